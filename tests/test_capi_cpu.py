"""The C ABI library on a machine without a GPU: it loads, exports every entry
point include/midfusion_b200.h declares, and fails loudly (an error code, no
CPU fallback) when asked to create a context without a device."""
import ctypes as C
import os
import re

import pytest

from mid_fusion_b200 import build, capi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", f)).read()
            names |= set(re.findall(r"^\s*(?:int|const char\*)\s+(mf_\w+)\s*\(", txt, re.M))
    return names


@pytest.fixture(scope="module")
def lib():
    build.build()
    return capi.load()


def test_every_declared_symbol_is_exported(lib):
    names = declared()
    assert len(names) >= 30
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing
    assert set(capi.EXPORTS) == names


def test_config_defaults(lib):
    cfg = capi.MfConfig()
    assert lib.mf_config_default(C.byref(cfg), 640, 480) == 0
    assert (cfg.width, cfg.height) == (640, 480)
    assert list(cfg.gn_iterations)[:3] == [10, 5, 4]
    assert abs(cfg.mu - 0.1) < 1e-7 and cfg.max_weight == 100
    assert abs(cfg.k[0] - 525.0) < 1e-4 and abs(cfg.k[2] - 319.5) < 1e-4
    assert lib.mf_config_default(None, 640, 480) == -1


def test_create_without_device_fails_loudly(lib):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    cfg = capi.MfConfig()
    lib.mf_config_default(C.byref(cfg), 64, 48)
    h = C.c_void_p()
    rc = lib.mf_create(C.byref(cfg), C.byref(h))
    assert rc == -2 and not h.value  # MF_E_CUDA, no context, no fallback


def test_bad_arguments_are_rejected(lib):
    cfg = capi.MfConfig()
    lib.mf_config_default(C.byref(cfg), 64, 48)
    cfg.max_instances = 1000
    h = C.c_void_p()
    assert lib.mf_create(C.byref(cfg), C.byref(h)) == -1


def test_tune_candidate_tables(lib):
    """The autotuner's candidate tables answer without a device; unknown stages
    and variants are rejected."""
    n_ray = capi.tune_candidates(capi.TUNE_RAYCAST)
    n_int = capi.tune_candidates(capi.TUNE_INTEGRATE)
    assert 1 < n_ray <= capi.TUNE_MAX_VARIANTS and 1 < n_int <= capi.TUNE_MAX_VARIANTS
    shapes = [capi.tune_describe(capi.TUNE_RAYCAST, v) for v in range(n_ray)]
    assert len(set(shapes)) == n_ray and shapes[0].startswith("raycast tile 16x8")
    assert capi.tune_describe(capi.TUNE_INTEGRATE, 0).startswith("integrate 4 x")
    n = C.c_int()
    assert lib.mf_tune_candidates(2, C.byref(n)) == -1
    buf = C.create_string_buffer(64)
    assert lib.mf_tune_describe(capi.TUNE_RAYCAST, n_ray, buf, 64) == -1
    assert lib.mf_tune_describe(capi.TUNE_INTEGRATE, -1, buf, 64) == -1
    assert lib.mf_tune_get(None, 0, C.byref(n)) == -1
    assert lib.mf_tune_set(None, 0, 0) == -1
    assert lib.mf_autotune(None, 3, None, None) == -1


def test_config_struct_layout_matches_header(tmp_path):
    """The ctypes mf_config (capi.MfConfig) has the header's field offsets and
    size, as a C compiler lays the struct out."""
    import subprocess
    fields = [f[0] for f in capi.MfConfig._fields_]
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "midfusion_b200.h"\n'
                   "int main(void) {\n"
                   + "".join(f'  printf("%zu\\n", offsetof(mf_config, {f}));\n' for f in fields)
                   + '  printf("%zu\\n", sizeof(mf_config));\n  return 0;\n}\n')
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), "-o", str(exe),
                    str(src)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True,
                                          text=True).stdout.split()]
    want = [getattr(capi.MfConfig, f).offset for f in fields] + [C.sizeof(capi.MfConfig)]
    assert got == want


def test_ray_record_sizes_match_header(tmp_path):
    """The byte sizes the sharded exchange allocates per pixel and instance
    (mid_fusion_b200.shard) equal the header's mf_ray_record / mf_ray_origin."""
    import subprocess
    from mid_fusion_b200 import shard
    src = tmp_path / "sizes.c"
    src.write_text('#include <stdio.h>\n#include "midfusion_b200.h"\n'
                   'int main(void) { printf("%zu %zu\\n", sizeof(mf_ray_record), '
                   'sizeof(mf_ray_origin)); return 0; }\n')
    exe = tmp_path / "sizes"
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), "-o", str(exe),
                    str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    assert [int(x) for x in out] == [shard.RECORD_BYTES, shard.ORIGIN_BYTES]
