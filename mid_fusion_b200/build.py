"""Build the MID-Fusion B200 CUDA library in-tree (sm_100a).

``python -m mid_fusion_b200.build`` compiles every ``csrc/*.cu`` file with nvcc
into ``mid_fusion_b200/_lib/libmidfusion_b200.so``.  -fmad=false keeps the
reference's IEEE single-precision evaluation order (no fused multiply-add), on
which the bit-exact allocation parity rests.
"""
from __future__ import annotations

import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB_DIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIB_DIR, "libmidfusion_b200.so")

NVCC_FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-lineinfo", "-O3", "-std=c++17", "-fmad=false",
    "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
    "-Xptxas", "-O3",
    "--shared",
]


def sources():
    return sorted(glob.glob(os.path.join(HERE, "csrc", "*.cu")))


def headers():
    return (glob.glob(os.path.join(HERE, "csrc", "*.cuh")) +
            glob.glob(os.path.join(HERE, "csrc", "*.h")) +
            glob.glob(os.path.join(ROOT, "include", "*.h")))


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in sources() + headers() + [__file__])


def build(force=False, verbose=False, extra=()):
    if not force and up_to_date():
        return LIB
    os.makedirs(LIB_DIR, exist_ok=True)
    nvcc = os.environ.get("NVCC", "nvcc")
    objs = []
    for src in sources():
        obj = os.path.join(LIB_DIR, os.path.basename(src)[:-3] + ".o")
        cmd = [nvcc, *NVCC_FLAGS[:-1], "-c", "-I", os.path.join(ROOT, "include"), *extra,
               src, "-o", obj]
        if verbose:
            print(" ".join(cmd), file=sys.stderr)
        subprocess.run(cmd, check=True)
        objs.append(obj)
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "--shared", *objs, "-o", LIB,
           "-lcudart"]
    subprocess.run(cmd, check=True)
    return LIB


TORCH_EXT_NAME = "mf_autograd_ext"
TORCH_EXT_DIR = os.path.join(LIB_DIR, "torch_ext")
TORCH_EXT_SRC = os.path.join(HERE, "csrc_torch", "mf_autograd.cpp")


def torch_ext_path():
    return os.path.join(TORCH_EXT_DIR, TORCH_EXT_NAME + ".so")


def build_torch_ext(verbose=False):
    """The libtorch autograd Function over mf_camera_cost
    (csrc_torch/mf_autograd.cpp), built in-tree against the CUDA library."""
    out = torch_ext_path()
    if (os.path.exists(out) and os.path.getmtime(out) >= os.path.getmtime(TORCH_EXT_SRC) and
            os.path.getmtime(out) >= os.path.getmtime(LIB)):
        return out
    from torch.utils import cpp_extension
    os.makedirs(TORCH_EXT_DIR, exist_ok=True)
    cpp_extension.load(
        name=TORCH_EXT_NAME, sources=[TORCH_EXT_SRC], build_directory=TORCH_EXT_DIR,
        extra_cflags=["-O2", "-std=c++17"],
        extra_ldflags=[f"-L{LIB_DIR}", "-lmidfusion_b200", f"-Wl,-rpath,{LIB_DIR}",
                       "-Wl,-rpath,$ORIGIN/.."],
        verbose=verbose, is_python_module=True)
    return out


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose=True,
          extra=["-Xptxas", "-v"] if "--ptxas-v" in sys.argv else [])
    print(LIB)
    print(build_torch_ext(verbose=True))
