"""The instance-sharded composite across ranks, on CPU: two gloo ranks each
hold and integrate half of the instances (mid_fusion_b200.shard.partition),
record their instances' raycasts (the oracle's restatement of
mf_raycast_records stands in for each rank's GPU), gather the records in
instance order (mid_fusion_b200.shard.gather_records, torch.distributed
all_gather), and fold them per pixel as mf_raycast_fold does.  Both ranks get
the single-process composite (raycastObjectList, rendering.cpp:9-181, as the
oracle restates it) bit for bit, over 3 frames of a 3-object scene and of the
12-object scene; the object poses tracked on their owning ranks are gathered
too."""
import ctypes as C
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as tmp

INVALID = np.float32(-2.0)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _records(orc, vol, T_w_o, label, T_w_c, k, W, H, eps_size):
    """One instance's records (the oracle's restatement of mf_raycast_records);
    the ray iterator's direction epsilon comes from the first octree's size."""
    eps = float(np.float32(2.0 ** -np.log2(eps_size)))
    lib = orc.lib
    f = lib.or_raycast_records
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_int, C.c_int,
                  C.c_float, C.c_float, C.c_float, C.c_float, C.c_void_p, C.c_void_p]
    rec = np.zeros((H, W, 12), np.float32)
    org = np.zeros(8, np.float32)
    Two = np.ascontiguousarray(T_w_o, np.float32).reshape(16)
    Twc = np.ascontiguousarray(T_w_c, np.float32).reshape(16)
    kk = np.ascontiguousarray(k, np.float32)
    f(vol.h, Two.ctypes.data, int(label), Twc.ctypes.data, kk.ctypes.data, W, H, 0.1, 4.0, 0.1,
      eps, rec.ctypes.data, org.ctypes.data)
    return rec, org


def fold(rec, org, poses, labels, vertex, normal, label_img, far=4.0):
    """mf_raycast_fold restated per pixel: the instances in order, each with
    its march's crossing if that lies before min(nearest, far), else its zero
    hit; the reference's nearest / foreground / tie tests; the winner's vertex
    and normal (a zero gradient writes only normal.x)."""
    H, W = label_img.shape
    n = len(labels)
    for y in range(H):
        for x in range(W):
            nearest = np.float32(1.0e3)
            high_fg = 0.0
            miss = 0
            win = None
            last_full = None
            for o in range(n):
                r = rec[o, y, x]
                nfar = min(nearest, np.float32(far))
                if r[4] < nfar:
                    hit, fg, nrm, zero = r[0:4], float(r[5]), r[6:9], r[9] != 0
                else:
                    hit = np.zeros(4, np.float32)
                    fg, nrm, zero = float(org[o, 0]), org[o, 1:4], org[o, 4] != 0
                hd = np.float32(hit[3] + np.float32(0.05)) if labels[o] == 0 else hit[3]
                if hd > nearest:
                    miss += 1
                    continue
                if fg <= 0.5:
                    miss += 1
                    continue
                if hd == nearest:
                    if not fg > high_fg:
                        miss += 1
                        continue
                elif hd < nearest:
                    nearest = hd
                high_fg = fg
                if win is not None and not win[3]:
                    last_full = win[2]
                win = (o, hit, nrm, zero)
            if win is None:
                if miss == n:
                    vertex[y, x] = 0
                    normal[y, x] = (INVALID, 0, 0)
                    label_img[y, x] = -2
                continue
            o, hit, nrm, zero = win
            label_img[y, x] = labels[o]
            vertex[y, x] = _xform(poses[o], hit[:3])
            if not zero:
                normal[y, x] = nrm
            else:
                normal[y, x, 0] = INVALID
                if last_full is not None:
                    normal[y, x, 1:] = last_full[1:]


def _xform(T, p):
    """Matrix4 * float3 in float32 with the reference's operation order
    (utils/math_utils.h:105-110: dot of the row's xyz, then + w)."""
    T = T.astype(np.float32)
    out = np.zeros(3, np.float32)
    for i in range(3):
        d = np.float32(T[i, 0] * p[0]) + np.float32(T[i, 1] * p[1])
        d = np.float32(d + np.float32(T[i, 2] * p[2]))
        out[i] = np.float32(d + T[i, 3])
    return out


def _rank(rank, world, port, preset, out):
    import datetime
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path[:0] = [root, os.path.join(root, "tests")]
    import torch
    import torch.distributed as dist
    import _oracle as O
    from mid_fusion_b200 import shard
    from mid_fusion_b200.scene import generalize_masks, make_scene
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world, timeout=datetime.timedelta(seconds=120))
    try:
        W, H = 48, 36
        if preset == "multi":
            s = make_scene("multi", W, H, n_frames=3, seed=5, bg_size=128, obj_size=64,
                           n_objects=3)
        else:
            s = make_scene("uneven", W, H, n_frames=3, seed=23, n_objects=12)
        labels = [i.label for i in s.instances]
        n = len(labels)
        parts = shard.partition([i.size for i in s.instances], world)
        mine = parts[rank]
        orc = O.oracle()
        eps = s.instances[0].size
        vols = {i: orc.volume(s.instances[i].size, s.instances[i].dim) for i in mine}
        ok = True
        for f in range(s.n_frames):
            d, rgb, lab = s.render(f)
            masks = generalize_masks(lab, labels)
            T = s.cam_poses[f].astype(np.float32)
            poses = [P.astype(np.float32) for P in s.volume_poses(f)]
            rgb3 = rgb.astype(np.float32) / np.float32(255)
            recs, orgs = [], []
            for i in mine:
                vols[i].integrate(d, rgb3, masks[i], T, poses[i], s.k, 0.1)
                r, o = _records(orc, vols[i], poses[i], labels[i], T, s.k, W, H, eps)
                recs.append(r.view(np.uint8).reshape(H, W, 48))
                orgs.append(o.view(np.uint8))
            grec, gorg = shard.gather_records(torch.from_numpy(np.stack(recs)),
                                              torch.from_numpy(np.stack(orgs)), parts, n)
            rec = grec.numpy().view(np.float32).reshape(n, H, W, 12)
            org = gorg.numpy().view(np.float32).reshape(n, 8)
            # each rank "tracked" its own objects: the gathered poses are everyone's
            mp = torch.from_numpy(np.stack([poses[i] for i in mine]))
            gp = shard.gather_poses(mp, parts, n).numpy()
            ok &= np.array_equal(gp, np.stack(poses))
            v, nr, lb = (np.zeros((H, W, 3), np.float32), np.zeros((H, W, 3), np.float32),
                         np.zeros((H, W), np.int32))
            if f > 0:
                v, nr, lb = prev
            fold(rec, org, gp, labels, v, nr, lb)
            prev = (v, nr, lb)
            # the single-process composite, every volume on one "GPU"
            allv = [orc.volume(i.size, i.dim) for i in s.instances]
            for ff in range(f + 1):
                dd, rr, ll = s.render(ff)
                mm = generalize_masks(ll, labels)
                for i, vv in enumerate(allv):
                    vv.integrate(dd, rr.astype(np.float32) / np.float32(255), mm[i],
                                 s.cam_poses[ff].astype(np.float32),
                                 s.volume_poses(ff)[i].astype(np.float32), s.k, 0.1)
            vo, no, lo = want_prev if f > 0 else (np.zeros((H, W, 3), np.float32),
                                                  np.zeros((H, W, 3), np.float32),
                                                  np.zeros((H, W), np.int32))
            vo, no, lo = vo.copy(), no.copy(), lo.copy()
            orc.raycast_objects(allv, poses, labels, T, s.k, W, H, eps_size=eps, vertex=vo,
                                normal=no, label_img=lo)
            want_prev = (vo, no, lo)
            same = (np.array_equal(v, vo) and np.array_equal(nr, no) and np.array_equal(lb, lo))
            ok &= bool(same)
            ok &= bool((lo >= 0).mean() > 0.3)
        out.put((rank, bool(ok), mine))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("preset", ["multi", "uneven"])
def test_sharded_composite_over_two_gloo_ranks(preset):
    world = 2
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, world, port, preset, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = dict((r, (ok, mine)) for r, ok, mine in (q.get(timeout=300) for _ in procs))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    owned = sorted(i for r in res for i in res[r][1])
    assert owned == list(range(len(owned))) and len(owned) >= 4
    assert all(len(res[r][1]) > 0 for r in res)
    for r in res:
        assert res[r][0], f"rank {r}: the folded maps differ from the composite"


def test_partition_balances_instances():
    from mid_fusion_b200 import shard
    sizes = [512, 256, 32, 64, 128, 256, 32, 64]
    p = shard.partition(sizes, 3)
    assert p[0][0] == 0 and sorted(i for r in p for i in r) == list(range(len(sizes)))
    load = [sum(sizes[i] ** 3 for i in r) for r in p]
    assert max(load[1:]) <= 2 * 256 ** 3
    assert shard.partition([256], 4) == [[0], [], [], []]
