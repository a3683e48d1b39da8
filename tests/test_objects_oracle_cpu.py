"""Known-answer checks of the oracle's object spawning statistics
(Kfusion::spawnNewObjectKernel, kfusion.cpp:1080-1150) and semantic fusion
(Object::fuseSemanticLabel, object.cpp:223-252), worked out by hand."""
import numpy as np

import _oracle as O


def test_spawn_statistics_by_hand():
    W, H = 4, 2
    depth = np.ones((H, W), np.float32)
    mask = np.zeros((H, W), np.uint8)
    mask[0, 0] = mask[1, 3] = 1
    k = [1.0, 1.0, 0.0, 0.0]            # vertex = (x, y, 1)
    T, size, resol, n = O.spawn_object(depth, mask, k, np.eye(4))
    assert n == 2
    # extents (3, 1, 0 / 2) -> max 3 -> min(7.5, 5) = 5 -> 2048 voxels
    assert size == 5.0 and resol == 2048
    # mean (1.5, 0.5, 1) minus size / 2
    np.testing.assert_array_equal(T[:3, 3], np.float32([-1.0, -2.0, -1.5]))
    np.testing.assert_array_equal(T[:3, :3], np.eye(3, dtype=np.float32))
    # a masked pixel without depth contributes the camera centre
    depth[1, 3] = 0
    T2, size2, resol2, _ = O.spawn_object(depth, mask, k, np.eye(4))
    assert size2 == np.float32(2.5 * 0.5) and resol2 == 512   # extents (0, 0, 0.5)
    np.testing.assert_array_equal(T2[:3, 3], np.float32([0 - 0.625, 0 - 0.625, 0.5 - 0.625]))


def test_semantic_fusion_by_hand():
    f, ft, cid = O.fuse_semantics([0.5, 0.5, 0.0], 1, [0.0, 1.0, 0.0], recog_times=1)
    np.testing.assert_array_equal(f, np.float32([0.25, 0.75, 0.0]))
    assert ft == 2 and cid == 2
    f, ft, cid = O.fuse_semantics(f, ft, [1.0, 0.0, 0.0], recog_times=2)
    np.testing.assert_array_equal(f, np.float32([0.625, 0.375, 0.0]))   # (0.5 + 2) / 4
    assert ft == 4 and cid == 1
    # ties keep the first index
    _, _, cid = O.fuse_semantics([0.4, 0.4], 1, [0.4, 0.4])
    assert cid == 1
