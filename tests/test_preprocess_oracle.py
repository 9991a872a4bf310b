"""Known answers for the oracle's restatement of the driver preprocessing
(pcl::getMinMax3D, pcl::VoxelGrid as src/alignment.cpp:79-87,246-253 use
them).  PCL itself is not installed, so these hand-computed cases pin the
restatement."""
import numpy as np


def test_voxel_grid_known_answer(oracle):
    # leaf 1.0: voxels (0,0,0) and (1,0,0); linear order x fastest
    xyz = np.array([[0.1, 0.2, 0.3], [1.5, 0.5, 0.5], [0.3, 0.4, 0.1], [1.7, 0.1, 0.9],
                    [np.nan, 0.0, 0.0]], np.float32)
    nrm = np.array([[0, 0, 1], [1, 0, 0], [0, 1, 0], [1, 0, 0], [0, 0, 1]], np.float32)
    p, n = oracle.voxel_downsample(xyz, nrm, 1.0)
    assert p.shape == (2, 3)
    np.testing.assert_array_equal(p[0], (xyz[0] + xyz[2]) / np.float32(2))
    np.testing.assert_array_equal(p[1], (xyz[1] + xyz[3]) / np.float32(2))
    np.testing.assert_array_equal(n[0], np.float32([0, 0.5, 0.5]))  # normals are not renormalised
    np.testing.assert_array_equal(n[1], np.float32([1, 0, 0]))
    lo, hi = oracle.cloud_extent(xyz)
    np.testing.assert_array_equal(lo, np.float32([0.1, 0.1, 0.1]))
    np.testing.assert_array_equal(hi, np.float32([1.7, 0.5, 0.9]))


def test_voxel_grid_linear_order_and_overflow(oracle):
    rng = np.random.default_rng(3)
    xyz = rng.uniform(-1, 1, (500, 3)).astype(np.float32)
    nrm = rng.normal(size=(500, 3)).astype(np.float32)
    p, _ = oracle.voxel_downsample(xyz, nrm, 0.25)
    # voxels come out in linear index order: z slowest, then y, then x
    ijk = np.floor(p / np.float32(0.25)).astype(np.int64)
    key = (ijk[:, 2] * 10000 + ijk[:, 1]) * 10000 + ijk[:, 0]
    assert np.all(np.diff(key) > 0)
    # a grid beyond 2^31 - 1 cells returns the cloud unchanged, as PCL 1.8 does
    p2, n2 = oracle.voxel_downsample(xyz, nrm, 1e-4)
    np.testing.assert_array_equal(p2, xyz)
    np.testing.assert_array_equal(n2, nrm)
