"""GPU driver preprocessing against the oracle: cloud extent and voxel-grid
downsampling (points, normals, count) bit for bit, host and device inputs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("leaf", [0.004, 0.01, 0.03])
def test_voxel_downsample_equals_oracle(pkg, ctx, oracle, leaf):
    spec = pkg.synthetic.config_plain(seed=131)
    sc = spec.scene
    p, n = pkg.voxel_downsample(sc, leaf, context=ctx)
    op, on = oracle.voxel_downsample(sc.points, sc.normals, leaf)
    assert 0 < len(p) < len(sc)
    np.testing.assert_array_equal(p, op)
    np.testing.assert_array_equal(n, on)


def test_extent_and_d_dist_equal_oracle(pkg, ctx, oracle):
    spec = pkg.synthetic.config_multi_model(seed=1001)
    for m, t in zip(spec.models, (0.03, 0.035, 0.03, 0.05)):
        lo, hi = pkg.cloud_extent(m, context=ctx)
        olo, ohi = oracle.cloud_extent(m.points)
        np.testing.assert_array_equal(lo, olo)
        np.testing.assert_array_equal(hi, ohi)
        assert pkg.model_d_dist(m, t, context=ctx) == float(np.float32(t) * np.max(ohi - olo))


def test_device_inputs_and_overflow(pkg, ctx, oracle):
    import torch

    spec = pkg.synthetic.config_plain(seed=132, n_plane=3000, n_box=1000)
    sc = spec.scene
    dev = (torch.from_numpy(sc.points).cuda(), torch.from_numpy(sc.normals).cuda())
    torch.cuda.synchronize()
    p, n = pkg.voxel_downsample(dev, 0.01, context=ctx)
    op, on = oracle.voxel_downsample(sc.points, sc.normals, 0.01)
    np.testing.assert_array_equal(p, op)
    np.testing.assert_array_equal(n, on)
    # grid beyond 2^31 cells: the input comes back unchanged
    p, n = pkg.voxel_downsample(sc, 1e-5, context=ctx)
    np.testing.assert_array_equal(p, sc.points)
    np.testing.assert_array_equal(n, sc.normals)


def test_preprocessed_registration_finds_pose(pkg, ctx):
    spec = pkg.synthetic.config_plain(seed=133, n_model=3000, n_plane=9000, n_box=3000)
    scenes, models, d = pkg.preprocess([spec.scene], spec.models, [0.05], 0.004, context=ctx)
    pose = pkg.ppf_registration(scenes, models, d, 5, 0.3, context=ctx)[0][0]
    G = spec.instances[0].pose
    assert np.linalg.norm(pose[:3, 3] - G[:3, 3]) < 0.1 * spec.diameters[0]
