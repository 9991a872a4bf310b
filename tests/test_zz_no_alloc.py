"""The allocation-free vote pass (ppf_model_vote_cells_noalloc) against the
allocating entry points on the same model and scene.

The file name sorts last, so in a full run it goes after every other GPU
test; `pytest tests/test_zz_no_alloc.py -m gpu` runs it alone in a fresh
process.  Each comparison is made on two calls in a row, since the second
call reuses the static scratch the first one left behind.  Vote cells are
integers, so the comparison is exact.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(a, dtype):
    import torch

    return torch.as_tensor(np.ascontiguousarray(a), dtype=dtype, device="cuda")


def _scene_dev(cloud):
    import torch

    return _dev(cloud.points, torch.float32), _dev(cloud.normals, torch.float32)


def _outputs(n):
    import torch

    return (torch.zeros(n, dtype=torch.int64, device="cuda"),
            torch.zeros(n, dtype=torch.int32, device="cuda"))


def _cells(codes, counts, n):
    c = codes[:n].cpu().numpy().view(np.uint64)
    k = counts[:n].cpu().numpy().view(np.uint32)
    return c, k


@pytest.fixture(scope="module")
def small(pkg, ctx):
    # one m_r chunk; every nonzero cell fits a modest output
    spec = pkg.synthetic.config_plain(seed=71, n_model=500, n_plane=1200, n_box=400)
    d = spec.d_dists[0]
    model = pkg.Model(spec.models[0], d, spec.vote_count_threshold, context=ctx)
    scene = pkg.Scene(spec.scene, d, spec.ref_point_df, context=ctx)
    return spec, model, scene


@pytest.fixture(scope="module")
def chunked(pkg, ctx):
    # 3500 model points: three m_r chunks of the vote accumulator
    spec = pkg.synthetic.config_plain(seed=72, n_model=3500, n_plane=3000, n_box=1000)
    d = spec.d_dists[0]
    model = pkg.Model(spec.models[0], d, spec.vote_count_threshold, context=ctx)
    scene = pkg.Scene(spec.scene, d, spec.ref_point_df, context=ctx)
    return spec, model, scene


def test_every_nonzero_cell_matches_all_votes(small):
    spec, model, scene = small
    ref_codes, ref_counts = model.all_votes(scene)
    assert len(ref_codes) > 0
    xyz, nxyz = _scene_dev(spec.scene)
    codes, counts = _outputs(len(ref_codes) + 1000)
    for _ in range(2):
        codes.zero_()
        counts.zero_()
        n, mx = model.vote_cells_noalloc(xyz, nxyz, spec.ref_point_df, 0.0, codes, counts)
        c, k = _cells(codes, counts, n)
        order = np.argsort(c, kind="stable")
        assert n == len(ref_codes)
        assert np.array_equal(c[order], ref_codes) and np.array_equal(k[order], ref_counts)
        assert mx == int(ref_counts.max())


@pytest.mark.parametrize("which", ["small", "chunked"])
def test_threshold_cells_match_lookup(which, request):
    spec, model, scene = request.getfixturevalue(which)
    model.ppf_lookup(scene)
    ref_codes, ref_counts = model.get_votes()
    xyz, nxyz = _scene_dev(spec.scene)
    codes, counts = _outputs(16_000_000)
    for _ in range(2):
        n, mx = model.vote_cells_noalloc(xyz, nxyz, spec.ref_point_df, -1.0, codes, counts)
        assert mx == int(ref_counts.max())
        c, k = _cells(codes, counts, n)
        floor = np.float32(model.vote_count_threshold) * np.float32(mx)
        keep = k.astype(np.float32) > floor
        c, k = c[keep], k[keep]
        order = np.lexsort((c, -k.astype(np.int64)))  # count descending, then code ascending
        assert np.array_equal(c[order], ref_codes) and np.array_equal(k[order], ref_counts)


def test_small_output_reports_needed_cells(pkg, small):
    spec, model, scene = small
    xyz, nxyz = _scene_dev(spec.scene)
    codes, counts = _outputs(16)
    with pytest.raises(pkg.PPFError) as e:
        model.vote_cells_noalloc(xyz, nxyz, spec.ref_point_df, 0.0, codes, counts)
    assert pkg._capi.STATUS_NAMES[e.value.status] == "PPF_ERR_OUT_OF_MEMORY"
    assert "too small" in str(e.value)
    needed = e.value.needed
    codes, counts = _outputs(needed)
    n, _ = model.vote_cells_noalloc(xyz, nxyz, spec.ref_point_df, 0.0, codes, counts)
    assert n == needed == len(model.all_votes(scene)[0])


def test_sizes_beyond_the_limit_are_rejected(pkg, small):
    import torch

    spec, model, _ = small
    big = torch.zeros((65537, 3), dtype=torch.float32, device="cuda")
    codes, counts = _outputs(16)
    with pytest.raises(pkg.PPFError) as e:
        model.vote_cells_noalloc(big, big, 1, 0.0, codes, counts)
    assert pkg._capi.STATUS_NAMES[e.value.status] == "PPF_ERR_INVALID_ARGUMENT"
    assert "exceeds the allocation-free limit of 65536" in str(e.value)
    # host memory is refused at the C boundary too
    import ctypes as C

    host = np.zeros((100, 3), np.float32)
    n = C.c_uint64()
    st = pkg.api._lib().ppf_model_vote_cells_noalloc(
        model.handle, C.c_void_p(host.ctypes.data), C.c_void_p(host.ctypes.data), 100, 1, 0.0,
        C.c_void_p(codes.data_ptr()), C.c_void_p(counts.data_ptr()), 16, C.byref(n), None)
    assert pkg._capi.STATUS_NAMES[st] == "PPF_ERR_INVALID_ARGUMENT"


def test_work_items_beyond_the_limit_are_rejected(pkg, ctx):
    """A scene within the point limit whose reference points times the model's
    chunks exceed the 262144 work items the static scratch holds is refused
    before any GPU work."""
    import torch

    spec = pkg.synthetic.config_plain(seed=73, n_model=9000, n_plane=10, n_box=10)
    model = pkg.Model(spec.models[0], spec.d_dists[0], 0.3, context=ctx)
    chunks = model.num_chunks
    n_scene = 60000
    assert n_scene <= 65536 and n_scene * chunks > 262144, chunks
    xyz = torch.zeros((n_scene, 3), dtype=torch.float32, device="cuda")
    codes, counts = _outputs(16)
    launches = ctx.kernel_launches
    with pytest.raises(pkg.PPFError) as e:
        model.vote_cells_noalloc(xyz, xyz, 1, 0.0, codes, counts)
    assert pkg._capi.STATUS_NAMES[e.value.status] == "PPF_ERR_INVALID_ARGUMENT"
    assert "work items" in str(e.value)
    assert ctx.kernel_launches == launches


def test_tensors_on_another_device_are_refused(small):
    """The Python wrapper compares each tensor's device with the model's
    context before the call (a stand-in context on another device index
    makes the mismatch with one GPU)."""
    spec, model, _ = small
    xyz, nxyz = _scene_dev(spec.scene)
    codes, counts = _outputs(16)

    class OtherDevice:
        device = xyz.device.index + 1

    real = model.ctx
    model.ctx = OtherDevice()
    try:
        with pytest.raises(ValueError, match="context on cuda:"):
            model.vote_cells_noalloc(xyz, nxyz, spec.ref_point_df, 0.0, codes, counts)
    finally:
        model.ctx = real
