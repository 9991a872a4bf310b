"""Failure detection without a GPU fault.

The reference exits the process on any CUDA error (include/impl/util.hpp:18-26).
This engine returns a status instead, and these tests make the failures on
purpose in forms that leave the GPU healthy:

* a radix sort tile that never publishes its look-back status (a test hook
  armed through PPF_B200_TEST_SORT_STALL=1 when the context is created): the
  tiles that wait on it give up after a few thousand bounded spins, the
  kernel returns, and the call reports PPF_ERR_TIMEOUT;
* a device allocation that fails (PPF_B200_TEST_FAIL_ALLOC=<n>: the n-th
  allocation after the context is created), reported as
  PPF_ERR_OUT_OF_MEMORY.

In both cases the same context then builds the model and registers the scene
with the result a clean context gives.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def case(pkg, ctx):
    spec = pkg.synthetic.config_plain(seed=181, n_model=400, n_plane=800, n_box=300)
    m, s, d = spec.models[0], spec.scene, spec.d_dists[0]
    model = pkg.Model(m, d, 0.3, context=ctx)
    pose = model.ppf_lookup(pkg.Scene(s, d, 5, context=ctx)).copy()
    return spec, pose, model.get_votes()


def _register(pkg, spec, context):
    m, s, d = spec.models[0], spec.scene, spec.d_dists[0]
    model = pkg.Model(m, d, 0.3, context=context)
    pose = model.ppf_lookup(pkg.Scene(s, d, 5, context=context)).copy()
    return pose, model.get_votes()


def _status(pkg, err):
    return pkg._capi.STATUS_NAMES[err.value.status]


def test_sort_lookback_timeout_is_reported_and_the_context_recovers(pkg, case, monkeypatch):
    spec, pose_ref, votes_ref = case
    monkeypatch.setenv("PPF_B200_TEST_SORT_STALL", "1")
    c = pkg.Context(0)
    monkeypatch.delenv("PPF_B200_TEST_SORT_STALL")
    with pytest.raises(pkg.PPFError) as e:
        _register(pkg, spec, c)
    assert _status(pkg, e) == "PPF_ERR_TIMEOUT"
    assert "look-back timed out" in str(e.value)
    pose, votes = _register(pkg, spec, c)
    assert np.array_equal(pose, pose_ref)
    assert all(np.array_equal(a, b) for a, b in zip(votes, votes_ref))


@pytest.mark.parametrize("nth", [1, 4, 9, 15, 22])
def test_failed_allocation_is_reported_and_the_context_recovers(pkg, case, monkeypatch, nth):
    spec, pose_ref, votes_ref = case
    monkeypatch.setenv("PPF_B200_TEST_FAIL_ALLOC", str(nth))
    c = pkg.Context(0)
    monkeypatch.delenv("PPF_B200_TEST_FAIL_ALLOC")
    with pytest.raises(pkg.PPFError) as e:
        _register(pkg, spec, c)
    assert _status(pkg, e) == "PPF_ERR_OUT_OF_MEMORY"
    assert "(injected)" in str(e.value)
    pose, votes = _register(pkg, spec, c)
    assert np.array_equal(pose, pose_ref)
    assert all(np.array_equal(a, b) for a, b in zip(votes, votes_ref))
