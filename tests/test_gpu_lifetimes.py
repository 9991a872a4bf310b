"""Handle lifetimes at the C boundary: contexts, models, scenes and servers
may be destroyed in any order (each model and scene holds a reference on its
context, a server on its library models).  Python's garbage collector
finalises objects of a reference cycle in no fixed order, so a model can be
finalised after its context; these calls make that order explicit."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _handles(pkg, spec, ctx_h):
    L = pkg.api._lib()
    m, s, d = spec.models[0], spec.scene, spec.d_dists[0]
    mp, mn = np.ascontiguousarray(m.points), np.ascontiguousarray(m.normals)
    sp, sn = np.ascontiguousarray(s.points), np.ascontiguousarray(s.normals)
    mh, sh = C.c_void_p(), C.c_void_p()
    assert L.ppf_model_create(ctx_h, C.c_void_p(mp.ctypes.data), C.c_void_p(mn.ctypes.data), len(mp), d, 0.3,
                              0, 0, 0, C.byref(mh)) == 0
    assert L.ppf_scene_create(ctx_h, C.c_void_p(sp.ctypes.data), C.c_void_p(sn.ctypes.data), len(sp), d, 5,
                              C.byref(sh)) == 0
    return mh, sh


def _lookup(pkg, mh, sh):
    pose = np.zeros(16, np.float32)
    assert pkg.api._lib().ppf_model_lookup(mh, sh, C.c_void_p(pose.ctypes.data), None) == 0
    return pose


def test_context_destroyed_before_its_model_and_scene(pkg):
    L = pkg.api._lib()
    spec = pkg.synthetic.config_plain(seed=201, n_model=300, n_plane=500, n_box=200)
    ch = C.c_void_p()
    assert L.ppf_context_create(0, C.byref(ch)) == 0
    mh, sh = _handles(pkg, spec, ch)
    before = _lookup(pkg, mh, sh)
    assert L.ppf_context_destroy(ch) == 0  # the model and scene keep it alive
    after = _lookup(pkg, mh, sh)
    assert np.array_equal(before, after)
    assert L.ppf_model_destroy(mh) == 0
    assert L.ppf_scene_destroy(sh) == 0  # the last reference: the context goes here


def test_server_keeps_its_library_models(pkg):
    L = pkg.api._lib()
    spec = pkg.synthetic.config_plain(seed=202, n_model=300, n_plane=500, n_box=200)
    ch = C.c_void_p()
    assert L.ppf_context_create(0, C.byref(ch)) == 0
    mh, sh = _handles(pkg, spec, ch)
    want = _lookup(pkg, mh, sh)
    lib = (C.c_void_p * 1)(mh.value)
    srv = C.c_void_p()
    assert L.ppf_server_create(0, 1, lib, 8 << 30, 1, 4, C.byref(srv)) == 0
    assert L.ppf_scene_destroy(sh) == 0
    assert L.ppf_model_destroy(mh) == 0
    assert L.ppf_context_destroy(ch) == 0  # all held by the server's reference on the model
    s = spec.scene
    sp, sn = np.ascontiguousarray(s.points), np.ascontiguousarray(s.normals)
    ids = np.zeros(1, np.uint32)
    t = C.c_uint64()
    assert L.ppf_server_submit(srv, C.c_void_p(sp.ctypes.data), C.c_void_p(sn.ctypes.data), len(sp), 5, 1,
                               C.c_void_p(ids.ctypes.data), C.byref(t)) == 0
    pose = np.zeros(16, np.float32)
    assert L.ppf_server_wait(srv, t.value, C.c_void_p(pose.ctypes.data), None, None) == 0
    assert np.array_equal(pose, want)
    assert L.ppf_server_destroy(srv) == 0
