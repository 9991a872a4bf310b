"""ctypes access to the oracle builds -- TEST INFRASTRUCTURE ONLY.

Imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg,
only as the checker / the timed CPU baseline; the product never calls it.

* ``Oracle``    -> oracle/libppf_oracle.so, the CPU restatement (ppf_oracle.cpp)
* ``RefHost``   -> oracle/_ref/libppfref_host.so, the reference's own helpers
                   built for the host (pins the restatement)
* ``RefGPU``    -> oracle/_ref/libppfref_gpu.so, the reference's own kernels on
                   the GPU, driven in model.cu order (the bit-exact oracle)
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_fp = C.POINTER(C.c_float)
_dp = C.POINTER(C.c_double)
_u32p = C.POINTER(C.c_uint32)
_u64p = C.POINTER(C.c_uint64)


def _f32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.float32))


def _p(a, t=_fp):
    return a.ctypes.data_as(t)


class orc_result(C.Structure):
    _fields_ = [
        ("n_votes", C.c_uint64),
        ("n_unique", C.c_uint64),
        ("max_count", C.c_uint32),
        ("min_votecount", C.c_float),
        ("n_kept", C.c_uint64),
        ("codes", _u64p),
        ("counts", _u32p),
        ("weighted", _fp),
        ("transforms", _fp),
        ("trans", _fp),
        ("quats", _fp),
        ("cell_keys", _u32p),
        ("scores", _fp),
        ("max_idx", C.c_uint64),
        ("pose", C.c_float * 16),
        ("status", C.c_int),
        ("n_clusters", C.c_int),
        ("cpu_poses", C.c_float * 48),
        ("cpu_votes", C.c_uint32 * 3),
        ("t_build", C.c_double),
        ("t_vote", C.c_double),
        ("n_refs", C.c_uint64),
    ]


class orc_params(C.Structure):
    _fields_ = [
        ("d_dist", C.c_float),
        ("ref_point_df", C.c_uint32),
        ("vote_count_threshold", C.c_float),
        ("cpu_clustering", C.c_int),
        ("use_l1_norm", C.c_int),
        ("use_averaged_clusters", C.c_int),
        ("n_threads", C.c_int),
        ("sr_begin", C.c_int64),
        ("sr_end", C.c_int64),
        ("sr_step", C.c_int64),
        ("votes_only", C.c_int),
    ]


def _arr(ptr, n, dtype, shape=None):
    if n == 0 or not ptr:
        return np.zeros((0,) if shape is None else (0,) + shape[1:], dtype)
    a = np.ctypeslib.as_array(ptr, shape=(int(n),) if shape is None else shape).copy()
    return a.astype(dtype, copy=False)


class Oracle:
    def __init__(self, path=None):
        p = Path(path or HERE / "libppf_oracle.so")
        if not p.exists():
            raise RuntimeError(f"{p} missing: run `make -C oracle`")
        L = C.CDLL(str(p))
        L.orc_fnv1a.restype = C.c_uint32
        L.orc_fnv1a.argtypes = [C.c_void_p, C.c_int, C.c_uint32]
        L.orc_pair_feature.argtypes = [_fp, _fp, _fp, _fp, C.c_float, _fp]
        L.orc_feature_key.restype = C.c_uint32
        L.orc_feature_key.argtypes = [_fp]
        L.orc_trans_model_scene.restype = C.c_uint32
        L.orc_trans_model_scene.argtypes = [_fp] * 6
        L.orc_vote_pose.argtypes = [C.c_uint32, _fp, _fp, _fp, _fp, _fp]
        L.orc_vote_pose_f64.argtypes = [C.c_uint32, _fp, _fp, _fp, _fp, _dp]
        L.orc_hrotmat2quat.argtypes = [_fp, _fp]
        L.orc_trans_cell_keys.restype = C.c_uint32
        L.orc_trans_cell_keys.argtypes = [_fp, C.c_float, _u32p]
        L.orc_pair_keys.argtypes = [_fp, _fp, C.c_int64, C.c_uint32, C.c_float, _u32p, C.c_int]
        L.orc_hash_array.restype = C.c_int64
        L.orc_hash_array.argtypes = [_u32p, C.c_int64, _u32p, _u32p, _u32p, _u32p, _u32p]
        L.orc_register.restype = C.POINTER(orc_result)
        L.orc_register.argtypes = [_fp, _fp, C.c_int64, _fp, _fp, C.c_int64, _fp, C.POINTER(orc_params)]
        L.orc_result_free.argtypes = [C.POINTER(orc_result)]
        L.orc_vote_counts.argtypes = [_u32p, C.c_int64, _u32p, _u32p, C.c_int64, _u64p]
        L.orc_cluster_poses.restype = C.c_int
        L.orc_cluster_poses.argtypes = [_fp, _u32p, C.c_int64, C.c_float, C.c_float, _fp, _u32p]
        L.orc_cloud_extent.argtypes = [_fp, C.c_int64, _fp, _fp]
        L.orc_voxel_downsample.argtypes = [_fp, _fp, C.c_int64, C.c_float, _fp, _fp]
        L.orc_voxel_downsample.restype = C.c_int64
        self.L = L

    # -- single items
    def pair_feature(self, p1, n1, p2, n2, d_dist):
        out = np.zeros(4, np.float32)
        a = [_f32(x) for x in (p1, n1, p2, n2)]
        self.L.orc_pair_feature(*[_p(x) for x in a], float(d_dist), _p(out))
        return out

    def feature_key(self, f):
        return int(self.L.orc_feature_key(_p(_f32(f))))

    def alpha_bin(self, m_r, n_m, m_i, s_r, n_s, s_i):
        a = [_f32(x) for x in (m_r, n_m, m_i, s_r, n_s, s_i)]
        return int(self.L.orc_trans_model_scene(*[_p(x) for x in a]))

    def vote_pose(self, b, m_r, n_m, s_r, n_s, f64=False):
        a = [_f32(x) for x in (m_r, n_m, s_r, n_s)]
        if f64:
            out = np.zeros(16, np.float64)
            self.L.orc_vote_pose_f64(int(b), *[_p(x) for x in a], out.ctypes.data_as(_dp))
        else:
            out = np.zeros(16, np.float32)
            self.L.orc_vote_pose(int(b), *[_p(x) for x in a], _p(out))
        return out.reshape(4, 4)

    def quat(self, T):
        q = np.zeros(4, np.float32)
        self.L.orc_hrotmat2quat(_p(_f32(T).ravel()), _p(q))
        return q

    def cell_keys(self, t, d_dist):
        adj = np.zeros(27, np.uint32)
        k = self.L.orc_trans_cell_keys(_p(_f32(t)), float(d_dist), _p(adj, _u32p))
        return int(k), adj

    # -- stages
    def pair_keys(self, points, normals, d_dist, ref_df=1, n_threads=0):
        p, q = _f32(points), _f32(normals)
        n = p.shape[0]
        out = np.zeros(n * n, np.uint32)
        self.L.orc_pair_keys(_p(p), _p(q), n, int(ref_df), float(d_dist), _p(out, _u32p), int(n_threads))
        return out.reshape(n, n)

    def hash_array(self, keys):
        k = np.ascontiguousarray(np.asarray(keys, np.uint32).ravel())
        n = k.size
        sk = np.zeros(n, np.uint32)
        mp = np.zeros(n, np.uint32)
        uq = np.zeros(n, np.uint32)
        ct = np.zeros(n, np.uint32)
        fi = np.zeros(n, np.uint32)
        K = self.L.orc_hash_array(_p(k, _u32p), n, _p(sk, _u32p), _p(mp, _u32p), _p(uq, _u32p),
                                  _p(ct, _u32p), _p(fi, _u32p))
        return {"sorted_keys": sk, "map": mp, "keys": uq[:K].copy(), "counts": ct[:K].copy(), "first": fi[:K].copy()}

    def vote_counts(self, scene_keys, uniq, counts):
        sk = np.ascontiguousarray(np.asarray(scene_keys, np.uint32).ravel())
        u = np.ascontiguousarray(np.asarray(uniq, np.uint32))
        c = np.ascontiguousarray(np.asarray(counts, np.uint32))
        out = np.zeros(sk.size, np.uint64)
        self.L.orc_vote_counts(_p(sk, _u32p), sk.size, _p(u, _u32p), _p(c, _u32p), u.size, _p(out, _u64p))
        return out

    def register(self, model, scene, d_dist, ref_df=1, thr=0.4, cpu_clustering=False, use_l1_norm=False,
                 use_averaged_clusters=False, weights=None, n_threads=0, sr_range=None, sr_step=0,
                 votes_only=False):
        mp, mn = _f32(model[0]), _f32(model[1])
        sp, sn = _f32(scene[0]), _f32(scene[1])
        prm = orc_params(float(d_dist), int(ref_df), float(thr), int(cpu_clustering), int(use_l1_norm),
                         int(use_averaged_clusters), int(n_threads),
                         sr_range[0] if sr_range else 0, sr_range[1] if sr_range else -1, int(sr_step),
                         int(bool(votes_only)))
        w = _f32(weights) if weights is not None else None
        r = self.L.orc_register(_p(mp), _p(mn), mp.shape[0], _p(sp), _p(sn), sp.shape[0],
                                _p(w) if w is not None else None, C.byref(prm))
        R = r.contents
        U = int(R.n_kept)
        out = {
            "n_votes": int(R.n_votes),
            "n_unique": int(R.n_unique),
            "max_count": int(R.max_count),
            "min_votecount": float(R.min_votecount),
            "n_kept": U,
            "status": int(R.status),
            "codes": _arr(R.codes, U, np.uint64),
            "counts": _arr(R.counts, U, np.uint32),
            "weighted": _arr(R.weighted, U, np.float32),
            "transforms": _arr(R.transforms, U * 16, np.float32).reshape(-1, 16),
            "trans": _arr(R.trans, U * 3, np.float32).reshape(-1, 3),
            "quats": _arr(R.quats, U * 4, np.float32).reshape(-1, 4),
            "cell_keys": _arr(R.cell_keys, U, np.uint32),
            "scores": _arr(R.scores, U, np.float32),
            "max_idx": int(R.max_idx),
            "pose": np.array(R.pose[:], np.float32).reshape(4, 4),
            "n_clusters": int(R.n_clusters),
            "cpu_poses": np.array(R.cpu_poses[:], np.float32).reshape(3, 4, 4)[: int(R.n_clusters)],
            "cpu_votes": np.array(R.cpu_votes[:], np.uint32)[: int(R.n_clusters)],
            "t_build": float(R.t_build),
            "t_vote": float(R.t_vote),
            "n_refs": int(R.n_refs),
        }
        self.L.orc_result_free(r)
        return out

    def cluster_poses(self, poses, votes, trans_thresh, rot_thresh):
        P = _f32(poses).reshape(-1)
        v = np.ascontiguousarray(np.asarray(votes, np.uint32))
        out = np.zeros(48, np.float32)
        ov = np.zeros(3, np.uint32)
        nc = self.L.orc_cluster_poses(_p(P), _p(v, _u32p), v.size, float(trans_thresh), float(rot_thresh),
                                      _p(out), _p(ov, _u32p))
        return out.reshape(3, 4, 4)[:nc], ov[:nc]


    def cloud_extent(self, xyz):
        p = _f32(xyz)
        lo, hi = np.zeros(3, np.float32), np.zeros(3, np.float32)
        ok = self.L.orc_cloud_extent(_p(p), p.shape[0], _p(lo), _p(hi))
        return (lo, hi) if ok else None

    def voxel_downsample(self, xyz, nxyz, leaf):
        p, q = _f32(xyz), _f32(nxyz)
        ox, on = np.zeros_like(p), np.zeros_like(q)
        k = self.L.orc_voxel_downsample(_p(p), _p(q), p.shape[0], float(leaf), _p(ox), _p(on))
        return ox[:k], on[:k]


class RefHost:
    """The reference's own helpers, host build (oracle/_ref/libppfref_host.so)."""

    def __init__(self, path=None):
        p = Path(path or HERE / "_ref" / "libppfref_host.so")
        if not p.exists():
            raise RuntimeError(f"{p} missing: run `make -C oracle ref` where the reference sources exist")
        L = C.CDLL(str(p))
        L.ref_hash.restype = C.c_uint32
        L.ref_hash.argtypes = [C.c_void_p, C.c_int]
        L.ref_pair_feature.argtypes = [_fp, _fp, _fp, _fp, C.c_float, _fp]
        L.ref_feature_key.restype = C.c_uint32
        L.ref_feature_key.argtypes = [_fp]
        L.ref_trans_model_scene.restype = C.c_uint32
        L.ref_trans_model_scene.argtypes = [_fp] * 6
        L.ref_vote_pose.argtypes = [C.c_uint32, _fp, _fp, _fp, _fp, _fp]
        L.ref_hrotmat2quat.argtypes = [_fp, _fp]
        L.ref_trans_cell_keys.restype = C.c_uint32
        L.ref_trans_cell_keys.argtypes = [_fp, C.c_float, _u32p]
        self.L = L

    def pair_feature(self, p1, n1, p2, n2, d_dist):
        out = np.zeros(4, np.float32)
        a = [_f32(x) for x in (p1, n1, p2, n2)]
        self.L.ref_pair_feature(*[_p(x) for x in a], float(d_dist), _p(out))
        return out

    def feature_key(self, f):
        return int(self.L.ref_feature_key(_p(_f32(f))))

    def alpha_bin(self, m_r, n_m, m_i, s_r, n_s, s_i):
        a = [_f32(x) for x in (m_r, n_m, m_i, s_r, n_s, s_i)]
        return int(self.L.ref_trans_model_scene(*[_p(x) for x in a]))

    def vote_pose(self, b, m_r, n_m, s_r, n_s):
        a = [_f32(x) for x in (m_r, n_m, s_r, n_s)]
        out = np.zeros(16, np.float32)
        self.L.ref_vote_pose(int(b), *[_p(x) for x in a], _p(out))
        return out.reshape(4, 4)

    def quat(self, T):
        q = np.zeros(4, np.float32)
        self.L.ref_hrotmat2quat(_p(_f32(T).ravel()), _p(q))
        return q

    def cell_keys(self, t, d_dist):
        adj = np.zeros(27, np.uint32)
        k = self.L.ref_trans_cell_keys(_p(_f32(t)), float(d_dist), _p(adj, _u32p))
        return int(k), adj


class rh_result(C.Structure):
    _fields_ = [
        ("n_votes", C.c_ulonglong),
        ("n_unique", C.c_ulonglong),
        ("max_count", C.c_uint),
        ("min_votecount", C.c_float),
        ("n_kept", C.c_ulonglong),
        ("max_idx", C.c_ulonglong),
        ("pose", C.c_float * 16),
        ("elapsed_ms", C.c_float),
    ]


class RefGPU:
    """The reference's own kernels on the GPU (oracle/_ref/libppfref_gpu.so)."""

    def __init__(self, path=None):
        p = Path(path or HERE / "_ref" / "libppfref_gpu.so")
        if not p.exists():
            raise RuntimeError(f"{p} missing: run `make -C oracle ref` where the reference sources exist")
        L = C.CDLL(str(p))
        L.rh_last_error.restype = C.c_char_p
        L.rh_pair_keys.restype = C.c_int
        L.rh_pair_keys.argtypes = [_fp, _fp, C.c_int, C.c_float, C.c_uint, _u32p]
        L.rh_model_tables.restype = C.c_longlong
        L.rh_model_tables.argtypes = [_fp, _fp, C.c_int, C.c_float, _u32p, _u32p, _u32p, _u32p, C.c_longlong]
        L.rh_lookup.restype = C.c_int
        L.rh_lookup.argtypes = [
            _fp, _fp, C.c_int, _fp, _fp, C.c_int, C.c_float, C.c_uint, C.c_float, C.c_int, C.c_int, _fp,
            C.POINTER(rh_result), _u64p, _u32p, C.c_longlong, _u64p, _u32p, _fp, _fp, _fp, _fp,
            C.c_longlong, _u64p,
        ]
        L.rh_unique_votes.restype = C.c_int
        L.rh_unique_votes.argtypes = [_fp, _fp, C.c_int, _fp, _fp, C.c_int, C.c_float, C.c_uint,
                                      C.POINTER(rh_result), _u64p, _u32p, C.c_longlong]
        L.rh_post.restype = C.c_int
        L.rh_post.argtypes = [_fp, _fp, C.c_int, _fp, _fp, C.c_int, C.c_float, C.c_int, C.c_int, _fp, _u64p,
                              _u32p, C.c_longlong, C.POINTER(rh_result), _fp, _fp, _fp, _fp]
        self.L = L

    def _err(self, rc, what):
        if rc < 0:
            raise RuntimeError(f"{what} failed ({rc}): {self.L.rh_last_error().decode()}")

    def pair_keys(self, points, normals, d_dist, ref_df=1):
        p, q = _f32(points), _f32(normals)
        n = p.shape[0]
        out = np.zeros(n * n, np.uint32)
        self._err(self.L.rh_pair_keys(_p(p), _p(q), n, float(d_dist), int(ref_df), _p(out, _u32p)), "rh_pair_keys")
        return out.reshape(n, n)

    def model_tables(self, points, normals, d_dist):
        p, q = _f32(points), _f32(normals)
        n = p.shape[0]
        mp = np.zeros(n * n, np.uint32)
        cap = n * n
        u = np.zeros(cap, np.uint32)
        c = np.zeros(cap, np.uint32)
        f = np.zeros(cap, np.uint32)
        K = self.L.rh_model_tables(_p(p), _p(q), n, float(d_dist), _p(mp, _u32p), _p(u, _u32p), _p(c, _u32p),
                                   _p(f, _u32p), cap)
        self._err(K, "rh_model_tables")
        return {"keys": u[:K].copy(), "counts": c[:K].copy(), "first": f[:K].copy(), "map": mp}

    def lookup(self, model, scene, d_dist, ref_df=1, thr=0.4, use_l1_norm=False, use_averaged_clusters=False,
               weights=None, all_votes=False, pair_counts=False, cap=1 << 22):
        mp, mn = _f32(model[0]), _f32(model[1])
        sp, sn = _f32(scene[0]), _f32(scene[1])
        res = rh_result()
        acap = cap if all_votes else 0
        all_codes = np.zeros(acap, np.uint64)
        all_counts = np.zeros(acap, np.uint32)
        codes = np.zeros(cap, np.uint64)
        counts = np.zeros(cap, np.uint32)
        T = np.zeros(cap * 16, np.float32)
        t = np.zeros(cap * 3, np.float32)
        q = np.zeros(cap * 4, np.float32)
        s = np.zeros(cap, np.float32)
        ns = sp.shape[0]
        pc = np.zeros(ns * ns, np.uint64) if pair_counts else None
        w = _f32(weights) if weights is not None else None
        rc = self.L.rh_lookup(
            _p(mp), _p(mn), mp.shape[0], _p(sp), _p(sn), ns, float(d_dist), int(ref_df), float(thr),
            int(use_l1_norm), int(use_averaged_clusters), _p(w) if w is not None else None, C.byref(res),
            _p(all_codes, _u64p) if all_votes else None, _p(all_counts, _u32p) if all_votes else None, acap,
            _p(codes, _u64p), _p(counts, _u32p), _p(T), _p(t), _p(q), _p(s), cap,
            _p(pc, _u64p) if pc is not None else None,
        )
        self._err(rc, "rh_lookup")
        U = int(res.n_kept)
        nu = int(res.n_unique)
        if all_votes and nu > acap:
            # more unique vote cells than the buffer holds: run again with room for all
            return self.lookup(model, scene, d_dist, ref_df, thr, use_l1_norm, use_averaged_clusters, weights,
                               all_votes, pair_counts, cap=max(cap, nu))
        out = {
            "status": rc,
            "n_votes": int(res.n_votes),
            "n_unique": nu,
            "max_count": int(res.max_count),
            "min_votecount": float(res.min_votecount),
            "n_kept": U,
            "max_idx": int(res.max_idx),
            "pose": np.array(res.pose[:], np.float32).reshape(4, 4),
            "elapsed_ms": float(res.elapsed_ms),
        }
        if U <= cap:
            out.update(codes=codes[:U], counts=counts[:U], transforms=T[: U * 16].reshape(-1, 16),
                       trans=t[: U * 3].reshape(-1, 3), quats=q[: U * 4].reshape(-1, 4), scores=s[:U])
        if all_votes and nu <= acap:
            out.update(all_codes=all_codes[:nu], all_counts=all_counts[:nu])
        if pc is not None:
            out["pair_counts"] = pc.reshape(ns, ns)
        return out

    def unique_votes(self, model, scene, d_dist, ref_df=1, cap=1 << 24):
        """Every nonzero (s_r, m_r, alpha) vote cell in code order with its
        count (the reference's unique votes before the threshold)."""
        mp, mn = _f32(model[0]), _f32(model[1])
        sp, sn = _f32(scene[0]), _f32(scene[1])
        res = rh_result()
        codes = np.zeros(cap, np.uint64)
        counts = np.zeros(cap, np.uint32)
        rc = self.L.rh_unique_votes(_p(mp), _p(mn), mp.shape[0], _p(sp), _p(sn), sp.shape[0], float(d_dist),
                                    int(ref_df), C.byref(res), _p(codes, _u64p), _p(counts, _u32p), cap)
        self._err(rc, "rh_unique_votes")
        nu = int(res.n_unique)
        if nu > cap:
            return self.unique_votes(model, scene, d_dist, ref_df, cap=nu)
        return {"codes": codes[:nu], "counts": counts[:nu], "n_votes": int(res.n_votes),
                "elapsed_ms": float(res.elapsed_ms)}

    def post(self, model, scene, d_dist, codes, counts, use_l1_norm=False, use_averaged_clusters=False,
             weights=None):
        """Poses, weighted counts, clustering and the best pose of kept votes
        given in the reference's order (count descending, code ascending)."""
        mp, mn = _f32(model[0]), _f32(model[1])
        sp, sn = _f32(scene[0]), _f32(scene[1])
        c = np.ascontiguousarray(np.asarray(codes, np.uint64))
        k = np.ascontiguousarray(np.asarray(counts, np.uint32))
        U = c.size
        res = rh_result()
        T = np.zeros(U * 16, np.float32)
        t = np.zeros(U * 3, np.float32)
        q = np.zeros(U * 4, np.float32)
        s = np.zeros(U, np.float32)
        w = _f32(weights) if weights is not None else None
        rc = self.L.rh_post(_p(mp), _p(mn), mp.shape[0], _p(sp), _p(sn), sp.shape[0], float(d_dist),
                            int(use_l1_norm), int(use_averaged_clusters), _p(w) if w is not None else None,
                            _p(c, _u64p), _p(k, _u32p), U, C.byref(res), _p(T), _p(t), _p(q), _p(s))
        self._err(rc, "rh_post")
        return {"max_idx": int(res.max_idx), "pose": np.array(res.pose[:], np.float32).reshape(4, 4),
                "transforms": T.reshape(-1, 16), "trans": t.reshape(-1, 3), "quats": q.reshape(-1, 4),
                "scores": s, "elapsed_ms": float(res.elapsed_ms)}


def available(kind: str) -> bool:
    names = {"oracle": HERE / "libppf_oracle.so", "ref_host": HERE / "_ref" / "libppfref_host.so",
             "ref_gpu": HERE / "_ref" / "libppfref_gpu.so"}
    return names[kind].exists()


def n_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1
