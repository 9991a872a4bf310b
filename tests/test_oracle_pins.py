"""The CPU oracle against the reference's own code (CPU, no GPU needed).

The oracle (oracle/ppf_oracle.cpp) must reproduce, bit for bit, the
reference's __host__ build of its arithmetic helpers (src/cuda/kernel.cu,
built in place into oracle/_ref/libppfref_host.so) and the golden vectors in
tests/golden/ that were generated from that build.  NaN results compare equal
to NaN (the two builds produce different NaN payloads).
"""
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


def _same(a, b):
    a = np.asarray(a, np.float32)
    b = np.asarray(b, np.float32)
    return bool(np.all((a.view(np.uint32) == b.view(np.uint32)) | (np.isnan(a) & np.isnan(b))))


@pytest.fixture(scope="module")
def cfg(pkg):
    return pkg.synthetic.config_plain(seed=21, n_model=600, n_plane=800, n_box=300)


def test_pair_features_and_keys_match_reference(oracle, ref_host, cfg):
    m, s, d = cfg.models[0], cfg.scene, cfg.d_dists[0]
    rng = np.random.default_rng(1)
    for _ in range(3000):
        i, j = rng.integers(0, len(m), 2)
        k, l = rng.integers(0, len(s), 2)
        for P, N, a, b in ((m.points, m.normals, i, j), (s.points, s.normals, k, l)):
            fo = oracle.pair_feature(P[a], N[a], P[b], N[b], d)
            fr = ref_host.pair_feature(P[a], N[a], P[b], N[b], d)
            assert _same(fo, fr)
            assert oracle.feature_key(fo) == ref_host.feature_key(fr)


def test_alpha_bins_match_reference(oracle, ref_host, cfg):
    m, s = cfg.models[0], cfg.scene
    rng = np.random.default_rng(2)
    for _ in range(3000):
        i, j = rng.integers(0, len(m), 2)
        k, l = rng.integers(0, len(s), 2)
        args = (m.points[i], m.normals[i], m.points[j], s.points[k], s.normals[k], s.points[l])
        assert oracle.alpha_bin(*args) == ref_host.alpha_bin(*args)


def test_poses_quaternions_cells_match_reference(oracle, ref_host, cfg):
    m, s, d = cfg.models[0], cfg.scene, cfg.d_dists[0]
    rng = np.random.default_rng(3)
    for _ in range(2000):
        i = rng.integers(0, len(m))
        k = rng.integers(0, len(s))
        b = int(rng.integers(0, 31))
        To = oracle.vote_pose(b, m.points[i], m.normals[i], s.points[k], s.normals[k])
        Tr = ref_host.vote_pose(b, m.points[i], m.normals[i], s.points[k], s.normals[k])
        assert _same(To, Tr)
        assert _same(oracle.quat(Tr), ref_host.quat(Tr))
        ko, ao = oracle.cell_keys(Tr[:3, 3], d)
        kr, ar = ref_host.cell_keys(Tr[:3, 3], d)
        assert ko == kr and np.array_equal(ao, ar)


def test_fnv_signed_char_semantics(oracle):
    import ctypes as C

    for data in (b"\x00\x7f\x80\xff", b"\xff" * 16, bytes(range(256))[:16]):
        buf = C.create_string_buffer(data, len(data))
        h = 2166136261
        for byte in data:
            sb = byte - 256 if byte >= 128 else byte
            h ^= sb & 0xFFFFFFFF
            h = (h * 16777619) & 0xFFFFFFFF
        assert oracle.L.orc_fnv1a(buf, len(data), 2166136261) == h


def _golden(name):
    p = GOLDEN / name
    if not p.exists():
        pytest.skip(f"{p} not generated")
    return np.load(p)


def test_oracle_against_golden_vectors(oracle):
    g = _golden("reference_host_vectors.npz")
    for r in range(g["p1"].shape[0]):
        f = oracle.pair_feature(g["p1"][r], g["n1"][r], g["p2"][r], g["n2"][r], float(g["d_dist"]))
        assert _same(f, g["feature"][r])
        assert oracle.feature_key(f) == int(g["key"][r])
        a = oracle.alpha_bin(g["p1"][r], g["n1"][r], g["p2"][r], g["p3"][r], g["n3"][r], g["p4"][r])
        assert a == int(g["alpha"][r])
        T = oracle.vote_pose(int(g["bin"][r]), g["p1"][r], g["n1"][r], g["p3"][r], g["n3"][r])
        assert _same(T, g["pose"][r])
        assert _same(oracle.quat(T), g["quat"][r])
        k, adj = oracle.cell_keys(g["pose"][r][:3, 3], float(g["d_dist"]))
        assert k == int(g["cell"][r]) and np.array_equal(adj, g["adj"][r])


def test_hash_array_is_stable_sort(oracle):
    rng = np.random.default_rng(4)
    keys = rng.integers(0, 50, size=5000).astype(np.uint32)
    keys[rng.random(5000) < 0.1] = 0
    H = oracle.hash_array(keys)
    order = np.argsort(keys, kind="stable")
    assert np.array_equal(H["map"], order)
    u, first, counts = np.unique(keys[order], return_index=True, return_counts=True)
    assert np.array_equal(H["keys"], u) and np.array_equal(H["first"], first) and np.array_equal(H["counts"], counts)


def test_oracle_votes_match_literal_restatement(oracle, pkg):
    """The oracle's factored vote loop equals a literal per-vote
    trans_model_scene loop (same bits on the host) on a tiny case."""
    spec = pkg.synthetic.config_plain(seed=5, n_model=60, n_plane=60, n_box=30)
    m, s, d = spec.models[0], spec.scene, spec.d_dists[0]
    mk = oracle.pair_keys(m.points, m.normals, d)
    H = oracle.hash_array(mk)
    sk = oracle.pair_keys(s.points, s.normals, d, ref_df=5)
    acc = {}
    n_m, n_s = len(m), len(s)
    for r in range(0, n_s, 5):
        for i in range(n_s):
            k = sk[r, i]
            if k == 0:
                continue
            pos = np.searchsorted(H["keys"], k)
            if pos >= H["keys"].size or H["keys"][pos] != k:
                continue
            for e in range(H["first"][pos], H["first"][pos] + H["counts"][pos]):
                pr = int(H["map"][e])
                mr, mi = divmod(pr, n_m)
                b = oracle.alpha_bin(m.points[mr], m.normals[mr], m.points[mi], s.points[r], s.normals[r], s.points[i])
                code = (r << 32) | (mr << 6) | b
                acc[code] = acc.get(code, 0) + 1
    R = oracle.register((m.points, m.normals), (s.points, s.normals), d, 5, 0.0)
    assert R["n_unique"] == len(acc)
    assert R["max_count"] == max(acc.values())
    kept = {int(c): int(n) for c, n in zip(R["codes"], R["counts"])}
    thr = np.float32(0.0) * np.float32(R["max_count"])
    assert kept == {c: n for c, n in acc.items() if np.float32(n) > thr}
    # reference order: count descending, then code ascending
    order = sorted(kept.items(), key=lambda kv: (-kv[1], kv[0]))
    assert [c for c, _ in order] == [int(c) for c in R["codes"]]


def test_cpu_greedy_clustering_properties(oracle):
    rng = np.random.default_rng(6)
    poses, votes = [], []
    base = [np.eye(4), np.eye(4)]
    base[1][:3, 3] = [0.5, 0, 0]
    for k in range(40):
        T = base[k % 2].copy()
        T[:3, 3] += rng.normal(scale=1e-3, size=3)
        poses.append(T.astype(np.float32).ravel())
        votes.append(10 + (k % 2) * 5 + k)
    out, ov = oracle.cluster_poses(np.array(poses), np.array(votes, np.uint32), 0.01, np.deg2rad(12))
    assert len(out) == 2
    assert ov[0] >= ov[1]
    assert np.allclose(out[0][:3, :3], np.eye(3), atol=1e-5)
