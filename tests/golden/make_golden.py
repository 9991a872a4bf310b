"""Generates tests/golden/reference_host_vectors.npz from the reference's own
arithmetic helpers (src/cuda/kernel.cu compiled for the host in place, see
oracle/Makefile target `ref`).  Run where oracle/_ref/libppfref_host.so has
been built:

    make -C oracle ref && python tests/golden/make_golden.py

Vectors: 400 seeded random (model pair, scene pair) combinations from the
plain single-model workload, with the reference's discretised feature, key,
alpha bin, vote pose, quaternion and pose-cell keys for each.
"""
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import __graft_entry__ as ge  # noqa: E402


def main(n=400, seed=2024):
    pkg = ge.load_package()
    orc = ge.load_oracle()
    R = orc.RefHost()
    spec = pkg.synthetic.config_plain(seed=1000)
    m, s, d = spec.models[0], spec.scene, np.float32(spec.d_dists[0])
    rng = np.random.default_rng(seed)
    out = {k: [] for k in ("p1", "n1", "p2", "n2", "p3", "n3", "p4", "feature", "key", "alpha", "bin", "pose",
                           "quat", "cell", "adj")}
    for _ in range(n):
        i, j = rng.integers(0, len(m), 2)
        k, l = rng.integers(0, len(s), 2)
        b = int(rng.integers(0, 31))
        f = R.pair_feature(m.points[i], m.normals[i], m.points[j], m.normals[j], d)
        T = R.vote_pose(b, m.points[i], m.normals[i], s.points[k], s.normals[k])
        cell, adj = R.cell_keys(T[:3, 3], d)
        out["p1"].append(m.points[i]); out["n1"].append(m.normals[i])
        out["p2"].append(m.points[j]); out["n2"].append(m.normals[j])
        out["p3"].append(s.points[k]); out["n3"].append(s.normals[k]); out["p4"].append(s.points[l])
        out["feature"].append(f); out["key"].append(R.feature_key(f))
        out["alpha"].append(R.alpha_bin(m.points[i], m.normals[i], m.points[j], s.points[k], s.normals[k], s.points[l]))
        out["bin"].append(b); out["pose"].append(T); out["quat"].append(R.quat(T))
        out["cell"].append(cell); out["adj"].append(adj)
    arrs = {k: np.array(v) for k, v in out.items()}
    arrs["key"] = arrs["key"].astype(np.uint32)
    arrs["cell"] = arrs["cell"].astype(np.uint32)
    arrs["alpha"] = arrs["alpha"].astype(np.uint32)
    arrs["d_dist"] = np.float32(d)
    path = Path(__file__).resolve().parent / "reference_host_vectors.npz"
    np.savez_compressed(path, **arrs)
    print("wrote", path, {k: v.shape for k, v in arrs.items()})


if __name__ == "__main__":
    main()
