"""PLY ingest and ground-truth validation of the alignment driver
(src/alignment.cpp:212,241,300-335, src/cuda/linalg.cu:9-20), on the CPU
through the library's own reader."""
import struct

import numpy as np
import pytest


def _cloud(n=50, seed=0):
    rng = np.random.default_rng(seed)
    p = rng.normal(size=(n, 3)).astype(np.float32)
    q = rng.normal(size=(n, 3)).astype(np.float32)
    return p, q / np.linalg.norm(q, axis=1, keepdims=True)


def test_binary_round_trip(pkg, tmp_path):
    p, q = _cloud()
    pkg.save_ply(tmp_path / "a.ply", (p, q))
    rp, rq = pkg.load_ply(tmp_path / "a.ply")
    np.testing.assert_array_equal(rp, p)
    np.testing.assert_array_equal(rq, q)


def test_big_endian_doubles_with_faces(pkg, tmp_path):
    p, q = _cloud(7, 1)
    hdr = ("ply\nformat binary_big_endian 1.0\nelement vertex 7\nproperty double x\nproperty double y\n"
           "property double z\nproperty uchar red\nproperty double nx\nproperty double ny\nproperty double nz\n"
           "element face 2\nproperty list uchar int vertex_indices\nend_header\n").encode()
    body = b"".join(struct.pack(">dddBddd", *p[i], 200, *q[i]) for i in range(7))
    body += struct.pack(">Biii", 3, 0, 1, 2) + struct.pack(">Biiii", 4, 0, 1, 2, 3)
    (tmp_path / "b.ply").write_bytes(hdr + body)
    rp, rq = pkg.load_ply(tmp_path / "b.ply")
    np.testing.assert_array_equal(rp, p)
    np.testing.assert_array_equal(rq, q)


def test_ascii_with_pcl_normal_names(pkg, tmp_path):
    p, q = _cloud(5, 2)
    lines = ["ply", "format ascii 1.0", "element vertex 5", "property float x", "property float y",
             "property float z", "property float normal_x", "property float normal_y", "property float normal_z",
             "property float curvature", "element face 1", "property list uchar int vertex_indices", "end_header"]
    lines += [" ".join(f"{v:.9g}" for v in (*p[i], *q[i], 0.0)) for i in range(5)] + ["3 0 1 2"]
    (tmp_path / "c.ply").write_text("\n".join(lines) + "\n")
    rp, rq = pkg.load_ply(tmp_path / "c.ply")
    np.testing.assert_array_equal(rp, p)
    np.testing.assert_array_equal(rq, q)


def test_missing_normals_is_an_error(pkg, tmp_path):
    (tmp_path / "d.ply").write_text("ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\nproperty float y\n"
                                    "property float z\nend_header\n0 0 0\n")
    with pytest.raises(pkg.PPFError, match="normals"):
        pkg.load_ply(tmp_path / "d.ply")


def test_xf_and_ht_dist(pkg, tmp_path):
    T = np.eye(4, dtype=np.float32)
    T[:3, 3] = (0.1, -0.2, 0.3)
    (tmp_path / "g.xf").write_text("\n".join(" ".join(f"{v:g}" for v in row) for row in T) + "\n")
    G = pkg.load_xf(tmp_path / "g.xf")
    np.testing.assert_array_equal(G, T)
    c, s = np.cos(np.pi / 2), np.sin(np.pi / 2)
    R = np.eye(4, dtype=np.float32)
    R[:2, :2] = [[c, -s], [s, c]]
    R[:3, 3] = (0.1, -0.2, 0.3 + 0.05)
    td, rd = pkg.ht_dist(R, G)
    assert abs(td - 0.05) < 1e-6 and abs(rd - np.pi / 2) < 1e-6
    # 170 degrees about a tilted axis
    ax = np.array([1.0, 2.0, 2.0]) / 3.0
    th = np.deg2rad(170.0)
    K = np.array([[0, -ax[2], ax[1]], [ax[2], 0, -ax[0]], [-ax[1], ax[0], 0]])
    R2 = np.eye(4, dtype=np.float32)
    R2[:3, :3] = np.eye(3) + np.sin(th) * K + (1 - np.cos(th)) * K @ K
    assert abs(pkg.ht_dist(R2, np.eye(4))[1] - th) < 1e-5
    ok, _ = pkg.validate(R, G, model_diameter=1.0)
    assert not ok  # 90 degrees off
    ok, _ = pkg.validate(G, G, model_diameter=1.0)
    assert ok
