"""Pose-error bookkeeping of bench.py's recall report: rotation error modulo
each synthetic shape's symmetry, and the counts at the north star's bounds
(1% of the diameter, 2 degrees) and the reference driver's validation bounds
(0.1 diameter, 12 degrees; src/alignment.cpp:300-335)."""
import types

import numpy as np
import pytest

import bench


def _rot(axis, deg):
    a = np.radians(deg)
    c, s = np.cos(a), np.sin(a)
    return {"x": np.array([[1, 0, 0], [0, c, -s], [0, s, c]]),
            "y": np.array([[c, 0, s], [0, 1, 0], [-s, 0, c]]),
            "z": np.array([[c, -s, 0], [s, c, 0], [0, 0, 1]])}[axis]


def test_rotation_error_modulo_symmetry(pkg):
    err = pkg.synthetic.rotation_error_deg
    G = _rot("x", 20) @ _rot("y", -35)
    assert err(G, G) == pytest.approx(0.0, abs=1e-4)
    assert err(G @ _rot("z", 30), G) == pytest.approx(30.0, abs=1e-4)
    # the torus is symmetric about its axis and under a half-turn about x
    assert err(G @ _rot("z", 30), G, "torus") == pytest.approx(0.0, abs=1e-4)
    assert err(G @ _rot("x", 180), G, "torus") == pytest.approx(0.0, abs=1e-3)
    assert err(G @ _rot("x", 30), G, "torus") == pytest.approx(30.0, abs=1e-4)
    # the superellipsoid's three half-turns
    for ax in "xyz":
        assert err(G @ _rot(ax, 180), G, "superellipsoid") == pytest.approx(0.0, abs=1e-3)
    assert err(G @ _rot("z", 90), G, "superellipsoid") == pytest.approx(90.0, abs=1e-4)
    # the capsule union has no symmetry
    assert err(G @ _rot("y", 180), G, "capsules") == pytest.approx(180.0, abs=1e-3)


def test_recall_counts_at_both_bounds(pkg):
    G = np.eye(4)
    shifted = np.eye(4)
    shifted[0, 3] = 0.05  # half a diameter of 0.1
    turned = np.eye(4)
    turned[:3, :3] = _rot("z", 5)
    inst = [types.SimpleNamespace(model_index=k, pose=G) for k in range(3)]
    spec = types.SimpleNamespace(instances=inst, diameters=[0.1, 0.1, 0.1],
                                 models=[None] * 3, extra={"families": ["capsules", "capsules", "torus"]})
    r = bench.recall_of(spec, [np.eye(4), shifted, turned])
    assert r["at_1pct_2deg"] == "1/3"
    assert r["at_reference_bounds_0.1diam_12deg"] == "2/3"
    # the torus's 5 degrees about its own axis vanish modulo its symmetry
    assert r["modulo_shape_symmetry"]["at_1pct_2deg"] == "2/3"
    assert r["terr_over_diam_and_deg"][1][0] == pytest.approx(0.5)
