"""Batched lookups (ppf_lookup_batch) against one ppf_model_lookup per request.

A request's result must not depend on the other requests in its batch: the
pose, the vote statistics and the kept votes of every request equal those of
the same (model, scene) looked up alone.  Integer results and poses are
compared exactly.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("n_votes", "n_matched_pairs", "max_vote_count", "n_kept", "max_idx", "best_score")


@pytest.fixture(scope="module")
def library(pkg, ctx):
    specs = [pkg.synthetic.config_plain(seed=s, n_model=nm, n_plane=np_, n_box=nb)
             for s, nm, np_, nb in ((81, 700, 1500, 500), (82, 1800, 2500, 800), (83, 2600, 2000, 600))]
    models, scenes = [], []
    for k, spec in enumerate(specs):
        d = spec.d_dists[0]
        models.append(pkg.Model(spec.models[0], d, spec.vote_count_threshold, context=ctx))
        # every model against its own scene and the next spec's scene
        for j in (k, (k + 1) % len(specs)):
            scenes.append((k, pkg.Scene(specs[j].scene, d, specs[j].ref_point_df, context=ctx)))
    return specs, models, scenes


def _alone(model, scene):
    pose = model.ppf_lookup(scene, raise_on_no_votes=False).copy()
    codes, counts = model.get_votes()
    return pose, dict(model.stats), codes, counts


def _check_batch(pkg, ctx, models, scenes, order):
    ms = [models[scenes[i][0]] for i in order]
    ss = [scenes[i][1] for i in order]
    poses, stats = pkg.lookup_batch(ms, ss, context=ctx, return_stats=True, raise_on_no_votes=False)
    for j, i in enumerate(order):
        pose, st, _, _ = _alone(ms[j], ss[j])
        assert np.array_equal(poses[j], pose), (j, i)
        for k in KEYS:
            assert stats[j][k] == st[k], (j, i, k)
    return poses, stats


def test_batch_equals_single_lookups(pkg, ctx, library):
    _, models, scenes = library
    order = list(range(len(scenes)))
    _check_batch(pkg, ctx, models, scenes, order)
    # reversed, with the first model repeated, gives the same per-request results
    _check_batch(pkg, ctx, models, scenes, order[::-1] + [0, 1])


def test_batch_kept_votes_equal(pkg, ctx, library):
    _, models, scenes = library
    for i in range(len(scenes)):
        m, s = models[scenes[i][0]], scenes[i][1]
        _, _, codes, counts = _alone(m, s)
        pkg.lookup_batch([m], [s], context=ctx, raise_on_no_votes=False)
        c2, k2 = m.get_votes()
        assert np.array_equal(codes, c2) and np.array_equal(counts, k2)


def test_batch_candidate_growth(pkg, ctx, library, monkeypatch):
    _, models, scenes = library
    monkeypatch.setenv("PPF_B200_BATCH_CAP", "2048")
    poses, stats = _check_batch(pkg, ctx, models, scenes, list(range(len(scenes))))
    assert any(s["n_redo_items"] > 0 for s in stats)


def test_batch_request_without_votes(pkg, ctx, library):
    specs, models, scenes = library
    tiny = pkg.Scene((specs[0].scene.points[:1], specs[0].scene.normals[:1]), specs[0].d_dists[0], 1, context=ctx)
    ms = [models[0], models[0]]
    ss = [scenes[0][1], tiny]
    with pytest.raises(pkg.PPFError):
        pkg.lookup_batch(ms, ss, context=ctx)
    poses, stats = pkg.lookup_batch(ms, ss, context=ctx, return_stats=True, raise_on_no_votes=False)
    pose, _, _, _ = _alone(models[0], scenes[0][1])
    assert np.array_equal(poses[0], pose)
    assert stats[1]["n_kept"] == 0 and not poses[1].any()


def test_registration_scenes_by_models_equals_lookups(pkg, ctx, library):
    specs, _, _ = library
    scenes = [specs[0].scene, specs[2].scene]
    ms = [sp.models[0] for sp in specs]
    ds = [sp.d_dists[0] for sp in specs]
    poses, stats = pkg.ppf_registration(scenes, ms, ds, 5, 0.3, return_stats=True)
    for i, sc in enumerate(scenes):
        for j, (m, d) in enumerate(zip(ms, ds)):
            model = pkg.Model(m, d, 0.3, context=ctx)
            pose = model.ppf_lookup(pkg.Scene(sc, d, 5, context=ctx), raise_on_no_votes=False)
            assert np.array_equal(poses[i][j], pose), (i, j)
            assert stats[i][j]["n_votes"] == model.stats["n_votes"]
            assert stats[i][j]["n_kept"] == model.stats["n_kept"]


def test_batch_modes_equal_single_lookups(pkg, ctx, library):
    """L1, averaged-cluster and greedy (cpu_clustering) models in one batch:
    each request equals its single lookup."""
    specs, _, scenes = library
    sp = specs[1]
    d = sp.d_dists[0]
    kinds = [dict(use_l1_norm=True), dict(use_averaged_clusters=True), dict(cpu_clustering=True), {}]
    models = [pkg.Model(sp.models[0], d, sp.vote_count_threshold, context=ctx, **kw) for kw in kinds]
    scene = pkg.Scene(sp.scene, d, sp.ref_point_df, context=ctx)
    poses, stats = pkg.lookup_batch(models, [scene] * len(models), context=ctx, return_stats=True)
    for j, m in enumerate(models):
        pose, st, _, _ = _alone(m, scene)
        assert np.array_equal(poses[j], pose), kinds[j]
        for k in KEYS:
            assert stats[j][k] == st[k], (kinds[j], k)
