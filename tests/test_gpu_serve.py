"""The request loop (ppf_server_*) against plain lookups.

Requests submitted from two threads are admitted, batched and overlapped by
two workers; every target of every request must give the same pose and vote
statistics as Model.ppf_lookup of that (model, scene) alone, whatever the
mix it ran in.  Poses and integer statistics are compared exactly.
"""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def library(pkg, ctx):
    specs = [pkg.synthetic.config_plain(seed=s, n_model=nm, n_plane=np_, n_box=nb)
             for s, nm, np_, nb in ((121, 600, 1200, 400), (122, 1700, 2000, 700), (123, 2300, 1800, 500))]
    models = [pkg.Model(sp.models[0], sp.d_dists[0], sp.vote_count_threshold, context=ctx) for sp in specs]
    requests = []  # (scene cloud, ref_df, target ids)
    for k, sp in enumerate(specs):
        requests.append((sp.scene, 5, [k]))
        requests.append((sp.scene, 5, [0, 1, 2]))
        requests.append((sp.scene, 1 + 2 * k, [(k + 1) % 3, k]))
    return specs, models, requests


def _expected(pkg, ctx, specs, models, requests):
    out = []
    for cloud, df, ids in requests:
        poses, stats = [], []
        for j in ids:
            scene = pkg.Scene(cloud, specs[j].d_dists[0], df, context=ctx)
            poses.append(models[j].ppf_lookup(scene, raise_on_no_votes=False).copy())
            stats.append(dict(models[j].stats))
        out.append((poses, stats))
    return out


def _serve(pkg, models, requests, **kw):
    srv = pkg.Server(models, **kw)
    tickets = [None] * len(requests)

    def submit(idx):
        for i in idx:
            cloud, df, ids = requests[i]
            tickets[i] = srv.submit(cloud, ids, df)

    th = [threading.Thread(target=submit, args=(range(s, len(requests), 2),)) for s in (0, 1)]
    for t in th:
        t.start()
    for t in th:
        t.join()
    res = [srv.wait(t, raise_on_no_votes=False) for t in tickets]
    srv.close()
    return res


@pytest.mark.parametrize("kw", [dict(workers=2, max_batch=4), dict(workers=2, max_batch=16, memory_budget=1)])
def test_served_results_equal_plain_lookups(pkg, ctx, library, kw):
    specs, models, requests = library
    want = _expected(pkg, ctx, specs, models, requests)
    got = _serve(pkg, models, requests, **kw)
    for i, ((poses, stats), (gp, gs, lat)) in enumerate(zip(want, got)):
        assert lat > 0
        for t in range(len(poses)):
            assert np.array_equal(gp[t], poses[t]), (i, t)
            for key in ("n_votes", "max_vote_count", "n_kept", "max_idx", "best_score"):
                assert gs[t][key] == stats[t][key], (i, t, key)


def test_server_rejects_bad_requests(pkg, library):
    import torch

    specs, models, _ = library
    srv = pkg.Server(models, workers=1)
    with pytest.raises(pkg.PPFError):
        srv.submit(specs[0].scene, [7])
    dev = (torch.from_numpy(specs[0].scene.points).cuda(), torch.from_numpy(specs[0].scene.normals).cuda())
    with pytest.raises(pkg.PPFError):
        srv.submit(dev, [0])
    t = srv.submit(specs[0].scene, [0], 5)
    srv.wait(t)
    with pytest.raises(pkg.PPFError):
        srv.wait(t)
    srv.close()
