"""FP16-acc kernel variants the batched form's autotuner chooses between: the tile height (64 x 8
pixels per CTA with 8 warps, or 64 x 4 with 4) and the staging depth (4 or 8 quad loads in flight per
window row).  They change how work is grouped into CTAs and when loads are issued, never the
arithmetic of a pixel, so every variant must give the same bits - initial costs, whole solves (ragged
tiles at the view edges included), plans under both schedules, with and without the fused filter."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import cam_of

pytestmark = pytest.mark.gpu

VARIANTS = [(8, 4), (8, 8), (4, 4), (4, 8)]  # (tile_h, staging); (8, 4) is the default


@pytest.fixture(scope="module")
def setup(hp, scene_mod):
    s = scene_mod.plane_sphere(w=200, h=138, seed=3)  # ragged in x (200 = 3 x 64 + 8) and y (138 = 34 x 4 + 2)
    ctx = hp.Context(0)
    ids = [ctx.upload(v.image) for v in s.views]
    yield s, ctx, ids
    ctx.close()


def _job(hp, s, ids, r, iterations=3):
    srcs = s.sources[r]
    return hp.make_job(ids[r], [ids[i] for i in srcs], hp.make_camera(*cam_of(s, r)),
                       [hp.make_camera(*cam_of(s, i)) for i in srcs], *s.depth_range, seed=5 + r, view_id=r,
                       iterations=iterations)


def _params(hp, tile_h, staging, **kw):
    return hp.default_params(precision=hp.PRECISION_F16ACC, tile_h=tile_h, staging=staging, **kw)


@pytest.mark.parametrize("radius,stride", [(7, 2), (5, 1), (3, 2)])
def test_variants_give_the_same_cost(hp, setup, radius, stride):
    s, ctx, ids = setup
    job = _job(hp, s, ids, 1)
    m, d, n, _ = hp.host_maps(s.height, s.width)
    ctx.init_hypotheses(job, hp.default_params(), m)
    out = []
    for th, dd in VARIANTS:
        c = np.zeros(d.shape, np.float32)
        ctx.ncc_cost(job, _params(hp, th, dd, radius=radius, stride=stride), hp.maps_of(d.copy(), n.copy(), c))
        out.append(c)
    for c in out[1:]:
        assert np.array_equal(c, out[0])


@pytest.mark.parametrize("filtered", [False, True])
def test_variants_give_the_same_solve(hp, setup, filtered):
    s, ctx, ids = setup
    jobs = [_job(hp, s, ids, r) for r in s.refs]
    extra = dict(filter_min_consistent=2) if filtered else {}
    res = []
    for th, dd in VARIANTS:
        outs = [hp.host_maps(s.height, s.width, confidence=True) for _ in jobs]
        ctx.solve(jobs, _params(hp, th, dd, radius=7, stride=2, **extra), [o[0] for o in outs])
        res.append([o[1:] for o in outs])
    for r in res[1:]:
        for a, b in zip(r, res[0]):
            for x, y in zip(a, b):
                assert np.array_equal(x, y)


@pytest.mark.parametrize("schedule", [1, 2])
def test_tile4_plans_equal_solve(hp, setup, schedule):
    s, ctx, ids = setup
    jobs = [_job(hp, s, ids, r, iterations=it) for r, it in ((0, 3), (2, 2), (4, 1))]
    want = [hp.host_maps(s.height, s.width) for _ in jobs]
    ctx.solve(jobs, _params(hp, 8, 4, radius=7, stride=2, filter_min_consistent=2), [w[0] for w in want])
    got = [hp.host_maps(s.height, s.width) for _ in jobs]
    with hp.Plan(ctx, jobs, _params(hp, 4, 8, radius=7, stride=2, filter_min_consistent=2), [g[0] for g in got],
                 hp.plan_options(schedule=schedule)) as plan:
        for _ in range(2):
            plan.run()
            for g, w in zip(got, want):
                for x, y in zip(g[1:], w[1:]):
                    assert np.array_equal(x, y)


def test_tuner_chooses_tile_and_staging(hp, setup):
    """Left at 0, the tile height and staging depth are the autotuner's: it rebuilds the plan for the
    other tile height, times each combination, and the maps still equal hp_solve's."""
    s, ctx, ids = setup
    jobs = [_job(hp, s, ids, r) for r in (1, 3)]
    params = hp.default_params(precision=hp.PRECISION_F16ACC, radius=5, stride=2)
    want = [hp.host_maps(s.height, s.width) for _ in jobs]
    ctx.solve(jobs, params, [w[0] for w in want])
    got = [hp.host_maps(s.height, s.width) for _ in jobs]
    with hp.Plan(ctx, jobs, params, [g[0] for g in got]) as plan:
        best = plan.tune(repeats=1)
        assert best["tile_h"] in (4, 8) and best["staging"] in (4, 8)
        assert plan.info()["tile_h"] == best["tile_h"]
        for g, w in zip(got, want):
            for x, y in zip(g[1:], w[1:]):
                assert np.array_equal(x, y)
        plan.run()
        for g, w in zip(got, want):
            for x, y in zip(g[1:], w[1:]):
                assert np.array_equal(x, y)

