"""FP16-acc lane layouts: one lane per (pixel, candidate) item, or a lane pair splitting the window's
even and odd taps (hp_params.lanes_per_pixel).  The pair forms every FP16 value with the same
operations in the same order and flushes the row sums into FP32 in the one-lane order, so the two
layouts must agree bit for bit - costs of fixed hypotheses, whole solves (both plan schedules), at
several window shapes including odd widths and the bounds-checked border path."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import cam_of

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def setup(hp, scene_mod):
    s = scene_mod.plane_sphere(w=200, h=136, seed=3)
    ctx = hp.Context(0)
    ids = [ctx.upload(v.image) for v in s.views]
    yield s, ctx, ids
    ctx.close()


def _job(hp, s, ids, r, iterations=3):
    srcs = s.sources[r]
    return hp.make_job(ids[r], [ids[i] for i in srcs], hp.make_camera(*cam_of(s, r)),
                       [hp.make_camera(*cam_of(s, i)) for i in srcs], *s.depth_range, seed=5, view_id=r,
                       iterations=iterations)


@pytest.mark.parametrize("radius,stride", [(7, 2), (5, 2), (5, 1), (3, 1), (6, 2), (2, 2)])
def test_lane_pair_cost_equals_single_lane(hp, setup, radius, stride):
    s, ctx, ids = setup
    job = _job(hp, s, ids, 1)
    m, d, n, _ = hp.host_maps(s.height, s.width)
    ctx.init_hypotheses(job, hp.default_params(), m)
    out = []
    for lanes in (1, 2):
        c = np.zeros(d.shape, np.float32)
        ctx.ncc_cost(job, hp.default_params(radius=radius, stride=stride, precision=hp.PRECISION_F16ACC,
                                            lanes_per_pixel=lanes), hp.maps_of(d.copy(), n.copy(), c))
        out.append(c)
    assert np.array_equal(out[0], out[1]), float(np.abs(out[0] - out[1]).max())
    assert (out[0] < 2).mean() > 0.5


@pytest.mark.parametrize("radius,stride", [(7, 2), (4, 1)])
def test_lane_pair_solve_equals_single_lane(hp, setup, radius, stride):
    s, ctx, ids = setup
    jobs = [_job(hp, s, ids, r) for r in (0, 2, 4)]
    res = []
    for lanes in (1, 2):
        outs = [hp.host_maps(s.height, s.width) for _ in jobs]
        ctx.solve(jobs, hp.default_params(radius=radius, stride=stride, precision=hp.PRECISION_F16ACC,
                                          lanes_per_pixel=lanes), [o[0] for o in outs])
        res.append([o[1:] for o in outs])
    for a, b in zip(*res):
        for x, y in zip(a, b):
            assert np.array_equal(x, y)


@pytest.mark.parametrize("schedule", [1, 2])
def test_lane_pair_plans_equal_solve(hp, setup, schedule):
    s, ctx, ids = setup
    jobs = [_job(hp, s, ids, r, iterations=it) for r, it in ((1, 3), (3, 2))]
    p1 = hp.default_params(radius=7, stride=2, precision=hp.PRECISION_F16ACC, lanes_per_pixel=1)
    want = [hp.host_maps(s.height, s.width) for _ in jobs]
    ctx.solve(jobs, p1, [w[0] for w in want])
    p2 = hp.default_params(radius=7, stride=2, precision=hp.PRECISION_F16ACC, lanes_per_pixel=2)
    got = [hp.host_maps(s.height, s.width) for _ in jobs]
    with hp.Plan(ctx, jobs, p2, [g[0] for g in got], hp.plan_options(schedule=schedule)) as plan:
        plan.run()
    for g, w in zip(got, want):
        for x, y in zip(g[1:], w[1:]):
            assert np.array_equal(x, y)


def test_lanes_param_validated(hp, setup):
    s, ctx, ids = setup
    with pytest.raises(hp.HpError):
        ctx.solve([_job(hp, s, ids, 0)], hp.default_params(lanes_per_pixel=3), [hp.host_maps(s.height, s.width)[0]])
