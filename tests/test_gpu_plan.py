"""Plans (hp_plan_*): the batched form.  Views of uneven size, source count and
iteration count solved together; every schedule (per-pass launches or one
persistent launch, direct or replayed as a CUDA graph, any resident-CTA
count, the autotuner's pick) must give exactly what hp_solve gives - the
tolerance is bit-identity, because the per-pixel arithmetic never depends on
how tiles are scheduled.  A persistent dependency wait that runs out must end
the launch with HP_ERR_TIMEOUT and leave the context usable."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import cam_of

pytestmark = pytest.mark.gpu

HP_ERR_TIMEOUT = 5


@pytest.fixture(scope="module")
def batch(hp, scene_mod):
    a = scene_mod.plane_sphere(w=192, h=136, seed=7)  # 3 x 17 tiles, ragged bottom row
    b = scene_mod.plane_sphere(w=130, h=70, seed=8)   # ragged in x and y
    ctx = hp.Context(0)
    ids_a = [ctx.upload(v.image) for v in a.views]
    ids_b = [ctx.upload(v.image) for v in b.views]

    def job(s, ids, r, n_src, iters, seed):
        srcs = s.sources[r][:n_src]
        return hp.make_job(ids[r], [ids[i] for i in srcs], hp.make_camera(*cam_of(s, r)),
                           [hp.make_camera(*cam_of(s, i)) for i in srcs], *s.depth_range, seed=seed, view_id=r,
                           iterations=iters)

    jobs = [job(a, ids_a, 1, 4, 3, 11), job(b, ids_b, 0, 3, 2, 12), job(a, ids_a, 2, 2, 0, 13),
            job(b, ids_b, 3, 4, 1, 14)]
    shapes = [(136, 192), (70, 130), (136, 192), (70, 130)]
    yield ctx, jobs, shapes
    ctx.close()


def _reference(hp, ctx, jobs, shapes, params):
    outs = [hp.host_maps(h, w) for h, w in shapes]
    ctx.solve(jobs, params, [o[0] for o in outs])
    return [o[1:] for o in outs]


def _plan_outputs(hp, ctx, jobs, shapes, params, options, device, runs=2):
    import torch
    results = []
    if device:
        arrs = [(torch.full((h, w), -1.0, device="cuda"), torch.full((h, w, 3), -1.0, device="cuda"),
                 torch.full((h, w), -1.0, device="cuda")) for h, w in shapes]
        maps = [hp.maps_of(*a) for a in arrs]
    else:
        outs = [hp.host_maps(h, w) for h, w in shapes]
        maps = [o[0] for o in outs]
        arrs = [o[1:] for o in outs]
    with hp.Plan(ctx, jobs, params, maps, options) as plan:
        for _ in range(runs):
            plan.run()
            results.append([[t.cpu().numpy() if device else t.copy() for t in a] for a in arrs])
        info = plan.info()
    return results, info


@pytest.mark.parametrize("precision", [0, 1])
def test_every_schedule_matches_solve(hp, batch, precision):
    ctx, jobs, shapes = batch
    params = hp.default_params(radius=3, stride=1, precision=precision)
    want = _reference(hp, ctx, jobs, shapes, params)
    variants = [
        (dict(schedule=hp.SCHEDULE_PER_PASS, use_graph=1), True),
        (dict(schedule=hp.SCHEDULE_PER_PASS, use_graph=0), False),
        (dict(schedule=hp.SCHEDULE_PERSISTENT, use_graph=1, ctas_per_sm=1), True),
        (dict(schedule=hp.SCHEDULE_PERSISTENT, use_graph=1, ctas_per_sm=0), False),
        (dict(schedule=hp.SCHEDULE_PERSISTENT, use_graph=0), True),
    ]
    for opts, device in variants:
        results, info = _plan_outputs(hp, ctx, jobs, shapes, params, hp.plan_options(**opts), device)
        assert info["schedule"] == opts["schedule"]
        if opts["schedule"] == hp.SCHEDULE_PERSISTENT:
            assert info["launches_per_run"] == 1 and info["grid"] >= 1
            assert info["tickets"] == sum(((w + 63) // 64) * ((h + 7) // 8) * (2 * j.iterations + 2)
                                          for (h, w), j in zip(shapes, jobs))
        for got in results:
            for g, w in zip(got, want):
                for a, b in zip(g, w):
                    assert np.array_equal(a, b), (opts, device)


def test_autotuner_picks_a_candidate_and_keeps_results(hp, batch):
    ctx, jobs, shapes = batch
    params = hp.default_params(radius=5, stride=2, precision=1)
    want = _reference(hp, ctx, jobs, shapes, params)
    outs = [hp.host_maps(h, w) for h, w in shapes]
    with hp.Plan(ctx, jobs, params, [o[0] for o in outs]) as plan:
        best = plan.tune(repeats=2)
        assert best["schedule"] in (hp.SCHEDULE_PER_PASS, hp.SCHEDULE_PERSISTENT)
        assert best["tuned_ms"] > 0
        if best["schedule"] == hp.SCHEDULE_PERSISTENT:
            assert 1 <= best["ctas_per_sm"] <= best["max_ctas_per_sm"]
        assert plan.info()["schedule"] == best["schedule"]
        for o, w in zip(outs, want):
            for a, b in zip(o[1:], w):
                assert np.array_equal(a, b)
        plan.run()
        for o, w in zip(outs, want):
            for a, b in zip(o[1:], w):
                assert np.array_equal(a, b)


def test_persistent_wait_runs_out_cleanly(hp, batch):
    """A tile that never reports completion: its dependants' bounded waits give up, the launch ends with
    HP_ERR_TIMEOUT, and the context (and a plan without the stall) keeps working."""
    ctx, jobs, shapes = batch
    params = hp.default_params(radius=2, stride=1)
    outs = [hp.host_maps(h, w) for h, w in shapes]
    opts = hp.plan_options(schedule=hp.SCHEDULE_PERSISTENT, wait_limit_ms=100, debug_stall_view=0,
                           debug_stall_tile=4)
    with hp.Plan(ctx, jobs, params, [o[0] for o in outs], opts) as plan:
        for _ in range(2):
            with pytest.raises(hp.HpError) as ei:
                plan.run()
            assert ei.value.status == HP_ERR_TIMEOUT
    want = _reference(hp, ctx, jobs, shapes, params)
    results, _ = _plan_outputs(hp, ctx, jobs, shapes, params, hp.plan_options(schedule=hp.SCHEDULE_PERSISTENT),
                               device=False, runs=1)
    for g, w in zip(results[0], want):
        for a, b in zip(g, w):
            assert np.array_equal(a, b)


def test_plan_launch_wait_device_outputs(hp, batch):
    import torch
    ctx, jobs, shapes = batch
    params = hp.default_params(radius=3, stride=2, precision=1)
    want = _reference(hp, ctx, jobs, shapes, params)
    arrs = [(torch.zeros(h, w, device="cuda"), torch.zeros(h, w, 3, device="cuda"), torch.zeros(h, w, device="cuda"))
            for h, w in shapes]
    with hp.Plan(ctx, jobs, params, [hp.maps_of(*a) for a in arrs]) as plan:
        plan.launch()
        plan.wait()
        for a, w in zip(arrs, want):
            for t, b in zip(a, w):
                assert np.array_equal(t.cpu().numpy(), b)
    host = [hp.host_maps(h, w)[0] for h, w in shapes]
    with hp.Plan(ctx, jobs, params, host) as plan:
        with pytest.raises(hp.HpError):
            plan.launch()  # host outputs need hp_plan_run
