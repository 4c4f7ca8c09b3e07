"""The geometric-consistency filter as the last stage of a solve (hp_params.filter_*).

The reference runs geometric_consistency_filter_kernel view by view after the solve, in place, each
view against its sources' maps as they stand - earlier views already filtered, later ones not
(src/dense_recon/patchmatch_mvs.cu:668-781, :1267-1384).  Here the same check runs on the packed
plane state inside hp_solve, inside plans (per-pass launches and the persistent ticket schedule),
and on caller maps through hp_geometric_filter.  Tolerance: bit-identity between all of these (they
share one device function, every float operation explicitly rounded), and the confidence map is
exactly 1 - cost / 2.  Agreement with the reference kernel itself is in test_gpu_parity.py."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import cam_of

pytestmark = pytest.mark.gpu

FILTER = dict(filter_min_consistent=2, filter_depth_tol=0.12, filter_normal_cos=-1.0)


@pytest.fixture(scope="module")
def views(hp, scene_mod):
    s = scene_mod.plane_sphere(w=200, h=136, seed=5)  # 4 x 17 tiles, ragged in x
    ctx = hp.Context(0)
    ids = [ctx.upload(v.image) for v in s.views]
    jobs = [hp.make_job(ids[r], [ids[i] for i in s.sources[r]], hp.make_camera(*cam_of(s, r)),
                        [hp.make_camera(*cam_of(s, i)) for i in s.sources[r]], *s.depth_range,
                        seed=42 + 1_000_000 * r, view_id=r, iterations=4) for r in s.refs]
    yield s, ctx, jobs
    ctx.close()


def _solve(hp, ctx, jobs, shape, params):
    outs = [hp.host_maps(*shape, confidence=True) for _ in jobs]
    ctx.solve(jobs, params, [o[0] for o in outs])
    return [o[1:] for o in outs]


def _sequential_filter(hp, s, ctx, solved, cos=-1.0):
    """hp_solve's maps filtered on the host side of the ABI: view by view, in place, each against the
    maps of the views that solved its sources (the reference's loop)."""
    out = [tuple(a.copy() for a in m) for m in solved]
    for k, r in enumerate(s.refs):
        d, n, c, cf = out[k]
        srcs = [i for i in s.sources[r] if i in s.refs and i != r]
        if len(srcs) < 2:
            continue
        ctx.geometric_filter(hp.make_camera(*cam_of(s, r)), d, n, cf, [hp.make_camera(*cam_of(s, i)) for i in srcs],
                             [out[s.refs.index(i)][0] for i in srcs], [out[s.refs.index(i)][1] for i in srcs],
                             0.12, cos, 2)
        c[cf == 0] = 2.0
    return out


@pytest.mark.parametrize("precision", [0, 1])
def test_fused_filter_equals_solve_then_filter(hp, views, precision):
    s, ctx, jobs = views
    shape = (s.height, s.width)
    plain = _solve(hp, ctx, jobs, shape, hp.default_params(radius=4, stride=2, precision=precision))
    for d, n, c, cf in plain:
        assert np.array_equal(cf, (1.0 - c * np.float32(0.5)).astype(np.float32))
    fused = _solve(hp, ctx, jobs, shape, hp.default_params(radius=4, stride=2, precision=precision, **FILTER))
    want = _sequential_filter(hp, s, ctx, plain)
    rejected = 0
    for (d, n, c, cf), (wd, wn, wc, wcf), (pd, pn, pc, pcf) in zip(fused, want, plain):
        assert np.array_equal(d, wd) and np.array_equal(n, wn) and np.array_equal(cf, wcf) and np.array_equal(c, wc)
        assert np.array_equal(n, pn), "the filter keeps normals"
        assert np.array_equal(d[d > 0], pd[d > 0]), "kept depths are the solve's"
        rejected += int((d == 0).sum())
    total = len(fused) * shape[0] * shape[1]
    assert 0.01 * total < rejected < 0.9 * total, "the test scene exercises both outcomes"


def test_filter_order_is_sequential(hp, views):
    """Later views see earlier views filtered: filtering every view against the unfiltered maps
    (all at once) differs from the fused result, which equals the sequential loop."""
    s, ctx, jobs = views
    shape = (s.height, s.width)
    plain = _solve(hp, ctx, jobs, shape, hp.default_params(radius=4, stride=2))
    fused = _solve(hp, ctx, jobs, shape, hp.default_params(radius=4, stride=2, **FILTER))
    at_once = []
    for k, r in enumerate(s.refs):
        d, n, c, cf = (a.copy() for a in plain[k])
        srcs = [i for i in s.sources[r] if i in s.refs and i != r]
        ctx.geometric_filter(hp.make_camera(*cam_of(s, r)), d, n, cf, [hp.make_camera(*cam_of(s, i)) for i in srcs],
                             [plain[s.refs.index(i)][0] for i in srcs], [plain[s.refs.index(i)][1] for i in srcs],
                             0.12, -1.0, 2)
        at_once.append(d)
    assert np.array_equal(fused[0][0], at_once[0]), "the first view sees no filtered source"
    assert any(not np.array_equal(f[0], a) for f, a in zip(fused[1:], at_once[1:]))


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("schedule", [1, 2])
@pytest.mark.parametrize("device", [False, True])
def test_plans_run_the_filter_stage(hp, views, precision, schedule, device):
    """Both plan schedules - per-pass launches, and the persistent kernel whose filter tickets wait for
    the whole solve and for the previous view's filter - give hp_solve's filtered maps."""
    import torch
    s, ctx, jobs = views
    shape = (s.height, s.width)
    params = hp.default_params(radius=4, stride=2, precision=precision, **FILTER)
    want = _solve(hp, ctx, jobs, shape, params)
    if device:
        arrs = [tuple(torch.full(sh, -1.0, device="cuda") for sh in (shape, shape + (3,), shape, shape))
                for _ in jobs]
        maps = [hp.maps_of(*a) for a in arrs]
    else:
        outs = [hp.host_maps(*shape, confidence=True) for _ in jobs]
        maps = [o[0] for o in outs]
        arrs = [o[1:] for o in outs]
    with hp.Plan(ctx, jobs, params, maps, hp.plan_options(schedule=schedule)) as plan:
        for _ in range(2):  # a replay resets the counters and flags
            plan.run()
            got = [tuple(a.cpu().numpy() if device else a for a in t) for t in arrs]
            for g, w in zip(got, want):
                for a, b in zip(g, w):
                    assert np.array_equal(a, b)


def test_filter_params_validated(hp, views):
    s, ctx, jobs = views
    m = [hp.host_maps(s.height, s.width)[0] for _ in jobs]
    for bad in (dict(filter_min_consistent=9), dict(filter_min_consistent=-1),
                dict(filter_min_consistent=2, filter_depth_tol=float("nan"))):
        with pytest.raises(hp.HpError):
            ctx.solve(jobs, hp.default_params(**bad), m)


def test_cpp_stage_adapter_runs_like_the_python_stage(hp, scene_mod, tmp_path):
    """include/hpmvs_stage.hpp's runPatchMatchMVS, executed inside the reference's own translation unit
    (oracle/_ref/libpmstage.so), gives run_patchmatch_mvs's depth, normal and confidence bit for bit -
    with the filter fused into the solve, and with intermediates written (filter after the write)."""
    import pmref
    if not pmref.stage_available():
        pytest.skip("stage harness not built (needs the reference tree at build time)")
    s = scene_mod.plane_sphere(w=160, h=120, seed=9)
    cams = [(v.cam.K, v.cam.R, v.cam.t) for v in s.views]
    pos, tracks = scene_mod.sparse_points(s, n=300, seed=3)
    C = [hp.make_camera(*c) for c in cams]
    grays = [v.image_f32 for v in s.views]
    for pfm in (False, True):
        out_dir = tmp_path / ("pfm" if pfm else "fused")
        out_dir.mkdir()
        st, got = pmref.stage_run(grays, cams, pos, tracks, patch_size=11, iterations=3,
                                  output_dir=str(out_dir) if pfm else None)
        assert st == 0
        cfg = hp.MVSConfig(mvs_iterations=3, mvs_patch_size=11, save_intermediate=pfm,
                           output_dir=str(tmp_path / "py") if pfm else None)
        if pfm:
            (tmp_path / "py").mkdir(exist_ok=True)
        want = hp.run_patchmatch_mvs(grays, C, config=cfg, sfm=hp.SfmPoints(pos, tracks))
        assert sorted(got) == [m.image_id for m in want]
        assert any((m.depth == 0).any() for m in want), "the filter ran"
        for m in want:
            d, n, cf = got[m.image_id]
            assert np.array_equal(d, m.depth) and np.array_equal(n, m.normal) and np.array_equal(cf, m.confidence)
            if pfm:
                assert np.array_equal(hp.pfm_read(str(out_dir / f"depth_{m.image_id}.pfm")),
                                      hp.pfm_read(str(tmp_path / "py" / f"depth_{m.image_id}.pfm")))
