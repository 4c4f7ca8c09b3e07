"""The largest view size of the batched and serving mixes - 4000x3000 on a 9-view +-30 degree arc, the
serving form's cameras (fx = 3125) - pinned against the reference's own kernels.

The engine's FP32 hp_ncc_cost and the reference's cost kernels (compiled unmodified by oracle/ref_harness)
run on identical fixed hypotheses with the reference's own homography coefficients:
computePixelCost (src/dense_recon/patchmatch_mvs.cu:222-343) at radius 7 and compute_ncc_cost_kernel
(:349-513) at its radius limit 5, stride 1.  Warped coordinates here reach 4000 px, four times the ulp of
the sub-1024 px views the other parity tests use, so a texture weight flips wherever the two computations
of a coordinate differ by a rounding.  Bound: |engine - reference| <= 1e-5 on every pixel."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import cam_of

pytestmark = pytest.mark.gpu

REFS = (0, 8)  # the arc's ends: every source lies to one side, baselines up to 60 degrees


@pytest.fixture(scope="module")
def scene(scene_mod):
    return scene_mod.multi_object(seed=33, w=4000, h=3000, n_views=9, n_src=6, f=1500.0 * 4000 / 1920.0,
                                  n_refs=9)


@pytest.fixture(scope="module")
def ctx(hp):
    with hp.Context(0) as c:
        yield c


@pytest.fixture(scope="module")
def ids(ctx, scene):
    return [ctx.upload(v.image) for v in scene.views]


@pytest.fixture(scope="module")
def pmref():
    import pmref as m
    if not m.available():
        pytest.skip("reference harness not built (needs the reference tree at build time)")
    return m


@pytest.mark.parametrize("r", REFS)
@pytest.mark.parametrize("radius,kernel", [(7, "pixel"), (5, "ncc")])
def test_cost_matches_reference_at_4000x3000(hp, ctx, ids, scene, pmref, r, radius, kernel):
    s = scene
    srcs = s.sources[r]
    kinv, ab = pmref.setup_views(cam_of(s, r), [cam_of(s, i) for i in srcs])
    job = hp.make_job(ids[r], [ids[i] for i in srcs], hp.make_camera(*cam_of(s, r)),
                      [hp.make_camera(*cam_of(s, i)) for i in srcs], *s.depth_range, seed=7 + r, view_id=r,
                      iterations=1, coeffs=(kinv, ab))
    m, d, n, _ = hp.host_maps(s.height, s.width)
    ctx.init_hypotheses(job, hp.default_params(), m)
    planes = {"random": (d, n), "true": (s.views[r].depth_gt.astype(np.float32),
                                         np.ascontiguousarray(s.views[r].normal_gt, np.float32))}
    params = hp.default_params(radius=radius, stride=1)
    for tag, (dd, nn) in planes.items():
        c = np.zeros(dd.shape, np.float32)
        ctx.ncc_cost(job, params, hp.maps_of(dd.copy(), nn.copy(), c))
        want = pmref.ncc_cost(s.views[r].image_f32, [s.views[i].image_f32 for i in srcs], kinv, ab, dd, nn,
                              radius, kernel=kernel)
        err = np.abs(c.astype(np.float64) - want)
        assert err.max() <= 1e-5, (tag, float(err.max()), float((err > 0).mean()))
        if tag == "true":
            assert (want < 1.0).mean() > 0.5, "true planes correlate"


BAND = (2900, 2940)  # rows near the bottom edge: the quad plane's last block row, coordinates up to 4000 px


@pytest.mark.parametrize("planes", ["true", "random"])
def test_fp16_ncc_vs_fp64_oracle_at_4000x3000(hp, po, ctx, ids, scene, planes):
    """FP16-acc cost on fixed hypotheses against the FP64 oracle with the engine's sampler model (every
    source through the software sampler), over a band of rows at the bottom of a 4000x3000 view at an arc's
    end, with the FP32 path against its own FP64 model (the texture unit's weights) measured beside it.

    At this size a warped coordinate's FP32 ulp is 2.4e-4 px, and on random hypotheses both paths exceed
    1e-3 on about 0.1% of the band (measured: FP16 99.84%, FP32 99.89% within; largest errors about 0.02):
    windows whose taps sit on 8-bit weight boundaries or whose contrast is near the 1e-6 floor.  So the
    bound here is the FP32 path's own agreement, minus 0.1 point.  On the true planes every pixel is within
    1e-3 except validity flips (one side 2, the other finite: a tap on the valid-region edge turns the
    count rule), at most 1 in 10 000.  The oracle reads the images as the FP16 path stores them."""
    s, r = scene, 8
    srcs = s.sources[r]
    job = hp.make_job(ids[r], [ids[i] for i in srcs], hp.make_camera(*cam_of(s, r)),
                      [hp.make_camera(*cam_of(s, i)) for i in srcs], *s.depth_range, seed=11, view_id=r,
                      iterations=1)
    if planes == "true":
        d = s.views[r].depth_gt.astype(np.float32)
        n = np.ascontiguousarray(s.views[r].normal_gt, np.float32)
    else:
        m, d, n, _ = hp.host_maps(s.height, s.width)
        ctx.init_hypotheses(job, hp.default_params(), m)
    costs = {}
    for prec in (hp.PRECISION_F16ACC, hp.PRECISION_F32):
        c = np.zeros(d.shape, np.float32)
        ctx.ncc_cost(job, hp.default_params(radius=7, stride=2, precision=prec), hp.maps_of(d.copy(), n.copy(), c))
        costs[prec] = c
    as16 = lambda a: a.astype(np.float16).astype(np.float32)
    v16 = po.View(as16(s.views[r].image_f32), [as16(s.views[i].image_f32) for i in srcs], radius=7, stride=2,
                  ref_cam=cam_of(s, r), src_cams=[cam_of(s, i) for i in srcs])
    v32 = po.View(s.views[r].image_f32, [s.views[i].image_f32 for i in srcs], radius=7, stride=2,
                  ref_cam=cam_of(s, r), src_cams=[cam_of(s, i) for i in srcs])
    y0, y1 = BAND
    po.set_soft_sources(0xFF)
    try:
        q64 = v16.cost_rows_f64(d, n, y0, y1, quantized=True)
    finally:
        po.set_soft_sources(0)
    t64 = v32.cost_rows_f64(d, n, y0, y1, quantized=True)
    c16 = costs[hp.PRECISION_F16ACC][y0:y1].astype(np.float64)
    e16 = np.abs(c16 - q64)
    e32 = np.abs(costs[hp.PRECISION_F32][y0:y1].astype(np.float64) - t64)
    within16, within32 = float((e16 <= 1e-3).mean()), float((e32 <= 1e-3).mean())
    if planes == "random":
        assert within16 >= within32 - 1e-3, (within16, within32)
        assert max(float(e16.max()), float(e32.max())) < 0.1
    else:
        over = e16 > 1e-3
        flips = over & ((c16 == 2.0) != (q64 == 2.0))
        assert np.array_equal(over, flips), (float(e16[over & ~flips].max()) if (over & ~flips).any() else 0.0)
        assert over.mean() <= 1e-4, float(over.mean())


def test_filter_matches_reference_kernel_at_4000x3000(hp, ctx, scene, pmref):
    """The geometric-consistency check on caller maps (hp_geometric_filter, own arithmetic) against the
    reference's kernel (geometric_consistency_filter_kernel, patchmatch_mvs.cu:668-781) at 4000x3000: an
    arc-end view against its two nearest sources, depths with 8% multiplicative noise, the normal check
    off and at 30 degrees.  At least 99.99% of depths and confidences identical (the rest are projections
    within a rounding of a pixel boundary or of the tolerance, where the two arithmetics round apart)."""
    s = scene
    rng = np.random.default_rng(5)
    r, srcs = 8, s.sources[8][:2]
    maps = {}
    for i in [r] + srcs:
        d = s.views[i].depth_gt * (1 + rng.normal(0, 0.08, s.views[i].depth_gt.shape))
        maps[i] = (np.ascontiguousarray(d, np.float32), np.ascontiguousarray(s.views[i].normal_gt, np.float32))
    for cos_tol in (-1.0, float(np.cos(np.radians(30)))):
        de, ce = maps[r][0].copy(), np.full(maps[r][0].shape, 0.5, np.float32)
        ctx.geometric_filter(hp.make_camera(*cam_of(s, r)), de, maps[r][1], ce,
                             [hp.make_camera(*cam_of(s, i)) for i in srcs], [maps[i][0] for i in srcs],
                             [maps[i][1] for i in srcs], 0.12, cos_tol, 2)
        dr, cr = maps[r][0].copy(), np.full(maps[r][0].shape, 0.5, np.float32)
        pmref.geometric_filter(cam_of(s, r), dr, maps[r][1], cr, [cam_of(s, i) for i in srcs],
                               [maps[i][0] for i in srcs], [maps[i][1] for i in srcs], 0.12, cos_tol, 2)
        assert (de == dr).mean() >= 0.9999 and (ce == cr).mean() >= 0.9999, ((de == dr).mean(), (ce == cr).mean())
        assert 0.05 < (de == 0).mean() < 0.95, "the test maps exercise both outcomes"


@pytest.mark.parametrize("precision", [0, 1])
def test_persistent_plan_and_server_equal_solve_at_4000x3000(hp, ctx, ids, scene, precision):
    """Two 4000x3000 views (23 625 tiles each at 64x8) through one persistent plan and through the server
    give hp_solve's maps bit for bit: the ticket schedule at the largest view size of the mixes."""
    s = scene
    jobs = [hp.make_job(ids[r], [ids[i] for i in s.sources[r][:4]], hp.make_camera(*cam_of(s, r)),
                        [hp.make_camera(*cam_of(s, i)) for i in s.sources[r][:4]], *s.depth_range, seed=90 + r,
                        view_id=r, iterations=2) for r in (0, 8)]
    params = hp.default_params(radius=7, stride=2, precision=precision)
    want = [hp.host_maps(s.height, s.width) for _ in jobs]
    ctx.solve(jobs, params, [w[0] for w in want])
    got = [hp.host_maps(s.height, s.width) for _ in jobs]
    with hp.Plan(ctx, jobs, params, [g[0] for g in got], hp.plan_options(schedule=hp.SCHEDULE_PERSISTENT)) as plan:
        plan.run()
    for g, w in zip(got, want):
        for a, b in zip(g[1:], w[1:]):
            assert np.array_equal(a, b)
    srv_out = [hp.host_maps(s.height, s.width) for _ in jobs]
    with hp.Server(ctx, params, passes_per_step=3) as srv:
        for j, o in zip(jobs, srv_out):
            srv.submit(j, o[0])
        srv.drain(timeout_ms=120000)
        done = srv.poll(capacity=8)
    assert len(done) == 2 and all(c["status"] == 0 for c in done)
    for g, w in zip(srv_out, want):
        for a, b in zip(g[1:], w[1:]):
            assert np.array_equal(a, b)
