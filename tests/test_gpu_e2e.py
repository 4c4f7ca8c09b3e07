"""End-to-end behaviour of the CUDA path: accuracy against renderer ground truth
and against the reference's own solver, FP16 vs FP32 agreement, determinism,
batching invariance, the stage API, device-resident buffers and error paths."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import cam_of

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx(hp):
    with hp.Context(0) as c:
        yield c


@pytest.fixture(scope="module")
def ids_full(ctx, full_scene):
    return [ctx.upload(v.image) for v in full_scene.views]


def job_for(hp, scene, ids, r, iterations=8, seed=42):
    srcs = scene.sources[r]
    return hp.make_job(ids[r], [ids[i] for i in srcs], hp.make_camera(*cam_of(scene, r)),
                       [hp.make_camera(*cam_of(scene, i)) for i in srcs], *scene.depth_range, seed=seed,
                       view_id=r, iterations=iterations)


def solve(hp, ctx, scene, ids, refs, params, iterations=8):
    jobs, outs, res = [], [], []
    for r in refs:
        m, d, n, c = hp.host_maps(scene.height, scene.width)
        jobs.append(job_for(hp, scene, ids, r, iterations))
        outs.append(m)
        res.append((d, n, c))
    ctx.solve(jobs, params, outs)
    return res


def completeness(d, gt, tol=0.01):
    return float((np.abs(d - gt) / gt <= tol).mean())


def test_accuracy_matches_reference_solver(hp, ctx, ids_full, full_scene):
    """Engine FP32 vs the reference's own per-view solve (radius 5, stride 1, 8 iterations) on
    the same images and cameras, scored against renderer ground truth: completeness at 1%
    relative depth within 2 points of the reference's, mean relative error no worse than 1.1x."""
    import pmref
    if not pmref.available():
        pytest.skip("reference harness not built")
    s = full_scene
    p = hp.default_params(radius=5, stride=1)
    for r in (0, 2):
        d, _, _ = solve(hp, ctx, s, ids_full, [r], p)[0]
        srcs = s.sources[r]
        kinv, ab = pmref.setup_views(cam_of(s, r), [cam_of(s, i) for i in srcs])
        dr, _, _, _ = pmref.solve_view(s.views[r].image_f32, [s.views[i].image_f32 for i in srcs], kinv, ab,
                                       *s.depth_range, 5, 8, r)
        gt = s.views[r].depth_gt
        ce, cr = completeness(d, gt), completeness(dr, gt)
        ee, er = float((np.abs(d - gt) / gt).mean()), float((np.abs(dr - gt) / gt).mean())
        assert ce >= cr - 0.02 and ce > 0.6, (ce, cr)
        assert ee <= 1.1 * er + 1e-3, (ee, er)


def test_fp16acc_depth_agrees_with_fp32(hp, ctx, ids_full, full_scene):
    """>= 99% of pixels within 0.5% relative depth of the FP32 result."""
    s = full_scene
    p32 = hp.default_params(radius=5, stride=2)
    p16 = hp.default_params(radius=5, stride=2, precision=hp.PRECISION_F16ACC)
    refs = [0, 2, 4]
    a = solve(hp, ctx, s, ids_full, refs, p32)
    b = solve(hp, ctx, s, ids_full, refs, p16)
    for (d32, _, _), (d16, _, _) in zip(a, b):
        assert (np.abs(d16 - d32) / d32 <= 0.005).mean() >= 0.99


@pytest.mark.parametrize("precision", [0, 1])
def test_deterministic_and_batch_invariant(hp, ctx, ids_full, full_scene, precision):
    """A view's result is bit-identical run to run and alone vs inside a batch (the RNG is keyed
    on (seed, view, pixel, iteration) and no arithmetic crosses pixels)."""
    s = full_scene
    p = hp.default_params(radius=5, stride=2, precision=precision)
    alone = solve(hp, ctx, s, ids_full, [3], p)[0]
    again = solve(hp, ctx, s, ids_full, [3], p)[0]
    batch = solve(hp, ctx, s, ids_full, [1, 3, 4], p)[1]
    for a, b, c in zip(alone, again, batch):
        assert np.array_equal(a, b) and np.array_equal(a, c)


@pytest.mark.parametrize("precision", [0, 1])
def test_stored_cost_equals_recomputed_cost(hp, ctx, ids_full, full_scene, precision):
    """The cost a solve stores for a pixel is bit-identical to what the full-map cost kernel
    computes for the final plane.  The propagate kernel relies on this when it skips a neighbour
    plane equal to the current one: re-scoring it could not produce a lower number."""
    s = full_scene
    p = hp.default_params(radius=5, stride=2, precision=precision)
    d, n, c = solve(hp, ctx, s, ids_full, [2], p, iterations=3)[0]
    again = np.zeros_like(c)
    ctx.ncc_cost(job_for(hp, s, ids_full, 2), p, hp.maps_of(d, n, again))
    assert np.array_equal(c, again)


def test_uneven_iterations_in_one_batch(hp, ctx, ids_full, full_scene):
    s = full_scene
    p = hp.default_params(radius=5, stride=2)
    jobs, outs, res = [], [], []
    for r, it in [(0, 2), (1, 5), (2, 0)]:
        m, d, n, c = hp.host_maps(s.height, s.width)
        jobs.append(job_for(hp, s, ids_full, r, it))
        outs.append(m)
        res.append(d)
    ctx.solve(jobs, p, outs)
    for (r, it), d in zip([(0, 2), (1, 5), (2, 0)], res):
        alone = solve(hp, ctx, s, ids_full, [r], p, iterations=it)[0][0]
        assert np.array_equal(d, alone)


def test_stage_api_end_to_end(hp, full_scene, tmp_path):
    """run_patchmatch_mvs mirrors runPatchMatchMVS: 5 views, geometric filter, PFM output.
    EndToEndFilterAndAccuracy (tests/test_patchmatch.cpp:446-539) bounds on this scene:
    mean relative error of retained pixels < 0.15 (here < 0.02), retention >= 0.5.  As in the
    reference, the PFM files hold each view's depth before the filter (:1254-1257); the filtered maps
    are the same whether the filter ran fused into the solve or after the write."""
    s = full_scene
    cams = [hp.make_camera(*cam_of(s, i)) for i in range(len(s.views))]
    views = [hp.ViewParams(r, s.sources[r], *s.depth_range) for r in s.refs]
    imgs = [v.image for v in s.views]
    cfg = hp.MVSConfig(mvs_iterations=8, mvs_patch_size=11, window_stride=2, save_intermediate=True,
                       output_dir=str(tmp_path))
    maps = hp.run_patchmatch_mvs(imgs, cams, views, cfg)
    fused = hp.run_patchmatch_mvs(imgs, cams, views, hp.MVSConfig(mvs_iterations=8, mvs_patch_size=11,
                                                                   window_stride=2))
    raw = hp.run_patchmatch_mvs(imgs, cams, views, hp.MVSConfig(mvs_iterations=8, mvs_patch_size=11,
                                                                 window_stride=2, geometric_filter=False))
    assert [m.image_id for m in maps] == s.refs
    kept, err = [], []
    for m, f, r in zip(maps, fused, raw):
        gt = s.views[m.image_id].depth_gt
        k = m.depth > 0
        kept.append(k.mean())
        err.append((np.abs(m.depth[k] - gt[k]) / gt[k]).mean())
        assert ((m.confidence >= 0) & (m.confidence <= 1)).all()
        assert np.array_equal(m.depth, f.depth) and np.array_equal(m.confidence, f.confidence)
        assert np.array_equal(hp.pfm_read(str(tmp_path / f"depth_{m.image_id}.pfm")), r.depth)
    assert np.mean(kept) >= 0.5 and np.mean(err) < 0.02, (kept, err)


def test_device_resident_buffers(hp, ctx, full_scene):
    import torch
    s = full_scene
    dev_ids = [ctx.upload(torch.from_numpy(v.image).cuda()) for v in s.views]
    host_ids = [ctx.upload(v.image) for v in s.views]
    p = hp.default_params(radius=5, stride=2)
    jd = job_for(hp, s, dev_ids, 1)
    d = torch.zeros(s.height, s.width, device="cuda")
    n = torch.zeros(s.height, s.width, 3, device="cuda")
    c = torch.zeros(s.height, s.width, device="cuda")
    ctx.solve([jd], p, [hp.maps_of(d, n, c)])
    ref = solve(hp, ctx, s, host_ids, [1], p)[0]
    assert np.array_equal(d.cpu().numpy(), ref[0]) and np.array_equal(c.cpu().numpy(), ref[2])
    for i in dev_ids + host_ids:
        ctx.release(i)


def test_image_dtypes_agree(hp, ctx, full_scene):
    s = full_scene
    img = s.views[0].image_f32
    a = ctx.upload(s.views[0].image)
    b = ctx.upload(img)
    c16 = ctx.upload(img.astype(np.float16))
    assert ctx  # uploads succeeded; u8 and f32 of the same values give identical solves
    srcs = [ctx.upload(s.views[i].image) for i in s.sources[0]]
    p = hp.default_params(radius=3, stride=2)
    out = []
    for ref in (a, b):
        job = hp.make_job(ref, srcs, hp.make_camera(*cam_of(s, 0)), [hp.make_camera(*cam_of(s, i)) for i in s.sources[0]],
                          *s.depth_range, iterations=2)
        m, d, _, _ = hp.host_maps(s.height, s.width)
        ctx.solve([job], p, [m])
        out.append(d)
    assert np.array_equal(out[0], out[1])
    for i in [a, b, c16, *srcs]:
        ctx.release(i)


def test_error_paths(hp, ctx, ids_full, full_scene):
    s = full_scene
    job = job_for(hp, s, ids_full, 0)
    m, *_ = hp.host_maps(s.height, s.width)
    for bad in (dict(radius=8), dict(radius=0), dict(stride=3), dict(top_k=4), dict(precision=7),
                dict(refine_steps=9), dict(iter_decay=0.0)):
        with pytest.raises(hp.HpError) as e:
            ctx.solve([job], hp.default_params(**bad), [m])
        assert e.value.status == 1
    # Tile shapes: 64 x 8, and 64 x 4 on the FP16-acc path only.
    for tile in (dict(tile_w=32), dict(tile_h=16), dict(tile_h=4), dict(tile_h=4, precision=0)):
        with pytest.raises(hp.HpError) as e:
            ctx.solve([job], hp.default_params(**tile), [m])
        assert e.value.status == 6
    ctx.solve([job], hp.default_params(tile_w=64, tile_h=8), [m])
    ctx.solve([job], hp.default_params(tile_h=4, precision=1), [m])
    with pytest.raises(hp.HpError) as e:
        ctx.solve([job], hp.default_params(staging=6, precision=1), [m])
    assert e.value.status == 1
    bad_job = job_for(hp, s, ids_full, 0)
    bad_job.ref_image = 999999
    with pytest.raises(hp.HpError) as e:
        ctx.solve([bad_job], hp.default_params(), [m])
    assert e.value.status == 4 and "unknown ref image" in str(e.value)
    bad_job = job_for(hp, s, ids_full, 0)
    bad_job.depth_min, bad_job.depth_max = 3.0, 2.0
    with pytest.raises(hp.HpError):
        ctx.solve([bad_job], hp.default_params(), [m])
    small = ctx.upload(np.zeros((10, 12), np.uint8))
    bad_job = job_for(hp, s, ids_full, 0)
    bad_job.src_images[0] = small
    with pytest.raises(hp.HpError) as e:
        ctx.solve([bad_job], hp.default_params(), [m])
    assert "source 0" in str(e.value)
    with pytest.raises(hp.HpError):
        ctx.upload(np.zeros((1, 5), np.uint8))
    with pytest.raises(hp.HpError):
        ctx.release(123456)
    ctx.release(small)
    free, total = ctx.mem_info()
    assert 0 < free <= total
