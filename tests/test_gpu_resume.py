"""Checkpoint and resume of solver state through PFM files, and the device memory of uploads.

A view's solver state is exactly its (depth, normal, cost) maps: the random streams are keyed on
(seed, view, pixel, iteration), not on a running generator.  So a solve stopped after k iterations,
written to PFM (saveDepthMapPFM's format, extended to the 3-channel normal map), read back and
continued with hp_propagate_pass from iteration k must equal the uninterrupted solve bit for bit.
Tolerance: identity."""
from __future__ import annotations

import numpy as np
import pytest

from conftest import cam_of

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def rctx(hp):
    with hp.Context(0) as c:
        yield c


@pytest.mark.parametrize("precision", [0, 1])
def test_resume_from_pfm_checkpoint_is_exact(hp, rctx, small_scene, tmp_path, precision):
    s = small_scene
    ids = [rctx.upload(v.image) for v in s.views]
    try:
        r = 1
        srcs = s.sources[r]
        params = hp.default_params(radius=5, stride=1, precision=precision)

        def job(iters):
            return hp.make_job(ids[r], [ids[i] for i in srcs], hp.make_camera(*cam_of(s, r)),
                               [hp.make_camera(*cam_of(s, i)) for i in srcs], *s.depth_range, seed=9, view_id=r,
                               iterations=iters)

        full_m, full_d, full_n, full_c = hp.host_maps(s.height, s.width)
        rctx.solve([job(6)], params, [full_m])
        part_m, part_d, part_n, part_c = hp.host_maps(s.height, s.width)
        rctx.solve([job(3)], params, [part_m])
        for name, a in (("depth", part_d), ("normal", part_n), ("cost", part_c)):
            hp.pfm_write(str(tmp_path / f"{name}.pfm"), a)
        d = np.ascontiguousarray(hp.pfm_read(str(tmp_path / "depth.pfm")))
        n = np.ascontiguousarray(hp.pfm_read(str(tmp_path / "normal.pfm")))
        c = np.ascontiguousarray(hp.pfm_read(str(tmp_path / "cost.pfm")))
        assert np.array_equal(d, part_d) and np.array_equal(n, part_n) and np.array_equal(c, part_c)
        maps = hp.maps_of(d, n, c)
        for it in range(3, 6):
            rctx.propagate_pass(job(6), params, maps, it, 0)
            rctx.propagate_pass(job(6), params, maps, it, 1)
        assert np.array_equal(d, full_d) and np.array_equal(n, full_n) and np.array_equal(c, full_c)
    finally:
        for i in ids:
            rctx.release(i)


def test_uploads_release_their_device_memory(hp, rctx, small_scene):
    """Every upload holds FP32 / FP16 planes, two texture arrays and the sparse quad plane; releasing the
    images must give it all back (measured with the context's device-memory query)."""
    import torch
    img = small_scene.views[0].image
    big = np.ascontiguousarray(np.resize(img, (1500, 2100)).astype(np.uint8))
    rctx.set_image_cache(0)  # released images are freed, not kept for reuse
    rctx.synchronize()
    torch.cuda.synchronize()
    free0, _ = rctx.mem_info()
    for _ in range(3):
        ids = [rctx.upload(big) for _ in range(8)]
        held = free0 - rctx.mem_info()[0]
        assert held >= 8 * big.size * 18, held  # about 20 bytes per pixel per upload
        for i in ids:
            rctx.release(i)
        rctx.synchronize()
        assert abs(rctx.mem_info()[0] - free0) <= 64 << 20, (free0, rctx.mem_info()[0])
    # With the cache on, released images are kept and the next uploads of that size take them over.
    rctx.set_image_cache(4 << 30)
    for i in [rctx.upload(big) for _ in range(8)]:
        rctx.release(i)
    kept = rctx.mem_info()[0]
    assert free0 - kept >= 8 * big.size * 18
    ids = [rctx.upload(big) for _ in range(8)]
    assert rctx.mem_info()[0] >= kept - (16 << 20), "uploads of a cached size allocated new memory"
    for i in ids:
        rctx.release(i)
    rctx.set_image_cache(0)
    assert abs(rctx.mem_info()[0] - free0) <= 64 << 20


def test_upload_size_limit(hp, rctx):
    """Image sides are capped at 16384 px (the software sampler's fixed-point coordinate range)."""
    with pytest.raises(hp.HpError):
        rctx.upload(np.zeros((2, 16385), np.uint8))


def test_image_cache_reuse_gives_identical_results(hp, small_scene):
    """Released images lend their buffers to later uploads of the same size; solves over reused buffers
    (holding the same or different pixels) equal solves over fresh ones, and the cache stays bounded."""
    s = small_scene
    r, srcs = 0, s.sources[0]

    def solve(ctx, ids):
        job = hp.make_job(ids[r], [ids[i] for i in srcs], hp.make_camera(*cam_of(s, r)),
                          [hp.make_camera(*cam_of(s, i)) for i in srcs], *s.depth_range, seed=3, view_id=r,
                          iterations=3)
        m, d, n, c = hp.host_maps(s.height, s.width)
        ctx.solve([job], hp.default_params(radius=5, stride=2, precision=1), [m])
        return d, c

    with hp.Context(0) as fresh:
        want = solve(fresh, [fresh.upload(v.image) for v in s.views])
        flipped = [np.ascontiguousarray(v.image[:, ::-1]) for v in s.views]
        want_flipped = solve(fresh, [fresh.upload(x) for x in flipped])
    with hp.Context(0) as ctx:
        ids = [ctx.upload(x) for x in flipped]
        for i in ids:
            ctx.release(i)  # cached
        got = solve(ctx, [ctx.upload(v.image) for v in s.views])  # reuses the flipped images' buffers
        assert all(np.array_equal(a, b) for a, b in zip(got, want))
        ctx.set_image_cache(0)
        got2 = solve(ctx, [ctx.upload(x) for x in flipped])
        assert all(np.array_equal(a, b) for a, b in zip(got2, want_flipped))
