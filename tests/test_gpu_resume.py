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


def test_upload_size_limit(hp, rctx):
    """Image sides are capped at 16384 px (the software sampler's fixed-point coordinate range)."""
    with pytest.raises(hp.HpError):
        rctx.upload(np.zeros((2, 16385), np.uint8))
