"""hp_solve_static: the solve for callers that cannot let the library allocate device memory
(applications whose device memory belongs to their own pool or budget, or latency-critical loops
that cannot pay for cudaMalloc / cudaFree and their synchronisation).

Its scratch is a fixed, file-scope device array, so this file checks, through the C ABI, that two
calls in a row give exactly what hp_solve gives on the same inputs (the same kernels run; the
tolerance is the one the determinism tests use: bit-identical), that device memory does not move
across a call, and that views larger than the fixed maximum are refused.  The file name makes
pytest collect it last."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import cam_of

pytestmark = pytest.mark.gpu


def _texture(rt, t):
    """Linear-filter, clamp, unnormalised texture object over a contiguous device FP32 (H, W) tensor."""
    h, w = t.shape
    res = rt.cudaResourceDesc()
    res.resType = rt.cudaResourceType.cudaResourceTypePitch2D
    res.res.pitch2D.devPtr = t.data_ptr()
    res.res.pitch2D.desc = rt.cudaCreateChannelDesc(32, 0, 0, 0, rt.cudaChannelFormatKind.cudaChannelFormatKindFloat)[1]
    res.res.pitch2D.width = w
    res.res.pitch2D.height = h
    res.res.pitch2D.pitchInBytes = w * 4
    td = rt.cudaTextureDesc()
    td.addressMode = [rt.cudaTextureAddressMode.cudaAddressModeClamp] * 3
    td.filterMode = rt.cudaTextureFilterMode.cudaFilterModeLinear
    td.readMode = rt.cudaTextureReadMode.cudaReadModeElementType
    td.normalizedCoords = 0
    err, tex = rt.cudaCreateTextureObject(res, td, None)
    assert err == rt.cudaError_t.cudaSuccess, err
    return tex


def test_static_scratch_solve_matches_solve(hp, scene_mod):
    import torch
    from cuda.bindings import runtime as rt

    s = scene_mod.plane_sphere(w=192, h=128)
    r, srcs = 1, s.sources[1]
    H, W = s.height, s.width
    params = hp.default_params(radius=5, stride=2)

    # hp_solve through a context (it allocates its own scratch).
    with hp.Context(0) as ctx:
        ids = [ctx.upload(v.image) for v in s.views]
        job = hp.make_job(ids[r], [ids[i] for i in srcs], hp.make_camera(*cam_of(s, r)),
                          [hp.make_camera(*cam_of(s, i)) for i in srcs], *s.depth_range, seed=7, view_id=r,
                          iterations=4)
        want = (torch.zeros(H, W, device="cuda"), torch.zeros(H, W, 3, device="cuda"), torch.zeros(H, W, device="cuda"))
        ctx.solve([job], params, [hp.maps_of(*want)])
    want = [t.cpu().numpy() for t in want]

    # hp_solve_static on the same images (FP32 values u8/255, as the engine converts them).
    ref = torch.from_numpy(s.views[r].image_f32).cuda().contiguous()
    src_imgs = [torch.from_numpy(s.views[i].image_f32).cuda().contiguous() for i in srcs]
    texs = [_texture(rt, t) for t in src_imgs]
    try:
        outs = []
        for call in range(2):
            got = (torch.full((H, W), -1.0, device="cuda"), torch.full((H, W, 3), -1.0, device="cuda"),
                   torch.full((H, W), -1.0, device="cuda"))
            torch.cuda.synchronize()
            free_before = rt.cudaMemGetInfo()[1]
            hp.solve_static(job, params, ref, [int(t) for t in texs], hp.maps_of(*got))
            free_after = rt.cudaMemGetInfo()[1]
            if call == 1:
                assert free_after == free_before, "hp_solve_static allocated device memory"
            outs.append([t.cpu().numpy() for t in got])
        for got in outs:
            for a, b in zip(got, want):
                assert np.array_equal(a, b)
    finally:
        for t in texs:
            rt.cudaDestroyTextureObject(t)

    # Views above the fixed scratch size are refused before any device work.
    big = hp.make_job(0, [0], hp.make_camera(*cam_of(s, r)), [hp.make_camera(*cam_of(s, srcs[0]))], 1.0, 4.0)
    tex = (C.c_ulonglong * 1)(0)
    st = hp.lib.hp_solve_static(0, None, C.byref(big), ref.data_ptr(), 4096, 4096, 4096, tex, C.byref(params),
                                C.byref(hp.maps_of(*[torch.zeros(1, device="cuda")] * 3)))
    assert st == 6  # HP_ERR_UNSUPPORTED
    assert hp.STATIC_MAX_PIXELS == 1280 * 1024

    # A depth range hp_solve refuses is refused here too: a non-finite far plane.
    inf_job = hp.make_job(0, [0], hp.make_camera(*cam_of(s, r)), [hp.make_camera(*cam_of(s, srcs[0]))], 1.0,
                          float("inf"))
    st = hp.lib.hp_solve_static(0, None, C.byref(inf_job), ref.data_ptr(), W, W, H, tex, C.byref(params),
                                C.byref(hp.maps_of(*[torch.zeros(1, device="cuda")] * 3)))
    assert st == 1  # HP_ERR_INVALID_ARG
    # The Python wrapper checks the texture count against the job's sources.
    with pytest.raises(ValueError):
        hp.solve_static(job, params, ref, [0], hp.maps_of(*[torch.zeros(1, device="cuda")] * 3))
