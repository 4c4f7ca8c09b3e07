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
