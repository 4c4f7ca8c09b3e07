"""Generate golden vectors from the reference's own kernels (run on a GPU box).

Runs the reference's compute_ncc_cost_kernel / computePixelCost and
geometric_consistency_filter_kernel (oracle/_ref/libpmref.so, compiled
unmodified from src/dense_recon/patchmatch_mvs.cu) on small seeded inputs and
writes inputs and outputs to tests/golden/reference_kernels.npz.  The CPU
tests pin the oracle against these vectors, so the oracle is anchored to the
reference's actual outputs, not only to a restatement.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import importlib
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "oracle", "ref_harness")]

import pm_oracle as po  # noqa: E402
import pmref  # noqa: E402

scene = importlib.import_module("hemiphoto3d-private_b200.scene")


def main(out=os.path.join(HERE, "reference_kernels.npz")):
    s = scene.plane_sphere(seed=21, w=128, h=96)
    r = 2
    srcs = s.sources[r]
    cam = lambda i: (s.views[i].cam.K, s.views[i].cam.R, s.views[i].cam.t)
    kinv, ab = pmref.setup_views(cam(r), [cam(i) for i in srcs])
    ov = po.View(s.views[r].image_f32, [s.views[i].image_f32 for i in srcs], radius=5, ref_cam=cam(r),
                 src_cams=[cam(i) for i in srcs])
    d_rand, n_rand = ov.init(1.0, 4.0, 1234, r)
    d_gt = s.views[r].depth_gt.astype(np.float32)
    n_gt = np.ascontiguousarray(s.views[r].normal_gt, np.float32)
    ref_img = s.views[r].image_f32
    src_imgs = [s.views[i].image_f32 for i in srcs]
    res = {}
    for tag, (d, n) in {"rand": (d_rand, n_rand), "gt": (d_gt, n_gt)}.items():
        res[f"cost_r5_{tag}"] = pmref.ncc_cost(ref_img, src_imgs, kinv, ab, d, n, 5, "ncc")
        res[f"cost_r3_{tag}"] = pmref.ncc_cost(ref_img, src_imgs, kinv, ab, d, n, 3, "ncc")
        res[f"cost_r7_{tag}"] = pmref.ncc_cost(ref_img, src_imgs, kinv, ab, d, n, 7, "pixel")
    # Geometric filter on perturbed ground-truth maps of views 1..3 (view 2 is the reference).
    rng = np.random.default_rng(5)
    maps = {}
    for i in (1, 2, 3):
        d = s.views[i].depth_gt.astype(np.float32) * (1 + rng.normal(0, 0.08, s.views[i].depth_gt.shape)).astype(np.float32)
        maps[i] = (np.ascontiguousarray(d), np.ascontiguousarray(s.views[i].normal_gt, np.float32))
    fd, fc = maps[2][0].copy(), np.full(maps[2][0].shape, 0.75, np.float32)
    pmref.geometric_filter(cam(2), fd, maps[2][1], fc, [cam(1), cam(3)], [maps[1][0], maps[3][0]],
                           [maps[1][1], maps[3][1]], 0.12, float(np.cos(np.pi)), 2)
    cams = np.stack([np.concatenate([np.ravel(c) for c in cam(i)]) for i in range(len(s.views))])
    np.savez_compressed(
        out, ref_id=r, srcs=np.array(srcs), images=np.stack([v.image for v in s.views]), cams=cams, kinv=kinv, ab=ab,
        d_rand=d_rand, n_rand=n_rand, d_gt=d_gt, n_gt=n_gt,
        filter_depths=np.stack([maps[i][0] for i in (1, 2, 3)]), filter_normals=np.stack([maps[i][1] for i in (1, 2, 3)]),
        filter_out_depth=fd, filter_out_conf=fc, **res)
    print(f"wrote {out} ({os.path.getsize(out)} bytes)")


if __name__ == "__main__":
    main(*sys.argv[1:2])
