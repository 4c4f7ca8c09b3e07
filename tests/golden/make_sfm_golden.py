"""Generates tests/golden/sfm_select.npz: the reference's own selectSourceViews
(src/dense_recon/patchmatch_mvs.cu:74-157, run through oracle/ref_harness, which compiles the reference
source unmodified) on a synthetic sparse reconstruction of a 10-view scene (one camera unregistered),
for num_sources 4 and 8.  Needs the harness built (oracle/_ref/libpmref.so); no GPU.

    python tests/golden/make_sfm_golden.py
"""
import importlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle", "ref_harness")]


def main():
    import pmref
    sc = importlib.import_module("hemiphoto3d-private_b200.scene")
    s = sc.multi_object(seed=5, w=240, h=160, n_views=10, n_refs=0, f=190.0)
    cams = [(v.cam.K, v.cam.R, v.cam.t) for v in s.views]
    pos, tracks = sc.sparse_points(s, n=1500, seed=2)
    reg = [1] * len(cams)
    reg[6] = 0
    out = {"cams_krt": np.array([np.concatenate([np.ravel(K), np.ravel(R), np.ravel(t)]) for K, R, t in cams]),
           "registered": np.array(reg, np.int32), "positions": pos,
           "track_offset": np.concatenate([[0], np.cumsum([len(t) for t in tracks])]).astype(np.int32),
           "track_images": np.array([c for t in tracks for c in t], np.int32)}
    for ns in (4, 8):
        sel = pmref.select_sources(cams, reg, pos, tracks, ns)
        n = len(sel)
        src = np.full((n, 8), -1, np.int32)
        score = np.zeros((n, 8), np.float32)
        ang = np.zeros((n, 8), np.float32)
        for i, v in enumerate(sel):
            k = len(v["sources"])
            src[i, :k], score[i, :k], ang[i, :k] = v["sources"], v["scores"], v["baseline_deg"]
        out[f"ns{ns}_ref"] = np.array([v["ref"] for v in sel], np.int32)
        out[f"ns{ns}_count"] = np.array([len(v["sources"]) for v in sel], np.int32)
        out[f"ns{ns}_sources"], out[f"ns{ns}_scores"], out[f"ns{ns}_angles"] = src, score, ang
        out[f"ns{ns}_depth_min"] = np.array([v["depth_min"] for v in sel], np.float32)
        out[f"ns{ns}_depth_max"] = np.array([v["depth_max"] for v in sel], np.float32)
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "sfm_select.npz")
    np.savez_compressed(path, **out)
    print(path, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
