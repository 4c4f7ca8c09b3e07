"""ctypes binding of the GPU reference harness (oracle/_ref/libpmref.so) - TEST INFRASTRUCTURE.

libpmref.so is the reference's own src/dense_recon/patchmatch_mvs.cu compiled
unmodified (see Makefile and ref_harness.cu).  Tests call it as the parity
anchor; it is only built where the reference tree exists, so callers skip when
:func:`available` is False.  All arrays are host float32.
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "..", "_ref", "libpmref.so")

_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        L = C.CDLL(LIB_PATH)
        fp, dp, ip = C.c_void_p, C.c_void_p, C.c_int
        L.pmref_setup_views.argtypes = [dp, dp, ip, fp, fp]
        L.pmref_ncc_cost.argtypes = [fp, C.c_void_p, ip, ip, ip, fp, fp, fp, fp, ip, fp]
        L.pmref_pixel_cost.argtypes = [fp, C.c_void_p, ip, ip, ip, fp, fp, fp, fp, ip, fp]
        L.pmref_init.argtypes = [fp, ip, ip, C.c_float, C.c_float, C.c_uint64, fp, fp]
        L.pmref_propagate.argtypes = [fp, C.c_void_p, ip, ip, ip, fp, fp, fp, fp, fp, C.c_float, C.c_float, ip, ip,
                                      ip, C.c_uint64]
        L.pmref_solve_view.argtypes = [fp, C.c_void_p, ip, ip, ip, fp, fp, C.c_float, C.c_float, ip, ip, ip, fp, fp,
                                       fp, C.POINTER(C.c_float)]
        L.pmref_geometric_filter.argtypes = [fp, fp, fp, dp, fp, fp, dp, ip, ip, ip, C.c_float, C.c_float, ip]
        L.pmref_select_sources.argtypes = [dp, fp, ip, dp, fp, fp, ip, ip] + [fp] * 8
        L.pmref_run_stage.argtypes = [C.c_void_p, ip, ip, dp, fp, ip, dp, fp, fp, ip, ip, fp, fp, fp, fp]
        for f in ("pmref_setup_views", "pmref_ncc_cost", "pmref_pixel_cost", "pmref_init", "pmref_propagate",
                  "pmref_solve_view", "pmref_geometric_filter", "pmref_select_sources", "pmref_run_stage"):
            getattr(L, f).restype = C.c_int
        _lib = L
    return _lib


def _p(a):
    return a.ctypes.data


def _krt(cam):
    K, R, t = cam
    return np.concatenate([np.asarray(K, np.float64).ravel(), np.asarray(R, np.float64).ravel(),
                           np.asarray(t, np.float64).ravel()])


def setup_views(ref_cam, src_cams):
    """(kinv[9], ab[S,12]) float32 exactly as the reference computes them."""
    r = _krt(ref_cam)
    s = np.concatenate([_krt(c) for c in src_cams])
    kinv = np.empty(9, np.float32)
    ab = np.empty((len(src_cams), 12), np.float32)
    assert lib().pmref_setup_views(_p(r), _p(s), len(src_cams), _p(kinv), _p(ab)) == 0
    return kinv, ab


class _Images:
    def __init__(self, ref, srcs):
        self.ref = np.ascontiguousarray(ref, np.float32)
        self.srcs = [np.ascontiguousarray(s, np.float32) for s in srcs]
        self.ptrs = (C.c_void_p * len(self.srcs))(*[s.ctypes.data for s in self.srcs])


def ncc_cost(ref, srcs, kinv, ab, depth, normal, radius, kernel="ncc"):
    """compute_ncc_cost_kernel ('ncc', radius <= 5) or computePixelCost ('pixel') on fixed maps."""
    im = _Images(ref, srcs)
    h, w = im.ref.shape
    cost = np.empty((h, w), np.float32)
    fn = lib().pmref_ncc_cost if kernel == "ncc" else lib().pmref_pixel_cost
    kinv = np.ascontiguousarray(kinv, np.float32)
    ab = np.ascontiguousarray(ab, np.float32)
    depth = np.ascontiguousarray(depth, np.float32)
    normal = np.ascontiguousarray(normal, np.float32)
    st = fn(_p(im.ref), C.cast(im.ptrs, C.c_void_p), len(im.srcs), w, h, _p(kinv), _p(ab), _p(depth), _p(normal),
            radius, _p(cost))
    assert st == 0, st
    return cost


def solve_view(ref, srcs, kinv, ab, dmin, dmax, radius, iterations, ref_id):
    """The reference's per-view solve; returns (depth, normal, cost, gpu_ms)."""
    im = _Images(ref, srcs)
    h, w = im.ref.shape
    depth = np.empty((h, w), np.float32)
    normal = np.empty((h, w, 3), np.float32)
    cost = np.empty((h, w), np.float32)
    ms = C.c_float()
    kinv = np.ascontiguousarray(kinv, np.float32)
    ab = np.ascontiguousarray(ab, np.float32)
    st = lib().pmref_solve_view(_p(im.ref), C.cast(im.ptrs, C.c_void_p), len(im.srcs), w, h, _p(kinv), _p(ab), dmin,
                                dmax, radius, iterations, ref_id, _p(depth), _p(normal), _p(cost), C.byref(ms))
    assert st == 0, st
    return depth, normal, cost, ms.value


def geometric_filter(ref_cam, depth, normal, conf, src_cams, src_depths, src_normals, depth_tol=0.12,
                     normal_tol_cos=-1.0, min_consistent=2):
    """In place on depth / conf."""
    S = len(src_cams)
    h, w = depth.shape
    r = _krt(ref_cam)
    s = np.concatenate([_krt(c) for c in src_cams])
    sd = np.ascontiguousarray(np.stack(src_depths), np.float32)
    sn = np.ascontiguousarray(np.stack(src_normals), np.float32)
    assert lib().pmref_geometric_filter(_p(depth), _p(np.ascontiguousarray(normal, np.float32)), _p(conf), _p(r),
                                        _p(sd), _p(sn), _p(s), S, w, h, depth_tol, normal_tol_cos,
                                        min_consistent) == 0


def _sfm_arrays(cams, registered, positions, tracks):
    krt = np.ascontiguousarray(np.concatenate([_krt(c) for c in cams]))
    reg = np.ascontiguousarray(np.asarray(registered, np.int32))
    pos = np.ascontiguousarray(np.asarray(positions, np.float64).reshape(-1, 3))
    toff = np.zeros(len(tracks) + 1, np.int32)
    toff[1:] = np.cumsum([len(t) for t in tracks]) if len(tracks) else []
    timg = np.ascontiguousarray(np.asarray([c for t in tracks for c in t] or [0], np.int32))
    return krt, reg, pos, toff, timg


def select_sources(cams, registered, positions, tracks, num_sources):
    """The reference's selectSourceViews (host code; no GPU needed).  cams: (K, R, t) per camera."""
    krt, reg, pos, toff, timg = _sfm_arrays(cams, registered, positions, tracks)
    n = len(cams)
    ref, cnt = np.zeros(n, np.int32), np.zeros(n, np.int32)
    src = np.zeros(8 * n, np.int32)
    score, ang = np.zeros(8 * n, np.float32), np.zeros(8 * n, np.float32)
    dmin, dmax = np.zeros(n, np.float32), np.zeros(n, np.float32)
    n_out = np.zeros(1, np.int32)
    rc = lib().pmref_select_sources(_p(krt), _p(reg), n, _p(pos), _p(toff), _p(timg), len(tracks), num_sources,
                                    _p(ref), _p(cnt), _p(src), _p(score), _p(ang), _p(dmin), _p(dmax), _p(n_out))
    assert rc == 0
    out = []
    for i in range(int(n_out[0])):
        k = int(cnt[i])
        out.append({"ref": int(ref[i]), "sources": src[8 * i:8 * i + k].tolist(), "scores": score[8 * i:8 * i + k].tolist(),
                    "baseline_deg": ang[8 * i:8 * i + k].tolist(), "depth_min": float(dmin[i]),
                    "depth_max": float(dmax[i])})
    return out


def run_stage(grays: Sequence[np.ndarray], cams, positions, tracks, patch_size=11):
    """The reference's runPatchMatchMVS with 0 iterations (init + SfM seeding): {image id: (depth, normal)}."""
    H, W = grays[0].shape
    g = [np.ascontiguousarray(x, np.float32) for x in grays]
    ptrs = (C.c_void_p * len(g))(*[x.ctypes.data for x in g])
    krt, reg, pos, toff, timg = _sfm_arrays(cams, [1] * len(cams), positions, tracks)
    n = len(cams)
    ids = np.zeros(n, np.int32)
    depth = np.zeros((n, H, W), np.float32)
    normal = np.zeros((n, H, W, 3), np.float32)
    n_out = np.zeros(1, np.int32)
    rc = lib().pmref_run_stage(ptrs, W, H, _p(krt), _p(reg), n, _p(pos), _p(toff), _p(timg), len(tracks), patch_size,
                               _p(ids), _p(depth), _p(normal), _p(n_out))
    assert rc == 0
    return {int(ids[i]): (depth[i], normal[i]) for i in range(int(n_out[0]))}


# ------------------------------------------------------------------------------------------------
# The engine's C++ stage adapter (include/hpmvs_stage.hpp) run inside the reference's translation
# unit: oracle/_ref/libpmstage.so (stage_harness.cu).
STAGE_LIB_PATH = os.path.join(HERE, "..", "_ref", "libpmstage.so")
_stage = None


def stage_available() -> bool:
    return os.path.exists(STAGE_LIB_PATH)


def stage_run(grays: Sequence[np.ndarray], cams, positions, tracks, patch_size=11, iterations=3, output_dir=None):
    """hpmvs_stage::runPatchMatchMVS: (status, {image id: (depth, normal, confidence)})."""
    global _stage
    if _stage is None:
        L = C.CDLL(STAGE_LIB_PATH)
        L.pmstage_run.restype = C.c_int
        _stage = L
    H, W = grays[0].shape
    g = [np.ascontiguousarray(x, np.float32) for x in grays]
    ptrs = (C.c_void_p * len(g))(*[x.ctypes.data for x in g])
    krt, _, pos, toff, timg = _sfm_arrays(cams, [1] * len(cams), positions, tracks)
    n = len(cams)
    ids = np.zeros(n, np.int32)
    depth = np.zeros((n, H, W), np.float32)
    normal = np.zeros((n, H, W, 3), np.float32)
    conf = np.zeros((n, H, W), np.float32)
    n_out = np.zeros(1, np.int32)
    status = np.zeros(1, np.int32)
    rc = _stage.pmstage_run(ptrs, C.c_int(W), C.c_int(H), C.c_void_p(_p(krt)), C.c_int(n), C.c_void_p(_p(pos)),
                            C.c_void_p(_p(toff)), C.c_void_p(_p(timg)), C.c_int(len(tracks)), C.c_int(patch_size),
                            C.c_int(iterations), output_dir.encode() if output_dir else None, C.c_void_p(_p(ids)),
                            C.c_void_p(_p(depth)), C.c_void_p(_p(normal)), C.c_void_p(_p(conf)),
                            C.c_void_p(_p(n_out)), C.c_void_p(_p(status)))
    assert rc == 0
    return int(status[0]), {int(ids[i]): (depth[i], normal[i], conf[i]) for i in range(int(n_out[0]))}
