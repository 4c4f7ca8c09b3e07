"""ctypes binding of the CPU oracle (oracle/libpmoracle.so) - TEST INFRASTRUCTURE.

The oracle restates the reference's PatchMatch path on the CPU
(src/dense_recon/patchmatch_mvs.cu:164-216, :222-343, :519-655, :668-781); see
pm_oracle.h.  Only tests/, the smoke check and the bench's CPU-baseline leg use
it, always as the checker or the timed CPU baseline, never as the engine.
"""
from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from typing import Sequence

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libpmoracle.so")
REF_LIB_PATH = os.path.join(HERE, "_ref", "libpmref.so")
MAX_SOURCES = 8


class OrcCamera(C.Structure):
    _fields_ = [("K", C.c_double * 9), ("R", C.c_double * 9), ("t", C.c_double * 3)]


class OrcView(C.Structure):
    _fields_ = [
        ("W", C.c_int), ("H", C.c_int), ("S", C.c_int),
        ("ref", C.POINTER(C.c_float)), ("src", C.POINTER(C.c_float) * MAX_SOURCES),
        ("kinv", C.c_float * 9), ("ab", (C.c_float * 12) * MAX_SOURCES),
        ("kinv64", C.c_double * 9), ("ab64", (C.c_double * 12) * MAX_SOURCES),
        ("radius", C.c_int), ("stride", C.c_int), ("top_k", C.c_int),
    ]


class OrcFuseView(C.Structure):
    _fields_ = [("cam", OrcCamera), ("depth", C.POINTER(C.c_float)), ("normal", C.POINTER(C.c_float)),
                ("confidence", C.POINTER(C.c_float)), ("gray", C.POINTER(C.c_float)),
                ("neighbors", C.POINTER(C.c_int)), ("num_neighbors", C.c_int), ("W", C.c_int), ("H", C.c_int)]


class OrcRefine(C.Structure):
    _fields_ = [("refine_steps", C.c_int), ("iter_decay", C.c_float), ("step_decay", C.c_float)]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        P = C.POINTER
        fp, dp = P(C.c_float), P(C.c_double)
        sig = {
            "orc_set_tex_rounding": (None, [C.c_int]),
            "orc_set_soft_sources": (None, [C.c_uint]),
            "orc_get_soft_sources": (C.c_uint, []),
            "orc_philox4x32_10": (None, [P(C.c_uint32), P(C.c_uint32), P(C.c_uint32)]),
            "orc_u01": (C.c_float, [C.c_uint32]),
            "orc_setup_f64": (C.c_int, [P(OrcCamera), P(OrcCamera), C.c_int, dp, dp]),
            "orc_view_set_cameras": (C.c_int, [P(OrcView), P(OrcCamera), P(OrcCamera)]),
            "orc_tex_linear": (C.c_float, [fp, C.c_int, C.c_int, C.c_float, C.c_float]),
            "orc_pixel_cost_f32": (C.c_float, [P(OrcView), C.c_int, C.c_int, C.c_float, C.c_float, C.c_float,
                                               C.c_float]),
            "orc_pixel_cost_f64": (C.c_double, [P(OrcView), C.c_int, C.c_int, C.c_double, C.c_double, C.c_double,
                                                C.c_double, C.c_int]),
            "orc_cost_map_f32": (None, [P(OrcView), fp, fp, fp]),
            "orc_cost_map_f64": (None, [P(OrcView), fp, fp, C.c_int, dp]),
            "orc_cost_rows_f64": (None, [P(OrcView), fp, fp, C.c_int, dp, C.c_int, C.c_int]),
            "orc_cost_rows_f32": (None, [P(OrcView), fp, fp, fp, C.c_int, C.c_int]),
            "orc_propagate_rows": (None, [P(OrcView), fp, fp, fp, C.c_float, C.c_float, C.c_int, C.c_int, C.c_uint64,
                                          C.c_uint32, P(OrcRefine), C.c_int, C.c_int]),
            "orc_init": (None, [P(OrcView), C.c_float, C.c_float, C.c_uint64, C.c_uint32, fp, fp]),
            "orc_propagate_pass": (None, [P(OrcView), fp, fp, fp, C.c_float, C.c_float, C.c_int, C.c_int, C.c_uint64,
                                          C.c_uint32, P(OrcRefine)]),
            "orc_solve_view": (None, [P(OrcView), C.c_float, C.c_float, C.c_uint64, C.c_uint32, C.c_int,
                                      P(OrcRefine), fp, fp, fp]),
            "orc_geometric_filter": (None, [P(OrcCamera), C.c_int, C.c_int, fp, fp, fp, C.c_int, P(OrcCamera),
                                            P(fp), P(fp), C.c_float, C.c_float, C.c_int]),
            "orc_fuse": (C.c_longlong, [P(OrcFuseView), C.c_int, C.c_int, C.c_float, C.c_float, C.c_float, C.c_float,
                                        fp, fp, fp, C.c_longlong]),
            "orc_num_threads": (C.c_int, []),
            "orc_set_num_threads": (None, [C.c_int]),
        }
        for k, (r, a) in sig.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _lib = L
    return _lib


def _fp(a: np.ndarray):
    assert a.dtype == np.float32 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(C.POINTER(C.c_float))


def camera(K, R, t) -> OrcCamera:
    c = OrcCamera()
    c.K[:] = list(np.asarray(K, np.float64).ravel())
    c.R[:] = list(np.asarray(R, np.float64).ravel())
    c.t[:] = list(np.asarray(t, np.float64).ravel())
    return c


class View:
    """A reference view with its sources (FP32 images in [0, 1]); keeps the arrays alive."""

    def __init__(self, ref: np.ndarray, srcs: Sequence[np.ndarray], radius: int = 5, stride: int = 1,
                 top_k: int = 3, ref_cam=None, src_cams=None, coeffs=None):
        self.ref = np.ascontiguousarray(ref, np.float32)
        self.srcs = [np.ascontiguousarray(s, np.float32) for s in srcs]
        v = OrcView()
        v.H, v.W = self.ref.shape
        v.S = len(self.srcs)
        v.ref = _fp(self.ref)
        for i, s in enumerate(self.srcs):
            v.src[i] = _fp(s)
        v.radius, v.stride, v.top_k = radius, stride, top_k
        if ref_cam is not None:
            rc = camera(*ref_cam)
            scs = (OrcCamera * len(src_cams))(*[camera(*c) for c in src_cams])
            if lib().orc_view_set_cameras(C.byref(v), C.byref(rc), scs) != 0:
                raise ValueError("singular intrinsics")
        if coeffs is not None:  # float32 (kinv, ab) replace the FP32 copies; FP64 copies stay
            kinv, ab = coeffs
            v.kinv[:] = list(np.asarray(kinv, np.float32).ravel())
            ab = np.asarray(ab, np.float32).reshape(-1, 12)
            for s in range(ab.shape[0]):
                v.ab[s][:] = list(ab[s])
        self.c = v

    @property
    def kinv(self):
        return np.array(self.c.kinv[:], np.float32)

    @property
    def ab(self):
        return np.array([self.c.ab[s][:] for s in range(self.c.S)], np.float32)

    def cost_map_f32(self, depth, normal):
        cost = np.empty(depth.shape, np.float32)
        lib().orc_cost_map_f32(C.byref(self.c), _fp(depth), _fp(normal), _fp(cost))
        return cost

    def cost_map_f64(self, depth, normal, quantized=False):
        cost = np.empty(depth.shape, np.float64)
        lib().orc_cost_map_f64(C.byref(self.c), _fp(depth), _fp(normal), int(quantized),
                               cost.ctypes.data_as(C.POINTER(C.c_double)))
        return cost

    def cost_rows_f64(self, depth, normal, y0, y1, quantized=False):
        """Rows [y0, y1) of the FP64 cost map, as a (y1 - y0, W) array."""
        cost = np.zeros(depth.shape, np.float64)
        lib().orc_cost_rows_f64(C.byref(self.c), _fp(depth), _fp(normal), int(quantized),
                                cost.ctypes.data_as(C.POINTER(C.c_double)), y0, y1)
        return cost[y0:y1]

    def cost_rows_f32(self, depth, normal, cost, y0, y1):
        lib().orc_cost_rows_f32(C.byref(self.c), _fp(depth), _fp(normal), _fp(cost), y0, y1)

    def propagate_rows(self, depth, normal, cost, dmin, dmax, iteration, color, seed, view_id, y0, y1,
                       refine_steps=2, iter_decay=0.6, step_decay=0.5):
        rf = OrcRefine(refine_steps, iter_decay, step_decay)
        lib().orc_propagate_rows(C.byref(self.c), _fp(depth), _fp(normal), _fp(cost), dmin, dmax, iteration, color,
                                 seed, view_id, C.byref(rf), y0, y1)

    def pixel_cost_f32(self, x, y, d, n):
        return lib().orc_pixel_cost_f32(C.byref(self.c), x, y, d, *map(float, n))

    def init(self, dmin, dmax, seed, view_id):
        h, w = self.ref.shape
        depth = np.empty((h, w), np.float32)
        normal = np.empty((h, w, 3), np.float32)
        lib().orc_init(C.byref(self.c), dmin, dmax, seed, view_id, _fp(depth), _fp(normal))
        return depth, normal

    def propagate_pass(self, depth, normal, cost, dmin, dmax, iteration, color, seed, view_id,
                       refine_steps=2, iter_decay=0.6, step_decay=0.5):
        rf = OrcRefine(refine_steps, iter_decay, step_decay)
        lib().orc_propagate_pass(C.byref(self.c), _fp(depth), _fp(normal), _fp(cost), dmin, dmax, iteration, color,
                                 seed, view_id, C.byref(rf))

    def solve(self, dmin, dmax, seed, view_id, iterations, refine_steps=2, iter_decay=0.6, step_decay=0.5):
        h, w = self.ref.shape
        depth = np.empty((h, w), np.float32)
        normal = np.empty((h, w, 3), np.float32)
        cost = np.empty((h, w), np.float32)
        rf = OrcRefine(refine_steps, iter_decay, step_decay)
        lib().orc_solve_view(C.byref(self.c), dmin, dmax, seed, view_id, iterations, C.byref(rf), _fp(depth),
                             _fp(normal), _fp(cost))
        return depth, normal, cost


def philox(ctr, key):
    c = (C.c_uint32 * 4)(*ctr)
    k = (C.c_uint32 * 2)(*key)
    o = (C.c_uint32 * 4)()
    lib().orc_philox4x32_10(c, k, o)
    return list(o)


def geometric_filter(ref_cam, depth, normal, conf, src_cams, src_depths, src_normals, depth_tol=0.12,
                     normal_tol_cos=-1.0, min_consistent=2):
    """In place on depth / conf (float32 arrays)."""
    h, w = depth.shape
    n = len(src_cams)
    cams = (OrcCamera * max(1, n))(*[camera(*c) for c in src_cams])
    FP = C.POINTER(C.c_float)
    dps = (FP * max(1, n))(*[_fp(a) for a in src_depths])
    nps = (FP * max(1, n))(*[_fp(a) for a in src_normals])
    lib().orc_geometric_filter(C.byref(camera(*ref_cam)), w, h, _fp(depth), _fp(normal), _fp(conf), n, cams, dps,
                               nps, depth_tol, normal_tol_cos, min_consistent)


def fuse(maps, cams, neighbors=None, min_views=2, min_confidence=0.0, max_depth_rel=0.01, max_reproj_px=2.0,
         min_normal_cos=0.98480775):
    """Depth-map fusion (orc_fuse).  maps: per view (depth (H, W), normal (H, W, 3), confidence or None,
    gray or None), float32; cams: per view (K, R, t); neighbors: per view a list of view indices, or None for
    every other view.  Returns (positions, normals, colors), each (N, 3) float32."""
    n = len(maps)
    keep = []
    views = (OrcFuseView * n)()
    for i, (d, nr, cf, g) in enumerate(maps):
        arrs = [np.ascontiguousarray(a, np.float32) if a is not None else None for a in (d, nr, cf, g)]
        keep.append(arrs)
        v = views[i]
        v.cam = camera(*cams[i])
        v.depth, v.normal = _fp(arrs[0]), _fp(arrs[1])
        v.confidence = _fp(arrs[2]) if arrs[2] is not None else None
        v.gray = _fp(arrs[3]) if arrs[3] is not None else None
        v.H, v.W = arrs[0].shape
        if neighbors is not None and neighbors[i] is not None:
            nb = np.ascontiguousarray(neighbors[i], np.int32)
            keep.append(nb)
            v.neighbors = nb.ctypes.data_as(C.POINTER(C.c_int))
            v.num_neighbors = len(nb)
    args = (views, n, min_views, min_confidence, max_depth_rel, max_reproj_px, min_normal_cos)
    total = lib().orc_fuse(*args, None, None, None, 0)
    pos = np.zeros((total, 3), np.float32)
    nrm = np.zeros((total, 3), np.float32)
    col = np.zeros((total, 3), np.float32)
    if total:
        lib().orc_fuse(*args, _fp(pos), _fp(nrm), _fp(col), total)
    return pos, nrm, col


def set_tex_rounding(mode: int):
    lib().orc_set_tex_rounding(mode)


def set_soft_sources(mask: int):
    """Sources (bit per source) whose quantized-weight FP64 cost uses the FP16 path's
    software-sampler model (separable 8-bit weights, round-to-nearest coordinates)."""
    lib().orc_set_soft_sources(mask & 0xFF)


def soft_sources() -> int:
    return int(lib().orc_get_soft_sources())


def num_threads() -> int:
    return lib().orc_num_threads()


def set_num_threads(n: int):
    lib().orc_set_num_threads(n)


# ---------------------------------------------------------------------------------------------
# SfM front of the stage (patchmatch_mvs.cu:40-157, :1111-1177), restated in FP64 numpy scalars.
# Small cases only (pure Python loops).  Cameras are (K, R, t) tuples; tracks hold camera indices.
# ---------------------------------------------------------------------------------------------

_LIBM = None


def _sinf(x):
    """The C library's single-precision sine (the reference calls std::sin on a float)."""
    global _LIBM
    if _LIBM is None:
        _LIBM = C.CDLL("libm.so.6")
        _LIBM.sinf.restype, _LIBM.sinf.argtypes = C.c_float, [C.c_float]
    return np.float32(_LIBM.sinf(float(x)))


def _cam_centre(R, t):
    """-R^T t, summed left to right (CameraPose::cam_center, include/types.h:71-73)."""
    return np.array([(-R[0, i] * t[0] + -R[1, i] * t[1]) + -R[2, i] * t[2] for i in range(3)])


def _mv(M, v):
    return np.array([(M[i, 0] * v[0] + M[i, 1] * v[1]) + M[i, 2] * v[2] for i in range(3)])


def _unit(v):
    n = math.sqrt((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2])
    return v / n if n > 0 else v


def sfm_select_sources(cams, registered, positions, tracks, num_sources):
    """selectSourceViews (patchmatch_mvs.cu:74-157): per registered camera, sources scored by shared points x
    sin(clamped baseline angle at the centroid), best first (ties: lower index), and the 5/95-percentile depth
    range x0.5 / x1.5 (centroid depth x0.3 / x3 with fewer than two points)."""
    pos = [np.asarray(p, np.float64) for p in positions]
    cen = np.zeros(3)
    for p in pos:
        cen = cen + p
    if pos:
        cen = cen / float(len(pos))
    sets = [set(t) for t in tracks]
    out = []
    for ref, (K, R, t) in enumerate(cams):
        if not registered[ref]:
            continue
        R, t = np.asarray(R, np.float64), np.asarray(t, np.float64)
        cand = []
        for src, (Ks, Rs, ts) in enumerate(cams):
            if src == ref or not registered[src]:
                continue
            vi = _unit(cen - _cam_centre(R, t))
            vj = _unit(cen - _cam_centre(np.asarray(Rs, np.float64), np.asarray(ts, np.float64)))
            c = min(1.0, max(-1.0, (vi[0] * vj[0] + vi[1] * vj[1]) + vi[2] * vj[2]))
            ang = np.float32(math.acos(c) * 180.0 / math.pi)
            if ang < np.float32(5.0) or ang > np.float32(90.0):
                continue
            cl = min(max(ang, np.float32(5.0)), np.float32(30.0))
            b = _sinf(np.float32(cl * np.float32(math.pi) / np.float32(180.0)))
            shared = sum(1 for s in sets if ref in s and src in s)
            if shared == 0:
                continue
            cand.append((-(np.float32(shared) * b), src, np.float32(shared) * b, ang))
        cand.sort(key=lambda c: (c[0], c[1]))
        cand = cand[:num_sources]
        depths = []
        for p, s in zip(pos, sets):
            if ref in s:
                z = _mv(R, p)[2] + t[2]
                if z > 0:
                    depths.append(np.float32(z))
        if len(depths) >= 2:
            depths.sort()
            i5 = int(len(depths) * 0.05)
            i95 = min(int(len(depths) * 0.95), len(depths) - 1)
            dmin, dmax = depths[i5] * np.float32(0.5), depths[i95] * np.float32(1.5)
        else:
            d = np.float32(_mv(R, cen)[2] + t[2])
            dmin, dmax = d * np.float32(0.3), d * np.float32(3.0)
        out.append({"ref": ref, "sources": [c[1] for c in cand], "scores": [float(c[2]) for c in cand],
                    "baseline_deg": [float(c[3]) for c in cand], "depth_min": float(dmin), "depth_max": float(dmax)})
    return out


def sfm_project_seeds(cam, ref, depth_min, depth_max, positions, tracks):
    """The seeds of camera `ref` (patchmatch_mvs.cu:1122-1160): (x, y, depth, nx, ny, nz) per point it sees
    with positive depth inside [depth_min, depth_max], in point order."""
    K, R, t = (np.asarray(a, np.float64) for a in cam)
    c = _cam_centre(R, t)
    seeds = []
    for p, tr in zip(positions, tracks):
        if ref not in tr:
            continue
        p = np.asarray(p, np.float64)
        pc = _mv(R, p) + t
        if pc[2] <= 0:
            continue
        px = _mv(K, pc)
        x, y = _round_half_away(px[0] / px[2]), _round_half_away(px[1] / px[2])
        d = np.float32(pc[2])
        if d < np.float32(depth_min) or d > np.float32(depth_max):
            continue
        n = _mv(R, _unit(c - p))
        seeds.append((int(x), int(y), float(d), float(np.float32(n[0])), float(np.float32(n[1])),
                      float(np.float32(n[2]))))
    return seeds


def _round_half_away(v):
    """std::round: nearest integer, halves away from zero (v - floor(v) is exact here)."""
    a = abs(v)
    r = math.floor(a)
    r = r + 1 if a - r >= 0.5 else r
    return r if v >= 0 else -r


def paint_seeds(depth, normal, seeds, radius):
    """Overwrite the (2r+1)^2 square around each seed's pixel with its depth and normal, in list order."""
    H, W = depth.shape
    for x, y, d, nx, ny, nz in seeds:
        x0, x1 = max(0, x - radius), min(W - 1, x + radius)
        y0, y1 = max(0, y - radius), min(H - 1, y + radius)
        if x0 > x1 or y0 > y1:
            continue
        depth[y0:y1 + 1, x0:x1 + 1] = d
        normal[y0:y1 + 1, x0:x1 + 1] = (nx, ny, nz)
