"""ctypes binding of the CPU oracle (oracle/libpmoracle.so) - TEST INFRASTRUCTURE.

The oracle restates the reference's PatchMatch path on the CPU
(src/dense_recon/patchmatch_mvs.cu:164-216, :222-343, :519-655, :668-781); see
pm_oracle.h.  Only tests/, the smoke check and the bench's CPU-baseline leg use
it, always as the checker or the timed CPU baseline, never as the engine.
"""
from __future__ import annotations

import ctypes as C
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
