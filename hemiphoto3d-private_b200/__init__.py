"""B200 PatchMatch multi-view stereo: Python binding of the C ABI in include/hpmvs.h.

The engine is the CUDA library ``lib/libhpmvs.so`` built in-tree for sm_100a.
This module only binds it (ctypes) and mirrors the reference's stage call
``runPatchMatchMVS(images, cameras, sfm, config)``
(src/dense_recon/patchmatch_mvs.h:39-44) as :func:`run_patchmatch_mvs`, with the
SfM-derived inputs (source views, depth range) passed explicitly.  There is no
CPU fallback: importing without the built library raises ``ImportError``.
"""
from __future__ import annotations

import ctypes as C
import os
import threading
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# HP_ENGINE_LIB loads another build of the engine (the instrumented
# lib/libhpmvs_count.so of `make count`, for the bench's --count-taps).
LIB_PATH = os.environ.get("HP_ENGINE_LIB") or os.path.join(_HERE, "lib", "libhpmvs.so")

MAX_SOURCES = 8
MAX_RADIUS = 7

OK = 0
STATUS_NAMES = {
    0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of device memory", 4: "not found",
    5: "timed out", 6: "unsupported", 7: "I/O error", 8: "busy", 9: "cancelled",
}
DTYPE_U8, DTYPE_F16, DTYPE_F32 = 0, 1, 2
PRECISION_F32, PRECISION_F16ACC = 0, 1
# runPatchMatchMVS's geometric-filter constants (patchmatch_mvs.cu:1273-1276):
# 12% relative depth, normal check off (cos 180 deg), 2 agreeing sources.
GEOM_DEPTH_TOL = 0.12
GEOM_NORMAL_COS = -1.0
GEOM_MIN_CONSISTENT = 2
MEMORY_HOST, MEMORY_DEVICE = 0, 1


class HpError(RuntimeError):
    """A non-OK hp_status; ``status`` holds the code."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class Camera(C.Structure):
    _fields_ = [("K", C.c_double * 9), ("R", C.c_double * 9), ("t", C.c_double * 3)]


class Params(C.Structure):
    _fields_ = [
        ("radius", C.c_int), ("stride", C.c_int), ("top_k", C.c_int), ("precision", C.c_int),
        ("refine_steps", C.c_int), ("iter_decay", C.c_float), ("step_decay", C.c_float),
        ("tile_w", C.c_int), ("tile_h", C.c_int), ("soft_sources", C.c_int),
        ("filter_min_consistent", C.c_int), ("filter_depth_tol", C.c_float), ("filter_normal_cos", C.c_float),
        ("staging", C.c_int), ("debug_checked_taps", C.c_int),
    ]


class Job(C.Structure):
    _fields_ = [
        ("ref_image", C.c_int), ("num_sources", C.c_int), ("src_images", C.c_int * MAX_SOURCES),
        ("ref_cam", Camera), ("src_cams", Camera * MAX_SOURCES),
        ("depth_min", C.c_float), ("depth_max", C.c_float),
        ("seed", C.c_uint64), ("view_id", C.c_uint32), ("iterations", C.c_int),
        ("use_coeffs", C.c_int), ("kinv", C.c_float * 9), ("ab", (C.c_float * 12) * MAX_SOURCES),
        ("seeds", C.c_void_p), ("num_seeds", C.c_int), ("seed_radius", C.c_int),
    ]


class Maps(C.Structure):
    _fields_ = [("memory", C.c_int), ("depth", C.c_void_p), ("normal", C.c_void_p), ("cost", C.c_void_p),
                ("confidence", C.c_void_p)]


KERNEL_KINDS = ("init", "cost", "propagate", "other", "persistent")


class Profile(C.Structure):
    _fields_ = [("launches", C.c_uint64 * 5), ("device_ms", C.c_double * 5), ("timed", C.c_uint64 * 5)]

    def as_dict(self):
        return {k: {"launches": int(self.launches[i]), "device_ms": float(self.device_ms[i]),
                    "timed": int(self.timed[i])} for i, k in enumerate(KERNEL_KINDS)}


SCHEDULE_AUTO, SCHEDULE_PER_PASS, SCHEDULE_PERSISTENT = 0, 1, 2


class PlanOptions(C.Structure):
    _fields_ = [("schedule", C.c_int), ("ctas_per_sm", C.c_int), ("use_graph", C.c_int),
                ("wait_limit_ms", C.c_int), ("debug_stall_view", C.c_int), ("debug_stall_tile", C.c_int)]


class PlanInfo(C.Structure):
    _fields_ = [("schedule", C.c_int), ("ctas_per_sm", C.c_int), ("grid", C.c_int), ("max_ctas_per_sm", C.c_int),
                ("tickets", C.c_int), ("launches_per_run", C.c_int), ("views", C.c_int), ("use_graph", C.c_int),
                ("state_bytes", C.c_uint64), ("pixel_iterations", C.c_double), ("tuned_ms", C.c_float),
                ("tile_h", C.c_int), ("staging", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class Seed(C.Structure):
    _fields_ = [("x", C.c_int), ("y", C.c_int), ("depth", C.c_float), ("normal", C.c_float * 3)]


class SparsePoints(C.Structure):
    _fields_ = [("num_points", C.c_int), ("position", C.c_void_p), ("track_offset", C.c_void_p),
                ("track_images", C.c_void_p)]


class ViewSelection(C.Structure):
    _fields_ = [("ref_image", C.c_int), ("num_sources", C.c_int), ("sources", C.c_int * MAX_SOURCES),
                ("scores", C.c_float * MAX_SOURCES), ("baseline_deg", C.c_float * MAX_SOURCES),
                ("depth_min", C.c_float), ("depth_max", C.c_float)]


class ServerOptions(C.Structure):
    _fields_ = [("max_active", C.c_int), ("mem_fraction", C.c_float), ("mem_limit", C.c_uint64),
                ("passes_per_step", C.c_int), ("split_launches", C.c_int), ("ctas_per_sm", C.c_int),
                ("inflight_steps", C.c_int), ("wait_limit_ms", C.c_int), ("policy", C.c_int),
                ("step_budget_mpix", C.c_double), ("debug_stall_request", C.c_uint64),
                ("debug_stall_tile", C.c_int), ("debug_fail_step", C.c_int)]


class Completion(C.Structure):
    _fields_ = [("request_id", C.c_uint64), ("status", C.c_int), ("latency_ms", C.c_double),
                ("queue_ms", C.c_double)]


class ServerStats(C.Structure):
    _fields_ = [("submitted", C.c_uint64), ("admitted", C.c_uint64), ("completed", C.c_uint64),
                ("failed", C.c_uint64), ("steps", C.c_uint64), ("launches", C.c_uint64), ("queued", C.c_int),
                ("active", C.c_int), ("peak_active", C.c_int), ("p50_ms", C.c_double), ("p99_ms", C.c_double),
                ("mean_ms", C.c_double), ("max_ms", C.c_double), ("pixel_iterations", C.c_double),
                ("device_ms", C.c_double), ("state_bytes", C.c_uint64), ("peak_state_bytes", C.c_uint64),
                ("budget_bytes", C.c_uint64), ("failed_steps", C.c_uint64), ("pool_reserved_bytes", C.c_uint64),
                ("device_free_bytes", C.c_uint64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class FuseView(C.Structure):
    _fields_ = [("cam", Camera), ("depth", C.c_void_p), ("normal", C.c_void_p), ("confidence", C.c_void_p),
                ("gray", C.c_void_p), ("neighbors", C.POINTER(C.c_int)), ("num_neighbors", C.c_int),
                ("width", C.c_int), ("height", C.c_int)]


class FuseParams(C.Structure):
    _fields_ = [("memory", C.c_int), ("min_views", C.c_int), ("min_confidence", C.c_float),
                ("max_depth_rel", C.c_float), ("max_reproj_px", C.c_float), ("min_normal_cos", C.c_float)]


class PointCloudC(C.Structure):
    _fields_ = [("memory", C.c_int), ("positions", C.c_void_p), ("normals", C.c_void_p), ("colors", C.c_void_p),
                ("capacity", C.c_int64), ("count", C.c_int64)]


def _load() -> C.CDLL:
    if not os.path.exists(LIB_PATH):
        raise ImportError(
            f"{LIB_PATH} is not built; run `make -C {_HERE}` (or __graft_entry__.build()) first")
    lib = C.CDLL(LIB_PATH)
    P = C.POINTER
    sigs = {
        "hp_status_string": (C.c_char_p, [C.c_int]),
        "hp_params_default": (None, [P(Params)]),
        "hp_version": (C.c_char_p, []),
        "hp_ctx_create": (C.c_int, [C.c_int, P(C.c_void_p)]),
        "hp_ctx_destroy": (C.c_int, [C.c_void_p]),
        "hp_ctx_last_error": (C.c_char_p, [C.c_void_p]),
        "hp_ctx_synchronize": (C.c_int, [C.c_void_p]),
        "hp_ctx_mem_info": (C.c_int, [C.c_void_p, P(C.c_size_t), P(C.c_size_t)]),
        "hp_ctx_stream": (C.c_int, [C.c_void_p, P(C.c_void_p)]),
        "hp_ctx_set_profiling": (C.c_int, [C.c_void_p, C.c_int]),
        "hp_ctx_profile": (C.c_int, [C.c_void_p, P(Profile)]),
        "hp_ctx_profile_reset": (C.c_int, [C.c_void_p]),
        "hp_image_upload": (C.c_int, [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int, P(C.c_int)]),
        "hp_image_release": (C.c_int, [C.c_void_p, C.c_int]),
        "hp_ctx_set_image_cache": (C.c_int, [C.c_void_p, C.c_uint64]),
        "hp_image_size": (C.c_int, [C.c_void_p, C.c_int, P(C.c_int), P(C.c_int)]),
        "hp_setup_homographies": (C.c_int, [P(Camera), P(Camera), C.c_int, P(C.c_double), P(C.c_double)]),
        "hp_solve": (C.c_int, [C.c_void_p, P(Job), C.c_int, P(Params), P(Maps)]),
        "hp_init_hypotheses": (C.c_int, [C.c_void_p, P(Job), P(Params), P(Maps)]),
        "hp_ncc_cost": (C.c_int, [C.c_void_p, P(Job), P(Params), P(Maps)]),
        "hp_propagate_pass": (C.c_int, [C.c_void_p, P(Job), P(Params), P(Maps), C.c_int, C.c_int]),
        "hp_geometric_filter": (C.c_int, [C.c_void_p, P(Camera), C.c_int, C.c_int, C.c_void_p, C.c_void_p,
                                          C.c_void_p, C.c_int, P(Camera), P(C.c_void_p), P(C.c_void_p),
                                          C.c_int, C.c_float, C.c_float, C.c_int]),
        "hp_solve_static": (C.c_int, [C.c_int, C.c_void_p, P(Job), C.c_void_p, C.c_int, C.c_int, C.c_int,
                                      P(C.c_ulonglong), P(Params), P(Maps)]),
        "hp_plan_options_default": (None, [P(PlanOptions)]),
        "hp_plan_create": (C.c_int, [C.c_void_p, P(Job), C.c_int, P(Params), P(PlanOptions), P(Maps),
                                     P(C.c_void_p)]),
        "hp_plan_run": (C.c_int, [C.c_void_p]),
        "hp_plan_launch": (C.c_int, [C.c_void_p]),
        "hp_plan_wait": (C.c_int, [C.c_void_p]),
        "hp_plan_tune": (C.c_int, [C.c_void_p, C.c_int, P(PlanInfo)]),
        "hp_plan_get_info": (C.c_int, [C.c_void_p, P(PlanInfo)]),
        "hp_plan_destroy": (C.c_int, [C.c_void_p]),
        "hp_schedule_build": (C.c_int, [C.c_int, P(C.c_int), P(C.c_int), P(C.c_int), C.c_int, P(C.c_int),
                                        P(C.c_int), P(C.c_int), P(C.c_int)]),
        "hp_select_sources": (C.c_int, [P(Camera), P(C.c_int), C.c_int, P(SparsePoints), C.c_int,
                                        P(ViewSelection), P(C.c_int)]),
        "hp_project_seeds": (C.c_int, [P(Camera), C.c_int, C.c_float, C.c_float, P(SparsePoints), P(Seed),
                                       C.c_int, P(C.c_int)]),
        "hp_server_options_default": (None, [P(ServerOptions)]),
        "hp_server_create": (C.c_int, [C.c_void_p, P(Params), P(ServerOptions), P(C.c_void_p)]),
        "hp_submit": (C.c_int, [C.c_void_p, P(Job), P(Maps), P(C.c_uint64)]),
        "hp_poll": (C.c_int, [C.c_void_p, P(Completion), C.c_int, P(C.c_int), C.c_int]),
        "hp_server_drain": (C.c_int, [C.c_void_p, C.c_int]),
        "hp_server_stats_get": (C.c_int, [C.c_void_p, P(ServerStats)]),
        "hp_server_stats_reset": (C.c_int, [C.c_void_p]),
        "hp_server_last_error": (C.c_char_p, [C.c_void_p]),
        "hp_server_first_error": (C.c_char_p, [C.c_void_p]),
        "hp_server_destroy": (C.c_int, [C.c_void_p]),
        "hp_server_simulate": (C.c_int, [C.c_int, P(C.c_int), P(C.c_uint64), P(C.c_int), C.c_int, C.c_uint64,
                                         C.c_int, P(C.c_int), P(C.c_int), P(C.c_int)]),
        "hp_server_simulate_policy": (C.c_int, [C.c_int, P(C.c_int), P(C.c_uint64), P(C.c_int), P(C.c_double),
                                                C.c_int, C.c_uint64, C.c_int, C.c_int, C.c_double, P(C.c_int),
                                                P(C.c_int), P(C.c_int)]),
        "hp_fuse_params_default": (None, [P(FuseParams)]),
        "hp_fuse_depth_maps": (C.c_int, [C.c_void_p, P(FuseView), C.c_int, P(FuseParams), P(PointCloudC)]),
        "hp_pfm_write": (C.c_int, [C.c_char_p, C.c_void_p, C.c_int, C.c_int, C.c_int]),
        "hp_pfm_read": (C.c_int, [C.c_char_p, C.c_void_p, C.c_size_t, P(C.c_int), P(C.c_int), P(C.c_int)]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    return lib


lib = _load()

#: Every exported entry point of include/hpmvs.h (checked against the .so by the tests).
EXPORTS = (
    "hp_status_string", "hp_params_default", "hp_version", "hp_ctx_create", "hp_ctx_destroy",
    "hp_ctx_last_error", "hp_ctx_synchronize", "hp_ctx_mem_info", "hp_ctx_stream", "hp_ctx_set_profiling",
    "hp_ctx_profile", "hp_ctx_profile_reset", "hp_image_upload", "hp_image_release",
    "hp_image_size", "hp_setup_homographies", "hp_solve", "hp_init_hypotheses", "hp_ncc_cost",
    "hp_propagate_pass", "hp_geometric_filter", "hp_pfm_write", "hp_pfm_read", "hp_solve_static",
    "hp_plan_options_default", "hp_plan_create", "hp_plan_run", "hp_plan_launch", "hp_plan_wait", "hp_plan_tune",
    "hp_plan_get_info", "hp_plan_destroy", "hp_schedule_build", "hp_server_options_default", "hp_server_create",
    "hp_submit", "hp_poll", "hp_server_drain", "hp_server_stats_get", "hp_server_stats_reset",
    "hp_server_last_error", "hp_server_first_error", "hp_server_destroy", "hp_server_simulate", "hp_server_simulate_policy",
    "hp_select_sources", "hp_project_seeds",
    "hp_ctx_set_image_cache", "hp_fuse_params_default", "hp_fuse_depth_maps",
)
STATIC_MAX_PIXELS = 1280 * 1024  # HP_STATIC_MAX_PIXELS


def solve_static(job: Job, params: Params, ref_image, src_textures: Sequence[int], out: Maps, device: int = 0,
                 stream: int = 0):
    """hp_solve_static: the single-view FP32 solve for callers that cannot let the library allocate device
    memory.  ``ref_image`` is a contiguous device FP32 tensor (H, W); ``src_textures`` are texture-object
    handles over the FP32 source images (linear filter, clamp, unnormalised coordinates); ``out`` holds device
    maps.  No device memory is allocated: the state lives in a fixed array of HP_STATIC_MAX_PIXELS pixels."""
    if len(src_textures) != job.num_sources:
        raise ValueError(f"solve_static: {len(src_textures)} source textures for a job with {job.num_sources} sources")
    import torch
    if not (isinstance(ref_image, torch.Tensor) and ref_image.is_cuda and ref_image.dtype == torch.float32
            and ref_image.dim() == 2):
        raise ValueError("solve_static: ref_image must be a 2-D float32 CUDA tensor")
    if ref_image.stride(1) != 1:
        raise ValueError("solve_static: ref_image rows must be contiguous")
    h, w = ref_image.shape
    tex = (C.c_ulonglong * len(src_textures))(*src_textures)
    st = lib.hp_solve_static(device, stream or None, C.byref(job), int(ref_image.data_ptr()), int(ref_image.stride(0)), w, h, tex,
                             C.byref(params), C.byref(out))
    if st != OK:
        raise HpError(st, "hp_solve_static")


def default_params(**kw) -> Params:
    """hp_params_default() with keyword overrides (radius, stride, precision, ...)."""
    p = Params()
    lib.hp_params_default(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise TypeError(f"unknown parameter {k}")
        setattr(p, k, v)
    return p


def make_camera(K, R, t) -> Camera:
    c = Camera()
    c.K[:] = [float(v) for v in np.asarray(K, np.float64).ravel()]
    c.R[:] = [float(v) for v in np.asarray(R, np.float64).ravel()]
    c.t[:] = [float(v) for v in np.asarray(t, np.float64).ravel()]
    return c


def setup_homographies(ref: Camera, srcs: Sequence[Camera]):
    """FP64 (K_ref^-1, [A|b] per source) as the engine computes them."""
    n = len(srcs)
    kinv = (C.c_double * 9)()
    ab = (C.c_double * (12 * max(n, 1)))()
    arr = (Camera * max(n, 1))(*srcs)
    st = lib.hp_setup_homographies(C.byref(ref), arr, n, kinv, ab)
    if st != OK:
        raise HpError(st, "hp_setup_homographies")
    return np.array(kinv[:], np.float64).reshape(3, 3), np.array(ab[: 12 * n], np.float64).reshape(n, 12)


def _ptr(a) -> int:
    """Address of a numpy array (host) or a torch tensor (device)."""
    if isinstance(a, np.ndarray):
        if not a.flags["C_CONTIGUOUS"]:
            raise ValueError("arrays must be C-contiguous")
        return a.ctypes.data
    return int(a.data_ptr())


def _mem(a) -> int:
    return MEMORY_HOST if isinstance(a, np.ndarray) else MEMORY_DEVICE


class Context:
    """An engine context (hp_ctx): one device, one stream, resident images."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        st = lib.hp_ctx_create(device, C.byref(h))
        if st != OK:
            raise HpError(st, f"hp_ctx_create(device={device})")
        self._h = h
        self.device = device

    def close(self):
        if getattr(self, "_h", None):
            lib.hp_ctx_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _check(self, st: int, what: str):
        if st != OK:
            raise HpError(st, f"{what}: {lib.hp_ctx_last_error(self._h).decode()}")

    @property
    def handle(self):
        return self._h

    def synchronize(self):
        self._check(lib.hp_ctx_synchronize(self._h), "hp_ctx_synchronize")

    def set_image_cache(self, limit_bytes: int):
        """Bytes of released images kept for reuse by later uploads of the same size (0: none)."""
        self._check(lib.hp_ctx_set_image_cache(self._h, int(limit_bytes)), "hp_ctx_set_image_cache")

    def mem_info(self):
        f, t = C.c_size_t(), C.c_size_t()
        self._check(lib.hp_ctx_mem_info(self._h, C.byref(f), C.byref(t)), "hp_ctx_mem_info")
        return f.value, t.value

    @property
    def stream_handle(self) -> int:
        """The context's cudaStream_t as an integer (e.g. for torch.cuda.ExternalStream)."""
        s = C.c_void_p()
        self._check(lib.hp_ctx_stream(self._h, C.byref(s)), "hp_ctx_stream")
        return s.value or 0

    def set_profiling(self, on: bool):
        self._check(lib.hp_ctx_set_profiling(self._h, int(bool(on))), "hp_ctx_set_profiling")

    def profile(self) -> dict:
        p = Profile()
        self._check(lib.hp_ctx_profile(self._h, C.byref(p)), "hp_ctx_profile")
        return p.as_dict()

    def profile_reset(self):
        self._check(lib.hp_ctx_profile_reset(self._h), "hp_ctx_profile_reset")

    def upload(self, img) -> int:
        """Upload a grayscale image (numpy u8/f16/f32 on host, or a contiguous torch CUDA tensor)."""
        dt = {np.dtype(np.uint8): DTYPE_U8, np.dtype(np.float16): DTYPE_F16, np.dtype(np.float32): DTYPE_F32}
        if isinstance(img, np.ndarray):
            img = np.ascontiguousarray(img)
            code = dt.get(img.dtype)
        else:
            import torch
            code = {torch.uint8: DTYPE_U8, torch.float16: DTYPE_F16, torch.float32: DTYPE_F32}.get(img.dtype)
            if not img.is_contiguous():
                raise ValueError("device image must be contiguous")
        if code is None:
            raise TypeError(f"unsupported image dtype {img.dtype}")
        h, w = img.shape
        iid = C.c_int()
        self._check(lib.hp_image_upload(self._h, _ptr(img), _mem(img), w, h, code, C.byref(iid)), "hp_image_upload")
        return iid.value

    def release(self, image_id: int):
        self._check(lib.hp_image_release(self._h, image_id), "hp_image_release")

    def solve(self, jobs: Sequence[Job], params: Params, outs: Sequence[Maps]):
        jarr = (Job * len(jobs))(*jobs)
        marr = (Maps * len(outs))(*outs)
        self._check(lib.hp_solve(self._h, jarr, len(jobs), C.byref(params), marr), "hp_solve")

    def init_hypotheses(self, job: Job, params: Params, maps: Maps):
        self._check(lib.hp_init_hypotheses(self._h, C.byref(job), C.byref(params), C.byref(maps)),
                    "hp_init_hypotheses")

    def ncc_cost(self, job: Job, params: Params, maps: Maps):
        self._check(lib.hp_ncc_cost(self._h, C.byref(job), C.byref(params), C.byref(maps)), "hp_ncc_cost")

    def propagate_pass(self, job: Job, params: Params, maps: Maps, iteration: int, color: int):
        self._check(lib.hp_propagate_pass(self._h, C.byref(job), C.byref(params), C.byref(maps), iteration, color),
                    "hp_propagate_pass")

    def geometric_filter(self, ref_cam: Camera, depth, normal, confidence, src_cams: Sequence[Camera],
                         src_depths, src_normals, depth_tol=0.12, normal_tol_cos=-1.0, min_consistent=2):
        """In-place filter (depth and confidence); arrays all host numpy or all device tensors."""
        h, w = depth.shape[:2]
        n = len(src_cams)
        cams = (Camera * max(n, 1))(*src_cams)
        dps = (C.c_void_p * max(n, 1))(*[_ptr(a) for a in src_depths])
        nps = (C.c_void_p * max(n, 1))(*[_ptr(a) for a in src_normals])
        self._check(lib.hp_geometric_filter(self._h, C.byref(ref_cam), w, h, _ptr(depth), _ptr(normal),
                                            _ptr(confidence), n, cams, dps, nps, _mem(depth), depth_tol,
                                            normal_tol_cos, min_consistent), "hp_geometric_filter")

    def fuse_views(self, views: Sequence[FuseView], params: FuseParams, out: PointCloudC) -> int:
        """hp_fuse_depth_maps as is: fills ``out`` up to its capacity; returns the number of fused points."""
        varr = (FuseView * len(views))(*views)
        self._check(lib.hp_fuse_depth_maps(self._h, varr, len(views), C.byref(params), C.byref(out)),
                    "hp_fuse_depth_maps")
        return int(out.count)

    def fuse(self, cameras: Sequence[Camera], depths, normals, confidences=None, grays=None, neighbors=None,
             params: Optional[FuseParams] = None) -> "DensePointCloud":
        """Fuses per-view maps (all host numpy or all device tensors; confidences / grays may be None or
        hold None entries) into a DensePointCloud of the same kind.  ``neighbors``: per view a list of view
        indices, or None for every other view.  Counts first, then writes into arrays of exactly that size."""
        n = len(cameras)
        prm = FuseParams.from_buffer_copy(params if params is not None else fuse_params())
        prm.memory = _mem(depths[0])
        keep, views = [], []
        for i in range(n):
            v = FuseView()
            v.cam = cameras[i]
            v.height, v.width = depths[i].shape[:2]
            v.depth, v.normal = _ptr(depths[i]), _ptr(normals[i])
            cf = confidences[i] if confidences is not None else None
            g = grays[i] if grays is not None else None
            v.confidence = _ptr(cf) if cf is not None else None
            v.gray = _ptr(g) if g is not None else None
            if neighbors is not None and neighbors[i] is not None:
                nb = np.ascontiguousarray(neighbors[i], np.int32)
                keep.append(nb)
                v.neighbors = nb.ctypes.data_as(C.POINTER(C.c_int))
                v.num_neighbors = len(nb)
            views.append(v)
        out = PointCloudC()
        out.memory = prm.memory
        total = self.fuse_views(views, prm, out)
        if prm.memory == MEMORY_HOST:
            arrs = [np.zeros((total, 3), np.float32) for _ in range(3)]
        else:
            import torch
            arrs = [torch.zeros((total, 3), dtype=torch.float32, device=depths[0].device) for _ in range(3)]
        if total:
            out.positions, out.normals, out.colors = (_ptr(a) for a in arrs)
            out.capacity = total
            self.fuse_views(views, prm, out)
        return DensePointCloud(*arrs)


def fuse_params(**kw) -> FuseParams:
    """hp_fuse_params_default() with keyword overrides (min_views, max_depth_rel, ...)."""
    p = FuseParams()
    lib.hp_fuse_params_default(C.byref(p))
    for k, v in kw.items():
        if not hasattr(p, k):
            raise TypeError(f"unknown fusion parameter {k}")
        setattr(p, k, v)
    return p


@dataclass
class DensePointCloud:
    """DensePointCloud (include/types.h:93-106): world-frame positions, unit normals and colours, (N, 3)
    float32 each (host numpy or device tensors)."""
    positions: object
    normals: object
    colors: object

    def size(self) -> int:
        return int(self.positions.shape[0])


def plan_options(**kw) -> PlanOptions:
    o = PlanOptions()
    lib.hp_plan_options_default(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class Plan:
    """A batched solve prepared once (hp_plan): jobs, params and output maps bound at creation."""

    def __init__(self, ctx: "Context", jobs: Sequence[Job], params: Params, outs: Sequence[Maps],
                 options: PlanOptions | None = None):
        self.ctx = ctx
        self._outs = list(outs)  # keep the Maps (and their arrays) alive
        jarr = (Job * len(jobs))(*jobs)
        marr = (Maps * len(outs))(*outs)
        h = C.c_void_p()
        opts = options if options is not None else plan_options()
        ctx._check(lib.hp_plan_create(ctx.handle, jarr, len(jobs), C.byref(params), C.byref(opts), marr, C.byref(h)),
                   "hp_plan_create")
        self._h = h

    def run(self):
        self.ctx._check(lib.hp_plan_run(self._h), "hp_plan_run")

    def launch(self):
        self.ctx._check(lib.hp_plan_launch(self._h), "hp_plan_launch")

    def wait(self):
        self.ctx._check(lib.hp_plan_wait(self._h), "hp_plan_wait")

    def tune(self, repeats: int = 3) -> dict:
        info = PlanInfo()
        self.ctx._check(lib.hp_plan_tune(self._h, repeats, C.byref(info)), "hp_plan_tune")
        return info.as_dict()

    def info(self) -> dict:
        info = PlanInfo()
        self.ctx._check(lib.hp_plan_get_info(self._h, C.byref(info)), "hp_plan_get_info")
        return info.as_dict()

    def close(self):
        if getattr(self, "_h", None):
            lib.hp_plan_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def schedule_build(tiles: Sequence[int], stage_begin: Sequence[int], stage_end: Sequence[int]):
    """The persistent ticket order (hp_schedule_build): arrays (entry_ticket[n+1], entry_view[n], entry_stage[n])."""
    n = len(tiles)
    cap = sum(max(0, e - b) for b, e in zip(stage_begin, stage_end)) + 1
    arr = lambda xs: (C.c_int * max(1, len(xs)))(*xs)
    et, ev, es, ne = (C.c_int * (cap + 1))(), (C.c_int * cap)(), (C.c_int * cap)(), C.c_int()
    st = lib.hp_schedule_build(n, arr(tiles), arr(stage_begin), arr(stage_end), cap, et, ev, es, C.byref(ne))
    if st != OK:
        raise HpError(st, "hp_schedule_build")
    k = ne.value
    return np.array(et[:k + 1]), np.array(ev[:k]), np.array(es[:k])


def server_options(**kw) -> ServerOptions:
    o = ServerOptions()
    lib.hp_server_options_default(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


class Server:
    """Continuous-batching solve server (hp_server): submit jobs from any thread, poll completions.

    The output maps of a request are kept alive here until its completion has been polled."""

    def __init__(self, ctx: "Context", params: Params, options: ServerOptions | None = None, **kw):
        self.ctx = ctx
        opts = options if options is not None else server_options(**kw)
        h = C.c_void_p()
        ctx._check(lib.hp_server_create(ctx.handle, C.byref(params), C.byref(opts), C.byref(h)), "hp_server_create")
        self._h = h
        self._maps = {}
        self._lock = threading.Lock()

    def _fail(self, st: int, what: str):
        raise HpError(st, f"{what}: {lib.hp_server_last_error(self._h).decode()}")

    def submit(self, job: Job, maps: Maps) -> int:
        rid = C.c_uint64()
        # The maps are registered under the lock that poll() takes to release them, so a request that
        # completes before submit returns still finds its entry.
        with self._lock:
            st = lib.hp_submit(self._h, C.byref(job), C.byref(maps), C.byref(rid))
            if st == OK:
                self._maps[rid.value] = maps
        if st != OK:
            self._fail(st, "hp_submit")
        return rid.value

    def poll(self, timeout_ms: int = 0, capacity: int = 256) -> List[dict]:
        """Completed requests as dicts (request_id, status, latency_ms, queue_ms)."""
        buf = (Completion * capacity)()
        n = C.c_int()
        st = lib.hp_poll(self._h, buf, capacity, C.byref(n), int(timeout_ms))
        if st != OK:
            self._fail(st, "hp_poll")
        out = []
        for c in buf[:n.value]:
            out.append({"request_id": c.request_id, "status": c.status, "latency_ms": c.latency_ms,
                        "queue_ms": c.queue_ms})
            with self._lock:
                self._maps.pop(c.request_id, None)
        return out

    def drain(self, timeout_ms: int = -1):
        st = lib.hp_server_drain(self._h, int(timeout_ms))
        if st != OK:
            self._fail(st, "hp_server_drain")

    def stats(self) -> dict:
        s = ServerStats()
        st = lib.hp_server_stats_get(self._h, C.byref(s))
        if st != OK:
            self._fail(st, "hp_server_stats_get")
        return s.as_dict()

    def reset_stats(self):
        lib.hp_server_stats_reset(self._h)

    def last_error(self) -> str:
        """The server's most recent error message (a failed step names the request, stage and tile)."""
        return lib.hp_server_last_error(self._h).decode()

    def first_error(self) -> str:
        """The server's first error since creation ("" if none)."""
        return lib.hp_server_first_error(self._h).decode()

    def close(self):
        if getattr(self, "_h", None):
            lib.hp_server_destroy(self._h)
            self._h = None
            self._maps.clear()

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


SERVER_POLICY_ROUND_ROBIN, SERVER_POLICY_BUDGET = 0, 1


def server_simulate(arrive_step: Sequence[int], state_bytes: Sequence[int], stages: Sequence[int], max_active: int,
                    budget: int, passes_per_step: int, policy: int = 0, work: Optional[Sequence[float]] = None,
                    step_work: float = 0.0):
    """The server's admission and step policy without a device (hp_server_simulate_policy):
    (admit_step[n], finish_step[n], steps).  ``work`` is each request's work per stage (W * H * sources),
    ``step_work`` the budget policy's work per step in the same units."""
    n = len(arrive_step)
    m = max(1, n)
    a = (C.c_int * m)(*arrive_step)
    b = (C.c_uint64 * m)(*state_bytes)
    k = (C.c_int * m)(*stages)
    w = (C.c_double * m)(*(work if work is not None else [0.0] * n))
    adm, fin, steps = (C.c_int * m)(), (C.c_int * m)(), C.c_int()
    st = lib.hp_server_simulate_policy(n, a, b, k, w, max_active, budget, passes_per_step, policy, float(step_work),
                                       adm, fin, C.byref(steps))
    if st != OK:
        raise HpError(st, "hp_server_simulate_policy")
    return np.array(adm[:n]), np.array(fin[:n]), steps.value


class SfmPoints:
    """Sparse points and their tracks (hp_sparse_points) over numpy arrays kept alive here.
    ``positions``: (P, 3) float64 world points; ``tracks``: one sequence of camera indices per point."""

    def __init__(self, positions, tracks):
        self.positions = np.ascontiguousarray(np.asarray(positions, np.float64).reshape(-1, 3))
        self.offsets = np.zeros(len(tracks) + 1, np.int32)
        self.offsets[1:] = np.cumsum([len(t) for t in tracks]) if len(tracks) else []
        flat = [int(c) for t in tracks for c in t]
        self.images = np.ascontiguousarray(np.asarray(flat if flat else [0], np.int32))
        self.c = SparsePoints(len(tracks), self.positions.ctypes.data, self.offsets.ctypes.data,
                              self.images.ctypes.data)


def select_sources(cameras: Sequence[Camera], points: SfmPoints, num_sources: int, registered=None) -> List[dict]:
    """hp_select_sources (selectSourceViews, patchmatch_mvs.cu:74-157): per registered camera its sources
    (best first), their scores and baseline angles, and the depth range."""
    n = len(cameras)
    cams = (Camera * n)(*cameras)
    reg = (C.c_int * n)(*([1] * n if registered is None else [int(bool(r)) for r in registered]))
    out = (ViewSelection * n)()
    cnt = C.c_int()
    st = lib.hp_select_sources(cams, reg, n, C.byref(points.c), int(num_sources), out, C.byref(cnt))
    if st != OK:
        raise HpError(st, "hp_select_sources")
    res = []
    for v in out[:cnt.value]:
        k = v.num_sources
        res.append({"ref": v.ref_image, "sources": list(v.sources[:k]), "scores": list(v.scores[:k]),
                    "baseline_deg": list(v.baseline_deg[:k]), "depth_min": v.depth_min, "depth_max": v.depth_max})
    return res


def project_seeds(camera: Camera, ref: int, depth_min: float, depth_max: float, points: SfmPoints):
    """hp_project_seeds: the SfM seeds of reference camera ``ref`` as a ctypes Seed array (point order)."""
    n = C.c_int()
    st = lib.hp_project_seeds(C.byref(camera), int(ref), float(depth_min), float(depth_max), C.byref(points.c),
                              None, 0, C.byref(n))
    if st != OK:
        raise HpError(st, "hp_project_seeds")
    arr = (Seed * max(1, n.value))()
    st = lib.hp_project_seeds(C.byref(camera), int(ref), float(depth_min), float(depth_max), C.byref(points.c),
                              arr, n.value, C.byref(n))
    if st != OK:
        raise HpError(st, "hp_project_seeds")
    arr.count = n.value
    return arr


def with_seeds(job: Job, seeds, radius: int = 50) -> Job:
    """Attach seeds (from project_seeds) to a job; the job keeps the array alive."""
    job.seeds = C.cast(seeds, C.c_void_p).value if seeds is not None and seeds.count else None
    job.num_seeds = seeds.count if seeds is not None else 0
    job.seed_radius = int(radius)
    job._seeds = seeds
    return job


def make_job(ref_image: int, src_images: Sequence[int], ref_cam: Camera, src_cams: Sequence[Camera],
             depth_min: float, depth_max: float, seed: int = 42, view_id: int = 0, iterations: int = 12,
             coeffs=None) -> Job:
    """Build an hp_job.  ``coeffs`` = (kinv[9], ab[S,12]) float32 replaces the FP64 setup."""
    if not 1 <= len(src_images) <= MAX_SOURCES or len(src_images) != len(src_cams):
        raise ValueError("need 1..8 sources with one camera each")
    j = Job()
    j.ref_image = ref_image
    j.num_sources = len(src_images)
    for i, s in enumerate(src_images):
        j.src_images[i] = s
        j.src_cams[i] = src_cams[i]
    j.ref_cam = ref_cam
    j.depth_min, j.depth_max = float(depth_min), float(depth_max)
    j.seed, j.view_id, j.iterations = int(seed), int(view_id), int(iterations)
    if coeffs is not None:
        kinv, ab = coeffs
        j.use_coeffs = 1
        j.kinv[:] = [float(v) for v in np.asarray(kinv, np.float32).ravel()]
        ab = np.asarray(ab, np.float32).reshape(-1, 12)
        for s in range(ab.shape[0]):
            j.ab[s][:] = [float(v) for v in ab[s]]
    return j


def host_maps(h: int, w: int, confidence: bool = False):
    """(Maps, depth, normal, cost) with fresh host arrays; with ``confidence`` a
    fifth array, the confidence map, is bound and returned too."""
    depth = np.zeros((h, w), np.float32)
    normal = np.zeros((h, w, 3), np.float32)
    cost = np.zeros((h, w), np.float32)
    if confidence:
        conf = np.zeros((h, w), np.float32)
        return maps_of(depth, normal, cost, conf), depth, normal, cost, conf
    return maps_of(depth, normal, cost), depth, normal, cost


def maps_of(depth, normal, cost, confidence=None) -> Maps:
    """Maps over existing arrays (host numpy or device tensors, not mixed).

    ``confidence`` (optional) receives 1 - cost / 2, formed on the device.  The
    returned struct keeps the arrays alive (``.arrays``): the engine writes
    through its raw pointers, so the arrays must outlive every call using it.
    """
    m = Maps(_mem(depth), _ptr(depth), _ptr(normal), _ptr(cost),
             _ptr(confidence) if confidence is not None else None)
    m.arrays = (depth, normal, cost, confidence)
    return m


def pfm_write(path: str, data: np.ndarray):
    data = np.ascontiguousarray(data, np.float32)
    ch = 1 if data.ndim == 2 else data.shape[2]
    st = lib.hp_pfm_write(path.encode(), data.ctypes.data, data.shape[1], data.shape[0], ch)
    if st != OK:
        raise HpError(st, f"hp_pfm_write({path})")


def pfm_read(path: str) -> np.ndarray:
    w, h, ch = C.c_int(), C.c_int(), C.c_int()
    st = lib.hp_pfm_read(path.encode(), None, 0, C.byref(w), C.byref(h), C.byref(ch))
    if st != OK:
        raise HpError(st, f"hp_pfm_read({path})")
    out = np.empty((h.value, w.value, ch.value) if ch.value == 3 else (h.value, w.value), np.float32)
    st = lib.hp_pfm_read(path.encode(), out.ctypes.data, out.size, C.byref(w), C.byref(h), C.byref(ch))
    if st != OK:
        raise HpError(st, f"hp_pfm_read({path})")
    return out


# --------------------------------------------------------------------------------------------
# Mirror of the reference's stage API (types.h DepthMap / PipelineConfig, patchmatch_mvs.h).
# --------------------------------------------------------------------------------------------

@dataclass
class ViewParams:
    """MVSViewParams (src/dense_recon/patchmatch_mvs.h:22-28): a reference image, its sources, depth range."""
    ref_image_id: int
    source_ids: List[int]
    depth_min: float
    depth_max: float


@dataclass
class DepthMap:
    """DepthMap (include/types.h:85-91): depth (0 = invalid), camera-frame normal, confidence = 1 - cost/2."""
    image_id: int
    depth: np.ndarray
    normal: np.ndarray
    confidence: np.ndarray
    cost: np.ndarray = field(repr=False, default=None)

    @property
    def width(self):
        return self.depth.shape[1]

    @property
    def height(self):
        return self.depth.shape[0]


@dataclass
class MVSConfig:
    """The PipelineConfig fields the stage reads (include/types.h:120-169, patchmatch_mvs.cu:1065-1070)."""
    mvs_iterations: int = 12
    mvs_patch_size: int = 11
    window_stride: int = 1
    precision: int = PRECISION_F32
    geometric_filter: bool = True
    save_intermediate: bool = False
    output_dir: Optional[str] = None
    device: int = 0
    sfm_seeding: bool = True   # paint the SfM points' depths over the random init (:1111-1177)
    seed_radius: int = 50      # SEED_RADIUS (:1123)


def run_patchmatch_mvs(images: Sequence[np.ndarray], cameras: Sequence[Camera],
                       views: Optional[Sequence[ViewParams]] = None, config: MVSConfig = MVSConfig(),
                       ctx: Optional[Context] = None, sfm: Optional[SfmPoints] = None,
                       registered: Optional[Sequence[bool]] = None) -> List[DepthMap]:
    """runPatchMatchMVS (patchmatch_mvs.cu:1028-1388).

    With ``sfm`` (the sparse points and their tracks) and no ``views``, the views come from
    :func:`select_sources` with min(8, max(3, registered - 1)) sources (:1037-1039), and with
    ``config.sfm_seeding`` every view's hypotheses are seeded from the points it sees
    (:1111-1177).  Explicit ``views`` override the selection.
    Views without sources are skipped (:1089-1092); the per-view seed is
    42 + 1e6 * ref_id (:1106); radius = (patch_size - 1) / 2 clamped to 1..7;
    confidence = 1 - cost / 2 (:1246-1252); with iterations > 0 and >= 2 maps the
    geometric filter runs with tolerance 0.12, normal check off, 2 agreeing
    sources (:1267-1384); PFM depth is written per view when save_intermediate.
    """
    own = ctx is None
    ctx = ctx or Context(config.device)
    try:
        radius = min(MAX_RADIUS, max(1, (config.mvs_patch_size - 1) // 2))
        params = default_params(radius=radius, stride=config.window_stride, precision=config.precision)
        # The reference writes each view's depth before filtering (:1254-1257); with
        # intermediates wanted the filter therefore runs after the write, on the host
        # maps, through hp_geometric_filter (the same check, bit for bit).
        fused = config.geometric_filter and not (config.save_intermediate and config.output_dir)
        if fused:
            # The reference's constants (:1273-1276): 12% depth, normal check off, 2 sources.
            params.filter_min_consistent = GEOM_MIN_CONSISTENT
            params.filter_depth_tol = GEOM_DEPTH_TOL
            params.filter_normal_cos = GEOM_NORMAL_COS
        if views is None:
            if sfm is None:
                raise ValueError("run_patchmatch_mvs needs views or sfm points")
            reg = [True] * len(cameras) if registered is None else list(registered)
            ns = min(MAX_SOURCES, max(3, sum(bool(r) for r in reg) - 1))
            views = [ViewParams(v["ref"], v["sources"], v["depth_min"], v["depth_max"])
                     for v in select_sources(cameras, sfm, ns, reg)]
        ids = {}
        views = [v for v in views if v.source_ids]
        for v in views:
            for i in [v.ref_image_id, *v.source_ids]:
                if i not in ids:
                    ids[i] = ctx.upload(images[i])
        jobs, outs, maps = [], [], []
        for v in views:
            h, w = images[v.ref_image_id].shape[:2]
            m, d, n, c, cf = host_maps(h, w, confidence=True)
            job = make_job(ids[v.ref_image_id], [ids[s] for s in v.source_ids], cameras[v.ref_image_id],
                           [cameras[s] for s in v.source_ids], v.depth_min, v.depth_max,
                           seed=42 + 1_000_000 * v.ref_image_id, view_id=v.ref_image_id,
                           iterations=config.mvs_iterations)
            if sfm is not None and config.sfm_seeding:
                with_seeds(job, project_seeds(cameras[v.ref_image_id], v.ref_image_id, v.depth_min, v.depth_max,
                                              sfm), config.seed_radius)
            jobs.append(job)
            outs.append(m)
            maps.append((d, n, c, cf))
        if jobs:
            # The geometric filter is the solve's last stage (params.filter_*):
            # in place and in view order on the device, as the reference's loop.
            ctx.solve(jobs, params, outs)
        result = [DepthMap(v.ref_image_id, d, n, cf, c) for v, (d, n, c, cf) in zip(views, maps)]
        if config.save_intermediate and config.output_dir:
            for dm in result:
                pfm_write(os.path.join(config.output_dir, f"depth_{dm.image_id}.pfm"), dm.depth)
        if config.geometric_filter and not fused and config.mvs_iterations > 0 and len(result) >= 2:
            # In place and in view order: a later view sees earlier views filtered.
            by_id = {dm.image_id: dm for dm in result}
            for v, dm in zip(views, result):
                srcs = [s for s in v.source_ids
                        if s in by_id and s != v.ref_image_id and by_id[s].depth.shape == dm.depth.shape]
                if len(srcs) >= GEOM_MIN_CONSISTENT:
                    ctx.geometric_filter(cameras[v.ref_image_id], dm.depth, dm.normal, dm.confidence,
                                         [cameras[s] for s in srcs], [by_id[s].depth for s in srcs],
                                         [by_id[s].normal for s in srcs])
                    dm.cost[dm.confidence == 0] = 2.0
        for i in ids.values():
            ctx.release(i)
        return result
    finally:
        if own:
            ctx.close()


def _gray_f32(img) -> np.ndarray:
    a = np.asarray(img)
    if a.dtype == np.uint8:
        return (a.astype(np.float32) / np.float32(255.0)).astype(np.float32)
    return np.ascontiguousarray(a, np.float32)


def fuse_depth_maps(depth_maps: Sequence[DepthMap], cameras, images=None, params: Optional[FuseParams] = None,
                    neighbors=None, ctx: Optional[Context] = None) -> DensePointCloud:
    """fuseDepthMaps(depth_maps, poses, images) (src/dense_recon/point_cloud.h:7; a stub in the reference,
    point_cloud.cu:4-8) on the engine's fusion (hp_fuse_depth_maps).

    ``cameras`` and ``images`` are indexed by each map's ``image_id`` (as the reference's poses and images
    vectors are); the colour is the image's gray value (u8 scaled by 1/255, or float in [0, 1]).  Maps are
    host arrays as run_patchmatch_mvs returns them; ``neighbors`` lists, per map, the positions (in
    ``depth_maps``) of the maps to check, or None for all."""
    own = ctx is None
    ctx = ctx or Context(0)
    try:
        f32 = lambda a: np.ascontiguousarray(a, np.float32)
        return ctx.fuse([cameras[dm.image_id] for dm in depth_maps], [f32(dm.depth) for dm in depth_maps],
                        [f32(dm.normal) for dm in depth_maps], [f32(dm.confidence) for dm in depth_maps],
                        None if images is None else [_gray_f32(images[dm.image_id]) for dm in depth_maps],
                        neighbors, params)
    finally:
        if own:
            ctx.close()
