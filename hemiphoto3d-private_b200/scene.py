"""Seeded synthetic scenes with analytic ground truth for the engine's workloads.

Each scene is textured planes and spheres rendered by the host renderer in
``lib/libhpscene.so`` (ray casting, 2x2 supersampling) from pinhole cameras on
an arc aimed at a common target.  One albedo texture - uniform noise blurred
by a Gaussian of 1.5 texels, one texel about one pixel at the scene's typical
depth - covers every surface, so a surface point has the same value in every
view.  The renderer also returns per-pixel camera-z depth and camera-frame
normals, the ground truth the accuracy tests score against.

Workloads (all sizes, counts and ranges as stated):
  plane_sphere   5 views 640x480 u8, fx 500; plane z=3 + sphere r=0.5 at z=2.5;
                 2 m arc, 10 deg spacing; depth [1, 4]; r=5, s=2, S=4, 8 iterations
  multi_object   20 views 1920x1080 u8, fx 1500; 3 spheres + 2 tilted planes
                 (seeded) before a background plane at z=4.5; arc +-30 deg; depth [1, 6];
                 r=7, s=2, S=6, 12 iterations
  precision      32 views 3000x2000 FP16 + N(0, 0.01), fx 2400, multi_object
                 layout; r=7, S=8, 12 iterations
The arc convention: cameras at target + radius (sin a, 0, -cos a), looking at
the target (0, 0, radius), so the central camera sits at the world origin
looking down +z and the stated object depths are depths from it.
"""
from __future__ import annotations

import ctypes as C
import math
import os
from dataclasses import dataclass, field
from typing import List, Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
# The renderer library; HP_SCENE_LIB names another build of the same source
# (the bench's reference arm renders with one outside the engine's lib/).
SCENE_LIB_PATH = os.environ.get("HP_SCENE_LIB") or os.path.join(_HERE, "lib", "libhpscene.so")

PLANE, SPHERE = 0, 1


class _Obj(C.Structure):
    _fields_ = [
        ("kind", C.c_int), ("p", C.c_double * 3), ("n", C.c_double * 3), ("u", C.c_double * 3),
        ("v", C.c_double * 3), ("half_u", C.c_double), ("half_v", C.c_double), ("radius", C.c_double),
        ("tex_offset", C.c_double * 2),
    ]


_lib = None


def _scene_lib():
    global _lib
    if _lib is None:
        if not os.path.exists(SCENE_LIB_PATH):
            raise ImportError(f"{SCENE_LIB_PATH} is not built; run make in {_HERE}")
        _lib = C.CDLL(SCENE_LIB_PATH)
        P = C.POINTER
        _lib.hps_make_albedo.restype = C.c_int
        _lib.hps_make_albedo.argtypes = [C.c_int, C.c_double, C.c_uint64, C.c_float, P(C.c_float)]
        _lib.hps_render.restype = C.c_int
        _lib.hps_render.argtypes = [P(_Obj), C.c_int, P(C.c_float), C.c_int, C.c_double, P(C.c_double),
                                    P(C.c_double), P(C.c_double), C.c_int, C.c_int, C.c_int, C.c_float,
                                    P(C.c_float), P(C.c_float), P(C.c_float)]
    return _lib


@dataclass
class Obj:
    kind: int
    p: Sequence[float]
    n: Sequence[float] = (0.0, 0.0, -1.0)
    u: Sequence[float] = (1.0, 0.0, 0.0)
    v: Sequence[float] = (0.0, 1.0, 0.0)
    half_u: float = 0.0
    half_v: float = 0.0
    radius: float = 0.0
    tex_offset: Sequence[float] = (0.0, 0.0)

    def to_c(self) -> _Obj:
        o = _Obj()
        o.kind = self.kind
        o.p[:] = list(map(float, self.p))
        o.n[:] = list(map(float, self.n))
        o.u[:] = list(map(float, self.u))
        o.v[:] = list(map(float, self.v))
        o.half_u, o.half_v, o.radius = float(self.half_u), float(self.half_v), float(self.radius)
        o.tex_offset[:] = list(map(float, self.tex_offset))
        return o


@dataclass
class Cam:
    K: np.ndarray
    R: np.ndarray
    t: np.ndarray

    @property
    def center(self):
        return -self.R.T @ self.t


@dataclass
class View:
    image: np.ndarray          # u8 / f16 / f32, H x W
    image_f32: np.ndarray      # the same image in [0, 1] as float32
    depth_gt: np.ndarray       # camera z, 0 where the ray misses
    normal_gt: np.ndarray      # camera-frame normals
    cam: Cam


@dataclass
class Scene:
    name: str
    views: List[View]
    sources: List[List[int]]   # per reference view, its source view indices
    refs: List[int]            # reference views to solve
    depth_range: tuple
    radius: int
    stride: int
    iterations: int
    objects: List[Obj] = field(default_factory=list)

    @property
    def width(self):
        return self.views[0].image.shape[1]

    @property
    def height(self):
        return self.views[0].image.shape[0]

    def mpix_iter(self) -> float:
        return sum(self.views[r].image.shape[0] * self.views[r].image.shape[1] for r in self.refs) \
            * self.iterations / 1e6


def intrinsics(f: float, w: int, h: int) -> np.ndarray:
    return np.array([[f, 0, w / 2.0], [0, f, h / 2.0], [0, 0, 1]], np.float64)


def look_at(center, target, K) -> Cam:
    c = np.asarray(center, np.float64)
    z = np.asarray(target, np.float64) - c
    z /= np.linalg.norm(z)
    down = np.array([0.0, 1.0, 0.0])
    x = np.cross(down, z)
    x /= np.linalg.norm(x)
    y = np.cross(z, x)
    R = np.stack([x, y, z])
    return Cam(K, R, -R @ c)


def arc_cameras(n: int, angles_deg: Sequence[float], radius: float, K: np.ndarray) -> List[Cam]:
    target = np.array([0.0, 0.0, radius])
    cams = []
    for a in angles_deg:
        r = math.radians(a)
        cams.append(look_at(target + radius * np.array([math.sin(r), 0.0, -math.cos(r)]), target, K))
    return cams


_albedo_cache = {}


def albedo(seed: int, n: int = 2048, sigma: float = 1.5, contrast: float = 0.15) -> np.ndarray:
    key = (seed, n, sigma, contrast)
    if key not in _albedo_cache:
        out = np.empty((n, n), np.float32)
        st = _scene_lib().hps_make_albedo(n, sigma, seed, contrast, out.ctypes.data_as(C.POINTER(C.c_float)))
        if st != 0:
            raise RuntimeError("hps_make_albedo failed")
        _albedo_cache[key] = out
    return _albedo_cache[key]


def render(objs: Sequence[Obj], cam: Cam, w: int, h: int, tex: np.ndarray, texels_per_meter: float,
           spp: int = 2, background: float = 0.5):
    """(image f32, depth, normal) of one view."""
    arr = (_Obj * len(objs))(*[o.to_c() for o in objs])
    img = np.empty((h, w), np.float32)
    depth = np.empty((h, w), np.float32)
    normal = np.empty((h, w, 3), np.float32)
    K = np.ascontiguousarray(cam.K, np.float64)
    R = np.ascontiguousarray(cam.R, np.float64)
    t = np.ascontiguousarray(cam.t, np.float64)
    fp = C.POINTER(C.c_float)
    dp = C.POINTER(C.c_double)
    st = _scene_lib().hps_render(arr, len(objs), tex.ctypes.data_as(fp), tex.shape[0], texels_per_meter,
                                 K.ctypes.data_as(dp), R.ctypes.data_as(dp), t.ctypes.data_as(dp), w, h, spp,
                                 background, img.ctypes.data_as(fp), depth.ctypes.data_as(fp),
                                 normal.ctypes.data_as(fp))
    if st != 0:
        raise RuntimeError("hps_render failed")
    return img, depth, normal


def nearest_sources(cams: Sequence[Cam], ref: int, k: int, min_deg: float = 1.0) -> List[int]:
    """The k cameras whose viewing directions are closest in angle to the reference's (ties: lower index)."""
    zr = cams[ref].R[2]
    cand = []
    for i, c in enumerate(cams):
        if i == ref:
            continue
        ang = math.degrees(math.acos(max(-1.0, min(1.0, float(zr @ c.R[2])))))
        if ang >= min_deg:
            cand.append((ang, i))
    cand.sort()
    return [i for _, i in cand[:k]]


def quantize(img: np.ndarray, dtype: str, rng: Optional[np.random.Generator] = None, noise: float = 0.0):
    """Return (stored image, its float32 [0,1] value)."""
    x = img
    if noise > 0:
        x = np.clip(x + rng.normal(0.0, noise, x.shape).astype(np.float32), 0.0, 1.0)
    if dtype == "u8":
        q = np.clip(np.rint(x * 255.0), 0, 255).astype(np.uint8)
        return q, (q.astype(np.float32) / np.float32(255.0))
    if dtype == "f16":
        q = x.astype(np.float16)
        return q, q.astype(np.float32)
    q = x.astype(np.float32)
    return q, q


def _random_layout(rng: np.random.Generator, n_spheres: int, n_planes: int, background_z: float) -> List[Obj]:
    objs = [Obj(PLANE, (0.0, 0.0, background_z), n=(0.0, 0.0, -1.0), u=(1.0, 0.0, 0.0), v=(0.0, 1.0, 0.0))]
    for _ in range(n_spheres):
        objs.append(Obj(SPHERE, (rng.uniform(-1.0, 1.0), rng.uniform(-0.5, 0.5), rng.uniform(2.4, 4.0)),
                        radius=rng.uniform(0.3, 0.55), tex_offset=(rng.uniform(0, 5), rng.uniform(0, 5))))
    for _ in range(n_planes):
        tilt = math.radians(rng.uniform(15.0, 45.0))
        az = rng.uniform(0.0, 2 * math.pi)
        axis = np.array([math.cos(az), math.sin(az), 0.0])
        n0 = np.array([0.0, 0.0, -1.0])
        # Rodrigues rotation of n0 about axis by tilt
        n = n0 * math.cos(tilt) + np.cross(axis, n0) * math.sin(tilt) + axis * (axis @ n0) * (1 - math.cos(tilt))
        u = np.cross(np.array([0.0, 1.0, 0.0]), n)
        u /= np.linalg.norm(u)
        v = np.cross(n, u)
        objs.append(Obj(PLANE, (rng.uniform(-1.2, 1.2), rng.uniform(-0.5, 0.5), rng.uniform(2.0, 3.8)), n=n, u=u,
                        v=v, half_u=rng.uniform(0.35, 0.7), half_v=rng.uniform(0.3, 0.55),
                        tex_offset=(rng.uniform(0, 5), rng.uniform(0, 5))))
    return objs


def build_views(objs, cams, w, h, tex, tpm, dtype, rng, noise=0.0, spp=2) -> List[View]:
    views = []
    for c in cams:
        img, d, n = render(objs, c, w, h, tex, tpm, spp=spp)
        q, f = quantize(img, dtype, rng, noise)
        views.append(View(q, f, d, n, c))
    return views


def plane_sphere(seed: int = 7, w: int = 640, h: int = 480, n_views: int = 5, dtype: str = "u8") -> Scene:
    """5 views, plane z=3 + sphere (r 0.5, centre z 2.5), fx 500, 2 m arc at 10 deg."""
    rng = np.random.default_rng(seed)
    K = intrinsics(500.0 * w / 640.0, w, h)
    angles = [(i - (n_views - 1) / 2.0) * 10.0 for i in range(n_views)]
    cams = arc_cameras(n_views, angles, 2.0, K)
    objs = [Obj(PLANE, (0.0, 0.0, 3.0)), Obj(SPHERE, (0.0, 0.0, 2.5), radius=0.5, tex_offset=(1.3, 2.1))]
    tpm = K[0, 0] / 2.75
    views = build_views(objs, cams, w, h, albedo(seed), tpm, dtype, rng)
    refs = list(range(n_views))
    return Scene("plane_sphere", views, [nearest_sources(cams, r, 4) for r in refs], refs, (1.0, 4.0), 5, 2, 8, objs)


def multi_object(seed: int = 11, w: int = 1920, h: int = 1080, n_views: int = 20, n_src: int = 6, f: float = 1500.0,
                 dtype: str = "u8", noise: float = 0.0, radius: int = 7, stride: int = 2, iterations: int = 12,
                 n_refs: Optional[int] = None) -> Scene:
    """3 spheres + 2 tilted planes (seeded poses) before a background plane; arc +-30 deg."""
    rng = np.random.default_rng(seed)
    K = intrinsics(f, w, h)
    angles = list(np.linspace(-30.0, 30.0, n_views))
    cams = arc_cameras(n_views, angles, 3.0, K)
    objs = _random_layout(rng, 3, 2, 4.5)
    tpm = f / 3.5
    views = build_views(objs, cams, w, h, albedo(seed), tpm, dtype, rng, noise)
    refs = list(range(n_views if n_refs is None else n_refs))
    return Scene("multi_object", views, [nearest_sources(cams, r, n_src) for r in refs], refs, (1.0, 6.0), radius,
                 stride, iterations, objs)


def precision(seed: int = 13, w: int = 3000, h: int = 2000, n_views: int = 32, stride: int = 2,
              n_refs: Optional[int] = None) -> Scene:
    """32 views 3000x2000, FP16 + N(0, 0.01), fx 2400; r=7, S=8, 12 iterations."""
    return multi_object(seed, w, h, n_views, 8, 2400.0 * w / 3000.0, "f16", 0.01, 7, stride, 12, n_refs)


def depth_metrics(depth: np.ndarray, gt: np.ndarray, rel_tol: float = 0.01, mask: Optional[np.ndarray] = None):
    """(completeness, accuracy, mean rel err) over GT-valid pixels: completeness = share of valid GT pixels
    with a depth within rel_tol; accuracy = mean relative error of retained (depth > 0) pixels."""
    valid = gt > 0
    if mask is not None:
        valid &= mask
    rel = np.abs(depth - gt) / np.where(gt > 0, gt, 1)
    good = valid & (rel <= rel_tol)
    kept = valid & (depth > 0)
    comp = good.sum() / max(1, valid.sum())
    mean_err = float(rel[kept].mean()) if kept.any() else float("nan")
    return float(comp), float(kept.sum() / max(1, valid.sum())), mean_err


def sparse_points(scene: Scene, n: int = 2000, seed: int = 0, rel_tol: float = 0.02):
    """A stand-in for an SfM sparse reconstruction of a rendered scene: `n` surface points back-projected
    from random ground-truth pixels of random views, each with the track of views that see it (projection
    inside the image and ground-truth depth within rel_tol of the point's depth).  Points seen by fewer than
    two views are dropped.  Returns (positions (P, 3) float64, tracks list of camera-index lists)."""
    rng = np.random.default_rng(seed)
    H, W = scene.height, scene.width
    pts, tracks = [], []
    for _ in range(n):
        v = scene.views[int(rng.integers(0, len(scene.views)))]
        y, x = int(rng.integers(0, H)), int(rng.integers(0, W))
        d = float(v.depth_gt[y, x])
        if d <= 0:
            continue
        pc = np.linalg.solve(v.cam.K, np.array([x + 0.5, y + 0.5, 1.0])) * d
        pw = v.cam.R.T @ (pc - v.cam.t)
        tr = []
        for j, w in enumerate(scene.views):
            q = w.cam.R @ pw + w.cam.t
            if q[2] <= 0:
                continue
            u = w.cam.K @ q
            ux, uy = u[0] / u[2], u[1] / u[2]
            if not (0 <= ux < W and 0 <= uy < H):
                continue
            g = float(w.depth_gt[int(uy), int(ux)])
            if g > 0 and abs(g - q[2]) <= rel_tol * q[2]:
                tr.append(j)
        if len(tr) >= 2:
            pts.append(pw)
            tracks.append(tr)
    return np.array(pts, np.float64).reshape(-1, 3), tracks
