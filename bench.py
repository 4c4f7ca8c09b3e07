#!/usr/bin/env python
"""Headline benchmark: depth-map Mpix*iter/s of the PatchMatch engine on B200.

Workload (one "step"): the multi-object scene - 20 reference views of
1920x1080 u8 images, 6 sources each, 15x15 window sampled at stride 2, 12
red-black iterations, depth range [1, 6] m - solved in one batched hp_solve
(random init, initial cost, 24 half-pass launches over all 20 views).
Units per step = 20 * 1920 * 1080 * 12 = 497.7 Mpix*iter.

  value  device-resident: images uploaded once, outputs in device memory,
         K steps timed with CUDA events on the engine's stream.
  e2e    through the public API with host buffers: every step uploads the 20
         images from pinned host memory and reads depth, normal and cost of
         every view back to pinned host memory.

Inputs (20 x 2.07 Mpix images, 20 x 41 MB of state) exceed the 126 MB L2, so
no flush between steps is needed.  Multi-GPU (torchrun): views are
independent, each rank solves its own 20-view batch (weak scaling, no
collective on the data path); the step time is the max over ranks.

--impl reference times the reference's algorithm on the host cores (the CPU
restatement in oracle/, all threads): one red-black iteration of view 0 of the
same workload per step.  It loads nothing from the engine: the scene is
rendered by oracle/libpmscene.so (the renderer's source, built apart), and
where the reference's own kernels were compiled (oracle/_ref/libpmref.so) it
also times them on the GPU ("reference_gpu") at the parameters they support -
radius 5, stride 1 - which the engine arm times too ("reference_params").
"""
from __future__ import annotations

import argparse
import importlib
import importlib.util
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "oracle", "ref_harness")]
PKG = "hemiphoto3d-private_b200"

WORKLOAD = dict(name="multi_object_20x1920x1080", views=20, width=1920, height=1080, sources=6, radius=7, stride=2,
                iterations=12, depth_range=[1.0, 6.0], image_dtype="u8")
METRIC = "depth-map Mpix*iter/s on 1 B200 (FP16-acc vs plain FP32)"
# Serving form: Poisson arrivals, each request one depth-map solve on the FP16-acc path.
# Batched form: one plan over views of uneven sizes, autotuned schedule, replayed as a CUDA graph.
BATCHED = dict(name="batched_uneven_64", views=64, sizes=[[640, 480], [1280, 720], [1920, 1080], [4000, 3000]],
               sources=[2, 8], iterations=[6, 12], radius=7, stride=2, views_per_size=9, runs=2, tune_repeats=1)
SERVING = dict(name="serving_poisson", sizes=[[640, 480], [1920, 1080], [4000, 3000]], sources=[2, 8],
               iterations=[4, 12], radius=7, stride=2, requests=480, rate_per_s=10.0, views_per_size=9,
               mem_fraction=0.8, passes_per_step=32, policy=1, step_budget_mpix=1200.0)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["engine", "reference"], default="engine")
    ap.add_argument("--precision", choices=["f32", "f16acc"], default="f32",
                    help="headline arithmetic; the other is measured too and reported under 'variants'")
    ap.add_argument("--e2e-steps", type=int, default=None, help="end-to-end steps (default: --steps)")
    ap.add_argument("--cpu-rows", type=int, default=1080, help="rows of the CPU-baseline sample (1080: all of view 0)")
    ap.add_argument("--tile-h", type=int, default=0, choices=[0, 4, 8],
                    help="FP16-acc tile height of the headline solve (0: engine default)")
    ap.add_argument("--staging", type=int, default=0, choices=[0, 4, 8],
                    help="FP16-acc quad loads in flight per window row (0: engine default)")
    ap.add_argument("--count-taps", action="store_true",
                    help="with HP_ENGINE_LIB set to the instrumented engine (make -C <pkg> count): taps sampled per "
                         "pixel visit of the propagate half-passes, views 0 and 10, 12 iterations, both precisions")
    ap.add_argument("--no-reference-params", action="store_true",
                    help="skip timing the engine at the reference kernels' parameters")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-variants", action="store_true")
    ap.add_argument("--views", type=int, default=WORKLOAD["views"], help="reduce for profiling captures only")
    ap.add_argument("--no-serving", action="store_true", help="skip the serving leg (N = 1 only)")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched-plan leg (N = 1 only)")
    ap.add_argument("--precision-form", action="store_true",
                    help="print only the config-3 throughput (32 x 3000x2000, S 8, r 7, 12 it., FP32 and FP16-acc)")
    ap.add_argument("--no-precision-form", action="store_true", help="skip the config-3 throughput leg (N = 1 only)")
    ap.add_argument("--serve-requests", type=int, default=SERVING["requests"])
    ap.add_argument("--serve-rate", type=float, default=SERVING["rate_per_s"], help="Poisson arrivals per second")
    ap.add_argument("--serve-passes", type=int, default=SERVING["passes_per_step"], help="server stages per step")
    ap.add_argument("--serve-only", action="store_true", help="run only the serving leg (N = 1)")
    ap.add_argument("--serve-split", type=int, default=0, help="server: one launch per stage offset")
    ap.add_argument("--serve-policy", type=int, default=SERVING["policy"], choices=[0, 1],
                    help="server step policy: 0 round robin, 1 oldest first within a work budget")
    ap.add_argument("--serve-budget", type=float, default=SERVING["step_budget_mpix"],
                    help="budget policy: work per step, 1e6 pixel x source stage units")
    ap.add_argument("--serve-seed", type=int, default=2024, help="arrival and request draw seed")
    ap.add_argument("--serve-range", type=int, nargs=2, default=None, metavar=("FIRST", "END"),
                    help="replay only requests [FIRST, END) of the drawn stream, arrivals shifted to start at 0")
    ap.add_argument("--serve-log", default=None,
                    help="write a memory/progress timeline, the failed requests and the server's errors here (JSON)")
    return ap.parse_args()


# ------------------------------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi sampling (200 ms) during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([c.strip() for c in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            self.proc.wait(timeout=5)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 5 + i and r[5 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


# ------------------------------------------------------------------------------------------------
def rank_job_keys(rank: int, n_views: int):
    """(RNG seed, view id) of each of a rank's jobs.  Views are independent, so under torchrun every rank
    solves its own batch: the same scene, keyed differently, so no two ranks compute the same streams."""
    return [(42 + 1_000_003 * rank, r + 1000 * rank) for r in range(n_views)]


def max_over_ranks(x: float, dist, device) -> float:
    """The largest value over all ranks (device time of a step); x itself when running alone."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world: int, units_per_rank: float, steps: int, max_ms: float) -> float:
    """Whole-job Mpix*iter/s: all ranks' units over the slowest rank's time."""
    return world * units_per_rank * steps / (max_ms / 1e3)


def scene_module(standalone: bool = False):
    """The scene generator.  standalone: loaded from its file with the renderer built under oracle/, without
    importing the engine package (the reference arm must not load the engine)."""
    if not standalone:
        return importlib.import_module(PKG + ".scene")
    os.environ["HP_SCENE_LIB"] = os.path.join(ROOT, "oracle", "libpmscene.so")
    spec = importlib.util.spec_from_file_location("hp_scene_standalone", os.path.join(ROOT, PKG, "scene.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules[spec.name] = mod
    spec.loader.exec_module(mod)
    return mod


def build_scene(views: int, standalone: bool = False):
    scene = scene_module(standalone)
    # The full 20-view arc is always rendered, so a reduced --views case keeps the workload's geometry.
    return scene.multi_object(n_views=max(views, WORKLOAD["views"]), n_refs=views)


def workload_config(world: int, n_views: int) -> dict:
    """The `config` object of both arms' lines."""
    H, W = WORKLOAD["height"], WORKLOAD["width"]
    return {"workload": WORKLOAD["name"], "views_per_gpu": n_views, "width": W, "height": H,
            "sources": WORKLOAD["sources"], "window": f"{2 * WORKLOAD['radius'] + 1}x{2 * WORKLOAD['radius'] + 1}",
            "stride": WORKLOAD["stride"], "iterations": WORKLOAD["iterations"], "depth_range": WORKLOAD["depth_range"],
            "images": "u8", "parallelism": f"views/{world} ranks",
            "mpix_iter_per_step": round(n_views * H * W * WORKLOAD["iterations"] / 1e6 * world, 3),
            "l2": "inputs larger than L2 (20 x 2.07 Mpix images + 830 MB state per step), no flush"}


# Workloads the reference's own kernels can run (radius <= 5, no stride), timed on the same B200 by both arms:
# the engine arm through hp_solve ("reference_params"), the reference arm through oracle/_ref ("reference_gpu").
REF_PARAM_WORKLOADS = [
    dict(name="plane_sphere_5x640x480_r5_s1_it8", scene="plane_sphere", refs=[0, 1, 2, 3, 4], radius=5, stride=1,
         iterations=8),
    dict(name="multi_object_1920x1080_r5_s1_it12_2views", scene="multi_object", refs=[4, 13], radius=5, stride=1,
         iterations=12),
]


def ref_param_scenes(scene_mod):
    return {"plane_sphere": scene_mod.plane_sphere(), "multi_object": scene_mod.multi_object()}


def cpu_sample(s, rows: int, reps: int = 1):
    """Time one red-black iteration of a band of `rows` rows of view 0 on all host threads.
    Returns (Mpix*iter/s, seconds, threads, sample description)."""
    import pm_oracle as po
    r = 0
    srcs = s.sources[r]
    cam = lambda i: (s.views[i].cam.K, s.views[i].cam.R, s.views[i].cam.t)
    v = po.View(s.views[r].image_f32, [s.views[i].image_f32 for i in srcs], radius=WORKLOAD["radius"],
                stride=WORKLOAD["stride"], ref_cam=cam(r), src_cams=[cam(i) for i in srcs])
    H, W = s.views[r].image.shape
    y0 = (H - rows) // 2
    dmin, dmax = WORKLOAD["depth_range"]
    d, n = v.init(dmin, dmax, 42, r)
    c = np.zeros((H, W), np.float32)
    v.cost_rows_f32(d, n, c, y0, y0 + rows)
    best = None
    for it in range(reps):
        t = time.perf_counter()
        v.propagate_rows(d, n, c, dmin, dmax, it, 0, 42, r, y0, y0 + rows)
        v.propagate_rows(d, n, c, dmin, dmax, it, 1, 42, r, y0, y0 + rows)
        dt = time.perf_counter() - t
        best = dt if best is None else min(best, dt)
    mpix = rows * W / 1e6
    return mpix / best, best, po.num_threads(), (f"1 red-black iteration (the first) of rows [{y0},{y0 + rows}) x {W} "
                                                 f"of view 0 (r=7, s=2, S=6), {po.num_threads()} threads")


def measure_peaks():
    """On-chip ceilings measured live (lib/libhppeaks.so)."""
    import ctypes as C
    path = os.path.join(ROOT, PKG, "lib", "libhppeaks.so")
    L = C.CDLL(path)
    out = {}
    for name, fn, args in [("tex_f32_fetch_per_s", "hpk_tex_fetch_rate", (0,)),
                           ("tex_f16_fetch_per_s", "hpk_tex_fetch_rate", (1,)),
                           ("smem_bytes_per_s", "hpk_smem_read_rate", ()), ("fma_per_s", "hpk_fma_rate", ())]:
        v = C.c_double()
        f = getattr(L, fn)
        f.restype = C.c_int
        rc = f(*args, C.byref(v))
        out[name] = v.value if rc == 0 else None
    return out


def load_executed_taps(kind: str):
    """Taps actually sampled per pixel visit of the propagate launch, from the committed measurement
    (profiles/executed_taps.json, made by --count-taps on the instrumented engine)."""
    p = os.path.join(ROOT, "profiles", "executed_taps.json")
    try:
        e = json.load(open(p)).get(kind) or {}
        v = e.get("executed_taps_per_pixel_visit")
        return None if v is None else round(float(v), 1)
    except (OSError, ValueError, TypeError):
        return None


def load_ncu_traffic(kind: str):
    """DRAM bytes per propagate launch from the committed ncu summary, scaled to this workload."""
    p = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    if not os.path.exists(p):
        return None
    try:
        d = json.load(open(p))
        e = d.get(kind)
        return None if e is None else float(e["dram_bytes_per_pixel_visit"])
    except (ValueError, KeyError, TypeError):
        return None


# ------------------------------------------------------------------------------------------------
def run_engine(args, rank, world, local_rank):
    import torch
    hp = importlib.import_module(PKG)
    torch.cuda.set_device(local_rank)
    s = build_scene(args.views)
    dist = None
    if world > 1:
        import torch.distributed as dist
    H, W = WORKLOAD["height"], WORKLOAD["width"]
    n_views = args.views
    units_per_step = n_views * H * W * WORKLOAD["iterations"] / 1e6  # Mpix*iter per rank
    e2e_steps = args.e2e_steps or args.steps

    ctx = hp.Context(local_rank)
    stream = torch.cuda.ExternalStream(ctx.stream_handle, device=local_rank)
    ids = [ctx.upload(v.image) for v in s.views]

    def make_jobs(id_list):
        jobs = []
        for r, (seed, view_id) in enumerate(rank_job_keys(rank, n_views)):
            srcs = s.sources[r]
            cam = lambda i: hp.make_camera(s.views[i].cam.K, s.views[i].cam.R, s.views[i].cam.t)
            jobs.append(hp.make_job(id_list[r], [id_list[i] for i in srcs], cam(r), [cam(i) for i in srcs],
                                    *WORKLOAD["depth_range"], seed=seed, view_id=view_id,
                                    iterations=WORKLOAD["iterations"]))
        return jobs

    jobs = make_jobs(ids)
    dev_maps = []
    for _ in range(n_views):
        d = torch.empty(H, W, device="cuda")
        n = torch.empty(H, W, 3, device="cuda")
        c = torch.empty(H, W, device="cuda")
        dev_maps.append(hp.maps_of(d, n, c))

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    def timed(precision, steps, warmup):
        f16 = precision == "f16acc"
        params = hp.default_params(radius=WORKLOAD["radius"], stride=WORKLOAD["stride"],
                                   precision=hp.PRECISION_F16ACC if f16 else hp.PRECISION_F32,
                                   tile_h=args.tile_h if f16 else 0, staging=args.staging if f16 else 0)
        for _ in range(warmup):
            ctx.solve(jobs, params, dev_maps)
        ctx.profile_reset()
        ctx.set_profiling(True)
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with ClockSampler(local_rank) as clk:
            e0.record(stream)
            for _ in range(steps):
                ctx.solve(jobs, params, dev_maps)
            e1.record(stream)
            e1.synchronize()
        barrier()
        ctx.set_profiling(False)
        ms = max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
        prof = ctx.profile()
        return ms, prof, clk.summary()

    head = args.precision
    other = "f16acc" if head == "f32" else "f32"
    ms, prof, clocks = timed(head, args.steps, args.warmup)
    variants = {}
    if not args.no_variants:
        ms2, prof2, clocks2 = timed(other, args.steps, max(1, args.warmup))
        variants[other] = {"value": job_throughput(world, units_per_step, args.steps, ms2),
                           "ms_per_step": ms2 / args.steps,
                           "propagate_ms_per_launch": prof2["propagate"]["device_ms"] / max(1, prof2["propagate"]["timed"]),
                           "clocks": clocks2}

    # ---- end to end through the public API with pinned host buffers
    pinned_imgs = [torch.from_numpy(v.image).pin_memory() for v in s.views]
    host_out = [(torch.empty(H, W).pin_memory(), torch.empty(H, W, 3).pin_memory(), torch.empty(H, W).pin_memory())
                for _ in range(n_views)]
    params = hp.default_params(radius=WORKLOAD["radius"], stride=WORKLOAD["stride"],
                               precision=hp.PRECISION_F16ACC if head == "f16acc" else hp.PRECISION_F32)

    def host_maps(t3):
        m = hp.Maps(hp.MEMORY_HOST, t3[0].data_ptr(), t3[1].data_ptr(), t3[2].data_ptr())
        m.arrays = t3
        return m

    outs_h = [host_maps(t) for t in host_out]

    def upload_pinned(t):
        import ctypes as C
        iid = C.c_int()
        st = hp.lib.hp_image_upload(ctx.handle, t.data_ptr(), hp.MEMORY_HOST, W, H, hp.DTYPE_U8, C.byref(iid))
        if st != 0:
            raise hp.HpError(st, "hp_image_upload")
        return iid.value

    def e2e_step():
        step_ids = [upload_pinned(t) for t in pinned_imgs]
        ctx.solve(make_jobs(step_ids), params, outs_h)
        for i in step_ids:
            ctx.release(i)

    e2e_step()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(e2e_steps):
        e2e_step()
    e1.record(stream)
    e1.synchronize()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), dist, "cuda")
    barrier()
    h2d = sum(int(t.numel()) for t in pinned_imgs)
    d2h = n_views * H * W * (4 + 12 + 4)

    if rank != 0:
        ctx.close()
        return None

    # ---- roofline of the dominant kernel (the propagate half-pass)
    prop_launches = prof["propagate"]["timed"]
    prop_ms = prof["propagate"]["device_ms"] / max(1, prop_launches)
    visits = n_views * H * W / 2  # pixel visits per half-pass launch
    S, N_w = WORKLOAD["sources"], ((2 * WORKLOAD["radius"]) // WORKLOAD["stride"] + 1) ** 2
    taps_per_visit = 6 * S * N_w  # 4 neighbour + 2 refinement candidates, S sources, N_w taps
    b_img = 2 if head == "f16acc" else 4
    # compulsory DRAM bytes per visit: own plane+cost read & write (40), neighbour planes (16),
    # reference and source images once per launch ((1+S) * 2 visits' worth of pixels * b_img)
    hbm_bytes_per_visit = 40 + 16 + 2 * (1 + S) * b_img
    peaks_meas = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else {}
    hbm_peak = peaks_meas.get("hbm_gbs")
    hbm_src = "measured" if hbm_peak else "fallback"
    hbm_peak = hbm_peak or 6650.0
    achieved_hbm = visits * hbm_bytes_per_visit / (prop_ms * 1e-3) / 1e9
    traffic_per_visit = load_ncu_traffic(head)
    onchip = measure_peaks()
    tex_peak = onchip.get("tex_f16_fetch_per_s" if head == "f16acc" else "tex_f32_fetch_per_s")
    fetch_rate = visits * taps_per_visit / (prop_ms * 1e-3)
    fma_peak = onchip.get("fma_per_s")

    value = job_throughput(world, units_per_step, args.steps, ms)
    smem_peak = onchip.get("smem_bytes_per_s")
    l1_bytes_per_tap = 5 * b_img  # 4 bilinear source texels + 1 reference value, stored element width
    executed = load_executed_taps(head)
    line = {
        "metric": METRIC,
        "value": round(value, 2),
        "unit": "Mpix*iter/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(ms / args.steps, 3),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f16acc" if head == "f16acc" else "f32",
        "data": "synthetic: seeded planes+spheres scene, renderer ground truth (no dataset)",
        "config": workload_config(world, n_views),
        "e2e": {"value": round(job_throughput(world, units_per_step, e2e_steps, e2e_ms), 2), "unit": "Mpix*iter/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h, "steps": e2e_steps},
        # The survey's reported figure for the dominant kernel: algorithmic on-chip gather bytes (4 bilinear
        # texels of the source + 1 reference value per tap, at the stored element width; taps counted as
        # 6 candidates x S sources x N_w window taps per pixel visit, with no skips) per CUDA-event launch
        # duration, against the shared-memory/L1 read bandwidth measured live on the same GPU.
        "roofline": {"bound": "l1", "achieved": round(fetch_rate * l1_bytes_per_tap / 1e9, 1),
                     "peak": None if not smem_peak else round(smem_peak / 1e9, 1), "unit": "GB/s",
                     "frac": None if not smem_peak else round(fetch_rate * l1_bytes_per_tap / smem_peak, 4),
                     "peak_source": "measured live (shared-memory streaming microbenchmark, lib/libhppeaks.so)",
                     "traffic": None if traffic_per_visit is None else round(traffic_per_visit * visits),
                     "traffic_note": "DRAM bytes per launch (ncu dram__bytes_read+write, scaled per pixel visit)",
                     "kernel": ("propagate16_kernel<7,2>" if head == "f16acc" else "propagate_kernel<7,2>")
                               + " (red-black half-pass)",
                     "ms_per_launch": round(prop_ms, 4), "launches_timed": prop_launches,
                     "algorithmic_bytes_per_launch": int(visits * taps_per_visit * l1_bytes_per_tap),
                     "algorithmic_taps_per_visit": taps_per_visit,
                     "executed_taps_per_visit": executed,
                     "executed_note": "taps actually sampled per pixel visit, counted by the instrumented engine "
                                      "(duplicate neighbour planes and wholly-outside sources skip theirs), from "
                                      "profiles/executed_taps.json"},
        "roofline_hbm": {"bound": "hbm", "achieved": round(achieved_hbm, 2), "peak": hbm_peak, "unit": "GB/s",
                         "frac": round(achieved_hbm / hbm_peak, 5), "peak_source": hbm_src + " (MEASURED_PEAKS.json)",
                         "traffic": None if traffic_per_visit is None else round(traffic_per_visit * visits),
                         "algorithmic_bytes_per_launch": int(visits * hbm_bytes_per_visit),
                         "note": "compulsory DRAM bytes per launch; HBM does not bind this kernel"},
        "roofline_tex": {"bound": "texture-filter fetches" if head == "f32" else
                         "bilinear taps (software sampler; the texture rate is the reference ceiling)", "achieved": round(fetch_rate / 1e9, 2),
                         "peak": None if tex_peak is None else round(tex_peak / 1e9, 2), "unit": "Gfetch/s",
                         "frac": None if not tex_peak else round(fetch_rate / tex_peak, 4),
                         "peak_source": "measured live (L1-resident bilinear fetch microbenchmark)",
                         "algorithmic_fetches_per_launch": int(visits * taps_per_visit)},
        "roofline_fp32": {"achieved_fma_equiv": None if fma_peak is None else round(fetch_rate * 14 / 1e12, 3),
                          "peak_fma": None if fma_peak is None else round(fma_peak / 1e12, 3), "unit": "TFMA/s",
                          "note": "~14 FMA-equivalent issue slots per tap on the FP32 path (28 ops)"},
        "onchip_peaks": onchip,
        "gpu_launches": int(sum(v["launches"] for v in prof.values())),
        "kernel_launches": {k: v["launches"] for k, v in prof.items()},
        "clocks": clocks,
        "variants": variants,
    }
    for name, var in variants.items():
        b_v = 2 if name == "f16acc" else 4
        rate_v = visits * taps_per_visit / (var["propagate_ms_per_launch"] * 1e-3)
        var["taps_per_s"] = rate_v
        if onchip.get("smem_bytes_per_s"):
            var["roofline"] = {"bound": "l1", "achieved": round(rate_v * 5 * b_v / 1e9, 1), "unit": "GB/s",
                               "frac": round(rate_v * 5 * b_v / onchip["smem_bytes_per_s"], 4),
                               "kernel": ("propagate16_kernel<7,2>" if name == "f16acc" else "propagate_kernel<7,2>"),
                               "ms_per_launch": round(var["propagate_ms_per_launch"], 4),
                               "executed_taps_per_visit": load_executed_taps(name)}
    rates = {head: value, **{k: v["value"] for k, v in variants.items()}}
    if "f16acc" in rates and "f32" in rates:
        line["f16acc_over_f32"] = round(rates["f16acc"] / rates["f32"], 3)
    line["fusion"] = run_fusion(hp, ctx, s, dev_maps, n_views, stream)
    if world == 1 and not args.no_reference_params:
        line["reference_params"] = run_reference_params(hp, ctx, stream)
    if world == 1 and not args.no_serving:
        line["serving"] = run_serving(args, hp, local_rank)
    if world == 1 and not args.no_batched:
        bctx = hp.Context(local_rank)
        try:
            line["batched"] = run_batched(args, hp, bctx)
        finally:
            bctx.close()
    if world == 1 and not args.no_precision_form:
        line["precision_form"] = run_precision_form(hp, local_rank)
    if hasattr(hp.lib, "hp_debug_check"):  # self-checking engine: failed range checks of every leg since serving's
        import ctypes as C
        a8, a4 = (C.c_int * 12)(), (C.c_int * 12)()
        rc = hp.lib.hp_debug_check(a8, a4)
        line["self_check"] = {"rc": rc, "th8": list(a8), "th4": list(a4)}
    # CPU baseline (rank 0, N = 1)
    if world == 1 and not args.no_cpu_baseline:
        rate, secs, thr, desc = cpu_sample(s, args.cpu_rows)
        line["cpu_baseline"] = {"value": round(rate, 4), "unit": "Mpix*iter/s", "cores": thr, "kind": "port",
                                "sample": desc, "seconds": round(secs, 2)}
    ctx.close()
    return line


def view_pools(hp, ctx, sizes, seed0):
    """Per size, a 9-view arc of the multi-object generator (its own seeded layout), uploaded once."""
    scene = importlib.import_module(PKG + ".scene")
    pools = {}
    for k, (w, h) in enumerate(sizes):
        if (w, h) in pools:
            continue
        sc = scene.multi_object(seed=seed0 + k, w=w, h=h, n_views=9, n_src=8, f=1500.0 * w / 1920.0, n_refs=1)
        ids = [ctx.upload(v.image) for v in sc.views]
        cams = [hp.make_camera(v.cam.K, v.cam.R, v.cam.t) for v in sc.views]
        pools[(w, h)] = (sc, ids, cams, w, h)
    return pools


def run_batched(args, hp, ctx):
    """Batched form: BATCHED["views"] reference views of sizes drawn from BATCHED["sizes"], 2-8 sources and
    6-12 iterations each, in one plan.  The autotuner times the per-pass graph and the persistent kernel at
    every resident-CTA count and keeps the fastest; the plan then replays as one CUDA graph.  Reported:
    Mpix*iter/s of the tuned plan (device-resident, median of the timed runs) for both precisions."""
    import torch
    scene = importlib.import_module(PKG + ".scene")
    rng = np.random.default_rng(4096)
    pools = view_pools(hp, ctx, BATCHED["sizes"], 51)
    jobs, shapes = [], []
    for i in range(BATCHED["views"]):
        w, h = BATCHED["sizes"][int(rng.integers(0, len(BATCHED["sizes"])))]
        sc, ids, cams, _, _ = pools[(w, h)]
        r = int(rng.integers(0, len(sc.views)))
        S = int(rng.integers(BATCHED["sources"][0], BATCHED["sources"][1] + 1))
        srcs = scene.nearest_sources([v.cam for v in sc.views], r, S)
        it = int(rng.integers(BATCHED["iterations"][0], BATCHED["iterations"][1] + 1))
        jobs.append(hp.make_job(ids[r], [ids[j] for j in srcs], cams[r], [cams[j] for j in srcs], *sc.depth_range,
                                seed=1000 + i, view_id=i, iterations=it))
        shapes.append((h, w))
    outs = [hp.maps_of(torch.empty(h, w, device="cuda"), torch.empty(h, w, 3, device="cuda"),
                       torch.empty(h, w, device="cuda")) for h, w in shapes]
    stream = torch.cuda.ExternalStream(ctx.stream_handle)
    res = {"workload": BATCHED["name"], "views": len(jobs),
           "sizes_drawn": {f"{w}x{h}": sum(1 for s in shapes if s == (h, w)) for w, h in BATCHED["sizes"]}}
    for prec in ("f32", "f16acc"):
        params = hp.default_params(radius=BATCHED["radius"], stride=BATCHED["stride"],
                                   precision=hp.PRECISION_F16ACC if prec == "f16acc" else hp.PRECISION_F32)
        with hp.Plan(ctx, jobs, params, outs) as plan:
            info = plan.tune(BATCHED["tune_repeats"])
            times = []
            for _ in range(BATCHED["runs"]):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                plan.launch()
                e1.record(stream)
                plan.wait()
                e1.synchronize()
                times.append(e0.elapsed_time(e1))
            ms = float(np.median(times))
            res[prec] = {"mpix_iter_per_s": round(info["pixel_iterations"] / 1e6 / (ms / 1e3), 1),
                         "ms_per_run": round(ms, 2), "mpix_iter_per_run": round(info["pixel_iterations"] / 1e6, 1),
                         "schedule": {1: "per_pass", 2: "persistent"}[info["schedule"]],
                         "ctas_per_sm": info["ctas_per_sm"], "tile": f"{64}x{info['tile_h']}",
                         "staging": info["staging"] if prec == "f16acc" else None,
                         "launches_per_run": info["launches_per_run"],
                         "tuned_ms": round(info["tuned_ms"], 2), "graph": bool(info["use_graph"]),
                         "state_gb": round(info["state_bytes"] / 1e9, 2)}
    res["f16acc_over_f32"] = round(res["f16acc"]["mpix_iter_per_s"] / res["f32"]["mpix_iter_per_s"], 3)
    return res


def run_fusion(hp, ctx, s, dev_maps, n_views, stream):
    """Depth-map fusion (hp_fuse_depth_maps) of the last timed solve's device maps: each view's MVS sources
    as its neighbours, confidence 1 - cost/2, gray colour, device arrays in and out.  One call = counting
    pass, scan, writing pass (and the host read of the total between them), timed with CUDA events on
    the engine's stream.  The maps are unfiltered solver output."""
    import ctypes as C
    import torch
    H, W = dev_maps[0].arrays[0].shape
    cams = [hp.make_camera(v.cam.K, v.cam.R, v.cam.t) for v in s.views[:n_views]]
    conf = [1 - m.arrays[2] / 2 for m in dev_maps]
    grays = [torch.from_numpy(v.image_f32).cuda() for v in s.views[:n_views]]
    keep, views = [], []
    for r in range(n_views):
        v = hp.FuseView()
        v.cam = cams[r]
        v.height, v.width = H, W
        v.depth, v.normal = dev_maps[r].arrays[0].data_ptr(), dev_maps[r].arrays[1].data_ptr()
        v.confidence, v.gray = conf[r].data_ptr(), grays[r].data_ptr()
        nb = np.array([i for i in s.sources[r] if i < n_views], np.int32)
        keep.append(nb)
        v.neighbors, v.num_neighbors = nb.ctypes.data_as(C.POINTER(C.c_int)), len(nb)
        views.append(v)
    prm = hp.fuse_params(memory=hp.MEMORY_DEVICE)
    out = hp.PointCloudC()
    out.memory = hp.MEMORY_DEVICE
    total = ctx.fuse_views(views, prm, out)
    arrs = [torch.empty((max(total, 1), 3), device="cuda") for _ in range(3)]
    out.positions, out.normals, out.colors = (a.data_ptr() for a in arrs)
    out.capacity = total
    ctx.fuse_views(views, prm, out)
    times = []
    for _ in range(3):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.fuse_views(views, prm, out)
        e1.record(stream)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
    ms = float(np.median(times))
    mpix = n_views * H * W / 1e6
    return {"workload": f"{n_views} views {W}x{H}, {len(keep[0])} neighbours each", "ms": round(ms, 3),
            "mpix_per_s": round(mpix / (ms / 1e3), 1), "points": int(total), "params": "defaults"}


def run_serving(args, hp, device: int):
    """Serving form: requests of sizes drawn from SERVING["sizes"] (2-8 sources, 4-12 iterations, FP16-acc,
    r 7, s 2) arrive as a Poisson stream; images stay resident on the device (uploaded once per view pool), the
    server admits requests by free HBM (<= 80% of the device) and batches all admitted ones into its persistent
    launches.  Latency is submit -> completion; throughput is completed Mpix*iter over the span from the first
    submission to the last completion."""
    import torch
    scene = importlib.import_module(PKG + ".scene")
    rng = np.random.default_rng(args.serve_seed)
    ctx = hp.Context(device)
    pools = []
    for k, (w, h) in enumerate(SERVING["sizes"]):
        sc = scene.multi_object(seed=31 + k, w=w, h=h, n_views=SERVING["views_per_size"], n_src=8,
                                f=1500.0 * w / 1920.0, n_refs=1)
        ids = [ctx.upload(v.image) for v in sc.views]
        cams = [hp.make_camera(v.cam.K, v.cam.R, v.cam.t) for v in sc.views]
        pools.append((sc, ids, cams, w, h))
    reqs = []
    t = 0.0
    n_draw = max(args.serve_requests, args.serve_range[1]) if args.serve_range else args.serve_requests
    for i in range(n_draw):
        t += rng.exponential(1.0 / args.serve_rate)
        sc, ids, cams, w, h = pools[int(rng.integers(0, len(pools)))]
        r = int(rng.integers(0, len(sc.views)))
        S = int(rng.integers(SERVING["sources"][0], SERVING["sources"][1] + 1))
        srcs = scene.nearest_sources([v.cam for v in sc.views], r, S)
        it = int(rng.integers(SERVING["iterations"][0], SERVING["iterations"][1] + 1))
        job = hp.make_job(ids[r], [ids[j] for j in srcs], cams[r], [cams[j] for j in srcs], *sc.depth_range,
                          seed=7 + i, view_id=r, iterations=it)
        reqs.append((t, job, w, h, w * h * it))
    if args.serve_range:
        first, end = args.serve_range
        t0_arr = reqs[first][0] - (reqs[first][0] - reqs[first - 1][0] if first > 0 else 0.0)
        reqs = [(t - t0_arr, job, w, h, pi) for t, job, w, h, pi in reqs[first:end]]
    params = hp.default_params(radius=SERVING["radius"], stride=SERVING["stride"], precision=hp.PRECISION_F16ACC)
    srv = hp.Server(ctx, params, mem_fraction=SERVING["mem_fraction"], passes_per_step=args.serve_passes,
                    split_launches=args.serve_split, policy=args.serve_policy,
                    step_budget_mpix=args.serve_budget)
    # Warm-up: one request of each size, not counted.
    for sc, ids, cams, w, h in pools:
        m = hp.maps_of(torch.empty(h, w, device="cuda"), torch.empty(h, w, 3, device="cuda"),
                       torch.empty(h, w, device="cuda"))
        srv.submit(hp.make_job(ids[0], [ids[1], ids[2]], cams[0], [cams[1], cams[2]], *sc.depth_range,
                               iterations=2), m)
    srv.drain(timeout_ms=120000)
    srv.poll(capacity=16)
    srv.reset_stats()
    done = []
    first_failure = None

    def producer():
        # The server keeps each request's maps alive until its completion is polled.
        t0 = time.perf_counter()
        for t_arr, job, w, h, _ in reqs:
            dt = t_arr - (time.perf_counter() - t0)
            if dt > 0:
                time.sleep(dt)
            srv.submit(job, hp.maps_of(torch.empty(h, w, device="cuda"), torch.empty(h, w, 3, device="cuda"),
                                       torch.empty(h, w, device="cuda")))

    t_start = time.perf_counter()
    th = threading.Thread(target=producer)
    th.start()
    deadline = t_start + reqs[-1][0] + 600
    timeline, failures, t_next = [], [], 0.0
    while len(done) < len(reqs) and time.perf_counter() < deadline:
        for c in srv.poll(timeout_ms=100):
            c["done_s"] = round(time.perf_counter() - t_start, 3)
            done.append(c)
            c["index"] = c["request_id"] - (len(pools) + 1) + (args.serve_range[0] if args.serve_range else 0)
            if c["status"] != 0:
                if first_failure is None:
                    first_failure = {"at_s": c["done_s"], "status": c["status"], "server_error": srv.first_error()}
                if len(failures) < 64:
                    failures.append(c)
        if args.serve_log and time.perf_counter() - t_start >= t_next:
            t_next += 2.0
            st_now = srv.stats()
            timeline.append({"t": round(time.perf_counter() - t_start, 1), "done": len(done),
                             **{k: st_now[k] for k in ("completed", "failed", "active", "queued", "state_bytes",
                                                       "pool_reserved_bytes", "device_free_bytes", "budget_bytes",
                                                       "steps", "failed_steps")},
                             "torch_reserved": torch.cuda.memory_reserved()})
    wall = time.perf_counter() - t_start
    first_error, last_error = srv.first_error(), srv.last_error()
    th.join()
    st = srv.stats()
    srv.close()
    ctx.close()
    ok = [c for c in done if c["status"] == 0]
    statuses = {}
    for c in done:
        if c["status"] != 0:
            statuses[str(c["status"])] = statuses.get(str(c["status"]), 0) + 1
    check = None
    if hasattr(hp.lib, "hp_debug_check"):  # self-checking engine: the first failed range check, if any
        import ctypes as C
        a8, a4 = (C.c_int * 12)(), (C.c_int * 12)()
        rc = hp.lib.hp_debug_check(a8, a4)
        check = {"rc": rc, "th8": list(a8), "th4": list(a4)}
    if args.serve_log:
        with open(args.serve_log, "w") as f:
            json.dump({"first_error": first_error, "last_error": last_error, "first_failure": first_failure,
                       "failures": failures, "self_check": check, "timeline": timeline,
                       "first_request": args.serve_range[0] if args.serve_range else 0}, f)
    lat = np.array([c["latency_ms"] for c in ok]) if ok else np.zeros(1)
    pix_iter = sum(r[4] for r in reqs) / 1e6
    offered = pix_iter / reqs[-1][0]
    return {
        "workload": SERVING["name"], "requests": len(reqs), "completed": len(ok), "failed": len(done) - len(ok),
        "failed_by_status": statuses, "failed_steps": st["failed_steps"], "first_failure": first_failure,
        **({"self_check": check} if check is not None else {}),
        "rate_per_s": args.serve_rate, "offered_mpix_iter_per_s": round(offered, 1),
        "p50_ms": round(float(np.percentile(lat, 50)), 1), "p90_ms": round(float(np.percentile(lat, 90)), 1),
        "p99_ms": round(float(np.percentile(lat, 99)), 1),
        "mean_ms": round(float(lat.mean()), 1), "max_ms": round(float(lat.max()), 1),
        "queue_p50_ms": round(float(np.percentile([c["queue_ms"] for c in ok], 50)), 1) if ok else None,
        "mpix_iter_per_s": round(st["pixel_iterations"] / 1e6 / wall, 1),
        "device_mpix_iter_per_s": round(st["pixel_iterations"] / 1e6 / (st["device_ms"] / 1e3), 1)
        if st["device_ms"] else None,
        "device_busy_frac": round(st["device_ms"] / 1e3 / wall, 3), "wall_s": round(wall, 1),
        "peak_active": st["peak_active"], "steps": st["steps"], "launches": st["launches"],
        "passes_per_step": args.serve_passes,
        "policy": {0: "round_robin", 1: "budget"}[args.serve_policy],
        "step_budget_mpix": args.serve_budget if args.serve_policy == 1 else None,
        "seed": args.serve_seed,
        "peak_state_gb": round(st["peak_state_bytes"] / 1e9, 2),
        "config": {"sizes": SERVING["sizes"], "sources": SERVING["sources"], "iterations": SERVING["iterations"],
                   "window": "15x15", "stride": SERVING["stride"], "precision": "f16acc",
                   "admission": "state <= 80% of device memory", "images": "resident, u8 uploads, 9 views per size",
                   "arrivals": f"Poisson, {args.serve_rate}/s, {len(reqs)} requests"},
    }


def run_count_taps(args):
    """Executed taps: the instrumented engine counts, per sampled (candidate, source), its window's taps
    (wholly-outside sources and duplicate neighbour planes are skipped, as in the timed kernels).  Views 0 and
    10 of the headline workload are solved pass by pass (hp_propagate_pass), so only the half-passes count."""
    import ctypes as C
    hp = importlib.import_module(PKG)
    L = C.CDLL(hp.LIB_PATH)
    if not hasattr(L, "hp_debug_taps"):
        raise SystemExit("--count-taps needs HP_ENGINE_LIB=<pkg>/lib/libhpmvs_count.so (make -C <pkg> count)")
    f32c, f16c = C.c_ulonglong(), C.c_ulonglong()
    s = build_scene(WORKLOAD["views"])
    out = {}
    refs = [0, 10]
    with hp.Context(0) as ctx:
        ids = [ctx.upload(v.image) for v in s.views]
        cam = lambda i: hp.make_camera(s.views[i].cam.K, s.views[i].cam.R, s.views[i].cam.t)
        for name, prec in (("f32", hp.PRECISION_F32), ("f16acc", hp.PRECISION_F16ACC)):
            per_it = np.zeros(WORKLOAD["iterations"])
            for r in refs:
                job = hp.make_job(ids[r], [ids[i] for i in s.sources[r]], cam(r), [cam(i) for i in s.sources[r]],
                                  *WORKLOAD["depth_range"], seed=42, view_id=r, iterations=WORKLOAD["iterations"])
                p = hp.default_params(radius=WORKLOAD["radius"], stride=WORKLOAD["stride"], precision=prec)
                m, _, _, _ = hp.host_maps(s.height, s.width)
                ctx.init_hypotheses(job, p, m)
                ctx.ncc_cost(job, p, m)
                L.hp_debug_taps(C.byref(f32c), C.byref(f16c))
                for it in range(WORKLOAD["iterations"]):
                    for color in (0, 1):
                        ctx.propagate_pass(job, p, m, it, color)
                    L.hp_debug_taps(C.byref(f32c), C.byref(f16c))
                    per_it[it] += (f32c if name == "f32" else f16c).value
            visits_per_it = len(refs) * s.height * s.width  # two half-passes of W * H / 2 visits per view
            out[name] = {"executed_taps_per_pixel_visit": round(float(per_it.sum() / (visits_per_it * len(per_it))), 1),
                         "per_iteration": [round(float(x / visits_per_it), 1) for x in per_it],
                         "algorithmic_taps_per_pixel_visit": 6 * WORKLOAD["sources"] * 64, "views": refs}
    return out


def run_reference_params(hp, ctx, stream):
    """The engine at the parameters the reference's own kernels support (REF_PARAM_WORKLOADS: radius 5, stride 1),
    per view as the reference solves (one hp_solve per view), FP32 and FP16-acc, device-resident maps, CUDA
    events on the engine's stream.  The reference arm times the reference's kernels on the same workloads."""
    import torch
    scenes = ref_param_scenes(importlib.import_module(PKG + ".scene"))
    out = {}
    for wl in REF_PARAM_WORKLOADS:
        sc = scenes[wl["scene"]]
        ids = [ctx.upload(v.image) for v in sc.views]
        cam = lambda i: hp.make_camera(sc.views[i].cam.K, sc.views[i].cam.R, sc.views[i].cam.t)
        H, W = sc.height, sc.width
        maps = hp.maps_of(torch.empty(H, W, device="cuda"), torch.empty(H, W, 3, device="cuda"),
                          torch.empty(H, W, device="cuda"))
        res = {"views": len(wl["refs"]), "width": W, "height": H, "sources": len(sc.sources[wl["refs"][0]]),
               "radius": wl["radius"], "stride": wl["stride"], "iterations": wl["iterations"]}
        for prec, pk in (("f32", hp.PRECISION_F32), ("f16acc", hp.PRECISION_F16ACC)):
            params = hp.default_params(radius=wl["radius"], stride=wl["stride"], precision=pk)
            total = 0.0
            for r in wl["refs"]:
                job = hp.make_job(ids[r], [ids[i] for i in sc.sources[r]], cam(r), [cam(i) for i in sc.sources[r]],
                                  *sc.depth_range, seed=42 + 1_000_000 * r, view_id=r, iterations=wl["iterations"])
                ctx.solve([job], params, [maps])  # warm-up
                best = None
                for _ in range(3):
                    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    e0.record(stream)
                    ctx.solve([job], params, [maps])
                    e1.record(stream)
                    e1.synchronize()
                    t = e0.elapsed_time(e1)
                    best = t if best is None else min(best, t)
                total += best
            res[prec] = {"ms": round(total, 3),
                         "mpix_iter_per_s": round(len(wl["refs"]) * H * W * wl["iterations"] / 1e6 / (total / 1e3), 1)}
        for i in ids:
            ctx.release(i)
        out[wl["name"]] = res
    return out


def run_precision_form(hp, device: int):
    """Config 3 throughput (the precision form's workload): 32 views at 3000x2000 stored FP16 in [0, 1] with
    N(0, 0.01) noise, fx 2400, the 8 nearest sources each, r 7, 12 iterations, every view a reference - 2304
    Mpix*iter per solve.  One hp_solve over all 32 views with device-resident maps, FP32 and FP16-acc, at
    stride 2 (warm-up, then the best of 2) and stride 1 (one timed solve after the stride-2 runs), CUDA events on
    the engine's stream."""
    import torch
    scene = importlib.import_module(PKG + ".scene")
    s = scene.precision(n_refs=0)
    n = len(s.views)
    srcs = [scene.nearest_sources([v.cam for v in s.views], r, 8) for r in range(n)]
    ctx = hp.Context(device)
    try:
        stream = torch.cuda.ExternalStream(ctx.stream_handle)
        ids = [ctx.upload(v.image) for v in s.views]
        cam = lambda i: hp.make_camera(s.views[i].cam.K, s.views[i].cam.R, s.views[i].cam.t)
        jobs = [hp.make_job(ids[r], [ids[i] for i in srcs[r]], cam(r), [cam(i) for i in srcs[r]], *s.depth_range,
                            seed=42 + r, view_id=r, iterations=12) for r in range(n)]
        H, W = s.height, s.width
        maps = [hp.maps_of(torch.empty(H, W, device="cuda"), torch.empty(H, W, 3, device="cuda"),
                           torch.empty(H, W, device="cuda")) for _ in range(n)]
        units = n * H * W * 12 / 1e6
        out = {"workload": f"precision_form_{n}x{W}x{H}", "views": n, "sources": 8, "radius": 7, "iterations": 12,
               "images": "f16 + N(0, 0.01)", "mpix_iter_per_solve": round(units, 1)}

        def timed(params, reps):
            best = None
            for _ in range(reps):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                ctx.solve(jobs, params, maps)
                e1.record(stream)
                e1.synchronize()
                t = e0.elapsed_time(e1)
                best = t if best is None else min(best, t)
            return best

        for stride in (2, 1):
            rates = {}
            for prec, pk in (("f32", hp.PRECISION_F32), ("f16acc", hp.PRECISION_F16ACC)):
                params = hp.default_params(radius=7, stride=stride, precision=pk)
                if stride == 2:
                    ctx.solve(jobs, params, maps)  # warm-up
                ms = timed(params, 2 if stride == 2 else 1)
                rates[prec] = {"ms": round(ms, 1), "mpix_iter_per_s": round(units / (ms / 1e3), 1)}
            rates["f16acc_over_f32"] = round(rates["f16acc"]["mpix_iter_per_s"] / rates["f32"]["mpix_iter_per_s"], 3)
            out[f"stride{stride}"] = rates
        return out
    finally:
        ctx.close()


def run_reference_gpu(scene_mod):
    """The reference's own kernels (oracle/_ref/libpmref.so: patchmatch_mvs.cu compiled unmodified) on
    REF_PARAM_WORKLOADS, on this box's GPU: pmref.solve_view = init, initial cost and the red-black passes
    of runPatchMatchMVS (:1094-1107, :1189-1232) with its per-launch device synchronisations, timed by CUDA
    events from the init launch to the last pass; best of 3 per view."""
    import pmref
    if not pmref.available():
        return {"unavailable": "oracle/_ref/libpmref.so not built (needs the reference tree at build time)"}
    try:
        import torch
        if not torch.cuda.is_available():
            return {"unavailable": "no GPU"}
    except ImportError:
        return {"unavailable": "torch missing"}
    scenes = ref_param_scenes(scene_mod)
    out = {}
    for wl in REF_PARAM_WORKLOADS:
        sc = scenes[wl["scene"]]
        cam = lambda i: (sc.views[i].cam.K, sc.views[i].cam.R, sc.views[i].cam.t)
        total = 0.0
        for r in wl["refs"]:
            srcs = sc.sources[r]
            kinv, ab = pmref.setup_views(cam(r), [cam(i) for i in srcs])
            args = (sc.views[r].image_f32, [sc.views[i].image_f32 for i in srcs], kinv, ab, *sc.depth_range,
                    wl["radius"], wl["iterations"], r)
            pmref.solve_view(*args)  # warm-up
            total += min(pmref.solve_view(*args)[3] for _ in range(3))
        out[wl["name"]] = {"views": len(wl["refs"]), "width": sc.width, "height": sc.height,
                           "sources": len(sc.sources[wl["refs"][0]]), "radius": wl["radius"], "stride": wl["stride"],
                           "iterations": wl["iterations"], "ms": round(total, 3),
                           "mpix_iter_per_s": round(len(wl["refs"]) * sc.width * sc.height * wl["iterations"] / 1e6
                                                    / (total / 1e3), 1)}
    return out


def run_reference(args, rank, world):
    """The reference's algorithm on the host cores (CPU restatement, all threads), and - where the reference's
    kernels were compiled - those kernels on the GPU at the parameters they support.  Nothing of the engine is
    loaded: the scene comes from the renderer built under oracle/."""
    if rank != 0:
        return None
    scene_mod = scene_module(standalone=True)
    s = scene_mod.multi_object(n_views=WORKLOAD["views"], n_refs=1)
    rates = []
    desc = thr = None
    for i in range(args.warmup + args.steps):
        rate, secs, thr, desc = cpu_sample(s, args.cpu_rows)
        if i >= args.warmup:
            rates.append(rate)
    v = float(np.median(rates))
    sample_mpix = args.cpu_rows * WORKLOAD["width"] / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": round(v, 4), "unit": "Mpix*iter/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(sample_mpix / v * 1e3, 1),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic: seeded planes+spheres scene, renderer ground truth (no dataset)",
        "config": workload_config(world, WORKLOAD["views"]),
        "cpu_baseline": {"value": round(v, 4), "unit": "Mpix*iter/s", "cores": thr, "kind": "port", "sample": desc},
        "e2e": {"value": round(v, 4), "unit": "Mpix*iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if not args.no_reference_params:
        line["reference_gpu"] = run_reference_gpu(scene_mod)
    return line


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if world != args.gpus:
        print(f"warning: --gpus {args.gpus} but WORLD_SIZE {world}", file=sys.stderr)
    if args.count_taps:
        print(json.dumps({"executed_taps": run_count_taps(args)}))
        return
    if args.precision_form:
        hp = importlib.import_module(PKG)
        print(json.dumps({"precision_form": run_precision_form(hp, local_rank)}))
        return
    if args.serve_only:
        hp = importlib.import_module(PKG)
        print(json.dumps({"serving": run_serving(args, hp, local_rank)}))
        return
    if args.impl == "reference":
        line = run_reference(args, rank, world)
        if line:
            print(json.dumps(line))
        return
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180))
    try:
        line = run_engine(args, rank, world, local_rank)
        if line:
            print(json.dumps(line))
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
