"""The self-checking engine (``make check``, lib/libhpmvs_check.so): its FP16 stages range-check every
data-derived quad load, neighbour read, claimed ticket and view state pointer, record the first failed
check and skip that access instead of making it.  Solves at both tile heights, a persistent plan and a
server, on a wide camera arc where near edge-on plane hypotheses occur, must record no failed check.

The library runs in a child process (HP_ENGINE_LIB selects it), so this process keeps the shipped engine.
The check that found the corner test's conditioning fault (an x = -1 quad load from the unchecked form
on a near edge-on plane) ran through the same build."""
from __future__ import annotations

import json
import os
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CHECK_LIB = os.path.join(ROOT, "hemiphoto3d-private_b200", "lib", "libhpmvs_check.so")

SCRIPT = r"""
import ctypes as C, importlib, json, sys
sys.path.insert(0, ROOT)
hp = importlib.import_module("hemiphoto3d-private_b200")
scene = importlib.import_module("hemiphoto3d-private_b200.scene")
assert hasattr(hp.lib, "hp_debug_check"), "not the self-checking engine"
s = scene.multi_object(seed=5, w=640, h=480, n_views=9, n_src=8, f=500.0, n_refs=9)
cam = lambda i: hp.make_camera(s.views[i].cam.K, s.views[i].cam.R, s.views[i].cam.t)
with hp.Context(0) as ctx:
    ids = [ctx.upload(v.image) for v in s.views]
    jobs = [hp.make_job(ids[r], [ids[i] for i in s.sources[r]], cam(r), [cam(i) for i in s.sources[r]],
                        *s.depth_range, seed=100 + r, view_id=r, iterations=6) for r in range(9)]
    for tile_h in (8, 4):
        params = hp.default_params(radius=7, stride=2, precision=hp.PRECISION_F16ACC, tile_h=tile_h)
        ctx.solve(jobs, params, [hp.host_maps(s.height, s.width)[0] for _ in jobs])
    params = hp.default_params(radius=7, stride=2, precision=hp.PRECISION_F16ACC)
    outs = [hp.host_maps(s.height, s.width)[0] for _ in jobs]
    with hp.Plan(ctx, jobs, params, outs, hp.plan_options(schedule=hp.SCHEDULE_PERSISTENT)) as plan:
        plan.run()
    with hp.Server(ctx, params, passes_per_step=4, policy=1) as srv:
        for j in jobs:
            srv.submit(j, hp.host_maps(s.height, s.width)[0])
        srv.drain(timeout_ms=120000)
        done = srv.poll(capacity=64)
    assert len(done) == len(jobs) and all(c["status"] == 0 for c in done), done
a8, a4 = (C.c_int * 12)(), (C.c_int * 12)()
rc = hp.lib.hp_debug_check(a8, a4)
print(json.dumps({"rc": rc, "th8": list(a8), "th4": list(a4)}))
"""


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(CHECK_LIB), reason="self-checking engine not built (make -C <pkg> check)")
def test_self_checked_fp16_paths_record_no_out_of_range_access():
    env = dict(os.environ, HP_ENGINE_LIB=CHECK_LIB)
    out = subprocess.run([sys.executable, "-c", SCRIPT.replace("ROOT", repr(ROOT))], env=env, capture_output=True,
                         text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    rec = json.loads(out.stdout.strip().splitlines()[-1])
    assert rec["rc"] == 0
    # hits, kind, six integers, four floats (as bits): hits 0 = no failed check
    assert rec["th8"][0] == 0, f"64x8 kernels: failed range check {rec['th8']}"
    assert rec["th4"][0] == 0, f"64x4 kernels: failed range check {rec['th4']}"


SHORTCUTS = r"""
import hashlib, importlib, json, sys
sys.path.insert(0, ROOT)
hp = importlib.import_module("hemiphoto3d-private_b200")
scene = importlib.import_module("hemiphoto3d-private_b200.scene")
s = scene.multi_object(seed=5, w=320, h=240, n_views=7, n_src=6, f=250.0, n_refs=7)
cam = lambda i: hp.make_camera(s.views[i].cam.K, s.views[i].cam.R, s.views[i].cam.t)
out = {}
with hp.Context(0) as ctx:
    ids = [ctx.upload(v.image) for v in s.views]
    jobs = [hp.make_job(ids[r], [ids[i] for i in s.sources[r]], cam(r), [cam(i) for i in s.sources[r]],
                        *s.depth_range, seed=40 + r, view_id=r, iterations=4) for r in range(len(s.views))]
    for radius, stride in ((7, 2), (3, 1)):
        for tile_h in (8, 4):
            for checked in (0, 1):
                params = hp.default_params(radius=radius, stride=stride, precision=hp.PRECISION_F16ACC,
                                           tile_h=tile_h, debug_checked_taps=checked)
                maps = [hp.host_maps(s.height, s.width) for _ in jobs]
                ctx.solve(jobs, params, [m[0] for m in maps])
                h = hashlib.sha1()
                for m in maps:
                    for a in m[1:]:
                        h.update(a.tobytes())
                out[f"r{radius}s{stride}t{tile_h}c{checked}"] = h.hexdigest()
print(json.dumps(out))
"""


@pytest.mark.gpu
@pytest.mark.skipif(not os.path.exists(CHECK_LIB), reason="self-checking engine not built (make -C <pkg> check)")
def test_fp16_corner_shortcuts_change_no_bit():
    """The FP16 cost skips the per-tap bounds checks of windows the corner test proves inside, and skips
    sources it proves wholly outside.  With both shortcuts off (debug_checked_taps, a switch of the
    self-checking build: every window through the checked form, every source sampled) whole solves on a wide
    arc come out bit-identical, for two windows and both tile heights."""
    env = dict(os.environ, HP_ENGINE_LIB=CHECK_LIB)
    out = subprocess.run([sys.executable, "-c", SHORTCUTS.replace("ROOT", repr(ROOT))], env=env,
                         capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    h = json.loads(out.stdout.strip().splitlines()[-1])
    for key in [k for k in h if k.endswith("c0")]:
        assert h[key] == h[key[:-1] + "1"], key


@pytest.mark.gpu
def test_shipped_engine_refuses_the_checked_taps_switch(hp):
    """debug_checked_taps exists only in the self-checking build; the shipped engine refuses it."""
    if hasattr(hp.lib, "hp_debug_check"):
        pytest.skip("this process runs the self-checking engine")
    import importlib
    scene = importlib.import_module("hemiphoto3d-private_b200.scene")
    s = scene.plane_sphere(w=160, h=120)
    cam = lambda i: hp.make_camera(s.views[i].cam.K, s.views[i].cam.R, s.views[i].cam.t)
    with hp.Context(0) as ctx:
        ids = [ctx.upload(v.image) for v in s.views]
        job = hp.make_job(ids[0], [ids[i] for i in s.sources[0]], cam(0), [cam(i) for i in s.sources[0]],
                          *s.depth_range, iterations=1)
        params = hp.default_params(precision=hp.PRECISION_F16ACC, debug_checked_taps=1)
        with pytest.raises(hp.HpError) as ei:
            ctx.solve([job], params, [hp.host_maps(s.height, s.width)[0]])
        assert ei.value.status == 6  # HP_ERR_UNSUPPORTED
