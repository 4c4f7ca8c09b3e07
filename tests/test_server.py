"""The continuous-batching server (hp_server, include/hpmvs.h).

CPU: its admission and step-composition policy (hp_server_simulate) - strict
arrival order, slots and byte budget never exceeded, every admitted request
advancing every step, late arrivals joining running work.
GPU: requests of different sizes, source counts and iteration counts, submitted
while others run, each equal bit for bit to hp_solve of the same job alone
(tolerance 0: the per-pixel arithmetic does not depend on batching)."""
from __future__ import annotations

import math
import time

import numpy as np
import pytest

from conftest import cam_of


def _occupancy(adm, fin, bytes_, ticks):
    active = np.zeros(ticks, int)
    held = np.zeros(ticks, np.int64)
    for a, f, b in zip(adm, fin, bytes_):
        active[a:f + 1] += 1
        held[a:f + 1] += b
    return active, held


def test_simulated_policy_respects_slots_budget_and_order(hp):
    rng = np.random.default_rng(3)
    for trial in range(30):
        n = int(rng.integers(1, 40))
        arrive = np.sort(rng.integers(0, 30, n))
        bytes_ = rng.integers(1, 100, n)
        stages = 2 * rng.integers(0, 13, n) + 2
        slots = int(rng.integers(1, 9))
        budget = int(rng.integers(int(bytes_.max()), 400))
        passes = int(rng.integers(1, 6))
        adm, fin, steps = hp.server_simulate(arrive.tolist(), bytes_.tolist(), stages.tolist(), slots, budget, passes)
        assert (adm >= arrive).all()
        assert (np.diff(adm) >= 0).all(), "admission is in arrival order"
        # Admitted requests advance every step: finished ceil(stages / passes) - 1 steps after admission.
        assert (fin - adm == np.ceil(stages / passes).astype(int) - 1).all()
        active, held = _occupancy(adm, fin, bytes_, int(fin.max()) + 1)
        assert active.max() <= slots and held.max() <= budget
        assert steps == int((active > 0).sum())


def test_late_arrival_joins_running_work(hp):
    # A long request runs; a short one arriving two steps later is admitted at once and overtakes it.
    adm, fin, _ = hp.server_simulate([0, 2], [10, 10], [2 * 12 + 2, 2 * 2 + 2], 4, 100, 2)
    assert adm.tolist() == [0, 2]
    assert fin[1] < fin[0]
    # The same two with room for one: the short one waits for the long one (a queue alone).
    adm, fin, _ = hp.server_simulate([0, 2], [10, 10], [26, 6], 1, 100, 2)
    assert adm[1] == fin[0] + 1


def test_budget_policy_serves_the_oldest_first_and_stalls_none(hp):
    """HP_SERVER_POLICY_BUDGET: in admission order each request takes as many stages (up to
    passes_per_step) as the step's work budget still covers, and at least one - so the oldest request
    finishes first when the budget covers it, and every admitted request still advances every step."""
    # Two requests of 26 stages, work 10 a stage, budget 100 a step, cap 16: the first takes 10 stages
    # a step (finishing in 3 steps), the second 1 a step until the first is done.
    adm, fin, steps = hp.server_simulate([0, 0], [1, 1], [26, 26], 4, 100, 16, policy=hp.SERVER_POLICY_BUDGET,
                                         work=[10.0, 10.0], step_work=100.0)
    assert adm.tolist() == [0, 0]
    assert fin[0] == 2  # stages 10 + 10 + 6
    assert fin[1] > fin[0]
    rng = np.random.default_rng(5)
    for trial in range(30):
        n = int(rng.integers(1, 40))
        arrive = np.sort(rng.integers(0, 30, n))
        bytes_ = rng.integers(1, 100, n)
        stages = 2 * rng.integers(0, 13, n) + 2
        work = rng.uniform(1, 50, n)
        slots = int(rng.integers(1, 9))
        budget = int(rng.integers(int(bytes_.max()), 400))
        passes = int(rng.integers(1, 20))
        adm, fin, steps = hp.server_simulate(arrive.tolist(), bytes_.tolist(), stages.tolist(), slots, budget, passes,
                                             policy=hp.SERVER_POLICY_BUDGET, work=work.tolist(),
                                             step_work=float(rng.uniform(0, 200)))
        assert (adm >= arrive).all() and (np.diff(adm) >= 0).all()
        # At least one stage and at most `passes` a step: ceil(stages / passes) - 1 <= fin - adm <= stages - 1.
        assert (fin - adm >= np.ceil(stages / passes).astype(int) - 1).all() and (fin - adm <= stages - 1).all()
        active, held = _occupancy(adm, fin, bytes_, int(fin.max()) + 1)
        assert active.max() <= slots and held.max() <= budget
    with pytest.raises(hp.HpError):
        hp.server_simulate([0], [1], [4], 1, 10, 2, policy=7)


def test_budget_serialises_and_oversize_is_refused(hp):
    adm, fin, steps = hp.server_simulate([0, 0, 0], [60, 60, 60], [6, 6, 6], 8, 100, 3)
    assert adm.tolist() == [0, 2, 4] and fin.tolist() == [1, 3, 5] and steps == 6
    with pytest.raises(hp.HpError):
        hp.server_simulate([0], [101], [6], 8, 100, 3)


# ------------------------------------------------------------------------------------ GPU


@pytest.fixture(scope="module")
def scenes(scene_mod):
    return {"s": scene_mod.plane_sphere(w=160, h=120), "m": scene_mod.plane_sphere(seed=9, w=320, h=240)}


@pytest.fixture(scope="module")
def gctx(hp):
    with hp.Context(0) as c:
        yield c


@pytest.fixture(scope="module")
def ids(gctx, scenes):
    return {k: [gctx.upload(v.image) for v in s.views] for k, s in scenes.items()}


def _requests(hp, scenes, ids, n, seed):
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        key = "s" if k % 3 else "m"
        s = scenes[key]
        r = int(rng.integers(0, len(s.views)))
        others = [i for i in range(len(s.views)) if i != r]
        srcs = list(rng.choice(others, int(rng.integers(2, 5)), replace=False))
        it = int(rng.integers(1, 7))
        job = hp.make_job(ids[key][r], [ids[key][i] for i in srcs], hp.make_camera(*cam_of(s, r)),
                          [hp.make_camera(*cam_of(s, i)) for i in srcs], *s.depth_range, seed=100 + k, view_id=r,
                          iterations=it)
        out.append((job, s.height, s.width))
    return out


def _alone(hp, ctx, job, params, h, w):
    m, d, n, c = hp.host_maps(h, w)
    ctx.solve([job], params, [m])
    return d, n, c


def _request_bytes(h, w):
    a = lambda x: (x + 255) // 256 * 256
    tiles = math.ceil(w / 64) * math.ceil(h / 8)
    return a(a(h * w * 20) + tiles * 4)


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("split", [0, 1])
@pytest.mark.parametrize("policy", [0, 1])
def test_results_same_alone_and_in_the_mix(hp, gctx, scenes, ids, precision, split, policy):
    """Requests submitted in waves while earlier ones run; each result equals hp_solve alone, bit for bit,
    under either step policy (the budget here is small enough that requests take different stage counts)."""
    params = hp.default_params(radius=5, stride=2, precision=precision)
    reqs = _requests(hp, scenes, ids, 12, seed=precision * 10 + split)
    expect = [_alone(hp, gctx, j, params, h, w) for j, h, w in reqs]
    got = {}
    with hp.Server(gctx, params, max_active=6, passes_per_step=3, split_launches=split, policy=policy,
                   step_budget_mpix=0.5) as srv:
        rid = {}
        pending = list(enumerate(reqs))
        done = []
        deadline = time.time() + 120
        while pending or len(done) < len(reqs):
            assert time.time() < deadline, "server made no progress"

            for _ in range(min(len(pending), 4)):  # a wave of up to four arrivals
                k, (j, h, w) = pending.pop(0)
                m, d, n, c = hp.host_maps(h, w)
                rid[srv.submit(j, m)] = k
                got[k] = (d, n, c)
            done += srv.poll(timeout_ms=20 if pending else 2000)
        st = srv.stats()
    assert all(c["status"] == 0 for c in done) and len(done) == len(reqs)
    assert st["completed"] == len(reqs) and st["failed"] == 0
    assert st["peak_active"] > 1, "requests overlapped on the device"
    assert 0 < st["p50_ms"] <= st["p99_ms"] <= st["max_ms"]
    for k, (d, n, c) in got.items():
        ed, en, ec = expect[k]
        assert np.array_equal(d, ed) and np.array_equal(n, en) and np.array_equal(c, ec), f"request {k}"


@pytest.mark.gpu
def test_device_outputs_and_memory_budget(hp, gctx, scenes, ids):
    """Device-memory outputs; a byte budget that holds only the largest request alone still serves every
    request, and the state held never exceeds it."""
    import torch
    params = hp.default_params(radius=5, stride=2, precision=1)
    reqs = _requests(hp, scenes, ids, 5, seed=7)
    budget = max(_request_bytes(h, w) for _, h, w in reqs)
    with hp.Server(gctx, params, mem_limit=budget, passes_per_step=4) as srv:
        outs = []
        for j, h, w in reqs:
            t = (torch.empty(h, w, device="cuda"), torch.empty(h, w, 3, device="cuda"), torch.empty(h, w, device="cuda"))
            srv.submit(j, hp.maps_of(*t))
            outs.append(t)
        srv.drain(timeout_ms=60000)
        done = srv.poll(capacity=16)
        st = srv.stats()
        with pytest.raises(hp.HpError):  # a request larger than the whole budget is refused at submission
            big = scenes["m"]
            j = hp.make_job(ids["m"][0], [ids["m"][1]], hp.make_camera(*cam_of(big, 0)),
                            [hp.make_camera(*cam_of(big, 1))], *big.depth_range, iterations=1)
            srv2 = hp.Server(gctx, params, mem_limit=1024)
            try:
                m, *_ = hp.host_maps(big.height, big.width)
                srv2.submit(j, m)
            finally:
                srv2.close()
    assert len(done) == len(reqs) and all(c["status"] == 0 for c in done)
    # The budget holds one large request, or a few small ones together.
    assert st["peak_state_bytes"] <= budget
    assert st["peak_active"] <= budget // min(_request_bytes(h, w) for _, h, w in reqs)
    for (j, h, w), (d, n, c) in zip(reqs, outs):
        ed, en, ec = _alone(hp, gctx, j, params, h, w)
        assert np.array_equal(d.cpu().numpy(), ed) and np.array_equal(c.cpu().numpy(), ec)


HP_ERR_TIMEOUT = 5


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_a_failed_step_is_contained(hp, gctx, scenes, ids, precision):
    """A request with a tile that never reports completion (a test hook): the step's bounded waits run out
    after 100 ms, the requests admitted with it fail with HP_ERR_TIMEOUT, the server's error names the request,
    and requests submitted afterwards complete, bit-identical to hp_solve alone.  Before the shared abort
    flag and the recovery, every later step waited on the failed request's unfinished tiles and failed too."""
    params = hp.default_params(radius=5, stride=2, precision=precision)
    reqs = _requests(hp, scenes, ids, 6, seed=21 + precision)

    def run(srv, batch):
        got, rid = {}, {}
        for k, (j, h, w) in batch:
            m, d, n, c = hp.host_maps(h, w)
            rid[srv.submit(j, m)] = k
            got[k] = (d, n, c)
        srv.drain(timeout_ms=60000)
        return {rid[c["request_id"]]: c["status"] for c in srv.poll(capacity=64)}, got, rid

    with hp.Server(gctx, params, passes_per_step=4, wait_limit_ms=100, debug_stall_request=2,
                   debug_stall_tile=1) as srv:
        first, _, _ = run(srv, [(0, reqs[0])])
        assert first == {0: 0}
        # Request id 2 stalls; request 3 may be admitted beside it (and then fails with it) or after.
        mid, _, rid = run(srv, [(1, reqs[1]), (2, reqs[2])])
        assert mid[1] == HP_ERR_TIMEOUT and mid[2] in (0, HP_ERR_TIMEOUT)
        assert "request 2 " in srv.last_error() and "wait ran out" in srv.last_error()
        later, got, _ = run(srv, list(enumerate(reqs))[3:])
        st = srv.stats()
    assert later == {3: 0, 4: 0, 5: 0}
    assert st["failed_steps"] >= 1 and st["failed"] == sum(v != 0 for v in mid.values())
    for k, (d, n, c) in got.items():
        ed, en, ec = _alone(hp, gctx, *reqs[k][:1], params, *reqs[k][1:])
        assert np.array_equal(d, ed) and np.array_equal(n, en) and np.array_equal(c, ec), f"request {k}"


@pytest.mark.gpu
def test_queued_requests_are_cancelled_on_shutdown(hp, gctx, scenes, ids):
    params = hp.default_params(radius=5, stride=2, precision=1)
    reqs = _requests(hp, scenes, ids, 6, seed=11)
    srv = hp.Server(gctx, params, max_active=1, passes_per_step=1)
    for j, h, w in reqs:
        m, *_ = hp.host_maps(h, w)
        srv.submit(j, m)
    time.sleep(0.01)
    srv.close()  # returns once the admitted request has finished; the rest are cancelled


HP_ERR_CUDA = 2


@pytest.mark.gpu
def test_a_failed_launch_is_contained_without_waiting_out_the_limit(hp, gctx, scenes, ids):
    """A step whose launch fails on the host (a test hook injects it; nothing runs on the device): its
    requests fail with HP_ERR_CUDA, the launches queued behind it stop at once on the raised abort flag
    instead of waiting out the 30 s dependency limit, and later requests complete bit-identical to hp_solve."""
    params = hp.default_params(radius=5, stride=2, precision=1)
    reqs = _requests(hp, scenes, ids, 6, seed=31)
    t0 = time.time()
    with hp.Server(gctx, params, passes_per_step=2, wait_limit_ms=30000, debug_fail_step=2) as srv:
        got, rid = {}, {}
        for k, (j, h, w) in enumerate(reqs[:3]):
            m, d, n, c = hp.host_maps(h, w)
            rid[srv.submit(j, m)] = k
        srv.drain(timeout_ms=60000)
        first = {rid[c["request_id"]]: c["status"] for c in srv.poll(capacity=64)}
        assert "injected" in srv.first_error()
        for k, (j, h, w) in list(enumerate(reqs))[3:]:
            m, d, n, c = hp.host_maps(h, w)
            rid[srv.submit(j, m)] = k
            got[k] = (d, n, c)
        srv.drain(timeout_ms=60000)
        later = {rid[c["request_id"]]: c["status"] for c in srv.poll(capacity=64)}
        st = srv.stats()
    assert time.time() - t0 < 20, "a queued launch waited out the dependency limit"
    assert set(first.values()) <= {0, HP_ERR_CUDA} and HP_ERR_CUDA in first.values(), first
    assert later == {3: 0, 4: 0, 5: 0} and st["failed_steps"] >= 1
    for k, (d, n, c) in got.items():
        ed, en, ec = _alone(hp, gctx, *reqs[k][:1], params, *reqs[k][1:])
        assert np.array_equal(d, ed) and np.array_equal(n, en) and np.array_equal(c, ec), f"request {k}"


def test_server_option_defaults(hp):
    """hp_server_options_default: the budget policy (oldest first, at most 32 stages a request, 1200 M
    W*H*S units a step), 64 slots, 80% of device memory, 2 steps in flight, 2 s dependency limit, no
    test hooks."""
    o = hp.server_options()
    assert (o.policy, o.passes_per_step, o.step_budget_mpix) == (hp.SERVER_POLICY_BUDGET, 32, 1200.0)
    assert (o.max_active, o.inflight_steps, o.wait_limit_ms, o.split_launches) == (64, 2, 2000, 0)
    assert abs(o.mem_fraction - 0.8) < 1e-7 and o.mem_limit == 0
    assert (o.debug_stall_request, o.debug_stall_tile, o.debug_fail_step) == (0, 0, 0)
