"""The persistent ticket schedule (hp_schedule_build), checked on the host.

The persistent kernel runs (view, stage, tile) tickets in counter order, and a
stage-k tile waits for its own and its four neighbour tiles' stage k-1.  It can
never deadlock if every ticket waited on is smaller than the waiter's: the
CTA holding it took it earlier and is already running.  These tests check that
ordering property on random uneven batches (including the serving form, where
a launch starts each view at a later stage), that every (view, stage, tile) is
scheduled exactly once, and they replay the schedule with a simulated pool of
concurrent workers of every size to show it always completes."""
from __future__ import annotations

import numpy as np
import pytest


def _decode(et, ev, es, t):
    e = int(np.searchsorted(et, t, side="right")) - 1
    return int(ev[e]), int(es[e]), t - int(et[e])


def _random_batch(rng, n, serving=False):
    tx = rng.integers(1, 7, n)
    ty = rng.integers(1, 6, n)
    iters = rng.integers(0, 5, n)
    total = 2 * iters + 2
    kb = rng.integers(0, total) if serving else np.zeros(n, int)
    ke = np.minimum(total, kb + (rng.integers(1, 5, n) if serving else total))
    return tx, ty, kb, ke


@pytest.mark.parametrize("serving", [False, True])
def test_every_dependency_has_a_smaller_ticket(hp, serving):
    rng = np.random.default_rng(5)
    for trial in range(40):
        n = int(rng.integers(1, 7))
        tx, ty, kb, ke = _random_batch(rng, n, serving)
        et, ev, es = hp.schedule_build((tx * ty).tolist(), kb.tolist(), ke.tolist())
        total = int(et[-1])
        assert total == int(sum((tx * ty) * (ke - kb)))
        seen = {}
        for t in range(total):
            v, k, tile = _decode(et, ev, es, t)
            assert kb[v] <= k < ke[v] and 0 <= tile < tx[v] * ty[v]
            assert (v, k, tile) not in seen
            seen[(v, k, tile)] = t
        for (v, k, tile), t in seen.items():
            if k == kb[v]:
                continue  # its dependencies finished in an earlier launch
            x, y = tile % tx[v], tile // tx[v]
            for dx, dy in ((0, 0), (-1, 0), (1, 0), (0, -1), (0, 1)):
                if 0 <= x + dx < tx[v] and 0 <= y + dy < ty[v]:
                    assert seen[(v, k - 1, (y + dy) * tx[v] + x + dx)] < t


@pytest.mark.parametrize("workers", [1, 2, 3, 7, 64])
def test_simulated_concurrent_execution_completes(hp, workers):
    """Workers take tickets in order, wait for their dependencies, then run for a random time."""
    rng = np.random.default_rng(workers)
    tx, ty, kb, ke = _random_batch(rng, 5)
    et, ev, es = hp.schedule_build((tx * ty).tolist(), kb.tolist(), ke.tolist())
    total = int(et[-1])
    done = {}  # (v, tile) -> last finished stage
    nxt = 0
    running = []  # [ticket, remaining work or None while waiting]
    steps = 0
    while nxt < total or running:
        steps += 1
        assert steps < 100 * (total + 1), "schedule stalled"
        while len(running) < workers and nxt < total:
            running.append([nxt, None])
            nxt += 1
        for r in running:
            v, k, tile = _decode(et, ev, es, r[0])
            if r[1] is None:
                x, y = tile % tx[v], tile // tx[v]
                deps = [(v, (y + dy) * tx[v] + x + dx) for dx, dy in ((0, 0), (-1, 0), (1, 0), (0, -1), (0, 1))
                        if 0 <= x + dx < tx[v] and 0 <= y + dy < ty[v]]
                if k == kb[v] or all(done.get(d, -1) >= k - 1 for d in deps):
                    r[1] = int(rng.integers(1, 4))
            else:
                r[1] -= 1
        for r in [r for r in running if r[1] == 0]:
            v, k, tile = _decode(et, ev, es, r[0])
            done[(v, tile)] = k
            running.remove(r)
    assert all(done[(v, t)] == ke[v] - 1 for v in range(len(tx)) if ke[v] > kb[v] for t in range(tx[v] * ty[v]))


def test_schedule_build_rejects_bad_input(hp):
    with pytest.raises(hp.HpError):
        hp.schedule_build([2], [3], [1])
    et, ev, es = hp.schedule_build([4, 0, 2], [0, 0, 0], [2, 2, 1])
    assert list(ev) == [0, 2, 0] and list(es) == [0, 0, 1] and et[-1] == 4 + 2 + 4
