"""The SfM front of the stage: source-view selection and depth ranges (selectSourceViews,
patchmatch_mvs.cu:74-157) and the seeded initialisation (:1111-1177).

Pinned to the reference itself: tests/golden/sfm_select.npz holds the reference's own
selectSourceViews outputs (made by tests/golden/make_sfm_golden.py through the harness, which
compiles the reference source unmodified), and where the harness is built the live comparisons run
too.  Tolerance: identity (sources, scores, angles and depth ranges bit for bit; seeds bit for bit).
On the GPU, seeded hypotheses must equal the oracle's painting of the same seeds over the engine's
random initialisation, and the reference's runPatchMatchMVS on seeded pixels."""
from __future__ import annotations

import os

import numpy as np
import pytest

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "sfm_select.npz")


@pytest.fixture(scope="module")
def golden():
    g = np.load(GOLDEN)
    krt = g["cams_krt"]
    cams = [(k[:9].reshape(3, 3), k[9:18].reshape(3, 3), k[18:21]) for k in krt]
    off, img = g["track_offset"], g["track_images"]
    tracks = [img[off[i]:off[i + 1]].tolist() for i in range(len(off) - 1)]
    return g, cams, g["registered"].tolist(), g["positions"], tracks


def _expected(g, ns):
    out = []
    for i, ref in enumerate(g[f"ns{ns}_ref"]):
        k = int(g[f"ns{ns}_count"][i])
        out.append({"ref": int(ref), "sources": g[f"ns{ns}_sources"][i, :k].tolist(),
                    "scores": g[f"ns{ns}_scores"][i, :k].tolist(), "baseline_deg": g[f"ns{ns}_angles"][i, :k].tolist(),
                    "depth_min": float(g[f"ns{ns}_depth_min"][i]), "depth_max": float(g[f"ns{ns}_depth_max"][i])})
    return out


def _norm(sel):
    return [{k: ([float(np.float32(x)) for x in v] if isinstance(v, list) and k != "sources" else v)
             for k, v in s.items()} for s in sel]


@pytest.mark.parametrize("ns", [4, 8])
def test_oracle_selection_matches_reference_golden(po, golden, ns):
    g, cams, reg, pos, tracks = golden
    assert _norm(po.sfm_select_sources(cams, reg, pos, tracks, ns)) == _norm(_expected(g, ns))


@pytest.mark.parametrize("ns", [4, 8])
def test_engine_selection_matches_reference_golden(hp, golden, ns):
    g, cams, reg, pos, tracks = golden
    sel = hp.select_sources([hp.make_camera(*c) for c in cams], hp.SfmPoints(pos, tracks), ns, reg)
    assert _norm(sel) == _norm(_expected(g, ns))


def test_engine_selection_matches_live_reference(hp, scene_mod):
    import pmref
    if not pmref.available():
        pytest.skip("reference harness not built (needs the reference tree at build time)")
    for seed in range(3):
        s = scene_mod.multi_object(seed=20 + seed, w=200, h=120, n_views=8 + 2 * seed, n_refs=0, f=160.0)
        cams = [(v.cam.K, v.cam.R, v.cam.t) for v in s.views]
        pos, tracks = scene_mod.sparse_points(s, n=800, seed=seed)
        reg = [1] * len(cams)
        reg[seed] = 0
        for ns in (3, 6, 8):
            want = pmref.select_sources(cams, reg, pos, tracks, ns)
            got = hp.select_sources([hp.make_camera(*c) for c in cams], hp.SfmPoints(pos, tracks), ns, reg)
            assert _norm(got) == _norm(want), (seed, ns)


def test_seeds_match_oracle(hp, po, golden):
    g, cams, reg, pos, tracks = golden
    sel = po.sfm_select_sources(cams, reg, pos, tracks, 4)
    P = hp.SfmPoints(pos, tracks)
    total = 0
    for v in sel:
        r = v["ref"]
        got = hp.project_seeds(hp.make_camera(*cams[r]), r, v["depth_min"], v["depth_max"], P)
        got = [(q.x, q.y, q.depth, q.normal[0], q.normal[1], q.normal[2]) for q in got[:got.count]]
        want = po.sfm_project_seeds(cams[r], r, v["depth_min"], v["depth_max"], pos, tracks)
        assert got == want, r
        total += len(got)
    assert total > 1000


def test_selection_edge_cases(hp, golden):
    g, cams, reg, pos, tracks = golden
    C = [hp.make_camera(*c) for c in cams]
    # No points: no shared points, so no sources; depth range from the (zero) centroid's depth.
    empty = hp.select_sources(C, hp.SfmPoints(np.zeros((0, 3)), []), 4)
    assert len(empty) == len(C) and all(v["sources"] == [] for v in empty)
    for v, c in zip(empty, cams):
        d = np.float32(c[2][2])
        assert v["depth_min"] == d * np.float32(0.3) and v["depth_max"] == d * np.float32(3.0)
    # A single registered camera has no candidates.
    one = hp.select_sources(C, hp.SfmPoints(pos, tracks), 4, [1] + [0] * (len(C) - 1))
    assert len(one) == 1 and one[0]["sources"] == []
    # Invalid arguments are refused, not crashed on.
    with pytest.raises(hp.HpError):
        hp.select_sources(C, hp.SfmPoints(pos, tracks), 9)
    with pytest.raises(hp.HpError):
        hp.select_sources(C, hp.SfmPoints(pos, [[len(C) + 3]] * len(tracks)), 4)


# ------------------------------------------------------------------------------------ GPU


@pytest.mark.gpu
def test_seeded_init_matches_oracle_painting(hp, po, scene_mod, small_scene):
    s = small_scene
    cams = [(v.cam.K, v.cam.R, v.cam.t) for v in s.views]
    pos, tracks = scene_mod.sparse_points(s, n=300, seed=4)
    P = hp.SfmPoints(pos, tracks)
    with hp.Context(0) as ctx:
        ids = [ctx.upload(v.image) for v in s.views]
        for r, radius in [(0, 50), (2, 3), (4, 0)]:
            srcs = s.sources[r]
            job = hp.make_job(ids[r], [ids[i] for i in srcs], hp.make_camera(*cams[r]),
                              [hp.make_camera(*cams[i]) for i in srcs], *s.depth_range, seed=42, view_id=r)
            params = hp.default_params()
            m0, d0, n0, _ = hp.host_maps(s.height, s.width)
            ctx.init_hypotheses(job, params, m0)
            seeds = hp.project_seeds(hp.make_camera(*cams[r]), r, *s.depth_range, P)
            assert seeds.count > 10
            m1, d1, n1, _ = hp.host_maps(s.height, s.width)
            ctx.init_hypotheses(hp.with_seeds(job, seeds, radius), params, m1)
            want = po.sfm_project_seeds(cams[r], r, *s.depth_range, pos, tracks)
            po.paint_seeds(d0, n0, want, radius)
            assert np.array_equal(d1, d0) and np.array_equal(n1, n0), (r, radius)


@pytest.mark.gpu
def test_seeded_stage_matches_reference(hp, scene_mod, small_scene):
    """The reference's runPatchMatchMVS at 0 iterations (random init + SfM seeding) against the engine's
    seeded initialisation, on the pixels the seeds cover (elsewhere both are random, from different RNGs)."""
    import pmref
    if not pmref.available():
        pytest.skip("reference harness not built (needs the reference tree at build time)")
    s = small_scene
    cams = [(v.cam.K, v.cam.R, v.cam.t) for v in s.views]
    pos, tracks = scene_mod.sparse_points(s, n=300, seed=6)
    ref_maps = pmref.run_stage([v.image_f32 for v in s.views], cams, pos, tracks, patch_size=11)
    P = hp.SfmPoints(pos, tracks)
    C = [hp.make_camera(*c) for c in cams]
    sel = {v["ref"]: v for v in hp.select_sources(C, P, min(8, max(3, len(C) - 1)))}
    covered_total = 0
    with hp.Context(0) as ctx:
        ids = [ctx.upload(v.image_f32) for v in s.views]
        for r, (rd, rn) in ref_maps.items():
            v = sel[r]
            job = hp.make_job(ids[r], [ids[i] for i in v["sources"]], C[r], [C[i] for i in v["sources"]],
                              v["depth_min"], v["depth_max"], seed=42 + 1_000_000 * r, view_id=r)
            seeds = hp.project_seeds(C[r], r, v["depth_min"], v["depth_max"], P)
            m, d, n, _ = hp.host_maps(s.height, s.width)
            ctx.init_hypotheses(hp.with_seeds(job, seeds, 50), hp.default_params(), m)
            mask = np.zeros(d.shape, bool)
            for q in seeds[:seeds.count]:
                mask[max(0, q.y - 50):max(0, q.y + 51), max(0, q.x - 50):max(0, q.x + 51)] = True
            covered_total += int(mask.sum())
            assert np.array_equal(d[mask], rd[mask]) and np.array_equal(n[mask], rn[mask]), r
    assert covered_total > 0


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_seeded_jobs_in_plans_and_server_match_solve(hp, scene_mod, small_scene, precision):
    """Seeded jobs give the same maps through hp_solve, a plan (both schedules) and the server."""
    s = small_scene
    cams = [(v.cam.K, v.cam.R, v.cam.t) for v in s.views]
    pos, tracks = scene_mod.sparse_points(s, n=300, seed=8)
    P = hp.SfmPoints(pos, tracks)
    params = hp.default_params(radius=5, stride=2, precision=precision)
    with hp.Context(0) as ctx:
        ids = [ctx.upload(v.image) for v in s.views]
        jobs = []
        for r in (0, 3):
            srcs = s.sources[r]
            job = hp.make_job(ids[r], [ids[i] for i in srcs], hp.make_camera(*cams[r]),
                              [hp.make_camera(*cams[i]) for i in srcs], *s.depth_range, seed=5, view_id=r,
                              iterations=3)
            jobs.append(hp.with_seeds(job, hp.project_seeds(hp.make_camera(*cams[r]), r, *s.depth_range, P), 20))
        want = []
        for j in jobs:
            m, d, n, c = hp.host_maps(s.height, s.width)
            ctx.solve([j], params, [m])
            want.append((d, n, c))
        for sched in (hp.SCHEDULE_PER_PASS, hp.SCHEDULE_PERSISTENT):
            outs = [hp.host_maps(s.height, s.width) for _ in jobs]
            with hp.Plan(ctx, jobs, params, [o[0] for o in outs], hp.plan_options(schedule=sched)) as plan:
                plan.run()
            for (_, d, n, c), (wd, wn, wc) in zip(outs, want):
                assert np.array_equal(d, wd) and np.array_equal(n, wn) and np.array_equal(c, wc), sched
        outs = [hp.host_maps(s.height, s.width) for _ in jobs]
        with hp.Server(ctx, params, passes_per_step=3) as srv:
            for j, o in zip(jobs, outs):
                srv.submit(j, o[0])
            srv.drain(timeout_ms=60000)
            done = srv.poll(capacity=8)
        assert len(done) == 2 and all(c["status"] == 0 for c in done)
        for (_, d, n, c), (wd, wn, wc) in zip(outs, want):
            assert np.array_equal(d, wd) and np.array_equal(n, wn) and np.array_equal(c, wc)
