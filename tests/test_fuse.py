"""Depth-map fusion (hp_fuse_depth_maps, include/hpmvs.h): the consumer of the stage, filling the
reference's fuseDepthMaps (src/dense_recon/point_cloud.h:7), which is a stub there
(src/dense_recon/point_cloud.cu:4-8).  With no reference behaviour to match, the rule is the one
include/hpmvs.h states, restated in plain C by the oracle (orc_fuse).

CPU: the oracle against known answers (back-projection of one view, duplicate suppression between
identical views, points on the rendered surfaces), its edge cases (empty maps, thresholds, capacity).
GPU: the engine equals the oracle bit for bit (tolerance 0: the same FP32 operation order, no
contraction) on host and device maps, with explicit neighbour lists, on a solve's own filtered maps,
and under a short capacity; invalid arguments are refused."""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

from conftest import cam_of


def _gt_maps(s, noise=0.0, seed=0):
    rng = np.random.default_rng(seed)
    maps = []
    for v in s.views:
        d = v.depth_gt.astype(np.float32).copy()
        if noise:
            d *= (1 + noise * rng.standard_normal(d.shape)).astype(np.float32)
        conf = rng.uniform(0.0, 1.0, d.shape).astype(np.float32)
        maps.append((d, v.normal_gt.astype(np.float32), conf, v.image_f32.astype(np.float32)))
    return maps


def _backproject(K, R, t, depth):
    h, w = depth.shape
    ys, xs = np.mgrid[0:h, 0:w]
    rays = np.stack([xs, ys, np.ones_like(xs)], -1).astype(np.float64) @ np.linalg.inv(K).T
    pc = rays * depth[..., None]
    return (pc - t) @ R  # R^T (p - t), row vectors


# ------------------------------------------------------------------------------------------- CPU


def test_single_view_emits_every_valid_pixel(po, small_scene):
    s = small_scene
    v = s.views[0]
    d = v.depth_gt.astype(np.float32)
    pos, nrm, col = po.fuse([(d, v.normal_gt, None, v.image_f32)], [cam_of(s, 0)], min_views=1)
    valid = d > 0
    assert len(pos) == int(valid.sum())
    K, R, t = cam_of(s, 0)
    want = _backproject(K, R, t, d.astype(np.float64))[valid]
    assert np.allclose(pos, want, rtol=1e-5, atol=1e-5)
    assert np.allclose(nrm, (v.normal_gt.astype(np.float64) @ R)[valid], atol=1e-5)
    assert np.array_equal(col[:, 0], v.image_f32[valid]) and np.array_equal(col[:, 0], col[:, 2])


def test_identical_views_emit_each_point_once(po, small_scene):
    s = small_scene
    v = s.views[0]
    d = v.depth_gt.astype(np.float32)
    one = po.fuse([(d, v.normal_gt, None, None)], [cam_of(s, 0)], min_views=1)
    two = po.fuse([(d, v.normal_gt, None, None)] * 2, [cam_of(s, 0)] * 2)
    # View 1 agrees with view 0 everywhere and defers to it; view 0's points are two-view means of itself.
    assert len(two[0]) == len(one[0])
    assert np.allclose(two[0], one[0], rtol=1e-6, atol=1e-6)


def test_fused_points_lie_on_the_rendered_surfaces(po, small_scene):
    s = small_scene
    maps = _gt_maps(s)
    pos, nrm, col = po.fuse([(d, n, None, g) for d, n, _, g in maps], [cam_of(s, i) for i in range(len(maps))])
    assert len(pos) > 0.5 * (maps[0][0] > 0).sum()
    # Every point lies on the rendered surface seen by some view (points hidden from one view are
    # still on the surface of the view that saw them): best relative depth error over the views.
    best = np.full(len(pos), np.inf)
    for i in range(len(maps)):
        K, R, t = cam_of(s, i)
        pc = pos.astype(np.float64) @ R.T + t
        uv = pc @ K.T
        u, v = np.rint(uv[:, 0] / uv[:, 2]).astype(int), np.rint(uv[:, 1] / uv[:, 2]).astype(int)
        h, w = maps[i][0].shape
        ok = (u >= 0) & (u < w) & (v >= 0) & (v < h) & (pc[:, 2] > 0)
        gt = np.zeros(len(pos))
        gt[ok] = maps[i][0][v[ok], u[ok]]
        ok &= gt > 0
        rel = np.full(len(pos), np.inf)
        rel[ok] = np.abs(pc[ok, 2] - gt[ok]) / gt[ok]
        best = np.minimum(best, rel)
    assert (best < 0.01).mean() > 0.999, (best < 0.01).mean()
    assert np.allclose(np.linalg.norm(nrm, axis=1), 1.0, atol=1e-5)
    assert (col >= 0).all() and (col <= 1).all()


def test_edge_cases(po, small_scene):
    s = small_scene
    maps = _gt_maps(s, noise=0.002, seed=3)
    cams = [cam_of(s, i) for i in range(len(maps))]
    zero = [(np.zeros_like(d), n, c, g) for d, n, c, g in maps]
    assert len(po.fuse(zero, cams)[0]) == 0
    assert len(po.fuse(maps, cams, min_views=len(maps) + 1)[0]) == 0
    base = po.fuse(maps, cams)
    conf = po.fuse(maps, cams, min_confidence=0.5)
    assert 0 < len(conf[0]) < len(base[0])
    # Without neighbours, and one view required, each view emits all its (confident) pixels.
    alone = po.fuse(maps, cams, neighbors=[[]] * len(maps), min_views=1)
    assert len(alone[0]) == sum(int((d > 0).sum()) for d, *_ in maps)
    # A tight normal test keeps fewer points than the default.
    assert len(po.fuse(maps, cams, min_normal_cos=0.99999)[0]) < len(base[0])


def test_oracle_fusion_is_independent_of_thread_count(po, small_scene):
    """Points come in (view, row, column) order whatever the parallel split: one thread and eight
    give the same arrays."""
    s = small_scene
    maps = _gt_maps(s, noise=0.002, seed=9)
    cams = [cam_of(s, i) for i in range(len(maps))]
    n0 = po.num_threads()
    try:
        po.set_num_threads(1)
        one = po.fuse(maps, cams)
        po.set_num_threads(8)
        many = po.fuse(maps, cams)
    finally:
        po.set_num_threads(n0)
    assert len(one[0]) > 0
    assert all(np.array_equal(a, b) for a, b in zip(one, many))


def test_fusion_entry_points_are_exported_and_defaults(hp):
    for name in ("hp_fuse_params_default", "hp_fuse_depth_maps"):
        assert hasattr(hp.lib, name) and name in hp.EXPORTS
    p = hp.fuse_params()
    assert (p.memory, p.min_views) == (hp.MEMORY_HOST, 2)
    assert p.max_depth_rel == np.float32(0.01) and p.max_reproj_px == 2.0
    assert abs(p.min_normal_cos - np.cos(np.radians(10))) < 1e-7
    assert C.sizeof(hp.FuseView) == 224 and C.sizeof(hp.FuseParams) == 24 and C.sizeof(hp.PointCloudC) == 48
    with pytest.raises(TypeError):
        hp.fuse_params(tolerance=1)


# ------------------------------------------------------------------------------------------- GPU


def _engine(hp, ctx, s, maps, neighbors=None, device=False, **kw):
    import torch
    cams = [hp.make_camera(*cam_of(s, i)) for i in range(len(maps))]
    cols = list(zip(*maps))
    if device:
        cols = [[None if a is None else torch.from_numpy(np.ascontiguousarray(a)).cuda() for a in c] for c in cols]
    cloud = ctx.fuse(cams, cols[0], cols[1], cols[2], cols[3], neighbors, hp.fuse_params(**kw))
    if device:
        return tuple(a.cpu().numpy() for a in (cloud.positions, cloud.normals, cloud.colors))
    return cloud.positions, cloud.normals, cloud.colors


def _same(a, b):
    return all(x.shape == y.shape and np.array_equal(x, y) for x, y in zip(a, b))


@pytest.mark.gpu
@pytest.mark.parametrize("device", [False, True])
@pytest.mark.parametrize("kw", [{}, {"min_confidence": 0.3, "min_views": 3},
                                {"max_depth_rel": 0.002, "max_reproj_px": 0.75, "min_normal_cos": -1.0}])
def test_engine_matches_oracle(hp, po, small_scene, device, kw):
    s = small_scene
    maps = _gt_maps(s, noise=0.001, seed=5)
    with hp.Context(0) as ctx:
        got = _engine(hp, ctx, s, maps, device=device, **kw)
    want = po.fuse(maps, [cam_of(s, i) for i in range(len(maps))], **kw)
    assert len(want[0]) > 1000
    assert _same(got, want)


@pytest.mark.gpu
def test_engine_matches_oracle_with_neighbour_lists_and_no_colour(hp, po, small_scene):
    s = small_scene
    maps = [(d, n, None, None) for d, n, _, _ in _gt_maps(s, noise=0.001, seed=6)]
    nb = [[1, 2], [0, 2, 3], [4, 1], [2], [0, 3, 1]]
    with hp.Context(0) as ctx:
        got = _engine(hp, ctx, s, maps, neighbors=nb)
    want = po.fuse(maps, [cam_of(s, i) for i in range(len(maps))], neighbors=nb)
    assert len(want[0]) > 0 and _same(got, want)
    assert not got[2].any()


@pytest.mark.gpu
def test_fusion_of_a_solve(hp, po, small_scene):
    """The engine's own filtered maps (hp_solve + hp_geometric_filter), fused on the device."""
    import torch
    s = small_scene
    n = len(s.views)
    params = hp.default_params(radius=5, stride=1)
    with hp.Context(0) as ctx:
        ids = [ctx.upload(v.image) for v in s.views]
        cams = [hp.make_camera(*cam_of(s, i)) for i in range(n)]
        jobs = [hp.make_job(ids[r], [ids[i] for i in s.sources[r]], cams[r], [cams[i] for i in s.sources[r]],
                            *s.depth_range, seed=42 + r, view_id=r, iterations=6) for r in range(n)]
        outs = [(torch.empty(s.height, s.width, device="cuda"), torch.empty(s.height, s.width, 3, device="cuda"),
                 torch.empty(s.height, s.width, device="cuda")) for _ in range(n)]
        ctx.solve(jobs, params, [hp.maps_of(*o) for o in outs])
        conf = [1 - o[2] / 2 for o in outs]
        for r in range(n):
            srcs = s.sources[r]
            ctx.geometric_filter(cams[r], outs[r][0], outs[r][1], conf[r], [cams[i] for i in srcs],
                                 [outs[i][0] for i in srcs], [outs[i][1] for i in srcs])
        grays = [torch.from_numpy(v.image_f32).cuda() for v in s.views]
        cloud = ctx.fuse(cams, [o[0] for o in outs], [o[1] for o in outs], conf, grays, s.sources)
        got = tuple(a.cpu().numpy() for a in (cloud.positions, cloud.normals, cloud.colors))
        host = [(o[0].cpu().numpy(), o[1].cpu().numpy(), c.cpu().numpy(), v.image_f32)
                for o, c, v in zip(outs, conf, s.views)]
    want = po.fuse(host, [cam_of(s, i) for i in range(n)], neighbors=s.sources)
    assert _same(got, want)
    assert cloud.size() > 0.3 * s.height * s.width


@pytest.mark.gpu
def test_capacity_and_invalid_arguments(hp, po, small_scene):
    s = small_scene
    maps = _gt_maps(s, noise=0.001, seed=7)
    cams = [hp.make_camera(*cam_of(s, i)) for i in range(len(maps))]
    want = po.fuse(maps, [cam_of(s, i) for i in range(len(maps))])
    with hp.Context(0) as ctx:
        views = []
        for cam, (d, nr, c, g) in zip(cams, maps):
            v = hp.FuseView()
            v.cam = cam
            v.height, v.width = d.shape
            v.depth, v.normal, v.confidence, v.gray = (a.ctypes.data for a in (d, nr, c, g))
            views.append(v)
        prm = hp.fuse_params()
        out = hp.PointCloudC()
        assert ctx.fuse_views(views, prm, out) == len(want[0])  # capacity 0: count only
        k = len(want[0]) // 3
        pos = np.full((k + 1, 3), -7.0, np.float32)
        out.positions, out.capacity = pos.ctypes.data, k
        assert ctx.fuse_views(views, prm, out) == len(want[0])
        assert np.array_equal(pos[:k], want[0][:k]) and (pos[k] == -7.0).all()
        bad = hp.FuseView.from_buffer_copy(views[0])
        self_nb = np.array([0], np.int32)  # a view listing itself
        bad.neighbors, bad.num_neighbors = self_nb.ctypes.data_as(C.POINTER(C.c_int)), 1
        with pytest.raises(hp.HpError):
            ctx.fuse_views([bad] + views[1:], prm, hp.PointCloudC())
        with pytest.raises(hp.HpError):
            ctx.fuse_views(views, hp.fuse_params(min_views=0), hp.PointCloudC())
        sing = hp.FuseView.from_buffer_copy(views[0])
        sing.cam = hp.make_camera(np.zeros((3, 3)), np.eye(3), np.zeros(3))
        with pytest.raises(hp.HpError):
            ctx.fuse_views([sing] + views[1:], prm, hp.PointCloudC())


@pytest.mark.gpu
def test_fuse_depth_maps_on_the_stage_output(hp, po, small_scene):
    """fuse_depth_maps(depth_maps, cameras, images) - the reference's fuseDepthMaps signature - on the
    DepthMaps run_patchmatch_mvs returns (host maps, filtered, confidence 1 - cost / 2)."""
    s = small_scene
    n = len(s.views)
    cams = [hp.make_camera(*cam_of(s, i)) for i in range(n)]
    images = [v.image for v in s.views]
    views = [hp.ViewParams(r, list(s.sources[r]), *s.depth_range) for r in range(n)]
    maps = hp.run_patchmatch_mvs(images, cams, views, hp.MVSConfig(mvs_iterations=4, mvs_patch_size=11))
    cloud = hp.fuse_depth_maps(maps, cams, images)
    want = po.fuse([(dm.depth, dm.normal, dm.confidence, hp._gray_f32(images[dm.image_id])) for dm in maps],
                   [cam_of(s, dm.image_id) for dm in maps])
    assert cloud.size() > 0
    assert _same((cloud.positions, cloud.normals, cloud.colors), want)
