"""Shared fixtures.  Tests marked ``gpu`` need a B200 and the built engine;
everything else runs on the CPU (oracle, C ABI host entry points, scenes,
multi-rank host logic over gloo)."""
from __future__ import annotations

import importlib
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "oracle"), os.path.join(ROOT, "oracle", "ref_harness")):
    if p not in sys.path:
        sys.path.insert(0, p)

PKG = "hemiphoto3d-private_b200"
# The reference checkout, present only where fixtures are generated and its
# headers compiled against; HP_REFERENCE_TREE overrides the default.
REFERENCE_TREE = os.environ.get("HP_REFERENCE_TREE", "/root/reference")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built engine")


@pytest.fixture(scope="session")
def hp():
    return importlib.import_module(PKG)


@pytest.fixture(scope="session")
def scene_mod():
    return importlib.import_module(PKG + ".scene")


@pytest.fixture(scope="session")
def po():
    import pm_oracle
    pm_oracle.lib()
    return pm_oracle


@pytest.fixture(scope="session")
def small_scene(scene_mod):
    """plane_sphere at 160x120 (fx scaled), 5 views."""
    return scene_mod.plane_sphere(w=160, h=120)


@pytest.fixture(scope="session")
def full_scene(scene_mod):
    """plane_sphere at its stated 640x480."""
    return scene_mod.plane_sphere()


def cam_of(scene, i):
    v = scene.views[i].cam
    return (v.K, v.R, v.t)


def oracle_view(po, scene, r, radius=5, stride=1, coeffs=None, top_k=3):
    srcs = scene.sources[r]
    return po.View(scene.views[r].image_f32, [scene.views[i].image_f32 for i in srcs], radius=radius,
                   stride=stride, top_k=top_k, ref_cam=cam_of(scene, r), src_cams=[cam_of(scene, i) for i in srcs],
                   coeffs=coeffs)


def err_stats(a, b):
    e = np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)).ravel()
    return {"max": float(e.max()), "p999": float(np.quantile(e, 0.999)), "p99": float(np.quantile(e, 0.99)),
            "p90": float(np.quantile(e, 0.9)), "exact": float((e == 0).mean())}
