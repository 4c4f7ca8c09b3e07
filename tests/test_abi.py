"""C ABI checks that need no GPU: the library loads and exports every entry
point include/hpmvs.h declares, the Python struct mirrors match the C layout,
host-only entry points work, and device entry points fail cleanly."""
from __future__ import annotations

import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from conftest import REFERENCE_TREE, ROOT

HEADER = os.path.join(ROOT, "include", "hpmvs.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?[a-z_]+\*?\s+\*?(hp_[a-z0-9_]+)\s*\(", text, re.M)))


def test_header_declares_the_boundary():
    names = declared_functions()
    for must in ("hp_solve", "hp_ncc_cost", "hp_propagate_pass", "hp_init_hypotheses", "hp_geometric_filter",
                 "hp_image_upload", "hp_ctx_create", "hp_pfm_write", "hp_pfm_read", "hp_setup_homographies"):
        assert must in names


def test_library_exports_every_declared_symbol(hp):
    exported = subprocess.run(["nm", "-D", "--defined-only", hp.LIB_PATH], capture_output=True, text=True,
                              check=True).stdout
    syms = {line.split()[-1] for line in exported.splitlines() if line.strip()}
    missing = [f for f in declared_functions() if f not in syms]
    assert not missing, missing
    assert set(hp.EXPORTS) == set(declared_functions())


def test_struct_layout_matches_header(hp):
    src = r'''
#include <stdio.h>
#include <stddef.h>
#include "hpmvs.h"
int main(void) {
  printf("%zu %zu %zu %zu\n", sizeof(hp_job), sizeof(hp_params), sizeof(hp_camera), sizeof(hp_maps));
  printf("%zu %zu %zu %zu %zu %zu\n", offsetof(hp_job, ref_cam), offsetof(hp_job, depth_min), offsetof(hp_job, seed),
         offsetof(hp_job, use_coeffs), offsetof(hp_job, ab), offsetof(hp_maps, cost));
  return 0; }
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-std=c11", "-I", os.path.dirname(HEADER), "-o", exe, c], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split()
    want = [C.sizeof(hp.Job), C.sizeof(hp.Params), C.sizeof(hp.Camera), C.sizeof(hp.Maps),
            hp.Job.ref_cam.offset, hp.Job.depth_min.offset, hp.Job.seed.offset, hp.Job.use_coeffs.offset,
            hp.Job.ab.offset, hp.Maps.cost.offset]
    assert [int(v) for v in out] == want


# Every struct of the ABI and its ctypes mirror (field names are the header's).
MIRRORS = [("hp_camera", "Camera"), ("hp_params", "Params"), ("hp_seed", "Seed"), ("hp_job", "Job"),
           ("hp_maps", "Maps"), ("hp_profile", "Profile"), ("hp_plan_options", "PlanOptions"),
           ("hp_plan_info", "PlanInfo"), ("hp_server_options", "ServerOptions"), ("hp_completion", "Completion"),
           ("hp_server_stats", "ServerStats"), ("hp_sparse_points", "SparsePoints"),
           ("hp_view_selection", "ViewSelection"), ("hp_fuse_view", "FuseView"), ("hp_fuse_params", "FuseParams"),
           ("hp_point_cloud", "PointCloudC")]


def test_every_mirror_matches_the_header_field_by_field(hp):
    """sizeof and every field's offset of each ABI struct, from the C compiler, against the ctypes mirror."""
    lines = []
    for cname, pyname in MIRRORS:
        fields = [f[0] for f in getattr(hp, pyname)._fields_]
        lines.append(f'  printf("{cname} %zu", sizeof({cname}));')
        for f in fields:
            lines.append(f'  printf(" %zu", offsetof({cname}, {f}));')
        lines.append('  printf("\\n");')
    src = "#include <stdio.h>\n#include <stddef.h>\n#include \"hpmvs.h\"\nint main(void) {\n" + "\n".join(lines) + \
        "\n  return 0; }\n"
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(src)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-std=c11", "-I", os.path.dirname(HEADER), "-o", exe, c], check=True)
        out = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.splitlines()
    got = {ln.split()[0]: [int(v) for v in ln.split()[1:]] for ln in out}
    for cname, pyname in MIRRORS:
        cls = getattr(hp, pyname)
        want = [C.sizeof(cls)] + [getattr(cls, f[0]).offset for f in cls._fields_]
        assert got[cname] == want, f"{cname} vs {pyname}: C {got[cname]}, ctypes {want}"


def test_default_params_are_the_reference_constants(hp):
    p = hp.default_params()
    assert (p.radius, p.stride, p.top_k, p.refine_steps, p.precision) == (5, 1, 3, 2, 0)
    assert abs(p.iter_decay - 0.6) < 1e-7 and p.step_decay == 0.5


def test_status_strings(hp):
    assert hp.lib.hp_status_string(0) == b"ok"
    assert hp.lib.hp_status_string(3) == b"out of device memory"
    assert hp.lib.hp_version().count(b".") == 2


def test_context_creation_fails_cleanly_without_a_device(hp):
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    h = C.c_void_p()
    st = hp.lib.hp_ctx_create(0, C.byref(h))
    assert st == 2 and not h.value  # HP_ERR_CUDA, no handle
    assert hp.lib.hp_ctx_create(0, None) == 1


def test_null_context_is_rejected(hp):
    assert hp.lib.hp_ctx_destroy(None) == 1
    assert hp.lib.hp_solve(None, None, 0, None, None) == 1
    assert hp.lib.hp_ctx_last_error(None) == b"null context"


def test_setup_homographies_rejects_bad_input(hp):
    K = np.eye(3)
    ref = hp.make_camera(np.zeros((3, 3)), np.eye(3), np.zeros(3))  # singular K
    kinv = (C.c_double * 9)()
    ab = (C.c_double * 12)()
    src = (hp.Camera * 1)(hp.make_camera(K, np.eye(3), np.zeros(3)))
    assert hp.lib.hp_setup_homographies(C.byref(ref), src, 1, kinv, ab) == 1
    assert hp.lib.hp_setup_homographies(C.byref(hp.make_camera(K, np.eye(3), np.zeros(3))), src, 9, kinv, ab) == 1


def test_identity_homography(hp):
    K = np.array([[500.0, 0, 320], [0, 500, 240], [0, 0, 1]])
    c = hp.make_camera(K, np.eye(3), np.zeros(3))
    kinv, ab = hp.setup_homographies(c, [c])
    assert np.allclose(kinv @ K, np.eye(3))
    assert np.allclose(ab[0, :9].reshape(3, 3), np.eye(3)) and np.allclose(ab[0, 9:], 0)


@pytest.mark.parametrize("shape", [(7, 5), (4, 6, 3), (1, 1)])
def test_pfm_round_trip_bit_exact(hp, shape, tmp_path):
    """PFMSaveLoad (tests/test_patchmatch.cpp:192-222), 1- and 3-channel."""
    a = np.random.default_rng(3).standard_normal(shape).astype(np.float32)
    p = str(tmp_path / "x.pfm")
    hp.pfm_write(p, a)
    b = hp.pfm_read(p)
    assert b.shape == a.shape and np.array_equal(a, b)
    raw = open(p, "rb").read()
    assert raw.startswith(b"Pf\n" if a.ndim == 2 else b"PF\n") and b"\n-1.0\n" in raw
    # rows are stored bottom-to-top
    body = np.frombuffer(raw[-a.size * 4:], np.float32).reshape(a.shape)
    assert np.array_equal(body[0], a[-1])


def test_pfm_errors(hp, tmp_path):
    with pytest.raises(hp.HpError):
        hp.pfm_read(str(tmp_path / "missing.pfm"))
    bad = tmp_path / "bad.pfm"
    bad.write_bytes(b"P6\n2 2\n255\n")
    with pytest.raises(hp.HpError):
        hp.pfm_read(str(bad))
    trunc = tmp_path / "trunc.pfm"
    trunc.write_bytes(b"Pf\n4 4\n-1.0\n" + b"\0" * 8)
    with pytest.raises(hp.HpError):
        hp.pfm_read(str(trunc))


def test_stage_adapter_compiles_against_reference_headers(tmp_path):
    """include/hpmvs_stage.hpp (runPatchMatchMVS and fuseDepthMaps on the C ABI) compiles inside the reference's
    own translation-unit context: its types.h / patchmatch_mvs.h, with the test-only stand-ins
    for the Eigen and OpenCV headers those include."""
    ref = REFERENCE_TREE
    if not os.path.isdir(os.path.join(ref, "src", "dense_recon")):
        pytest.skip("reference tree not present")
    src = tmp_path / "adapter.cpp"
    src.write_text('#include "dense_recon/patchmatch_mvs.h"\n#include "dense_recon/point_cloud.h"\n'
                   '#include "hpmvs_stage.hpp"\n'
                   'auto* p = &hpmvs_stage::runPatchMatchMVS;\nauto* q = &hpmvs_stage::fuseDepthMaps;\n')
    subprocess.run(["g++", "-std=c++17", "-fsyntax-only", "-I", os.path.join(ROOT, "oracle", "ref_harness", "shim"),
                    "-I", os.path.join(ref, "include"), "-I", os.path.join(ref, "src"), "-I", os.path.join(ROOT, "include"),
                    "-I", "/usr/local/cuda/include", str(src)], check=True)
