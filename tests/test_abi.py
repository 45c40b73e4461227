"""The C ABI: the library loads, exports every entry point include/flsp_dg.h
declares, the ctypes mirrors match the C struct layouts, and without a GPU
the library fails loudly instead of falling back to the CPU."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import pytest

from felspa_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "flsp_dg.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(flsp_[a-z0-9_]+)\s*\(", text)))


def test_header_entry_points_exported(flsp):
    L = flsp.load()
    names = declared_functions()
    assert len(names) >= 25
    for n in names:
        assert hasattr(L, n), n
    out = subprocess.run(["nm", "-D", "--defined-only", flsp.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (flsp_\w+)", out))
    assert set(names) <= exported


def test_prototypes_cover_header(flsp):
    assert set(declared_functions()) == set(flsp.PROTOTYPES)


def test_struct_layouts_match_c():
    src = """
#include <stdio.h>
#include <stddef.h>
#include "flsp_dg.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\\n", sizeof(flsp_mesh_desc),
         sizeof(flsp_dg_opts), sizeof(flsp_factor), sizeof(flsp_vel_term), sizeof(flsp_velocity_desc),
         sizeof(flsp_ic_node), sizeof(flsp_ic_desc), sizeof(flsp_reinit_opts), sizeof(flsp_ls_opts),
         offsetof(flsp_ic_desc, waves), sizeof(flsp_train_opts), sizeof(flsp_learned_opts),
         offsetof(flsp_learned_opts, fallback), sizeof(flsp_learned_stats), sizeof(flsp_batch_tuning),
         offsetof(flsp_batch_tuning, adv_ms));
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write(src)
        gcc = "/usr/bin/gcc" if os.path.exists("/usr/bin/gcc") else "gcc"
        subprocess.run([gcc, "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        vals = [int(v) for v in subprocess.run([exe], capture_output=True, text=True).stdout.split()]
    mine = [C.sizeof(abi.MeshDesc), C.sizeof(abi.DGOpts), C.sizeof(abi.Factor), C.sizeof(abi.VelTerm),
            C.sizeof(abi.VelocityDesc), C.sizeof(abi.ICNode), C.sizeof(abi.ICDesc), C.sizeof(abi.ReinitOpts),
            C.sizeof(abi.LSOpts), abi.ICDesc.waves.offset, C.sizeof(abi.TrainOpts), C.sizeof(abi.LearnedOpts),
            abi.LearnedOpts.fallback.offset, C.sizeof(abi.LearnedStats), C.sizeof(abi.BatchTuning),
            abi.BatchTuning.adv_ms.offset]
    assert vals == mine


def test_defaults_are_reference_defaults(flsp):
    L = flsp.load()
    o = abi.DGOpts()
    L.flsp_default_dg_opts(C.byref(o))
    assert (o.rk_order, o.cfl_max, o.basis) == (3, 0.9, abi.BASIS_P)   # AdvectControl, FE_DGP
    r = abi.ReinitOpts()
    L.flsp_default_reinit_opts(C.byref(r))
    # ReinitControl (rktvd1, CFL 0.1-0.2) + AdditionalControl (max_iter 1000, band 4)
    assert (r.mode, r.rk_order, r.cfl_max, r.max_iter, r.band_width_coeff) == (abi.REINIT_BAND, 1, 0.2, 1000, 4.0)
    ls = abi.LSOpts()
    L.flsp_default_ls_opts(C.byref(ls))
    assert (ls.reinit_frequency, ls.execute_reinit) == (10, 1)   # LevelSetControl


def _cuda_visible():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.mark.skipif(_cuda_visible(), reason="a GPU is visible")
def test_no_gpu_fails_loudly(flsp):
    from felspa_b200.level_set import Mesh, Problem
    with pytest.raises(flsp.FlspError) as e:
        Problem(Mesh(2, (8, 8)), 1)
    assert e.value.code == abi.FLSP_ERR_NO_DEVICE


def test_bad_arguments_rejected(flsp):
    L = flsp.load()
    m = abi.mesh_desc(4, (8, 8, 8))
    o = abi.DGOpts()
    L.flsp_default_dg_opts(C.byref(o))
    h = C.c_void_p()
    assert L.flsp_create(C.byref(m), C.byref(o), C.byref(h)) == abi.FLSP_ERR_BAD_ARG
    assert b"dim" in L.flsp_last_error()
    m = abi.mesh_desc(3, (8, 8, 8))
    o.degree = 3
    assert L.flsp_create(C.byref(m), C.byref(o), C.byref(h)) == abi.FLSP_ERR_UNSUPPORTED
    assert L.flsp_create(None, C.byref(o), C.byref(h)) == abi.FLSP_ERR_BAD_ARG
    # handle-level entry points refuse a missing handle before touching a device
    d = C.c_double(0.0)
    t = (C.c_int * 3)()
    assert L.flsp_autotune(None, 3, t, None, None, None) == abi.FLSP_ERR_BAD_ARG
    assert L.flsp_stage_tile(None, t) == abi.FLSP_ERR_BAD_ARG
    assert L.flsp_curvature(None, abi.CURV_REFERENCE, C.byref(d), 1) == abi.FLSP_ERR_BAD_ARG
    assert L.flsp_eval_patches(None, 1, C.byref(d), 1) == abi.FLSP_ERR_BAD_ARG
    assert L.flsp_export_solutions(None, b"./", b"LevelSet") == abi.FLSP_ERR_BAD_ARG


def test_product_does_not_reference_oracle():
    """the product path never imports, links or loads the oracle"""
    pkg = os.path.join(ROOT, "felspa_b200")
    for dirpath, _, files in os.walk(pkg):
        for f in files:
            if f.endswith((".py", ".cu", ".cuh", ".h")):
                text = open(os.path.join(dirpath, f)).read()
                assert "oracle" not in text.lower(), f


def test_learned_and_batch_entry_points_without_gpu(flsp):
    """the network and batch entry points report a missing device or bad
    arguments instead of falling back to the CPU"""
    L = flsp.load()
    n = C.c_int64(0)
    assert L.flsp_mlp_n_params(C.byref(n)) == abi.FLSP_OK
    assert n.value == 256 * 82 + 256 + 3 * (256 * 256 + 256) + 9 * 256 + 9
    h = C.c_void_p()
    assert L.flsp_mlp_create(0, 1, C.byref(h)) == abi.FLSP_ERR_NO_DEVICE
    m = (abi.MeshDesc * 2)(abi.mesh_desc(2, (8, 8)), abi.mesh_desc(3, (8, 8, 8)))
    o = (abi.DGOpts * 2)()
    for i in range(2):
        L.flsp_default_dg_opts(C.byref(o[i]))
        o[i].basis = abi.BASIS_Q
    b = C.c_void_p()
    assert L.flsp_batch_create(2, m, o, C.byref(b)) == abi.FLSP_ERR_UNSUPPORTED   # a 3D member
    assert L.flsp_batch_create(0, m, o, C.byref(b)) == abi.FLSP_ERR_BAD_ARG
    t = abi.TrainOpts()
    L.flsp_default_train_opts(C.byref(t))
    assert (t.batch, t.lr, t.beta1, t.beta2) == (8192, 1e-3, 0.9, 0.999)
    lo = abi.LearnedOpts()
    L.flsp_default_learned_opts(C.byref(lo))
    assert (lo.band_cells, lo.max_residual, lo.fallback.mode, lo.fallback.narrow_band) == (6.0, 0.05, abi.REINIT_FIXED, 1)


def test_group_entry_points_without_gpu(flsp):
    """the group entry points reject bad arguments before touching a device"""
    L = flsp.load()
    g = C.c_void_p()
    hs = (C.c_void_p * 1)(None)
    assert L.flsp_group_create(hs, 0, C.byref(g)) == abi.FLSP_ERR_BAD_ARG
    assert L.flsp_group_create(hs, 1, C.byref(g)) == abi.FLSP_ERR_BAD_ARG   # a null member
    ctl = abi.default_ls_opts()
    assert L.flsp_group_run_periods(None, C.byref(ctl), 1) == abi.FLSP_ERR_BAD_ARG
    assert L.flsp_group_sync(None) == abi.FLSP_ERR_BAD_ARG
    L.flsp_group_destroy(None)


def test_patch_network_entry_points_without_gpu(flsp):
    """the 3D patch network and the graph-replayed learned periods reject
    bad arguments and report a missing device"""
    L = flsp.load()
    h = C.c_void_p()
    assert L.flsp_mlp_create_patch(7, 0, 1, C.byref(h)) in (abi.FLSP_ERR_BAD_ARG, abi.FLSP_ERR_NO_DEVICE)
    assert L.flsp_mlp_create_patch(abi.PATCH_3D_Q2, 0, 1, C.byref(h)) == abi.FLSP_ERR_NO_DEVICE
    assert L.flsp_mlp_info(None, None, None, None) == abi.FLSP_ERR_BAD_ARG
    lo = abi.LearnedOpts()
    L.flsp_default_learned_opts(C.byref(lo))
    assert L.flsp_ls_run_steps_learned(None, None, C.byref(lo), 10, 10) == abi.FLSP_ERR_BAD_ARG


def test_noalloc_argument_checks_without_gpu(flsp):
    """flsp_reduce_noalloc checks its arguments before any device call:
    a reduction that needs an IC or a comparison state without one, a bad
    reduction kind, a bad IC description (the pointers are never
    dereferenced on the host, so stand-in addresses suffice here)."""
    from felspa_b200 import fields as F
    from felspa_b200.level_set import Mesh, reduce_noalloc
    mesh = Mesh(2, (16, 16))
    fake = 0x100000   # stand-in device address
    for which in (abi.RED_MASS_ERROR, abi.RED_L2_ERROR_IC, abi.RED_L1_INTERFACE_IC):
        with pytest.raises(flsp.FlspError, match="needs an IC"):
            reduce_noalloc(mesh, 1, abi.BASIS_Q, abi.FP64, fake, which, fake)
    for which in (abi.RED_L1_INTERFACE, abi.RED_MEAN_ABS_DIFF):
        with pytest.raises(flsp.FlspError, match="needs ref_state"):
            reduce_noalloc(mesh, 1, abi.BASIS_Q, abi.FP64, fake, which, fake)
    for which in (-1, abi.RED_MASS_SHARP + 1):
        with pytest.raises(flsp.FlspError, match="bad reduction kind"):
            reduce_noalloc(mesh, 1, abi.BASIS_Q, abi.FP64, fake, which, fake)

    class BadIC:
        def __init__(self, **kw):
            self.d = F.zalesak_disk().desc()
            for k, v in kw.items():
                setattr(self.d, k, v)

        def desc(self):
            return self.d

    for kw in ({"n_nodes": 0}, {"root": 7}, {"n_waves": -1}, {"n_waves": 33}):
        with pytest.raises(flsp.FlspError, match="bad IC"):
            reduce_noalloc(mesh, 1, abi.BASIS_Q, abi.FP64, fake, abi.RED_MASS_ERROR, fake, ic=BadIC(**kw))
    with pytest.raises(flsp.FlspError, match="null argument"):
        reduce_noalloc(mesh, 1, abi.BASIS_Q, abi.FP64, 0, abi.RED_MASS, fake)


def test_noalloc_argument_checks_without_gpu(flsp):
    """flsp_reduce_noalloc refuses missing inputs and bad kinds before it
    touches a device (fake non-null addresses: nothing is read)"""
    from felspa_b200.level_set import Mesh, reduce_noalloc
    from felspa_b200.lib import FlspError
    from felspa_b200 import fields as F
    mesh = Mesh(2, (8, 8))
    fake = 0x1000
    with pytest.raises(FlspError, match="needs an IC"):
        reduce_noalloc(mesh, 1, abi.BASIS_Q, abi.FP64, fake, abi.RED_MASS_ERROR, fake)
    with pytest.raises(FlspError, match="needs ref_state"):
        reduce_noalloc(mesh, 1, abi.BASIS_Q, abi.FP64, fake, abi.RED_L1_INTERFACE, fake)
    with pytest.raises(FlspError, match="bad reduction kind"):
        reduce_noalloc(mesh, 1, abi.BASIS_Q, abi.FP64, fake, 99, fake)
    with pytest.raises(FlspError, match="bad basis"):
        reduce_noalloc(mesh, 1, 7, abi.FP64, fake, abi.RED_MASS, fake)
    with pytest.raises(FlspError, match="null argument"):
        reduce_noalloc(mesh, 1, abi.BASIS_Q, abi.FP64, fake, abi.RED_MASS, 0)
    bad_ic = F.sphere((0.5, 0.5), 0.2)
    d = bad_ic.desc()
    d.root = 99
    import ctypes as C
    L = flsp.load()
    md = mesh.desc()
    st = L.flsp_reduce_noalloc(C.byref(md), 1, abi.BASIS_Q, abi.FP64, C.c_void_p(fake), None,
                               abi.RED_L2_ERROR_IC, C.byref(d), C.c_void_p(fake), None)
    assert st == abi.FLSP_ERR_BAD_ARG
    assert b"bad IC" in L.flsp_last_error()
