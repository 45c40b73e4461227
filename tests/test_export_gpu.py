"""GPU: point values of the DG field for output (flsp_eval_patches) against
the oracle's basis functions, and the files flsp_export_solutions writes
(SimulatorBase::export_solutions, src/pde/pde_base.cc:93-115).

Bar: the device evaluates in FP64 from the stored coefficients, so against
the oracle on the same coefficients (FP32 states: the same FP32-rounded
coefficients) the relative max-norm difference is <= 1e-13.
"""
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from felspa_b200 import abi, fields as F
from felspa_b200.level_set import LevelSetSurface, Mesh, Problem, dealii_hypercube_order

from test_export import oracle_patches, parse_vtu

pytestmark = pytest.mark.gpu

TOL = 1e-13


def rel(a, b):
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


@pytest.mark.parametrize("dim,n,p,basis,prec,n_sub", [
    (2, (8, 8), 1, abi.BASIS_P, abi.FP64, 1),
    (2, (8, 8), 2, abi.BASIS_Q, abi.FP64, 1),
    (2, (8, 8), 3, abi.BASIS_Q, abi.FP64, 3),
    (2, (8, 8), 3, abi.BASIS_P, abi.FP32, 2),
    (3, (4, 4, 4), 2, abi.BASIS_Q, abi.FP32, 1),
    (3, (4, 4, 4), 2, abi.BASIS_P, abi.FP64, 2),
    (3, (4, 4, 4), 1, abi.BASIS_Q, abi.FP64, 1),
])
def test_eval_patches_vs_oracle(flsp, oracle, dim, n, p, basis, prec, n_sub):
    order = dealii_hypercube_order(dim, 2, int(np.log2(n[0] // 2)))
    pr = Problem(Mesh(dim, n, host_cell_order=order), p, basis=basis, precision=prec)
    orc = oracle.Problem(dim, n, p, basis)
    nb = orc.nb
    rng = np.random.default_rng(11 + dim + p)
    phi_host = rng.standard_normal(orc.n_dofs)
    if prec == abi.FP32:
        phi_host = phi_host.astype(np.float32).astype(np.float64)
    pr.set_state(phi_host)
    got = pr.eval_patches(n_sub)
    # host order -> lexicographic cells for the oracle
    lex = np.empty_like(phi_host).reshape(-1, nb)
    lex[order] = phi_host.reshape(-1, nb)
    want = oracle_patches(orc, lex.ravel(), dim, n_sub)[order]
    assert got.shape == want.shape
    assert rel(got, want) <= TOL
    pr.close()


def test_export_solutions_files(flsp, oracle, tmp_path):
    n = (16, 16)
    ls = LevelSetSurface(Mesh(2, n), 2, basis=abi.BASIS_Q, precision=abi.FP64, cfl_max=0.1)
    ls.initialize(F.zalesak_disk(), F.ccw_rotation())
    prefix = str(tmp_path) + "/"
    ls.export_solutions(prefix)
    v0 = ls.problem.eval_patches(1)
    ls.advance_time(0.01)
    t1 = ls.get_time()
    ls.export_solutions(prefix)
    v1 = ls.problem.eval_patches(1)
    for name, want in (("LevelSet_000000001.vtu", v0), ("LevelSet_000000002.vtu", v1)):
        v = parse_vtu(str(tmp_path / name))
        assert v["n_points"] == 4 * 256 and v["name"] == "LevelSet"
        np.testing.assert_array_equal(v["values"], want.ravel())
    assert not np.array_equal(v0, v1)
    ds = ET.parse(str(tmp_path / "LevelSet.pvd")).getroot().findall("Collection/DataSet")
    assert [d.get("file") for d in ds] == ["LevelSet_000000001.vtu", "LevelSet_000000002.vtu"]
    np.testing.assert_allclose([float(d.get("timestep")) for d in ds], [0.0, t1], rtol=0, atol=0)
    # the corner values are the field's: compare with the oracle on the state
    orc = oracle.Problem(2, n, 2, abi.BASIS_Q)
    want = oracle_patches(orc, ls.get_solution_vector(), 2, 1)
    assert rel(v1, want) <= TOL
    ls.problem.close()


def test_eval_patches_rejects_bad_sizes(flsp):
    from felspa_b200.lib import FlspError
    pr = Problem(Mesh(2, (4, 4)), 1)
    with pytest.raises(FlspError):
        pr.eval_patches(0)
    with pytest.raises(FlspError):
        pr.eval_patches(17)
    pr.close()


def test_cpp_driver_exports(flsp, tmp_path):
    """the C++ Zalesak driver writes the reference test's exports: before
    the loop, after the first and after the last outer step"""
    import os
    import subprocess
    exe = os.path.join(os.path.dirname(flsp.LIB_PATH), "examples", "zalesak_disk.bin")
    d = tmp_path / "ZalesaksDisk_Cycle0"
    d.mkdir()
    out = subprocess.run([exe, "2", "0.001", str(d) + "/"], capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr
    names = [f"LevelSet_00000000{k}.vtu" for k in (1, 2, 3)]
    for nm in names:
        v = parse_vtu(str(d / nm))
        assert v["n_points"] == 4 * 64 * 64 and np.all(np.isfinite(v["values"]))
    ds = ET.parse(str(d / "LevelSet.pvd")).getroot().findall("Collection/DataSet")
    assert [x.get("file") for x in ds] == names
    t = [float(x.get("timestep")) for x in ds]
    assert t[0] == 0.0 and 0.0 < t[1] < t[2]


def test_export_writes_synced_curvature(flsp, oracle, tmp_path):
    """as LevelSetSurface::export_solution (level_set.implement.h:325-330):
    the curvature estimate goes into the VTU as <label>Curvature while its
    time equals the solution's, and is left out once the solution moves on"""
    n = (16, 16)
    ls = LevelSetSurface(Mesh(2, n), 2, basis=abi.BASIS_Q, precision=abi.FP64, cfl_max=0.1)
    ls.initialize(F.sphere((0.5, 0.5), 0.3), F.ccw_rotation())
    kappa = ls.estimate_curvature(abi.CURV_NEIGHBOUR)
    prefix = str(tmp_path) + "/"
    ls.export_solutions(prefix)
    root = ET.parse(str(tmp_path / "LevelSet_000000001.vtu")).getroot()
    arrays = root.findall("UnstructuredGrid/Piece/PointData/DataArray")
    assert [a.get("Name") for a in arrays] == ["LevelSet", "LevelSetCurvature"]
    got = np.array(arrays[1].text.split(), dtype=np.float64)
    orc = oracle.Problem(2, n, 2, abi.BASIS_Q)
    want = oracle_patches(orc, kappa, 2, 1).ravel()
    assert rel(got, want) <= TOL
    ls.advance_time(0.01)
    ls.export_solutions(prefix)
    root = ET.parse(str(tmp_path / "LevelSet_000000002.vtu")).getroot()
    assert [a.get("Name") for a in root.findall("UnstructuredGrid/Piece/PointData/DataArray")] == ["LevelSet"]
    ls.problem.close()
