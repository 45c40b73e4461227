"""Host-side VTU / PVD writers (no GPU): layout of the files the library
writes for SimulatorBase::export_solutions (src/pde/pde_base.cc:93-115,
LevelSetSurface::export_solution, level_set.implement.h:313-342, deal.II
DataOut patches) and PVDCollector (src/base/io.cc:142-166).

The patch values fed to the writer come from the oracle's basis functions;
the GPU evaluation of the same values is checked in test_export_gpu.py.
"""
import xml.etree.ElementTree as ET

import numpy as np
import pytest

from felspa_b200 import abi
from felspa_b200.level_set import Mesh, write_pvd, write_vtu
from felspa_b200.lib import FlspError


def oracle_patches(orc, phi_lex, dim, n_sub):
    """values of every lexicographic cell at its (n_sub+1)^dim patch
    vertices (x fastest), from the oracle's basis functions"""
    ns1 = n_sub + 1
    pts = [(i / n_sub, j / n_sub, k / n_sub)
           for k in range(ns1 if dim == 3 else 1) for j in range(ns1) for i in range(ns1)]
    val, _ = orc.shape(np.array(pts, dtype=np.float64))
    return phi_lex.reshape(-1, orc.nb) @ val


def parse_vtu(path):
    root = ET.parse(path).getroot()
    piece = root.find("UnstructuredGrid/Piece")
    arr = lambda node, dt: np.array(node.text.split(), dtype=dt)
    pts = arr(piece.find("Points/DataArray"), np.float64).reshape(-1, 3)
    cells = {d.get("Name"): d for d in piece.findall("Cells/DataArray")}
    pd = piece.find("PointData")
    return {
        "n_points": int(piece.get("NumberOfPoints")),
        "n_cells": int(piece.get("NumberOfCells")),
        "points": pts,
        "conn": arr(cells["connectivity"], np.int64),
        "offsets": arr(cells["offsets"], np.int64),
        "types": arr(cells["types"], np.int64),
        "scalars": pd.get("Scalars"),
        "values": arr(pd.find("DataArray"), np.float64),
        "name": pd.find("DataArray").get("Name"),
    }


@pytest.mark.parametrize("n_sub", [1, 2])
def test_vtu_2d_patches(flsp, oracle, tmp_path, n_sub):
    n, p, lo, hi = (4, 3), 2, (0.0, 1.0), (2.0, 2.5)
    rng = np.random.default_rng(5)
    order = rng.permutation(n[0] * n[1]).astype(np.int64)
    mesh = Mesh(2, n, lo, hi, host_cell_order=order)
    orc = oracle.Problem(2, n, p, abi.BASIS_Q, lo + (0,), hi + (1,))
    phi = rng.standard_normal(orc.n_dofs)
    vals = oracle_patches(orc, phi, 2, n_sub)[order]          # host cell order
    f = tmp_path / "phi.vtu"
    write_vtu(mesh, vals, "LevelSet", str(f), n_sub=n_sub)
    v = parse_vtu(str(f))
    ncell, npt, nsc = n[0] * n[1], (n_sub + 1) ** 2, n_sub ** 2
    assert v["n_points"] == ncell * npt and v["n_cells"] == ncell * nsc
    assert v["scalars"] == "LevelSet" and v["name"] == "LevelSet"
    np.testing.assert_array_equal(v["values"], vals.ravel())   # %.17g round-trips doubles
    # every point is its host cell's patch vertex
    h = np.array([(hi[0] - lo[0]) / n[0], (hi[1] - lo[1]) / n[1]])
    for k, c in enumerate(order):
        ix, iy = c % n[0], c // n[0]
        for j in range(npt):
            s = np.array([j % (n_sub + 1), j // (n_sub + 1)]) / n_sub
            np.testing.assert_allclose(v["points"][k * npt + j, :2], np.array(lo) + h * (np.array([ix, iy]) + s),
                                       rtol=0, atol=1e-15)
            assert v["points"][k * npt + j, 2] == 0.0
    # quads: counter-clockwise, inside their own patch
    assert np.all(v["types"] == 9)
    np.testing.assert_array_equal(v["offsets"], 4 * np.arange(1, ncell * nsc + 1))
    quads = v["conn"].reshape(-1, 4)
    for q in quads:
        assert len({int(i) // npt for i in q}) == 1
        P = v["points"][q, :2]
        area = 0.5 * sum(P[i, 0] * P[(i + 1) % 4, 1] - P[(i + 1) % 4, 0] * P[i, 1] for i in range(4))
        np.testing.assert_allclose(area, h[0] * h[1] / nsc, rtol=1e-12)


def test_vtu_3d_hexahedra(flsp, oracle, tmp_path):
    n, p = (3, 2, 2), 1
    mesh = Mesh(3, n)
    orc = oracle.Problem(3, n, p, abi.BASIS_P)
    phi = np.random.default_rng(6).standard_normal(orc.n_dofs)
    vals = oracle_patches(orc, phi, 3, 1)
    f = tmp_path / "phi3.vtu"
    write_vtu(mesh, vals, "phi", str(f))
    v = parse_vtu(str(f))
    ncell = 12
    assert v["n_points"] == 8 * ncell and v["n_cells"] == ncell
    assert np.all(v["types"] == 12)
    np.testing.assert_array_equal(v["values"], vals.ravel())
    for hx in v["conn"].reshape(-1, 8):
        P = v["points"][hx]
        lo_f, up_f = P[:4], P[4:]
        assert np.all(lo_f[:, 2] == lo_f[0, 2]) and np.all(up_f[:, 2] > lo_f[0, 2])
        np.testing.assert_allclose(up_f[:, :2], lo_f[:, :2], atol=1e-15)
        # lower face counter-clockwise seen from +z
        a = sum(lo_f[i, 0] * lo_f[(i + 1) % 4, 1] - lo_f[(i + 1) % 4, 0] * lo_f[i, 1] for i in range(4))
        assert a > 0


def test_corner_values_of_a_linear_field_are_continuous(flsp, oracle, tmp_path):
    """a projected linear field is exact in Q1: the two one-sided values of
    every shared vertex coincide and equal the field"""
    n = (5, 4)
    orc = oracle.Problem(2, n, 1, abi.BASIS_Q)
    from felspa_b200 import fields as F
    ic = F.height_function(1, 0.3, [])        # phi = y - 0.3
    phi = orc.project(ic)
    vals = oracle_patches(orc, phi, 2, 1)
    f = tmp_path / "lin.vtu"
    write_vtu(Mesh(2, n), vals, "phi", str(f))
    v = parse_vtu(str(f))
    exact = np.array([oracle.eval_ic(ic, 2, (x, y, 0.0)) for x, y, _ in v["points"]])
    np.testing.assert_allclose(v["values"], exact, rtol=0, atol=1e-13)


def test_pvd_records(flsp, tmp_path):
    f = tmp_path / "LevelSet.pvd"
    recs = [(0.0, "LevelSet_000000001.vtu"), (0.125, "LevelSet_000000002.vtu")]
    write_pvd(str(f), recs)
    root = ET.parse(str(f)).getroot()
    assert root.get("type") == "Collection"
    ds = root.findall("Collection/DataSet")
    assert [(float(d.get("timestep")), d.get("file")) for d in ds] == recs


def test_writers_reject_bad_arguments(flsp, tmp_path):
    mesh = Mesh(2, (2, 2))
    with pytest.raises(ValueError):
        write_vtu(mesh, np.zeros(3), "phi", str(tmp_path / "a.vtu"))
    with pytest.raises(FlspError) as e:
        write_vtu(mesh, np.zeros(4 * 18 * 18), "phi", str(tmp_path / "a.vtu"), n_sub=17)
    assert e.value.code == abi.FLSP_ERR_BAD_ARG
    with pytest.raises(FlspError):
        write_vtu(mesh, np.zeros(16), "phi", str(tmp_path / "missing_dir" / "a.vtu"))
    with pytest.raises(FlspError):
        write_pvd(str(tmp_path / "missing_dir" / "a.pvd"), [])
    # labels and record names become XML attributes and file names
    with pytest.raises(FlspError):
        write_vtu(mesh, np.zeros(16), 'phi" evil="1', str(tmp_path / "b.vtu"))
    with pytest.raises(FlspError):
        write_pvd(str(tmp_path / "b.pvd"), [(0.0, "a<b.vtu")])


def test_rejected_pvd_leaves_existing_collection(flsp, tmp_path):
    """a call with a bad record name fails before the file is opened: the
    collection written earlier stays as it was"""
    f = tmp_path / "LevelSet.pvd"
    write_pvd(str(f), [(0.0, "LevelSet_000000000.vtu"), (0.5, "LevelSet_000000001.vtu")])
    before = f.read_bytes()
    with pytest.raises(FlspError):
        write_pvd(str(f), [(0.0, "LevelSet_000000000.vtu"), (1.0, "../x.vtu")])
    assert f.read_bytes() == before
