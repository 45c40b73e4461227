"""flsp_reduce_noalloc: the allocation-free reduction entry point.

It must give the same numbers as flsp_reduce (same kernels, same partial-sum
layout), twice in a row on the same device (its scratch array is reused, not
cleared), and reject meshes beyond its fixed scratch size.  This file is
collected last so that it also runs after everything else has used the
device."""
import ctypes as C

import numpy as np
import pytest

from felspa_b200 import abi, fields as F
from felspa_b200.level_set import Mesh, Problem, reduce_noalloc
from felspa_b200.lib import FlspError, check, load

pytestmark = pytest.mark.gpu

KINDS = [abi.RED_MASS, abi.RED_MASS_ERROR, abi.RED_L1_INTERFACE, abi.RED_MEAN_ABS_DIFF,
         abi.RED_GRAD_DEVIATION, abi.RED_MAX_ABS, abi.RED_L2_ERROR_IC, abi.RED_L1_INTERFACE_IC,
         abi.RED_MASS_SHARP]
NEEDS_IC = {abi.RED_MASS_ERROR, abi.RED_L2_ERROR_IC, abi.RED_L1_INTERFACE_IC}
NEEDS_REF = {abi.RED_L1_INTERFACE, abi.RED_MEAN_ABS_DIFF}


def _device_state(torch, prob):
    dt = torch.float64 if prob.precision == abi.FP64 else torch.float32
    return torch.from_numpy(prob.get_state()).to(device="cuda", dtype=dt)


@pytest.mark.parametrize("dim,n,p,basis,prec", [
    (2, (48, 40), 2, abi.BASIS_Q, abi.FP64),
    (2, (33, 47), 3, abi.BASIS_P, abi.FP32),
    (3, (12, 10, 14), 2, abi.BASIS_Q, abi.FP32),
    (3, (9, 11, 8), 1, abi.BASIS_P, abi.FP64),
])
def test_noalloc_matches_flsp_reduce(dim, n, p, basis, prec):
    torch = pytest.importorskip("torch")
    mesh = Mesh(dim, n)
    prob = Problem(mesh, p, basis=basis, precision=prec, cfl_max=0.2)
    if dim == 2:
        ic, vel = F.zalesak_disk(center=(0.4927, 0.7481)), F.ccw_rotation()
    else:
        ic, vel = F.sphere((0.35, 0.35, 0.35), 0.15), F.deformation_3d()
    prob.set_velocity(vel)
    prob.project(ic)
    ref = _device_state(torch, prob)
    prob.snapshot()
    check(load().flsp_advance(prob.h, 0.02, 0, C.byref(C.c_double(0.0))))
    state = _device_state(torch, prob)
    out = torch.full((len(KINDS), 2), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    # two calls in a row per kind, on the same stream, reusing the scratch array
    for i, w in enumerate(KINDS):
        for r in range(2):
            reduce_noalloc(mesh, p, basis, prec, state.data_ptr(), w, out[i, r:].data_ptr(),
                           ref_ptr=ref.data_ptr() if w in NEEDS_REF else None,
                           ic=ic if w in NEEDS_IC else None, stream=stream)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    for i, w in enumerate(KINDS):
        want = prob.reduce(w, ic=ic if w in NEEDS_IC else None)
        assert np.isfinite(want), w
        assert got[i, 0] == want, (w, got[i, 0], want)
        assert got[i, 1] == want, (w, got[i, 1], want)
    prob.close()


def test_noalloc_rejects_oversized_mesh():
    torch = pytest.importorskip("torch")
    mesh = Mesh(3, (256, 256, 129))   # 8.45M cells > FLSP_NOALLOC_MAX_CELLS
    assert mesh.n_cells > abi.NOALLOC_MAX_CELLS
    buf = torch.zeros(4, dtype=torch.float64, device="cuda")
    with pytest.raises(FlspError, match="at most"):
        reduce_noalloc(mesh, 1, abi.BASIS_Q, abi.FP64, buf.data_ptr(), abi.RED_MASS, buf.data_ptr())
