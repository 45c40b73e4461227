"""Generate the golden fixtures under tests/golden/ from the CPU oracle.

    python tests/golden/make_golden.py

The reference (deal.II-based FELSPA) cannot be built or run here and its
own tests hold no reference numbers, so these fixtures are regression pins
of the oracle: they freeze its outputs on small cases.  tests/test_oracle.py
checks the oracle against them, tests/test_gpu_parity.py checks the library
against them.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from felspa_b200 import abi, fields as F  # noqa: E402
from oracle import oracle as O  # noqa: E402


def cases():
    """name -> (dim, n, degree, basis, field, ic, what)"""
    return {
        "zalesak_p1_rhs": (2, (16, 16), 1, abi.BASIS_P, F.ccw_rotation(), F.zalesak_disk(), "rhs"),
        "zalesak_q2_rk3": (2, (16, 16), 2, abi.BASIS_Q, F.ccw_rotation(), F.zalesak_disk(), "advance"),
        "circles_q2_reinit": (2, (16, 16), 2, abi.BASIS_Q, F.ccw_rotation(),
                              F.sphere((0.4731, 0.5193), 0.25) + F.sphere((0.6817, 0.3109), 0.17), "reinit"),
        "sphere_q2_3d_rhs": (3, (6, 6, 6), 2, abi.BASIS_Q, F.deformation_3d(),
                             F.sphere((0.35, 0.35, 0.35), 0.15), "rhs"),
        "sphere_p2_3d_grad": (3, (6, 5, 4), 2, abi.BASIS_P, F.deformation_3d(),
                              F.sphere((0.45, 0.5, 0.55), 0.3), "grad"),
        "circles_q2_curvature": (2, (16, 16), 2, abi.BASIS_Q, F.ccw_rotation(),
                                 F.sphere((0.4731, 0.5193), 0.25) + F.sphere((0.6817, 0.3109), 0.17),
                                 "curvature"),
    }


def compute(name, spec):
    dim, n, p, basis, field, ic, what = spec
    pr = O.Problem(dim, n, p, basis)
    pr.set_velocity(field)
    phi0 = pr.project(ic)
    out = {"phi0": phi0}
    if what == "rhs":
        out["result"] = pr.advect_rhs(phi0, 0.2)
    elif what == "advance":
        phi = phi0.copy()
        pr.advance(phi, 0.05, single_cycle=False, cfl_max=0.1)
        out["result"] = phi
        out["t"] = np.array([pr.clock.t, pr.clock.n_substeps])
    elif what == "reinit":
        phi = phi0.copy()
        st, nit = pr.reinit(phi, abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=3))
        assert st == 0
        out["result"] = phi
    elif what == "grad":
        gl, gr = pr.hj_gradients(phi0)
        out["result"] = np.concatenate([gl.ravel(), gr.ravel()])
    elif what == "curvature":
        out["result"] = pr.curvature(phi0)
        out["result_neighbour"] = pr.curvature(phi0, to_neighbour=True)
    return out


def revolution_cases():
    """The Zalesak slotted disk of the 2D configuration: 128^2 cells of the
    unit square, degree 1 (Q and P), counter-clockwise rotation
    u = 2 pi (0.5 - y, x - 0.5), one revolution (T = 1), SSP-RK3 at CFL
    0.1, a fixed 5-pseudo-step reinit over every cell each 10 substeps
    (band 6 cells), without and with the reference test's LDG viscosity
    1e-3 (tests/test_zalesak_disk.cc:252,256).
    name -> (basis, viscosity, keep the full final state)"""
    return {
        # the inviscid Q1 sweep is unstable over a revolution (the field
        # degrades and rounding differences grow without bound): its state
        # is frozen at T = 0.05 as well
        "zalesak128_q1_nu0_t0.05": (abi.BASIS_Q, 0.0, True, 0.05),
        "zalesak128_q1_nu0": (abi.BASIS_Q, 0.0, False),
        "zalesak128_p1_nu0": (abi.BASIS_P, 0.0, False),
        "zalesak128_q1_nu1e-3": (abi.BASIS_Q, 1e-3, True),
        "zalesak128_p1_nu1e-3": (abi.BASIS_P, 1e-3, True),
        # the reference test's viscosity 1e-3 on its [-50, 50]^2 domain with
        # period 628, rescaled to the unit square with period 1:
        # 1e-3 * 628 / 100^2
        "zalesak128_q1_nu6.28e-5": (abi.BASIS_Q, 6.28e-5, True),
        "zalesak128_p1_nu6.28e-5": (abi.BASIS_P, 6.28e-5, True),
    }


def revolution_opts(viscosity):
    ro = abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=5, band_width_coeff=6.0,
                                 viscosity=viscosity)
    return abi.default_ls_opts(reinit_frequency=10, reinit=ro)


def compute_revolution(basis, viscosity, keep_state, t_end=1.0):
    import time
    ic = F.zalesak_disk()
    pr = O.Problem(2, (128, 128), 1, basis)
    pr.set_velocity(F.ccw_rotation())
    phi = pr.project(ic)
    area0 = pr.reduce(abi.RED_MASS, phi)
    t0 = time.perf_counter()
    pr.ls_advance(phi, t_end, revolution_opts(viscosity), single_step=False, rk_order=3, cfl_max=0.1)
    cpu_s = time.perf_counter() - t0
    nb = pr.nb
    out = {"t_end": np.array(pr.clock.t), "n_substeps": np.array(pr.clock.n_substeps),
           "area0": np.array(area0), "area1": np.array(pr.reduce(abi.RED_MASS, phi)),
           "l1_ic": np.array(pr.reduce(abi.RED_L1_INTERFACE_IC, phi, ic=ic)),
           "max_abs": np.array(np.abs(phi).max()),
           "cell_means": phi.reshape(-1, nb)[:, 0].copy(),
           "cpu_s": np.array(cpu_s), "threads": np.array(os.cpu_count() or 1)}
    if keep_state:
        out["result"] = phi
    return out


def main(names=None):
    for name, spec in cases().items():
        if names and name not in names:
            continue
        out = compute(name, spec)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, {k: v.shape for k, v in out.items()})
    # full revolutions take minutes each: only when named
    for name, spec in revolution_cases().items():
        if not names or name not in names:
            continue
        out = compute_revolution(*spec)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, {k: (v.shape if v.ndim else float(v)) for k, v in out.items()}, flush=True)


if __name__ == "__main__":
    main(sys.argv[1:])
