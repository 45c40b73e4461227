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


def main(names=None):
    for name, spec in cases().items():
        if names and name not in names:
            continue
        out = compute(name, spec)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main(sys.argv[1:])
