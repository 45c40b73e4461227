"""Learned reinitialisation: the tensor-core MLP of libflsp_dg.so.

No counterpart in the reference, whose ReinitSimulatorLDG
(src/level_set/reinit.cc:386-637) only has the HJ sweep; that sweep stays
as the source of the training targets and as the fallback where the
network's result is not distance-like enough (the cell mean of
||grad phi| - 1| above a threshold).

The network maps the 3 x 3 patch of a 2D degree-2 (Q basis) cell, 9
Legendre coefficients per cell divided by the cell size h, plus 64 h, to
the change of the centre cell's coefficients under the HJ sweep, divided
by h: 82 -> 256 x 4 (GELU) -> 9, BF16 weights on the tensor cores, FP32
accumulation, FP32 master weights and Adam.
"""
import ctypes as C

import numpy as np

from . import abi
from .lib import check, dp, fp, load

IN, HIDDEN, OUT = abi.MLP_IN, abi.MLP_HIDDEN, abi.MLP_OUT
WIDTHS = (IN, HIDDEN, HIDDEN, HIDDEN, HIDDEN, OUT)


def param_layout():
    """[(name, offset, shape)] of the flat parameter vector (W_l row-major [out][in])."""
    out, off = [], 0
    for l in range(5):
        ni, no = WIDTHS[l], WIDTHS[l + 1]
        out.append((f"W{l + 1}", off, (no, ni)))
        off += ni * no
        out.append((f"b{l + 1}", off, (no,)))
        off += no
    return out


def split_params(p):
    """W1, b1, ..., W5, b5 views of a flat parameter vector."""
    return {name: p[off:off + int(np.prod(shape))].reshape(shape) for name, off, shape in param_layout()}


def default_train_opts(**kw):
    o = abi.TrainOpts()
    load().flsp_default_train_opts(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def default_learned_opts(**kw):
    o = abi.LearnedOpts()
    load().flsp_default_learned_opts(C.byref(o))
    for k, v in kw.items():
        if k == "fallback_pseudo_steps":
            o.fallback.n_pseudo_steps = v
        else:
            setattr(o, k, v)
    return o


class MLP:
    def __init__(self, device=0, seed=0):
        L = load()
        h = C.c_void_p()
        check(L.flsp_mlp_create(int(device), C.c_uint64(seed), C.byref(h)))
        self.h = h
        n = C.c_int64(0)
        check(L.flsp_mlp_n_params(C.byref(n)))
        self.n_params = n.value

    def close(self):
        if getattr(self, "h", None):
            load().flsp_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def get_params(self):
        p = np.empty(self.n_params, dtype=np.float32)
        check(load().flsp_mlp_get_params(self.h, fp(p), p.size))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(load().flsp_mlp_set_params(self.h, fp(p), p.size))

    def forward(self, x):
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, IN)
        y = np.empty((x.shape[0], OUT), dtype=np.float32)
        check(load().flsp_mlp_forward(self.h, fp(x), x.shape[0], fp(y)))
        return y

    def backward(self, x, dy):
        """gradient of sum(dy * net(x)) w.r.t. the parameters, summed over the batch"""
        x = np.ascontiguousarray(x, dtype=np.float32).reshape(-1, IN)
        dy = np.ascontiguousarray(dy, dtype=np.float32).reshape(-1, OUT)
        g = np.empty(self.n_params, dtype=np.float32)
        check(load().flsp_mlp_backward(self.h, fp(x), fp(dy), x.shape[0], fp(g)))
        return g

    def collect(self, problem, band_cells=6.0, target=None):
        """training pairs from a Problem (its state is reinitialised by `target`)"""
        if target is None:
            target = abi.ReinitOpts()
            load().flsp_default_reinit_opts(C.byref(target))
            target.mode = abi.REINIT_FIXED
            target.n_pseudo_steps = 20
        n = C.c_int64(0)
        check(load().flsp_mlp_collect(self.h, problem.h, float(band_cells), C.byref(target), C.byref(n)))
        return n.value

    @property
    def n_pairs(self):
        n = C.c_int64(0)
        check(load().flsp_mlp_n_pairs(self.h, C.byref(n)))
        return n.value

    def clear_pairs(self):
        check(load().flsp_mlp_clear_pairs(self.h))

    def train(self, steps, batch=8192, lr=1e-3, seed=1):
        o = default_train_opts(steps=int(steps), batch=int(batch), lr=float(lr), seed=int(seed))
        loss = C.c_double(0.0)
        check(load().flsp_mlp_train(self.h, C.byref(o), C.byref(loss)))
        return loss.value

    def eval(self):
        loss = C.c_double(0.0)
        check(load().flsp_mlp_eval(self.h, C.byref(loss)))
        return loss.value

    def reinit(self, problem, opts=None):
        """learned reinitialisation of a Problem's state; returns the stats"""
        o = opts if opts is not None else default_learned_opts()
        st = abi.LearnedStats()
        check(load().flsp_reinit_learned(problem.h, self.h, C.byref(o), C.byref(st)))
        return {"n_band": st.n_band, "n_fallback": st.n_fallback, "hj_ran": bool(st.hj_ran)}
