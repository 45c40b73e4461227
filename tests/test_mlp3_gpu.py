"""The 3D patch network of the learned reinitialisation (3 x 3 x 3 cells of a
3D degree-2 Q state, 27 coefficients each, plus 64 h: 730 -> 256 x 4 ->
27): tensor-core forward and backward against the oracle's FP64 MLP (the
730-wide input takes the column-blocked weight-gradient GEMM), training on
pairs from the 3D HJ sweep, and the band / fallback logic in 3D.

Tolerances as for the 2D network: BF16 weights, inputs and activations on
the GPU, the oracle fed the same rounded weights and inputs; 2e-2 of the
largest output, 3e-2 relative Frobenius per parameter gradient.
"""
import ctypes as C

import numpy as np
import pytest

from felspa_b200 import abi, fields as F
from felspa_b200.learned import MLP, default_learned_opts, param_layout, split_params, widths
from felspa_b200.level_set import Mesh, Problem
from felspa_b200.lib import check, load

pytestmark = pytest.mark.gpu


def bf16(a):
    torch = pytest.importorskip("torch")
    return torch.tensor(np.asarray(a, dtype=np.float32)).to(torch.bfloat16).float().numpy().astype(np.float64)


def random_params(rng):
    p = []
    for name, off, shape in param_layout(3):
        if name.startswith("W"):
            p.append(rng.uniform(-1.5, 1.5, size=shape) / np.sqrt(shape[1]))
        else:
            p.append(rng.uniform(-0.1, 0.1, size=shape))
    return np.concatenate([a.ravel() for a in p]).astype(np.float32)


def oracle_weights(p):
    v = split_params(p.astype(np.float64), 3)
    return [bf16(v[f"W{l}"]) for l in range(1, 6)], [v[f"b{l}"].copy() for l in range(1, 6)]


@pytest.fixture(scope="module")
def net():
    n = MLP(device=0, seed=3, dim=3)
    yield n
    n.close()


def test_dimensions(net):
    W = widths(3)
    assert (net.n_in, net.n_out) == (W[0], W[-1]) == (730, 27)
    assert net.n_params == sum(int(np.prod(s)) for _, _, s in param_layout(3))


def test_forward_matches_oracle(net, oracle):
    rng = np.random.default_rng(21)
    p = random_params(rng)
    net.set_params(p)
    x = rng.standard_normal((300, 730)).astype(np.float32)
    y = net.forward(x)
    Ws, bs = oracle_weights(p)
    ref = oracle.mlp_forward(Ws, bs, bf16(x))
    assert y.shape == (300, 27) and np.all(np.isfinite(y))
    assert np.max(np.abs(y - ref)) <= 2e-2 * np.max(np.abs(ref))


def test_backward_matches_oracle(net, oracle):
    rng = np.random.default_rng(22)
    p = random_params(rng)
    net.set_params(p)
    B = 384
    x = rng.standard_normal((B, 730)).astype(np.float32)
    dy = (rng.standard_normal((B, 27)) / B).astype(np.float32)
    g = net.backward(x, dy)
    Ws, bs = oracle_weights(p)
    dW, db = oracle.mlp_backward(Ws, bs, bf16(x), bf16(dy))
    gv = split_params(g.astype(np.float64), 3)
    for l in range(5):
        for got, ref in ((gv[f"W{l + 1}"], dW[l]), (gv[f"b{l + 1}"], db[l])):
            err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
            assert err <= 3e-2, (l, err)
    # every column block of the first layer's weight gradient
    for c0 in (0, 256, 512):
        blk = slice(c0, min(c0 + 256, 730))
        err = np.linalg.norm(gv["W1"][:, blk] - dW[0][:, blk]) / np.linalg.norm(dW[0][:, blk])
        assert err <= 3e-2, (c0, err)


def make_problem(n=20, seed=0, precision=abi.FP32):
    pb = Problem(Mesh(3, (n, n, n)), 2, basis=abi.BASIS_Q, precision=precision, cfl_max=0.1)
    pb.set_velocity(F.deformation_3d())
    r = np.random.default_rng(500 + seed)
    c = r.uniform(0.35, 0.65, 3)
    pb.project(F.sphere(tuple(float(v) for v in c), float(r.uniform(0.15, 0.25))))
    return pb


def advance(pb, n_steps):
    check(load().flsp_advance_steps(pb.h, int(n_steps), 1e30))


def target_opts():
    return abi.default_reinit_opts(mode=abi.REINIT_FIXED, n_pseudo_steps=5)


def test_network_dimension_must_match_problem():
    net2 = MLP(device=0, seed=1, dim=2)
    pb = make_problem(8, 0)
    with pytest.raises(Exception):
        net2.reinit(pb, default_learned_opts())
    pb.close()
    net2.close()


def test_training_reduces_loss_3d():
    """pairs from states scaled by random factors (the same interface, not
    a distance function): the sweep's correction is learnable"""
    net = MLP(device=0, seed=5, dim=3)
    rng = np.random.default_rng(5)
    for s in range(3):
        pb = make_problem(20, s)
        for _ in range(3):
            advance(pb, 15)
            pb.set_state(pb.get_state() * float(rng.uniform(0.5, 2.0)))
            net.collect(pb, band_cells=6.0, target=target_opts())
        pb.close()
    assert net.n_pairs > 2000
    before = net.eval()
    last = net.train(steps=400, batch=1024, lr=1e-3, seed=2)
    after = net.eval()
    assert np.isfinite(last) and np.isfinite(after)
    assert after < 0.5 * before, (before, after)
    net.close()


def test_learned_band_and_forced_fallback_3d():
    net = MLP(device=0, seed=6, dim=3)
    n = 16
    pb = make_problem(n, 7, precision=abi.FP64)
    advance(pb, 10)
    pre = pb.get_state()
    band = np.abs(pre.reshape(-1, 27)[:, 0]) <= 6.0 / n
    # every band cell fails a zero residual bound: the HJ sweep fills the band
    st = net.reinit(pb, default_learned_opts(max_residual=1e-12))
    assert st["n_band"] == int(band.sum()) and st["n_band"] > 0
    assert st["n_fallback"] == st["n_band"] and st["hj_ran"]
    got = pb.get_state().reshape(-1, 27)
    pb.set_state(pre)
    o = abi.ReinitOpts()
    load().flsp_default_reinit_opts(C.byref(o))
    o.mode = abi.REINIT_FIXED
    o.n_pseudo_steps = 20
    o.narrow_band = 1
    o.band_cells = 6.0
    nit = C.c_int(0)
    check(load().flsp_reinit(pb.h, C.byref(o), C.byref(nit)))
    hj = pb.get_state().reshape(-1, 27)
    assert np.array_equal(got[band], hj[band])
    assert np.array_equal(got[~band], pre.reshape(-1, 27)[~band])
    pb.close()
    net.close()


def test_zero_network_leaves_band_unchanged():
    """a network with all parameters zero predicts no change: without the
    fallback the state comes back exactly"""
    net = MLP(device=0, seed=9, dim=3)
    net.set_params(np.zeros(net.n_params, dtype=np.float32))
    pb = make_problem(12, 3, precision=abi.FP64)
    advance(pb, 5)
    pre = pb.get_state()
    st = net.reinit(pb, default_learned_opts(max_residual=1e30))
    assert st["n_band"] > 0 and st["n_fallback"] == 0 and not st["hj_ran"]
    assert np.array_equal(pb.get_state(), pre)
    pb.close()
    net.close()
