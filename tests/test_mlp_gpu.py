"""Learned reinitialisation on the GPU: the tensor-core MLP (BF16
operands, FP32 accumulation) against the oracle's FP64 MLP, training on
pairs produced by the HJ sweep, and the band / fallback logic of
flsp_reinit_learned.

Tolerances: the GPU rounds weights, inputs and every hidden activation to
BF16 (8-bit mantissa); with the weights and inputs rounded the same way
for the oracle, the remaining difference is the activations' rounding,
bounded here by 2e-2 of the largest output and 3e-2 (relative Frobenius)
for each parameter gradient.
"""
import numpy as np
import pytest

from felspa_b200 import abi, fields as F
from felspa_b200.learned import MLP, WIDTHS, default_learned_opts, param_layout, split_params
from felspa_b200.level_set import Mesh, Problem

pytestmark = pytest.mark.gpu


def bf16(a):
    torch = pytest.importorskip("torch")
    return torch.tensor(np.asarray(a, dtype=np.float32)).to(torch.bfloat16).float().numpy().astype(np.float64)


def random_params(rng):
    p = []
    for name, off, shape in param_layout():
        if name.startswith("W"):
            p.append(rng.uniform(-1.5, 1.5, size=shape) / np.sqrt(shape[1]))
        else:
            p.append(rng.uniform(-0.1, 0.1, size=shape))
    return np.concatenate([a.ravel() for a in p]).astype(np.float32)


def oracle_weights(p):
    v = split_params(p.astype(np.float64))
    Ws = [bf16(v[f"W{l}"]) for l in range(1, 6)]
    bs = [v[f"b{l}"].copy() for l in range(1, 6)]
    return Ws, bs


@pytest.fixture(scope="module")
def net():
    n = MLP(device=0, seed=3)
    yield n
    n.close()


def test_forward_matches_oracle(net, oracle):
    rng = np.random.default_rng(11)
    p = random_params(rng)
    net.set_params(p)
    x = rng.standard_normal((300, WIDTHS[0])).astype(np.float32)
    y = net.forward(x)
    Ws, bs = oracle_weights(p)
    ref = oracle.mlp_forward(Ws, bs, bf16(x))
    assert np.all(np.isfinite(y))
    assert np.max(np.abs(y - ref)) <= 2e-2 * np.max(np.abs(ref))


def test_backward_matches_oracle(net, oracle):
    rng = np.random.default_rng(12)
    p = random_params(rng)
    net.set_params(p)
    B = 384
    x = rng.standard_normal((B, WIDTHS[0])).astype(np.float32)
    dy = (rng.standard_normal((B, WIDTHS[-1])) / B).astype(np.float32)
    g = net.backward(x, dy)
    Ws, bs = oracle_weights(p)
    dW, db = oracle.mlp_backward(Ws, bs, bf16(x), bf16(dy))
    gv = split_params(g.astype(np.float64))
    for l in range(5):
        for got, ref in ((gv[f"W{l + 1}"], dW[l]), (gv[f"b{l + 1}"], db[l])):
            err = np.linalg.norm(got - ref) / np.linalg.norm(ref)
            assert err <= 3e-2, (l, err)


def test_backward_two_calls_identical(net):
    rng = np.random.default_rng(13)
    net.set_params(random_params(rng))
    x = rng.standard_normal((256, WIDTHS[0])).astype(np.float32)
    dy = rng.standard_normal((256, WIDTHS[-1])).astype(np.float32)
    assert np.array_equal(net.backward(x, dy), net.backward(x, dy))


def make_problem(n=64, seed=0, precision=abi.FP32):
    pb = Problem(Mesh(2, (n, n)), 2, basis=abi.BASIS_Q, precision=precision, cfl_max=0.1)
    pb.set_velocity(F.fourier_stream_2d(seed=1000 + seed))
    pb.project(F.circles_union(1000 + seed))
    return pb


def advance(pb, n_steps):
    from felspa_b200.lib import check, load
    check(load().flsp_advance_steps(pb.h, int(n_steps), 1e30))


def test_training_reduces_loss():
    net = MLP(device=0, seed=5)
    for s in range(6):
        pb = make_problem(64, s)
        for _ in range(3):
            advance(pb, 20)
            net.collect(pb, band_cells=6.0)
        pb.close()
    assert net.n_pairs > 2000
    before = net.eval()
    last = net.train(steps=300, batch=1024, lr=1e-3, seed=2)
    after = net.eval()
    assert np.isfinite(last) and np.isfinite(after)
    assert after < 0.5 * before, (before, after)
    net.close()


def test_learned_band_and_forced_fallback():
    net = MLP(device=0, seed=6)
    pb = make_problem(48, 7, precision=abi.FP64)
    advance(pb, 30)
    pre = pb.get_state()
    h = 1.0 / 48
    band = np.abs(pre.reshape(-1, 9)[:, 0]) <= 6.0 * h
    # every band cell fails a zero residual bound: the HJ sweep fills the band
    st = net.reinit(pb, default_learned_opts(max_residual=1e-12))
    assert st["n_band"] == int(band.sum()) and st["n_band"] > 0
    assert st["n_fallback"] == st["n_band"] and st["hj_ran"]
    got = pb.get_state().reshape(-1, 9)
    pb.set_state(pre)
    from felspa_b200.lib import check, load
    import ctypes as C
    o = abi.ReinitOpts()
    load().flsp_default_reinit_opts(C.byref(o))
    o.mode = abi.REINIT_FIXED
    o.n_pseudo_steps = 20
    o.narrow_band = 1     # the fallback's default: the sweep restricted to the failed cells,
    # here every band cell (|mean phi| <= 6 h; the sweep's band is measured
    # in cell diameters, sqrt(2) h)
    o.band_cells = 6.0 / np.sqrt(2.0)
    nit = C.c_int(0)
    check(load().flsp_reinit(pb.h, C.byref(o), C.byref(nit)))
    hj = pb.get_state().reshape(-1, 9)
    assert np.array_equal(got[band], hj[band])
    assert np.array_equal(got[~band], pre.reshape(-1, 9)[~band])
    pb.close()
    net.close()


def test_learned_reinit_after_training():
    net = MLP(device=0, seed=8)
    for s in range(4):
        pb = make_problem(64, 20 + s)
        for _ in range(3):
            advance(pb, 20)
            net.collect(pb, band_cells=6.0)
        pb.close()
    net.train(steps=400, batch=2048, lr=1e-3, seed=3)
    pb = make_problem(64, 40)
    advance(pb, 40)
    st = net.reinit(pb, default_learned_opts())
    out = pb.get_state()
    assert np.all(np.isfinite(out))
    assert st["n_band"] > 0 and 0 <= st["n_fallback"] <= st["n_band"]
    pb.close()
    net.close()


def test_learned_graph_periods_match_host_loop():
    """learned periods replayed from CUDA graphs equal the host-driven loop
    (advance, then the learned reinit with no fallback) bit for bit"""
    import ctypes as C
    from felspa_b200.lib import check, load
    net = MLP(device=0, seed=9)
    lo = default_learned_opts(max_residual=1e30)
    a, b = make_problem(48, 11), make_problem(48, 11)
    for _ in range(3):
        advance(a, 8)
        st = net.reinit(a, lo)
        assert st["n_fallback"] == 0 and st["n_band"] > 0
    check(load().flsp_ls_run_steps_learned(b.h, net.h, C.byref(lo), 8, 3 * 8))
    check(load().flsp_sync(b.h))
    assert a.get_time() == b.get_time()
    sa, sb = a.get_state(), b.get_state()
    assert np.all(np.isfinite(sb)) and np.array_equal(sa, sb)
    a.close()
    b.close()
    net.close()


@pytest.mark.parametrize("max_residual", [1e-12, 0.3, 1e30])
def test_learned_graph_periods_with_fallback_match_host_loop(max_residual):
    """learned periods replayed from CUDA graphs with the residual test and
    the HJ fallback decided on the device equal the host loop (advance,
    then flsp_reinit_learned, whose host decides) bit for bit: every band
    cell failing, some failing, none failing (the gated sweep finds no
    tile)"""
    import ctypes as C
    from felspa_b200.lib import check, load
    net = MLP(device=0, seed=12)    # untrained: many cells fail a moderate bound
    lo = default_learned_opts(max_residual=max_residual, fallback_pseudo_steps=4)
    a, b = make_problem(40, 13), make_problem(40, 13)
    fails = []
    for _ in range(3):
        advance(a, 6)
        st = net.reinit(a, lo)
        fails.append(st["n_fallback"])
    check(load().flsp_ls_run_steps_learned(b.h, net.h, C.byref(lo), 6, 3 * 6))
    check(load().flsp_sync(b.h))
    if max_residual < 1e-6:
        assert min(fails) > 0
    if max_residual > 1e6:
        assert max(fails) == 0
    assert a.get_time() == b.get_time()
    sa, sb = a.get_state(), b.get_state()
    assert np.all(np.isfinite(sb)) and np.array_equal(sa, sb)
    a.close()
    b.close()
    net.close()


def test_trained_network_beats_untrained_and_no_reinit_on_held_out_instances():
    """trained on the plain sweep's pairs of some instances, the network
    predicts the sweep's change on instances it has not seen with less
    error than the untrained network and than doing nothing (a zero
    network: the state left as it is)"""
    from felspa_b200.learned import collect_training_pairs
    trained, untrained, zero = MLP(device=0, seed=21), MLP(device=0, seed=21), MLP(device=0, seed=22)
    zero.set_params(np.zeros(zero.n_params, dtype=np.float32))
    collect_training_pairs(trained, n=96, instances=12, periods=6, every=40)
    trained.train(steps=3000, batch=8192, lr=1e-3, seed=4)
    mse = {}
    for name, net in (("trained", trained), ("untrained", untrained), ("zero", zero)):
        net.clear_pairs()
        # held-out instances (seeds the training did not use), the same pairs for every network
        collect_training_pairs(net, n=96, instances=4, periods=3, every=40, first=40)
        mse[name] = net.eval()
    # measured: 0.59 of the zero network's error, 0.47 of the untrained one's
    assert mse["trained"] < 0.75 * mse["zero"], mse
    assert mse["trained"] < 0.75 * mse["untrained"], mse
    for net in (trained, untrained, zero):
        net.close()
