"""The learned warm start on the GPU: the network's forward and gradient
kernels against the CPU restatement, training on the device, and what the
trained network gains over the plain guess du = v h at the same residual
tolerance."""
import numpy as np
import pytest

from icflow_b200.implicit_model import ImplicitModel3
from icflow_b200.warm_start import MLP, LearnedWarmStart, init_params
from oracle.mlp_oracle import NI, NO, check_trace, forward, loss_and_grad
from tests.test_gpu_newton import _prms, fast_cantilever

pytestmark = pytest.mark.gpu


def _setup(seed=0, n=3000):
    rng = np.random.default_rng(seed)
    p = init_params(seed)
    p[-(NO * 64 + NO):] = rng.normal(0, 0.2, NO * 64 + NO).astype(np.float32)
    norm = np.concatenate([rng.normal(size=NI), rng.uniform(0.5, 2, NI), np.ones(NO)]).astype(np.float32)
    x = rng.normal(size=(n, NI)).astype(np.float32) / norm[NI:2 * NI] + norm[:NI]
    return p, norm, x


def test_forward_matches_cpu():
    """Layer by layer (oracle.mlp_oracle.check_trace): every float32
    pre-activation within the float32 summation bound of the float64 value
    from the kernel's own previous layer, every bf16 activation the correct
    rounding of GELU of the kernel's pre-activation (or, within float32
    error of a rounding boundary, its neighbour).  End to end: within 1e-4 of
    the restatement (max-norm relative) on every node where the two made the
    same bf16 roundings; elsewhere a rounding boundary moves one activation
    by one bf16 unit, within 2e-3."""
    p, norm, x = _setup(0, 1037)  # not a multiple of 16
    net = MLP()
    net.set_params(p, norm)
    y = net.forward(x)
    tr = net.forward_trace(x)
    assert np.array_equal(tr["y"], y)
    rep = check_trace(p, norm, x, tr)
    assert rep["mismatched"] == 0 and max(rep["z1"], rep["z2"], rep["z3"]) <= 1.0, rep
    c = forward(p, norm, x)
    ref = c["y"]
    same = (tr["h1"] == c["h1"]).all(axis=1) & (tr["h2"] == c["h2"]).all(axis=1)
    scale = np.abs(ref).max()
    err_same = np.abs(y - ref)[same].max() / scale
    err_all = np.abs(y - ref).max() / scale
    print(f"MLP forward: layer bound ratios {rep}; nodes with equal roundings {same.sum()}/{len(x)}, "
          f"error there {err_same:.1e}, over all nodes {err_all:.1e}")
    assert same.sum() >= len(x) // 2  # measured: 874 of 1037 (the rest hold a near-tie activation)
    assert err_same <= 1e-4, err_same
    assert err_all <= 2e-3, err_all
    net.close()


def test_gradient_matches_cpu():
    p, norm, x = _setup(1, 777)
    t = np.random.default_rng(2).normal(size=(len(x), NO)).astype(np.float32)
    net = MLP()
    net.set_params(p, norm)
    g, loss = net.grad(x, t)
    lref, gref = loss_and_grad(p, norm, x, t)
    assert abs(loss - lref) <= 1e-5 * lref, (loss, lref)
    err = np.abs(g - gref).max() / np.abs(gref).max()
    print(f"MLP gradient vs CPU restatement: {err:.2e} (max-norm relative)")
    assert err <= 1e-5, err
    # identical on a second run (fixed-order reductions)
    g2, _ = net.grad(x, t)
    assert np.array_equal(g, g2)
    net.close()


def test_training_fits_a_smooth_map():
    rng = np.random.default_rng(3)
    x = rng.normal(size=(20000, NI)).astype(np.float32)
    t = np.stack([np.sin(x[:, 0]) + 0.5 * x[:, 3], x[:, 6] * x[:, 9] * 0.3, np.tanh(x[:, 12] - x[:, 1])], 1)
    net = MLP()
    net.set_params(init_params(0), np.concatenate([np.zeros(NI), np.ones(NI), np.ones(NO)]).astype(np.float32))
    _, l0 = net.grad(x, t)
    l1 = net.train(x, t, epochs=40, batch=1024, lr=3e-3, seed=1)
    print(f"training: loss {l0:.3e} -> {l1:.3e}")
    assert l1 < 0.05 * l0
    net.close()


def test_learned_warm_start_reduces_newton_iterations():
    """Train on the method's own trajectories (tip driven at 0.015, 0.02 and
    0.03 m/s, 40 steps each) with the residual-weighted loss, calibrate the
    network's gain on another (0.022 m/s), then run a new one (0.025 m/s)
    with the plain guess du = v h and with the learned one, both to a
    residual tolerance of 1e-8 of the zero-increment residual, minIterations
    1, and compare Newton iterations per step."""
    p = _prms()
    p.minIterations = 1
    p.maxIterations = 20
    ws = LearnedWarmStart(seed=0)
    for rate in (0.015, 0.02, 0.03):
        g = ImplicitModel3(fast_cantilever(rate), p, convergence="residual", res_tol=1e-8,
                           step_control=False)
        g.recorder = ws
        for _ in range(40):
            assert g.Step().converged
        g.close()
    loss = ws.fit_residual(epochs=40, lr=3e-4)
    cal = ImplicitModel3(fast_cantilever(0.022), p, convergence="residual", res_tol=1e-8,
                           step_control=False)
    for _ in range(3):
        cal.Step()
    by_gain = ws.calibrate(cal, 12)
    cal.close()
    its = {}
    for name, warm in (("plain", None), ("learned", ws)):
        m = ImplicitModel3(fast_cantilever(0.025), p, convergence="residual", res_tol=1e-8,
                           step_control=False)
        for _ in range(40):
            s = m.Step(warm_start=warm)
            assert s.converged
        its[name] = np.mean([s.iterations for s in m.history[2:]])
        m.close()
    red = 1 - its["learned"] / its["plain"]
    print(f"warm start: training loss {loss:.3e} (1.0 = extrapolation alone); first-iterate log10 residual by "
          f"gain { {k: round(v, 2) for k, v in by_gain.items()} }, gain {ws.gain}; Newton iterations/step "
          f"plain {its['plain']:.2f}, learned {its['learned']:.2f} ({100 * red:.0f}% fewer)")
    assert its["learned"] <= its["plain"]
    ws.close()
