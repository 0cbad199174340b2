"""The warm-start network's CPU restatement (oracle/mlp_oracle.py): its
gradient against central finite differences, and its bf16 rounding."""
import numpy as np

from oracle.mlp_oracle import NI, NO, bf16, loss_and_grad


def _params(seed):
    rng = np.random.default_rng(seed)
    sizes = [64 * NI, 64, 64 * 64, 64, NO * 64, NO]
    return np.concatenate([rng.normal(0, 0.3, n) for n in sizes])


def test_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = _params(1)
    norm = np.concatenate([rng.normal(size=NI), rng.uniform(0.5, 2, NI), np.ones(NO)])
    x = rng.normal(size=(40, NI))
    t = rng.normal(size=(40, NO))
    _, g = loss_and_grad(p, norm, x, t, round=False)
    for i in rng.choice(len(p), 40, replace=False):
        e = np.zeros_like(p)
        e[i] = 1e-6
        fd = (loss_and_grad(p + e, norm, x, t, False)[0] - loss_and_grad(p - e, norm, x, t, False)[0]) / 2e-6
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(g[i])), (i, fd, g[i])


def test_bf16_rounding():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -9, -3.140625, 0.0, 1e-30], np.float32)
    r = bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # the midpoint 1 + 2^-8 ties to the even neighbour
    assert r[2] == np.float32(1.0 + 2 ** -7)  # 1 + 1.5 ulp rounds up
    assert r[3] == np.float32(-3.140625) and r[4] == 0.0
    # bf16 keeps 8 significant bits
    assert np.all(np.abs(r - x) <= np.abs(x) * 2 ** -8 + 1e-38)


def test_trace_check_accepts_the_restatement_and_catches_planted_errors():
    """check_trace on the restatement's own float32 trace passes; a hidden
    activation moved by one bf16 unit, or a pre-activation moved well beyond
    float32 summation error, fails it (the mistakes are planted in the
    restatement's trace, on the CPU)."""
    from oracle.mlp_oracle import check_trace, forward

    rng = np.random.default_rng(4)
    p = _params(4).astype(np.float32)
    norm = np.concatenate([rng.normal(size=NI), rng.uniform(0.5, 2, NI), np.ones(NO)]).astype(np.float32)
    x = (rng.normal(size=(300, NI)) / norm[NI:2 * NI] + norm[:NI]).astype(np.float32)
    c = forward(p, norm, x)
    tr = {k: c[k] for k in ("z1", "h1", "z2", "h2", "y")}
    rep = check_trace(p, norm, x, tr)
    assert rep["mismatched"] == 0 and max(rep["z1"], rep["z2"], rep["z3"]) <= 1.0, rep
    h1 = tr["h1"].copy()
    h1.view(np.uint32)[7, 11] += 0x10000
    assert check_trace(p, norm, x, dict(tr, h1=h1))["mismatched"] == 1
    z2 = tr["z2"].copy()
    z2[3, 4] += 1e-2 * (abs(z2[3, 4]) + 1)
    assert check_trace(p, norm, x, dict(tr, z2=z2))["z2"] > 1.0
