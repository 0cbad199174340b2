"""Whole time steps on the device (ImplicitModel3 mirror): N-step parity of
displacements and damage state with the CPU twin (oracle assembly + direct
solve), without and with contact, FP32-mixed against FP64 at equal converged
displacements."""
import numpy as np
import pytest

from icflow_b200 import mesh as M
from icflow_b200.implicit_model import ImplicitModel3
from icflow_b200.model_prms import config_prms
from tests.newton_oracle import OracleModel

pytestmark = pytest.mark.gpu


def fast_cantilever(rate=0.2):
    """cfg0 beam with the tip driven at `rate` m/s so that the mid-span CZs
    damage within a few dozen steps."""
    c = M.cantilever()
    m = c.meshes[0]
    tip = np.isclose(m.x0[:, 0], 0.6)
    m.forced = [(tip, 0.0, 0.0, rate, 1.0)]
    return c


def _prms(eps=0.005):
    p = config_prms()
    p.InitialTimeStep = 1e-4
    p.ConvergenceEpsilon = eps
    return p


def _rel(a, b):
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-300))


def test_newton_steps_match_oracle():
    """40 steps at a fixed time step (step control off in both): per-step
    iteration counts equal; displacements, velocities and CZ damage state
    (pmax, tmax, failed) match the CPU twin."""
    c = fast_cantilever()
    p = _prms()
    g = ImplicitModel3(c, p, step_control=False)
    o = OracleModel(c, p, step_control=False)
    for _ in range(40):
        sg = g.Step()
        so = o.Step()
        assert sg.iterations == so
    u, v, a, cz = g.state()
    assert _rel(u, o.u) <= 1e-8, _rel(u, o.u)
    assert _rel(v, o.v) <= 1e-6, _rel(v, o.v)
    assert o.pmax.max() > 0, "no damage developed; the case does not test the CZ commit"
    assert _rel(cz["pmax"], o.pmax) <= 1e-8 and _rel(cz["tmax"], o.tmax) <= 1e-8
    assert np.array_equal(cz["failed"], o.failed)
    g.close()


def test_step_control_matches_oracle():
    """Step control (_checkDamage, _adjustTimeStep, the accept rule;
    ImplicitModel3.cs:198-212, 259-287, 417-421) against the CPU twin: the
    cantilever's tip driven at 3 m/s damages more than 1 % of its 32 CZs in
    one step, so attempts are discarded and the time scale factor doubles
    up to FrameInfo.Parts, then relaxes after converged steps.  Per attempt:
    equal iterations, time scale factor and accept decision; afterwards
    equal displacements, velocities and CZ state."""
    c = fast_cantilever(3.0)
    p = _prms()
    g = ImplicitModel3(c, p)
    o = OracleModel(c, p)
    for k in range(60):
        sg = g.Step()
        so = o.Step()
        assert (sg.iterations, sg.time_scale, sg.accepted) == (so, o.scales[-1], o.accepted[-1]), (k, sg)
    discards = sum(not s.accepted for s in g.history)
    assert discards >= 10 and max(s.time_scale for s in g.history) == 32768, discards
    u, v, a, cz = g.state()
    assert _rel(u, o.u) <= 1e-8, _rel(u, o.u)
    assert _rel(v, o.v) <= 1e-6, _rel(v, o.v)
    assert _rel(cz["pmax"], o.pmax) <= 1e-8 and _rel(cz["tmax"], o.tmax) <= 1e-8
    assert np.array_equal(cz["failed"], o.failed)
    print(f"step control: 60 attempts, {discards} discarded, simulated time {g.t:.3e} s, u {_rel(u, o.u):.1e}")
    g.close()


def test_fp32_mixed_equal_converged_displacements():
    """FP32 Hessians converge to the FP64 displacements within 1e-6 relative
    (the rhs, and so the converged solution, is FP64 in both)."""
    c = fast_cantilever()
    p = _prms(eps=1e-9)
    runs = []
    for prec in (0, 1):
        g = ImplicitModel3(c, p, precision=prec, step_control=False)
        for _ in range(30):
            g.Step()
        u, _, _, cz = g.state()
        runs.append((u, cz, [s.iterations for s in g.history]))
        g.close()
    (u64, cz64, it64), (u32, cz32, it32) = runs
    err = _rel(u32, u64)
    print(f"FP32-mixed vs FP64 after 30 steps: displacement {err:.2e}; iterations {sum(it32)} vs {sum(it64)}")
    assert err <= 1e-6
    # damage history: the openings are ~1e-8 m, so their absolute error is of
    # the order of the displacement error (~1e-13 m), a few 1e-5 of pmax
    assert _rel(cz32["pmax"], cz64["pmax"]) <= 1e-3
    assert np.array_equal(cz32["failed"], cz64["failed"])


def test_contact_steps_converge():
    """Polycrystal between closing platens: the Newton loop with device narrow
    phase, pattern rebuild, assembly and MINRES converges every step."""
    # penalty scaled to the 1 mm specimen so that contact stresses stay near
    # the CZ strengths (with 1e6 and above the first contact steps crush
    # whole grain boundaries and the Newton loop diverges, as the reference's
    # would without its time-step reduction)
    c = M.polycrystal(n=6, grains=6, seed=1, platens=True, gap=-0.01)
    p = config_prms(penaltyK=1e3)
    p.InitialTimeStep = 1e-5
    p.CollisionScheme = 1
    sig = M.lognormal_strengths(len(c.czs), seed=1, granule_pairs=c.meshes[0].cz_grains)
    g = ImplicitModel3(c, p, strengths=sig, contact=True, step_control=False)
    for _ in range(8):
        s = g.Step()
        assert s.converged and not s.diverged, s
    assert any(s.n_impacts > 0 for s in g.history)
    g.close()


def test_contact_steps_match_oracle():
    """20 steps of a polycrystal pressed between closing platens, contact on
    (platen contact and contact across the grain boundaries): every Newton
    iteration's impacts (device broad phase, narrow phase and closest face)
    against the CPU twin's (host pair rule, oracle narrow phase and closest
    face), equal iteration counts, and matching displacements and CZ damage
    state.  The two runs' solves differ by rounding (device MINRES, host
    SuperLU), and a penetrating split-node copy often lies on an edge shared
    by two faces, so the closest face is a tie that rounding decides: the
    twin alone, its solve perturbed by 1e-13, changes such faces too.  So per
    iteration the impacting nodes must be equal, and a face may differ only
    where both faces are at the same distance from the node (to 1e-12 of the
    element size).  Step control is on in both (_checkDamage,
    _adjustTimeStep, ImplicitModel3.cs:198-212, 259-287): every attempt is
    accepted or discarded alike."""
    c = M.polycrystal(n=6, grains=6, seed=1, platens=True, gap=-0.01)
    p = config_prms(penaltyK=1e3)
    p.InitialTimeStep = 1e-5
    p.CollisionScheme = 1
    sig = M.lognormal_strengths(len(c.czs), seed=1, granule_pairs=c.meshes[0].cz_grains)
    g = ImplicitModel3(c, p, strengths=sig, contact=True)
    g.trace = []
    o = OracleModel(c, p, strengths=sig, contact=True)
    for step in range(20):
        sg = g.Step()
        so = o.Step()
        assert sg.iterations == so, (step, sg.iterations, so)
        assert sg.accepted == o.accepted[-1] and sg.time_scale == g.history[-1].time_scale, (step, sg)
        assert sg.accepted <= sg.converged, (step, sg)
    assert len(g.trace) == len(o.trace)
    from oracle.oracle import Oracle

    O = Oracle()
    h_el = float(np.linalg.norm(c.x0[c.elems[0, 1]] - c.x0[c.elems[0, 0]]))
    ties = 0
    for i, (a, b, x) in enumerate(zip(g.trace, o.trace, o.trace_x)):
        assert a.shape == b.shape and np.array_equal(a[:, 0], b[:, 0]), f"impacting nodes differ at iteration {i}"
        for r in np.nonzero((a != b).any(axis=1))[0]:
            p_ = x[a[r, 0]]
            da = O.dtn(x[a[r, 1:]].ravel(), p_)
            db = O.dtn(x[b[r, 1:]].ravel(), p_)
            assert abs(np.sqrt(da) - np.sqrt(db)) <= 1e-12 * h_el, (i, a[r].tolist(), b[r].tolist(), da, db)
            ties += 1
    assert sum(len(t) for t in o.trace) > 0, "no contact: the case does not test the contact path"
    u, v, a, cz = g.state()
    assert _rel(u, o.u) <= 1e-8, _rel(u, o.u)
    assert _rel(v, o.v) <= 1e-6, _rel(v, o.v)
    if o.pmax.max() > 0:
        assert _rel(cz["pmax"], o.pmax) <= 1e-8 and _rel(cz["tmax"], o.tmax) <= 1e-8
    assert np.array_equal(cz["failed"], o.failed)
    print(f"contact parity: 20 steps, {sum(o.iterations)} iterations, "
          f"{sum(len(t) for t in o.trace)} impacts over the iterations ({ties} closest-face ties decided "
          f"differently), u {_rel(u, o.u):.1e}")
    g.close()
