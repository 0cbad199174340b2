"""The device cohesive law, case by case, against the reference.

icf_cz_law_eval runs the law exactly as the assembly's CZ kernel does
(cohesive_law_thermodynamically_consistent, cz_kernels9/cz_kernels.h:37-174,
on the PPR functions of PPR_math.h:2-57): the fast law, and where it leaves a
failure test within rounding of its threshold, the reference's own expressions
with pow correctly rounded.

Bar: the contact and failure flags and the updated pmax/tmax equal the
oracle's; the tractions within 1e-12 of max(|T|, strength) and the tangents
within 1e-12 of max(|D|, strength/del) per state (the law's own scales: at a
zero opening Tn_ and Tt_ are rounding noise of order 1e-16 of the strength).
"""
from __future__ import annotations

from pathlib import Path

import numpy as np
import pytest

from tests.harness import Oracle, orc_prms_from
from tests.law_cases import oracle_law, pinned, threshold_cases

from icflow_b200.gpu_functionality import GPU_Functionality
from icflow_b200.model_prms import config_prms

GOLDEN = Path(__file__).resolve().parent / "golden"
TOL = 1e-12


@pytest.fixture(scope="module")
def law_env():
    prms = config_prms()
    gf = GPU_Functionality(0)
    gf.prms = prms
    gf.SetConstants()
    O = Oracle()
    p = orc_prms_from(O, prms)
    yield gf, O, p
    gf.close()


def _value_errors(law_ref, law_dev, sig, deln):
    dT = np.abs(law_dev[:, :2] - law_ref[:, :2]).max(axis=1)
    sT = np.maximum(np.abs(law_ref[:, :2]).max(axis=1), sig)
    dD = np.abs(law_dev[:, 2:5] - law_ref[:, 2:5]).max(axis=1)
    sD = np.maximum(np.abs(law_ref[:, 2:5]).max(axis=1), sig / deln)
    return float((dT / sT).max()), float((dD / sD).max())


@pytest.mark.gpu
def test_law_matches_reference_golden(law_env):
    """The 400 golden states the reference kernel code evaluated (all branches)."""
    gf, O, p = law_env
    g = np.load(GOLDEN / "cz_law.npz")
    pm, tm, law, fl = gf.CZLaw(g["pmax"], g["tmax"], g["opn"], g["opt"])
    assert np.array_equal(fl[:, 0], g["flags"][:, 0]), "contact flags differ"
    assert np.array_equal(fl[:, 1], g["flags"][:, 1]), "failure flags differ"
    assert np.array_equal(pm, g["pmax_out"]) and np.array_equal(tm, g["tmax_out"])
    eT, eD = _value_errors(g["law"][:, :5], law, 1e6, p.ppr.deln)
    assert eT <= TOL and eD <= TOL, (eT, eD)


@pytest.mark.gpu
def test_law_random_states_with_per_cz_strengths(law_env):
    """20k random states, lognormal strengths, every branch of the law."""
    gf, O, p = law_env
    rng = np.random.default_rng(11)
    n = 20000
    sig = np.exp(rng.normal(np.log(1e6) - 0.0196, 0.198, n))
    qs = [O.ppr_for(p, s, s) for s in sig]
    dn = np.array([q.deln for q in qs])
    dt = np.array([q.delt for q in qs])
    pmx = rng.random(n) * dn * 0.8 * (rng.random(n) > 0.3)
    tmx = rng.random(n) * dt * 0.8 * (rng.random(n) > 0.3)
    opn = (rng.random(n) * 2.1 - 1.0) * dn
    opt = rng.random(n) * 1.05 * dt
    cases = np.stack([pmx, tmx, opn, opt, sig], axis=1)
    pm_o, tm_o, law_o, fl_o = oracle_law(O, p, cases)
    pm, tm, law, fl = gf.CZLaw(pmx, tmx, opn, opt, np.stack([sig, sig], axis=1))
    assert np.array_equal(fl[:, :2], fl_o), np.nonzero((fl[:, :2] != fl_o).any(axis=1))[0][:10]
    assert np.array_equal(pm, pm_o) and np.array_equal(tm, tm_o)
    ok = fl_o[:, 1] == 0
    eT, eD = _value_errors(law_o[ok], law[ok], sig[ok, None].ravel(), dn[ok])
    assert eT <= TOL and eD <= TOL, (eT, eD)
    print(f"random states: T {eT:.1e}, D {eD:.1e}; settled exactly: {int(fl[:, 2].sum())}")


@pytest.mark.gpu
def test_law_flags_at_the_thresholds(law_env):
    """States a few ulps either side of every flip of the oracle's failure
    flag: the 5 % tests past the peak (normal, tangential, in contact), the
    -1e-9 test at zero opening (where the reference's rounding noise decides,
    at the strength where it crosses), and the comparisons on the inputs.
    Every state whose pow calls the host C library rounds correctly (all of
    them here) must give the oracle's flags exactly."""
    gf, O, p = law_env
    cases = threshold_cases(O, p)
    pm_o, tm_o, law_o, fl_o = oracle_law(O, p, cases)
    pm, tm, law, fl = gf.CZLaw(cases[:, 0], cases[:, 1], cases[:, 2], cases[:, 3],
                               np.stack([cases[:, 4], cases[:, 4]], axis=1))
    pin = np.array([pinned(O.ppr_for(p, s, s), a, b) for (_, _, a, b, s) in cases])
    assert pin.mean() > 0.95
    bad = np.nonzero(pin & (fl[:, :2] != fl_o).any(axis=1))[0]
    assert len(bad) == 0, [(cases[i].tolist(), fl[i].tolist(), fl_o[i].tolist()) for i in bad[:5]]
    assert np.array_equal(pm[pin], pm_o[pin]) and np.array_equal(tm[pin], tm_o[pin])
    # both outcomes occur at every kind of threshold
    assert 0.2 < fl_o[:, 1].mean() < 0.8
    print(f"threshold states: {len(cases)}, pinned {int(pin.sum())}, "
          f"settled with the reference's rounding: {int(fl[:, 2].sum())}")
