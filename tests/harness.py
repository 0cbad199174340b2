"""Parity harness shared by the tests and smoke(): runs the CUDA path through
the C ABI and the CPU oracle on the same seeded state and compares them.

Tolerances (FP64): per-unit and per-block-row normwise relative error
<= 1e-12 (max |difference| over a block row of the matrix divided by the max
|entry| of that row; the whole rhs vector in the infinity norm), because the
reference sums contributions with atomics in arbitrary order, so entrywise
relative error on cancelling entries is meaningless.  Integer outputs
(pattern, slot maps, masks, impacts, flags) must be bit-exact.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

from oracle.oracle import Oracle  # noqa: E402

from icflow_b200.model_prms import ModelPrms  # noqa: E402

FP64_TOL = 1e-12


def orc_prms_from(O: Oracle, prms: ModelPrms):
    keys = ("Y", "nu", "rho", "dampingMass", "dampingStiffness", "gravity", "NewmarkBeta",
            "NewmarkGamma", "alpha", "beta", "lambda_n", "lambda_t", "phi_n", "phi_t", "sigma_max",
            "tau_max", "penaltyK", "DistanceEpsilon")
    return O.prms(**{k: getattr(prms, k) for k in keys})


def random_state(coll, seed: int, du: float, dv: float = 1.0, da: float = 1.0):
    """Tentative un, vn, an with displacements of magnitude `du`; anchored
    nodes keep zero displacement."""
    rng = np.random.default_rng(seed)
    n = len(coll.x0)
    un = (rng.random((n, 3)) - 0.5) * du
    vn = (rng.random((n, 3)) - 0.5) * dv
    an = (rng.random((n, 3)) - 0.5) * da
    un[coll.anchored] = 0.0
    return un, vn, an


def rowwise_rel(rows: np.ndarray, ref: np.ndarray, got: np.ndarray) -> float:
    """max over block rows of max|got-ref| / max|ref| within the row."""
    d = np.abs(got - ref).reshape(len(ref), -1).max(axis=1)
    m = np.abs(ref).reshape(len(ref), -1).max(axis=1)
    row_of = np.repeat(np.arange(len(rows) - 1), np.diff(rows))
    dm = np.zeros(len(rows) - 1)
    mm = np.zeros(len(rows) - 1)
    np.maximum.at(dm, row_of, d)
    np.maximum.at(mm, row_of, m)
    ok = mm > 0
    if np.any(~ok & (dm > 0)):
        return np.inf
    return float((dm[ok] / mm[ok]).max()) if ok.any() else 0.0


def vec_rel(ref, got) -> float:
    s = np.abs(ref).max()
    return float(np.abs(got - ref).max() / s) if s > 0 else float(np.abs(got).max())


def oracle_assemble(O, p, coll, state, h, pmax, tmax, impacts, cz_sigma=None, cz_live=None):
    """Structure, slot maps and assembly by the oracle.  cz_live selects the
    CZs in the static pattern (those not failed when it is first built)."""
    un, vn, an = state
    czs = coll.czs if cz_live is None else coll.czs[cz_live]
    N, rows, cols = O.build_structure(coll.alt, coll.elems, czs, impacts)
    ep = O.pcsr(coll.elems, 4, coll.alt, rows, cols, N)
    cp = O.pcsr(coll.czs, 6, coll.alt, rows, cols, N)
    ip_ = O.pcsr(impacts, 4, coll.alt, rows, cols, N)
    q = None
    if cz_sigma is not None:
        q = [O.ppr_for(p, s, t) for s, t in zip(*cz_sigma)]
    live = np.ones(len(coll.czs), bool) if cz_live is None else cz_live
    czsel = np.nonzero(live)[0]
    res = O.assemble(p, h, coll.x0, un, vn, an, coll.elems, ep, coll.czs[czsel], cp[czsel],
                     pmax[czsel], tmax[czsel], impacts, ip_, len(cols), N,
                     cz_ppr=None if q is None else [q[i] for i in czsel])
    res.update(N=N, rows=rows, cols=cols, epcsr=ep, cpcsr=cp, ipcsr=ip_, czsel=czsel)
    return res


def gpu_assemble(gf, coll, state, h, pmax, tmax, failed, impacts=None, pairs=None):
    """icflow_b200 path through the C ABI.  Either `impacts` (given list) or
    `pairs` (narrow phase on the device) supplies the contacts."""
    un, vn, an = state
    gf.TransferNodesToGPU(un, vn, an)
    gf.TransferPCSR(pmax, tmax, failed)
    if pairs is not None:
        gf.NarrowPhaseCollisionDetection(pairs)
    elif impacts is not None:
        gf.SetImpacts(impacts)
    N, nnz = gf.CreateStructure()
    cnt = gf.AssembleElemsAndCZs(h)
    vals, rhs = gf.TransferLinearSystemToHost()
    tent, flags, avg = gf.GetCZTentative()
    return dict(N=N, rows=gf.linearSystem.csr_rows.copy(), cols=gf.linearSystem.csr_cols.copy(),
                vals=vals.reshape(-1, 3, 3).copy(), rhs=rhs.copy(), tent=tent, flags=flags, avg=avg,
                counts=cnt, epcsr=gf.GetPCSR(0), cpcsr=gf.GetPCSR(1),
                ipcsr=gf.GetPCSR(2) if gf.nImpacts else np.zeros((0, 20), np.int32))


def compare(gpu: dict, orc: dict, check_cz: bool = True) -> dict:
    """Returns the error report; raises AssertionError on any parity failure."""
    rep = {}
    assert gpu["N"] == orc["N"], (gpu["N"], orc["N"])
    assert np.array_equal(gpu["rows"], orc["rows"]), "csr_rows differ"
    assert np.array_equal(gpu["cols"], orc["cols"]), "csr_cols differ"
    assert np.array_equal(gpu["epcsr"], orc["epcsr"]), "element slot maps differ"
    assert np.array_equal(gpu["cpcsr"], orc["cpcsr"]), "CZ slot maps differ"
    if len(orc["ipcsr"]):
        assert np.array_equal(gpu["ipcsr"], orc["ipcsr"]), "impact slot maps differ"
    rep["vals_rowwise"] = rowwise_rel(orc["rows"], orc["vals"], gpu["vals"])
    rep["rhs"] = vec_rel(orc["rhs"], gpu["rhs"])
    assert rep["vals_rowwise"] <= FP64_TOL, rep
    assert rep["rhs"] <= FP64_TOL, rep
    if check_cz and len(orc["czsel"]):
        sel = orc["czsel"]
        assert np.array_equal(gpu["flags"][sel], orc["flags"]), "CZ flags differ"
        rep["tent"] = vec_rel(orc["tent"], gpu["tent"][sel]) if orc["tent"].size else 0.0
        rep["avg"] = vec_rel(orc["avg"], gpu["avg"][sel]) if orc["avg"].size else 0.0
        assert rep["tent"] <= FP64_TOL and rep["avg"] <= FP64_TOL, rep
    return rep
