"""CPU twin of icflow_b200.implicit_model.ImplicitModel3 for N-step parity:
the same time step (ImplicitModel3.Step, ImplicitModel3.cs:369-435) with the
oracle's assembly (oracle/icf_oracle.c), the oracle's Newmark predictor and
commit (Node.cs:62-97) and a direct sparse solve (SuperLU on the symmetric
matrix, standing in for PARDISO, LinearSystem.cs:48-64).  With contact, every
Newton iteration runs the oracle's narrow phase and closest-face search on the
candidate pairs of the tentative positions, adds the impacts to the structure
(_addCollidingNodesToStructure, :177-196) and assembles their penalty terms.
Test infrastructure only."""
from __future__ import annotations

import numpy as np
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from icflow_b200.implicit_model import prescribed_displacement
from oracle.oracle import Oracle


def full_matrix(N: int, rows: np.ndarray, cols: np.ndarray, vals: np.ndarray) -> sp.csr_matrix:
    """A = U + U^T - diag(U) from the upper-triangular 3x3 BCSR."""
    U = sp.bsr_matrix((vals.reshape(-1, 3, 3), cols, rows), shape=(3 * N, 3 * N)).tocsr()
    D = sp.bsr_matrix((vals.reshape(-1, 3, 3) * (cols == np.repeat(np.arange(N), np.diff(rows)))[:, None, None],
                       cols, rows), shape=(3 * N, 3 * N)).tocsr()
    return (U + U.T - D).tocsc()


class OracleModel:
    def __init__(self, coll, prms, strengths=None, v0=None, contact=False):
        self.O = O = Oracle()
        keys = ("Y", "nu", "rho", "dampingMass", "dampingStiffness", "gravity", "NewmarkBeta", "NewmarkGamma",
                "alpha", "beta", "lambda_n", "lambda_t", "phi_n", "phi_t", "sigma_max", "tau_max", "penaltyK",
                "DistanceEpsilon")
        self.p = O.prms(**{k: getattr(prms, k) for k in keys})
        self.prms = prms
        self.coll = coll
        n = len(coll.x0)
        nc = len(coll.czs)
        self.u = np.zeros((n, 3))
        self.v = np.zeros((n, 3)) if v0 is None else np.array(v0, float)
        self.v[coll.anchored] = 0
        self.a = np.zeros((n, 3))
        self.pmax = np.zeros((nc, 3))
        self.tmax = np.zeros((nc, 3))
        self.failed = np.zeros(nc, np.int32)
        self.q = None if strengths is None else [O.ppr_for(self.p, s, s) for s in strengths]
        self.t = 0.0
        self.active = ~coll.anchored
        self.iterations = []
        self.contact = contact
        self.trace = []  # per Newton iteration: the impact list
        self.trace_x = []  # ... and the tentative positions it was found at
        # per step: CZs newly damaged and failed (the counters _checkDamage reads)
        self.damage_counts = []
        imps = np.zeros((0, 4), np.int32)
        # static pattern from every CZ (never shrinks), as the device keeps it
        self.N, self.rows, self.cols = O.build_structure(coll.alt, coll.elems, coll.czs, imps)
        self.ep = O.pcsr(coll.elems, 4, coll.alt, self.rows, self.cols, self.N)
        self.cp = O.pcsr(coll.czs, 6, coll.alt, self.rows, self.cols, self.N)

    def _check(self, norm, it, st):
        p = self.prms
        if it == 0:
            st["E0"] = norm if norm != 0 else p.ConvergenceEpsilon
            return False, False
        if norm < p.ConvergenceCutoff:
            return True, False
        rel = np.sqrt(norm / st["E0"])
        return rel <= p.ConvergenceEpsilon, rel > 1.01

    def Step(self):
        O, p, c = self.O, self.prms, self.coll
        h = p.InitialTimeStep
        t1 = self.t + h
        du = np.zeros_like(self.u)
        du[self.active] = (self.v * h)[self.active]
        pres = c.anchored
        du[pres] = prescribed_displacement(c, t1)[pres] - self.u[pres]
        it = 0
        st = {}
        imps = np.zeros((0, 4), np.int32)
        ip = np.zeros((0, 20), np.int32)
        alt = c.alt
        act = np.nonzero(alt >= 0)[0]
        N, rows, cols, ep, cp = self.N, self.rows, self.cols, self.ep, self.cp
        while True:
            un, vn, an, xt = O.newmark_infer(h, p.NewmarkBeta, p.NewmarkGamma, c.x0, self.u, self.v, self.a, du)
            if self.contact:
                from icflow_b200 import mesh as M

                pairs = M.candidate_pairs(c, xt)
                if len(pairs):
                    masks = O.narrow_phase(pairs, c.selem, xt)
                    imps = O.impacts(pairs, masks, c.selem, c.adj_off, c.adj, c.faces, xt)
                else:
                    imps = np.zeros((0, 4), np.int32)
                self.trace.append(imps.copy())
                self.trace_x.append(xt.copy())
                N, rows, cols = O.build_structure(c.alt, c.elems, c.czs, imps)
                ep = O.pcsr(c.elems, 4, c.alt, rows, cols, N)
                cp = O.pcsr(c.czs, 6, c.alt, rows, cols, N)
                ip = O.pcsr(imps, 4, c.alt, rows, cols, N)
            live = np.nonzero(self.failed == 0)[0]
            res = O.assemble(self.p, h, c.x0, un, vn, an, c.elems, ep, c.czs[live], cp[live],
                             self.pmax[live], self.tmax[live], imps, ip, len(cols), N,
                             cz_ppr=None if self.q is None else [self.q[i] for i in live])
            A = full_matrix(N, rows, cols, res["vals"])
            dx = spla.spsolve(A, res["rhs"].ravel()).reshape(-1, 3)
            du[act] += dx[alt[act]]
            norm = float((dx * dx).sum())
            conv, div = self._check(norm, it, st)
            it += 1
            if not (it < p.minIterations or (not div and not conv and it < p.maxIterations)):
                break
        self.u, self.v, self.a, _, _ = O.newmark_accept(h, c.x0, self.u, self.v, self.a, un, du)
        tent, flags = res["tent"], res["flags"]
        self.damage_counts.append((int((flags[:, 1] != 0).sum()), int((flags[:, 2] != 0).sum())))
        self.pmax[live] = tent[:, :1]
        self.tmax[live] = tent[:, 1:2]
        self.failed[live] |= (flags[:, 2] != 0).astype(np.int32)
        self.t = t1
        self.iterations.append(it)
        return it
