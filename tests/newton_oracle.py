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
    def __init__(self, coll, prms, strengths=None, v0=None, contact=False, step_control=True):
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
        self.accepted = []  # per attempt: accepted by step control
        self.scales = []  # per attempt: its time scale factor
        self.contact = contact
        # step control, as ImplicitModel3 (icflow_b200/implicit_model.py)
        self.step_control = step_control
        self.time_scale = 1
        self.steps_with_factor = 0
        self.int_time = 0
        self.n_damaged_frame = 0
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

    def _damaged_at_level(self):
        """_acceptFrame's count (ImplicitModel3.cs:304-317): non-failed CZs
        with pmax[0] > deln lambda_n or tmax[0] > delt lambda_t."""
        p = self.p
        nc = len(self.failed)
        if self.q is None:
            dn = np.full(nc, p.ppr.deln)
            dt = np.full(nc, p.ppr.delt)
        else:
            dn = np.array([q.deln for q in self.q])
            dt = np.array([q.delt for q in self.q])
        hit = (self.pmax[:, 0] > dn * p.lambda_n) | (self.tmax[:, 0] > dt * p.lambda_t)
        return int((hit & (self.failed == 0)).sum())

    def Step(self):
        """One attempt; returns its Newton iterations (self.accepted[-1] says
        whether step control kept it)."""
        from icflow_b200.implicit_model import HOLD_FACTOR_DELAY, PARTS

        O, p, c = self.O, self.prms, self.coll
        tsf, swf = self.time_scale, self.steps_with_factor
        ticks = PARTS // tsf
        h = p.InitialTimeStep * ticks / PARTS
        t1 = (self.int_time + ticks) * p.InitialTimeStep / PARTS
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
        nc0 = len(self.failed)
        explodes = conv = div = False
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
            flags = res["flags"]
            n_dmg, n_fail = int((flags[:, 1] != 0).sum()), int((flags[:, 2] != 0).sum())
            # _checkDamage (ImplicitModel3.cs:198-212)
            explodes = (self.step_control and tsf != PARTS and nc0 > 0 and
                        ((n_dmg - self.n_damaged_frame) / nc0 > p.maxDamagePerStep or n_fail / nc0 > p.maxFailPerStep))
            A = full_matrix(N, rows, cols, res["vals"])
            dx = spla.spsolve(A, res["rhs"].ravel()).reshape(-1, 3)
            du[act] += dx[alt[act]]
            norm = float((dx * dx).sum())
            conv, div = self._check(norm, it, st)
            it += 1
            if not (it < p.minIterations or (not explodes and not div and not conv and it < p.maxIterations)):
                break
        accept = True
        if self.step_control:
            if explodes:
                self.time_scale = min(tsf * 2, PARTS)
                self.steps_with_factor = HOLD_FACTOR_DELAY
            elif (div or not conv) and tsf < PARTS and p.maxIterations > 1:
                self.time_scale = tsf * 2
                self.steps_with_factor = HOLD_FACTOR_DELAY
            elif conv and tsf > 1:
                if swf > 0:
                    swf -= 1
                else:
                    tsf = max(tsf // 2, 1)
                    swf = 2
            accept = (p.maxIterations == 1 or tsf == PARTS or (not conv and tsf >= PARTS) or
                      (not explodes and not div and conv))
        self.iterations.append(it)
        self.accepted.append(accept)
        self.scales.append(PARTS // ticks)
        self.damage_counts.append((n_dmg, n_fail))
        if not accept:
            return it
        self.u, self.v, self.a, _, _ = O.newmark_accept(h, c.x0, self.u, self.v, self.a, un, du)
        tent = res["tent"]
        self.pmax[live] = tent[:, :1]
        self.tmax[live] = tent[:, 1:2]
        self.failed[live] |= (flags[:, 2] != 0).astype(np.int32)
        self.t = t1
        self.int_time += ticks
        if self.step_control:
            self.time_scale, self.steps_with_factor = tsf, swf
            self.n_damaged_frame = self._damaged_at_level()
        return it
