"""Host driver of one implicit time step, mirroring ImplicitModel3
(v3Library/Simulation/ImplicitModel3.cs) on top of the device path.

Per step (ImplicitModel3.Step, :369-435):
  _beginStep (:117-157)      prescribed nodes (anchored surfaces moved by
                              SurfaceFragment dx/dy/dz with applicationTime,
                              non-deformable meshes by their translation) get
                              du = target(t + h) - u; active nodes get the
                              initial guess, du = v h (:149-156) or a learned
                              warm start (warm_start.LearnedWarmStart);
  Newton loop                 InferTentativeValues (device) -> contact pairs
                              and narrow phase -> CreateStructure -> assembly
                              -> linear solve (device MINRES for PARDISO)
                              -> _checkDivergence (:214-245) -> _XtoDU, until
                              minIterations are done and the increment norm
                              converged, diverged or maxIterations ran out;
  accept (:404-417)           AcceptTentativeValues (device) and the CZ
                              damage commit (TransferUpdatedStateToHost).

The time step is fixed: _adjustTimeStep's time-scale factor (:259-287) and the
damage-explosion frame discard are not reproduced.  The node state, the
contact detection, the matrix and the Newton increment stay on the device;
the host reads v once per step (for the guess).  Contact detection is one
device call without a pair list by default (broad_phase="device"); "pairs"
runs the device broad phase and the narrow phase on its pair list, and
"host" the host grid generator (the tentative positions then cross to the
host every iteration).  All three give the same impacts.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field

import numpy as np

from icflow_b200 import mesh as M
from icflow_b200.gpu_functionality import GPU_Functionality
from icflow_b200.model_prms import ModelPrms


@dataclass
class StepStats:
    step: int
    time: float
    iterations: int
    converged: bool
    diverged: bool
    rel_error: float
    cg_iterations: list = field(default_factory=list)
    n_impacts: int = 0
    n_damaged: int = 0
    n_failed_this_step: int = 0
    seconds: float = 0.0


def prescribed_displacement(coll: M.Collection, t: float) -> np.ndarray:
    """Displacement of every prescribed node at time t: anchored surfaces with
    a forcing (Mesh.forced = (mask, dx, dy, dz, applicationTime), attenuated
    by t / applicationTime until it reaches 1, ImplicitModel3.cs:125-133) and
    non-deformable meshes translated with their velocity
    (_positionNonDeformables, :160-175).  Other nodes: zero."""
    d = np.zeros_like(coll.x0)
    off = 0
    for m in coll.meshes:
        n = m.n_nodes
        if not m.isDeformable:
            vel = getattr(m, "velocity", None)
            if vel is not None:
                d[off:off + n] = np.asarray(vel, float) * t
        for (mask, dx, dy, dz, t_app) in getattr(m, "forced", None) or []:
            att = 1.0 if t_app <= t else t / t_app
            idx = off + np.nonzero(mask)[0]
            d[idx] = att * np.array([dx, dy, dz])
        off += n
    return d


class ImplicitModel3:
    """One simulation: a mesh collection, its parameters and the device
    context.  `strengths` gives per-CZ sigma_max (= tau_max)."""

    def __init__(self, coll: M.Collection, prms: ModelPrms, strengths: np.ndarray | None = None,
                 device: int = 0, precision: int = 0, contact: bool = False, rel_tol: float = 1e-12,
                 v0: np.ndarray | None = None, convergence: str = "increment", res_tol: float = 1e-8,
                 broad_phase: str = "device"):
        """convergence: "increment" is the reference's test on NormOfDx
        (_checkDivergence); "residual" stops when ||rhs|| <= res_tol * ||rhs
        at zero increment||, a scale that does not depend on the initial
        guess (used to compare initial guesses)."""
        if convergence not in ("increment", "residual"):
            raise ValueError("convergence is 'increment' or 'residual'")
        self.convergence = convergence
        self.res_tol = res_tol
        if broad_phase not in ("device", "pairs", "host"):
            raise ValueError("broad_phase is 'device', 'pairs' or 'host'")
        self.broad_phase = broad_phase
        self.coll = coll
        self.prms = prms
        self.contact = contact
        self.rel_tol = rel_tol
        gf = self.gf = GPU_Functionality(device)
        gf.prms = prms
        gf.mc = coll
        gf.SetConstants()
        gf.SetPrecision(precision)
        gf.TransferStaticDataToDevice()
        if strengths is not None:
            gf.SetCZStrengths(strengths, strengths)
        n = len(coll.x0)
        nc = len(coll.czs)
        gf.TransferPCSR(np.zeros((nc, 3)), np.zeros((nc, 3)), np.zeros(nc, np.int32))
        v = np.zeros((n, 3)) if v0 is None else np.array(v0, float)
        v[coll.anchored] = 0.0
        gf.SetNodeState(np.zeros((n, 3)), v, np.zeros((n, 3)))
        self.t = 0.0
        self.step_no = 0
        self.active = ~coll.anchored
        self.history: list[StepStats] = []
        self.cz_state = None
        # object with record(model, h, u, v, a, du_prev, du_prev2, du_accepted),
        # called after every accepted step (training data for a warm start)
        self.recorder = None
        # when a list: the impact list of every Newton iteration (contact runs)
        self.trace = None
        # accepted increments of the two previous steps (learned warm start inputs)
        self.du_prev = np.zeros((n, 3))
        self.du_prev2 = np.zeros((n, 3))
        if contact and gf.prms.CollisionScheme == 0:
            raise ValueError("contact needs ModelPrms.CollisionScheme = 1")

    # ---- _beginStep ---------------------------------------------------------
    def initial_guess(self, h: float, u, v, a) -> np.ndarray:
        """du = v h for the active nodes (ImplicitModel3.cs:149-156)."""
        return v * h

    def _check(self, norm: float, it: int, st: dict) -> tuple[bool, bool]:
        """_checkDivergence (ImplicitModel3.cs:214-245) on NormOfDx."""
        p = self.prms
        if it == 0:
            st["E0"] = norm if norm != 0 else p.ConvergenceEpsilon
            st["rel"] = 1.0
            return False, False
        if norm < p.ConvergenceCutoff:
            st["rel"] = -1.0
            return True, False
        rel = float(np.sqrt(norm / st["E0"]))
        st["rel"] = rel
        return rel <= p.ConvergenceEpsilon, rel > 1.01

    def guess_residuals(self, guesses) -> list[float]:
        """Residual norm of the first Newton iterate for each initial guess (du
        of the active nodes, all nodes' shape), relative to the residual at
        zero increment, at the start of the next step; the state is left as
        it was (used to calibrate initial guesses)."""
        gf, p, coll = self.gf, self.prms, self.coll
        h = p.InitialTimeStep
        u, v, a, _ = gf.GetNodeState()
        pres = coll.anchored
        base = np.zeros_like(u)
        base[pres] = prescribed_displacement(coll, self.t + h)[pres] - u[pres]

        def resid(du):
            gf.SetDU(du)
            gf.InferTentativeValues(h)
            if self.contact:
                self._contact()
            gf.CreateStructure(copy_back=False)
            gf.AssembleElemsAndCZs(h)
            return gf.ResidualNorm()

        r0 = resid(base)
        out = []
        for g in guesses:
            du = base.copy()
            du[self.active] = g[self.active]
            out.append(resid(du) / r0 if r0 > 0 else 0.0)
        gf.SetDU(np.zeros_like(u))
        return out

    def _contact(self):
        """Broad and narrow phase at the tentative positions: on the device
        in one call without a pair list ("device"), on the device through the
        pair list ("pairs", which never leaves the device), or with the host
        grid generator ("host").  All three give the same impacts."""
        gf = self.gf
        if self.broad_phase == "device":
            gf.DetectContacts()
        elif self.broad_phase == "pairs":
            gf.BroadPhase()
            gf.NarrowPhaseCollisionDetection(None)
        else:
            uu, _, _, duc = gf.GetNodeState()
            gf.NarrowPhaseCollisionDetection(M.candidate_pairs(self.coll, self.coll.x0 + uu + duc))

    def Step(self, warm_start=None) -> StepStats:
        t0 = time.perf_counter()
        gf, p, coll = self.gf, self.prms, self.coll
        h = p.InitialTimeStep
        t1 = self.t + h
        u, v, a, _ = gf.GetNodeState()
        du = np.zeros_like(u)
        guess = self.initial_guess(h, u, v, a) if warm_start is None else warm_start(self, h, u, v, a)
        du[self.active] = guess[self.active]
        pres = coll.anchored
        du[pres] = prescribed_displacement(coll, t1)[pres] - u[pres]
        it = 0
        st: dict = {}
        converged = diverged = False
        cg = []
        self._n_imp = 0

        def assemble():
            gf.InferTentativeValues(h)
            if self.contact:
                self._contact()
                self._n_imp = gf.nImpacts
                if self.trace is not None:
                    self.trace.append(gf.c_itet.copy())
            gf.CreateStructure(copy_back=False)
            return gf.AssembleElemsAndCZs(h)

        if self.convergence == "residual":
            du0 = np.zeros_like(du)
            du0[pres] = du[pres]
            gf.SetDU(du0)
            assemble()
            r_ref = gf.ResidualNorm()
            gf.SetDU(du)
            while True:
                cnt = assemble()
                r = gf.ResidualNorm()
                st["rel"] = r / r_ref if r_ref > 0 else 0.0
                converged = st["rel"] <= self.res_tol
                if (converged and it >= p.minIterations) or it >= p.maxIterations:
                    break
                k, _, _ = gf.Solve(self.rel_tol)
                cg.append(k)
                gf.ApplyDx()
                it += 1
        else:
            gf.SetDU(du)
            while True:
                cnt = assemble()
                k, _, _ = gf.Solve(self.rel_tol)
                cg.append(k)
                norm = gf.ApplyDx()
                converged, diverged = self._check(norm, it, st)
                it += 1
                if not (it < p.minIterations or (not diverged and not converged and it < p.maxIterations)):
                    break
        n_imp = self._n_imp
        u_before = u
        gf.AcceptTentativeValues(h)
        self.cz_state = gf.TransferUpdatedStateToHost(want_forces=False)
        u_after, _, _, _ = gf.GetNodeState()
        du_acc = u_after - u_before
        if self.recorder is not None:
            self.recorder.record(self, h, u, v, a, self.du_prev, self.du_prev2, du_acc)
        self.du_prev2 = self.du_prev
        self.du_prev = du_acc
        self.t = t1
        self.step_no += 1
        s = StepStats(self.step_no, self.t, it, converged, diverged, st.get("rel", 0.0), cg, n_imp,
                      cnt.nCZDamaged, cnt.nCZFailedThisStep, time.perf_counter() - t0)
        self.history.append(s)
        return s

    def state(self):
        """(u, v, a) of all nodes and the committed CZ state (pmax, tmax,
        failed, averages) of the last accepted step."""
        u, v, a, _ = self.gf.GetNodeState()
        return u, v, a, self.cz_state

    def close(self):
        self.gf.close()
