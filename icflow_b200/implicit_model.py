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
    # step control (_checkDamage, _adjustTimeStep): the attempt's time step
    # and time scale factor, whether the damage check fired and whether the
    # frame was accepted (a discarded attempt leaves the state as it was)
    time_step: float = 0.0
    time_scale: int = 1
    explodes: bool = False
    accepted: bool = True


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


# FrameInfo.Parts = Factor2 (FrameInfo.cs:12-13): the time step is
# InitialTimeStep / TimeScaleFactor, the factor a power of two up to PARTS
PARTS = 1024 * 32
HOLD_FACTOR_DELAY = 4  # ImplicitModel3.cs:257


class ImplicitModel3:
    """One simulation: a mesh collection, its parameters and the device
    context.  `strengths` gives per-CZ sigma_max (= tau_max).

    Step control follows the reference: an attempt whose new damage or new
    failures exceed maxDamagePerStep / maxFailPerStep of the initial CZs
    (_checkDamage, ImplicitModel3.cs:198-212), that diverges or does not
    converge, is discarded and retried with the time scale factor doubled
    (time step halved); after converged steps the factor halves again, each
    change held for a few steps (_adjustTimeStep, :259-287); the accept rule
    is Step's (:417-421).  step_control=False keeps the time step fixed and
    accepts every attempt."""

    def __init__(self, coll: M.Collection, prms: ModelPrms, strengths: np.ndarray | None = None,
                 device: int = 0, precision: int = 0, contact: bool = False, rel_tol: float = 1e-12,
                 v0: np.ndarray | None = None, convergence: str = "increment", res_tol: float = 1e-8,
                 broad_phase: str = "device", step_control: bool = True):
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
        # their time steps (0: no such step yet)
        self.h_prev = 0.0
        self.h_prev2 = 0.0
        # step control: the current frame's TimeScaleFactor and
        # StepsWithCurrentFactor, the integer simulation time in 1/PARTS of
        # InitialTimeStep, the last accepted frame's nCZDamaged, nCZ_Initial
        self.step_control = step_control
        self.time_scale = 1
        self.steps_with_factor = 0
        self.int_time = 0
        self.n_damaged_frame = 0
        self.n_cz_initial = nc
        self.attempts = 0
        if contact and gf.prms.CollisionScheme == 0:
            raise ValueError("contact needs ModelPrms.CollisionScheme = 1")

    # ---- _beginStep ---------------------------------------------------------
    def initial_guess(self, h: float, u, v, a) -> np.ndarray:
        """du = v h for the active nodes (ImplicitModel3.cs:149-156)."""
        return v * h

    def history_increments(self, h: float):
        """The two previous accepted increments scaled to the step h (each
        divided by its own step, times h; zero where there is no such step)."""
        d1 = self.du_prev * (h / self.h_prev) if self.h_prev > 0 else np.zeros_like(self.du_prev)
        d2 = self.du_prev2 * (h / self.h_prev2) if self.h_prev2 > 0 else np.zeros_like(self.du_prev2)
        return d1, d2

    def extrapolation(self, h: float, v) -> np.ndarray:
        """v h + (du_-1 - du_-2) with the increments scaled to h: with the
        reference's accept (v h = du_-1 at a constant step) the linear
        extrapolation of the increments."""
        d1, d2 = self.history_increments(h)
        return v * h + (d1 - d2)

    def time_step(self) -> tuple[float, int]:
        """The next attempt's time step and ticks (FrameInfo.IncrementTime,
        FrameInfo.cs:160-176)."""
        ticks = PARTS // self.time_scale if self.step_control else PARTS
        return self.prms.InitialTimeStep * ticks / PARTS, ticks

    def _check_damage(self, cnt, time_scale: int) -> bool:
        """_checkDamage (ImplicitModel3.cs:198-212)."""
        if not self.step_control or time_scale == PARTS or self.n_cz_initial == 0:
            return False
        p = self.prms
        dn_damaged = (cnt.nCZDamaged - self.n_damaged_frame) / self.n_cz_initial
        dn_failed = cnt.nCZFailedThisStep / self.n_cz_initial
        return dn_damaged > p.maxDamagePerStep or dn_failed > p.maxFailPerStep

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
        h, ticks = self.time_step()
        t1 = (self.int_time + ticks) * p.InitialTimeStep / PARTS
        u, v, a, _ = gf.GetNodeState()
        pres = coll.anchored
        base = np.zeros_like(u)
        base[pres] = prescribed_displacement(coll, t1)[pres] - u[pres]

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
        """One attempt of ImplicitModel3.Step (:369-435): returns its
        statistics; `accepted` is False when step control discarded it."""
        t0 = time.perf_counter()
        gf, p, coll = self.gf, self.prms, self.coll
        # _beginStep: the tentative frame copies the current one
        tsf, swf = self.time_scale, self.steps_with_factor
        tsf_used = tsf
        h, ticks = self.time_step()
        t1 = (self.int_time + ticks) * p.InitialTimeStep / PARTS
        u, v, a, _ = gf.GetNodeState()
        du = np.zeros_like(u)
        guess = self.initial_guess(h, u, v, a) if warm_start is None else warm_start(self, h, u, v, a)
        du[self.active] = guess[self.active]
        pres = coll.anchored
        du[pres] = prescribed_displacement(coll, t1)[pres] - u[pres]
        it = 0
        st: dict = {}
        converged = diverged = explodes = False
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
                explodes = self._check_damage(cnt, tsf)
                r = gf.ResidualNorm()
                st["rel"] = r / r_ref if r_ref > 0 else 0.0
                converged = st["rel"] <= self.res_tol
                if it >= p.minIterations and (converged or explodes or it >= p.maxIterations):
                    break
                k, _, _ = gf.Solve(self.rel_tol)
                cg.append(k)
                gf.ApplyDx()
                it += 1
        else:
            gf.SetDU(du)
            while True:
                cnt = assemble()
                explodes = self._check_damage(cnt, tsf)
                k, _, _ = gf.Solve(self.rel_tol)
                cg.append(k)
                norm = gf.ApplyDx()
                converged, diverged = self._check(norm, it, st)
                it += 1
                if not (it < p.minIterations or
                        (not explodes and not diverged and not converged and it < p.maxIterations)):
                    break
        n_imp = self._n_imp
        accept = True
        if self.step_control:
            # _adjustTimeStep (:259-287): the current frame's factor doubles
            # on a discard; the tentative frame's halves after converged steps
            self.attempts += 1
            if explodes:
                self.time_scale = min(tsf * 2, PARTS)
                self.steps_with_factor = HOLD_FACTOR_DELAY
            elif (diverged or not converged) and tsf < PARTS and p.maxIterations > 1:
                self.time_scale = tsf * 2
                self.steps_with_factor = HOLD_FACTOR_DELAY
            elif converged and tsf > 1:
                if swf > 0:
                    swf -= 1
                else:
                    tsf = max(tsf // 2, 1)
                    swf = 2
            accept = (p.maxIterations == 1 or tsf == PARTS or (not converged and tsf >= PARTS) or
                      (not explodes and not diverged and converged))
        if accept:
            u_before = u
            gf.AcceptTentativeValues(h)
            self.cz_state = gf.TransferUpdatedStateToHost(want_forces=False)
            u_after, _, _, _ = gf.GetNodeState()
            du_acc = u_after - u_before
            if self.recorder is not None:
                self.recorder.record(self, h, u, v, a, self.du_prev, self.du_prev2, du_acc)
            self.du_prev2, self.h_prev2 = self.du_prev, self.h_prev
            self.du_prev, self.h_prev = du_acc, h
            self.t = t1
            self.int_time += ticks
            self.step_no += 1
            if self.step_control:
                # _acceptFrame: the tentative frame becomes the current one
                self.time_scale, self.steps_with_factor = tsf, swf
                self.n_damaged_frame = gf.CountDamagedCZs()
        s = StepStats(self.step_no, t1, it, converged, diverged, st.get("rel", 0.0), cg, n_imp,
                      cnt.nCZDamaged, cnt.nCZFailedThisStep, time.perf_counter() - t0, h, tsf_used, explodes, accept)
        self.history.append(s)
        return s

    def state(self):
        """(u, v, a) of all nodes and the committed CZ state (pmax, tmax,
        failed, averages) of the last accepted step."""
        u, v, a, _ = self.gf.GetNodeState()
        return u, v, a, self.cz_state

    def close(self):
        self.gf.close()
