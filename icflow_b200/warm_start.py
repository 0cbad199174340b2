"""The learned Newton warm start (no counterpart in the reference).

icFlow starts every Newton loop from du = v h (ImplicitModel3.cs:149-156).
LearnedWarmStart replaces that guess for the active nodes with

    du = v h + (d1 - d2) + gain * out_scale * net(x),
    x = (u, v, a, d1, d2)

where d1, d2 are the increments of the two previous accepted steps, each
scaled to the current step (du_k h / h_k; step control changes h), and net is
the per-node MLP of the library (icf_mlp: 15 -> 64 -> 64 -> 3, GELU, BF16
weights, FP32 accumulation, trained on the GPU by the library's own forward
and backward kernels).  Training data are the method's own trajectories:
every accepted step contributes, per active node, the inputs seen at the
start of the step and the correction the Newton loop found beyond the
extrapolation, du_accepted - v h - (d1 - d2).  (With the reference's accept,
v h = du_{n-1} at a constant step, so the first two terms extrapolate the
increments linearly.)

The network is trained per node on displacements, but what the Newton loop
pays for is the force residual of the guess: per-node errors that are not
spatially coherent cost far more force than they save displacement, and
where the extrapolation is already close (free flight, slow loading) any
correction only adds error.  So the correction is judged before it is used:
`calibrate` picks one gain from a separate trajectory, and with
`select_gains` set each step picks the gain whose guess has the smallest
residual (one assembly per candidate, gain 0 being the extrapolation alone).
The plain guess v h stays the fallback and the judge: every arm runs to the
same residual tolerance.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from icflow_b200 import _lib

NI, NO = 15, 3


def features(u, v, a, du1, du2) -> np.ndarray:
    return np.concatenate([u, v, a, du1, du2], axis=1).astype(np.float32)


class MLP:
    """Handle on the library's network (icf_mlp)."""

    def __init__(self, device: int = 0):
        self.lib = _lib.load()
        h = C.c_void_p()
        rc = self.lib.icf_mlp_create(device, C.byref(h))
        if rc:
            raise _lib.ICFError(rc, "icf_mlp_create failed")
        self.h = h
        self.npar = self.lib.icf_mlp_param_count()

    def _check(self, rc):
        if rc:
            raise _lib.ICFError(rc, self.lib.icf_mlp_last_error(self.h).decode())

    def set_params(self, params: np.ndarray, norm: np.ndarray | None = None):
        p = np.ascontiguousarray(params, np.float32)
        assert p.size == self.npar
        n = None if norm is None else np.ascontiguousarray(norm, np.float32)
        self._check(self.lib.icf_mlp_set_params(self.h, p.ctypes.data_as(C.c_void_p),
                                                 None if n is None else n.ctypes.data_as(C.c_void_p)))

    def get_params(self):
        p = np.zeros(self.npar, np.float32)
        n = np.zeros(2 * NI + NO, np.float32)
        self._check(self.lib.icf_mlp_get_params(self.h, p.ctypes.data_as(C.c_void_p), n.ctypes.data_as(C.c_void_p)))
        return p, n

    def forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32).reshape(-1, NI)
        y = np.zeros((len(x), NO), np.float32)
        self._check(self.lib.icf_mlp_forward(self.h, len(x), x.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p)))
        return y

    def forward_trace(self, x: np.ndarray) -> dict:
        """z1, h1, z2, h2 [n, 64] and y [n, 3] of the forward (layer-by-layer checks)."""
        x = np.ascontiguousarray(x, np.float32)
        n = len(x)
        out = {k: np.zeros((n, 64), np.float32) for k in ("z1", "h1", "z2", "h2")}
        out["y"] = np.zeros((n, 3), np.float32)
        ptr = lambda a: a.ctypes.data_as(C.c_void_p)
        self._check(self.lib.icf_mlp_forward_trace(self.h, n, ptr(x), ptr(out["z1"]), ptr(out["h1"]), ptr(out["z2"]),
                                                   ptr(out["h2"]), ptr(out["y"])))
        return out

    def grad(self, x: np.ndarray, y: np.ndarray):
        x = np.ascontiguousarray(x, np.float32).reshape(-1, NI)
        y = np.ascontiguousarray(y, np.float32).reshape(-1, NO)
        g = np.zeros(self.npar, np.float32)
        loss = C.c_float()
        self._check(self.lib.icf_mlp_grad(self.h, len(x), x.ctypes.data_as(C.c_void_p), y.ctypes.data_as(C.c_void_p),
                                          g.ctypes.data_as(C.c_void_p), C.byref(loss)))
        return g, loss.value

    def grad_dy(self, x: np.ndarray, dy: np.ndarray):
        """Backward pass for a caller-defined loss (dy = dL/d output); the
        gradient stays on the device for adam_step."""
        x = np.ascontiguousarray(x, np.float32).reshape(-1, NI)
        dy = np.ascontiguousarray(dy, np.float32).reshape(-1, NO)
        self._check(self.lib.icf_mlp_grad_dy(self.h, len(x), x.ctypes.data_as(C.c_void_p),
                                             dy.ctypes.data_as(C.c_void_p), None))

    def adam_step(self, lr: float):
        self._check(self.lib.icf_mlp_adam_step(self.h, None, float(lr)))

    def train(self, x, y, epochs=20, batch=4096, lr=1e-3, seed=0) -> float:
        x = np.ascontiguousarray(x, np.float32).reshape(-1, NI)
        y = np.ascontiguousarray(y, np.float32).reshape(-1, NO)
        loss = C.c_float()
        self._check(self.lib.icf_mlp_train(self.h, len(x), x.ctypes.data_as(C.c_void_p),
                                           y.ctypes.data_as(C.c_void_p), int(epochs), int(batch), float(lr),
                                           int(seed), C.byref(loss)))
        return loss.value

    def close(self):
        if self.h:
            self.lib.icf_mlp_destroy(self.h)
            self.h = None


def init_params(seed: int = 0) -> np.ndarray:
    """He-style initialisation, last layer zero (the untrained guess is the
    plain one)."""
    rng = np.random.default_rng(seed)
    p = []
    p.append(rng.normal(0, np.sqrt(2 / NI), (64, NI)))
    p.append(np.zeros(64))
    p.append(rng.normal(0, np.sqrt(2 / 64), (64, 64)))
    p.append(np.zeros(64))
    p.append(np.zeros((NO, 64)))
    p.append(np.zeros(NO))
    return np.concatenate([a.ravel() for a in p]).astype(np.float32)


class LearnedWarmStart:
    """Records trajectories, trains the network and serves as the `warm_start`
    of ImplicitModel3.Step."""

    def __init__(self, device: int = 0, seed: int = 0):
        self.net = MLP(device)
        self.net.set_params(init_params(seed))
        self.xs: list[np.ndarray] = []
        self.ys: list[np.ndarray] = []
        self.mats: list = []
        self.norm = None
        self.seed = seed
        self.gain = 1.0

    # ---- data -----------------------------------------------------------------
    def record(self, model, h, u, v, a, du1, du2, du_acc):
        act = model.active
        d1, d2 = model.history_increments(h)
        self.xs.append(features(u, v, a, d1, d2)[act])
        self.ys.append((du_acc - model.extrapolation(h, v))[act].astype(np.float32))
        # the step's last assembled matrix (at the accepted iterate), for the
        # residual-weighted loss
        gf = model.gf
        vals, _ = gf.TransferLinearSystemToHost()
        N = gf.linearSystem.N
        rows = np.zeros(N + 1, np.int32)
        cols = np.zeros(gf.linearSystem.nnz, np.int32)
        _lib.check(gf.ctx, gf.lib.icf_get_structure(gf.ctx, _lib.iptr(rows), _lib.iptr(cols)))
        self.mats.append((N, rows, cols, vals.copy(), model.coll.alt[act].copy()))

    def dataset(self):
        return np.concatenate(self.xs), np.concatenate(self.ys)

    # ---- training ---------------------------------------------------------------
    def fit(self, epochs=30, batch=4096, lr=2e-3) -> float:
        x, y = self.dataset()
        shift = x.mean(axis=0)
        sd = x.std(axis=0)
        scale = 1.0 / np.where(sd > 0, sd, 1.0)
        osd = y.std(axis=0)
        out_scale = np.where(osd > 0, osd, 1.0)
        self.norm = np.concatenate([shift, scale, out_scale]).astype(np.float32)
        p, _ = self.net.get_params()
        self.net.set_params(p, self.norm)
        return self.net.train(x, y / out_scale, epochs=epochs, batch=min(batch, len(x)), lr=lr, seed=self.seed)

    def fit_residual(self, epochs=40, lr=3e-4, warm_epochs=0) -> float:
        """Training on what the Newton loop pays for: per recorded step, the
        force residual the prediction error causes, ||A e||^2, with A the
        step's assembled matrix (symmetric, from its upper blocks) and e the
        error of the predicted correction, normalised by the mean over the
        steps of ||A y||^2 for the true corrections y (so 1.0 is the zero
        network, i.e. the extrapolation alone).  The matrix products run on
        the host (scipy); the network's forward and backward run on the
        device.  Returns the mean loss of the last epoch."""
        import scipy.sparse as sp

        x_all, y_all = self.dataset()
        shift = x_all.mean(axis=0)
        sd = x_all.std(axis=0)
        scale = 1.0 / np.where(sd > 0, sd, 1.0)
        osd = y_all.std(axis=0)
        out_scale = np.where(osd > 0, osd, 1.0)
        self.norm = np.concatenate([shift, scale, out_scale]).astype(np.float32)
        p, _ = self.net.get_params()
        self.net.set_params(p, self.norm)
        if warm_epochs:
            self.net.train(x_all, y_all / out_scale, epochs=warm_epochs, batch=min(2048, len(x_all)), lr=lr,
                           seed=self.seed)
        mats = []
        for (N, rows, cols, vals, alt) in self.mats:
            U = sp.bsr_matrix((vals.reshape(-1, 3, 3), cols, rows), shape=(3 * N, 3 * N)).tocsr()
            diag = cols == np.repeat(np.arange(N), np.diff(rows))
            D = sp.bsr_matrix((vals.reshape(-1, 3, 3) * diag[:, None, None], cols, rows), shape=(3 * N, 3 * N)).tocsr()
            mats.append(((U + U.T - D).tocsr(), N, alt))
        dens = []
        for (A, N, alt), y in zip(mats, self.ys):
            yy = np.zeros((N, 3))
            yy[alt] = y
            dens.append(float(np.square(A @ yy.ravel()).sum()))
        den = float(np.mean(dens)) + 1e-300
        rng = np.random.default_rng(self.seed)
        last = 0.0
        for _ in range(epochs):
            tot = 0.0
            for s in rng.permutation(len(self.xs)):
                A, N, alt = mats[s]
                x, y = self.xs[s], self.ys[s].astype(np.float64)
                pred = self.net.forward(x).astype(np.float64) * out_scale
                e = np.zeros((N, 3))
                e[alt] = pred - y
                r = A @ e.ravel()
                tot += float(r @ r) / den
                g = (2.0 / den) * (A @ r).reshape(N, 3)[alt]
                self.net.grad_dy(x, g * out_scale)
                self.net.adam_step(lr)
            last = tot / len(self.xs)
        return last

    # ---- the guess --------------------------------------------------------------
    def guess(self, model, h, u, v, a, gain=None):
        g = self.gain if gain is None else gain
        du = model.extrapolation(h, v)
        if self.norm is None or g == 0:
            return du
        x = features(u, v, a, *model.history_increments(h))
        corr = self.net.forward(x).astype(np.float64) * self.norm[2 * NI:]
        return du + g * corr

    def __call__(self, model, h, u, v, a):
        if self.select_gains:
            return self.judged_guess(model, h, u, v, a)
        return self.guess(model, h, u, v, a)

    # per step, the network's correction is judged before it is used: the
    # first-iterate residual of the guess at each candidate gain (one assembly
    # each, no solve) picks the gain; 0 is the extrapolation alone
    select_gains: tuple = ()
    chosen: list = None

    def judged_guess(self, model, h, u, v, a):
        gains = self.select_gains
        guesses = [self.guess(model, h, u, v, a, gain=g) for g in gains]
        rs = model.guess_residuals(guesses)
        k = int(np.argmin(rs))
        if self.chosen is not None:
            self.chosen.append(gains[k])
        return guesses[k]

    def calibrate(self, model, steps: int, gains=(0.0, 0.05, 0.2, 0.5, 1.0)) -> dict:
        """Runs `steps` attempts of `model` (extrapolation guess) and, before
        each, the first-iterate residual of the learned guess at each gain;
        keeps the gain with the smallest mean log residual.  Returns that mean
        per gain."""
        logs = {g: [] for g in gains}
        for _ in range(steps):
            h = model.time_step()[0]
            u, v, a, _ = model.gf.GetNodeState()
            rs = model.guess_residuals([self.guess(model, h, u, v, a, gain=g) for g in gains])
            for g, r in zip(gains, rs):
                logs[g].append(np.log10(max(r, 1e-300)))
            model.Step(warm_start=lambda m, hh, uu, vv, aa: m.extrapolation(hh, vv))
        mean = {g: float(np.mean(logs[g])) for g in gains}
        self.gain = min(mean, key=mean.get)
        return mean

    def close(self):
        self.net.close()


# ---- the three-arm comparison on the ice-block impact ------------------------------
def ice_model(speed: float, seed: int, n: int = 8):
    """Two ice blocks (the ice-impact geometry at n hexes per short side: n = 8
    gives 1,536 tets per block, 8 grains) approaching at 2 x speed, penalty
    contact, dt 5 us, Newton to a residual of 1e-8 of the zero-increment
    residual, with the reference's step control."""
    from icflow_b200 import mesh as M
    from icflow_b200.implicit_model import ImplicitModel3
    from icflow_b200.model_prms import config_prms

    c, v0 = M.ice_impact(n=n, grains=8, seed=seed, speed=speed)
    sig = np.concatenate([M.lognormal_strengths(len(m.czs), seed=seed * 10 + i, granule_pairs=m.cz_grains)
                          for i, m in enumerate(c.meshes)])
    p = config_prms(penaltyK=1e8)
    p.InitialTimeStep = 5e-6
    p.CollisionScheme = 1
    p.minIterations = 1
    p.maxIterations = 12
    return ImplicitModel3(c, p, strengths=sig, contact=True, v0=v0, convergence="residual", res_tol=1e-8,
                          rel_tol=1e-10)


def run_arm(warm, speed: float = 2.5, seed: int = 1, recorder=None, t_end: float = 40 * 5e-6):
    """(Newton iterations, attempts, accepted steps) of one run to t_end with
    the guess `warm` (None: the reference's v h)."""
    g = ice_model(speed, seed)
    g.recorder = recorder
    while g.t < t_end * (1 - 1e-9):
        g.Step(warm_start=warm)
    its = sum(s.iterations for s in g.history)
    attempts, accepted = len(g.history), sum(s.accepted for s in g.history)
    g.close()
    return its, attempts, accepted


def three_arms(t_end: float = 40 * 5e-6, train=((2.0, 2), (3.0, 3), (2.5, 4), (1.5, 5))) -> dict:
    """The same span of the ice impact under three guesses, each to the same
    residual tolerance: v h, the extrapolation v h + (d1 - d2), and the
    extrapolation plus the network's correction, judged per attempt (gains
    0, 0.5, 1).  The network is trained on the device on other impacts
    (`train`: (speed, grain seed) pairs)."""
    extrap = lambda m, h, u, v, a: m.extrapolation(h, v)  # noqa: E731
    plain = run_arm(None, t_end=t_end)
    ext = run_arm(extrap, t_end=t_end)
    ws = LearnedWarmStart(seed=0)
    for speed, seed in train:
        run_arm(extrap, speed, seed, recorder=ws, t_end=t_end)
    loss = ws.fit(epochs=80, batch=4096, lr=2e-3)
    ws.select_gains = (0.0, 0.5, 1.0)
    ws.chosen = []
    net = run_arm(ws, t_end=t_end)
    used = sum(g > 0 for g in ws.chosen)
    n_chosen = len(ws.chosen)
    ws.close()
    return {"plain": plain, "extrapolation": ext, "network": net, "network_used": used,
            "attempts_judged": n_chosen, "training_loss": loss}
