"""Python access to the CHECKERS: the C restatement (liboracle.so) and the
reference's own kernel sources built for the host (_ref/libicf_ref.so).

TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg import this module; the product (icflow_b200) never does.

`RefKernels` drives the reference kernels unmodified, with the strided
structure-of-arrays layouts GPU_Functionality builds on the host
(v3Library/Simulation/GPU/GPU_Functionality.cs:141-149, 255-416, 539-676):
stride = n rounded up to a multiple of 128, field f of unit i at [i + stride*f].
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_LIB = HERE / "liboracle.so"
REF_LIB = HERE / "_ref" / "libicf_ref.so"

dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int)


def _d(a):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous, (a.dtype, a.flags)
    return a.ctypes.data_as(dp)


def _i(a):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous, (a.dtype, a.flags)
    return a.ctypes.data_as(ip)


class orc_ppr(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "G_fn", "G_ft", "f_tn", "f_tt", "alpha", "beta", "rn", "rt",
        "p_m", "p_n", "deln", "delt", "pMtn", "pMnt", "gam_n", "gam_t")]


class orc_prms(C.Structure):
    _fields_ = [(n, C.c_double) for n in (
        "Y", "nu", "rho", "dampingMass", "dampingStiffness", "gravity",
        "NewmarkBeta", "NewmarkGamma",
        "alpha", "beta", "lambda_n", "lambda_t", "phi_n", "phi_t", "sigma_max", "tau_max",
        "penaltyK", "DistanceEpsilon")] + [
        ("E", C.c_double * 36), ("M", C.c_double * 144), ("sf", C.c_double * 9),
        ("B", C.c_double * 162), ("ppr", orc_ppr),
        ("nThreshold", C.c_double), ("tThreshold", C.c_double)]


# ModelPrms defaults (v3Library/Simulation/DataSheets/ModelPrms.cs:29-209)
DEFAULTS = dict(Y=1e10, nu=0.3, rho=916.2, dampingMass=0.0005, dampingStiffness=0.0005,
                gravity=-9.8, NewmarkBeta=0.25, NewmarkGamma=0.5, alpha=3.0, beta=3.0,
                lambda_n=0.02, lambda_t=0.02, phi_n=30.0, phi_t=30.0, sigma_max=4e5,
                tau_max=15e5, penaltyK=50.0, DistanceEpsilon=1e-15)


class Oracle:
    """The C restatement of the reference algorithm (icf_oracle.c)."""

    def __init__(self):
        if not ORACLE_LIB.exists():
            raise RuntimeError("oracle/liboracle.so is not built (make -C oracle)")
        L = C.CDLL(str(ORACLE_LIB))
        L.orc_pt.restype = C.c_double
        L.orc_dtn.restype = C.c_double
        self.L = L

    # -- parameters --
    def prms(self, **kw) -> orc_prms:
        p = orc_prms()
        for k, v in {**DEFAULTS, **kw}.items():
            setattr(p, k, float(v))
        self.L.orc_prms_derive(C.byref(p))
        return p

    def ppr_for(self, p: orc_prms, sigma_max: float, tau_max: float) -> orc_ppr:
        q = orc_ppr()
        self.L.orc_ppr_derive(C.byref(q), C.c_double(p.alpha), C.c_double(p.beta),
                              C.c_double(p.lambda_n), C.c_double(p.lambda_t),
                              C.c_double(p.phi_n), C.c_double(p.phi_t),
                              C.c_double(sigma_max), C.c_double(tau_max))
        return q

    # -- per-unit functions --
    def ppr_eval(self, p, dn, dt):
        out = np.zeros(5)
        self.L.orc_ppr_eval(C.byref(p.ppr), C.c_double(dn), C.c_double(dt), _d(out))
        return out

    def cz_law(self, p, pmax, tmax, opn, opt, q=None):
        pm, tm = C.c_double(pmax), C.c_double(tmax)
        out = np.zeros(6)
        fl = np.zeros(2, np.int32)
        self.L.orc_cz_law(C.byref(q or p.ppr), C.byref(pm), C.byref(tm), C.c_double(opn),
                          C.c_double(opt), _d(out), _i(fl))
        return pm.value, tm.value, out, fl

    def elem_F_Df(self, p, x0, un):
        f = np.zeros(12)
        Df = np.zeros(144)
        V = C.c_double()
        self.L.orc_elem_F_Df(C.byref(p), _d(np.ascontiguousarray(x0, np.float64)),
                             _d(np.ascontiguousarray(un, np.float64)), _d(f), _d(Df), C.byref(V))
        return f, Df.reshape(12, 12), V.value

    def elem_local(self, p, h, x0, un, vn, an):
        lhs = np.zeros(144)
        rhs = np.zeros(12)
        c = lambda a: _d(np.ascontiguousarray(a, np.float64))  # noqa: E731
        self.L.orc_elem_local(C.byref(p), C.c_double(h), c(x0), c(un), c(vn), c(an), _d(lhs), _d(rhs))
        return lhs.reshape(12, 12), rhs

    def cz_local(self, p, x0, un, pmax, tmax, q=None):
        keff = np.zeros(324)
        rhs = np.zeros(18)
        tent = np.zeros(2)
        fl = np.zeros(3, np.int32)
        avg = np.zeros(4)
        c = lambda a: _d(np.ascontiguousarray(a, np.float64))  # noqa: E731
        self.L.orc_cz_local(C.byref(p), C.byref(q or p.ppr), c(x0), c(un), c(pmax), c(tmax),
                            _d(keff), _d(rhs), _d(tent), _i(fl), _d(avg))
        return keff.reshape(18, 18), rhs, tent, fl, avg

    def pt(self, x):
        fd = np.zeros(12)
        sd = np.zeros(144)
        s, t = C.c_double(), C.c_double()
        br = C.c_int()
        d = self.L.orc_pt(_d(np.ascontiguousarray(x, np.float64)), _d(fd), _d(sd), C.byref(s),
                          C.byref(t), C.byref(br))
        return d, fd, sd.reshape(12, 12), s.value, t.value, br.value

    def dtn(self, f9, p3):
        return self.L.orc_dtn(_d(np.ascontiguousarray(f9, np.float64)),
                              _d(np.ascontiguousarray(p3, np.float64)))

    def narrow_mask(self, xa, xb, na, nb):
        return self.L.orc_narrow_mask(_d(np.ascontiguousarray(xa, np.float64)),
                                      _d(np.ascontiguousarray(xb, np.float64)),
                                      _i(np.ascontiguousarray(na, np.int32)),
                                      _i(np.ascontiguousarray(nb, np.int32)))

    def contact_local(self, p, x):
        lhs = np.zeros(144)
        rhs = np.zeros(12)
        ok = self.L.orc_contact_local(C.byref(p), _d(np.ascontiguousarray(x, np.float64)), _d(lhs),
                                      _d(rhs))
        return ok, lhs.reshape(12, 12), rhs

    # -- structure --
    def build_structure(self, alt, elems, czs, imps):
        alt = np.ascontiguousarray(alt, np.int32)
        e = np.ascontiguousarray(elems, np.int32).reshape(-1, 4)
        c = np.ascontiguousarray(czs, np.int32).reshape(-1, 6)
        m = np.ascontiguousarray(imps, np.int32).reshape(-1, 4)
        nnz = C.c_int()
        rows = np.zeros(len(alt) + 2, np.int32)
        N = self.L.orc_build_structure(len(alt), _i(alt), len(e), _i(e), len(c), _i(c), len(m), _i(m),
                                       _i(rows), None, C.byref(nnz), C.c_longlong(0))
        if N < 0:
            raise RuntimeError(f"orc_build_structure failed ({N})")
        cols = np.zeros(max(nnz.value, 1), np.int32)
        N = self.L.orc_build_structure(len(alt), _i(alt), len(e), _i(e), len(c), _i(c), len(m), _i(m),
                                       _i(rows), _i(cols), C.byref(nnz), C.c_longlong(len(cols)))
        return N, rows[:N + 1].copy(), cols[:nnz.value].copy()

    def pcsr(self, units, k, alt, rows, cols, N):
        u = np.ascontiguousarray(units, np.int32).reshape(-1, k)
        out = np.zeros(len(u) * (k * k + k), np.int32)
        if len(u):
            self.L.orc_pcsr(len(u), k, _i(u), _i(np.ascontiguousarray(alt, np.int32)), _i(rows),
                            _i(cols), N, _i(out))
        return out.reshape(len(u), k * k + k)

    def assemble(self, p, h, coll_x0, un, vn, an, elems, epcsr, czs, cpcsr, pmax, tmax, imps, ipcsr,
                 nnz, N, cz_ppr=None):
        n = len(coll_x0)
        x0 = np.ascontiguousarray(coll_x0, np.float64)
        un = np.ascontiguousarray(un, np.float64)
        xt = x0 + un
        vals = np.zeros(9 * max(nnz, 1))
        rhs = np.zeros(3 * max(N, 1))
        F = np.zeros(3 * n)
        nc = len(czs)
        tent = np.zeros(2 * max(nc, 1))
        flags = np.zeros(3 * max(nc, 1), np.int32)
        avg = np.zeros(4 * max(nc, 1))
        ppr_arr = None
        if cz_ppr is not None:
            ppr_arr = (orc_ppr * nc)(*cz_ppr)
        e = np.ascontiguousarray(elems, np.int32)
        c = np.ascontiguousarray(czs, np.int32).reshape(-1, 6)
        m = np.ascontiguousarray(imps, np.int32).reshape(-1, 4)
        self.L.orc_assemble(C.byref(p), C.c_double(h), n, _d(x0), _d(un),
                            _d(np.ascontiguousarray(vn, np.float64)), _d(np.ascontiguousarray(an, np.float64)),
                            _d(xt), len(e), _i(e), _i(np.ascontiguousarray(epcsr, np.int32)),
                            nc, _i(c), _i(np.ascontiguousarray(cpcsr, np.int32)),
                            ppr_arr, _d(np.ascontiguousarray(pmax, np.float64)),
                            _d(np.ascontiguousarray(tmax, np.float64)), len(m), _i(m),
                            _i(np.ascontiguousarray(ipcsr, np.int32)), _d(vals), _d(rhs), _d(F),
                            _d(tent), _i(flags), _d(avg))
        return dict(vals=vals[:9 * nnz].reshape(-1, 3, 3), rhs=rhs[:3 * N], nodeF=F.reshape(-1, 3),
                    tent=tent[:2 * nc].reshape(-1, 2), flags=flags[:3 * nc].reshape(-1, 3),
                    avg=avg[:4 * nc].reshape(-1, 4))

    def narrow_phase(self, pairs, selem, xt):
        pairs = np.ascontiguousarray(pairs, np.int32)
        masks = np.zeros(max(len(pairs), 1), np.int32)
        self.L.orc_narrow_phase(len(pairs), _i(pairs), _i(np.ascontiguousarray(selem, np.int32)),
                                _d(np.ascontiguousarray(xt, np.float64)), _i(masks))
        return masks[:len(pairs)]

    def candidate_pairs(self, selem, xt, group=None, pad: float = 0.0, cap: int = 80_000_000):
        """The device broad phase's pair rule on the host (grid; boxes
        overlap, no shared node, a vertex of one in the other's box)."""
        selem = np.ascontiguousarray(selem, np.int32)
        out = np.zeros(2 * cap, np.int32)
        g = None if group is None else np.ascontiguousarray(group, np.int32)
        self.L.orc_candidate_pairs.restype = C.c_longlong
        n = self.L.orc_candidate_pairs(len(selem), _i(selem), _i(g), _d(np.ascontiguousarray(xt, np.float64)),
                                       C.c_double(pad), _i(out), C.c_longlong(cap))
        if n < 0:
            raise RuntimeError("candidate pair buffer too small")
        return out[:2 * n].reshape(-1, 2).copy()

    def kdop_pairs(self, selem, xt, cap: int = 20_000_000):
        """The element pairs the reference's k-DOP-24 BVH reports (all
        unordered surface-element pairs whose k-DOPs overlap), ascending."""
        selem = np.ascontiguousarray(selem, np.int32)
        out = np.zeros(2 * cap, np.int32)
        n = self.L.orc_kdop_pairs(len(selem), _i(selem), _d(np.ascontiguousarray(xt, np.float64)), _i(out),
                                  C.c_longlong(cap))
        if n < 0:
            raise RuntimeError("k-DOP pair buffer too small")
        return out[:2 * n].reshape(-1, 2).copy()

    def impacts(self, pairs, masks, selem, adj_off, adj, faces, xt):
        pairs = np.ascontiguousarray(pairs, np.int32)
        cap = 8 * max(len(pairs), 1)
        out = np.zeros(4 * cap, np.int32)
        n = self.L.orc_impacts(len(pairs), _i(pairs), _i(np.ascontiguousarray(masks, np.int32)),
                               _i(np.ascontiguousarray(selem, np.int32)),
                               _i(np.ascontiguousarray(adj_off, np.int32)),
                               _i(np.ascontiguousarray(adj, np.int32)),
                               _i(np.ascontiguousarray(faces, np.int32)),
                               _d(np.ascontiguousarray(xt, np.float64)), _i(out), cap)
        return out[:4 * n].reshape(-1, 4)

    def newmark_infer(self, h, beta, gamma, x0, u, v, a, du):
        n = len(x0)
        un, vn, an, xt = (np.zeros((n, 3)) for _ in range(4))
        c = lambda a_: _d(np.ascontiguousarray(a_, np.float64))  # noqa: E731
        self.L.orc_newmark_infer(n, C.c_double(h), C.c_double(beta), C.c_double(gamma), c(x0), c(u),
                                 c(v), c(a), c(du), _d(un), _d(vn), _d(an), _d(xt))
        return un, vn, an, xt

    def newmark_accept(self, h, x0, u, v, a, un, du):
        u, v, a, du = (np.array(z, np.float64, order="C") for z in (u, v, a, du))
        xc = np.zeros_like(u)
        self.L.orc_newmark_accept(len(x0), C.c_double(h), _d(np.ascontiguousarray(x0, np.float64)),
                                  _d(u), _d(v), _d(a), _d(np.ascontiguousarray(un, np.float64)),
                                  _d(du), _d(xc))
        return u, v, a, du, xc


def ref_available() -> bool:
    return REF_LIB.exists()


def _stride(n: int) -> int:
    """ComputeStrides (GPU_Functionality.cs:141-149): n rounded up to 128."""
    return ((n + 127) // 128) * 128


@dataclass
class RefState:
    """Reference-layout arrays for one assembly."""
    dn: np.ndarray
    nd_stride: int


class RefKernels:
    """The reference kernel sources compiled for the host, run unmodified."""

    def __init__(self, nthreads: int = 0):
        if not REF_LIB.exists():
            raise RuntimeError("oracle/_ref/libicf_ref.so is not built (reference sources absent?)")
        L = C.CDLL(str(REF_LIB))
        L.ref_pt.restype = C.c_double
        L.ref_dtn.restype = C.c_double
        self.L = L
        self.nthreads = nthreads

    def set_constants(self, p: orc_prms, q: orc_ppr | None = None):
        """SetConstants (GPU_Functionality.cs:151-194)."""
        q = q or p.ppr
        E = np.array(p.E[:], np.float64)
        M = np.array(p.M[:], np.float64)
        self.L.ref_elem_set_constants(_d(E), _d(M), C.c_double(p.NewmarkBeta), C.c_double(p.NewmarkGamma),
                                      C.c_double(p.dampingMass), C.c_double(p.dampingStiffness),
                                      C.c_double(p.rho), C.c_double(p.gravity), C.c_double(p.Y))
        s = np.array([p.NewmarkBeta, p.NewmarkGamma, p.dampingMass, p.dampingStiffness, p.rho, p.gravity,
                      q.G_fn, q.G_ft, q.f_tn, q.f_tt, q.alpha, q.beta, q.rn, q.rt, q.p_m, q.p_n,
                      q.deln, q.delt, q.pMtn, q.pMnt, q.gam_n, q.gam_t], np.float64)
        B = np.array(p.B[:], np.float64)
        sf = np.array(p.sf[:], np.float64)
        self.L.ref_cz_set_constants(_d(s), _d(M), _d(B), _d(sf))

    # -- per-unit entry points --
    def F_and_Df(self, x0, un):
        x0 = np.ascontiguousarray(x0, np.float64).reshape(-1, 12)
        un = np.ascontiguousarray(un, np.float64).reshape(-1, 12)
        n = len(x0)
        f = np.zeros((n, 12))
        Df = np.zeros((n, 144))
        V = np.zeros(n)
        self.L.ref_elem_F_and_Df(n, _d(x0), _d(un), _d(f), _d(Df), _d(V))
        return f, Df.reshape(n, 12, 12), V

    def ppr(self, dn, dt):
        dn = np.ascontiguousarray(dn, np.float64)
        dt = np.ascontiguousarray(dt, np.float64)
        out = np.zeros((len(dn), 5))
        self.L.ref_cz_ppr(len(dn), _d(dn), _d(dt), _d(out))
        return out

    def cz_law(self, pmax, tmax, opn, opt):
        pmax = np.array(pmax, np.float64)
        tmax = np.array(tmax, np.float64)
        out = np.zeros((len(pmax), 6))
        fl = np.zeros((len(pmax), 2), np.int32)
        self.L.ref_cz_law(len(pmax), _d(pmax), _d(tmax), _d(np.ascontiguousarray(opn, np.float64)),
                          _d(np.ascontiguousarray(opt, np.float64)), _d(out), _i(fl))
        return pmax, tmax, out, fl

    def pt(self, x):
        fd = np.zeros(12)
        sd = np.zeros(144)
        s, t = C.c_double(), C.c_double()
        br = C.c_int()
        d = self.L.ref_pt(_d(np.ascontiguousarray(x, np.float64)), _d(fd), _d(sd), C.byref(s),
                          C.byref(t), C.byref(br))
        return d, fd, sd.reshape(12, 12), s.value, t.value, br.value

    def dtn(self, f9, p3):
        return self.L.ref_dtn(_d(np.ascontiguousarray(f9, np.float64)),
                              _d(np.ascontiguousarray(p3, np.float64)))

    # -- reference layouts (GPU_Functionality host packing) --
    @staticmethod
    def pack_nodes(x0, un, vn, an):
        """TransferNodesToGPU (:307-343): 18 fields per node, F zeroed."""
        n = len(x0)
        st = _stride(n)
        dn = np.zeros(18 * st)
        for f, arr in ((0, x0), (3, un), (6, vn), (9, an), (15, np.asarray(x0) + np.asarray(un))):
            for k in range(3):
                dn[st * (f + k): st * (f + k) + n] = arr[:, k]
        return RefState(dn, st)

    @staticmethod
    def node_field(state: RefState, f: int, n: int):
        st = state.nd_stride
        return np.stack([state.dn[st * (f + k): st * (f + k) + n] for k in range(3)], axis=1)

    def elem_kernel(self, state: RefState, h, elems, epcsr, vals, rhs):
        """kelElementElasticityForce over all units with the g_ie_pcsr layout
        (TransferPCSR, :351-372): ids at fields 0..3, pcsr at 4..23."""
        ne = len(elems)
        st = _stride(ne)
        ie = np.zeros(28 * st, np.int32)
        for i in range(4):
            ie[st * i: st * i + ne] = elems[:, i]
        for j in range(20):
            ie[st * (4 + j): st * (4 + j) + ne] = epcsr[:, j]
        self.L.ref_elem_kernel(_i(ie), _d(state.dn), C.c_double(h), _d(vals), _d(rhs), ne, st,
                               state.nd_stride, self.nthreads)

    def cz_kernel(self, state: RefState, h, czs, cpcsr, pmax, tmax, vals, rhs, per_cz=None):
        """kczCZForce with the g_icz / g_dcz layouts (TransferPCSR, :375-413).
        Returns (tentative pmax, tentative tmax, flags [contact, damaged,
        failed], averages) as the reference leaves them in its buffers."""
        nc = len(czs)
        st = _stride(nc)
        icz = np.zeros(58 * st, np.int32)
        dcz = np.zeros(16 * st)
        for i in range(6):
            icz[st * (4 + i): st * (4 + i) + nc] = czs[:, i]
        for j in range(42):
            icz[st * (10 + j): st * (10 + j) + nc] = cpcsr[:, j]
        for j in range(3):
            dcz[st * j: st * j + nc] = pmax[:, j]
            dcz[st * (3 + j): st * (3 + j) + nc] = tmax[:, j]
        arrs = [None] * 4
        if per_cz is not None:
            arrs = [np.ascontiguousarray(a, np.float64) for a in per_cz]
        self.L.ref_cz_kernel(_d(dcz), _i(icz), _d(state.dn), _d(vals), _d(rhs), C.c_double(h), nc, st,
                             state.nd_stride, *(_d(a) for a in arrs), self.nthreads)
        tp = np.stack([dcz[st * (6 + j): st * (6 + j) + nc] for j in range(3)], 1)
        tt = np.stack([dcz[st * (9 + j): st * (9 + j) + nc] for j in range(3)], 1)
        flags = np.stack([icz[st * 1: st + nc], icz[st * 2: 2 * st + nc], icz[st * 3: 3 * st + nc]], 1)
        avg = np.stack([dcz[st * (12 + j): st * (12 + j) + nc] for j in range(4)], 1)
        return tp, tt, flags, avg

    def collision_kernel(self, state: RefState, h, imps, ipcsr, vals, rhs, k, eps):
        """kCollisionResponseForce with the g_icr layout (collisionResponse,
        :633-665): ids at 0..3, pcsr at 4..23."""
        ni = len(imps)
        st = _stride(ni)
        icr = np.zeros(28 * st, np.int32)
        for i in range(4):
            icr[st * i: st * i + ni] = imps[:, i]
        for j in range(20):
            icr[st * (4 + j): st * (4 + j) + ni] = ipcsr[:, j]
        self.L.ref_collision_kernel(_i(icr), _d(state.dn), C.c_double(h), _d(vals), _d(rhs), ni, st,
                                    state.nd_stride, C.c_double(k), C.c_double(eps), self.nthreads)

    def narrow_phase_kernel(self, state: RefState, n_nodes, pairs, selem, adj_off, adj):
        """kNarrowPhase_new with the g_ie / g_itet layouts (:255-280, :549-560)."""
        ns = len(selem)
        st = _stride(ns)
        maxadj = int(np.max(np.diff(adj_off))) if ns else 0
        ie = np.zeros(st * (5 + maxadj), np.int32)
        for i in range(4):
            ie[st * i: st * i + ns] = selem[:, i]
        ie[st * 4: st * 4 + ns] = np.diff(adj_off)
        for e in range(ns):
            fl = adj[adj_off[e]:adj_off[e + 1]]
            ie[e + st * (5 + np.arange(len(fl)))] = fl
        itet = np.ascontiguousarray(pairs, np.int32).reshape(-1).copy()
        self.L.ref_narrow_phase_kernel(len(pairs), _d(state.dn), _i(ie), _i(itet), st, state.nd_stride,
                                       self.nthreads)
        return itet[0::2].copy(), ie, st

    def closest_face_kernel(self, state: RefState, node_elem, ie, el_stride, faces):
        """kFindClosestFace (:586-612) on (node, element) tuples."""
        n = len(node_elem)
        ts = _stride(n)
        it = np.zeros(ts * 4, np.int32)
        it[:n] = node_elem[:, 0]
        it[ts: ts + n] = node_elem[:, 1]
        nf = len(faces)
        fs = _stride(nf)
        fc = np.zeros(3 * fs, np.int32)
        for i in range(3):
            fc[fs * i: fs * i + nf] = faces[:, i]
        self.L.ref_closest_face_kernel(n, ts, _i(it), _d(state.dn), _i(ie), _i(fc), state.nd_stride,
                                       el_stride, fs, self.nthreads)
        return np.stack([it[:n], it[ts:ts + n], it[2 * ts:2 * ts + n], it[3 * ts:3 * ts + n]], 1)
