"""GPU_Functionality: the host-side class of icFlow's assembly path
(v3Library/Simulation/GPU/GPU_Functionality.cs:13-678), same method names and
call order, implemented over the C ABI of libicflow_b200.

Differences from the C# original, by design:
  * The device builds the sparsity pattern (CSRDictionary.CreateStructure) and
    the per-unit slot maps (TransferPCSR); LinearSystem.CreateStructure here
    calls icf_create_structure and copies csr_rows/csr_cols back.
  * AssembleElemsAndCZs assembles elements, CZs and the impacts of the
    current structure in one deterministic pass; collisionResponse is kept
    for call compatibility and only records the impact counters.
  * CZ damage state stays on the device between iterations;
    TransferUpdatedStateToHost commits it there and copies it back.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import _lib
from ._lib import check, dptr, iptr
from .mesh import Collection
from .model_prms import ModelPrms


@dataclass
class FrameInfo:
    """The counters of FrameInfo.cs that the assembly path fills."""

    TimeStep: float = 0.0
    nElems: int = 0
    nCZ: int = 0
    nCZDamaged: int = 0
    nCZFailedThisStep: int = 0
    nCollisions: int = 0
    nImpactsActive: int = 0


@dataclass
class LinearSystem:
    """Structure and value arrays of the linear system (LinearSystem.cs)."""

    N: int = 0
    nnz: int = 0
    csr_rows: np.ndarray = field(default_factory=lambda: np.zeros(1, np.int32))
    csr_cols: np.ndarray = field(default_factory=lambda: np.zeros(0, np.int32))
    vals: np.ndarray = field(default_factory=lambda: np.zeros(0))
    rhs: np.ndarray = field(default_factory=lambda: np.zeros(0))
    dx: np.ndarray = field(default_factory=lambda: np.zeros(0))

    @property
    def dvalsSize(self) -> int:
        return self.nnz * 9

    @property
    def dxSize(self) -> int:
        return self.N * 3

    def NormOfDx(self) -> float:
        return float(np.dot(self.dx, self.dx))


class GPU_Functionality:
    def __init__(self, deviceID: int = 0):
        self.lib = _lib.load()
        self.ctx = C.c_void_p()
        rc = self.lib.icf_create(deviceID, C.byref(self.ctx))
        if rc != 0:
            raise _lib.ICFError(rc, "icf_create: no usable sm_100 device")
        self.prms: ModelPrms | None = None
        self.mc: Collection | None = None
        self.linearSystem = LinearSystem()
        self.cf = FrameInfo()
        self.nImpacts = 0
        self.c_itet = np.zeros((0, 4), np.int32)

    def __del__(self):
        try:
            if self.ctx:
                self.lib.icf_destroy(self.ctx)
                self.ctx = C.c_void_p()
        except Exception:
            pass

    def close(self):
        self.__del__()

    # -- SetConstants (:151-194) --
    def SetConstants(self):
        self._icf_prms = self.prms.to_icf()
        check(self.ctx, self.lib.icf_set_constants(self.ctx, C.byref(self._icf_prms)))

    def SetPrecision(self, precision: int):
        check(self.ctx, self.lib.icf_set_precision(self.ctx, precision))

    def SetCZStrengths(self, sigma_max: np.ndarray | None, tau_max: np.ndarray | None):
        s = None if sigma_max is None else np.ascontiguousarray(sigma_max, np.float64)
        t = None if tau_max is None else np.ascontiguousarray(tau_max, np.float64)
        n = 0 if s is None else len(s)
        check(self.ctx, self.lib.icf_set_cz_strength(self.ctx, n, dptr(s), dptr(t)))

    # -- TransferStaticDataToDevice (:255-302) --
    def TransferStaticDataToDevice(self):
        self._groups_same_mesh = True  # a new context has no groups: every pair
        mc = self.mc
        x0 = np.ascontiguousarray(mc.x0, np.float64)
        el = np.ascontiguousarray(mc.elems, np.int32)
        cz = np.ascontiguousarray(mc.czs, np.int32)
        se = np.ascontiguousarray(mc.selem, np.int32)
        check(self.ctx, self.lib.icf_transfer_static(
            self.ctx, len(x0), dptr(x0), iptr(np.ascontiguousarray(mc.alt, np.int32)),
            len(el), iptr(el), len(cz), iptr(cz), len(se), iptr(se),
            iptr(np.ascontiguousarray(mc.adj_off, np.int32)), iptr(np.ascontiguousarray(mc.adj, np.int32)),
            len(mc.faces), iptr(np.ascontiguousarray(mc.faces, np.int32))))
        self.cf.nElems = len(el)
        self.cf.nCZ = len(cz)

    # -- TransferNodesToGPU (:307-343) --
    def TransferNodesToGPU(self, un: np.ndarray, vn: np.ndarray, an: np.ndarray):
        un, vn, an = (np.ascontiguousarray(a, np.float64) for a in (un, vn, an))
        check(self.ctx, self.lib.icf_transfer_nodes(self.ctx, len(un), dptr(un), dptr(vn), dptr(an)))

    # -- TransferPCSR, CZ state part (:374-413) --
    def TransferPCSR(self, pmax: np.ndarray, tmax: np.ndarray, failed: np.ndarray):
        pmax, tmax = (np.ascontiguousarray(a, np.float64) for a in (pmax, tmax))
        failed = np.ascontiguousarray(failed, np.int32)
        check(self.ctx, self.lib.icf_transfer_cz_state(self.ctx, len(failed), dptr(pmax), dptr(tmax),
                                                       iptr(failed)))

    # -- broad phase on the device (replaces the host BVH, BVHT.cs:29-77) --
    def _set_groups(self, same_mesh: bool):
        if getattr(self, "_groups_same_mesh", None) != same_mesh:
            grp = None if same_mesh else np.ascontiguousarray(self.mc.selem_mesh, np.int32)
            check(self.ctx, self.lib.icf_set_surface_groups(self.ctx, len(self.mc.selem_mesh),
                                                            iptr(grp) if grp is not None else None))
            self._groups_same_mesh = same_mesh

    def BroadPhase(self, pad: float = 0.0, same_mesh: bool = True) -> int:
        """Candidate surface-element pairs with overlapping boxes at the
        current positions that share no node, as the reference's BVH lists
        them (BVHT.cs:29-77: every surface element of every mesh, so pairs of
        one mesh too); same_mesh=False keeps only pairs of different meshes.
        The pairs stay on the device for NarrowPhaseCollisionDetection(None)."""
        self._set_groups(same_mesh)
        n = C.c_int()
        check(self.ctx, self.lib.icf_broad_phase(self.ctx, float(pad), C.byref(n)))
        self.nPairs = n.value
        return n.value

    def DetectContacts(self, pad: float = 0.0, same_mesh: bool = True, copy_back: bool = True):
        """The impacts BroadPhase(pad, same_mesh) followed by
        NarrowPhaseCollisionDetection(None) gives, found without the pair
        list (one query per surface node in a grid of the surface elements).
        Returns the impact list (node, face vertices) as
        NarrowPhaseCollisionDetection does.  With copy_back=False the list
        stays on the device, where CreateStructure and the assembly read it,
        and only its length is returned."""
        self._set_groups(same_mesh)
        n = C.c_int()
        check(self.ctx, self.lib.icf_detect_contacts(self.ctx, float(pad), C.byref(n)))
        self.nImpacts = self.cf.nCollisions = n.value
        if not copy_back:
            return n.value
        self.c_itet = np.zeros((n.value, 4), np.int32)
        if n.value:
            check(self.ctx, self.lib.icf_get_impacts(self.ctx, n.value, iptr(self.c_itet)))
        return self.c_itet

    def GetPairs(self) -> np.ndarray:
        out = np.zeros((max(self.nPairs, 1), 2), np.int32)
        check(self.ctx, self.lib.icf_get_pairs(self.ctx, len(out), iptr(out)))
        return out[:self.nPairs]

    # -- NarrowPhaseCollisionDetection (:539-616) --
    def NarrowPhaseCollisionDetection(self, narrowList: np.ndarray | None):
        """narrowList: [n, 2] surface-element pairs, or None for the pairs of
        the last BroadPhase (already on the device)."""
        n = C.c_int()
        if narrowList is None:
            check(self.ctx, self.lib.icf_narrow_phase(self.ctx, -1, None, C.byref(n)))
        else:
            pairs = np.ascontiguousarray(narrowList, np.int32).reshape(-1, 2)
            check(self.ctx, self.lib.icf_narrow_phase(self.ctx, len(pairs), iptr(pairs), C.byref(n)))
        self.nImpacts = self.cf.nCollisions = n.value
        self.c_itet = np.zeros((n.value, 4), np.int32)
        if n.value:
            check(self.ctx, self.lib.icf_get_impacts(self.ctx, n.value, iptr(self.c_itet)))
        return self.c_itet

    def NarrowPhaseMasks(self, n_pairs: int) -> np.ndarray:
        m = np.zeros(max(n_pairs, 1), np.int32)
        check(self.ctx, self.lib.icf_get_narrow_masks(self.ctx, len(m), iptr(m)))
        return m[:n_pairs]

    def SetImpacts(self, impacts: np.ndarray):
        imp = np.ascontiguousarray(impacts, np.int32).reshape(-1, 4)
        check(self.ctx, self.lib.icf_set_impacts(self.ctx, len(imp), iptr(imp)))
        self.nImpacts = self.cf.nCollisions = len(imp)

    # -- LinearSystem.CreateStructure (LinearSystem.cs:29-43) --
    def CreateStructure(self, copy_back: bool = True):
        N, nnz = C.c_int(), C.c_int()
        check(self.ctx, self.lib.icf_create_structure(self.ctx, C.byref(N), C.byref(nnz)))
        ls = self.linearSystem
        ls.N, ls.nnz = N.value, nnz.value
        if copy_back:
            ls.csr_rows = np.zeros(ls.N + 1, np.int32)
            ls.csr_cols = np.zeros(max(ls.nnz, 1), np.int32)
            check(self.ctx, self.lib.icf_get_structure(self.ctx, iptr(ls.csr_rows), iptr(ls.csr_cols)))
            ls.csr_cols = ls.csr_cols[:ls.nnz]
        return ls.N, ls.nnz

    def GetPCSR(self, kind: int) -> np.ndarray:
        n = {0: self.cf.nElems, 1: self.cf.nCZ, 2: self.nImpacts}[kind]
        w = 42 if kind == 1 else 20
        out = np.zeros(max(n * w, 1), np.int32)
        check(self.ctx, self.lib.icf_get_pcsr(self.ctx, kind, len(out), iptr(out)))
        return out[:n * w].reshape(n, w)

    # -- AssembleElemsAndCZs (:439-479) --
    def AssembleElemsAndCZs(self, h: float | None = None):
        h = self.cf.TimeStep if h is None else h
        cnt = _lib.icf_counts()
        check(self.ctx, self.lib.icf_assemble(self.ctx, float(h), C.byref(cnt)))
        self.cf.nCZDamaged = cnt.nCZDamaged
        self.cf.nCZFailedThisStep = cnt.nCZFailedThisStep
        self.cf.nImpactsActive = cnt.nImpactsActive
        return cnt

    def ProfileAssembly(self, h: float | None = None, reps: int = 10):
        """Per-kernel mean device time of the assembly (no reference
        counterpart): list of {name, bytes, ms}."""
        h = self.cf.TimeStep if h is None else h
        t = _lib.icf_kernel_times()
        check(self.ctx, self.lib.icf_profile_assembly(self.ctx, float(h), int(reps), C.byref(t)))
        return t.as_list()

    def Autotune(self, h: float | None = None, reps: int = 10):
        """Times every launch variant of the tet kernel and the gathers on this
        model and keeps the fastest (no reference counterpart)."""
        h = self.cf.TimeStep if h is None else h
        r = _lib.icf_tune_report()
        check(self.ctx, self.lib.icf_autotune(self.ctx, float(h), int(reps), C.byref(r)))
        return r.as_list()

    def SetVariant(self, kind: int, variant: int):
        check(self.ctx, self.lib.icf_set_variant(self.ctx, int(kind), int(variant)))

    # -- collisionResponse (:627-676): folded into the assembly --
    def collisionResponse(self):
        return self.cf.nImpactsActive

    # -- TransferLinearSystemToHost (:481-485) --
    def TransferLinearSystemToHost(self, vals: np.ndarray | None = None, rhs: np.ndarray | None = None):
        ls = self.linearSystem
        if vals is None:
            vals = np.zeros(ls.nnz * 9)
        if rhs is None:
            rhs = np.zeros(ls.N * 3)
        check(self.ctx, self.lib.icf_transfer_linear_system(self.ctx, dptr(vals), dptr(rhs)))
        ls.vals, ls.rhs = vals, rhs
        return vals, rhs

    # -- TransferUpdatedStateToHost (:487-528) --
    def TransferUpdatedStateToHost(self, want_forces: bool = True):
        nc = self.cf.nCZ
        pmax = np.zeros((max(nc, 1), 3))
        tmax = np.zeros((max(nc, 1), 3))
        failed = np.zeros(max(nc, 1), np.int32)
        avg = np.zeros((max(nc, 1), 4))
        F = np.zeros((len(self.mc.x0), 3)) if want_forces else None
        check(self.ctx, self.lib.icf_transfer_updated_state(self.ctx, dptr(pmax), dptr(tmax), iptr(failed),
                                                            dptr(avg), dptr(F)))
        return dict(pmax=pmax[:nc], tmax=tmax[:nc], failed=failed[:nc], avg=avg[:nc], nodeF=F)

    def CountDamagedCZs(self) -> int:
        """Non-failed committed CZs damaged at the level _acceptFrame counts
        (ImplicitModel3.cs:304-317): the accepted frame's nCZDamaged."""
        n = C.c_int()
        check(self.ctx, self.lib.icf_count_damaged(self.ctx, C.byref(n)))
        return n.value

    def GetCZTentative(self):
        nc = self.cf.nCZ
        tent = np.zeros((max(nc, 1), 2))
        flags = np.zeros((max(nc, 1), 3), np.int32)
        avg = np.zeros((max(nc, 1), 4))
        check(self.ctx, self.lib.icf_get_cz_tentative(self.ctx, dptr(tent), iptr(flags), dptr(avg)))
        return tent[:nc], flags[:nc], avg[:nc]

    def CZLaw(self, pmax, tmax, opn, opt, strength=None):
        """The cohesive law of the CZ kernel (cz_kernels.h:37-174) evaluated on
        the device for arrays of Gauss-point states; strength[n, 2] =
        (sigma_max, tau_max) per state or None for the constants.  Returns
        pmax', tmax', law[n, 5] (Tn, Tt, Dnn, Dtt, Dnt), flags[n, 3]
        (contact, failed, settled with the reference's rounding)."""
        pmax, tmax, opn, opt = (np.ascontiguousarray(z, np.float64).ravel() for z in (pmax, tmax, opn, opt))
        n = len(pmax)
        st = None if strength is None else np.ascontiguousarray(strength, np.float64).reshape(n, 2)
        pm, tm = np.zeros(n), np.zeros(n)
        law = np.zeros((n, 5))
        fl = np.zeros((n, 3), np.int32)
        check(self.ctx, self.lib.icf_cz_law_eval(self.ctx, n, dptr(pmax), dptr(tmax), dptr(opn), dptr(opt),
                                                 dptr(st) if st is not None else None, dptr(pm), dptr(tm),
                                                 dptr(law), iptr(fl)))
        return pm, tm, law, fl

    def DeviceBuffers(self) -> _lib.icf_device_buffers:
        b = _lib.icf_device_buffers()
        check(self.ctx, self.lib.icf_get_device_buffers(self.ctx, C.byref(b)))
        return b

    # -- Node kinematics on the device (Node.cs:62-97) --
    def SetNodeState(self, u, v, a):
        u, v, a = (np.ascontiguousarray(z, np.float64) for z in (u, v, a))
        check(self.ctx, self.lib.icf_set_node_state(self.ctx, len(u), dptr(u), dptr(v), dptr(a)))

    def GetNodeState(self):
        n = len(self.mc.x0)
        u, v, a, du = (np.zeros((n, 3)) for _ in range(4))
        check(self.ctx, self.lib.icf_get_node_state(self.ctx, dptr(u), dptr(v), dptr(a), dptr(du)))
        return u, v, a, du

    def SetDU(self, du):
        du = np.ascontiguousarray(du, np.float64)
        check(self.ctx, self.lib.icf_set_du(self.ctx, len(du), dptr(du)))

    def InferTentativeValues(self, h: float):
        check(self.ctx, self.lib.icf_infer_tentative(self.ctx, float(h)))

    def XtoDU(self, dx: np.ndarray) -> float:
        dx = np.ascontiguousarray(dx, np.float64)
        nrm = C.c_double()
        check(self.ctx, self.lib.icf_add_dx(self.ctx, dptr(dx), C.byref(nrm)))
        return nrm.value

    def Solve(self, rel_tol: float = 1e-12, max_iter: int = 20000, want_dx: bool = False):
        """Device MINRES solve of the last assembled system (replaces
        LinearSystem.Solve / PARDISO).  Returns (iterations, relative residual,
        dx or None)."""
        it, rr = C.c_int(), C.c_double()
        dx = np.zeros((self.linearSystem.N, 3)) if want_dx else None
        check(self.ctx, self.lib.icf_solve(self.ctx, float(rel_tol), int(max_iter), dptr(dx), C.byref(it),
                                           C.byref(rr)))
        return it.value, rr.value, dx

    def ApplyDx(self) -> float:
        """_XtoDU with the device solution; returns NormOfDx (sum of dx^2)."""
        nrm = C.c_double()
        check(self.ctx, self.lib.icf_apply_dx(self.ctx, C.byref(nrm)))
        return nrm.value

    def ResidualNorm(self) -> float:
        """||rhs|| of the last assembly."""
        n2 = C.c_double()
        check(self.ctx, self.lib.icf_residual_norm(self.ctx, C.byref(n2)))
        return float(np.sqrt(n2.value))

    def AcceptTentativeValues(self, h: float):
        check(self.ctx, self.lib.icf_accept_tentative(self.ctx, float(h)))
