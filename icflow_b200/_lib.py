"""ctypes binding of libicflow_b200.so (the C ABI in include/icflow_b200.h).

The library is loaded from the package directory.  There is no fallback: if
the shared library is missing or cannot be loaded, importing a function that
needs it raises, so a GPU run can never silently use another code path.
"""
from __future__ import annotations

import ctypes as C  # noqa: N812
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libicflow_b200.so"

ICF_OK = 0
ICF_ERR_ARG = -1
ICF_ERR_SIZE = -2
ICF_ERR_CUDA = -3
ICF_ERR_STATE = -4
ICF_ERR_NUMERIC = -5
ICF_ERR_NODEVICE = -6
ICF_FP64 = 0
ICF_FP32_MIXED = 1

ERR_NAMES = {
    ICF_ERR_ARG: "ICF_ERR_ARG",
    ICF_ERR_SIZE: "ICF_ERR_SIZE",
    ICF_ERR_CUDA: "ICF_ERR_CUDA",
    ICF_ERR_STATE: "ICF_ERR_STATE",
    ICF_ERR_NUMERIC: "ICF_ERR_NUMERIC",
    ICF_ERR_NODEVICE: "ICF_ERR_NODEVICE",
}


class icf_params(C.Structure):
    """Mirror of struct icf_params (ModelPrms fields, then the derived block)."""

    _fields_ = [
        ("InitialTimeStep", C.c_double),
        ("Y", C.c_double), ("nu", C.c_double), ("rho", C.c_double),
        ("dampingMass", C.c_double), ("dampingStiffness", C.c_double), ("gravity", C.c_double),
        ("NewmarkBeta", C.c_double), ("NewmarkGamma", C.c_double),
        ("ConvergenceEpsilon", C.c_double), ("ConvergenceCutoff", C.c_double),
        ("maxDamagePerStep", C.c_double), ("maxFailPerStep", C.c_double),
        ("maxIterations", C.c_int), ("minIterations", C.c_int),
        ("alpha", C.c_double), ("beta", C.c_double), ("lambda_n", C.c_double),
        ("lambda_t", C.c_double), ("phi_n", C.c_double), ("phi_t", C.c_double),
        ("sigma_max", C.c_double), ("tau_max", C.c_double),
        ("CollisionScheme", C.c_int),
        ("penaltyK", C.c_double), ("DistanceEpsilon", C.c_double),
        ("E", C.c_double * 36), ("M", C.c_double * 144), ("sf", C.c_double * 9),
        ("B", C.c_double * 162),
        ("G_fn", C.c_double), ("G_ft", C.c_double), ("f_tn", C.c_double), ("f_tt", C.c_double),
        ("rn", C.c_double), ("rt", C.c_double), ("p_m", C.c_double), ("p_n", C.c_double),
        ("deln", C.c_double), ("delt", C.c_double), ("pMtn", C.c_double), ("pMnt", C.c_double),
        ("gam_n", C.c_double), ("gam_t", C.c_double),
        ("nThreshold", C.c_double), ("tThreshold", C.c_double),
    ]


class icf_counts(C.Structure):
    _fields_ = [(n, C.c_int) for n in (
        "nElems", "nCZ", "nCZDamaged", "nCZFailedThisStep", "nCZContact",
        "nImpacts", "nImpactsActive", "nonFinite", "nLawExact")]


class icf_kernel_times(C.Structure):
    _fields_ = [("n_kernels", C.c_int), ("name", (C.c_char * 32) * 16),
                ("bytes", C.c_longlong * 16), ("ms", C.c_double * 16)]

    def as_list(self):
        return [{"name": bytes(self.name[k]).split(b"\0")[0].decode(), "bytes": int(self.bytes[k]),
                 "ms": float(self.ms[k])} for k in range(self.n_kernels)]


class icf_tune_report(C.Structure):
    _fields_ = [("n", C.c_int), ("kernel", (C.c_char * 16) * 64), ("variant", (C.c_char * 32) * 64),
                ("ms", C.c_double * 64), ("chosen", C.c_int * 64)]

    def as_list(self):
        s = lambda b: bytes(b).split(b"\0")[0].decode()  # noqa: E731
        return [{"kernel": s(self.kernel[i]), "variant": s(self.variant[i]), "ms": float(self.ms[i]),
                 "chosen": bool(self.chosen[i])} for i in range(self.n)]


class icf_device_buffers(C.Structure):
    _fields_ = [
        ("vals", C.c_void_p), ("rhs", C.c_void_p), ("csr_rows", C.c_void_p),
        ("csr_cols", C.c_void_p), ("stream", C.c_void_p), ("N", C.c_int), ("nnz", C.c_int),
    ]


P = C.c_void_p
I = C.c_int
D = C.c_double
dp = C.POINTER(C.c_double)
ip = C.POINTER(C.c_int)

# name: (restype, argtypes)
SIGNATURES = {
    "icf_version": (C.c_char_p, []),
    "icf_create": (I, [I, C.POINTER(P)]),
    "icf_destroy": (I, [P]),
    "icf_last_error": (C.c_char_p, [P]),
    "icf_params_derive": (I, [C.POINTER(icf_params)]),
    "icf_set_constants": (I, [P, C.POINTER(icf_params)]),
    "icf_set_precision": (I, [P, I]),
    "icf_set_cz_strength": (I, [P, I, dp, dp]),
    "icf_transfer_static": (I, [P, I, dp, ip, I, ip, I, ip, I, ip, ip, ip, I, ip]),
    "icf_transfer_nodes": (I, [P, I, dp, dp, dp]),
    "icf_transfer_cz_state": (I, [P, I, dp, dp, ip]),
    "icf_narrow_phase": (I, [P, I, ip, ip]),
    "icf_get_impacts": (I, [P, I, ip]),
    "icf_set_impacts": (I, [P, I, ip]),
    "icf_get_narrow_masks": (I, [P, I, ip]),
    "icf_create_structure": (I, [P, ip, ip]),
    "icf_get_structure": (I, [P, ip, ip]),
    "icf_get_pcsr": (I, [P, I, C.c_longlong, ip]),
    "icf_assemble": (I, [P, D, C.POINTER(icf_counts)]),
    "icf_assemble_async": (I, [P, D]),
    "icf_set_graph": (I, [P, I]),
    "icf_read_counts": (I, [P, C.POINTER(icf_counts)]),
    "icf_profile_assembly": (I, [P, D, I, C.POINTER(icf_kernel_times)]),
    "icf_autotune": (I, [P, D, I, C.POINTER(icf_tune_report)]),
    "icf_solve": (I, [P, D, I, P, C.POINTER(C.c_int), C.POINTER(C.c_double)]),
    "icf_apply_dx": (I, [P, C.POINTER(C.c_double)]),
    "icf_residual_norm": (I, [P, C.POINTER(C.c_double)]),
    "icf_set_surface_groups": (I, [P, I, P]),
    "icf_broad_phase": (I, [P, D, C.POINTER(C.c_int)]),
    "icf_detect_contacts": (I, [P, D, C.POINTER(C.c_int)]),
    "icf_count_damaged": (I, [P, C.POINTER(C.c_int)]),
    "icf_get_pairs": (I, [P, I, P]),
    "icf_mlp_create": (I, [I, C.POINTER(P)]),
    "icf_mlp_destroy": (I, [P]),
    "icf_mlp_last_error": (C.c_char_p, [P]),
    "icf_mlp_param_count": (I, []),
    "icf_mlp_set_params": (I, [P, P, P]),
    "icf_mlp_get_params": (I, [P, P, P]),
    "icf_mlp_forward": (I, [P, I, P, P]),
    "icf_mlp_forward_trace": (I, [P, I, P, P, P, P, P, P]),
    "icf_mlp_grad": (I, [P, I, P, P, P, C.POINTER(C.c_float)]),
    "icf_mlp_train": (I, [P, I, P, P, I, I, C.c_float, C.c_ulonglong, C.POINTER(C.c_float)]),
    "icf_mlp_grad_dy": (I, [P, I, P, P, P]),
    "icf_mlp_adam_step": (I, [P, P, C.c_float]),
    "icf_set_variant": (I, [P, I, I]),
    "icf_assemble_noalloc": (I, [P, D, P, P, P, P, P, C.POINTER(icf_counts)]),
    "icf_transfer_linear_system": (I, [P, dp, dp]),
    "icf_transfer_updated_state": (I, [P, dp, dp, ip, dp, dp]),
    "icf_get_cz_tentative": (I, [P, dp, ip, dp]),
    "icf_cz_law_eval": (I, [P, I, dp, dp, dp, dp, dp, dp, dp, dp, ip]),
    "icf_get_device_buffers": (I, [P, C.POINTER(icf_device_buffers)]),
    "icf_set_node_state": (I, [P, I, dp, dp, dp]),
    "icf_get_node_state": (I, [P, dp, dp, dp, dp]),
    "icf_set_du": (I, [P, I, dp]),
    "icf_infer_tentative": (I, [P, D]),
    "icf_add_dx": (I, [P, dp, dp]),
    "icf_accept_tentative": (I, [P, D]),
}

_lib = None


def load() -> C.CDLL:
    """Loads the library (once).  Raises if it is missing: there is no fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise RuntimeError(
            f"{LIB_PATH.name} is not built; run `python -m icflow_b200.build` (needs nvcc)")
    lib = C.CDLL(str(LIB_PATH))
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def exported_symbols() -> list[str]:
    return sorted(SIGNATURES)


class ICFError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERR_NAMES.get(code, code)}: {msg}")
        self.code = code


def check(ctx, rc: int) -> None:
    if rc != ICF_OK:
        msg = load().icf_last_error(ctx) if ctx else b""
        raise ICFError(rc, (msg or b"").decode(errors="replace"))


def dptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(dp)


def iptr(a: np.ndarray | None):
    if a is None:
        return None
    assert a.dtype == np.int32 and a.flags.c_contiguous
    return a.ctypes.data_as(ip)
