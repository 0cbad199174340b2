"""The C ABI without a GPU: the library loads, exports every function that
include/icflow_b200.h declares, its host-only parameter derivation matches the
oracle bit for bit, and device calls fail cleanly with an error code."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

from icflow_b200 import _lib
from icflow_b200.model_prms import ModelPrms, config_prms

HEADER = Path(__file__).resolve().parents[1] / "include" / "icflow_b200.h"


def declared():
    txt = re.sub(r"/\*.*?\*/", "", HEADER.read_text(), flags=re.S)
    return sorted(set(re.findall(r"\b(icf_[a-z_0-9]+)\s*\(", txt)))


def test_every_declared_symbol_is_exported_and_bound():
    lib = _lib.load()
    names = declared()
    assert len(names) >= 30
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)
    assert lib.icf_version().startswith(b"icflow_b200")


def test_no_device_is_reported_not_crashed():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    lib = _lib.load()
    ctx = C.c_void_p()
    assert lib.icf_create(0, C.byref(ctx)) == _lib.ICF_ERR_NODEVICE
    assert lib.icf_destroy(None) == _lib.ICF_ERR_ARG
    assert lib.icf_last_error(None) == b"null context"
    assert lib.icf_assemble(None, 1e-4, None) == _lib.ICF_ERR_ARG


@pytest.mark.parametrize("prms", [ModelPrms(), config_prms(), config_prms(phi_n=2.0, phi_t=5.0, alpha=3.5)])
def test_params_derive_matches_oracle(prms):
    from oracle.oracle import Oracle

    p = prms.to_icf()
    O = Oracle()
    keys = ("Y", "nu", "rho", "dampingMass", "dampingStiffness", "gravity", "NewmarkBeta", "NewmarkGamma",
            "alpha", "beta", "lambda_n", "lambda_t", "phi_n", "phi_t", "sigma_max", "tau_max", "penaltyK",
            "DistanceEpsilon")
    o = O.prms(**{k: getattr(prms, k) for k in keys})
    for arr in ("E", "M", "sf", "B"):
        assert np.array_equal(np.array(getattr(p, arr)[:]), np.array(getattr(o, arr)[:])), arr
    for k in ("G_fn", "G_ft", "f_tn", "f_tt", "rn", "rt", "p_m", "p_n", "deln", "delt", "pMtn", "pMnt",
              "gam_n", "gam_t"):
        assert getattr(p, k) == getattr(o.ppr, k), k
    assert p.nThreshold == o.nThreshold and p.tThreshold == o.tThreshold


def test_model_prms_defaults_mirror_reference():
    """ModelPrms.cs:29-209 defaults."""
    m = ModelPrms()
    assert (m.InitialTimeStep, m.alpha, m.beta, m.lambda_n, m.phi_n, m.sigma_max, m.tau_max) == (
        0.025, 3.0, 3.0, 0.02, 30.0, 4e5, 15e5)
    assert (m.Y, m.rho, m.nu, m.penaltyK, m.DistanceEpsilon) == (1e10, 916.2, 0.3, 50.0, 1e-15)
    assert (m.NewmarkBeta, m.NewmarkGamma, m.ConvergenceEpsilon, m.ConvergenceCutoff) == (0.25, 0.5, 0.005, 1e-8)
    assert (m.maxIterations, m.minIterations, m.gravity) == (10, 3, -9.8)
