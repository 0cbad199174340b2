"""ModelPrms: the simulation parameters of icFlow
(v3Library/Simulation/DataSheets/ModelPrms.cs), same names and defaults.

The derived quantities (elasticity matrix, mass pattern, PPR constants, Gauss
point shape functions) are computed by the library's icf_params_derive, the
native counterpart of ModelPrms.SetComputedVariables (:237-322).
"""
from __future__ import annotations

from dataclasses import asdict, dataclass

from . import _lib


@dataclass
class ModelPrms:
    # Simulation (:29-33)
    InitialTimeStep: float = 0.025
    MaxSteps: int = 300
    # CZ (:38-65)
    alpha: float = 3.0
    beta: float = 3.0
    lambda_n: float = 0.02
    lambda_t: float = 0.02
    phi_n: float = 30.0
    phi_t: float = 30.0
    sigma_max: float = 4e5
    tau_max: float = 15e5
    # Material (:135-151)
    Y: float = 1e10
    rho: float = 916.2
    dampingMass: float = 0.0005
    dampingStiffness: float = 0.0005
    nu: float = 0.3
    # Collisions (:160-174); CollisionScheme 0 = None, 1 = Everything
    CollisionScheme: int = 1
    penaltyK: float = 50.0
    DistanceEpsilon: float = 1e-15
    ReconstructBVH: int = 10
    # Integration (:179-209)
    NewmarkBeta: float = 0.25
    NewmarkGamma: float = 0.5
    ConvergenceEpsilon: float = 0.005
    ConvergenceCutoff: float = 1e-8
    maxDamagePerStep: float = 0.01
    maxFailPerStep: float = 0.01
    maxIterations: int = 10
    minIterations: int = 3
    gravity: float = -9.8

    def to_icf(self) -> _lib.icf_params:
        p = _lib.icf_params()
        names = {f[0] for f in _lib.icf_params._fields_}
        for k, v in asdict(self).items():
            if k in names:
                setattr(p, k, type(getattr(p, k))(v))
        rc = _lib.load().icf_params_derive(p)
        if rc != 0:
            raise _lib.ICFError(rc, "icf_params_derive")
        return p

    def derived(self) -> dict:
        p = self.to_icf()
        return {n: (list(getattr(p, n)) if hasattr(getattr(p, n), "__len__") else getattr(p, n))
                for n, _ in _lib.icf_params._fields_}


def config_prms(**kw) -> ModelPrms:
    """Parameters shared by the benchmark configurations: E = 9 GPa, nu = 0.3,
    rho = 916 kg/m^3, PPR phi = 3 J/m^2, sigma = tau = 1 MPa, alpha = beta = 4,
    lambda = 0.02, Newmark beta = 0.25, gamma = 0.5."""
    base = dict(Y=9e9, nu=0.3, rho=916.0, phi_n=3.0, phi_t=3.0, sigma_max=1e6, tau_max=1e6,
                alpha=4.0, beta=4.0, lambda_n=0.02, lambda_t=0.02, NewmarkBeta=0.25,
                NewmarkGamma=0.5)
    base.update(kw)
    return ModelPrms(**base)
