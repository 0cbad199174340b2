"""icf_assemble_noalloc: the assembly entry point for callers that cannot
allocate device memory while they assemble (their device memory comes from a
pool they sized up front, or their loop must not enter the allocator).

It must produce what icf_assemble produces, from the caller's device arrays
into the caller's device arrays, with its temporaries in the library's fixed
static device array.  Checked on two calls in a row (two different node
states, so the second call cannot reuse anything the first left in the shared
array), on the cantilever and on a small polycrystal pressed by platens, in
FP64 and FP32-mixed precision, with the list gathers and with the row-tile
gather.  This file is collected last so a failure here cannot hide the other
tests.
"""
import ctypes as C

import numpy as np
import pytest

from icflow_b200 import _lib
from icflow_b200 import mesh as M
from icflow_b200.gpu_functionality import GPU_Functionality
from icflow_b200.model_prms import config_prms
from tests.harness import FP64_TOL, random_state, rowwise_rel, vec_rel

pytestmark = pytest.mark.gpu
H = 1e-4


def _setup(coll, prms, state, pairs=None, precision=0, tiles=False):
    gf = GPU_Functionality(0)
    gf.prms = prms
    gf.mc = coll
    gf.SetConstants()
    gf.SetPrecision(precision)
    gf.TransferStaticDataToDevice()
    nc = len(coll.czs)
    gf.TransferPCSR(np.zeros((nc, 3)), np.zeros((nc, 3)), np.zeros(nc, np.int32))
    gf.TransferNodesToGPU(*state)
    if pairs is not None:
        gf.NarrowPhaseCollisionDetection(pairs)
    gf.CreateStructure()
    if tiles:
        gf.SetVariant(6, 1)
        names = [k["name"] for k in gf.ProfileAssembly(H, reps=1)]
        assert "k_gather_tile" in names, names
    return gf


@pytest.mark.parametrize("case,precision,tiles", [("cantilever", 0, False), ("polycrystal_contact", 0, False),
                                                  ("cantilever", 1, False), ("polycrystal_contact", 1, True),
                                                  ("polycrystal_contact", 0, True)])
def test_noalloc_matches_assemble_twice(case, precision, tiles):
    import torch

    if case == "cantilever":
        coll = M.cantilever()
        prms = config_prms()
        du = 3e-6
    else:
        coll = M.polycrystal(n=6, grains=5, seed=4, platens=True, gap=-0.3)
        prms = config_prms(penaltyK=1e8)
        du = 1e-6
    states = [random_state(coll, seed, du=du) for seed in (11, 12)]
    pairs = None
    if case != "cantilever":
        pairs = M.candidate_pairs(coll, coll.x0 + states[0][0])
    gf = _setup(coll, prms, states[0], pairs, precision, tiles)
    lib = _lib.load()
    ls = gf.linearSystem
    dev = torch.device("cuda", 0)
    vals_d = torch.empty(9 * ls.nnz, dtype=torch.float64, device=dev)
    rhs_d = torch.empty(3 * ls.N, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()

    for call, state in enumerate(states):
        # the existing entry point on the same state
        gf.TransferNodesToGPU(*state)
        gf.AssembleElemsAndCZs(H)
        vals_ref, rhs_ref = gf.TransferLinearSystemToHost()
        vals_ref, rhs_ref = vals_ref.copy(), rhs_ref.copy()
        # the allocation-free entry point from device inputs into device outputs
        ins = [torch.from_numpy(np.ascontiguousarray(a)).to(dev) for a in state]
        vals_d.fill_(np.nan)
        rhs_d.fill_(np.nan)
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info(dev)[0]
        cnt = _lib.icf_counts()
        rc = lib.icf_assemble_noalloc(gf.ctx, H, *(C.c_void_p(t.data_ptr()) for t in ins),
                                      C.c_void_p(vals_d.data_ptr()), C.c_void_p(rhs_d.data_ptr()),
                                      C.byref(cnt))
        _lib.check(gf.ctx, rc)
        free1 = torch.cuda.mem_get_info(dev)[0]
        if call == 1:  # after the first call everything it touches is loaded
            assert free1 == free0, "icf_assemble_noalloc changed free device memory"
        vals = vals_d.cpu().numpy()
        rhs = rhs_d.cpu().numpy()
        assert np.all(np.isfinite(vals)) and np.all(np.isfinite(rhs))
        assert rowwise_rel(ls.csr_rows, vals_ref.reshape(-1, 3, 3), vals.reshape(-1, 3, 3)) <= FP64_TOL
        assert vec_rel(rhs_ref, rhs) <= FP64_TOL
        assert cnt.nElems == len(coll.elems) and cnt.nImpacts == gf.nImpacts
    gf.close()


def test_noalloc_rejects_models_beyond_its_scratch():
    coll = M.polycrystal(n=20, grains=16, seed=1, platens=False)  # ~15 MB of temporaries
    prms = config_prms()
    state = random_state(coll, 1, du=1e-7)
    gf = _setup(coll, prms, state)
    lib = _lib.load()
    import torch

    dev = torch.device("cuda", 0)
    ins = [torch.zeros(len(coll.x0) * 3, dtype=torch.float64, device=dev) for _ in range(3)]
    out = torch.zeros(9 * gf.linearSystem.nnz + 3 * gf.linearSystem.N, dtype=torch.float64, device=dev)
    rc = lib.icf_assemble_noalloc(gf.ctx, H, *(C.c_void_p(t.data_ptr()) for t in ins),
                                  C.c_void_p(out.data_ptr()), C.c_void_p(out.data_ptr() + 8 * 9 * gf.linearSystem.nnz),
                                  None)
    assert rc == _lib.ICF_ERR_SIZE
    assert b"bytes of scratch" in lib.icf_last_error(gf.ctx)
    gf.close()
