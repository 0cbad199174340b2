"""CUDA path vs the CPU oracle through the C ABI (needs a B200)."""
import ctypes as C

import numpy as np
import pytest

from icflow_b200 import mesh as M
from icflow_b200.gpu_functionality import GPU_Functionality
from icflow_b200.model_prms import config_prms
from tests.harness import (FP64_TOL, Oracle, compare, gpu_assemble, oracle_assemble,
                           orc_prms_from, random_state, rowwise_rel, vec_rel)

pytestmark = pytest.mark.gpu
H = 1e-4


@pytest.fixture(scope="module")
def O():
    return Oracle()


def _gf(coll, prms):
    gf = GPU_Functionality(0)
    gf.prms = prms
    gf.mc = coll
    gf.SetConstants()
    gf.TransferStaticDataToDevice()
    return gf


def _zeros_cz(coll):
    nc = len(coll.czs)
    return np.zeros((nc, 3)), np.zeros((nc, 3)), np.zeros(nc, np.int32)


@pytest.mark.parametrize("seed,du", [(0, 1e-7), (1, 2e-6), (2, 8e-6), (3, 3e-5)])
def test_cantilever_parity(O, seed, du):
    coll = M.cantilever()
    prms = config_prms()
    gf = _gf(coll, prms)
    pmax, tmax, failed = _zeros_cz(coll)
    state = random_state(coll, seed, du=du)
    g = gpu_assemble(gf, coll, state, H, pmax, tmax, failed)
    o = oracle_assemble(O, orc_prms_from(O, prms), coll, state, H, pmax, tmax, np.zeros((0, 4), np.int32))
    compare(g, o)
    assert g["counts"].nCZFailedThisStep == int(o["flags"][:, 2].sum())
    assert g["counts"].nCZDamaged == int(o["flags"][:, 1].sum())
    gf.close()


def test_damaged_and_failed_state(O):
    """Pre-damaged CZs (unload/reload branches), CZs committed as failed before
    the pattern is built, and per-CZ strengths."""
    coll = M.polycrystal(n=6, grains=6, seed=3, platens=False)
    prms = config_prms()
    p = orc_prms_from(O, prms)
    rng = np.random.default_rng(5)
    nc = len(coll.czs)
    q = p.ppr
    pmax = rng.random((nc, 3)) * q.deln * 0.3
    tmax = rng.random((nc, 3)) * q.delt * 0.3
    pmax[rng.random(nc) < 0.3] = 0
    failed = (rng.random(nc) < 0.1).astype(np.int32)
    sig = M.lognormal_strengths(nc, seed=2, granule_pairs=coll.meshes[0].cz_grains)
    gf = _gf(coll, prms)
    gf.SetCZStrengths(sig, sig)
    state = random_state(coll, 9, du=2e-6)
    g = gpu_assemble(gf, coll, state, H, pmax, tmax, failed)
    live = failed == 0
    o = oracle_assemble(O, p, coll, state, H, pmax, tmax, np.zeros((0, 4), np.int32),
                        cz_sigma=(sig, sig), cz_live=live)
    rep = compare(g, o)
    assert rep["vals_rowwise"] <= FP64_TOL
    gf.close()


def test_contact_parity(O):
    """Platens overlapping a small polycrystal: narrow-phase masks, the impact
    set and the pattern with contact pairs are bit-exact; the assembled matrix
    matches to 1e-12."""
    coll = M.polycrystal(n=8, grains=8, seed=1, platens=True, gap=-0.3)
    prms = config_prms(penaltyK=1e8)
    p = orc_prms_from(O, prms)
    pmax, tmax, failed = _zeros_cz(coll)
    state = random_state(coll, 4, du=1e-7)
    xt = coll.x0 + state[0]
    pairs = M.candidate_pairs(coll, xt)
    assert len(pairs) > 0
    gf = _gf(coll, prms)
    g = gpu_assemble(gf, coll, state, H, pmax, tmax, failed, pairs=pairs)
    masks_g = gf.NarrowPhaseMasks(len(pairs))
    masks_o = O.narrow_phase(pairs, coll.selem, xt)
    assert np.array_equal(masks_g, masks_o)
    imp_o = O.impacts(pairs, masks_o, coll.selem, coll.adj_off, coll.adj, coll.faces, xt)
    assert len(imp_o) > 0
    assert np.array_equal(gf.c_itet, imp_o)
    o = oracle_assemble(O, p, coll, state, H, pmax, tmax, imp_o)
    rep = compare(g, o)
    assert g["counts"].nImpacts == len(imp_o)
    gf.close()


def test_contact_regions_parity(O):
    """Every Voronoi region of the point-triangle distance (interior, the three
    edges, the three vertices: point_triange_v2.h:589-841) through the impact
    derivative kernel: 400 impacts of random nodes against random faces of
    the cantilever, injected with SetImpacts, some with anchored vertices (the
    root face).  The oracle's own region of each impact is tallied to show
    the coverage; the assembled matrix and rhs match it to 1e-12."""
    coll = M.cantilever()
    prms = config_prms(penaltyK=1e8)
    p = orc_prms_from(O, prms)
    pmax, tmax, failed = _zeros_cz(coll)
    state = random_state(coll, 11, du=2e-6)
    rng = np.random.default_rng(5)
    faces = coll.faces[rng.integers(0, len(coll.faces), 400)]
    nodes = rng.integers(0, len(coll.x0), 400)
    keep = ~np.any(faces == nodes[:, None], axis=1)
    imps = np.concatenate([nodes[keep, None], faces[keep]], 1).astype(np.int32)
    # at least one vertex of each impact off the anchors (the others respond nothing)
    imps = imps[~np.all(coll.anchored[imps], axis=1)]
    xt = coll.x0 + state[0]
    branches = [O.pt(xt[i].ravel())[5] for i in imps]
    assert len(set(branches)) >= 7, sorted(set(branches))
    gf = _gf(coll, prms)
    g = gpu_assemble(gf, coll, state, H, pmax, tmax, failed, impacts=imps)
    o = oracle_assemble(O, p, coll, state, H, pmax, tmax, imps)
    rep = compare(g, o)
    print("contact regions:", {b: branches.count(b) for b in sorted(set(branches))}, rep)
    gf.close()


def test_deterministic(O):
    coll = M.polycrystal(n=6, grains=5, seed=2, platens=True, gap=-0.3)
    prms = config_prms(penaltyK=1e8)
    gf = _gf(coll, prms)
    pmax, tmax, failed = _zeros_cz(coll)
    state = random_state(coll, 1, du=1e-6)
    pairs = M.candidate_pairs(coll, coll.x0 + state[0])
    a = gpu_assemble(gf, coll, state, H, pmax, tmax, failed, pairs=pairs)
    b = gpu_assemble(gf, coll, state, H, pmax, tmax, failed, pairs=pairs)
    assert np.array_equal(a["vals"], b["vals"]) and np.array_equal(a["rhs"], b["rhs"])
    gf.close()


def test_node_forces_and_commit(O):
    coll = M.cantilever()
    prms = config_prms()
    p = orc_prms_from(O, prms)
    gf = _gf(coll, prms)
    pmax, tmax, failed = _zeros_cz(coll)
    state = random_state(coll, 3, du=4e-6)
    gpu_assemble(gf, coll, state, H, pmax, tmax, failed)
    st = gf.TransferUpdatedStateToHost()
    o = oracle_assemble(O, p, coll, state, H, pmax, tmax, np.zeros((0, 4), np.int32))
    assert vec_rel(o["nodeF"], st["nodeF"]) <= FP64_TOL
    assert np.array_equal(st["failed"], o["flags"][:, 2])
    assert vec_rel(o["tent"][:, 0], st["pmax"][:, 0]) <= FP64_TOL
    assert vec_rel(o["tent"][:, 1], st["tmax"][:, 2]) <= FP64_TOL
    gf.close()


def test_newmark_on_device(O):
    coll = M.cantilever()
    prms = config_prms()
    gf = _gf(coll, prms)
    rng = np.random.default_rng(0)
    n = len(coll.x0)
    u, v, a, du = (rng.random((n, 3)) - 0.5 for _ in range(4))
    u *= 1e-4
    du *= 1e-6
    gf.SetNodeState(u, v, a)
    gf.SetDU(du)
    gf.InferTentativeValues(H)
    un_o, vn_o, an_o, xt_o = O.newmark_infer(H, 0.25, 0.5, coll.x0, u, v, a, du)
    gf.CreateStructure(copy_back=False)
    dx = rng.random(3 * gf.linearSystem.N) - 0.5
    nrm = gf.XtoDU(dx)
    assert abs(nrm - float(dx @ dx)) <= 1e-13 * float(dx @ dx)
    gf.AcceptTentativeValues(H)
    u2, v2, a2, du2 = gf.GetNodeState()
    uo, vo, ao, duo, _ = O.newmark_accept(H, coll.x0, u, v, a, un_o, du)
    assert np.allclose(u2, uo, rtol=0, atol=1e-18) and np.array_equal(du2, np.zeros_like(du2))
    assert vec_rel(vo, v2) <= 1e-12 and vec_rel(ao, a2) <= 1e-12
    gf.close()


def test_error_paths():
    """Bad arguments are rejected on the host with an error code; nothing
    reaches the GPU."""
    from icflow_b200 import _lib

    coll = M.cantilever()
    gf = _gf(coll, config_prms())
    lib = _lib.load()
    assert lib.icf_assemble(gf.ctx, 1e-4, None) == _lib.ICF_ERR_STATE
    bad = np.array([[0, 1, 2, 10 ** 7]], np.int32)
    assert lib.icf_set_impacts(gf.ctx, 1, _lib.iptr(bad)) == _lib.ICF_ERR_ARG
    assert b"out of range" in lib.icf_last_error(gf.ctx)
    pairs = np.array([[0, 10 ** 7]], np.int32)
    n = _lib.C.c_int()
    assert lib.icf_narrow_phase(gf.ctx, 1, _lib.iptr(pairs), _lib.C.byref(n)) == _lib.ICF_ERR_ARG
    gf.CreateStructure()
    assert lib.icf_assemble(gf.ctx, -1.0, None) == _lib.ICF_ERR_ARG
    gf.close()


def test_non_finite_state_is_reported():
    """A NaN in the node state reaches the matrix: the assembly returns
    ICF_ERR_NUMERIC (counts.nonFinite = 1) and the context stays usable."""
    from icflow_b200 import _lib

    coll = M.cantilever()
    prms = config_prms()
    gf = _gf(coll, prms)
    pmax, tmax, failed = _zeros_cz(coll)
    un, vn, an = random_state(coll, 5, du=1e-6)
    gf.TransferPCSR(pmax, tmax, failed)
    gf.CreateStructure()
    bad_v = vn.copy()
    bad_v[np.nonzero(coll.alt >= 0)[0][7]] = np.nan
    lib = _lib.load()
    try:
        gf.TransferNodesToGPU(un, bad_v, an)
    except _lib.ICFError as e:  # rejected on the host: also acceptable
        assert e.code == _lib.ICF_ERR_ARG
    else:
        cnt = _lib.icf_counts()
        assert lib.icf_assemble(gf.ctx, H, C.byref(cnt)) == _lib.ICF_ERR_NUMERIC
        assert cnt.nonFinite == 1 or b"non-finite" in lib.icf_last_error(gf.ctx)
    gf.TransferNodesToGPU(un, vn, an)
    cnt = gf.AssembleElemsAndCZs(H)
    assert cnt.nonFinite == 0
    gf.close()


def test_graph_matches_direct_launch(O):
    """The captured fork/join graph and direct launches give identical bits,
    and a changed time step or pattern re-captures the graph."""
    from icflow_b200 import _lib

    coll = M.polycrystal(n=6, grains=5, seed=4, platens=True, gap=-0.3)
    prms = config_prms(penaltyK=1e8)
    gf = _gf(coll, prms)
    pmax, tmax, failed = _zeros_cz(coll)
    state = random_state(coll, 2, du=1e-6)
    pairs = M.candidate_pairs(coll, coll.x0 + state[0])
    lib = _lib.load()
    outs = []
    for graph in (1, 0, 1):
        _lib.check(gf.ctx, lib.icf_set_graph(gf.ctx, graph))
        outs.append(gpu_assemble(gf, coll, state, H, pmax, tmax, failed, pairs=pairs))
    for o in outs[1:]:
        assert np.array_equal(o["vals"], outs[0]["vals"]) and np.array_equal(o["rhs"], outs[0]["rhs"])
    a = gpu_assemble(gf, coll, state, 2 * H, pmax, tmax, failed, pairs=pairs)
    p = orc_prms_from(O, prms)
    imp = gf.c_itet
    o = oracle_assemble(O, p, coll, state, 2 * H, pmax, tmax, imp)
    compare(a, o)
    gf.close()


def test_structure_kept_for_the_same_impacts(O):
    """A structure request with the impact list the current structure holds
    keeps it (same pattern, same bits); a different list rebuilds it, and
    the assembly matches the oracle either way."""
    coll = M.polycrystal(n=6, grains=5, seed=4, platens=True, gap=-0.3)
    prms = config_prms(penaltyK=1e8)
    gf = _gf(coll, prms)
    pmax, tmax, failed = _zeros_cz(coll)
    p = orc_prms_from(O, prms)
    state = random_state(coll, 2, du=1e-6)
    pairs = M.candidate_pairs(coll, coll.x0 + state[0])
    a = gpu_assemble(gf, coll, state, H, pmax, tmax, failed, pairs=pairs)
    assert len(gf.c_itet) > 0
    b = gpu_assemble(gf, coll, state, H, pmax, tmax, failed, pairs=pairs)  # same impacts
    for k in ("rows", "cols", "vals", "rhs", "ipcsr"):
        assert np.array_equal(a[k], b[k]), k
    # fewer pairs, fewer impacts: a new structure
    c = gpu_assemble(gf, coll, state, H, pmax, tmax, failed, pairs=pairs[: len(pairs) // 2])
    compare(c, oracle_assemble(O, p, coll, state, H, pmax, tmax, gf.c_itet))
    # and back to the first list
    d = gpu_assemble(gf, coll, state, H, pmax, tmax, failed, pairs=pairs)
    for k in ("rows", "cols", "vals", "rhs"):
        assert np.array_equal(a[k], d[k]), k
    # the list grows past the impact buffer (which is then reallocated) and
    # returns to a list a structure was built from: the structure (and the
    # captured graph, which holds the buffer's address) must be rebuilt
    imps = gf.c_itet.copy()
    small = imps[: max(1, len(imps) // 8)]
    f = gpu_assemble(gf, coll, state, H, pmax, tmax, failed, impacts=small)
    big = np.concatenate([imps] * 32)  # repeats are allowed; beyond the buffer's capacity
    gpu_assemble(gf, coll, state, H, pmax, tmax, failed, impacts=big)
    f2 = gpu_assemble(gf, coll, state, H, pmax, tmax, failed, impacts=small)
    for k in ("rows", "cols", "vals", "rhs"):
        assert np.array_equal(f[k], f2[k]), k
    compare(f2, oracle_assemble(O, p, coll, state, H, pmax, tmax, small))
    # contact ends: an empty list after impacts whose blocks the off-diagonal
    # gather also writes (the impact-add launches must all go)
    e = gpu_assemble(gf, coll, state, H, pmax, tmax, failed, impacts=np.zeros((0, 4), np.int32))
    compare(e, oracle_assemble(O, p, coll, state, H, pmax, tmax, np.zeros((0, 4), np.int32)))
    assert e["counts"].nImpacts == 0
    gf.close()


def test_profile_assembly_kernels(O):
    """Per-kernel timing runs the same kernels: same bits as the graph, every
    kernel of the step listed with a positive time and byte count."""
    coll = M.polycrystal(n=6, grains=5, seed=4, platens=True, gap=-0.3)
    prms = config_prms(penaltyK=1e8)
    gf = _gf(coll, prms)
    pmax, tmax, failed = _zeros_cz(coll)
    state = random_state(coll, 2, du=1e-6)
    pairs = M.candidate_pairs(coll, coll.x0 + state[0])
    a = gpu_assemble(gf, coll, state, H, pmax, tmax, failed, pairs=pairs)
    ks = gf.ProfileAssembly(H, reps=3)
    names = [k["name"] for k in ks]
    assert {"k_tet_unit", "k_cz_gp", "k_gather_off", "k_gather_diag"} <= set(names)
    if len(gf.c_itet):
        assert {"k_imp_deriv", "k_imp_add"} <= set(names)
    assert all(k["ms"] > 0 and k["bytes"] > 0 for k in ks)
    vals, rhs = gf.TransferLinearSystemToHost()
    assert np.array_equal(vals.ravel(), a["vals"].ravel()) and np.array_equal(rhs.ravel(), a["rhs"].ravel())
    gf.close()


def test_every_launch_variant_and_autotune(O):
    """Each launch variant of the tet kernel and of both gathers gives blocks
    and rhs within the FP64 bar against the oracle; the autotuner reports a
    timing for every variant and keeps one of each kind."""
    from icflow_b200 import _lib

    coll = M.polycrystal(n=6, grains=5, seed=4, platens=True, gap=-0.3)
    prms = config_prms(penaltyK=1e8)
    gf = _gf(coll, prms)
    pmax, tmax, failed = _zeros_cz(coll)
    state = random_state(coll, 3, du=1e-6)
    pairs = M.candidate_pairs(coll, coll.x0 + state[0])
    ref = gpu_assemble(gf, coll, state, H, pmax, tmax, failed, pairs=pairs)
    p = orc_prms_from(O, prms)
    o = oracle_assemble(O, p, coll, state, H, pmax, tmax, gf.c_itet)
    compare(ref, o)
    lib = _lib.load()
    counts = {}
    for kind in (3, 6, 5, 7, 0, 1, 2, 4):
        v = 0
        while lib.icf_set_variant(gf.ctx, kind, v) == 0:
            gf.AssembleElemsAndCZs(H)
            vals, rhs = gf.TransferLinearSystemToHost()
            assert rowwise_rel(o["rows"], o["vals"], vals.reshape(-1, 3, 3)) <= FP64_TOL, (kind, v)
            assert vec_rel(o["rhs"], rhs) <= FP64_TOL, (kind, v)
            v += 1
        counts[kind] = v
        _lib.check(gf.ctx, lib.icf_set_variant(gf.ctx, kind, 0))
    assert all(n >= 2 for n in counts.values()), counts
    # the per-tet record layout, split and single lists, with every gather variant
    _lib.check(gf.ctx, lib.icf_set_variant(gf.ctx, 3, 0))
    for split in (0, 1):
        _lib.check(gf.ctx, lib.icf_set_variant(gf.ctx, 5, split))
        for kind in (1, 2):
            for v in range(counts[kind]):
                _lib.check(gf.ctx, lib.icf_set_variant(gf.ctx, kind, v))
                gf.AssembleElemsAndCZs(H)
                vals, rhs = gf.TransferLinearSystemToHost()
                assert rowwise_rel(o["rows"], o["vals"], vals.reshape(-1, 3, 3)) <= FP64_TOL, ("records", split, kind, v)
                assert vec_rel(o["rhs"], rhs) <= FP64_TOL
            _lib.check(gf.ctx, lib.icf_set_variant(gf.ctx, kind, 0))
    # the split lists give the same bits as the single ones
    _lib.check(gf.ctx, lib.icf_set_variant(gf.ctx, 5, 0))
    gf.AssembleElemsAndCZs(H)
    v0, r0 = gf.TransferLinearSystemToHost()
    v0, r0 = v0.copy(), r0.copy()
    _lib.check(gf.ctx, lib.icf_set_variant(gf.ctx, 5, 1))
    gf.AssembleElemsAndCZs(H)
    v1, r1 = gf.TransferLinearSystemToHost()
    assert np.array_equal(v0, v1) and np.array_equal(r0, r1)
    names = {k["name"] for k in gf.ProfileAssembly(H, reps=2)}
    assert {"k_gather_off", "k_gather_off_cz", "k_gather_diag", "k_gather_diag_cz"} <= names
    _lib.check(gf.ctx, lib.icf_set_variant(gf.ctx, 3, 1))
    rep = gf.Autotune(H, reps=3)
    kinds = {r["kernel"] for r in rep}
    assert {"layout", "k_tet_unit", "k_cz_gp"} <= kinds
    layout = [r["variant"] for r in rep if r["kernel"] == "layout" and r["chosen"]]
    assert ("gather" in kinds) == (layout == ["per-tet records"]), (layout, kinds)
    if "split" in kinds:  # the list gathers' choices are timed only when the lists run
        assert {"k_gather_off", "k_gather_diag"} <= kinds
    kind_of = {"layout": 3, "gather": 6, "split": 5, "streams": 7, "k_tet_unit": 0, "k_gather_off": 1,
               "k_gather_diag": 2, "k_cz_gp": 4}
    for k in kinds:  # every variant of a timed kind is timed
        assert sum(r["kernel"] == k for r in rep) == counts[kind_of[k]], k
    for k in kinds:
        assert sum(r["chosen"] for r in rep if r["kernel"] == k) == 1
    vals, rhs = gf.TransferLinearSystemToHost()
    assert rowwise_rel(o["rows"], o["vals"], vals.reshape(-1, 3, 3)) <= FP64_TOL
    gf.AssembleElemsAndCZs(H)
    vals2, rhs2 = gf.TransferLinearSystemToHost()
    assert np.array_equal(vals, vals2) and np.array_equal(rhs, rhs2)
    gf.close()


FP32_TOL = 1e-5  # FP32-mixed blocks, normwise per block row against the FP64 oracle


@pytest.mark.parametrize("case", ["cantilever_damaged", "polycrystal_contact"])
def test_fp32_mixed_error_report(O, case):
    """FP32-mixed assembly against the FP64 oracle, per field: Hessian blocks
    within FP32_TOL normwise per block row; rhs, tentative CZ state and flags
    as in FP64 (the law, tractions, forces and rhs stay FP64)."""
    from icflow_b200 import _lib

    prms = config_prms(penaltyK=1e8)
    if case == "cantilever_damaged":
        coll = M.cantilever()
        state = random_state(coll, 7, du=8e-6)
        pairs = None
    else:
        coll = M.polycrystal(n=8, grains=6, seed=2, platens=True, gap=-0.3)
        state = random_state(coll, 8, du=2e-6)
        pairs = M.candidate_pairs(coll, coll.x0 + state[0])
    gf = _gf(coll, prms)
    _lib.check(gf.ctx, gf.lib.icf_set_precision(gf.ctx, 1))
    pmax, tmax, failed = _zeros_cz(coll)
    a = gpu_assemble(gf, coll, state, H, pmax, tmax, failed, pairs=pairs)
    p = orc_prms_from(O, prms)
    o = oracle_assemble(O, p, coll, state, H, pmax, tmax, gf.c_itet if pairs is not None else
                        np.zeros((0, 4), np.int32))
    assert np.array_equal(a["rows"], o["rows"]) and np.array_equal(a["cols"], o["cols"])
    err_vals = rowwise_rel(o["rows"], o["vals"], a["vals"])
    err_rhs = vec_rel(o["rhs"], a["rhs"])
    assert 0 < err_vals <= FP32_TOL, err_vals
    assert err_rhs <= FP64_TOL, err_rhs
    sel = o["czsel"]
    if len(sel):
        assert np.array_equal(a["flags"][sel], o["flags"])
        assert vec_rel(o["tent"], a["tent"][sel]) <= FP64_TOL
    print(f"{case}: FP32-mixed vs FP64 oracle: blocks {err_vals:.2e} (rowwise), rhs {err_rhs:.2e}")
    gf.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_tiled_gather(O, precision):
    """The row-tile gather (one CTA per tile, tet records and codes staged in
    shared memory) against the oracle, in both precisions, for two structures
    of the same model (the contact blocks move the merged slots); its
    off-diagonal blocks equal the list gather's bit for bit (one lane per
    block, same code order).  The fused tiles (tets computed in shared
    memory, no tet kernel) give the tile gather's bits, node forces included."""
    from icflow_b200 import _lib

    prms = config_prms(penaltyK=1e8)
    coll = M.polycrystal(n=8, grains=6, seed=2, platens=True, gap=-0.3)
    gf = _gf(coll, prms)
    lib = _lib.load()
    _lib.check(gf.ctx, lib.icf_set_precision(gf.ctx, precision))
    p = orc_prms_from(O, prms)
    tol = FP64_TOL if precision == 0 else FP32_TOL
    for seed in (8, 9):
        state = random_state(coll, seed, du=2e-6)
        pmax, tmax, failed = _zeros_cz(coll)
        pairs = M.candidate_pairs(coll, coll.x0 + state[0])
        _lib.check(gf.ctx, lib.icf_set_variant(gf.ctx, 6, 0))
        a = gpu_assemble(gf, coll, state, H, pmax, tmax, failed, pairs=pairs)
        _lib.check(gf.ctx, lib.icf_set_variant(gf.ctx, 6, 1))
        gf.AssembleElemsAndCZs(H)
        vals, rhs = gf.TransferLinearSystemToHost()
        vals = vals.reshape(-1, 3, 3)
        names = {k["name"] for k in gf.ProfileAssembly(H, reps=2)}
        assert "k_gather_tile" in names and "k_gather_off" not in names, names
        o = oracle_assemble(O, p, coll, state, H, pmax, tmax, gf.c_itet)
        assert np.array_equal(a["rows"], o["rows"]) and np.array_equal(a["cols"], o["cols"])
        assert rowwise_rel(o["rows"], o["vals"], vals) <= tol
        assert vec_rel(o["rhs"], rhs) <= FP64_TOL
        row_of = np.repeat(np.arange(len(a["rows"]) - 1), np.diff(a["rows"]))
        off = a["cols"] != row_of
        assert np.array_equal(vals[off], a["vals"][off])
        cnt = gf.AssembleElemsAndCZs(H)
        assert cnt.nonFinite == 0
        # the fused tiles compute the tets in shared memory with the tet
        # kernel's arithmetic and sum the same values in the same order
        _lib.check(gf.ctx, lib.icf_set_variant(gf.ctx, 6, 2))
        gf.AssembleElemsAndCZs(H)
        vf, rf = gf.TransferLinearSystemToHost()
        names = {k["name"] for k in gf.ProfileAssembly(H, reps=2)}
        assert "k_tile_fused" in names and "k_tet_unit" not in names, names
        assert np.array_equal(vf.reshape(-1, 3, 3), vals) and np.array_equal(rf, rhs)
        # node forces need the tet rhs, which the fused tiles never stage
        F_fused = gf.TransferUpdatedStateToHost(want_forces=True)["nodeF"]
        _lib.check(gf.ctx, lib.icf_set_variant(gf.ctx, 6, 0))
        gf.AssembleElemsAndCZs(H)
        F_lists = gf.TransferUpdatedStateToHost(want_forces=True)["nodeF"]
        assert np.array_equal(F_fused, F_lists)
    gf.close()


def test_device_broad_phase_matches_host_pairs(O):
    """The device broad phase gives the host generator's pair set, and the
    narrow phase from those device-resident pairs gives the same impacts."""
    for seed, gap in ((1, -0.3), (2, -0.05), (3, 0.2)):
        coll = M.polycrystal(n=7, grains=5, seed=seed, platens=True, gap=gap)
        prms = config_prms(penaltyK=1e8)
        gf = _gf(coll, prms)
        un, vn, an = random_state(coll, seed, du=3e-6)
        gf.TransferNodesToGPU(un, vn, an)
        n = gf.BroadPhase()
        dev = gf.GetPairs()
        host = M.candidate_pairs(coll, coll.x0 + un)
        assert n == len(host) and np.array_equal(dev, host), (seed, n, len(host))
        imps_dev = gf.NarrowPhaseCollisionDetection(None).copy()
        imps_host = gf.NarrowPhaseCollisionDetection(host).copy()
        assert np.array_equal(imps_dev, imps_host)
        # pairs of different meshes only, through (cell, group) keys and,
        # for group ids that do not fit them (a negative one), the per-cell scan
        from icflow_b200 import _lib
        cross = M.candidate_pairs(coll, coll.x0 + un, same_mesh=False)
        assert len(cross) < len(host)  # none when the platens stand clear (gap > 0)
        for shift in (0, -1):
            grp = np.ascontiguousarray(coll.selem_mesh, np.int32) + shift
            _lib.check(gf.ctx, gf.lib.icf_set_surface_groups(gf.ctx, len(grp), _lib.iptr(grp)))
            n2 = C.c_int()
            _lib.check(gf.ctx, gf.lib.icf_broad_phase(gf.ctx, 0.0, C.byref(n2)))
            gf.nPairs = n2.value
            assert n2.value == len(cross) and np.array_equal(gf.GetPairs(), cross), shift
        gf.close()


def test_detect_contacts_matches_the_pair_pipeline(O):
    """icf_detect_contacts (one query per surface node in a grid of the
    surface elements, no pair list) gives the impact list of the device broad
    phase + narrow phase + closest face, entry for entry: platen contact at
    several gaps, rotated meshes, a widened box (pad), groups (also with a
    negative group id), and two ice blocks driven into each other."""
    from icflow_b200 import _lib

    # "ice_far": the blocks half a metre apart, so the grid over the boxes' hull
    # has more cells than the first guess of its buffers (one per surface
    # element): the first call grows them and runs again
    cases = [("poly", 1, -0.3, None, 0.0), ("poly", 2, -0.05, _rot([1, 1, 0], 35), 0.0),
             ("poly", 3, 0.2, None, 0.0), ("poly", 4, -0.25, _rot([1, 0, 2], 60), 2e-3), ("ice", 5, 0, None, 0.0),
             ("ice_far", 6, 0.5, None, 0.0)]
    for kind, seed, gap, R, pad in cases:
        if kind == "poly":
            coll = M.polycrystal(n=7, grains=5, seed=seed, platens=True, gap=gap)
            if R is not None:
                coll = _rotate(coll, R)
            un, vn, an = random_state(coll, seed, du=3e-6)
        elif kind == "ice":
            coll, _ = M.ice_impact(n=6, grains=6, seed=seed, size=(0.02, 0.02, 0.01))
            un, vn, an = random_state(coll, seed, du=1e-6)
            na = coll.meshes[0].n_nodes
            un[:na, 2] += 2e-4  # block A driven 0.1 mm into block B
        else:
            coll, _ = M.ice_impact(n=6, grains=6, seed=seed, size=(0.02, 0.02, 0.01), gap=gap)
            un, vn, an = random_state(coll, seed, du=1e-5)
        gf = _gf(coll, config_prms(penaltyK=1e8))
        gf.TransferNodesToGPU(un, vn, an)
        for same_mesh in (True, False):
            gf.BroadPhase(pad=pad, same_mesh=same_mesh)
            ref = gf.NarrowPhaseCollisionDetection(None).copy()
            det = gf.DetectContacts(pad=pad, same_mesh=same_mesh).copy()
            assert np.array_equal(det, ref), (kind, seed, same_mesh, len(det), len(ref))
            if same_mesh:
                n_same = len(ref)
        assert n_same > 0 or gap > 0, (kind, seed)
        # a negative group id
        grp = np.ascontiguousarray(coll.selem_mesh, np.int32) - 1
        _lib.check(gf.ctx, gf.lib.icf_set_surface_groups(gf.ctx, len(grp), _lib.iptr(grp)))
        n2 = C.c_int()
        _lib.check(gf.ctx, gf.lib.icf_broad_phase(gf.ctx, pad, C.byref(n2)))
        ref = gf.NarrowPhaseCollisionDetection(None).copy()
        _lib.check(gf.ctx, gf.lib.icf_detect_contacts(gf.ctx, pad, C.byref(n2)))
        det = np.zeros((n2.value, 4), np.int32)
        if n2.value:
            _lib.check(gf.ctx, gf.lib.icf_get_impacts(gf.ctx, n2.value, _lib.iptr(det)))
        assert np.array_equal(det, ref), (kind, seed, "negative groups")
        print(f"{kind} seed {seed}: {n_same} impacts (all meshes), equal to the pair pipeline")
        gf.close()


def _rotate(coll, R, mesh=None):
    """A copy of the collection with the nodes of one mesh (all meshes when
    None) rotated by R about that part's centroid."""
    import copy

    c = copy.deepcopy(coll)
    off = 0
    for i, m in enumerate(c.meshes):
        n = m.n_nodes
        if mesh is None or i == mesh:
            sl = slice(off, off + n)
            cen = c.x0[sl].mean(axis=0) if mesh is not None else coll.x0.mean(axis=0)
            c.x0[sl] = cen + (c.x0[sl] - cen) @ R.T
            m.x0 = c.x0[sl].copy()
        off += n
    return c


def _rot(axis, deg):
    a = np.asarray(axis, float) / np.linalg.norm(axis)
    t = np.radians(deg)
    K = np.array([[0, -a[2], a[1]], [a[2], 0, -a[0]], [-a[1], a[0], 0]])
    return np.eye(3) + np.sin(t) * K + (1 - np.cos(t)) * K @ K


def test_broad_phase_covers_the_reference_kdop_pairs(O):
    """The reference's broad phase is a k-DOP-24 BVH over all surface elements
    (BVHT.cs:29-77, BVHN.cs:39-194, kDOP24.cs:69-169); its self-collide lists
    every unordered pair of overlapping k-DOPs, same-mesh pairs included (and
    across a grain boundary those give impacts).  The device grid broad phase
    lists the pairs with overlapping boxes that share no node and where a
    vertex of one lies in the other's box.  An impact needs a vertex of one
    element inside the other, so such a pair overlaps in every k-DOP
    direction, shares no node (the narrow phase skips those) and has that
    vertex in the other's box: every k-DOP pair that can give an impact must
    be a device pair.  Checked: that containment, and equal impact lists from
    the two pair sets (the oracle's narrow phase on all k-DOP pairs against
    the device's on its own), with rotated meshes, where boxes and k-DOPs
    differ most."""
    cases = [(1, -0.3, None, None), (2, -0.05, _rot([1, 1, 0], 35), None),
             (3, -0.2, _rot([0, 1, 0], 10), 1), (4, -0.25, _rot([1, 0, 2], 60), None)]
    for seed, gap, R, mesh in cases:
        coll = M.polycrystal(n=7, grains=5, seed=seed, platens=True, gap=gap)
        if R is not None:
            coll = _rotate(coll, R, mesh)
        prms = config_prms(penaltyK=1e8)
        gf = _gf(coll, prms)
        un, vn, an = random_state(coll, seed, du=3e-6)
        gf.TransferNodesToGPU(un, vn, an)
        xt = coll.x0 + un
        n_dev = gf.BroadPhase()
        dev = gf.GetPairs()
        kd = O.kdop_pairs(coll.selem, xt)
        se = coll.selem
        lo, hi = xt[se].min(axis=1), xt[se].max(axis=1)
        a, b = kd[:, 0], kd[:, 1]
        shared = (se[a][:, :, None] == se[b][:, None, :]).any(axis=(1, 2))
        va, vb = xt[se[a]], xt[se[b]]
        vib = (np.all((va >= lo[b][:, None]) & (va <= hi[b][:, None]), axis=2).any(axis=1) |
               np.all((vb >= lo[a][:, None]) & (vb <= hi[a][:, None]), axis=2).any(axis=1))
        can = kd[~shared & vib]
        dev_set = set(map(tuple, dev.tolist()))
        assert all(tuple(p) in dev_set for p in can.tolist()), (seed, "k-DOP pair missing from the device set")
        cross = kd[coll.selem_mesh[a] != coll.selem_mesh[b]]
        imp_dev = gf.NarrowPhaseCollisionDetection(None).copy()
        masks = O.narrow_phase(kd, coll.selem, xt)
        imp_ref = O.impacts(kd, masks, coll.selem, coll.adj_off, coll.adj, coll.faces, xt)
        assert len(imp_ref) > 0, seed
        assert np.array_equal(imp_dev, imp_ref), (seed, len(imp_dev), len(imp_ref))
        assert np.array_equal(gf.DetectContacts(), imp_ref), seed
        print(f"seed {seed}: device pairs {n_dev}, k-DOP pairs {len(kd)} ({len(cross)} across meshes, "
              f"{len(can)} that can give an impact), impacts {len(imp_ref)}")
        gf.close()
