"""Parity at the sizes the benchmark measures, on exactly its workloads.

bench.build_workload builds the benchmark's seeded synthetic inputs (mesh,
compressed state, per-boundary strengths, broad-phase pairs); these tests
assemble the same inputs through the C ABI, with the launch variants the
autotuner picks (as bench.py does), and compare with the CPU oracle:

  cfg1  polycrystal compression, 196,608 tets, 34,819 CZs, ~22,700 impacts
        (platens and grain boundaries): the device broad phase's pair set
        equals the host rule's; masks, impacts (also from the detection
        without a pair list), csr_rows/cols and every slot map bit-exact; blocks
        within 1e-12 per block row; rhs within 1e-12; CZ flags equal;
        tentative state and averages within 1e-12.
  cfg2  the same at 1,572,864 tets in FP64 (same bar), then in FP32-mixed with
        each field's error reported against the FP64 oracle.
  cfg3  the batched path (one collection of uneven specimens, one graph per
        assembly) on the first 8 of the 64 specimens, FP64 and FP32-mixed.

Effects that only appear at scale are exercised here: thousands of
sliced-ELL windows, the 24/26-bit unit fields of the contribution codes,
structure merges with thousands of contact keys, graph updates.
"""
from __future__ import annotations

import numpy as np
import pytest

import bench
from tests.harness import (Oracle, compare, gpu_assemble, orc_prms_from, oracle_assemble, rowwise_rel,
                           vec_rel)

from icflow_b200 import mesh as M
from icflow_b200.gpu_functionality import GPU_Functionality
from icflow_b200.model_prms import config_prms

H = bench.H
MIXED_BLOCK_TOL = 1e-5  # FP32 Hessians (2^-24 ~ 6e-8 per product, sums of ~30 terms)


def _gf(coll, sig, precision, tune):
    prms = config_prms(penaltyK=1e8)
    gf = GPU_Functionality(0)
    gf.prms = prms
    gf.mc = coll
    gf.SetConstants()
    gf.SetPrecision(precision)
    gf.TransferStaticDataToDevice()
    gf.SetCZStrengths(sig, sig)
    return gf, prms


def _oracle(O, prms, coll, state, sig, pairs):
    """The oracle's narrow phase, impacts and assembly on the given pairs."""
    p = orc_prms_from(O, prms)
    xt = coll.x0 + state[0]
    masks = O.narrow_phase(pairs, coll.selem, xt) if len(pairs) else np.zeros(0, np.int32)
    imps = (O.impacts(pairs, masks, coll.selem, coll.adj_off, coll.adj, coll.faces, xt) if len(pairs)
            else np.zeros((0, 4), np.int32))
    nc = len(coll.czs)
    o = oracle_assemble(O, p, coll, state, H, np.zeros((nc, 3)), np.zeros((nc, 3)), imps, cz_sigma=(sig, sig))
    return o, masks, imps


def _device_pairs(gf, coll, state):
    """The device broad phase's pairs at the state's positions (as bench.py
    builds the workload)."""
    un, vn, an = state
    gf.TransferNodesToGPU(un, vn, an)
    gf.BroadPhase()
    return gf.GetPairs()


def _gpu(gf, coll, state, pairs, tune):
    nc = len(coll.czs)
    z3 = np.zeros((nc, 3))
    if tune:
        # the bench's order: structure, autotune, then the assembly it measures
        un, vn, an = state
        gf.TransferNodesToGPU(un, vn, an)
        gf.TransferPCSR(z3, z3, np.zeros(nc, np.int32))
        if len(pairs):
            gf.NarrowPhaseCollisionDetection(pairs)
        gf.CreateStructure(copy_back=False)
        gf.Autotune(H, reps=3)
    return gpu_assemble(gf, coll, state, H, z3, z3, np.zeros(nc, np.int32),
                        pairs=pairs if len(pairs) else None,
                        impacts=None if len(pairs) else np.zeros((0, 4), np.int32))


def _mixed_report(g, o):
    sel = o["czsel"]
    rep = {"blocks_rowwise": rowwise_rel(o["rows"], o["vals"], g["vals"]),
           "rhs": vec_rel(o["rhs"], g["rhs"]),
           "cz_flags_equal": bool(np.array_equal(g["flags"][sel], o["flags"])),
           "tentative": vec_rel(o["tent"], g["tent"][sel]),
           "averages": vec_rel(o["avg"], g["avg"][sel])}
    assert np.array_equal(g["rows"], o["rows"]) and np.array_equal(g["cols"], o["cols"])
    assert rep["cz_flags_equal"], rep
    assert rep["blocks_rowwise"] <= MIXED_BLOCK_TOL, rep
    # rhs, law, damage state and averages are FP64 in the mixed mode too
    assert rep["rhs"] <= 1e-12 and rep["tentative"] <= 1e-12 and rep["averages"] <= 1e-12, rep
    return rep


@pytest.mark.gpu
def test_cfg1_bench_workload_parity():
    coll, state, sig, _, _ = bench.build_workload("cfg1", 0)
    O = Oracle()
    gf, prms = _gf(coll, sig, 0, True)
    pairs = _device_pairs(gf, coll, state)
    # the broad phase's pair set is the host rule's (oracle/icf_oracle.c)
    assert np.array_equal(pairs, O.candidate_pairs(coll.selem, coll.x0 + state[0]))
    g = _gpu(gf, coll, state, pairs, tune=True)
    o, masks, imps = _oracle(O, prms, coll, state, sig, pairs)
    assert np.array_equal(gf.NarrowPhaseMasks(len(pairs)), masks)
    assert len(imps) > 1000 and np.array_equal(gf.c_itet, imps)
    rep = compare(g, o)
    assert g["counts"].nImpacts == len(imps) and g["counts"].nLawExact == 0
    # contact detection without the pair list: the same impacts
    assert np.array_equal(gf.DetectContacts(), imps)
    gf.close()
    print("cfg1 parity:", {k: f"{v:.1e}" for k, v in rep.items()})


@pytest.mark.gpu
def test_cfg2_bench_workload_fp64_parity_and_mixed_error():
    coll, state, sig, _, _ = bench.build_workload("cfg2", 0)
    O = Oracle()
    gf, prms = _gf(coll, sig, 0, True)
    pairs = _device_pairs(gf, coll, state)
    g = _gpu(gf, coll, state, pairs, tune=False)
    o, masks, imps = _oracle(O, prms, coll, state, sig, pairs)
    assert np.array_equal(gf.NarrowPhaseMasks(len(pairs)), masks)
    assert np.array_equal(gf.c_itet, imps)
    rep = compare(g, o)
    assert np.array_equal(gf.DetectContacts(), imps)
    print("cfg2 FP64 parity:", {k: f"{v:.1e}" for k, v in rep.items()})
    gf.SetPrecision(1)
    g32 = _gpu(gf, coll, state, pairs, tune=True)
    mrep = _mixed_report(g32, o)
    gf.close()
    print("cfg2 FP32-mixed error vs the FP64 oracle:", mrep)


@pytest.mark.gpu
def test_cfg3_batched_specimens_parity():
    coll, info = M.batched_specimens(bench.N_SPECIMENS, seed=0, only=list(range(8)))
    sig = np.concatenate([M.lognormal_strengths(len(m.czs), seed=i, granule_pairs=m.cz_grains)
                          for (i, _, _), m in zip(info, coll.meshes)])
    state = bench._state(coll, 0)
    pairs = np.zeros((0, 2), np.int32)
    O = Oracle()
    gf, prms = _gf(coll, sig, 0, True)
    g = _gpu(gf, coll, state, pairs, tune=True)
    o, _, _ = _oracle(O, prms, coll, state, sig, pairs)
    rep = compare(g, o)
    print(f"cfg3 (8 specimens, {len(coll.elems)} tets) FP64 parity:", {k: f"{v:.1e}" for k, v in rep.items()})
    gf.SetPrecision(1)
    g32 = _gpu(gf, coll, state, pairs, tune=True)
    mrep = _mixed_report(g32, o)
    gf.close()
    print("cfg3 FP32-mixed error vs the FP64 oracle:", mrep)
