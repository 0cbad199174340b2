"""Benchmark of the icFlow assembly path on B200.

One step = one Newton assembly (zero + tetrahedra + cohesive zones with damage
state and flags + contact response -> BCSR values and rhs) of a fixed
structure.  Workloads (--workload):
  cfg1            polycrystal compression: 1 mm cube, 32^3 hexahedra split into
                  196,608 tets, 128 Voronoi grains with cohesive zones on every
                  grain boundary (per-boundary lognormal strengths, mean 1 MPa,
                  cv 0.2), two rigid platens overlapping the cube by a quarter
                  cell (penalty 1e8), dt = 1e-5 s, FP64;
  cfg2 (default)  the same at 64^3 hexahedra (1,572,864 tets), 2048 grains: the
                  1.5M-tet size the throughput target is stated at; the line
                  also carries the FP32-mixed measurement of the same workload;
  cfg3            64 independent cubes of uneven size (tets U[5k, 60k], grains
                  U[8, 64]) assembled together in one graph launch, launch
                  variants autotuned, FP32-mixed by default.
Inputs are synthetic (seeded), as icFlow ships no setups.

  value  assemblies/s with inputs resident in HBM (device events around each
         step; L2 is flushed between steps by writing a 256 MiB buffer, outside
         the timed region)
  e2e    the same through the C ABI with host buffers: H2D of the tentative
         node state (un, vn, an) from pinned memory, assembly, D2H of vals and
         rhs into pinned memory, every step

`--impl reference` times the reference's own kernels compiled for the host
(oracle/_ref, all host threads) on the same workload.  Under torchrun, for
cfg1/cfg2 each rank assembles its own specimen (seed = rank, weak scaling);
for cfg3 the 64 specimens are split across the ranks (strong scaling).  No
collective touches the data path; timing is max over ranks.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Newton assemblies/s (elem+CZ+contact->BCSR)"
H = 1e-5
FLUSH_BYTES = 256 << 20


WORKLOADS = {
    # polycrystal compression, 1 mm cube: (hexes per side, grains); one
    # specimen per rank (weak scaling)
    "cfg1": (32, 128),    # 196,608 tets, ~35k CZs
    "cfg2": (64, 2048),   # 1,572,864 tets, ~396k CZs
    # 64 uneven specimens (tets U[5k, 60k], grains U[8, 64]) assembled together
    # in one graph launch; the specimens are split across ranks (strong scaling)
    "cfg3": None,
}
N_SPECIMENS = 64


def workload_name(workload: str, n: int = 0, grains: int = 0) -> str:
    if workload == "cfg3":
        return (f"{N_SPECIMENS} independent polycrystal cubes, tets U[5k,60k], grains U[8,64], CZs on grain "
                "boundaries, per-boundary lognormal strengths, one graph launch per assembly, dt 1e-5")
    return (f"polycrystal compression, 1 mm cube, {n}^3 hex -> 6 tets ({6 * n ** 3} tets), {grains} grains, "
            "CZs on grain boundaries, rigid platens in contact, dt 1e-5")


def _state(coll, seed):
    rng = np.random.default_rng(seed + 101)
    nn = len(coll.x0)
    # a compressed state: uniform strain 1e-4 toward each specimen's mid-plane plus noise
    zc = 0.5e-3
    un = np.zeros((nn, 3))
    un[:, 2] = -1e-4 * (coll.x0[:, 2] - zc)
    un += (rng.random((nn, 3)) - 0.5) * 2e-9
    un[coll.anchored] = 0.0
    vn = (rng.random((nn, 3)) - 0.5) * 1e-3
    an = (rng.random((nn, 3)) - 0.5) * 1e-1
    return un, vn, an


def build_workload(workload: str, seed: int, rank: int = 0, world: int = 1):
    """(collection, (un, vn, an), per-CZ strengths, candidate pairs, units of
    the metric this rank's collection holds).  The polycrystal workloads'
    pairs are None: they come from the broad phase at the state's positions
    (every overlapping surface-element pair sharing no node, same mesh
    included, as the reference's BVH lists them)."""
    from icflow_b200 import mesh as M

    if workload == "cfg3":
        from icflow_b200.shard import shard

        mine = shard(N_SPECIMENS, rank, world)
        coll, info = M.batched_specimens(N_SPECIMENS, seed=seed, only=mine)
        sig = np.concatenate([M.lognormal_strengths(len(m.czs), seed=1000 * seed + i, granule_pairs=m.cz_grains)
                              for (i, _, _), m in zip(info, coll.meshes)])
        pairs = np.zeros((0, 2), np.int32)
        return coll, _state(coll, seed), sig, pairs, len(mine) / N_SPECIMENS
    n, grains = WORKLOADS[workload]
    coll = M.polycrystal(n=n, grains=grains, seed=seed, platens=True, gap=-0.25)
    un, vn, an = _state(coll, seed)
    sig = M.lognormal_strengths(len(coll.czs), seed=seed, granule_pairs=coll.meshes[0].cz_grains)
    return coll, (un, vn, an), sig, None, 1.0


def algorithmic_bytes(nnz, n_active, n_nodes, n_tet, n_cz, n_imp) -> int:
    """Compulsory traffic of one assembly, FP64 layout, each item once:
    72 B per 3x3 block written, 24 B per rhs row, 96 B per node (x0, u, v, a),
    56 B per tet (4 ids + 10 upper-block slots), 240 B per CZ (6 ids, 21 slots,
    6 state in, 6 tentative out, 4 averages, flags), 56 B per impact."""
    return 72 * nnz + 24 * n_active + 96 * n_nodes + 56 * n_tet + 240 * n_cz + 56 * n_imp


def kernel_share_bytes(name, nnz, n_rows, n_nodes, n_tet, n_cz, n_imp) -> int:
    """The part of algorithmic_bytes a kernel is responsible for: the node
    state and tet ids to the tet kernel, the CZ items to the CZ kernel, the
    off-diagonal blocks (contact-only ones included) to the off-diagonal
    gather, the diagonal blocks and rhs rows to the diagonal gather, the
    impact items to the impact derivatives; the row-tile gather writes both
    kinds of blocks.  Summed over one assembly's kernels this is
    algorithmic_bytes."""
    return {"k_tet_unit": 96 * n_nodes + 56 * n_tet,
            "k_cz_gp": 240 * n_cz,
            "k_gather_off": 72 * (nnz - n_rows),
            "k_gather_diag": 72 * n_rows + 24 * n_rows,
            "k_gather_tile": 72 * nnz + 24 * n_rows,
            "k_imp_deriv": 56 * n_imp}.get(name, 0)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 7:
                continue
            try:
                sm.append(float(parts[0]))
                mx.append(float(parts[1]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[3:7]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_env():
    from icflow_b200.shard import dist_env as env

    return env()


def cpu_model() -> str:
    try:
        for ln in open("/proc/cpuinfo"):
            if ln.startswith("model name"):
                return ln.split(":", 1)[1].strip() + f" ({os.cpu_count()} logical CPUs)"
    except OSError:
        pass
    return f"{os.cpu_count()} logical CPUs"


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def ncu_traffic(workload: str, precision: str):
    """DRAM bytes (read + write) per launch of each kernel, from the committed
    summary of an ncu capture of this workload (profiles/dram_traffic.json,
    which names the command and the code it was taken on), or {}."""
    p = ROOT / "profiles" / "dram_traffic.json"
    if p.exists():
        try:
            d = json.loads(p.read_text()).get(workload, {})
            return d.get(precision, {}) if isinstance(d.get(precision), dict) else {}
        except (ValueError, OSError):
            return {}
    return {}


def cpu_baseline(coll, state, sig, pairs, bound_s: float = 12.0, nthreads: int = 0):
    """The reference's own kernels (oracle/_ref) on the host over the same
    workload; returns (assemblies/s, threads, kind, sample)."""
    from oracle.oracle import Oracle, RefKernels, ref_available

    O = Oracle()
    kind = "reference" if ref_available() else "port"
    from icflow_b200.model_prms import config_prms

    prms = config_prms(penaltyK=1e8)
    keys = ("Y", "nu", "rho", "dampingMass", "dampingStiffness", "gravity", "NewmarkBeta", "NewmarkGamma",
            "alpha", "beta", "lambda_n", "lambda_t", "phi_n", "phi_t", "sigma_max", "tau_max", "penaltyK",
            "DistanceEpsilon")
    p = O.prms(**{k: getattr(prms, k) for k in keys})
    un, vn, an = state
    xt = coll.x0 + un
    if pairs is None:  # the broad phase's rule, on the host
        pairs = O.candidate_pairs(coll.selem, xt)
    masks = O.narrow_phase(pairs, coll.selem, xt)
    imps = O.impacts(pairs, masks, coll.selem, coll.adj_off, coll.adj, coll.faces, xt)
    N, rows, cols = O.build_structure(coll.alt, coll.elems, coll.czs, imps)
    ep = O.pcsr(coll.elems, 4, coll.alt, rows, cols, N)
    cp = O.pcsr(coll.czs, 6, coll.alt, rows, cols, N)
    ipc = O.pcsr(imps, 4, coll.alt, rows, cols, N)
    nc = len(coll.czs)
    pmax = np.zeros((nc, 3))
    tmax = np.zeros((nc, 3))
    threads = nthreads or os.cpu_count()
    if kind == "reference":
        R = RefKernels(nthreads=threads)
        R.set_constants(p)
        qs = [O.ppr_for(p, s, s) for s in sig]
        per_cz = (sig, sig, np.array([q.deln for q in qs]), np.array([q.delt for q in qs]))

        def one():
            st = R.pack_nodes(coll.x0, un, vn, an)
            vals = np.zeros(9 * len(cols))
            rhs = np.zeros(3 * N)
            R.elem_kernel(st, H, coll.elems, ep, vals, rhs)
            R.cz_kernel(st, H, coll.czs, cp, pmax, tmax, vals, rhs, per_cz=per_cz)
            R.collision_kernel(st, H, imps, ipc, vals, rhs, prms.penaltyK, prms.DistanceEpsilon)
    else:
        threads = 1
        qs = [O.ppr_for(p, s, s) for s in sig]

        def one():
            O.assemble(p, H, coll.x0, un, vn, an, coll.elems, ep, coll.czs, cp, pmax, tmax, imps, ipc,
                       len(cols), N, cz_ppr=qs)
    one()  # warm-up
    n = 0
    t0 = time.perf_counter()
    while True:
        one()
        n += 1
        if time.perf_counter() - t0 > bound_s:
            break
    dt = time.perf_counter() - t0
    return n / dt, threads, kind, f"{n} full assemblies of the workload in {dt:.1f} s"


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    coll, state, sig, pairs, _ = build_workload(args.workload, 0)
    steps = max(args.steps, 1)
    rate, threads, kind, sample = cpu_baseline(coll, state, sig, pairs,
                                               bound_s=min(60.0, 2.0 * steps))
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": "assemblies/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 / rate, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "config": {"workload": workload_name(args.workload, *(WORKLOADS[args.workload] or ())),
                       "tets": int(len(coll.elems)), "czs": int(len(coll.czs))},
            "cpu_baseline": {"value": rate, "unit": "assemblies/s", "cores": threads, "kind": kind,
                             "sample": sample},
            "e2e": {"value": rate, "unit": "assemblies/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def _device_ms(gf, lib, stream, flush, steps, warmup, barrier, H_):
    """Mean device time of `steps` assemblies (graph launches) with the inputs
    resident in HBM: CUDA events on the launching stream around each launch, L2
    flushed by a 256 MiB write between launches, outside the events."""
    import torch

    from icflow_b200 import _lib

    for _ in range(warmup):
        rc = lib.icf_assemble_async(gf.ctx, H_)
        if rc:
            _lib.check(gf.ctx, rc)
    cnt = _lib.icf_counts()
    _lib.check(gf.ctx, lib.icf_read_counts(gf.ctx, C.byref(cnt)))
    starts = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    ends = [torch.cuda.Event(enable_timing=True) for _ in range(steps)]
    barrier()
    with torch.cuda.stream(stream):
        for i in range(steps):
            flush.zero_()
            starts[i].record(stream)
            rc = lib.icf_assemble_async(gf.ctx, H_)
            if rc:
                _lib.check(gf.ctx, rc)
            ends[i].record(stream)
    barrier()
    _lib.check(gf.ctx, lib.icf_read_counts(gf.ctx, C.byref(cnt)))
    return float(np.mean([a.elapsed_time(b) for a, b in zip(starts, ends)])), cnt


def run_ours(args):
    import torch

    from icflow_b200 import _lib
    from icflow_b200.gpu_functionality import GPU_Functionality
    from icflow_b200.model_prms import config_prms

    ws, rank, local = dist_env()
    if ws > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = local if ws > 1 else 0
    torch.cuda.set_device(dev)

    # cfg1/cfg2: one specimen per rank (seed = rank); cfg3: this rank's share
    # of the 64 specimens (seed 0 for all ranks)
    batched = args.workload == "cfg3"
    coll, state, sig, pairs, units = build_workload(args.workload, 0 if batched else rank, rank, ws)
    prms = config_prms(penaltyK=1e8)
    gf = GPU_Functionality(dev)
    gf.prms = prms
    gf.mc = coll
    gf.SetConstants()
    precision = args.precision or ("mixed" if batched else "fp64")
    other = "fp64" if precision == "mixed" else "mixed"
    gf.SetPrecision(1 if precision == "mixed" else 0)
    gf.TransferStaticDataToDevice()
    gf.SetCZStrengths(sig, sig)
    un, vn, an = state
    gf.TransferNodesToGPU(un, vn, an)
    nc = len(coll.czs)
    gf.TransferPCSR(np.zeros((nc, 3)), np.zeros((nc, 3)), np.zeros(nc, np.int32))
    if pairs is None:  # the device broad phase at the state's positions
        gf.BroadPhase()
        imps = gf.NarrowPhaseCollisionDetection(None)
        pairs = gf.GetPairs()
    else:
        imps = gf.NarrowPhaseCollisionDetection(pairs)
    N, nnz = gf.CreateStructure(copy_back=False)
    if args.layout != "auto":
        _lib.check(gf.ctx, gf.lib.icf_set_variant(gf.ctx, 3, 0 if args.layout == "records" else 1))
    tune = [] if args.no_tune else gf.Autotune(H, reps=10)
    lib = gf.lib
    bufs = gf.DeviceBuffers()
    stream = torch.cuda.ExternalStream(bufs.stream, device=dev)
    flush = torch.empty(FLUSH_BYTES // 4, dtype=torch.int32, device=dev)

    def barrier():
        if ws > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(dev)

    with ClockSampler(dev) as clk:
        ms_dev, cnt = _device_ms(gf, lib, stream, flush, args.steps, args.warmup, barrier, H)

        # end to end through the C ABI with pinned host buffers: H2D of un, vn,
        # an; the assembly; D2H of vals and rhs, every step
        pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
        hun, hvn, han = pin(un), pin(vn), pin(an)
        hvals = torch.empty(9 * nnz, dtype=torch.float64).pin_memory().numpy()
        hrhs = torch.empty(3 * N, dtype=torch.float64).pin_memory().numpy()
        for _ in range(max(1, args.warmup // 2)):
            gf.TransferNodesToGPU(hun, hvn, han)
            gf.AssembleElemsAndCZs(H)
            gf.TransferLinearSystemToHost(hvals, hrhs)
        barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            gf.TransferNodesToGPU(hun, hvn, han)
            gf.AssembleElemsAndCZs(H)
            gf.TransferLinearSystemToHost(hvals, hrhs)
        e1.record(stream)
        barrier()
        ms_e2e = e0.elapsed_time(e1) / args.steps
    clocks = clk.summary()

    # per-kernel device times: the same kernels in the graph's order on one
    # stream with an event after each (no overlap between streams); the last
    # entry is the per-commit CZ history refresh
    kernels = gf.ProfileAssembly(H, reps=max(args.steps, 10))
    hist = [k for k in kernels if k["name"] == "k_cz_hist"]
    kernels = [k for k in kernels if k["name"] != "k_cz_hist"]

    # the same workload in the other precision, measured the same way
    other_line = None
    if not args.no_other:
        gf.SetPrecision(1 if other == "mixed" else 0)
        tune_o = [] if args.no_tune else gf.Autotune(H, reps=10)
        with ClockSampler(dev) as clk_o:
            ms_o, _ = _device_ms(gf, lib, stream, flush, args.steps, args.warmup, barrier, H)
        k_o = [k for k in gf.ProfileAssembly(H, reps=max(args.steps, 10)) if k["name"] != "k_cz_hist"]
        gf.SetPrecision(1 if precision == "mixed" else 0)
        other_line = {"precision": other, "ms_per_step": ms_o, "clocks": clk_o.summary(),
                      "launch_variants": {t["kernel"]: t["variant"] for t in tune_o if t["chosen"]} or "defaults",
                      "kernels": [{"name": k["name"], "ms": round(k["ms"], 5)} for k in k_o]}

    # a whole Newton iteration without the solve: contact detection (one
    # device call, no pair list, as ImplicitModel3 runs it), structure
    # request, assembly; host wall clock.  The broad phase + narrow phase
    # pipeline through the pair list is timed beside it.
    full_iter = None
    if not batched:
        reps = 5

        def pipeline():
            gf.BroadPhase()
            gf.NarrowPhaseCollisionDetection(None)

        for _ in range(2):
            pipeline()
            gf.DetectContacts(copy_back=False)
            gf.CreateStructure(copy_back=False)
            gf.AssembleElemsAndCZs(H)
        torch.cuda.synchronize(dev)
        t_s = [0.0, 0.0, 0.0]
        for _ in range(reps):
            t0 = time.perf_counter()
            pipeline()
            torch.cuda.synchronize(dev)
            t1 = time.perf_counter()
            gf.DetectContacts(copy_back=False)
            gf.CreateStructure(copy_back=False)
            torch.cuda.synchronize(dev)
            t2 = time.perf_counter()
            gf.AssembleElemsAndCZs(H)
            torch.cuda.synchronize(dev)
            t3 = time.perf_counter()
            t_s[0] += t1 - t0
            t_s[1] += t2 - t1
            t_s[2] += t3 - t2
        full_iter = {"value": reps / (t_s[1] + t_s[2]), "unit": "iterations/s",
                     "detection_and_structure_ms": 1000 * t_s[1] / reps, "assembly_ms": 1000 * t_s[2] / reps,
                     "pair_pipeline_ms": 1000 * t_s[0] / reps,
                     "pairs": gf.nPairs, "impacts": gf.nImpacts,
                     "scope": "contact detection without a pair list (the impact list stays on the device) + "
                              "structure request (kept when the impact list is unchanged, as here) + synchronous "
                              "assembly, host wall clock; no linear solve.  pair_pipeline_ms: device broad phase + "
                              "narrow phase on its pair list, the same impacts"}

    from icflow_b200.shard import reduce_max, reduce_sum

    ms_list = [ms_dev, ms_e2e] + ([other_line["ms_per_step"]] if other_line else [])
    ms_list = reduce_max(ms_list, device=dev)
    ms_dev, ms_e2e = ms_list[0], ms_list[1]
    if other_line:
        other_line["ms_per_step"] = ms_list[2]
    total_units = reduce_sum([units], device=dev)[0]

    n_nodes, n_tet = len(coll.x0), len(coll.elems)
    B = algorithmic_bytes(nnz, N, n_nodes, n_tet, nc, len(imps))
    peak, peak_kind = measured_peak()
    achieved = B / (ms_dev * 1e-3) / 1e9
    traffic = ncu_traffic(args.workload, precision)
    top = max(kernels, key=lambda k: k["ms"])
    k_sum = sum(k["ms"] for k in kernels)
    for k in kernels:
        k["alg"] = kernel_share_bytes(k["name"], nnz, N, n_nodes, n_tet, nc, len(imps))
        k["share"] = k["ms"] / k_sum
    line = None
    if rank == 0:
        top_ach = top["alg"] / (top["ms"] * 1e-3) / 1e9
        traffic_asm = sum(v for v in traffic.values()) if traffic else None
        line = {
            "metric": METRIC, "value": total_units * 1000.0 / ms_dev, "unit": "assemblies/s", "n_gpus": ws,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_dev,
            "higher_is_better": True, "scaling": "strong" if batched else "weak", "vs_baseline": None,
            "dtype": "f64" if precision == "fp64" else "f32 Hessians, f64 rotation/law/rhs/accumulation",
            "data": "synthetic (seeded polycrystal; no public dataset exists for this path)",
            "config": {"workload": workload_name(args.workload, *(WORKLOADS[args.workload] or ())),
                       "specimens_per_assembly": N_SPECIMENS if batched else 1,
                       "specimens_rank0": int(len(coll.meshes)) if batched else 1,
                       "tets": int(n_tet), "czs": int(nc), "nodes": int(n_nodes),
                       "active_rows": int(N), "blocks": int(nnz), "impacts": int(len(imps)),
                       "pairs": int(len(pairs)),
                       "l2": "flushed between steps (256 MiB write), outside the timed region",
                       "launch_variants": {t["kernel"]: t["variant"] for t in tune if t["chosen"]} or "defaults"},
            # whole assembly against the HBM roofline: the compulsory bytes of
            # one assembly (72 nnzb + 24 N_a + 96 N + 56 n_t + 240 n_c + 56 n_i)
            # over the device time of one graph launch
            "roofline": {"bound": "hbm", "kernel": "one assembly (graph launch)", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": traffic_asm,
                         "algorithmic_bytes": B,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                         else "fallback",
                         "traffic_source": "profiles/dram_traffic.json: sum over one assembly's kernels of ncu "
                                           "dram__bytes_read.sum + dram__bytes_write.sum" if traffic else None,
                         "dominant_kernel": {
                             "name": top["name"], "launch_ms": top["ms"], "algorithmic_bytes": top["alg"],
                             "achieved": top_ach, "frac": top_ach / peak, "touched_bytes": top["bytes"],
                             "traffic": traffic.get(top["name"]),
                             "scope": "its share of the assembly's compulsory bytes over its serialised launch "
                                      "time; touched_bytes counts the staging records it reads back as well"},
                         "kernels": [{"name": k["name"], "ms": round(k["ms"], 5), "share": round(k["share"], 4),
                                      "algorithmic_bytes": k["alg"], "touched_bytes": k["bytes"],
                                      "frac": round(k["alg"] / (k["ms"] * 1e-3) / 1e9 / peak, 4),
                                      "traffic": traffic.get(k["name"])} for k in kernels]},
            "e2e": {"value": total_units * 1000.0 / ms_e2e, "unit": "assemblies/s",
                    "h2d_bytes_per_step": int(un.nbytes + vn.nbytes + an.nbytes),
                    "d2h_bytes_per_step": int(8 * (9 * nnz + 3 * N))},
            "gpu_launches": len(kernels) * args.steps,
            "autotune": [{k: (round(v, 5) if isinstance(v, float) else v) for k, v in t.items()} for t in tune],
            "full_iteration": full_iter,
            "clocks": clocks,
        }
        if cnt.nLawExact:
            line["law_exact_repeats"] = int(cnt.nLawExact)
        if hist:
            # once per committed step; the reference's minimum of three Newton
            # iterations per step (ModelPrms.cs:206) bounds its share per assembly
            line["cz_history_refresh"] = {"ms_per_commit": hist[0]["ms"],
                                          "ms_per_assembly_at_3_iterations": hist[0]["ms"] / 3,
                                          "scope": "k_cz_hist runs when the committed damage state changes "
                                                   "(once per accepted step), outside the assembly's graph"}
        if other_line:
            other_line["value"] = total_units * 1000.0 / other_line["ms_per_step"]
            other_line["speedup_vs_line"] = ms_dev / other_line["ms_per_step"]
            line[other] = other_line
        if not args.no_cpu:
            rate, threads, kind, sample = cpu_baseline(coll, state, sig, pairs, bound_s=args.cpu_seconds)
            rate1, _, _, sample1 = cpu_baseline(coll, state, sig, pairs, bound_s=args.cpu_seconds, nthreads=1)
            line["cpu_baseline"] = {"value": rate, "unit": "assemblies/s", "cores": threads, "kind": kind,
                                    "sample": sample, "cpu_model": cpu_model(),
                                    "single_core": {"value": rate1, "sample": sample1}}
    gf.close()
    if ws > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


def run_learned(args):
    """The second metric, Newton iterations per attempt with the learned warm
    start against the plain guess: the same 200 us of the ice-block impact
    (two blocks of 1,536 tets, 8 grains each, 5 m/s, dt 5 us, the reference's
    step control, Newton to 1e-8 of the zero-increment residual) under v h,
    the extrapolation, and the extrapolation plus the network trained on the
    device on four other impacts.  One JSON line on rank 0."""
    ws, rank, local = dist_env()
    if rank != 0:
        return
    import torch

    from icflow_b200.warm_start import three_arms

    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    r = three_arms()
    wall = time.perf_counter() - t0
    plain, ext, net = r["plain"], r["extrapolation"], r["network"]
    line = {"metric": "iters/step learned vs plain", "value": net[0] / net[1], "unit": "Newton iterations per attempt",
            "higher_is_better": False, "n_gpus": 1, "data": "synthetic (seeded)",
            "config": {"workload": "ice-block impact, 2 x 1,536 tets, 8 grains each, 5 m/s relative, dt 5 us, "
                                   "200 us simulated, residual tolerance 1e-8, reference step control"},
            "arms": {k: {"iterations": v[0], "attempts": v[1], "accepted": v[2], "per_attempt": v[0] / v[1]}
                     for k, v in (("plain", plain), ("extrapolation", ext), ("network", net))},
            "fewer_than_plain": 1 - net[0] / plain[0], "extrapolation_fewer_than_plain": 1 - ext[0] / plain[0],
            "network_fewer_than_extrapolation": 1 - net[0] / ext[0],
            "network_used": r["network_used"], "attempts_judged": r["attempts_judged"],
            "training_loss": r["training_loss"], "wall_s": wall}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--workload", default="cfg2", choices=sorted(WORKLOADS))
    ap.add_argument("--no-other", action="store_true",
                    help="skip the measurement of the same workload in the other precision")
    ap.add_argument("--no-tune", action="store_true", help="keep the default launch variants")
    ap.add_argument("--layout", default="auto", choices=["auto", "records", "contrib"],
                    help="staging layout of the tet contributions (auto: the autotuner's choice)")
    ap.add_argument("--precision", default=None, choices=["fp64", "mixed"],
                    help="fp64, or FP32 Hessian arithmetic with FP64 rotation, law, rhs and accumulation "
                         "(default: fp64 for cfg1/cfg2, mixed for cfg3); the line also carries the other")
    ap.add_argument("--learned", action="store_true",
                    help="measure the second metric instead: Newton iterations per attempt, learned warm start "
                         "against the plain guess, on the ice-block impact")
    args = ap.parse_args()
    if args.learned:
        run_learned(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
