"""Generates the golden fixtures in this directory from the REFERENCE's own
kernel code built for the host (oracle/_ref, compiled from the reference
sources by oracle/Makefile), on seeded synthetic inputs.

    python tests/golden/make_golden.py

The fixtures pin the CPU oracle (tests/test_oracle_golden.py) on machines where
the reference sources are not available.  Inputs are seeded; every output here
is what the reference code computes for them.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

from oracle.oracle import Oracle, RefKernels  # noqa: E402

from icflow_b200 import mesh as M  # noqa: E402

OUT = Path(__file__).resolve().parent
# parameters of the benchmark configurations (E 9 GPa, nu 0.3, rho 916,
# PPR phi 3 J/m^2, sigma = tau = 1 MPa, alpha = beta = 4, lambda 0.02)
PRMS = dict(Y=9e9, nu=0.3, rho=916.0, phi_n=3.0, phi_t=3.0, sigma_max=1e6, tau_max=1e6,
            alpha=4.0, beta=4.0, lambda_n=0.02, lambda_t=0.02, penaltyK=1e8)


def random_tets(rng, n):
    x0 = rng.random((n, 4, 3)) * 0.1
    V = M._jdet(x0)
    x0[V < 0] = x0[V < 0][:, [0, 1, 3, 2]]
    # a few slivers
    x0[: n // 10, 3] = x0[: n // 10, 0] + 0.02 * (x0[: n // 10, 3] - x0[: n // 10, 0])
    V = M._jdet(x0)
    x0[V < 0] = x0[V < 0][:, [0, 1, 3, 2]]
    return x0.reshape(n, 12)


def rotation(rng):
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def main():
    O = Oracle()
    R = RefKernels(nthreads=1)
    p = O.prms(**PRMS)
    R.set_constants(p)
    rng = np.random.default_rng(20240)
    q = p.ppr

    # elements: random, slivers, rotated + stretched states
    n = 64
    x0 = random_tets(rng, n)
    un = (rng.random((n, 12)) - 0.5) * 0.004
    for i in range(n // 4, n // 2):  # large rigid rotations plus small strain
        Rm = rotation(rng)
        c = x0[i].reshape(4, 3)
        un[i] = ((c @ Rm.T) - c).ravel() + (rng.random(12) - 0.5) * 1e-4
    f, Df, V = R.F_and_Df(x0, un)
    np.savez_compressed(OUT / "elem_f_df.npz", x0=x0, un=un, f=f, Df=Df, V=V)

    # PPR functions and the cohesive law over all branches
    m = 400
    dn = rng.random(m) * q.deln * 0.999
    dt = rng.random(m) * q.delt * 0.999
    ppr = R.ppr(dn, dt)
    pm = rng.random(m) * q.deln * 0.8 * (rng.random(m) > 0.3)
    tm = rng.random(m) * q.delt * 0.8 * (rng.random(m) > 0.3)
    opn = (rng.random(m) * 2.1 - 1.0) * q.deln
    opt = rng.random(m) * 1.05 * q.delt
    pm2, tm2, law, flags = R.cz_law(pm, tm, opn, opt)
    early = (opn > q.deln) | (opt > q.delt)
    law[early, 5] = np.nan  # Dtn is left unset by the reference on this path
    np.savez_compressed(OUT / "cz_law.npz", dn=dn, dt=dt, ppr=ppr, pmax=pm, tmax=tm, opn=opn, opt=opt,
                        pmax_out=pm2, tmax_out=tm2, law=law, flags=flags)

    # point-triangle distance with derivatives: all regions
    k = 600
    xs = rng.random((k, 12))
    xs[:50, 0:3] = 0.25 * (xs[:50, 3:6] + xs[:50, 6:9] + xs[:50, 9:12]) + 0.05 * (rng.random((50, 3)) - 0.5)
    res = [R.pt(x) for x in xs]
    np.savez_compressed(OUT / "pt.npz", x=xs, dsq=np.array([r[0] for r in res]),
                        fd=np.array([r[1] for r in res]), sd=np.array([r[2] for r in res]),
                        s=np.array([r[3] for r in res]), t=np.array([r[4] for r in res]),
                        branch=np.array([r[5] for r in res], np.int32))
    ft = rng.random((300, 12))
    np.savez_compressed(OUT / "dtn.npz", x=ft, d=np.array([R.dtn(v[:9], v[9:]) for v in ft]))

    # assembled system of the cantilever (2304 tets, 32 CZs) from a seeded state
    c = M.cantilever()
    nn = len(c.x0)
    r2 = np.random.default_rng(7)
    un = (r2.random((nn, 3)) - 0.5) * 4e-6
    un[c.anchored] = 0
    vn = r2.random((nn, 3)) - 0.5
    an = r2.random((nn, 3)) - 0.5
    nc = len(c.czs)
    pmax = r2.random((nc, 3)) * q.deln * 0.2
    tmax = r2.random((nc, 3)) * q.delt * 0.2
    N, rows, cols = O.build_structure(c.alt, c.elems, c.czs, np.zeros((0, 4), np.int32))
    ep = O.pcsr(c.elems, 4, c.alt, rows, cols, N)
    cp = O.pcsr(c.czs, 6, c.alt, rows, cols, N)
    st = R.pack_nodes(c.x0, un, vn, an)
    vals = np.zeros(9 * len(cols))
    rhs = np.zeros(3 * N)
    h = 1e-4
    R.elem_kernel(st, h, c.elems, ep, vals, rhs)
    tp, tt, fl, avg = R.cz_kernel(st, h, c.czs, cp, pmax, tmax, vals, rhs)
    F = R.node_field(st, 12, nn)
    np.savez_compressed(OUT / "cantilever_assembly.npz", un=un, vn=vn, an=an, pmax=pmax, tmax=tmax, h=h,
                        N=N, rows=rows, cols=cols, vals=vals, rhs=rhs, tent_pmax=tp, tent_tmax=tt, flags=fl,
                        avg=avg, nodeF=F)

    # contact: a small polycrystal pressed by platens; narrow phase, closest
    # face and the penalty response, all from the reference kernels
    c = M.polycrystal(n=5, grains=4, seed=2, platens=True, gap=-0.3)
    nn = len(c.x0)
    r3 = np.random.default_rng(9)
    un = (r3.random((nn, 3)) - 0.5) * 2e-7
    un[c.anchored] = 0
    xt = c.x0 + un
    pairs = M.candidate_pairs(c, xt, same_mesh=False, vertex_in_box=False)
    st = R.pack_nodes(c.x0, un, np.zeros((nn, 3)), np.zeros((nn, 3)))
    masks, ie, el_stride = R.narrow_phase_kernel(st, nn, pairs, c.selem, c.adj_off, c.adj)
    keys = set()
    for i, mk in enumerate(masks):
        ea, eb = pairs[i]
        for b in range(4):
            if mk & (1 << b):
                keys.add((int(c.selem[eb][b]), int(ea)))
            if mk & (16 << b):
                keys.add((int(c.selem[ea][b]), int(eb)))
    node_elem = np.array(sorted(keys), np.int32).reshape(-1, 2)
    imps = R.closest_face_kernel(st, node_elem, ie, el_stride, c.faces)
    N, rows, cols = O.build_structure(c.alt, c.elems, c.czs, imps)
    ipc = O.pcsr(imps, 4, c.alt, rows, cols, N)
    vals = np.zeros(9 * len(cols))
    rhs = np.zeros(3 * N)
    R.collision_kernel(st, 1e-5, imps, ipc, vals, rhs, p.penaltyK, p.DistanceEpsilon)
    np.savez_compressed(OUT / "contact.npz", un=un, pairs=pairs, masks=masks, node_elem=node_elem,
                        impacts=imps, N=N, rows=rows, cols=cols, vals=vals, rhs=rhs)
    for f_ in sorted(OUT.glob("*.npz")):
        print(f_.name, f_.stat().st_size)


if __name__ == "__main__":
    main()
