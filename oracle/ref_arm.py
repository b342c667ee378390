"""Reference arm of bench.py: the reference's step algorithm on host cores.

TEST / BASELINE INFRASTRUCTURE ONLY (called by ``bench.py --impl
reference``).  The reference program itself cannot be built here (its solve
needs Eigen, which is absent), so this times the oracle's FP64 NumPy port of
the reference's step, with all host threads, on a bounded sample per step:

* pencil phase (getUVW + padded s2p of six fields, padded p2s of three Lamb
  components, rhsNonlinear, no-pad s2p, CN right-hand sides, v and omega
  solves with explicit inverses) on S pencils, scaled by H / S;
* plane phase (2D C2R of six fields, Lamb vector with rotation, 2D R2C of
  three) on P wall-normal planes, scaled by Py / P.

Operator inverses of the sampled pencils are built before timing (setup, as
in the reference's initAuxMatrix).
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import time

import numpy as np

from . import rpcf_oracle as O


def _ddz(a):
    return O.ddz(a)


def _pencil_phase(args):
    (V, Om, Nvp, Nop, ia, ib, inv_v, inv_o, sz, p, T0, T2, T4, U, dU, ddU) = args
    nz, mz = sz.nz, sz.mz
    kmn = ia * ia + ib * ib
    with np.errstate(divide="ignore", invalid="ignore"):
        k1 = np.where(kmn > 0, 1.0 / kmn, 0.0)
    # getUVW + padded s2p of six fields (source/velocity.cu:90-170, transform.cu:416-453)
    Dw = _ddz(V)
    u = (1j * ia * k1)[:, None] * Dw - (1j * ib * k1)[:, None] * Om
    v = (1j * ib * k1)[:, None] * Dw + (1j * ia * k1)[:, None] * Om
    ox = _ddz(v) - 1j * ib[:, None] * V
    oy = -_ddz(u) + 1j * ia[:, None] * V
    for f in (u, v, V, ox, oy, Om):
        S = np.zeros((f.shape[0], mz), dtype=np.complex128)
        S[:, :nz] = f
        O.cheby_s2p(S, mz, pad=True)
    # padded p2s of three Lamb components (stand-in values), rhsNonlinear, no-pad s2p
    lam = [np.zeros((V.shape[0], mz), dtype=np.complex128) for _ in range(3)]
    for L in lam:
        L[:, :sz.pz] = 1e-3
    c = [O.cheby_p2s(L, mz, pad=True)[:, :nz] for L in lam]
    hv = kmn[:, None] * c[2] + 1j * ia[:, None] * _ddz(c[0]) + 1j * ib[:, None] * _ddz(c[1])
    ho = 1j * ia[:, None] * c[1] - 1j * ib[:, None] * c[0]
    H = np.zeros((V.shape[0], mz), dtype=np.complex128)
    H[:, :nz] = hv
    Nv = O.cheby_s2p(H, mz, pad=False)[:, :nz]
    H[:, :nz] = ho
    No = O.cheby_s2p(H, mz, pad=False)[:, :nz]
    # CN right-hand sides + AB2 and the two solves (source/linear.cpp, solver.cpp:107-123)
    dt, Re = p.dt, p.Re
    r = np.arange(4, nz)
    P0, P2, P4 = V @ T0[r - 2].T, V @ T2[r - 2].T, V @ T4[r - 2].T
    km = kmn[:, None]
    al = ia[:, None]
    rv = np.zeros_like(V)
    rv[:, 4:] = (P4 * dt * 0.5 / Re + (1 - km * dt / Re) * P2 - km * (1 - km * dt * 0.5 / Re) * P0
                 + 1j * (-al * dt * 0.5 * U[r - 2] * P2
                         + (km * al * dt * 0.5 * U[r - 2] + al * dt * 0.5 * ddU[r - 2]) * P0)
                 + (Nv[:, r - 2] * 1.5 - Nvp[:, r - 2] * 0.5) * dt)
    vn = np.einsum("pij,pj->pi", inv_v, rv)
    i = np.arange(2, nz)
    Q0, Q2, S0 = Om @ T0[i - 1].T, Om @ T2[i - 1].T, (V + vn) @ T0[i - 1].T
    ro = np.zeros_like(Om)
    ro[:, 2:] = (Q2 * 0.5 / Re * dt + (1 - km * dt * 0.5 / Re) * Q0 - 1j * al * dt * 0.5 * U[i - 1] * Q0
                 - 1j * 0.5 * ib[:, None] * dU[i - 1] * dt * S0 + (No[:, i - 1] * 1.5 - Nop[:, i - 1] * 0.5) * dt)
    return np.einsum("pij,pj->pi", inv_o, ro)


def _plane_phase(args):
    C6, sz, Ro, meanU = args
    phys = [np.fft.irfft2(C, s=(sz.my, sz.mx), axes=(-2, -1)) * (sz.my * sz.mx) for C in C6]
    u, v, w, ox, oy, oz = phys
    lx = oz * v - oy * w - Ro * w
    ly = ox * w - oz * u
    lz = oy * u - ox * v + Ro * (u + meanU)
    return [np.fft.rfft2(L, axes=(-2, -1)) / (sz.mx * sz.my) for L in (lx, ly, lz)]


def run(args, CFG, METRIC):
    from importlib import util as _u  # noqa: F401
    threads = os.cpu_count() or 1
    p = O.Params(CFG["mx"], CFG["my"], CFG["mz"], Re=CFG["Re"], Ro=CFG["Ro"], dt=CFG["dt"])
    pb = O.Problem(p)
    sz = pb.sz
    rng = np.random.default_rng(0)
    S = 512
    P = 8
    sel = rng.choice(sz.ny * sz.hnx, size=S, replace=False)
    ky, kx = np.unravel_index(sel, (sz.ny, sz.hnx))
    N = sz.nz - 1
    inv_v = np.empty((S, sz.nz, sz.nz), dtype=np.complex128)
    inv_o = np.empty_like(inv_v)
    for n, (a, b) in enumerate(zip(ky, kx)):
        inv_v[n] = np.linalg.inv(O.coef_v(N, pb.U, pb.ddU, pb.T0, pb.T2, pb.T4, p.Re, p.dt, pb.kmn[a, b], pb.ia[a, b]))
        inv_o[n] = np.linalg.inv(O.coef_omega(N, pb.U, pb.T0, pb.T2, p.Re, p.dt, pb.kmn[a, b], pb.ia[a, b]))
    V = rng.standard_normal((S, sz.nz)) + 1j * rng.standard_normal((S, sz.nz))
    Om = rng.standard_normal((S, sz.nz)) + 1j * rng.standard_normal((S, sz.nz))
    Nvp = np.zeros_like(V)
    Nop = np.zeros_like(V)
    ia, ib = pb.ia[ky, kx], pb.ib[ky, kx]
    C6 = [rng.standard_normal((P, sz.my, sz.mx // 2 + 1)) + 1j * rng.standard_normal((P, sz.my, sz.mx // 2 + 1))
          for _ in range(6)]
    meanU = O.base_profile(np.cos(np.arange(P) / (sz.pz - 1) * O.PI), p.prof)[0][:, None, None]
    chunks = np.array_split(np.arange(S), threads)
    pchunks = np.array_split(np.arange(P), min(threads, P))
    ex = cf.ThreadPoolExecutor(max_workers=threads)

    def sample():
        t0 = time.perf_counter()
        list(ex.map(_pencil_phase, [(V[c], Om[c], Nvp[c], Nop[c], ia[c], ib[c], inv_v[c], inv_o[c], sz, p,
                                     pb.T0, pb.T2, pb.T4, pb.U, pb.dU, pb.ddU) for c in chunks if len(c)]))
        t1 = time.perf_counter()
        list(ex.map(_plane_phase, [([C[c] for C in C6], sz, p.Ro, meanU[c]) for c in pchunks if len(c)]))
        t2 = time.perf_counter()
        return (t1 - t0) * (sz.ny * sz.hnx) / S + (t2 - t1) * sz.pz / P

    for _ in range(args.warmup):
        sample()
    ts = [sample() for _ in range(args.steps)]
    ex.shutdown()
    step_s = float(np.mean(ts))
    value = 1.0 / step_s
    sample_desc = (f"oracle FP64 NumPy port of the reference step at {CFG['mx']}x{CFG['my']}x{CFG['mz']} "
                   f"(mx,my,mz): pencil phase on {S} of {sz.ny * sz.hnx} pencils and plane phase on "
                   f"{P} of {sz.pz} wall-normal planes per step, scaled; {threads} host threads; "
                   "the reference program itself needs Eigen (absent) and is not built")
    return {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "steps/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(step_s * 1e3, 2), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"rotating plane Couette {args.config} modes, Re {CFG['Re']:g}, "
                               f"Ro {CFG['Ro']:g}, dt {CFG['dt']:g}"},
        "cpu_baseline": {"value": round(value, 4), "unit": "steps/s", "cores": threads, "kind": "port",
                         "sample": sample_desc},
        "e2e": {"value": round(value, 4), "unit": "steps/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
