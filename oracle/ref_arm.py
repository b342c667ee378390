"""Reference arm of bench.py.

TEST / BASELINE INFRASTRUCTURE ONLY (called by ``bench.py --impl
reference``).

Where the reference program has been built from its own sources
(oracle/_ref/ref_program, oracle/ref_build/build_ref_program.py) the arm runs
it: its own run_simulation, cuFFT on the GPU for the nonlinear phase and
OpenMP on every host core for the right-hand sides and the explicit-inverse
solves, and reads its own per-step timer (source/main_loop.cpp:81-102) for
every timed step.  The reference caps Ny at MAX_NZ = 100 (include/data.h:30),
so it runs the bench workload's horizontal grid, flow and parameters at the
largest wall-normal resolution it supports, 256 x 97 x 256 modes (mx, my, mz =
384, 384, 384), a smaller problem than the 256 x 129 x 256 of the bench.

Otherwise it times the oracle's FP64 NumPy port of the reference's step on
one host core, on a bounded sample per step:

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


REF_PROGRAM = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_ref", "ref_program")


def run_program(args, CFG, METRIC, max_timed=20):
    """The reference program at 256 x 97 x 256 (mz = 384): W warm-up steps and
    min(K, max_timed) timed steps of its own loop, its own event timer."""
    import platform
    import subprocess
    import tempfile
    mx, my, mz = CFG["mx"], CFG["my"], min(CFG["mz"], 384)
    K = max(1, min(args.steps, max_timed))
    W = args.warmup
    base = "/dev/shm" if os.path.isdir("/dev/shm") else None
    cores = os.cpu_count() or 1
    with tempfile.TemporaryDirectory(dir=base) as d:
        os.makedirs(os.path.join(d, "input"))
        os.makedirs(os.path.join(d, "run", "out"))
        with open(os.path.join(d, "input", "parameter.txt"), "w") as f:
            f.write(f"{mx} {my} {mz}\n4.0 2.0\n{CFG['Re']} {CFG['Ro']} {CFG['dt']}\n"
                    f"0 1 {W + K} 1000000000 1000000000\nout/o\nout/r\n")
        env = dict(os.environ, OMP_NUM_THREADS=str(cores))
        t0 = time.perf_counter()
        r = subprocess.run([REF_PROGRAM], cwd=os.path.join(d, "run"), env=env, capture_output=True, text=True,
                           timeout=3000)
        wall = time.perf_counter() - t0
    steps = [float(x.split(":")[1]) for x in r.stdout.splitlines() if x.startswith("Time cost of current step:")]
    # the reference never joins its worker thread: std::terminate at exit
    # (status -6) after the last step is expected
    if len(steps) != W + K or r.returncode not in (0, -6):
        raise RuntimeError(f"reference program: status {r.returncode}, {len(steps)} of {W + K} steps; "
                           f"{r.stderr[-500:]}")
    timed = steps[W:]
    step_s = float(np.mean(timed))
    value = 1.0 / step_s
    cpu = platform.processor() or ""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                cpu = line.split(":", 1)[1].strip()
                break
    except OSError:
        pass
    sample = (f"the reference program (its own sources, cuFFT nonlinear phase on the GPU, OpenMP right-hand "
              f"sides and explicit-inverse solves on {cores} host threads, {cpu}) at 256x97x256 modes "
              f"(mx,my,mz={mx},{my},{mz}; Ny capped at MAX_NZ = 100), rotating Couette Re {CFG['Re']:g}, Ro "
              f"{CFG['Ro']:g}, dt {CFG['dt']:g}: {K} timed steps after {W} warm-up, its own per-step timer; "
              f"whole run incl. set-up {wall:.0f} s")
    return {
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "steps/s",
        "n_gpus": 1, "steps": K, "warmup": W,
        "ms_per_step": round(step_s * 1e3, 2), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "the reference's analytic initial field (initFlow)",
        "config": {"workload": (f"rotating plane Couette 256x97x256 modes (mx,my,mz={mx},{my},{mz}), "
                                f"Re {CFG['Re']:g}, Ro {CFG['Ro']:g}, dt {CFG['dt']:g}; the reference's "
                                f"MAX_NZ = 100 rules out the bench's 256x129x256")},
        "cpu_baseline": {"value": round(value, 4), "unit": "steps/s", "cores": cores, "kind": "reference",
                         "sample": sample},
        "e2e": {"value": round(value, 4), "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "step_seconds_timed": [round(x, 5) for x in timed],
    }


def run(args, CFG, METRIC):
    if os.path.exists(REF_PROGRAM):
        return run_program(args, CFG, METRIC)
    return run_port(args, CFG, METRIC)


def run_port(args, CFG, METRIC):
    # one host core: NumPy's element-wise work holds the interpreter, so a
    # thread pool over the pencils gains nothing
    threads = 1
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
                   f"{P} of {sz.pz} wall-normal planes per step, scaled; {threads} host thread; "
                   "the reference program is not built on this host")
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
