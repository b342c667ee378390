#!/usr/bin/env python
"""DNS steps/s at 256x129x256 (Nx x Ny x Nz modes; reference parameters
mx, my, mz = 384, 384, 512; physical grid 384 x 257 x 384), rotating plane
Couette, Re = 3000, rotation number 0.02, dt = 0.001, seeded divergence-free
initial field (seed 0, amplitude 0.1).

The headline `value` is the mixed form (FP32 transforms and Lamb vector,
FP64 operators, solves and AB2/CN state) in steps/s with the state resident
in HBM; the plain FP64 form is timed in the same run and the mixed form's
relative L2 error against it is reported (must be <= 1e-6).  `e2e` is the
mixed step through the public C ABI with the state copied in from pinned host
memory and back out every step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With --gpus N > 1 (launched by torchrun) every rank runs an independent
replica of the problem; the time is the maximum over ranks and `value` sums
the replicas' steps/s.  --decomposed runs one problem split over the ranks
instead (the slab decomposition, NCCL all-to-all exchanges, strong scaling),
or over --slab-ranks R ranks on one device.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "gpu-spectral-channel-dns_b200")

METRIC = "DNS steps/s at 256x129x256: mixed vs FP64 form at 1e-6 rel err; % HBM roofline"
CONFIGS = {
    # the headline workload (mixed vs FP64)
    "256x129x256": dict(Nx=256, Ny=129, Nz=256, mx=384, my=384, mz=512, Re=3000.0, Ro=0.02,
                        dt=0.001, amplitude=0.1, seed=0),
    # smaller grids of the same family, for profiling captures and parity runs
    "128x65x128": dict(Nx=128, Ny=65, Nz=128, mx=192, my=192, mz=256, Re=3000.0, Ro=0.02,
                       dt=0.001, amplitude=0.1, seed=0),
    "32x33x32": dict(Nx=32, Ny=33, Nz=32, mx=48, my=48, mz=128, Re=1300.0, Ro=0.1, dt=0.005,
                     amplitude=0.05, seed=0),
}
CFG = CONFIGS["256x129x256"]
KERNELS = ["y3_uvw_s2p", "zb_span_inverse", "x_c2r_lamb_r2c", "zf_span_forward", "y1_p2s_rhs",
           "y2_solve"]


def load_pkg():
    if "dns_b200" in sys.modules:
        return sys.modules["dns_b200"]
    spec = importlib.util.spec_from_file_location(
        "dns_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["dns_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


# ---------------------------------------------------------------------------
# algorithmic bytes per kernel launch (one step), element size c (16 FP64 /
# 8 FP32 complex); s = 16 (FP64 state / operator complex)
# ---------------------------------------------------------------------------
WALL_BANDS = {0: (4, 8, 2, 4), 1: (5, 9, 3, 6), 2: (6, 10, 4, 8)}  # v kl, ku; omega kl, ku


def wall_dims(g, U):
    """Rows per pencil of the banded systems and bytes of the packed factors
    (groups of 16 operator slots; v rows: kl + 1 + ku + 2 entries, omega
    rows: kl + 1 + ku entries, complex FP64)."""
    delta = 2 if U[2] else (1 if U[1] else 0)
    klv, kuv, klo, kuo = WALL_BANDS[delta]
    n = g["Ny"] + delta
    slots = g["Kx"] * (g["Nz"] // 2 + 1)
    groups = (slots + 15) // 16
    per_group = 16 * (n * (klv + 1 + kuv + 2) + n * (klo + 1 + kuo))
    return n, groups * per_group * 16


def kernel_bytes(g, c, U=(0.5, 0.5, 0.0)):
    """Algorithmic bytes per launch, by the pencil-pass model: each pass reads
    its input fields once and writes its output fields once (padded
    transforms at c bytes per complex value); the FP64 state and the AB2
    history (16 B complex) are read and written once per step.  The banded
    factors the wall solve streams are implementation cost, reported apart
    (factor_bytes)."""
    Kx, Nz, Ny, Py, Pz = g["Kx"], g["Nz"], g["Ny"], g["Py"], g["Pz"]
    H = Kx * Nz
    s = 16
    return {
        "y3_uvw_s2p": s * 2 * H * Ny + c * 6 * H * Py,                  # v, omega in; 6 fields out
        "zb_span_inverse": c * 6 * H * Py + c * 6 * Kx * Pz * Py,       # pad Nz -> Pz
        "x_c2r_lamb_r2c": c * 6 * Kx * Pz * Py + c * 3 * Kx * Pz * Py,  # read 6, write 3
        "zf_span_forward": c * 3 * Kx * Pz * Py + c * 3 * H * Py,       # truncate Pz -> Nz
        # lambda in; v, omega, history in; history out
        "y1_p2s_rhs": c * 3 * H * Py + s * 6 * H * Ny,
        # v, omega out
        "y2_solve": s * 2 * H * Ny,
    }


def factor_bytes(g, U=(0.5, 0.5, 0.0)):
    return wall_dims(g, U)[1]


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    def __init__(self, index):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-lms", "50"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
            # nvidia-smi takes a while to start: wait for its first sample,
            # then keep only the samples taken from here on (the timed region)
            t0 = time.perf_counter()
            while not self.rows and time.perf_counter() - t0 < 10.0 and self.proc.poll() is None:
                time.sleep(0.01)
            self.rows = []
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 8:
                self.rows.append(parts)

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = sorted(float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit())
        mx = max((float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()), default=None)
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for n, v in zip(names, r[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def cpu_baseline():
    """Time the oracle (FP64 NumPy port of the reference step) on the host:
    the full nonlinear phase at 256x129x256 plus the CN/AB2 right-hand sides
    and the two solves on a sample of pencils, scaled to all pencils."""
    os.environ.setdefault("OPENBLAS_NUM_THREADS", "1")
    import numpy as np
    sys.path.insert(0, ROOT)
    from oracle import rpcf_oracle as O
    pkg = load_pkg()
    p = O.Params(CFG["mx"], CFG["my"], CFG["mz"], Re=CFG["Re"], Ro=CFG["Ro"], dt=CFG["dt"])
    pb = O.Problem(p)
    sz = pb.sz
    V, Om = pkg.seeded_state(sz.nx, sz.nz, sz.ny, p.n_pi_x, p.n_pi_y, CFG["amplitude"], CFG["seed"])
    pb.set_state(V, Om)
    t0 = time.perf_counter()
    Nv, No = pb.nonlinear()
    t_nl = time.perf_counter() - t0
    # linear RHS + solves on S pencils (their inverses built outside the timing)
    S = 256
    rng = np.random.default_rng(0)
    sel = rng.choice(sz.ny * sz.hnx, size=S, replace=False)
    ky, kx = np.unravel_index(sel, (sz.ny, sz.hnx))
    N = sz.nz - 1
    invs = []
    for a, b in zip(ky, kx):
        Av = O.coef_v(N, pb.U, pb.ddU, pb.T0, pb.T2, pb.T4, p.Re, p.dt, pb.kmn[a, b], pb.ia[a, b])
        Ao = O.coef_omega(N, pb.U, pb.T0, pb.T2, p.Re, p.dt, pb.kmn[a, b], pb.ia[a, b])
        invs.append((np.linalg.inv(Av), np.linalg.inv(Ao)))
    t0 = time.perf_counter()
    sub = O.Problem(p)
    sub.kmn = pb.kmn[ky, kx][None, :]
    sub.ia = pb.ia[ky, kx][None, :]
    sub.ib = pb.ib[ky, kx][None, :]
    Vs = V[ky, kx][None]
    Os = Om[ky, kx][None]
    rv = sub.linear_v(Vs)
    k = np.arange(4, sz.nz)
    rv[..., 4:] += (Nv[ky, kx][None][..., k - 2] * 1.5 - Nv[ky, kx][None][..., k - 2] * 0.5) * p.dt
    vn = np.stack([iv @ r for (iv, _), r in zip(invs, rv[0])])[None]
    ro = sub.linear_omega(Os, vn, Vs)
    on = np.stack([io @ r for (_, io), r in zip(invs, ro[0])])
    t_lin = (time.perf_counter() - t0) * (sz.ny * sz.hnx) / S
    step_s = t_nl + t_lin
    return {"value": 1.0 / step_s, "unit": "steps/s", "cores": 1, "kind": "port",
            "sample": (f"oracle FP64 NumPy step at 256x129x256: full nonlinear phase ({t_nl:.1f} s) "
                       f"+ CN/AB2 rhs and solves on {S} of {sz.ny * sz.hnx} pencils scaled "
                       f"({t_lin:.2f} s); operator inverses excluded as setup"),
            "step_seconds": step_s}


def dist_max(x):
    """Maximum over the ranks of a time-like float, on the process group's
    device (CUDA for NCCL, host for gloo)."""
    import torch
    dev = "cuda" if torch.distributed.get_backend() == "nccl" else "cpu"
    t = torch.tensor([float(x)], device=dev, dtype=torch.float64)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replica_value(n_ranks, ms_per_step_max):
    """Whole-job steps/s of n independent replicas timed as the slowest rank."""
    return n_ranks * 1000.0 / ms_per_step_max


def run_ours(args, rank, world):
    import numpy as np
    import torch
    pkg = load_pkg()
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    V0, O0 = pkg.seeded_state(CFG["Nx"], CFG["Ny"], CFG["Nz"], 4.0, 2.0, CFG["amplitude"], CFG["seed"])

    def make(prec):
        ctx = pkg.Context(pkg.make_params(CFG["mx"], CFG["my"], CFG["mz"], Re=CFG["Re"], Ro=CFG["Ro"],
                                          dt=CFG["dt"], precision=prec, device=dev))
        ctx.set_state(V0, O0)
        ctx.bootstrap()
        return ctx

    def timed(ctx, K, W):
        ctx.step(W)
        ctx.synchronize()
        s = torch.cuda.ExternalStream(ctx.stream)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()
        e0.record(s)
        ctx.step(K)
        e1.record(s)
        ctx.synchronize()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if world > 1:
            ms = dist_max(ms)
        return ms / K

    def rel(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    def components(ctx, V, Om):
        """getUVW of a state through the library (FP64 kernel): the six
        velocity / vorticity coefficient fields, in standard axis names."""
        Nz, Kx, Ny = V.shape
        mz = CFG["mz"]
        f = [torch.zeros((Nz, Kx, mz), dtype=torch.complex128, device="cuda") for _ in range(6)]
        f[2][..., :Ny] = torch.from_numpy(V).cuda()
        f[5][..., :Ny] = torch.from_numpy(Om).cuda()
        torch.cuda.synchronize()
        ctx.get_uvw([t.data_ptr() for t in f], mz * 16)
        ctx.synchronize()
        ref = [t[..., :Ny].cpu().numpy() for t in f]
        # reference axes (u, v span, w wall-normal, omega_x, omega_y span,
        # omega_z wall-normal) -> standard (u, v wall-normal, w span, ...)
        return {"u": ref[0], "v": ref[2], "w": ref[1], "omega_x": ref[3], "omega_y": ref[5],
                "omega_z": ref[4]}

    def comp_errors(ctx, A, B):
        ca, cb = components(ctx, *A), components(ctx, *B)
        return {k: rel(ca[k], cb[k]) for k in ca}

    K, W = args.steps, args.warmup
    t_setup = time.perf_counter()
    c64 = make(pkg.PREC_FP64)
    setup_s = time.perf_counter() - t_setup
    cmx = make(pkg.PREC_MIXED)
    # the autotuner times every compiled variant of each tunable pass on this
    # grid and keeps the fastest (per context, before any timed step)
    tune = {}
    for tag, ctx in (("mixed", cmx), ("fp64", c64)):
        times = ctx.autotune()
        tune[tag] = {pkg.PASS_NAMES[p]: {"ms": {pkg.VARIANT_NAMES[p][v]: round(t, 4) for v, t in vt.items()},
                                         "picked": pkg.VARIANT_NAMES[p][ctx.get_variant(p)]}
                     for p, vt in times.items()}
    # accuracy of the mixed form against the FP64 form: (1) accumulated over
    # ACC steps from the seeded state; (2) per step: both forms advance one
    # step from the FP64 state and history reached after ACC steps
    ACC = 20
    c64.step(ACC)
    cmx.step(ACC)
    V64, O64 = c64.get_state()
    Vmx, Omx = cmx.get_state()
    acc = comp_errors(c64, (Vmx, Omx), (V64, O64))
    Nv64, No64 = c64.get_history()
    cmx.set_state(V64, O64)
    cmx.set_history(Nv64, No64)
    c64.step(1)
    cmx.step(1)
    V64, O64 = c64.get_state()
    Vmx, Omx = cmx.get_state()
    err = comp_errors(c64, (Vmx, Omx), (V64, O64))
    # timing, each form from the seeded state again
    for ctx in (c64, cmx):
        ctx.set_state(V0, O0)
        ctx.bootstrap()
    ms64 = timed(c64, K, W)
    with ClockSampler(dev) as clk:
        msmx = timed(cmx, K, W)
    # per-kernel durations, measured with CUDA events on the launching stream
    kms64 = c64.step_profiled(K)
    kmsmx = cmx.step_profiled(K)
    c64.close()
    # end to end through the C ABI with pinned host buffers
    Vh = torch.empty((cmx.Nz, cmx.Kx, cmx.Ny), dtype=torch.complex128, pin_memory=True)
    Oh = torch.empty_like(Vh, pin_memory=True)
    Vh.copy_(torch.from_numpy(V0))
    Oh.copy_(torch.from_numpy(O0))
    pitch = cmx.Ny * 16
    vp, op = Vh.data_ptr(), Oh.data_ptr()
    lib = cmx.lib
    import ctypes
    for _ in range(2):
        lib.dns_set_state(cmx.h, ctypes.c_void_p(vp), ctypes.c_void_p(op), pitch, pkg.HOST)
        cmx.step(1)
        lib.dns_get_state(cmx.h, ctypes.c_void_p(vp), ctypes.c_void_p(op), pitch, pkg.HOST)
    if world > 1:
        torch.distributed.barrier()
    t0 = time.perf_counter()
    for _ in range(K):
        st = lib.dns_set_state(cmx.h, ctypes.c_void_p(vp), ctypes.c_void_p(op), pitch, pkg.HOST)
        cmx.step(1)
        st |= lib.dns_get_state(cmx.h, ctypes.c_void_p(vp), ctypes.c_void_p(op), pitch, pkg.HOST)
        if st:
            raise RuntimeError(lib.dns_last_error().decode())
    e2e_ms = (time.perf_counter() - t0) * 1e3 / K
    if world > 1:
        e2e_ms = dist_max(e2e_ms)
    geo = dict(Kx=cmx.Kx, Nz=cmx.Nz, Ny=cmx.Ny, Py=cmx.Py, Pz=cmx.Pz)
    mem = cmx.memory_bytes()
    cmx.close()
    return dict(ms64=ms64, msmx=msmx, err=err, acc=acc, acc_steps=ACC, autotune=tune,
                kms64=kms64, kmsmx=kmsmx,
                e2e_ms=e2e_ms, geo=geo, clocks=clk.summary(), setup_s=setup_s, mem=mem,
                state_bytes=2 * geo["Kx"] * geo["Nz"] * geo["Ny"] * 16)


def run_one(args):
    """One context of one precision: bootstrap, W warm-up steps, K steps,
    per-kernel CUDA-event times (profiling runs; no comparison, no e2e)."""
    import torch
    pkg = load_pkg()
    torch.cuda.set_device(0)
    V0, O0 = pkg.seeded_state(CFG["Nx"], CFG["Ny"], CFG["Nz"], 4.0, 2.0, CFG["amplitude"], CFG["seed"])
    prec = pkg.PREC_MIXED if args.only == "mixed" else pkg.PREC_FP64
    ctx = pkg.Context(pkg.make_params(CFG["mx"], CFG["my"], CFG["mz"], Re=CFG["Re"], Ro=CFG["Ro"],
                                      dt=CFG["dt"], precision=prec, device=0))
    ctx.set_state(V0, O0)
    if args.variant:
        # fixed variants, no timing of candidates: under a profiler the
        # autotuner's event times mean nothing
        by_name = {pkg.PASS_NAMES[p]: (p, {n: v for v, n in pkg.VARIANT_NAMES[p].items()})
                   for p in range(pkg.NUM_PASSES)}
        for item in args.variant:
            pname, vname = item.split("=")
            p, names = by_name[pname]
            ctx.set_variant(p, names[vname])
    else:
        ctx.autotune()
    variant = {pkg.PASS_NAMES[p]: pkg.VARIANT_NAMES[p][ctx.get_variant(p)] for p in range(pkg.NUM_PASSES)}
    ctx.bootstrap()
    ctx.step(args.warmup)
    kms = ctx.step_profiled(args.steps)
    ctx.synchronize()
    ctx.close()
    return {"only": args.only, "config": args.config, "variants": variant,
            "kernel_ms": {k: round(v, 4) for k, v in kms.items()}}


ENSEMBLE_SIZES = [(48, 48, 128), (96, 96, 192), (144, 144, 256), (192, 192, 384)]


def ensemble_members(n_per_size=12):
    """The 48-run ensemble: 12 runs each of 32x33x32, 64x49x64, 96x65x96 and
    128x97x128 modes; run m draws Re ~ U[500, 3000] and Ro ~ U[0, 0.3] from
    default_rng(1000 + m) and seeds its field with 1000 + m (amplitude 0.1),
    dt 0.002."""
    import numpy as np
    out = []
    for si, (mx, my, mz) in enumerate(ENSEMBLE_SIZES):
        for j in range(n_per_size):
            m = 12 * si + j
            r = np.random.default_rng(1000 + m)
            out.append(dict(mx=mx, my=my, mz=mz, Re=float(r.uniform(500.0, 3000.0)),
                            Ro=float(r.uniform(0.0, 0.3)), dt=0.002, seed=1000 + m))
    return out


def run_ensemble(args):
    """Aggregate steps/s of the 48 independent runs in mixed precision: the
    12 runs of each grid as one batch context (dns_create_batch: one launch
    per pass for all 12), the four batches stepped concurrently
    (dns_step_many); beside it the same runs as 48 separate contexts, all
    concurrent (one stream each) and one after another.  Per-run error of the
    batched runs against each run's own FP64 result after min(K, 20) steps:
    at dt 0.002 the 128x97x128 runs pass the explicit term's stability limit
    (their FP64 runs overflow between steps 80 and 200, finite at dt 0.001),
    and the mixed form, seeded by FP32 rounding, diverges earlier."""
    import numpy as np
    import torch
    pkg = load_pkg()
    torch.cuda.set_device(0)
    K, W = args.steps, args.warmup
    mem = ensemble_members()
    states = []
    for c in mem:
        Nx, Nz, Ny = c["mx"] // 3 * 2, c["my"] // 3 * 2, c["mz"] // 4 + 1
        states.append(pkg.seeded_state(Nx, Ny, Nz, 4.0, 2.0, 0.1, c["seed"]))

    def params(c, prec=pkg.PREC_MIXED):
        return pkg.make_params(c["mx"], c["my"], c["mz"], Re=c["Re"], Ro=c["Ro"], dt=c["dt"], precision=prec)

    groups = [list(range(12 * i, 12 * i + 12)) for i in range(len(ENSEMBLE_SIZES))]
    batches = []
    for grp in groups:
        b = pkg.BatchContext([params(mem[m]) for m in grp])
        b.set_state(np.stack([states[m][0] for m in grp]), np.stack([states[m][1] for m in grp]))
        b.bootstrap()
        batches.append(b)
    # accuracy: KE steps of every run, batched mixed vs its own FP64 run alone
    KE = min(K, 20)
    pkg.step_many(batches, KE)
    err = {}
    for grp, b in zip(groups, batches):
        b.synchronize()
        Vm, Om = b.get_state()
        for j, m in enumerate(grp):
            c = mem[m]
            f = pkg.Context(params(c, pkg.PREC_FP64))
            f.set_state(*states[m])
            f.bootstrap()
            f.step(KE)
            f.synchronize()
            Vf, Of = f.get_state()
            f.close()
            key = f"{c['mx'] // 3 * 2}x{c['mz'] // 4 + 1}x{c['my'] // 3 * 2}"
            e = max(float(np.linalg.norm(Vm[j] - Vf) / np.linalg.norm(Vf)),
                    float(np.linalg.norm(Om[j] - Of) / np.linalg.norm(Of)))
            err[key] = max(err.get(key, 0.0), e)

    def timed(ctxs, launch):
        streams = [torch.cuda.ExternalStream(ctx.stream) for ctx in ctxs]
        pkg.step_many(ctxs, W)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        ends = [torch.cuda.Event(enable_timing=True) for _ in ctxs]
        e0.record(streams[0])
        launch(ctxs, streams)
        for e, s in zip(ends, streams):
            e.record(s)
        torch.cuda.synchronize()
        return max(e0.elapsed_time(e) for e in ends)

    def concurrent(ctxs, streams):
        pkg.step_many(ctxs, K)

    def one_by_one(ctxs, streams):
        # each context's K steps after the previous one's (events order the streams)
        prev = None
        for ctx, s in zip(ctxs, streams):
            if prev is not None:
                s.wait_event(prev)
            ctx.step(K)
            prev = torch.cuda.Event()
            prev.record(s)

    for grp, b in zip(groups, batches):
        b.set_state(np.stack([states[m][0] for m in grp]), np.stack([states[m][1] for m in grp]))
        b.bootstrap()
    with ClockSampler(0) as clk:
        ms_batch = timed(batches, concurrent)
    for b in batches:
        b.close()
    singles = []
    for c, (V0, O0) in zip(mem, states):
        ctx = pkg.Context(params(c))
        ctx.set_state(V0, O0)
        ctx.bootstrap()
        singles.append(ctx)
    ms_conc = timed(singles, concurrent)
    ms_seq = timed(singles, one_by_one)
    for ctx in singles:
        ctx.close()
    runs = len(mem)
    rate = lambda ms: round(runs * K / (ms * 1e-3), 1)  # noqa: E731
    return {
        "metric": "ensemble run-steps/s: 48 rotating-Couette runs (12 each of 32x33x32, 64x49x64, "
                  "96x65x96, 128x97x128 modes), mixed precision, batched launches per grid",
        "value": rate(ms_batch), "unit": "run-steps/s",
        "steps": K, "warmup": W, "runs": runs, "ms_all_runs_K_steps": round(ms_batch, 3),
        "batches": "one batch context per grid (12 runs, one launch per pass), 4 batches concurrent",
        "separate_contexts_concurrent": {"value": rate(ms_conc), "ms": round(ms_conc, 3)},
        "one_after_another": {"value": rate(ms_seq), "ms": round(ms_seq, 3)},
        "max_rel_l2_err_vs_own_fp64_run": {k: float("%.3g" % v) for k, v in err.items()},
        "err_after_steps": KE,
        "clocks": clk.summary(),
        "timing": "CUDA events: one before the first launch, one at the end of each context's stream; max",
        "data": "synthetic seeded divergence-free fields (seeds 1000..1047, amplitude 0.1)",
    }


def run_solve(args):
    """The solve-only workload: both wall-normal systems of every pencil
    (dns_solve_wall, the banded factors of the step), Re 3000, dt 0.001,
    Couette base flow, right-hand sides 0.9^n N(0,1) (complex, seed 3) on
    the device; CUDA events on the library's stream around each call."""
    import numpy as np
    import torch
    pkg = load_pkg()
    torch.cuda.set_device(0)
    mx, my, mz = (int(v) for v in args.solve_grid.split(","))
    ctx = pkg.Context(pkg.make_params(mx, my, mz, Re=3000.0, Ro=0.0, dt=0.001))
    Nz, Kx, Ny = ctx.Nz, ctx.Kx, ctx.Ny
    rng = np.random.default_rng(3)
    damp = 0.9 ** np.arange(Ny)
    z = rng.standard_normal((4, Nz, Kx, Ny))
    bv = torch.from_numpy((z[0] + 1j * z[1]) * damp).cuda()
    bo = torch.from_numpy((z[2] + 1j * z[3]) * damp).cuda()
    del z
    wv, wo = bv.clone(), bo.clone()
    s = torch.cuda.ExternalStream(ctx.stream)

    def one_call():
        wv.copy_(bv)
        wo.copy_(bo)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        ctx.solve_wall(wv.data_ptr(), wo.data_ptr(), Ny * 16)
        e1.record(s)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1)

    # the solve's block shape chosen by timing every variant on this grid
    tune = {}
    for v, name in pkg.VARIANT_NAMES[pkg.PASS_Y2].items():
        try:
            ctx.set_variant(pkg.PASS_Y2, v)
        except pkg.DnsError:
            continue
        t = [one_call() for _ in range(5)]  # the first builds the factors and the graph
        tune[name] = round(float(np.median(t[2:])), 4)
    pick = min(tune, key=tune.get)
    ctx.set_variant(pkg.PASS_Y2, {n: v for v, n in pkg.VARIANT_NAMES[pkg.PASS_Y2].items()}[pick])
    ms = []
    for i in range(args.warmup + args.steps):
        wv.copy_(bv)
        wo.copy_(bo)
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        ctx.solve_wall(wv.data_ptr(), wo.data_ptr(), Ny * 16)  # the first call also builds the factors
        e1.record(s)
        torch.cuda.synchronize()
        if i >= args.warmup:
            ms.append(e0.elapsed_time(e1))
    # the last call's solutions against the operators themselves
    res = ctx.solve_residual(bv.data_ptr(), bo.data_ptr(), wv.data_ptr(), wo.data_ptr(), Ny * 16)
    ctx.close()
    t = float(np.median(ms))
    H = Kx * Nz
    return {"metric": f"wall-normal solves (v and omega_y pairs) per second at {Kx * 2 - 2}x{Ny}x{Nz} modes",
            "value": round(H / (t * 1e-3), 1), "unit": "pairs/s", "ms_per_call": round(t, 4),
            "pairs": H, "Ny": Ny, "steps": args.steps, "warmup": args.warmup,
            "rhs_and_solution_bytes": 4 * H * Ny * 16,
            "residual": {"max_pencil_rel_v": float(f"{res[0]:.3e}"), "max_pencil_rel_omega": float(f"{res[1]:.3e}"),
                         "rel_v": float(f"{res[2]:.3e}"), "rel_omega": float(f"{res[3]:.3e}"),
                         "max_backward_err_v": float(f"{res[4]:.3e}"),
                         "max_backward_err_omega": float(f"{res[5]:.3e}"),
                         "definition": "||A x - b|| / ||b|| with A the reference's collocation operators; "
                                       "backward error ||r||inf / (||A||inf ||x||inf + ||b||inf)"},
            "graph": "one CUDA graph per call (right-hand sides to integrated banded form, banded solve of all "
                     "pencils in one launch, finish)",
            "autotune": {"y2_solve": {"ms": tune, "picked": pick}},
            "l2": f"right-hand sides re-copied before each call (2 x {H * Ny * 16 / 1e6:.0f} MB"
                  f"{', > L2' if 2 * H * Ny * 16 > 126e6 else ''})",
            "timing": "CUDA events on the library stream around each synchronous call, median"}


def other_workloads(args):
    """The solve-only workload (384x193x384) and the 48-run ensemble, each
    with its own metric (not the headline); a failure is reported, not
    raised, so the headline line is always printed."""
    import copy
    res = {}
    for name, fn, steps, keys in (
            ("solve_384x193x384", run_solve, 5, ("metric", "value", "unit", "ms_per_call", "pairs", "residual",
                                                  "graph", "autotune", "timing")),
            ("ensemble_48_runs", run_ensemble, 10, ("metric", "value", "unit", "steps", "ms_all_runs_K_steps",
                                                    "batches", "separate_contexts_concurrent",
                                                    "one_after_another", "max_rel_l2_err_vs_own_fp64_run",
                                                    "err_after_steps", "clocks"))):
        a = copy.copy(args)
        a.steps, a.warmup, a.solve_grid = steps, 3, "576,576,768"
        try:
            r = fn(a)
            res[name] = {k: r[k] for k in keys}
        except Exception as e:  # noqa: BLE001
            res[name] = {"error": f"{type(e).__name__}: {e}"}
    return res


def measured_traffic(kernel, config, prec):
    """DRAM bytes per launch (dram__bytes_read.sum + dram__bytes_write.sum)
    of one ncu capture, from the committed summary profiles/dram_traffic.json
    (None when that kernel, workload and precision were not captured)."""
    try:
        with open(os.path.join(ROOT, "profiles", "dram_traffic.json")) as f:
            d = json.load(f)
        e = d["captures"][f"{config}/{prec}/{kernel}"]
        return int(e["read"] + e["write"])
    except Exception:
        return None


def roofline(kms, geo, c, peak, config="256x129x256", prec="mixed"):
    kb = kernel_bytes(geo, c)
    top = max(kms, key=kms.get)
    achieved = kb[top] / (kms[top] * 1e-3) / 1e9
    return top, {"bound": "hbm", "kernel": top, "achieved": round(achieved, 1), "peak": peak,
                 "unit": "GB/s", "frac": round(achieved / peak, 4),
                 "traffic": measured_traffic(top, config, prec),
                 "bytes_per_launch": kb[top], "ms_per_launch": round(kms[top], 4)}


def run_decomposed(args, rank, world):
    """The slab-decomposed mixed step (dns_slab_part) of the headline
    workload: with N ranks one per GPU and the two exchanges as NCCL
    all-to-all collectives (strong scaling: one problem over N GPUs); in one
    process with --slab-ranks R > 1, R ranks on one device with the
    exchanges as device copies (the decomposition's own cost, no scaling).
    CUDA events around the timed steps, maximum over ranks."""
    import importlib
    import numpy as np
    import torch
    pkg = load_pkg()
    slab = importlib.import_module(pkg.__name__ + ".slab")
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(dev)
    params = pkg.make_params(CFG["mx"], CFG["my"], CFG["mz"], Re=CFG["Re"], Ro=CFG["Ro"], dt=CFG["dt"],
                             precision=pkg.PREC_MIXED, device=dev)
    V0, O0 = pkg.seeded_state(CFG["Nx"], CFG["Ny"], CFG["Nz"], 4.0, 2.0, CFG["amplitude"], CFG["seed"])
    R = world if world > 1 else max(1, args.slab_ranks)
    ctxs = [pkg.SlabContext(params, R, r) for r in ([rank] if world > 1 else range(R))]
    for c in ctxs:
        c.scatter_state(V0, O0)
        try:  # the tensor-core wall-normal pass where the grid has it
            c.set_variant(pkg.PASS_Y3, pkg.Y3_TENSOR)
        except pkg.DnsError:
            pass
    K, W = args.steps, args.warmup
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    if world > 1:
        bufs = slab.step_dist(ctxs[0], boot=True)
        slab.step_dist(ctxs[0], W, bufs=bufs)
        ctxs[0].synchronize()
        torch.distributed.barrier()
        torch.cuda.synchronize()
        s = torch.cuda.ExternalStream(ctxs[0].stream)
        with ClockSampler(dev) as clk:
            e0.record(s)
            slab.step_dist(ctxs[0], K, bufs=bufs)
            e1.record(s)
            ctxs[0].synchronize()
            torch.cuda.synchronize()
        ms = dist_max(e0.elapsed_time(e1)) / K
        xbytes = sum(sum(bufs.split[x][0]) for x in (0, 1))
        xbytes = int(dist_max(xbytes))  # the busiest rank's bytes sent per step
    else:
        bufs = slab.step_local(ctxs, boot=True)
        slab.step_local(ctxs, W, bufs=bufs)
        torch.cuda.synchronize()
        with ClockSampler(dev) as clk:
            e0.record()
            slab.step_local(ctxs, K, bufs=bufs)
            e1.record()
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1) / K
        xbytes = max(sum(sum(b.split[x][0]) for x in (0, 1)) for b in bufs)
    finite = all(np.isfinite(c.get_local(pkg.SLAB_V)).all() for c in ctxs)
    # kernels per step and rank: y3 and y1 per run, one copy per segment and
    # exchange direction at both ends, zb, x, zf and the solve
    launches = 0
    for c in ctxs:
        nseg = sum(len(pkg.slab_segments(CFG["mx"], CFG["my"], CFG["mz"], R, c.rank, role))
                   for role in (pkg.SLAB_PENCILS, pkg.SLAB_PLANES))
        launches += 2 * len(c.runs) + 2 * nseg + 4
    if world > 1:
        launches = int(dist_max(launches))
    for c in ctxs:
        c.close()
    return {"metric": METRIC, "value": round(1000.0 / ms, 2), "unit": "steps/s", "n_gpus": world,
            "steps": K, "warmup": W, "ms_per_step": round(ms, 4), "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None,
            "dtype": "f32 transforms/Lamb + f64 solves/state (mixed)",
            "data": "synthetic seeded divergence-free field (seed 0, amplitude 0.1)",
            "config": {"workload": f"rotating plane Couette {args.config} modes, slab-decomposed step",
                       "parallelism": (f"slab x{world} (NCCL all-to-all)" if world > 1 else
                                       f"slab x{R} ranks on one device (exchanges as device copies)"),
                       "l2": "inputs larger than L2 (no flush)"},
            "exchange_bytes_per_step_max_rank": xbytes, "state_finite": bool(finite),
            "clocks": clk.summary(), "gpu_launches": launches * K}


def launch_ranks(n):
    """Run this command as n local ranks under torch.distributed.run (one
    process per GPU, rendezvous on 127.0.0.1) and return its exit status."""
    import socket
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", f"--nproc-per-node={n}",
           "--master-addr=127.0.0.1", f"--master-port={port}", os.path.abspath(__file__), *sys.argv[1:]]
    return subprocess.call(cmd)


def check_launch(rank, world):
    """Join the process group (NCCL with GPUs, else gloo) and have rank 0
    print the job's rank count: the launch path without device work."""
    import datetime
    import torch
    backend = "nccl" if torch.cuda.is_available() else "gloo"
    if backend == "nccl":
        torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    torch.distributed.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    t = torch.ones(1, device="cuda" if backend == "nccl" else "cpu")
    torch.distributed.all_reduce(t)
    if rank == 0:
        print(json.dumps({"n_gpus": world, "ranks_joined": int(t.item()), "backend": backend}))
    torch.distributed.barrier()
    torch.distributed.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="skip the solve-only and ensemble workloads appended to the line")
    ap.add_argument("--config", default="256x129x256", choices=sorted(CONFIGS))
    ap.add_argument("--only", choices=["fp64", "mixed"], default=None,
                    help="run one precision only (bootstrap + warm-up + timed steps), for "
                         "profiling captures; prints per-kernel times, not the bench line")
    ap.add_argument("--variant", action="append", default=[],
                    help="with --only: PASS=VARIANT (names as in the bench line's autotune block) "
                         "instead of the autotuner; repeatable")
    ap.add_argument("--solve", action="store_true",
                    help="the solve-only workload (dns_solve_wall): prints its own line")
    ap.add_argument("--solve-grid", default="576,576,768",
                    help="mx,my,mz of --solve (default 384x193x384 modes)")
    ap.add_argument("--ensemble", action="store_true",
                    help="the 48-run ensemble (concurrent runs, one GPU): prints its own line")
    ap.add_argument("--check-launch", action="store_true",
                    help="start the ranks and print their count only (no device work)")
    ap.add_argument("--decomposed", action="store_true",
                    help="the slab-decomposed step: one problem over the N ranks (NCCL all-to-all "
                         "exchanges), or over --slab-ranks ranks on one device")
    ap.add_argument("--slab-ranks", type=int, default=2,
                    help="with --decomposed on one process: ranks emulated on the device")
    args = ap.parse_args()
    global CFG
    CFG = CONFIGS[args.config]
    args.warmup = max(args.warmup, 3)
    if "WORLD_SIZE" not in os.environ and args.gpus > 1:
        # not started by torchrun: start the N ranks here, one process per GPU
        sys.exit(launch_ranks(args.gpus))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if world != args.gpus:
        sys.exit(f"bench.py: --gpus {args.gpus} but WORLD_SIZE={world}: launch one rank per GPU")
    if args.check_launch:
        check_launch(rank, world)
        return

    if args.impl == "reference":
        # the reference's algorithm on the host (oracle port): rank 0 only
        if rank == 0:
            sys.path.insert(0, ROOT)
            from oracle import ref_arm
            print(json.dumps(ref_arm.run(args, CFG, METRIC)))
        return

    if world > 1:
        import datetime
        import torch
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    if args.only:
        print(json.dumps(run_one(args)))
        return
    if args.solve:
        if rank == 0:
            print(json.dumps(run_solve(args)))
        return
    if args.ensemble:
        if rank == 0:
            print(json.dumps(run_ensemble(args)))
        return
    if args.decomposed:
        r = run_decomposed(args, rank, world)
        if rank == 0:
            print(json.dumps(r))
        if world > 1:
            import torch
            torch.distributed.barrier()
            torch.distributed.destroy_process_group()
        return
    r = run_ours(args, rank, world)
    peak, peak_kind = measured_peaks()
    top64, roof64 = roofline(r["kms64"], r["geo"], 16, peak, args.config, "fp64")
    topmx, roofmx = roofline(r["kmsmx"], r["geo"], 8, peak, args.config, "mixed")
    step_bytes64 = sum(kernel_bytes(r["geo"], 16).values())
    step_bytes_mx = sum(kernel_bytes(r["geo"], 8).values())
    out = None
    if rank == 0:
        cpu = None if (args.no_cpu_baseline or world > 1 or args.config != "256x129x256") else cpu_baseline()
        n = world
        value = replica_value(n, r["msmx"])
        out = {
            "metric": METRIC,
            "value": round(value, 2),
            "unit": "steps/s",
            "n_gpus": n,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": round(r["msmx"], 4),
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32 transforms/Lamb + f64 solves/state (mixed)",
            "data": "synthetic seeded divergence-free field (seed 0, amplitude 0.1)",
            "config": {"workload": (f"rotating plane Couette {args.config} modes (mx,my,mz="
                                    f"{CFG['mx']},{CFG['my']},{CFG['mz']}; physical {CFG['mx']}x"
                                    f"{CFG['mz'] // 2 + 1}x{CFG['my']}), Re {CFG['Re']:g}, "
                                    f"Ro {CFG['Ro']:g}, dt {CFG['dt']:g}"),
                       "parallelism": f"replicas x{n}" if n > 1 else "single GPU",
                       "l2": ("inputs larger than L2: each step streams ~3.7 GB (mixed) / ~6.8 GB (FP64) "
                              "through HBM, buffers of 0.3-0.8 GB per field set >> 126 MB L2 (no flush)")},
            "fp64": {"steps_per_s": round(replica_value(n, r["ms64"]), 2), "ms_per_step": round(r["ms64"], 4),
                     "roofline": roof64, "step_bytes_algorithmic": step_bytes64,
                     "step_frac_of_peak": round(step_bytes64 / (r["ms64"] * 1e-3) / 1e9 / peak, 4)},
            "mixed_vs_fp64": {"speedup": round(r["ms64"] / r["msmx"], 3),
                              "per_step_rel_l2_err": r["err"],
                              "within_1e-6": bool(all(r["err"][k] <= 1e-6 for k in ("u", "v", "w", "omega_y"))),
                              "accumulated_rel_l2_err": r["acc"],
                              "accumulated_after_steps": r["acc_steps"],
                              "axes": "standard: u streamwise, v wall-normal, w spanwise"},
            "roofline": dict(roofmx, peak_kind=f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"),
            "step_frac_of_peak": round(step_bytes_mx / (r["msmx"] * 1e-3) / 1e9 / peak, 4),
            "step_bytes_algorithmic": step_bytes_mx,
            "factor_bytes_per_step": factor_bytes(r["geo"]),
            "autotune": r["autotune"],
            "kernel_ms": {"fp64": {k: round(v, 4) for k, v in r["kms64"].items()},
                          "mixed": {k: round(v, 4) for k, v in r["kmsmx"].items()}},
            "e2e": {"value": round(replica_value(n, r["e2e_ms"]), 2), "unit": "steps/s",
                    "h2d_bytes_per_step": r["state_bytes"], "d2h_bytes_per_step": r["state_bytes"]},
            "gpu_launches": 6 * args.steps,
            "cpu_baseline": cpu,
            "clocks": r["clocks"],
            "setup_seconds": round(r["setup_s"], 2),
            "device_bytes": r["mem"],
        }
        if world == 1 and args.config == "256x129x256" and not args.no_extras:
            out["other_workloads"] = other_workloads(args)
        print(json.dumps(out))
    if world > 1:
        import torch
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
