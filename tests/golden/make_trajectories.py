"""Generate the FP64 trajectory fixtures of the oracle (tests/golden/traj_*.npz).

Test infrastructure: run on the CPU from the repository root,

    python tests/golden/make_trajectories.py config1     # ~15 min, 8 cores
    python tests/golden/make_trajectories.py config2     # ~15 min

Each fixture holds the oracle's trajectory (the reference's algorithm,
explicit inverses as source/solver.cpp:107-123 multiplies by) from the
seeded state, on a fixed sample of pencils at a few steps, so that the
device test can run the full trajectory on the GPU without running the
oracle live:

* ``ky, kx``        the sampled pencils (always including the mean pencil
                    (0,0) and the lowest modes);
* ``steps``         the snapshot steps;
* ``V, O``          (len(steps), P, Ny) complex: v-hat and omega_y-hat (the
                    reference's rhs_v / rhs_omega_y after nextStep) at the
                    sampled pencils;
* ``norm_V, norm_O`` full-field L2 norms after every step (1..nsteps);
* ``spread``        (len(steps), 6): relative L2, over the full field, of each
                    getUVW component (u, v span, w, omega_x, omega_y span,
                    omega_z) between the oracle with explicit inverses and the
                    oracle with LU solves: the oracle's own rounding floor;
* the parameters of the run.
"""
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle.rpcf_oracle as O  # noqa: E402
from conftest import load_package  # noqa: E402

CONFIGS = {
    # Poiseuille U = 1 - y^2 at Re_b = 5600 (Re = 1.5 Re_b = 8400 in the
    # centreline scaling), 128 x 65 x 128 modes.  150 steps: the reference's
    # algorithm (and the oracle with it) is unstable at these parameters --
    # the norm of the nonlinear term grows ~100x by step 150 and the state
    # overflows between steps 150 and 160 -- so the 200 steps of the
    # workload have no finite end state to compare.
    "config1": dict(mx=192, my=192, mz=256, Re=8400.0, Ro=0.0, dt=0.002, prof=(1.0, 0.0, -1.0),
                    amp=0.1, seed=0, nsteps=150, steps=(1, 2, 10, 50, 100, 150), npencils=256,
                    solvers=("inverse", "lu")),
    # rotating Couette at 256 x 129 x 256 modes in FP64, 3 steps
    "config2": dict(mx=384, my=384, mz=512, Re=3000.0, Ro=0.02, dt=0.001, prof=(0.5, 0.5, 0.0),
                    amp=0.1, seed=0, nsteps=3, steps=(1, 2, 3), npencils=256,
                    solvers=("batched", "batched-lu")),
}


def sample_pencils(sz, n, seed=7):
    rng = np.random.default_rng(seed)
    fixed = [(0, 0), (0, 1), (1, 0), (1, 1), (sz.ny - 1, 1), (2, 3), (sz.ny // 2, 0),
             (0, sz.hnx - 1)]
    H = sz.ny * sz.hnx
    ids = {y * sz.hnx + x for (y, x) in fixed}
    while len(ids) < n:
        ids.add(int(rng.integers(H)))
    ids = np.array(sorted(ids))
    return ids // sz.hnx, ids % sz.hnx


def run(cfg, solver, ky, kx, log):
    pkg = load_package()
    p = O.Params(cfg["mx"], cfg["my"], cfg["mz"], Re=cfg["Re"], Ro=cfg["Ro"], dt=cfg["dt"],
                 prof=cfg["prof"])
    pb = O.Problem(p)
    pb.solver = solver
    sz = pb.sz
    V, Om = pkg.seeded_state(sz.nx, sz.nz, sz.ny, p.n_pi_x, p.n_pi_y, cfg["amp"], cfg["seed"])
    pb.set_state(V, Om)
    pb.bootstrap()
    snapV, snapO, full, nV, nO = [], [], [], [], []
    t0 = time.time()
    for k in range(1, cfg["nsteps"] + 1):
        pb.step()
        nV.append(np.linalg.norm(pb.V))
        nO.append(np.linalg.norm(pb.O))
        if k in cfg["steps"]:
            snapV.append(pb.V[ky, kx].copy())
            snapO.append(pb.O[ky, kx].copy())
            full.append([f.copy() for f in pb.spectral_fields()])
            log(f"{solver}: step {k} ({time.time() - t0:.0f} s)")
    return np.array(snapV), np.array(snapO), full, np.array(nV), np.array(nO)


def main(name):
    cfg = CONFIGS[name]
    sz = O.Sizes(cfg["mx"], cfg["my"], cfg["mz"])
    ky, kx = sample_pencils(sz, cfg["npencils"])
    log = lambda m: print(m, flush=True)  # noqa: E731
    a = run(cfg, cfg["solvers"][0], ky, kx, log)
    b = run(cfg, cfg["solvers"][1], ky, kx, log)
    spread = np.array([[np.linalg.norm(fa - fb) / np.linalg.norm(fb) for fa, fb in zip(A, B)]
                       for A, B in zip(a[2], b[2])])
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), f"traj_{name}.npz")
    np.savez_compressed(out, ky=ky, kx=kx, steps=np.array(cfg["steps"]), V=a[0], O=a[1],
                        norm_V=a[3], norm_O=a[4], spread=spread,
                        mx=cfg["mx"], my=cfg["my"], mz=cfg["mz"], Re=cfg["Re"], Ro=cfg["Ro"],
                        dt=cfg["dt"], prof=np.array(cfg["prof"]), amp=cfg["amp"], seed=cfg["seed"],
                        nsteps=cfg["nsteps"])
    log(f"wrote {out}")
    for s, row in zip(cfg["steps"], spread):
        log(f"step {s}: spread " + " ".join(f"{e:.2e}" for e in row))


if __name__ == "__main__":
    main(sys.argv[1])
