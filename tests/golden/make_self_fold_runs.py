"""Generates the FP64 oracle fixtures of the self-fold full runs.

Test infrastructure: runs the oracle (the C++ restatement of the reference's
CPU step, FP64 and FP32 "ref32" modes) over the whole self-fold configuration
and stores checkpoints that tests/test_gpu_contact_runs.py compares the GPU's
free run against. The FP64 run takes several minutes on one core, too long to
repeat inside a GPU test.

Configuration (both runs): a 0.2 m x 2.0 m ribbon of 40 x 400 cells (16441
vertices) rotated 45 degrees about x, orthotropic membrane (warp 1e3, weft
6e2, element stiffness 1e3), dihedral bending 1e-4, density 150 g/m^2,
ground y = 0, self contact with 1-ring exclusion (thickness 1.5 d_hat),
d_hat = 5e-4 m read as a distance (barrier_d_hat = d_hat^2), matrix dt =
step dt = 1/120 s, kappa from estimate_initial_kappa with the mean vertex mass
(runner.rs:190-195), AL <= 5, 10 PD iterations, 300 steps.

  drop   lowest point 0.5 m above the ground, as the configuration states;
  near   lowest point 1 mm above the ground, so that ground contact acts
         from the first steps.

Output: self_fold_<name>.npz with the FP64 positions (float32) after steps
100, 200 and 300, and per step the max |x_ref32 - x_fp64| (the reference's
own FP32 spread) and the FP64 run's active-contact count.

With --literal N it instead steps the reference's literal wiring of the
configuration for N steps and prints each step's lowest point, highest
point, largest displacement and active contacts (no fixture): the system
matrix assembled with dt = 1/60 while the steps use 1/120, and d_hat = 5e-4
passed as barrier_d_hat (a squared distance), thickness 1.5 d_hat.

Usage: python tests/golden/make_self_fold_runs.py [drop|near ...]
       python tests/golden/make_self_fold_runs.py --literal N [precision]
"""
from __future__ import annotations

import os
import sys
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle_api as O  # noqa: E402
from vistio_b200 import scenarios  # noqa: E402

DT = 1.0 / 120.0
D_HAT = 5e-4
STEPS = 300
CHECKPOINTS = (100, 200, 300)
LOWEST = {"drop": 0.5, "near": 0.001}


def params():
    return O.init_params(model=O.MODEL_ORTHO, stiffness=1e3, warp=1e3, weft=6e2, bend_stiffness=1e-4,
                         density_gsm=150.0, matrix_dt=DT)


def contact(mesh):
    c = O.Contact()
    c.has_ground, c.ground_height = 1, 0.0
    c.self_collision, c.bvh_faithful = 1, 0
    c.thickness = 1.5 * D_HAT
    probe = O.OracleSim(mesh, params(), O.default_config(), precision=1)
    c.kappa = float(O.lib().orc_estimate_kappa(0.0, float(probe.masses().mean()), 9.81, D_HAT * D_HAT))
    return c


def run(name):
    mesh = scenarios.self_fold(40, 400, 0.2, 2.0, lowest=LOWEST[name])
    cfg = O.default_config(max_iterations=10, al_max_iterations=5, barrier_d_hat=D_HAT * D_HAT)
    c = contact(mesh)
    sims = [O.OracleSim(mesh, params(), cfg, precision=p) for p in (1, 0)]
    for s in sims:
        s.set_ground(1, 0.0)
    spread, active, keep = [], [], {}
    for n in range(1, STEPS + 1):
        res = [None, None]

        def one(k):
            res[k] = sims[k].step_ipc(DT, c)

        th = [threading.Thread(target=one, args=(k,)) for k in range(2)]
        for t in th:
            t.start()
        for t in th:
            t.join()
        p64, p32 = sims[0].state()[0], sims[1].state()[0]
        spread.append(float(np.abs(p32 - p64).max()))
        active.append(int(res[0].active_contacts))
        if n in CHECKPOINTS:
            keep[f"pos_{n}"] = p64.astype(np.float32)
        if n % 25 == 0:
            print(f"{name} step {n}: ref32 spread {spread[-1]:.3e} active {active[-1]} "
                  f"lowest {p64[:, 1].min():.4f}", flush=True)
    out = os.path.join(HERE, f"self_fold_{name}.npz")
    np.savez_compressed(out, kappa=np.float32(c.kappa), ref32_spread=np.array(spread, np.float32),
                        active=np.array(active, np.uint32), **keep)
    print("wrote", out)


def literal(nsteps, precision=1):
    mesh = scenarios.self_fold(40, 400, 0.2, 2.0, lowest=0.5)
    prm = O.init_params(model=O.MODEL_ORTHO, stiffness=1e3, warp=1e3, weft=6e2, bend_stiffness=1e-4,
                        density_gsm=150.0, matrix_dt=1.0 / 60.0)
    cfg = O.default_config(max_iterations=10, al_max_iterations=5, barrier_d_hat=D_HAT)
    sim = O.OracleSim(mesh, prm, cfg, precision=precision)
    sim.set_ground(1, 0.0)
    c = O.Contact()
    c.has_ground, c.ground_height = 1, 0.0
    c.self_collision, c.bvh_faithful = 1, 0
    c.thickness = 1.5 * D_HAT
    c.kappa = float(O.lib().orc_estimate_kappa(0.0, float(sim.masses().mean()), 9.81, D_HAT))
    prev = sim.state()[0]
    for n in range(1, nsteps + 1):
        r = sim.step_ipc(DT, c)
        p = sim.state()[0]
        print(f"literal step {n}: lowest {p[:, 1].min():.4f} highest {p[:, 1].max():.4f} "
              f"max displacement {np.abs(p - prev).max():.4f} active {r.active_contacts} finite {np.isfinite(p).all()}",
              flush=True)
        if not np.isfinite(p).all():
            break
        prev = p


if __name__ == "__main__":
    if sys.argv[1:2] == ["--literal"]:
        literal(int(sys.argv[2]), int(sys.argv[3]) if len(sys.argv) > 3 else 1)
    else:
        for nm in sys.argv[1:] or list(LOWEST):
            run(nm)
