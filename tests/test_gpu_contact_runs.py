"""Full-run parity of step_with_ipc: the GPU runs a whole contact configuration
freely (never re-seeded from the oracle) and is compared with the FP64 oracle
run of the same steps, beside the reference's own FP32 arithmetic (the
oracle's ref32 mode) on the same run.

* Sphere drape, 64 x 64 cells (4225 vertices), 180 steps: the sheet falls
  0.2 m onto a sphere of radius 0.3 m; with these light vertices (8e-5 kg)
  the kappa = 1e4 barrier throws the centre back up within the step it enters
  the contact zone, and the sheet keeps bouncing. Rounding differences grow
  about tenfold every ten steps after the first bounce: ref32 is 2.5e-4 m
  from FP64 at step 16 and tenths of a metre at step 180. No FP32 solver can
  stay within 1e-4 m of FP64 over that run, so the GPU is held to the bar
  while the reference's own FP32 meets it, must leave it no earlier than
  ref32 does, and at the end stays within twice ref32's largest spread.
* Self fold, 40 x 400 cells (16441 vertices), 300 steps at dt = 1/120 with
  ground and self contact, from 0.5 m (as configured) and from 1 mm (ground
  contact from the first steps). The FP64 runs take minutes on one core, so
  their checkpoints are fixtures written by tests/golden/make_self_fold_runs.py.
  At every checkpoint the GPU is within 1e-4 m of FP64, or within ref32's
  own spread where that is wider.
"""
import os
import threading

import numpy as np
import pytest

import oracle_api as O
from vistio_b200 import api, scenarios

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
BAR = 1e-4  # m: the position bar against FP64 after a run


def first_above(err, thr):
    """First step (1-based) whose error exceeds thr, or len(err) + 1."""
    idx = np.nonzero(np.asarray(err) > thr)[0]
    return int(idx[0]) + 1 if len(idx) else len(err) + 1


def test_sphere_drape_full_run():
    dt, steps = 1.0 / 60.0, 180
    mesh = scenarios.sphere_drape(side=64, length=1.5, height=0.5)
    contact = api.Contact(has_ground=True, ground_height=-0.3, has_sphere=True, sphere_center=(0.0, 0.0, 0.0),
                          sphere_radius=0.3, kappa=1e4)
    cfg = api.drape_config(max_iterations=15, al_max_iterations=5, barrier_d_hat=1e-3, barrier_kappa=1e4)
    setup = api.SetupDesc(stiffness=1e3, bend_stiffness=1e-4, density_gsm=150.0)
    gpu = api.ProjectiveDynamicsSolver().init_explicit(mesh, cfg, setup)

    oc = O.default_config(max_iterations=15, al_max_iterations=5, barrier_d_hat=1e-3)
    c = O.Contact()
    c.has_ground, c.ground_height, c.has_sphere = 1, -0.3, 1
    c.sphere_center[:] = (0.0, 0.0, 0.0)
    c.sphere_radius, c.kappa = 0.3, 1e4
    ref = {}
    for prec in (1, 0):
        ref[prec] = O.OracleSim(mesh, O.init_params(stiffness=1e3, bend_stiffness=1e-4, density_gsm=150.0), oc,
                                precision=prec)
        ref[prec].set_ground(1, -0.3)
    traj = {1: [], 0: []}

    def oracle_run(prec):
        for _ in range(steps):
            ref[prec].step_ipc(dt, c)
            traj[prec].append(ref[prec].state()[0])

    threads = [threading.Thread(target=oracle_run, args=(p,)) for p in (1, 0)]
    for t in threads:
        t.start()
    gp = []
    for _ in range(steps):
        gpu.step_with_ipc(dt, contact)
        gp.append(gpu.state()[0])
    for t in threads:
        t.join()
    e_gpu = [float(np.abs(g - r).max()) for g, r in zip(gp, traj[1])]
    e_32 = [float(np.abs(a - r).max()) for a, r in zip(traj[0], traj[1])]
    n32, ngpu = first_above(e_32, BAR), first_above(e_gpu, BAR)
    n32m, ngpum = first_above(e_32, 1e-3), first_above(e_gpu, 1e-3)
    for n in (10, 16, 20, 30, 40, 60, 90, 120, 150, 180):
        print(f"step {n}: gpu {e_gpu[n - 1]:.2e} ref32 {e_32[n - 1]:.2e}")
    print(f"first step above 1e-4 m: gpu {ngpu}, ref32 {n32}; above 1e-3 m: gpu {ngpum}, ref32 {n32m}")
    # while the reference's own FP32 meets the bar, so does the GPU
    assert max(e_gpu[: n32 - 1]) <= BAR, (n32, max(e_gpu[: n32 - 1]))
    # and the GPU leaves the bar (and 1e-3 m) no earlier than ref32
    assert ngpu >= n32 and ngpum >= n32m, (ngpu, n32, ngpum, n32m)
    # at the end the GPU's error is within twice the reference FP32's largest spread
    assert e_gpu[-1] <= max(BAR, 2.0 * max(e_32)), (e_gpu[-1], max(e_32))
    # no vertex inside the sphere or below the ground at any step
    for p in gp:
        assert np.isfinite(p).all()
        assert float(np.linalg.norm(p, axis=1).min()) >= 0.3 - 1e-3
        assert float(p[:, 1].min()) >= -0.3 - 1e-3


@pytest.mark.parametrize("name,lowest", [("drop", 0.5), ("near", 0.001)])
def test_self_fold_full_run(name, lowest):
    fx = np.load(os.path.join(GOLDEN, f"self_fold_{name}.npz"))
    dt, d_hat, steps = 1.0 / 120.0, 5e-4, 300
    mesh = scenarios.self_fold(40, 400, 0.2, 2.0, lowest=lowest)
    setup = api.SetupDesc(model=api.MODEL_ORTHOTROPIC, stiffness=1e3, warp_stiffness=1e3, weft_stiffness=6e2,
                          bend_stiffness=1e-4, density_gsm=150.0, matrix_dt=dt)
    cfg = api.drape_config(max_iterations=10, al_max_iterations=5, barrier_d_hat=d_hat * d_hat, barrier_kappa=0.0)
    # kappa 0: the library estimates it from the garment's mean vertex mass, as the fixture did
    contact = api.Contact(has_ground=True, ground_height=0.0, self_collision=True, kappa=0.0,
                          thickness=1.5 * d_hat)
    gpu = api.ProjectiveDynamicsSolver().init_explicit(mesh, cfg, setup, pinned=mesh.pinned)
    active, lowest_y = 0, 1.0
    worst, worst32 = 0.0, 0.0
    for n in range(1, steps + 1):
        r = gpu.step_with_ipc(dt, contact)
        active = max(active, r.active_contacts)
        key = f"pos_{n}"
        if key in fx.files:
            p = gpu.state()[0]
            assert np.isfinite(p).all()
            lowest_y = min(lowest_y, float(p[:, 1].min()))
            e = float(np.abs(p - fx[key]).max())
            s32 = float(fx["ref32_spread"][n - 1])
            worst, worst32 = max(worst, e), max(worst32, s32)
            print(f"self_fold {name} step {n}: gpu {e:.2e} ref32 {s32:.2e} fp64 active {int(fx['active'][n - 1])}")
            # within the bar, or within the reference FP32's own spread where that is wider
            assert e <= max(BAR, s32), (n, e, s32)
    print(f"self_fold {name}: worst {worst:.2e} (ref32 {worst32:.2e}), max active {active}, lowest {lowest_y:.4f}")
    if name == "near":
        assert active > 0 and int(fx["active"].max()) > 0
    assert lowest_y >= -1.5 * d_hat
