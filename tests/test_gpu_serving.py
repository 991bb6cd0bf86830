"""GPU tests of the serving layer (vistio_server_*): continuous batching of
drape requests of different sizes, materials and kinds.

* Each request's result in the mix equals the same request run alone on a
  standalone solver (within 1e-6 m; the kernels compute every garment from
  its own data, so they agree bit for bit).
* Requests submitted while others are on the GPU are admitted before those
  finish (their work overlaps), and several cohorts are active at once.
* A repeated garment with the same material and dt reuses the cached set-up.
* With a device-memory budget that holds one cohort at a time, requests
  wait for memory and still complete; one that can never fit fails with
  VISTIO_ERR_OOM.
"""
import dataclasses
import time

import numpy as np
import pytest

from vistio_b200 import api, scenarios

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0
SPHERE = api.Contact(has_ground=True, ground_height=-0.3, has_sphere=True, sphere_center=(0.0, 0.0, 0.0),
                     sphere_radius=0.3, kappa=1e4)


def plain_request(side, length, stiffness, bend, density, steps):
    mesh = scenarios.hanging_sheet(side, length)
    cfg = api.drape_config(max_iterations=10)
    setup = api.SetupDesc(stiffness=stiffness, bend_stiffness=bend, density_gsm=density)
    return dict(mesh=mesh, config=cfg, setup=setup, steps=steps, dt=DT, contact=None, ipc=False, pinned=mesh.pinned)


def sphere_request(side, steps, density=150.0):
    mesh = scenarios.sphere_drape(side=side, length=1.5, height=0.35)
    cfg = api.drape_config(max_iterations=15, al_max_iterations=5, barrier_d_hat=1e-3, barrier_kappa=1e4)
    setup = api.SetupDesc(stiffness=1e3, bend_stiffness=1e-4, density_gsm=density)
    return dict(mesh=mesh, config=cfg, setup=setup, steps=steps, dt=DT, contact=SPHERE, ipc=True, pinned=mesh.pinned)


def run_alone(req):
    s = api.ProjectiveDynamicsSolver().init_explicit(req["mesh"], req["config"], req["setup"], pinned=req["pinned"])
    for _ in range(req["steps"]):
        if req["ipc"]:
            s.step_with_ipc(req["dt"], req["contact"])
        else:
            s.step(req["dt"])
    return s.state()


def submit(server, req):
    return server.submit(req["mesh"], req["config"], req["setup"], req["steps"], req["dt"], contact=req["contact"],
                         ipc=req["ipc"], pinned=req["pinned"])


def test_requests_in_the_mix_equal_requests_alone():
    first = [plain_request(12, 0.8, 800.0, 1e-4, 120.0, 40), sphere_request(16, 30),
             plain_request(20, 1.2, 3000.0, 5e-4, 250.0, 40)]
    later = [plain_request(9, 0.5, 400.0, 2e-5, 90.0, 40),   # same step configuration as the first plain ones
             sphere_request(12, 30, density=200.0),
             plain_request(12, 0.8, 800.0, 1e-4, 120.0, 40)]  # repeats first[0]: cached set-up
    srv = api.Server(hbm_budget_bytes=4 << 30, max_cohort=8, setup_threads=3, steps_per_slice=5)
    ids = [submit(srv, r) for r in first]
    # run until the first wave is on the GPU, then submit the second wave
    t0 = time.time()
    while not all(srv.query(i)["state"] == "running" for i in ids):
        srv.tick()
        assert time.time() - t0 < 120
    ids += [submit(srv, r) for r in later]
    srv.drain(600)
    info = [srv.query(i) for i in ids]
    assert all(q["state"] == "done" for q in info), info
    # the second wave was admitted while the first was still running
    first_done = min(q["done_s"] for q in info[:3])
    assert any(q["start_s"] < first_done for q in info[3:]), info
    st = srv.stats()
    print(st)
    assert st["max_cohorts_active"] >= 2
    assert info[5]["cache_hit"]
    assert st["completed"] == 6 and st["failed"] == 0
    assert 0 < st["p50_latency_s"] <= st["p99_latency_s"]
    worst = 0.0
    for rid, req in zip(ids, first + later):
        pos, vel = srv.result(rid)
        p1, v1 = run_alone(req)
        worst = max(worst, float(np.abs(pos - p1).max()), float(np.abs(vel - v1).max()) * DT)
    print(f"max |mix - alone| = {worst:.3e} m")
    assert worst <= 1e-6, worst
    srv.close()


def test_memory_budget_admission_and_oversize_request():
    reqs = [plain_request(12, 0.6, 600.0, 1e-4, 150.0, 20), plain_request(14, 0.9, 900.0, 1e-4, 150.0, 20),
            plain_request(13, 0.7, 700.0, 1e-4, 150.0, 20)]
    from vistio_b200 import _lib
    import ctypes as C
    needs = []
    for r in reqs:
        # as the server's set-up threads build it: factorized on the host
        cfg = dataclasses.replace(r["config"], host_factorization=True)
        probe = api.ProjectiveDynamicsSolver().init_explicit(r["mesh"], cfg, r["setup"], pinned=r["pinned"])
        need = C.c_uint64()
        _lib.check(_lib.lib().vistio_solver_device_bytes(probe.h, 0, C.byref(need)))
        needs.append(need.value)
    # room for the largest request alone, and for no two of the three together
    budget = max(needs) + min(needs) // 2
    assert budget < sorted(needs)[0] + sorted(needs)[1]
    srv = api.Server(hbm_budget_bytes=budget, max_cohort=8, setup_threads=2, steps_per_slice=5)
    ids = [submit(srv, r) for r in reqs]
    big = plain_request(40, 1.0, 1e3, 1e-4, 150.0, 5)  # never fits this budget
    big_id = submit(srv, big)
    srv.drain(600)
    st = srv.stats()
    assert st["max_cohorts_active"] == 1, st
    assert st["completed"] == 3 and st["failed"] == 1, st
    q = srv.query(big_id)
    assert q["state"] == "failed" and q["status"] == 10, q  # VISTIO_ERR_OOM
    for rid, req in zip(ids, reqs):
        pos, _ = srv.result(rid)
        assert np.abs(pos - run_alone(req)[0]).max() <= 1e-6
    srv.close()


def test_admission_window_forms_larger_cohorts():
    """With an admission window, requests of one step configuration that
    become ready while a cohort runs wait (bounded) for company: the second
    wave's five requests start as one cohort instead of trickling into
    several, and every result still equals the request run alone."""
    blocker = plain_request(32, 1.0, 1000.0, 1e-4, 150.0, 300)
    wave = [plain_request(8 + k, 0.5 + 0.1 * k, 500.0 + 100 * k, 1e-4, 120.0, 30) for k in range(5)]
    srv = api.Server(hbm_budget_bytes=4 << 30, max_cohort=16, setup_threads=1, steps_per_slice=5, admit_wait_ms=400)
    b_id = submit(srv, blocker)
    t0 = time.time()
    while srv.query(b_id)["state"] != "running":
        srv.tick()
        assert time.time() - t0 < 120
    ids = [submit(srv, r) for r in wave]  # one set-up thread: they become ready one by one
    srv.drain(600)
    info = [srv.query(i) for i in ids]
    assert all(q["state"] == "done" for q in info), info
    assert len({q["cohort"] for q in info}) == 1, info  # one cohort for the whole wave
    st = srv.stats()
    assert st["cohorts_started"] == 2, st
    for rid, req in zip(ids, wave):
        pos, _ = srv.result(rid)
        assert np.abs(pos - run_alone(req)[0]).max() <= 1e-6
    srv.close()
