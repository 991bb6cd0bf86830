"""Benchmark: batched drape steps/s on B200 (the batched-sheets workload).

Workload: 512 hanging sheets of uneven size (grid side 8 distinct values drawn
uniformly from 16..128 and assigned round-robin, side length U[0.5, 2] m,
stretch log-U[2e2, 5e3] N/m, bending log-U[1e-5, 1e-3] N m, density
U[0.08, 0.30] kg/m^2), plain PD step with 10 local-global iterations,
dt = 1/60 s, seeded synthetic inputs. One step advances every instance once;
the metric is instance-steps per second over the whole job.

Arms:
  default            the CUDA batch (one CUDA graph per step over ragged SoA);
  --impl reference   the reference CPU path (the oracle's FP32 restatement,
                     since the Rust reference cannot be built here) on all
                     host threads, rank 0 only.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import dataclasses
import json
import math
import os
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "batched drape steps/sec vs plain GPU PD at <=1e-4 m err; p50/p99 latency"
UNIT = "instance-steps/s"
DT = 1.0 / 60.0
ITERS = 10
ERR_STEPS = 120  # steps of the batched workload checked against the FP64 oracle


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--instances", type=int, default=512)
    ap.add_argument("--no-baselines", action="store_true", help="skip the CPU and plain-GPU side measurements")
    ap.add_argument("--ipc-instances", type=int, default=64,
                    help="sphere drapes of the contact measurement (0: skip it)")
    ap.add_argument("--ipc-only", action="store_true", help="run only the contact measurement and print it")
    ap.add_argument("--serve-only", action="store_true", help="run only the served stream and print it")
    ap.add_argument("--serve-gpu-factorization", action="store_true",
                    help="served stream: factorize each set-up on the GPU at cohort start (host threads otherwise)")
    ap.add_argument("--serve-seconds", type=float, default=1.0,
                    help="arrival window of the served-stream measurement (0 skips it)")
    ap.add_argument("--sustain-rate", type=float, default=16.0,
                    help="arrival rate (req/s) of the second served stream, one that one GPU sustains")
    ap.add_argument("--sustain-seconds", type=float, default=10.0, help="its arrival window")
    ap.add_argument("--pin-sweep", default=None,
                    help="after tuning, use this sweep configuration instead of the tuner's choice: "
                         "KIND,WARP_LIMIT,GROUP_LIMIT,BLOCKS_PER_SM,TRIANGLES,HINGES (e.g. grouped,12288,64,4,2,2); "
                         "for profiling runs, where the tuner's timings are distorted")
    ap.add_argument("--refine", type=int, default=None,
                    help="FP64 refinement sweeps of the global solve (default: the solver's default)")
    return ap.parse_args()


def workload(n_instances, rank=0):
    from vistio_b200 import scenarios
    return scenarios.batched_specs(n_instances=n_instances, seed=scenarios.SEED + rank)


def max_over_ranks(x, world, device):
    """The largest of every rank's x (a device-timed duration): the job's time."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_value(instances_per_rank, world, steps, total_ms):
    """Whole-job instance-steps per second: every rank advances its own
    instances (weak scaling), timed by the slowest rank."""
    return instances_per_rank * world * steps / (total_ms / 1e3)


def config_block(n, gpus, refine=None):
    return {"workload": f"batched hanging sheets: {n} instances/GPU, grid side 16-128 (8 topologies), "
                        f"{ITERS} PD iterations, dt=1/60 s",
            "instances_per_gpu": n, "iterations": ITERS, "dt": DT, "parallelism": f"instances sharded, {gpus} GPU",
            "refinement_sweeps": solver_config(refine).refinement_sweeps,
            "l2": "inputs larger than L2 (factor panels alone exceed 126 MB)"}


def cpu_info():
    """The host CPU's model string and the threads this process may use."""
    model = None
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"cpu_model": model, "nproc": os.cpu_count()}


# ------------------------------------------------------------------ clocks
class ClockSampler:
    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"vistio_clocks_{os.getpid()}.csv")

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.fh.close()

    def summary(self):
        try:
            rows = [l.split(",") for l in open(self.path) if l.strip()]
        except Exception:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = float(r[2])
                for k, nm in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(nm)
            except Exception:
                continue
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- oracle CPU
def oracle_sample(specs_sample, steps, threads):
    """Times the oracle's FP32 restatement of the reference step (the
    reference CPU path) on the given instances; returns (seconds, instance-steps)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_api as O
    from vistio_b200 import scenarios
    sims = []
    for s in specs_sample:
        m = scenarios.hanging_sheet(s.side, s.length)
        p = O.init_params(stiffness=s.stretch, bend_stiffness=s.bending, density_gsm=s.density_gsm)
        sims.append(O.OracleSim(m, p, O.default_config(max_iterations=ITERS), precision=0))

    def run(sim):
        for _ in range(steps):
            sim.step(DT)

    t0 = time.perf_counter()
    if threads <= 1:
        for sm in sims:
            run(sm)
    else:
        with cf.ThreadPoolExecutor(threads) as ex:
            list(ex.map(run, sims))
    return time.perf_counter() - t0, len(sims) * steps


def cpu_sample_specs(specs):
    """One instance of each topology (each topology is 1/8 of the instances)."""
    seen, out = set(), []
    for s in specs:
        if s.side not in seen:
            seen.add(s.side)
            out.append(s)
    return out


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    specs = workload(args.instances)
    sample = cpu_sample_specs(specs)
    threads = os.cpu_count() or 1
    # every step is one step of a bounded sample: each topology x (threads // 8 + 1) copies
    copies = max(1, threads // len(sample))
    batch = [s for s in sample for _ in range(copies)]
    for _ in range(args.warmup):
        oracle_sample(batch[: len(sample)], 1, threads)
    secs, units = oracle_sample(batch, args.steps, threads)
    v = units / secs
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * secs / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 Cholesky)", "data": "synthetic",
            "config": config_block(args.instances, args.gpus, args.refine),
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"{len(batch)} instances ({copies} of each of the {len(sample)} topologies) "
                                       f"per step, one instance per host thread"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference is Rust (no toolchain here): its CPU path is timed through the oracle restatement"}
    print(json.dumps(line), flush=True)


# ----------------------------------------------------------- served stream
D_HAT_IPC = 1e-3  # m, a distance: barrier_d_hat = D_HAT_IPC^2, self-contact thickness 1.5 D_HAT_IPC


def apply_pin(batch, tune, pin):
    """Replaces the autotuner's choice by the sweep configuration `pin`
    ("KIND,WARP_LIMIT,GROUP_LIMIT,BLOCKS_PER_SM,TRIANGLES,HINGES"), for
    profiling runs whose tuner timings the profiler distorts."""
    if not pin:
        return tune
    kind, wl, gl, blocks, tri, hin = pin.split(",")
    batch.set_sweep_mode(kind)
    batch.set_warp_limit(int(wl))
    if kind == "grouped":
        batch.set_group_limit(int(gl))
    batch.set_sweep_blocks(int(blocks))
    batch.set_local_shape(int(tri), int(hin))
    return dict(tune, pinned=pin, sweep_mode=kind, sweep_blocks_per_sm=int(blocks))


def ipc_batch(n, steps=10, warmup=5, threads=None, pool=None, pin=None):
    """Batched contact drapes: `n` sphere drapes with the batched workload's grid
    sides and materials, each starting 1 mm above a sphere of radius 0.3 m (so
    the barriers are active from the first step), ground and sphere barriers
    and self-collision, d_hat = 1e-3 m read as a distance (barrier_d_hat =
    1e-6 m^2, self-contact thickness 1.5e-3 m; read as a squared distance, a
    3.2 cm zone on a 1.2-9 cm mesh puts every non-adjacent neighbour in
    contact and the sheets explode), kappa 1e4, AL <= 5, 15 PD iterations per
    AL pass; `steps` step_with_ipc steps timed with CUDA events after
    `warmup`. With a `pool`, the first drape of each grid side is also run by
    the oracle in FP64 over the same warmup + steps steps (the error), and
    stepped alone on the GPU (the plain one-garment-per-launch rate)."""
    from vistio_b200 import api, scenarios
    specs = workload(n, 0)
    dh2 = D_HAT_IPC * D_HAT_IPC
    cfg = api.drape_config(max_iterations=15, al_max_iterations=5, barrier_d_hat=dh2, barrier_kappa=1e4)
    contact = api.Contact(has_ground=True, ground_height=-0.3, has_sphere=True, sphere_center=(0.0, 0.0, 0.0),
                          sphere_radius=0.3, self_collision=True, kappa=1e4, thickness=1.5 * D_HAT_IPC)

    def mesh(sp):
        return scenarios.sphere_drape(side=sp.side, length=1.5, height=0.301)

    def make(sp):
        setup = api.SetupDesc(stiffness=sp.stretch, bend_stiffness=sp.bending, density_gsm=sp.density_gsm)
        return api.ProjectiveDynamicsSolver().init_explicit(mesh(sp), cfg, setup)

    first = {}
    for k, sp in enumerate(specs):
        first.setdefault(sp.side, k)
    refs = {}
    if pool is not None:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_api as O
        oc = O.default_config(max_iterations=15, al_max_iterations=5, barrier_d_hat=dh2)
        c = _oracle_contact(True, -0.3, ((0.0, 0.0, 0.0), 0.3), self_collision=True, kappa=1e4,
                            thickness=1.5 * D_HAT_IPC)
        for side, k in first.items():
            sp = specs[k]
            prm = O.init_params(stiffness=sp.stretch, bend_stiffness=sp.bending, density_gsm=sp.density_gsm)
            for prec in (1, 0):  # FP64, and the reference's FP32 for the spread of the runs
                refs[(k, prec)] = pool.submit(
                    lambda m=mesh(sp), prm=prm, prec=prec: _oracle_run(_oracle(m, prm, oc, prec, ground=-0.3),
                                                                       warmup + steps, DT, c)[1])
    with cf.ThreadPoolExecutor(threads or (os.cpu_count() or 4)) as ex:
        solvers = list(ex.map(make, specs))
    batch = api.Batch(solvers)
    tune = apply_pin(batch, batch.tune(), pin)
    ms = timed_steps(batch, steps, warmup, contact)
    info = batch.info()
    value = n * steps / (ms / 1e3)
    # the dominant kernel is the global solve (75 per step): its roofline, from
    # the autotuner's time of the chosen sweeps on this batch and the
    # algorithmic bytes of the oracle's factors of these meshes
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_api as O
    nnz = {}
    for sp in specs:
        if sp.side not in nnz:
            nnz[sp.side] = O.OracleSim(mesh(sp), O.init_params(), O.default_config()).factor_nnz()
    alg = 2 * (8 * sum(nnz[sp.side] for sp in specs) + 12 * info["vertices"])
    mode = tune["sweep_mode"]
    key = str(tune["group_limit"]) if mode == "grouped" else str(tune["warp_item_limit"])
    sweep_ms = tune["sweep_ms"].get(mode, {}).get(key, -1.0)
    occ_ms = tune["sweep_blocks_ms"].get(str(tune["sweep_blocks_per_sm"]), -1.0)
    if occ_ms > 0 and "pinned" not in tune:  # the chosen compiled form's time (the candidates ran the five-block form)
        sweep_ms = occ_ms
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else None
    peak = peaks["hbm_gbs"] if peaks else 6650.0
    solves = 15 * 5  # PD iterations per AL pass x AL passes (at most; passes end early when converged)
    roofline = {"bound": "hbm", "kernel": "the sweeps of one global solve", "algorithmic_bytes": alg,
                "kernel_ms": sweep_ms, "achieved": alg / (sweep_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                "peak_source": "measured" if peaks else "fallback",
                "solves_per_step_max": solves, "solve_share_of_step_max": min(1.0, solves * sweep_ms / (ms / steps))}
    roofline["frac"] = roofline["achieved"] / peak
    if sweep_ms <= 0:  # a pinned configuration the tuner did not time
        roofline.update(kernel_ms=None, achieved=None, frac=None, solve_share_of_step_max=None)
    out = {"value": value, "unit": UNIT, "instances": n, "steps": steps, "warmup": warmup,
           "ms_per_step": ms / steps, "vertices": info["vertices"], "triangles": info["triangles"],
           "launches_per_step": batch.launches_per_step(), "sweep": tune["sweep_mode"], "sweep_blocks_per_sm": tune["sweep_blocks_per_sm"],
           "autotune": {k: tune[k] for k in ("warp_item_limit", "group_limit", "triangles_per_thread",
                                             "hinges_per_thread", "pinned") if k in tune},
           "roofline": roofline,
           "how": "sphere drapes with ground, sphere and self-contact barriers (IPC, AL <= 5 x 15 iterations, "
                  "d_hat 1 mm as a distance), grid sides and materials of the batched workload, CUDA events over "
                  "the timed steps"}
    if pool is not None:
        errs = {str(specs[k].side): float(np.abs(batch.state(k)[0] - refs[(k, 1)].result()).max())
                for k in first.values()}
        errs32 = {str(specs[k].side): float(np.abs(refs[(k, 0)].result() - refs[(k, 1)].result()).max())
                  for k in first.values()}
        out["error_vs_fp64"] = {"max_m": max(errs.values()), "per_side_m": errs, "steps": warmup + steps,
                                "ref32_max_m": max(errs32.values()), "ref32_per_side_m": errs32,
                                "how": "first drape of each grid side vs the FP64 oracle run of the same steps; "
                                       "ref32: the oracle's restatement of the reference's FP32 step on the same "
                                       "runs (the sheets bounce on the sphere, and rounding differences grow "
                                       "after the first bounce in both)"}
        # plain: the same drapes, one garment per step call
        plain_steps, secs = 3, 0.0
        for k in first.values():
            g = make(specs[k])
            g.step_with_ipc(DT, contact)
            t0 = time.perf_counter()
            for _ in range(plain_steps):
                g.step_with_ipc(DT, contact)
            secs += time.perf_counter() - t0
            g.close()
        plain = len(first) * plain_steps / secs
        out["plain_gpu"] = {"value": plain, "unit": UNIT, "batched_over_plain": value / plain,
                            "how": "the first drape of each grid side stepped alone, one step_with_ipc call per "
                                   "garment-step (each call returns after its step)"}
    batch.close()
    return out


def stream_arrivals(window_s, rate=200.0, seed=20261203):
    """Poisson arrivals at `rate` req/s during `window_s` seconds: half sphere
    drapes, half hanging sheets, grid side log-uniform in [20, 192], materials
    as in the batched workload."""
    rng = np.random.default_rng(seed)
    t, arrivals = 0.0, []
    while True:
        t += rng.exponential(1.0 / rate)
        if t >= window_s:
            break
        side = int(round(math.exp(rng.uniform(math.log(20), math.log(192)))))
        arrivals.append(dict(t=t, sphere=bool(rng.random() < 0.5), side=side,
                             stretch=float(math.exp(rng.uniform(math.log(2e2), math.log(5e3)))),
                             bending=float(math.exp(rng.uniform(math.log(1e-5), math.log(1e-3)))),
                             density=float(rng.uniform(0.08, 0.30) * 1000.0)))
    return arrivals


def _request(a):
    """(mesh, config, set-up, contact or None) of one arrival: sphere drapes at
    the drawn side (IPC d_hat 1e-3, kappa 1e4, AL <= 5, 15 iterations), hanging
    sheets with 10 iterations."""
    from vistio_b200 import api, scenarios
    setup = api.SetupDesc(stiffness=a["stretch"], bend_stiffness=a["bending"], density_gsm=a["density"])
    if a["sphere"]:
        sphere = api.Contact(has_ground=True, ground_height=-0.3, has_sphere=True, sphere_center=(0.0, 0.0, 0.0),
                             sphere_radius=0.3, kappa=1e4)
        cfg = api.drape_config(max_iterations=15, al_max_iterations=5, barrier_d_hat=1e-3, barrier_kappa=1e4)
        return scenarios.sphere_drape(side=a["side"], length=1.5, height=0.5), cfg, setup, sphere
    return scenarios.hanging_sheet(a["side"], 1.0), api.drape_config(max_iterations=ITERS), setup, None


ADMIT_WAIT_MS = 250


def served_stream(window_s, rate=200.0, seed=20261203, threads=None, gpu_factorization=False,
                  admit_wait_ms=ADMIT_WAIT_MS):
    """The served drape stream: the arrivals of stream_arrivals, 300 steps
    each, 120 GB admission budget, cohorts of up to 64 requests formed with an
    admission window of `admit_wait_ms`. Latency runs from a request's arrival
    to its completion."""
    from vistio_b200 import api
    arrivals = stream_arrivals(window_s, rate, seed)
    srv = api.Server(hbm_budget_bytes=120 << 30, max_cohort=64, setup_threads=threads or (os.cpu_count() or 4),
                     steps_per_slice=10, cache_bytes=2 << 30, gpu_factorization=gpu_factorization,
                     admit_wait_ms=admit_wait_ms)
    sym0 = api.symbolic_cache_info()
    t0 = time.perf_counter()
    k = 0
    while k < len(arrivals):
        now = time.perf_counter() - t0
        while k < len(arrivals) and arrivals[k]["t"] <= now:
            m, cfg, setup, contact = _request(arrivals[k])
            if contact is not None:
                srv.submit(m, cfg, setup, 300, DT, contact=contact, ipc=True)
            else:
                srv.submit(m, cfg, setup, 300, DT, pinned=m.pinned)
            k += 1
        srv.tick()
        time.sleep(0.0005)
    srv.drain(3600)
    st = srv.stats()
    srv.close()
    sym1 = api.symbolic_cache_info()
    return {"window_s": window_s, "rate_per_s": rate, "requests": len(arrivals),
            "sphere_requests": sum(a["sphere"] for a in arrivals),
            "completed": st["completed"], "failed": st["failed"],
            "throughput_instance_steps_per_s": st["throughput"],
            "latency_s": {"p50": st["p50_latency_s"], "p99": st["p99_latency_s"], "mean": st["mean_latency_s"]},
            "max_cohorts_active": st["max_cohorts_active"], "peak_device_bytes": st["max_bytes_in_use"],
            "setup_cache": {"hits": st["cache_hits"], "misses": st["cache_misses"]},
            "factorization": "GPU (cohort start)" if gpu_factorization else "host (set-up threads)",
            "symbolic_cache": {"hits": sym1["hits"] - sym0["hits"], "misses": sym1["misses"] - sym0["misses"]},
            "admit_wait_ms": admit_wait_ms, "cohorts_started": st["cohorts_started"],
            "how": "Poisson arrivals at the stated rate during the window, then drained; each request 300 steps"}


def batched_same_mix(window_s, rate=200.0, seed=20261203, threads=None):
    """The served stream's requests run offline as two batches (the sphere
    drapes, the hanging sheets), all present from the start, 300 steps each:
    the batched rate on the same mix, device-timed with CUDA events."""
    import torch
    from vistio_b200 import api
    arrivals = stream_arrivals(window_s, rate, seed)
    total_ms, units = 0.0, 0
    for sphere in (True, False):
        reqs = [_request(a) for a in arrivals if a["sphere"] == sphere]
        if not reqs:
            continue

        def make(r):
            m, cfg, setup, _ = r
            return api.ProjectiveDynamicsSolver().init_explicit(m, cfg, setup,
                                                                pinned=None if sphere else m.pinned)

        with cf.ThreadPoolExecutor(threads or (os.cpu_count() or 4)) as ex:
            solvers = list(ex.map(make, reqs))
        batch = api.Batch(solvers)
        batch.tune()
        contact = reqs[0][3]
        batch.step(DT, 1, contact=contact)
        torch.cuda.synchronize()
        stream = torch.cuda.ExternalStream(batch.stream())
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            e0.record(stream)
            batch.step(DT, 299, contact=contact)
            e1.record(stream)
        torch.cuda.synchronize()
        total_ms += e0.elapsed_time(e1) * 300.0 / 299.0
        units += 300 * len(reqs)
        batch.close()
        for sv in solvers:
            sv.close()
    return {"value": units / (total_ms / 1e3), "unit": UNIT, "requests": len(arrivals),
            "how": "the same requests as two batches (sphere drapes with IPC, hanging sheets), 300 steps each, "
                   "one batch after the other, CUDA events"}


# ------------------------------------------------- single-garment configs
def _oracle(mesh, params, cfg, precision, ground=None):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_api as O
    sim = O.OracleSim(mesh, params, cfg, precision=precision)
    if ground is not None:
        sim.set_ground(1, ground)
    return sim


def _oracle_contact(has_ground=False, ground=0.0, sphere=None, self_collision=False, kappa=0.0, thickness=0.0):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_api as O
    c = O.Contact()
    c.has_ground, c.ground_height = int(has_ground), ground
    if sphere is not None:
        c.has_sphere = 1
        c.sphere_center[:] = sphere[0]
        c.sphere_radius = sphere[1]
    c.self_collision, c.bvh_faithful = int(self_collision), 0
    c.kappa, c.thickness = kappa, thickness
    return c


def _oracle_run(sim, steps, dt, contact=None, keep=False):
    out = []
    t0 = time.perf_counter()
    for _ in range(steps):
        if contact is None:
            sim.step(dt)
        else:
            sim.step_ipc(dt, contact)
        if keep:
            out.append(sim.state()[0])
    return time.perf_counter() - t0, (out if keep else sim.state()[0])


def _gpu_run(make, steps, dt, contact=None, keep=False, warmup=3):
    """One garment stepped alone, one step per call (each call returns after
    its step); a separate instance takes the warm-up steps."""
    w = make()
    for _ in range(warmup):
        (w.step(dt) if contact is None else w.step_with_ipc(dt, contact))
    w.close()
    g = make()
    traj = []
    t0 = time.perf_counter()
    for _ in range(steps):
        (g.step(dt) if contact is None else g.step_with_ipc(dt, contact))
        if keep:
            traj.append(g.state()[0])
    secs = time.perf_counter() - t0
    return secs, (traj if keep else g.state()[0])


def single_configs(pool):
    """The three single-garment configurations, each stepped alone on the GPU
    (one step per call, host wall clock around the synchronous calls), with
    its error against the oracle's FP64 run:
      hanging_sheet  20x20, 120 steps, plain PD, 10 iterations;
      sphere_drape   64x64, 180 steps, IPC (d_hat 1e-3, kappa 1e4, AL <= 5, 15 iterations);
      self_fold      40x400 dropped from 0.5 m, 300 steps at dt 1/120, ground and self contact,
                     d_hat 5e-4 m as a distance, matrix dt 1/120 (FP64 checkpoints from the
                     committed fixture tests/golden/self_fold_drop.npz)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_api as O
    from vistio_b200 import api, scenarios
    out = {}
    setup = api.SetupDesc(stiffness=1e3, bend_stiffness=1e-4, density_gsm=150.0)
    prm = O.init_params(stiffness=1e3, bend_stiffness=1e-4, density_gsm=150.0)

    m0 = scenarios.hanging_sheet(20, 1.0)
    cfg0 = api.drape_config(max_iterations=ITERS)
    ref0 = pool.submit(lambda: _oracle_run(_oracle(m0, prm, O.default_config(max_iterations=ITERS), 1), 120, DT))
    secs, p = _gpu_run(lambda: api.ProjectiveDynamicsSolver().init_explicit(m0, cfg0, setup, pinned=m0.pinned),
                       120, DT)
    out["hanging_sheet"] = {"gpu": {"value": 120 / secs, "unit": "steps/s", "ms_per_step": 1e3 * secs / 120,
                                    "steps": 120},
                            "error_vs_fp64_m": float(np.abs(p - ref0.result()[1]).max())}

    m1 = scenarios.sphere_drape(side=64, length=1.5, height=0.5)
    cfg1 = api.drape_config(max_iterations=15, al_max_iterations=5, barrier_d_hat=1e-3, barrier_kappa=1e4)
    sph = api.Contact(has_ground=True, ground_height=-0.3, has_sphere=True, sphere_center=(0.0, 0.0, 0.0),
                      sphere_radius=0.3, kappa=1e4)
    oc1 = O.default_config(max_iterations=15, al_max_iterations=5, barrier_d_hat=1e-3)
    c1 = _oracle_contact(True, -0.3, ((0.0, 0.0, 0.0), 0.3), kappa=1e4)
    ref1 = {pr: pool.submit(lambda pr=pr: _oracle_run(_oracle(m1, prm, oc1, pr, ground=-0.3), 180, DT, c1, True))
            for pr in (1, 0)}
    secs, traj = _gpu_run(lambda: api.ProjectiveDynamicsSolver().init_explicit(m1, cfg1, setup), 180, DT, sph,
                          keep=True)
    t64, t32 = ref1[1].result()[1], ref1[0].result()[1]
    e_gpu = [float(np.abs(a - b).max()) for a, b in zip(traj, t64)]
    e_32 = [float(np.abs(a - b).max()) for a, b in zip(t32, t64)]

    def first_above(e, thr):
        idx = [k for k, v in enumerate(e) if v > thr]
        return idx[0] + 1 if idx else None

    out["sphere_drape"] = {"gpu": {"value": 180 / secs, "unit": "steps/s", "ms_per_step": 1e3 * secs / 180,
                                   "steps": 180},
                           "error_vs_fp64_m": e_gpu[-1], "ref32_error_vs_fp64_m": e_32[-1],
                           "first_step_above_1e-4_m": {"gpu": first_above(e_gpu, 1e-4),
                                                       "ref32": first_above(e_32, 1e-4)},
                           "note": "the sheet bounces on the sphere: rounding differences grow about tenfold per "
                                   "ten steps after the first bounce, for the reference's FP32 as for the GPU"}

    fx = np.load(os.path.join(ROOT, "tests", "golden", "self_fold_drop.npz"))
    dt2, d_hat = 1.0 / 120.0, 5e-4
    m2 = scenarios.self_fold(40, 400, 0.2, 2.0, lowest=0.5)
    setup2 = api.SetupDesc(model=api.MODEL_ORTHOTROPIC, stiffness=1e3, warp_stiffness=1e3, weft_stiffness=6e2,
                           bend_stiffness=1e-4, density_gsm=150.0, matrix_dt=dt2)
    cfg2 = api.drape_config(max_iterations=10, al_max_iterations=5, barrier_d_hat=d_hat * d_hat, barrier_kappa=0.0)
    con2 = api.Contact(has_ground=True, ground_height=0.0, self_collision=True, kappa=0.0, thickness=1.5 * d_hat)
    secs, p = _gpu_run(lambda: api.ProjectiveDynamicsSolver().init_explicit(m2, cfg2, setup2), 300, dt2, con2)
    out["self_fold"] = {"gpu": {"value": 300 / secs, "unit": "steps/s", "ms_per_step": 1e3 * secs / 300,
                                "steps": 300},
                        "error_vs_fp64_m": float(np.abs(p - fx["pos_300"]).max()),
                        "ref32_error_vs_fp64_m": float(fx["ref32_spread"][-1])}
    return out


def single_configs_cpu():
    """The reference CPU path (oracle ref32, one core) on bounded samples of
    the three single-garment configurations; steps/s."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_api as O
    from vistio_b200 import scenarios
    prm = O.init_params(stiffness=1e3, bend_stiffness=1e-4, density_gsm=150.0)
    res = {}
    m0 = scenarios.hanging_sheet(20, 1.0)
    secs, _ = _oracle_run(_oracle(m0, prm, O.default_config(max_iterations=ITERS), 0), 120, DT)
    res["hanging_sheet"] = {"value": 120 / secs, "unit": "steps/s", "cores": 1, "kind": "port",
                            "sample": "all 120 steps"}
    m1 = scenarios.sphere_drape(side=64, length=1.5, height=0.5)
    oc1 = O.default_config(max_iterations=15, al_max_iterations=5, barrier_d_hat=1e-3)
    c1 = _oracle_contact(True, -0.3, ((0.0, 0.0, 0.0), 0.3), kappa=1e4)
    secs, _ = _oracle_run(_oracle(m1, prm, oc1, 0, ground=-0.3), 60, DT, c1)
    res["sphere_drape"] = {"value": 60 / secs, "unit": "steps/s", "cores": 1, "kind": "port",
                           "sample": "the first 60 of the 180 steps"}
    dt2, d_hat = 1.0 / 120.0, 5e-4
    m2 = scenarios.self_fold(40, 400, 0.2, 2.0, lowest=0.5)
    p2 = O.init_params(model=O.MODEL_ORTHO, stiffness=1e3, warp=1e3, weft=6e2, bend_stiffness=1e-4,
                       density_gsm=150.0, matrix_dt=dt2)
    oc2 = O.default_config(max_iterations=10, al_max_iterations=5, barrier_d_hat=d_hat * d_hat)
    sim = _oracle(m2, p2, oc2, 0, ground=0.0)
    kappa = float(O.lib().orc_estimate_kappa(0.0, float(sim.masses().mean()), 9.81, d_hat * d_hat))
    c2 = _oracle_contact(True, 0.0, self_collision=True, kappa=kappa, thickness=1.5 * d_hat)
    secs, _ = _oracle_run(sim, 15, dt2, c2)
    res["self_fold"] = {"value": 15 / secs, "unit": "steps/s", "cores": 1, "kind": "port",
                        "sample": "the first 15 of the 300 steps"}
    return res


# ------------------------------------------------------------------- our arm
def solver_config(refine):
    from vistio_b200 import api
    kw = {} if refine is None else {"refinement_sweeps": refine}
    return api.drape_config(max_iterations=ITERS, **kw)


def batch_order(specs):
    """Instances in the batch's grid order: big garments first."""
    return sorted(range(len(specs)), key=lambda k: -specs[k].side)


def build_batch(specs, threads, refine, order):
    from vistio_b200 import api, scenarios
    cfg = solver_config(refine)
    ctx = api.default_context()

    def make(s):
        m = scenarios.hanging_sheet(s.side, s.length)
        setup = api.SetupDesc(stiffness=s.stretch, bend_stiffness=s.bending, density_gsm=s.density_gsm)
        return api.ProjectiveDynamicsSolver(ctx).init_explicit(m, cfg, setup, pinned=m.pinned)

    with cf.ThreadPoolExecutor(threads) as ex:
        solvers = list(ex.map(make, [specs[k] for k in order]))
    return api.Batch(solvers), solvers


def first_of_each_topology(specs, order):
    """Batch index of the first instance of each grid side."""
    first = {}
    for k, idx in enumerate(order):
        first.setdefault(specs[idx].side, k)
    return sorted(first.values())


def fp64_runs(specs, order, nsteps, pool, precision=1):
    """Starts the oracle's runs (precision 1: FP64; 0: the reference's FP32
    arithmetic) of the first instance of each topology over nsteps steps on
    `pool`; returns {batch index: future of positions}."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_api as O
    from vistio_b200 import scenarios

    def run(k):
        s = specs[order[k]]
        m = scenarios.hanging_sheet(s.side, s.length)
        p = O.init_params(stiffness=s.stretch, bend_stiffness=s.bending, density_gsm=s.density_gsm)
        sim = O.OracleSim(m, p, O.default_config(max_iterations=ITERS), precision=precision)
        for _ in range(nsteps):
            sim.step(DT)
        return sim.state()[0]

    return {k: pool.submit(run, k) for k in first_of_each_topology(specs, order)}


def fp64_error(specs, order, states, refs, nsteps, refs32=None):
    """Max |x_gpu - x_fp64| (m) after nsteps steps on the first instance of
    each topology (states: batch index -> GPU positions); with refs32, also
    the reference FP32 restatement's own distance from FP64."""
    res = [(specs[order[k]].side, float(np.abs(states[k] - refs[k].result()).max())) for k in sorted(states)]
    out = {"max_m": max(e for _, e in res), "per_side_m": {str(side): e for side, e in res}, "steps": nsteps,
           "how": "first instance of each topology vs the FP64 oracle run of the same steps"}
    if refs32 is not None:
        out["ref32_max_m"] = max(float(np.abs(refs32[k].result() - refs[k].result()).max()) for k in refs)
    return out


def timed_steps(batch, steps, warmup, contact=None):
    """Device time (ms) of `steps` batch steps after `warmup`, CUDA events on the batch stream."""
    import torch
    for _ in range(warmup):
        batch.step(DT, 1, contact=contact)
    torch.cuda.synchronize()
    stream = torch.cuda.ExternalStream(batch.stream())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        batch.step(DT, steps, contact=contact)
        e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def oracle_nnz_by_side(specs):
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_api as O
    from vistio_b200 import scenarios
    out = {}
    for s in cpu_sample_specs(specs):
        m = scenarios.hanging_sheet(s.side, 1.0)
        out[s.side] = O.OracleSim(m, O.init_params(), O.default_config()).factor_nnz()
    return out


def main():
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
        return
    import torch
    import torch.distributed as dist

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from vistio_b200 import api
    api._default_ctx = api.Context(local)
    if args.ipc_only:
        if rank == 0:
            print(json.dumps({"ipc": ipc_batch(args.ipc_instances, args.steps, args.warmup, pin=args.pin_sweep)}),
                  flush=True)
        if world > 1:
            dist.destroy_process_group()
        return
    if args.serve_only:
        if rank == 0:
            srv = served_stream(args.serve_seconds, gpu_factorization=args.serve_gpu_factorization)
            srv["batched_same_mix"] = batched_same_mix(args.serve_seconds)
            srv["served_over_batched_same_mix"] = srv["throughput_instance_steps_per_s"] / srv["batched_same_mix"]["value"]
            print(json.dumps({"serving": srv}), flush=True)
        if world > 1:
            dist.destroy_process_group()
        return

    threads = max(1, (os.cpu_count() or 1) // max(1, world))
    specs = workload(args.instances, rank)
    order = batch_order(specs)
    e2e_steps = max(3, min(args.steps, 10))
    err_steps = max(ERR_STEPS, args.warmup + args.steps + e2e_steps)
    # the oracle's FP64 runs that the measured batch is checked against run on
    # the host beside the GPU work (rank 0, full runs only)
    pool = cf.ThreadPoolExecutor(max(1, os.cpu_count() or 1)) if rank == 0 and not args.no_baselines else None
    refs = fp64_runs(specs, order, err_steps, pool) if pool else None
    refs32 = fp64_runs(specs, order, err_steps, pool, precision=0) if pool else None
    from vistio_b200 import api as _api
    sym0 = _api.symbolic_cache_info()
    t0 = time.time()
    batch, solvers = build_batch(specs, threads, args.refine, order)
    setup_s = time.time() - t0
    sym1 = _api.symbolic_cache_info()
    symbolic = {"hits": sym1["hits"] - sym0["hits"], "misses": sym1["misses"] - sym0["misses"],
                "host_threads": threads}
    tune = apply_pin(batch, batch.tune(), args.pin_sweep)  # level schedule picked by timing this batch's sweeps
    info = batch.info()
    V = info["vertices"]
    stream = torch.cuda.ExternalStream(batch.stream())

    def barrier():
        if world > 1:
            dist.barrier(device_ids=[local])

    device = f"cuda:{local}"

    for _ in range(args.warmup):
        batch.step(DT, 1)
    torch.cuda.synchronize()
    launches_per_step = batch.launches_per_step()

    # ---- device-timed region: K steps, per-step events on the batch stream
    evs = [torch.cuda.Event(enable_timing=True) for _ in range(args.steps + 1)]
    barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        with torch.cuda.stream(stream):
            evs[0].record(stream)
            for k in range(args.steps):
                batch.step(DT, 1)
                evs[k + 1].record(stream)
        torch.cuda.synchronize()
    barrier()
    step_ms = [evs[k].elapsed_time(evs[k + 1]) for k in range(args.steps)]
    total_ms = max_over_ranks(evs[0].elapsed_time(evs[-1]), world, device)
    value = job_value(len(specs), world, args.steps, total_ms)
    clocks = clk.summary()

    # ---- end to end: positions from pinned host memory in, positions back out, each step
    # two pinned buffers: each step uploads the positions the previous step downloaded
    host = [torch.empty((V, 3), dtype=torch.float32, pin_memory=True).numpy() for _ in range(2)]
    batch.download_positions(host[0])
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        e0.record(stream)
        for k in range(e2e_steps):
            batch.upload_positions(host[k % 2])
            batch.step(DT, 1)
            batch.download_positions(host[(k + 1) % 2])
        e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    e2e_ms = max_over_ranks(e0.elapsed_time(e1), world, device)
    e2e_value = job_value(len(specs), world, e2e_steps, e2e_ms)

    # ---- per-kernel timing of one plain iteration's phases (live, CUDA events)
    phases = ["membrane", "bending", "gather", "solve"]
    reps = 5
    kern_ms = {}
    with torch.cuda.stream(stream):
        for ph in phases:
            tot = 0.0
            for _ in range(reps):
                if ph == "solve":
                    batch.launch_phase("gather")  # a fresh residual for the sweep
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                batch.launch_phase(ph)
                b.record(stream)
                b.synchronize()
                tot += a.elapsed_time(b)
            kern_ms[ph] = tot / reps
    torch.cuda.synchronize()
    dom = max(kern_ms, key=kern_ms.get)

    # algorithmic bytes per launch: per-unit figures (V vertices, T triangles, H hinges,
    # nnz(L) of the oracle's ordering) times the units of the launch
    nnz_ref = oracle_nnz_by_side(specs)
    nnz_total = sum(nnz_ref[s.side] for s in specs)
    T, H = info["triangles"], info["hinges"]
    alg = {"solve": 2 * (8 * nnz_total + 12 * V), "membrane": 32 * T + 12 * V + 36 * T,
           "bending": 40 * H + 12 * H, "gather": 12 * V * 3 + 36 * T + 12 * H}
    peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json"))) if os.path.exists(
        os.path.join(ROOT, "MEASURED_PEAKS.json")) else None
    peak = peaks["hbm_gbs"] if peaks else 6650.0  # fallback: an earlier copy-bandwidth measurement
    achieved = alg[dom] / (kern_ms[dom] * 1e-3) / 1e9
    solve_kernels = {"dataflow": "k_red_reset + k_sweep + k_update",
                     "grouped": "k_red_reset + k_gsweep<0> + k_sweep + k_gsweep<1> + k_update",
                     "levels": "k_red_reset + k_subtree<0> + k_level<0> x L + k_level<1> x L + k_subtree<1> + k_update"
                     }[batch.sweep_mode()[0]]
    roofline = {"bound": "hbm", "kernel": {"solve": solve_kernels, "membrane": "k_tri", "bending": "k_hinge",
                                          "gather": "k_gather"}[dom],
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": "measured" if peaks else "fallback",
                "traffic": None, "kernel_ms": kern_ms[dom],
                "phase_ms": kern_ms, "algorithmic_bytes": alg[dom],
                "kernel_declared_bytes": batch.phase_bytes(dom)}
    prof = os.path.join(ROOT, "profiles", "k_solve_traffic.json")
    if os.path.exists(prof):
        try:
            tr = json.load(open(prof))
            if dom == "solve" and tr.get("bytes_per_vertex"):
                roofline["traffic"] = tr["bytes_per_vertex"] * V
                roofline["traffic_source"] = tr.get("source")
        except Exception:
            pass

    out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 factorization)", "data": "synthetic",
           "config": dict(config_block(len(specs), world, args.refine), autotune=tune),
           "latency_ms": {"p50": float(np.percentile(step_ms, 50)), "p99": float(np.percentile(step_ms, 99))},
           "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": 12 * V * world,
                   "d2h_bytes_per_step": 12 * V * world, "steps": e2e_steps},
           "gpu_launches": launches_per_step * args.steps, "launches_per_step": launches_per_step,
           "clocks": clocks, "roofline": roofline,
           "batch": {"vertices": V, "triangles": T, "hinges": H, "factor_bytes": info["factor_bytes"],
                     "setup_s": setup_s, "symbolic_cache": symbolic,
                     "factorization": dict(batch.factor_stats(), where="GPU, multifrontal FP64, every garment")}}

    if pool is not None:
        # accuracy of the measured run, taken to ERR_STEPS steps: the metric is
        # quoted at <= 1e-4 m against FP64
        done = args.warmup + args.steps + e2e_steps
        if done < err_steps:
            batch.step(DT, err_steps - done)
        states = {k: batch.state(k)[0] for k in refs}
        batch.close()
        # the FP32+FP64-refined solver (one refinement sweep per solve) on the same workload
        batch2, _ = build_batch(specs, threads, 1, order)
        tune2 = batch2.tune()
        ms2 = timed_steps(batch2, args.steps, args.warmup)
        batch2.step(DT, err_steps - args.warmup - args.steps)
        states2 = {k: batch2.state(k)[0] for k in refs}
        batch2.close()
        out["error_vs_fp64"] = fp64_error(specs, order, states, refs, err_steps, refs32)
        v2 = job_value(len(specs), 1, args.steps, ms2)
        out["refined"] = {"refinement_sweeps": 1, "value": v2, "unit": UNIT, "ms_per_step": ms2 / args.steps,
                          "over_default": v2 / value, "sweep_mode": tune2["sweep_mode"],
                          "error_vs_fp64": fp64_error(specs, order, states2, refs, err_steps),
                          "how": "the same workload with one FP64-residual refinement sweep after the last "
                                 "iteration's solve of every step, CUDA events over the same K steps"}

        # plain one-instance-per-launch GPU PD on one instance of each topology
        from vistio_b200 import api, scenarios
        sample = cpu_sample_specs(specs)
        cfg = solver_config(args.refine)
        plain = []
        for s in sample:
            m = scenarios.hanging_sheet(s.side, s.length)
            setup = api.SetupDesc(stiffness=s.stretch, bend_stiffness=s.bending, density_gsm=s.density_gsm)
            plain.append(api.ProjectiveDynamicsSolver().init_explicit(m, cfg, setup, pinned=m.pinned))
        for p in plain:
            p.step(DT)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        psteps = 5
        for _ in range(psteps):
            for p in plain:
                p.step(DT)
        torch.cuda.synchronize()
        plain_v = len(plain) * psteps / (time.perf_counter() - t0)
        for p in plain:
            p.close()
        # the host's numeric FP64 factorization of the same garments, one thread,
        # for comparison with the batch's device factorization above
        host_ms = 0.0
        for s in sample:
            m = scenarios.hanging_sheet(s.side, s.length)
            setup = api.SetupDesc(stiffness=s.stretch, bend_stiffness=s.bending, density_gsm=s.density_gsm)
            t = []
            for host in (True, False):
                c = dataclasses.replace(cfg, host_factorization=host)
                t1 = time.perf_counter()
                api.ProjectiveDynamicsSolver().init_explicit(m, c, setup, pinned=m.pinned).close()
                t.append(time.perf_counter() - t1)
            host_ms += 1e3 * max(0.0, t[0] - t[1]) * len(specs) / len(sample)
        out["batch"]["factorization"]["host_1thread_ms_est"] = host_ms
        out["plain_gpu"] = {"value": plain_v, "unit": UNIT,
                            "how": "each instance stepped alone (one graph launch per instance-step, result read "
                                   "back each step), one instance of each topology",
                            "batched_over_plain": value / world / plain_v,
                            "e2e_batched_over_plain": e2e_value / world / plain_v}
        if args.ipc_instances > 0:
            out["ipc"] = ipc_batch(args.ipc_instances, pool=pool)
        out["configs"] = single_configs(pool)
        pool.shutdown(wait=True)
        # CPU baselines, timed with no other host work running: the oracle's
        # FP32 restatement, single thread
        cpu_steps = 30
        secs, units = oracle_sample(sample, cpu_steps, 1)
        out["cpu_baseline"] = dict(
            {"value": units / secs, "unit": UNIT, "cores": 1, "kind": "port",
             "sample": f"one instance of each of the {len(sample)} topologies x {cpu_steps} steps "
                       f"({secs:.1f} s); each topology is 1/8 of the workload"}, **cpu_info())
        for name, cpu in single_configs_cpu().items():
            out["configs"][name]["cpu_ref32"] = cpu
            out["configs"][name]["gpu_over_cpu"] = out["configs"][name]["gpu"]["value"] / cpu["value"]
        if args.serve_seconds > 0:
            out["serving"] = served_stream(args.serve_seconds, gpu_factorization=args.serve_gpu_factorization)
            mix = batched_same_mix(args.serve_seconds)
            out["serving"]["batched_same_mix"] = mix
            out["serving"]["served_over_batched_same_mix"] = \
                out["serving"]["throughput_instance_steps_per_s"] / mix["value"]
            # a stream at a rate one GPU sustains, beside the specified burst
            out["serving_sustained"] = served_stream(args.sustain_seconds, rate=args.sustain_rate, seed=20261204,
                                                     gpu_factorization=args.serve_gpu_factorization)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
