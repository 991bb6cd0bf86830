"""GPU parity of the plain PD step (SolverStrategy::step) against the oracle.

Tolerances (positions, metres; the sheet spans about 1 m):
* one step from an identical state: relative L2 error <= 1e-5 against the
  FP64 oracle and against the FP32 reference restatement;
* a full 120-step hanging_sheet run: max |x_gpu - x_fp64| <= 1e-4 m.
"""
import numpy as np
import pytest

import oracle_api as O
from vistio_b200 import api, scenarios

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


def sheet_pair(side=20, length=1.0, stiffness=1e3, bend=1e-4, density=150.0, iters=10, model=0, bending=1,
               warp=0.0, weft=0.0, bend_warp=0.0, bend_weft=0.0, precision=1, refine=0):
    mesh = scenarios.hanging_sheet(side, length)
    cfg = api.drape_config(max_iterations=iters, refinement_sweeps=refine)
    setup = api.SetupDesc(model=model, bending=bending, stiffness=stiffness, bend_stiffness=bend, density_gsm=density,
                          warp_stiffness=warp, weft_stiffness=weft, bend_warp=bend_warp, bend_weft=bend_weft)
    gpu = api.ProjectiveDynamicsSolver().init_explicit(mesh, cfg, setup, pinned=mesh.pinned)
    p = O.init_params(stiffness=stiffness, bend_stiffness=bend, density_gsm=density, model=model, bending=bending,
                      warp=warp, weft=weft, bend_warp=bend_warp, bend_weft=bend_weft)
    ref = O.OracleSim(mesh, p, O.default_config(max_iterations=iters), precision=precision)
    return mesh, gpu, ref


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_lumped_masses_match_oracle():
    """compute_lumped_masses (pd_solver.rs:1219-1242) in f32: bit-identical."""
    mesh, gpu, ref = sheet_pair(precision=0)
    assert np.array_equal(gpu.lumped_masses(), ref.masses())


def test_one_step_from_rest_matches_fp64_and_ref32():
    mesh, gpu, ref64 = sheet_pair(precision=1)
    _, _, ref32 = sheet_pair(precision=0)
    r = gpu.step(DT)
    ref64.step(DT)
    ref32.step(DT)
    pg, vg = gpu.state()
    p64, v64 = ref64.state()
    p32, _ = ref32.state()
    assert r.iterations == 10
    assert rel(pg, p64) <= 1e-5, rel(pg, p64)
    assert rel(pg, p32) <= 1e-5, rel(pg, p32)
    assert np.abs(vg - v64).max() <= 1e-3  # velocities = dx / dt
    # pinned vertices stay where they are (solver_tests.rs:419-450)
    pin = mesh.pinned.astype(bool)
    x0 = np.stack([mesh.px, mesh.py, mesh.pz], 1)
    assert np.abs(pg[pin] - x0[pin]).max() <= 1e-6


def test_per_step_parity_along_a_trajectory():
    """At checkpoints of an oracle trajectory, one GPU step from the oracle's
    state stays within 1e-5 relative of the oracle's next state."""
    mesh, gpu, ref = sheet_pair(precision=1)
    worst = 0.0
    for s in range(60):
        if s % 10 == 5:
            p, v = ref.state()
            gpu.set_state(p, v)
            ref.step(DT)
            gpu.step(DT)
            worst = max(worst, rel(gpu.state()[0], ref.state()[0]))
        else:
            ref.step(DT)
    assert worst <= 1e-5, worst


@pytest.mark.parametrize("refine", [0, 1, 2])
def test_full_hanging_sheet_run_within_1e4_m_of_fp64(refine):
    """hanging_sheet, 120 steps, 10 iterations: the GPU run stays within 1e-4 m
    of the FP64 run; gravity lowers the centroid (solver_tests.rs:453-483).
    Also with 1 and 2 FP64 refinement sweeps of the last solve of each step."""
    mesh, gpu, ref = sheet_pair(precision=1, refine=refine)
    for _ in range(120):
        gpu.step(DT)
        ref.step(DT)
    pg, _ = gpu.state()
    pr, _ = ref.state()
    err = float(np.abs(pg - pr).max())
    print(f"120-step hanging_sheet, refinement {refine}: max |x_gpu - x_fp64| = {err:.3e} m")
    assert err <= 1e-4, err
    assert pg[:, 1].mean() < mesh.py.mean() - 0.1


@pytest.mark.parametrize("model,bending,warp,weft", [
    (api.MODEL_COROTATIONAL, api.BENDING_DIHEDRAL, 0.0, 0.0),
    (api.MODEL_ORTHOTROPIC, api.BENDING_DISCRETE_SHELLS, 1e3, 6e2),
    (api.MODEL_ANISOTROPIC, api.BENDING_DISCRETE_SHELLS_ANISOTROPIC, 0.8, 0.3),
    (api.MODEL_ISOTROPIC_LINEAR, api.BENDING_DISCRETE_SHELLS, 0.0, 0.0),
    (api.MODEL_ARAP, api.BENDING_NONE, 0.0, 0.0),
])
def test_material_models_one_step(model, bending, warp, weft):
    mesh, gpu, ref = sheet_pair(side=16, length=0.8, model=model, bending=bending, warp=warp, weft=weft,
                                bend_warp=0.02, bend_weft=0.01)
    for _ in range(3):
        p, v = ref.state()
        gpu.set_state(p, v)
        ref.step(DT)
        gpu.step(DT)
        assert rel(gpu.state()[0], ref.state()[0]) <= 1e-5


def test_batch_equals_individual_solvers_bitwise():
    """Instances advanced together in one ragged batch give exactly the
    results they give alone."""
    specs = [(12, 0.7, 400.0, 2e-5, 90.0), (20, 1.3, 3000.0, 5e-4, 250.0), (9, 0.5, 900.0, 1e-4, 150.0)]
    cfg = api.drape_config(max_iterations=10)
    solo, grouped = [], []
    for side, length, k, kb, rho in specs:
        mesh = scenarios.hanging_sheet(side, length)
        setup = api.SetupDesc(stiffness=k, bend_stiffness=kb, density_gsm=rho)
        solo.append(api.ProjectiveDynamicsSolver().init_explicit(mesh, cfg, setup, pinned=mesh.pinned))
        grouped.append(api.ProjectiveDynamicsSolver().init_explicit(mesh, cfg, setup, pinned=mesh.pinned))
    batch = api.Batch(grouped)
    batch.step(DT, 5)
    for k, s in enumerate(solo):
        for _ in range(5):
            s.step(DT)
        assert np.array_equal(s.state()[0], batch.state(k)[0])


def test_batch_whole_position_copies():
    """download_positions returns every instance's positions in instance
    order; upload_positions writes them back exactly (velocities untouched)."""
    cfg = api.drape_config(max_iterations=4)
    solvers = []
    for side, length in [(7, 0.4), (13, 0.9), (4, 0.3)]:
        mesh = scenarios.hanging_sheet(side, length)
        solvers.append(api.ProjectiveDynamicsSolver().init(mesh, cfg, pinned=mesh.pinned))
    batch = api.Batch(solvers)
    batch.step(DT, 3)
    allpos = batch.download_positions()
    parts = [batch.state(k)[0] for k in range(3)]
    assert np.array_equal(allpos, np.concatenate(parts))
    vel_before = [batch.state(k)[1] for k in range(3)]
    moved = (allpos + np.float32(0.25)).astype(np.float32)
    batch.upload_positions(moved)
    for k in range(3):
        off = sum(len(p) for p in parts[:k])
        assert np.array_equal(batch.state(k)[0], moved[off: off + len(parts[k])])
        assert np.array_equal(batch.state(k)[1], vel_before[k])


def test_sparse_solver_reference_cases():
    """The reference's FaerSolver tests (math_tests.rs:115-273) through the
    SparseSolver mirror."""
    s = api.SparseSolver()
    assert not s.is_factorized()
    s.factorize([0, 1, 2, 3], [0, 1, 2], [1.0, 1.0, 1.0], 3)
    assert s.is_factorized()
    assert np.abs(s.solve([3.0, 7.0, -2.0]) - [3.0, 7.0, -2.0]).max() < 1e-5
    s = api.SparseSolver()
    s.factorize([0, 2, 5, 7], [0, 1, 0, 1, 2, 1, 2], [4, 1, 1, 3, 1, 1, 2], 3)
    x = s.solve([1.0, 2.0, 3.0])
    A = np.array([[4, 1, 0], [1, 3, 1], [0, 1, 2]], np.float64)
    assert np.abs(A @ x - [1, 2, 3]).max() < 1e-4
    s = api.SparseSolver()
    s.factorize([0, 1, 2, 3], [0, 1, 2], [2.0, 3.0, 5.0], 3)
    assert np.abs(s.solve([4.0, 9.0, 25.0]) - [2, 3, 5]).max() < 1e-5
    assert np.abs(s.solve([1.0, 1.0, 1.0]) - [0.5, 1 / 3, 0.2]).max() < 1e-5
    n = 100
    rows, cols, vals = [], [], []
    for i in range(n):
        for j, v in ((i - 1, -1.0), (i, 2.1), (i + 1, -1.0)):
            if 0 <= j < n:
                rows.append(i); cols.append(j); vals.append(v)
    rp = np.searchsorted(rows, np.arange(n + 1))
    s = api.SparseSolver()
    s.factorize(rp, cols, vals, n)
    x = s.solve(np.ones(n))
    A = np.zeros((n, n))
    A[rows, cols] = vals
    assert np.abs(A @ x - 1.0).max() < 1e-3
    with pytest.raises(Exception):
        api.SparseSolver().solve([1.0])


def test_not_spd_is_reported():
    s = api.SparseSolver()
    with pytest.raises(api.L.VistioError) as e:
        s.factorize([0, 1, 2], [0, 1], [1.0, -1.0], 2)
    assert e.value.status == 11


def test_bounded_device_wait_reports_timeout_and_context_survives():
    """A device wait that nothing completes ends with VISTIO_ERR_TIMEOUT after
    its poll limit (no hang, no fault), and the same context steps normally
    afterwards."""
    from vistio_b200 import _lib
    ctx = api.default_context()
    st = _lib.lib().vistio_diag_wait_timeout(ctx.h, 1 << 12)
    assert st == 9, st  # VISTIO_ERR_TIMEOUT
    assert b"gave up" in _lib.lib().vistio_last_error(ctx.h)
    mesh, gpu, ref = sheet_pair(side=8, length=0.5)
    gpu.step(DT)
    ref.step(DT)
    assert rel(gpu.state()[0], ref.state()[0]) <= 1e-5


@pytest.mark.parametrize("cols", [30, 40])
def test_long_ribbon_steps_match_fp64(cols):
    """A long unpinned ribbon (cols x 400 cells, rotated 45 degrees, dt 1/120
    with the matrix at the same dt): its nested dissection gives separators of
    30-45 columns whose diagonal blocks a warp stages in column chunks wider
    than the warp; three plain steps stay within 1e-5 relative of FP64."""
    dt = 1.0 / 120.0
    mesh = scenarios.self_fold(cols, 400, 0.2, 2.0, lowest=0.5)
    setup = api.SetupDesc(stiffness=1e3, bend_stiffness=1e-4, density_gsm=150.0, matrix_dt=dt)
    gpu = api.ProjectiveDynamicsSolver().init_explicit(mesh, api.drape_config(max_iterations=10), setup,
                                                       pinned=mesh.pinned)
    ref = O.OracleSim(mesh, O.init_params(stiffness=1e3, bend_stiffness=1e-4, density_gsm=150.0, matrix_dt=dt),
                      O.default_config(max_iterations=10), precision=1)
    for _ in range(3):
        gpu.step(dt)
        ref.step(dt)
    e = rel(gpu.state()[0], ref.state()[0])
    print(f"ribbon {cols}x400: 3 steps, rel error {e:.2e}")
    assert e <= 1e-5, e


def test_level_schedules_and_autotuner():
    """Every candidate schedule of the autotuner (from all top-level
    supernodes on whole blocks to every narrow one on a single warp) steps a
    batch of uneven sheets and a long ribbon to within 1e-5 of FP64, with
    one launch per level and with the dependency-driven sweeps; the two sweep
    kinds give bit-identical results (the same arithmetic per supernode). The
    tuner picks one of the candidates and times them all."""
    dt = 1.0 / 120.0
    meshes = [(scenarios.hanging_sheet(40, 1.0), 1.0 / 60.0), (scenarios.hanging_sheet(23, 0.6), 1.0 / 60.0),
              (scenarios.self_fold(30, 400, 0.2, 2.0, lowest=0.5), dt)]
    cfg = api.drape_config(max_iterations=10)
    for lim in api.Batch.TUNE_LIMITS:
        for mesh, h in meshes:
            setup = api.SetupDesc(stiffness=1e3, bend_stiffness=1e-4, density_gsm=150.0, matrix_dt=h)
            out = {}
            for mode in ("levels", "dataflow"):  # one garment: no garment groups
                s = api.ProjectiveDynamicsSolver().init_explicit(mesh, cfg, setup, pinned=mesh.pinned)
                batch = api.Batch([s])
                batch.set_warp_limit(lim)
                batch.set_sweep_mode(mode)
                assert batch.sweep_mode() == (mode, lim)
                batch.step(h, 2)
                out[mode] = batch.state(0)[0]
            ref = O.OracleSim(mesh, O.init_params(stiffness=1e3, bend_stiffness=1e-4, density_gsm=150.0, matrix_dt=h),
                              O.default_config(max_iterations=10), precision=1)
            ref.step(h)
            ref.step(h)
            e = rel(out["levels"], ref.state()[0])
            assert e <= 1e-5, (lim, mesh.nv, e)
            assert np.array_equal(out["levels"], out["dataflow"]), (lim, mesh.nv)
    solvers = [api.ProjectiveDynamicsSolver().init(scenarios.hanging_sheet(sd, 1.0), cfg,
                                                   pinned=scenarios.hanging_sheet(sd, 1.0).pinned) for sd in (31, 47, 64)]
    batch = api.Batch(solvers)
    t = batch.tune()
    print(t)
    assert t["warp_item_limit"] in api.Batch.TUNE_LIMITS
    assert t["sweep_mode"] in api.Batch.SWEEP_MODES
    assert batch.sweep_mode() == (t["sweep_mode"], t["warp_item_limit"])
    assert all(v > 0 for m in t["sweep_ms"].values() for v in m.values())
    batch.step(1.0 / 60.0, 1)


def test_dataflow_sweeps_match_levels_on_a_mixed_batch():
    """A batch of many garments of different sizes (so that the dependency-
    driven sweeps interleave supernodes of different levels and garments)
    steps bit-identically with both sweep kinds, plain and with IPC. Sides 2
    and 3 are garments whose whole elimination tree is one bottom subtree: in
    the single dependency-driven launch their backward unit waits on their own
    forward."""
    sides = [12, 37, 20, 64, 9, 48, 31, 25, 2, 3] * 3
    cfg = api.drape_config(max_iterations=10, al_max_iterations=3, barrier_d_hat=1e-3, barrier_kappa=1e4)
    contact = api.Contact(has_ground=True, ground_height=0.6, kappa=1e4)
    res = {}
    for mode in ("levels", "dataflow"):  # at most 3 garments per topology: no garment groups
        solvers = []
        for k, sd in enumerate(sides):
            m = scenarios.hanging_sheet(sd, 0.5 + 0.03 * k)
            setup = api.SetupDesc(stiffness=800.0 + 50 * k, bend_stiffness=1e-4, density_gsm=150.0)
            solvers.append(api.ProjectiveDynamicsSolver().init_explicit(m, cfg, setup, pinned=m.pinned))
        batch = api.Batch(solvers)
        batch.set_sweep_mode(mode)
        batch.step(DT, 3)
        batch.step(DT, 3, contact=contact)
        res[mode] = [batch.state(k)[0] for k in range(len(sides))]
    for a, b in zip(res["levels"], res["dataflow"]):
        assert np.array_equal(a, b)


def grouped_batch_solvers(cfg, sides):
    """Hanging sheets of the given grid sides, each with its own length and
    material (same topology per side, different numbers)."""
    solvers = []
    for k, sd in enumerate(sides):
        m = scenarios.hanging_sheet(sd, 0.5 + 0.011 * k)
        setup = api.SetupDesc(stiffness=300.0 + 37.0 * k, bend_stiffness=1e-5 * (1 + k % 7), density_gsm=90.0 + 3 * k)
        solvers.append(api.ProjectiveDynamicsSolver().init_explicit(m, cfg, setup, pinned=m.pinned))
    return solvers


# 20 garments of side 12 (one group of 20 lanes), 40 of side 9 (a group of 32
# and one of 8), 35 of side 16 (a group of 32, 3 left per garment), singles
# (among them sides 2 and 3, whose whole tree is one bottom subtree), all
# interleaved in batch order
GROUPED_SIDES = ([12] * 20 + [9] * 40 + [16] * 35 + [31, 2, 3, 24])
GROUPED_SIDES = [GROUPED_SIDES[(k * 37) % len(GROUPED_SIDES)] for k in range(len(GROUPED_SIDES))]


@pytest.mark.parametrize("refine", [0, 1])
def test_grouped_sweeps_bit_identical_to_dataflow_and_to_solo(refine):
    """Garment groups (8 or more garments of one mesh topology, swept one
    lane per garment at the bottom of their trees) give exactly the results
    of the per-garment dependency-driven sweeps, plain and with IPC, with and
    without a refinement sweep, and exactly what the garments give stepped
    alone; the dependency-driven kernel's three compiled forms (five and four
    eight-warp blocks per SM, two sixteen-warp blocks) agree bit for bit. A batch with groups starts in the
    grouped kind."""
    assert len(set(GROUPED_SIDES)) == 7 and len(GROUPED_SIDES) == 99
    cfg = api.drape_config(max_iterations=8, al_max_iterations=3, barrier_d_hat=1e-3, barrier_kappa=1e4,
                           refinement_sweeps=refine)
    contact = api.Contact(has_ground=True, ground_height=0.3, kappa=1e4)
    res = {}
    for mode, glimit, blocks in (("dataflow", None, 5), ("grouped", 0, 5), ("grouped", 256, 5), ("grouped", 6144, 5),
                                 ("dataflow", None, 4), ("grouped", 256, 4), ("dataflow", None, 2), ("grouped", 256, 2)):
        batch = api.Batch(grouped_batch_solvers(cfg, GROUPED_SIDES))
        assert batch.sweep_mode()[0] == "grouped" and batch.sweep_blocks()[0] == 4
        batch.set_sweep_mode(mode)
        batch.set_sweep_blocks(blocks)
        assert batch.sweep_blocks()[0] == blocks
        if glimit is not None:
            batch.set_group_limit(glimit)
            assert batch.group_limit() == glimit
        batch.step(DT, 3)
        batch.step(DT, 3, contact=contact)
        res[(mode, glimit, blocks)] = [batch.state(k)[0] for k in range(len(GROUPED_SIDES))]
        batch.close()
    for key in res:
        for k, (a, b) in enumerate(zip(res[("dataflow", None, 5)], res[key])):
            assert np.array_equal(a, b), (key, k, GROUPED_SIDES[k], float(np.abs(a - b).max()))
    res["grouped"] = res[("grouped", 6144, 5)]
    # garments of each group, stepped alone
    solo = grouped_batch_solvers(cfg, GROUPED_SIDES)
    for k in (0, 1, 2, 5, 7, 11):
        for _ in range(3):
            solo[k].step(DT)
        for _ in range(3):
            solo[k].step_with_ipc(DT, contact)
        assert np.array_equal(solo[k].state()[0], res["grouped"][k]), (k, GROUPED_SIDES[k])


def test_local_step_shapes_bit_identical_and_tuned():
    """The membrane and bending steps with one or two elements per thread give
    bit-identical trajectories; the autotuner times both shapes of each."""
    cfg = api.drape_config(max_iterations=6)
    out = {}
    for shape in ((1, 1), (2, 2), (1, 2), (2, 1)):
        batch = api.Batch(grouped_batch_solvers(cfg, [12, 31, 9, 47, 20]))
        batch.set_local_shape(*shape)
        batch.step(DT, 3)
        out[shape] = [batch.state(k)[0] for k in range(5)]
        batch.close()
    for shape in out:
        for a, b in zip(out[shape], out[(2, 1)]):
            assert np.array_equal(a, b), shape
    batch = api.Batch(grouped_batch_solvers(cfg, [12, 31, 9, 47, 20]))
    t = batch.tune()
    assert t["triangles_per_thread"] in (1, 2) and t["hinges_per_thread"] in (1, 2)
    assert all(v > 0 for m in t["local_ms"].values() for v in m.values())


def test_grouped_kind_needs_groups_and_tunes():
    """The grouped kind is refused for a batch without garment groups; with
    groups the autotuner times it beside the other two kinds."""
    cfg = api.drape_config(max_iterations=6)
    few = api.Batch(grouped_batch_solvers(cfg, [12, 12, 9]))
    assert few.sweep_mode()[0] == "dataflow"
    with pytest.raises(Exception):
        few.set_sweep_mode("grouped")
    batch = api.Batch(grouped_batch_solvers(cfg, [12] * 16 + [20] * 9))
    t = batch.tune()
    print(t)
    assert set(t["sweep_ms"]) == {"levels", "dataflow", "grouped"}
    assert t["sweep_blocks_per_sm"] in (2, 4, 5)
    if t["sweep_mode"] != "levels":  # the two compiled forms of the dependency-driven kernel were timed
        assert all(v > 0 for v in t["sweep_blocks_ms"].values())
    assert all(v > 0 for m in t["sweep_ms"].values() for v in m.values())
    batch.step(DT, 2)


@pytest.mark.parametrize("side,length", [(20, 1.0), (48, 1.5)])
def test_device_factorization_matches_host_factorization(side, length):
    """The FP64 Cholesky factor computed on the GPU (multifrontal, the default)
    and the one computed on the host give the same trajectories: both are
    FP64 factors of the same matrix rounded to FP32 for the sweeps, so they
    differ by FP64 rounding only (<= 1e-6 m after 10 steps). A batch holding
    one garment of each kind gives each the result it gives alone."""
    mesh = scenarios.hanging_sheet(side, length)
    setup = api.SetupDesc(stiffness=1e3, bend_stiffness=1e-4, density_gsm=150.0)
    runs = {}
    for host in (False, True):
        cfg = api.drape_config(max_iterations=10, host_factorization=host)
        s = api.ProjectiveDynamicsSolver().init_explicit(mesh, cfg, setup, pinned=mesh.pinned)
        for _ in range(10):
            s.step(DT)
        runs[host] = s.state()[0]
    diff = float(np.abs(runs[False] - runs[True]).max())
    print(f"max |device factor - host factor| after 10 steps = {diff:.3e} m")
    assert diff <= 1e-6, diff
    pair = [api.ProjectiveDynamicsSolver().init_explicit(mesh, api.drape_config(max_iterations=10, host_factorization=h),
                                                         setup, pinned=mesh.pinned) for h in (False, True)]
    batch = api.Batch(pair)
    batch.step(DT, 10)
    assert np.array_equal(batch.state(0)[0], runs[False])
    assert np.array_equal(batch.state(1)[0], runs[True])
