"""GPU parity of step_with_ipc and of the contact boundary queries.

* broad phase: the GPU candidate triangle pairs equal, as sorted integer
  lists, the complete set {(ta < tb) : inflated AABBs overlap} the oracle
  computes on the same f32 positions (bit-exact);
* CCD: the GPU vertex-triangle hit set over those pairs equals the oracle's,
  both evaluated in FP64 (bit-exact), with the same minimum TOI;
* IPC step (ground, sphere, cylinder, box): every step from an identical state within 1e-5
  relative of the FP64 oracle, with the same AL pass count, active contacts
  and step size. The reference's own FP32 arithmetic (the oracle's ref32 mode)
  misses that bar on these steps (up to ~8e-4: the FP32 polar decomposition of
  compressed triangles and the backtracking test amplify its rounding); the
  GPU forms those parts in FP64 and is printed beside it.
* self-contact step (VT + EE barriers, FP64 inside 10 d_hat, FP64 gradient
  accumulation): within 1e-5 relative of FP64 (ref32: ~1.2e-4).
  Short runs stay within 1e-4 m of FP64.
"""
import numpy as np
import pytest

import oracle_api as O
from vistio_b200 import api, scenarios

pytestmark = pytest.mark.gpu

DT = 1.0 / 60.0


def rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def folded_ribbon(cols=8, rows=60, width=0.1, height=0.6, gap=0.004, seed=0):
    """A ribbon folded in half over itself with the layers `gap` apart, plus a
    small deterministic jitter, so many triangle pairs are close."""
    px, py, pz, tris = scenarios.quad_grid(cols, rows, width, height)
    t = (py - py.min()) / (py.max() - py.min())  # 0..1 along the ribbon
    L = height
    s = t * L
    half = L / 2
    x = px.copy()
    y = np.where(s < half, s, L - s).astype(np.float32)
    z = np.where(s < half, 0.0, gap).astype(np.float32)
    bend = np.abs(s - half) < L / rows
    z = np.where(bend, gap / 2, z).astype(np.float32)
    rng = np.random.default_rng(seed)
    z = (z + rng.uniform(-gap / 8, gap / 8, size=z.shape)).astype(np.float32)
    pos = np.stack([x, y + 0.5, z], 1).astype(np.float32)
    return pos, tris


@pytest.mark.parametrize("gap,margin", [(0.004, 7.5e-4), (0.002, 1.5e-3), (0.01, 7.5e-4)])
def test_broadphase_pairs_bit_exact(gap, margin):
    pos, tris = folded_ribbon(gap=gap)
    ref = O.tri_pairs(pos, tris, margin, mode=0)
    got = api.broadphase_pairs(pos, tris, margin)
    assert got.shape == ref.shape, (got.shape, ref.shape)
    assert np.array_equal(got, ref)
    # the reference's median-split tree drops some of these pairs (bvh.rs:205-209)
    faithful = O.tri_pairs(pos, tris, margin, mode=1)
    assert len(faithful) <= len(ref)
    fset = set(map(tuple, faithful))
    assert fset <= set(map(tuple, ref))


def test_broadphase_pairs_independent_of_triangle_order():
    """The LBVH sorts triangles by the Morton code of their centroids, so a
    mesh stored in a random triangle order gives the same complete pair set
    (bit-exact against the oracle on the permuted mesh)."""
    pos, tris = folded_ribbon(gap=0.004)
    perm = np.random.default_rng(7).permutation(len(tris))
    shuffled = np.ascontiguousarray(tris[perm])
    ref = O.tri_pairs(pos, shuffled, 7.5e-4, mode=0)
    got = api.broadphase_pairs(pos, shuffled, 7.5e-4)
    assert np.array_equal(got, ref)
    # and, mapped back to the original triangle ids, the unshuffled set
    back = np.sort(perm[got], axis=1)
    back = back[np.lexsort((back[:, 1], back[:, 0]))]
    assert np.array_equal(back, O.tri_pairs(pos, tris, 7.5e-4, mode=0))


def test_broadphase_empty_and_degenerate():
    pos = np.zeros((3, 3), np.float32)
    tris = np.array([[0, 1, 2]], np.uint32)
    assert len(api.broadphase_pairs(pos, tris, 1e-3)) == 0
    pos, tris = folded_ribbon(cols=1, rows=2)
    ref = O.tri_pairs(pos, tris, 1e-3, mode=0)
    assert np.array_equal(api.broadphase_pairs(pos, tris, 1e-3), ref)


def test_ccd_hits_bit_exact():
    pos, tris = folded_ribbon(gap=0.004)
    rng = np.random.default_rng(3)
    # move the upper layer through the lower one
    p1 = pos.copy()
    upper = pos[:, 2] > 0.002
    p1[upper, 2] -= 0.008
    p1 += rng.uniform(-1e-4, 1e-4, size=p1.shape).astype(np.float32)
    pairs = O.tri_pairs(pos, tris, 7.5e-4, mode=0)
    assert len(pairs) > 0
    hr, tr = O.ccd_hits(pos, p1, tris, pairs)
    hg, tg = api.ccd_hits(pos, p1, tris, pairs)
    assert len(hr) > 0
    assert np.array_equal(hg, hr)
    assert abs(tg - tr) <= 1e-6 * max(1.0, abs(tr))


def step_errors(gpu, ref64, ref32, c, contact, dt=DT):
    """One step of each from the FP64 oracle's state; returns (gpu error,
    ref32 error) relative to the FP64 result, and the three step results."""
    p, v = ref64.state()
    gpu.set_state(p, v)
    ref32.set_state(p, v)
    r64 = ref64.step_ipc(dt, c)
    r32 = ref32.step_ipc(dt, c)
    rg = gpu.step_with_ipc(dt, contact)
    x64 = ref64.state()[0]
    return rel(gpu.state()[0], x64), rel(ref32.state()[0], x64), rg, r64, r32


def ipc_pair(mesh, contact: api.Contact, d_hat=1e-3, kappa=1e4, iters=15, al=5, precision=1, setup=None,
             params=None, refine=0):
    cfg = api.drape_config(max_iterations=iters, al_max_iterations=al, barrier_d_hat=d_hat, barrier_kappa=kappa,
                           refinement_sweeps=refine)
    setup = setup or api.SetupDesc(stiffness=1e3, bend_stiffness=1e-4, density_gsm=150.0)
    gpu = api.ProjectiveDynamicsSolver().init_explicit(mesh, cfg, setup, pinned=mesh.pinned)
    oc = O.default_config(max_iterations=iters, al_max_iterations=al, barrier_d_hat=d_hat)
    params = params or O.init_params(stiffness=1e3, bend_stiffness=1e-4, density_gsm=150.0)
    ref = O.OracleSim(mesh, params, oc, precision=precision)
    c = O.Contact()
    c.has_ground, c.ground_height = int(contact.has_ground), contact.ground_height
    c.has_sphere = int(contact.has_sphere)
    c.sphere_center[:] = contact.sphere_center
    c.sphere_radius = contact.sphere_radius
    c.self_collision, c.bvh_faithful = int(contact.self_collision), 0
    c.kappa, c.thickness = contact.kappa, contact.thickness
    c.has_cylinder = int(contact.has_cylinder)
    (c.cylinder_center_x, c.cylinder_center_z, c.cylinder_top_y, c.cylinder_radius) = contact.cylinder
    c.has_box = int(contact.has_box)
    c.box_min[:] = contact.box_min
    c.box_max[:] = contact.box_max
    if contact.has_ground:
        ref.set_ground(1, contact.ground_height)
    return gpu, ref, c


SPHERE = api.Contact(has_ground=True, ground_height=-0.3, has_sphere=True, sphere_center=(0.0, 0.0, 0.0),
                     sphere_radius=0.3, kappa=1e4)


def test_sphere_drape_steps_match_fp64():
    """sphere_drape geometry on a 24x24 sheet: every step from the oracle's
    state within 1e-5 relative of FP64 (see module doc); contacts become
    active and the backtracking line search engages during the run."""
    mesh = scenarios.sphere_drape(side=24, length=1.5, height=0.35)
    gpu, ref, c = ipc_pair(mesh, SPHERE)
    _, ref32, _ = ipc_pair(mesh, SPHERE, precision=0)
    active, backtracked = 0, 0
    for s in range(40):
        e, e32, rg, r64, r32 = step_errors(gpu, ref, ref32, c, SPHERE)
        print(f"step {s}: gpu {e:.2e} ref32 {e32:.2e} alpha {rg.last_alpha} / {r64.last_alpha}")
        assert e <= 1e-5, (s, e, e32)
        assert rg.al_iterations == r64.al_iterations
        assert rg.active_contacts == r64.active_contacts
        assert rg.last_alpha == r64.last_alpha
        active = max(active, rg.active_contacts)
        backtracked += rg.last_alpha < 1.0
    assert active > 0, "the sheet never reached the sphere"
    assert backtracked > 0


@pytest.mark.parametrize("refine", [0, 1])
def test_sphere_drape_run_within_1e4_m(refine):
    """45 steps onto the sphere (also with every solve FP64-refined)."""
    mesh = scenarios.sphere_drape(side=20, length=1.5, height=0.35)
    gpu, ref, c = ipc_pair(mesh, SPHERE, refine=refine)
    for _ in range(45):
        ref.step_ipc(DT, c)
        gpu.step_with_ipc(DT, SPHERE)
    err = float(np.abs(gpu.state()[0] - ref.state()[0]).max())
    print(f"45-step sphere_drape 20x20, refinement {refine}: max |x_gpu - x_fp64| = {err:.3e} m")
    assert err <= 1e-4, err
    # non-penetration of the sphere within 2 cm (bench_tests.rs:138-225)
    r = np.linalg.norm(gpu.state()[0], axis=1)
    assert r.min() >= 0.3 - 0.02


def estimated_kappa(mesh, d_hat=1e-3):
    """estimate_initial_kappa (barrier.rs:97-116) from the garment's mean lumped
    vertex mass, as the runner does from its vertex mass."""
    sim = O.OracleSim(mesh, O.init_params(stiffness=1e3, bend_stiffness=1e-4, density_gsm=150.0),
                      O.default_config())
    m = sim.masses()
    return float(O.lib().orc_estimate_kappa(0.0, float(m[mesh.pinned == 0].mean()), 9.81, d_hat))


def test_cusick_drape_steps_match_fp64():
    """The Cusick drape disc (circular_grid(0.15, 64), 829 vertices) starting
    3 cm above the pedestal cylinder of runner.rs:83-86 (top 0.3, radius 0.09,
    ground -0.3; cylinder.rs: barrier off the top face, the wall and the rim,
    CCD on the wall and the top face): every step from the oracle's state
    within 1e-5 relative of FP64, with the same AL pass count, active contacts
    and step size; the barrier becomes active and the line search engages."""
    mesh = scenarios.cusick_drape(height=0.33)
    pedestal = api.Contact(has_ground=True, ground_height=-0.3, has_cylinder=True, cylinder=(0.0, 0.0, 0.3, 0.09),
                           kappa=estimated_kappa(mesh))
    gpu, ref, c = ipc_pair(mesh, pedestal)
    _, ref32, _ = ipc_pair(mesh, pedestal, precision=0)
    active, backtracked = 0, 0
    for s in range(40):
        e, e32, rg, r64, r32 = step_errors(gpu, ref, ref32, c, pedestal)
        print(f"step {s}: gpu {e:.2e} ref32 {e32:.2e} active {rg.active_contacts} alpha {rg.last_alpha}")
        assert e <= 1e-5, (s, e, e32)
        assert rg.al_iterations == r64.al_iterations
        assert rg.active_contacts == r64.active_contacts
        assert rg.last_alpha == r64.last_alpha
        active = max(active, rg.active_contacts)
        backtracked += rg.last_alpha < 1.0
    assert active > 0, "the disc never reached the pedestal"
    assert backtracked > 0


def test_cusick_drape_no_penetration():
    """bench_tests.rs:225-300: the Cusick drape for 1 s with the reference's
    default configuration (IPC, d_hat 1e-3, kappa from the 2 g vertex mass)
    over a cylinder of radius 0.18 with its top at 0.2 and the ground at
    -0.3: no vertex below the top face comes within 2 cm inside the wall."""
    mesh = scenarios.cusick_drape()
    cfg = api.SolverConfig()
    kappa = O.lib().orc_estimate_kappa(cfg.barrier_kappa, 0.002, abs(cfg.gravity[1]), cfg.barrier_d_hat)
    contact = api.Contact(has_ground=True, ground_height=-0.3, has_cylinder=True, cylinder=(0.0, 0.0, 0.2, 0.18),
                          kappa=kappa)
    s = api.ProjectiveDynamicsSolver().init(mesh, cfg, pinned=mesh.pinned)
    for _ in range(60):
        s.step_with_ipc(DT, contact)
        x = s.state()[0]
        below = x[:, 1] < 0.2
        if below.any():
            r = np.sqrt(x[below, 0] ** 2 + x[below, 2] ** 2)
            assert r.min() >= 0.18 - 0.02, r.min()


def test_box_drape_steps_match_fp64():
    """A 0.6 m sheet starting 3 cm above a 0.4 x 0.2 x 0.4 m box (box_collider.rs:
    barrier off the faces, edges and corners; slab CCD): every step from the
    oracle's state within 1e-5 relative of FP64, with the same AL pass count,
    active contacts and step size."""
    mesh = scenarios.sphere_drape(side=20, length=0.6, height=0.13)
    box = api.Contact(has_ground=True, ground_height=-0.3, has_box=True, box_min=(-0.2, -0.1, -0.2),
                      box_max=(0.2, 0.1, 0.2), kappa=estimated_kappa(mesh))
    gpu, ref, c = ipc_pair(mesh, box)
    _, ref32, _ = ipc_pair(mesh, box, precision=0)
    active = 0
    for s in range(30):
        e, e32, rg, r64, r32 = step_errors(gpu, ref, ref32, c, box)
        print(f"step {s}: gpu {e:.2e} ref32 {e32:.2e} active {rg.active_contacts} alpha {rg.last_alpha}")
        assert e <= 1e-5, (s, e, e32)
        assert rg.al_iterations == r64.al_iterations
        assert rg.active_contacts == r64.active_contacts
        assert rg.last_alpha == r64.last_alpha
        active = max(active, rg.active_contacts)
    assert active > 0, "the sheet never reached the box"


def test_ground_contact_steps_match_fp64():
    mesh = scenarios.sphere_drape(side=16, length=0.8, height=0.02)
    ground = api.Contact(has_ground=True, ground_height=0.0, kappa=1e4)
    gpu, ref, c = ipc_pair(mesh, ground)
    _, ref32, _ = ipc_pair(mesh, ground, precision=0)
    for s in range(20):
        e, e32, rg, r64, r32 = step_errors(gpu, ref, ref32, c, ground)
        assert e <= 1e-5, (s, e, e32)
        assert rg.active_contacts == r64.active_contacts


@pytest.mark.parametrize("iters,al", [(2, 1), (10, 3)])
def test_self_contact_step_matches(iters, al):
    """A self-contact step (VT + EE barriers with 1-ring exclusion, thickness
    barrier, self CCD) on a folded ribbon with ~15k active contacts: same
    active-contact count as the oracle, positions within the reference's FP32
    noise of FP64."""
    pos, tris = folded_ribbon(cols=6, rows=40, gap=0.003)
    mesh = scenarios.Mesh(pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy(), tris,
                          np.zeros(len(pos), np.uint8))
    d_hat = 5e-4
    self_c = api.Contact(self_collision=True, kappa=1e3, thickness=1.5 * d_hat)
    gpu, ref, c = ipc_pair(mesh, self_c, d_hat=d_hat, kappa=1e3, iters=iters, al=al)
    _, ref32, _ = ipc_pair(mesh, self_c, d_hat=d_hat, kappa=1e3, iters=iters, al=al, precision=0)
    e, e32, rg, r64, r32 = step_errors(gpu, ref, ref32, c, self_c)
    print(f"self contact: gpu {e:.2e} ref32 {e32:.2e} active {rg.active_contacts} / {r64.active_contacts}")
    assert rg.active_contacts == r64.active_contacts
    assert e <= 1e-5, (e, e32)


def crossing_sheets(n=10, size=0.1, squeeze=0.25):
    """Two square sheets in one mesh: a flat one at y = 0.5, and above it a
    second whose rest shape is a plane tilted 17 degrees through it (its low
    edge 1 cm below the first sheet), started squeezed to `squeeze` of its
    size about its centre, clear of the first sheet. Springing back along its
    plane drives its low side through the first sheet within the first PD
    iteration, so the self CCD must bound that step."""
    px, py, _, tris = scenarios.quad_grid(n, n, size, size)
    nv = len(px)
    bottom = np.stack([px, np.full(nv, 0.5, np.float32), py], 1)
    rest_top = np.stack([px, 0.49 + 0.3 * (px + size / 2), py], 1)
    c = rest_top.mean(0)
    top = c + squeeze * (rest_top - c)
    rest = np.concatenate([bottom, rest_top]).astype(np.float32)
    state = np.concatenate([bottom, top]).astype(np.float32)
    t = np.concatenate([tris, tris + nv]).astype(np.uint32)
    mesh = scenarios.Mesh(rest[:, 0].copy(), rest[:, 1].copy(), rest[:, 2].copy(), t, np.zeros(2 * nv, np.uint8))
    assert state[nv:, 1].min() > 0.5 + 1e-3  # clear of the first sheet at the start
    return mesh, state


def test_self_ccd_test_list_bit_identical_to_every_pair_test():
    """The self CCD over its deduplicated vertex-triangle tests (each test of
    the candidate pairs once, the default) against every test of every pair,
    as compute_max_step_size runs them (ccd.rs:238-292): a batch of crossing
    sheets (the self CCD bounds their steps), folded ribbons and sphere drapes
    steps bit-identically both ways."""
    d_hat = 5e-4
    contact = api.Contact(has_ground=True, ground_height=-0.3, has_sphere=True, sphere_center=(0.0, 0.0, 0.0),
                          sphere_radius=0.3, self_collision=True, kappa=1e3, thickness=1.5 * d_hat)
    cfg = api.drape_config(max_iterations=8, al_max_iterations=3, barrier_d_hat=d_hat * d_hat, barrier_kappa=1e3)
    setup = api.SetupDesc(stiffness=1e3, bend_stiffness=1e-4, density_gsm=150.0)
    meshes, states = [], []
    for n in (10, 13):
        m, st = crossing_sheets(n)
        meshes.append(m)
        states.append(st)
    for k in range(2):
        pos, tris = folded_ribbon(cols=6, rows=40, gap=0.003, seed=k)
        meshes.append(scenarios.Mesh(pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy(), tris,
                                     np.zeros(len(pos), np.uint8)))
        states.append(None)
    for side in (16, 23):
        meshes.append(scenarios.sphere_drape(side=side, length=1.5, height=0.301))
        states.append(None)

    def run(dedup, nsteps=6):
        solvers = [api.ProjectiveDynamicsSolver().init_explicit(m, cfg, setup, pinned=m.pinned) for m in meshes]
        batch = api.Batch(solvers)
        batch.set_self_ccd_dedup(dedup)
        for k, st in enumerate(states):
            if st is not None:
                batch.set_state(k, st)
        out = []
        for _ in range(nsteps):
            batch.step(DT, 1, contact)
            out.append([batch.state(k)[0].copy() for k in range(len(meshes))])
        batch.close()
        for s_ in solvers:
            s_.close()
        return out

    a, b = run(True), run(False)
    for sa, sb in zip(a, b):
        for pa, pb in zip(sa, sb):
            assert np.array_equal(pa, pb)
    # the self CCD bounds the first PD iteration of the crossing sheets: their
    # first step, stopped after that iteration, takes a step below 1 (the CCD
    # scales its bound by 0.8), and both forms land on the same positions
    cfg1 = api.drape_config(max_iterations=1, al_max_iterations=1, barrier_d_hat=d_hat * d_hat, barrier_kappa=1e3)
    solo = api.ProjectiveDynamicsSolver().init_explicit(meshes[0], cfg1, setup, pinned=meshes[0].pinned)
    solo.set_state(states[0])
    alpha = solo.step_with_ipc(DT, contact).last_alpha
    solo.close()
    assert alpha < 0.9, alpha
    first = []
    for dedup in (True, False):
        solo = api.ProjectiveDynamicsSolver().init_explicit(meshes[0], cfg1, setup, pinned=meshes[0].pinned)
        batch = api.Batch([solo])
        batch.set_self_ccd_dedup(dedup)
        batch.set_state(0, states[0])
        batch.step(DT, 1, contact)
        first.append(batch.state(0)[0])
        batch.close()
        solo.close()
    assert np.array_equal(first[0], first[1])


def steps_from_oracle(gpu, ref, c, contact, nsteps, dt=DT):
    """nsteps GPU steps, each from the FP64 oracle's state; returns the worst
    relative error and the last GPU step result."""
    worst, rg = 0.0, None
    for _ in range(nsteps):
        p, v = ref.state()
        gpu.set_state(p, v)
        ref.step_ipc(dt, c)
        rg = gpu.step_with_ipc(dt, contact)
        worst = max(worst, rel(gpu.state()[0], ref.state()[0]))
    return worst, rg


def test_sphere_drape_64_configuration():
    """The sphere-drape configuration at full size: 64x64 cells (4225
    vertices), 1.5 m sheet at y = 0.5, sphere r = 0.3 at the origin, ground
    -0.3, d_hat 1e-3, kappa 1e4, AL <= 5, 15 iterations. With these light
    vertices (8e-5 kg) the barrier throws the sheet's centre back up within
    the step in which it enters the contact zone (the reference's dynamics:
    the oracle shows the same bounce). Steps 9-22, each from the FP64
    oracle's state, cover two bounces and are each within 1e-5 of FP64."""
    mesh = scenarios.sphere_drape(side=64, length=1.5, height=0.5)
    assert mesh.nv == 4225 and mesh.nt == 8192
    gpu, ref, c = ipc_pair(mesh, SPHERE)
    centre = 32 * 65 + 32
    for _ in range(9):
        ref.step_ipc(DT, c)
    worst, rose = 0.0, False
    for _ in range(14):
        p, v = ref.state()
        gpu.set_state(p, v)
        ref.step_ipc(DT, c)
        gpu.step_with_ipc(DT, SPHERE)
        pg = gpu.state()[0]
        worst = max(worst, rel(pg, ref.state()[0]))
        rose |= bool(pg[centre, 1] > p[centre, 1] + 0.01)  # only the barrier can lift the centre
    print(f"sphere_drape 64x64: worst step error {worst:.2e}")
    assert worst <= 1e-5, worst
    assert rose, "the sheet never reached the sphere's barrier"


def test_self_fold_configuration():
    """The self-fold configuration at full size: a 0.2 m x 2.0 m ribbon of
    40x400 cells (16441 vertices) rotated 45 degrees about x, orthotropic
    membrane (warp 1e3, weft 6e2, element stiffness 1e3), self contact with
    1-ring exclusion, ground y = 0, dt = 1/120, kappa from
    estimate_initial_kappa with the mean vertex mass (runner.rs:190-195).
    Two readings differ from the reference's literal wiring, because that
    wiring makes the reference's own step diverge here (checked with the
    oracle, FP64 and FP32 alike):
    * the system matrix is assembled with the step's dt (1/120); with the
      reference's fixed 1/60 the ribbon's height grows about 4x per step even
      without contact;
    * d_hat = 5e-4 m is a distance (barrier_d_hat = d_hat^2, thickness
      1.5 d_hat); as a squared distance it puts every triangle pair within
      3.2 cm of this 5 mm mesh in contact (1.4 M contacts).
    The ribbon starts 1 mm above the ground so that contact begins at once;
    each step is within 1e-5 of FP64."""
    dt = 1.0 / 120.0
    mesh = scenarios.self_fold(40, 400, 0.2, 2.0, lowest=0.001)
    assert mesh.nv == 16441 and mesh.nt == 32000
    d_hat = 5e-4
    setup = api.SetupDesc(model=api.MODEL_ORTHOTROPIC, stiffness=1e3, warp_stiffness=1e3, weft_stiffness=6e2,
                          bend_stiffness=1e-4, density_gsm=150.0, matrix_dt=dt)
    params = O.init_params(model=O.MODEL_ORTHO, stiffness=1e3, warp=1e3, weft=6e2, bend_stiffness=1e-4,
                           density_gsm=150.0, matrix_dt=dt)
    probe = api.ProjectiveDynamicsSolver().init_explicit(mesh, api.drape_config(), setup, pinned=mesh.pinned)
    kappa = float(O.lib().orc_estimate_kappa(0.0, float(probe.lumped_masses().mean()), 9.81, d_hat * d_hat))
    # kappa <= 0 makes the library estimate it the same way
    contact = api.Contact(has_ground=True, ground_height=0.0, self_collision=True, kappa=0.0, thickness=1.5 * d_hat)
    gpu, ref, c = ipc_pair(mesh, contact, d_hat=d_hat * d_hat, kappa=0.0, iters=10, al=5, setup=setup, params=params)
    c.kappa = kappa
    worst, active = 0.0, 0
    for _ in range(4):
        w, rg = steps_from_oracle(gpu, ref, c, contact, 1, dt=dt)
        worst, active = max(worst, w), max(active, rg.active_contacts)
    print(f"self_fold 40x400: kappa {kappa:.4g}, worst step error {worst:.2e}, active contacts {active}")
    assert worst <= 1e-5, worst
    assert active > 0


def test_device_barrier_gradient_matches_oracle():
    """vistio_barrier_grad: the device's FP64 barrier gradient (barrier.rs:35-46,
    78-87, and the C-IPC form 138-163) against the oracle's FP32 restatement
    over six decades of squared distance, within 1e-4 relative (the oracle
    rounds its inputs and result to f32), zero at and beyond d_hat, and the
    known answers of barrier_tests.rs."""
    d_hat, kappa = 1e-3, 1e4
    d2 = np.concatenate([np.geomspace(1e-9, 2e-3, 400), [0.0, d_hat, 2 * d_hat]])
    g = api.barrier_grad(d2, d_hat, kappa)
    L = O.lib()
    ref = np.array([L.orc_scaled_barrier_gradient(float(x), d_hat, kappa) for x in d2], np.float64)
    inside = (d2 > 0) & (d2 < d_hat * (1 - 1e-6))
    assert np.all(np.abs(g[inside] - ref[inside]) <= 1e-4 * np.abs(ref[inside]) + 1e-6)
    assert np.all(g[d2 >= d_hat] == 0.0) and np.all(g[inside] < 0.0)
    # thickness form: d_eff = d2 - t^2; at or below the thickness the clamped maximum
    t = 1.5e-3
    gt = api.barrier_grad(d2, d_hat, kappa, thickness=t)
    reft = np.array([kappa * L.orc_barrier_gradient_thick(float(x), d_hat, t) for x in d2], np.float64)
    deff = d2 - t * t
    ins = (deff > 1e-12) & (deff < d_hat * (1 - 1e-6))
    assert np.all(np.abs(gt[ins] - reft[ins]) <= 1e-4 * np.abs(reft[ins]) + 1e-6)
    assert np.all(gt[deff <= 0] == gt[deff <= 0][0]) and gt[deff <= 0][0] < 0
    # barrier_tests.rs: repulsive inside, massive at d <= 0 (unscaled < -5)
    assert api.barrier_grad([0.005], 0.01, 1.0)[0] < 0.0
    assert api.barrier_grad([0.0], 0.01, 1.0)[0] < -5.0
