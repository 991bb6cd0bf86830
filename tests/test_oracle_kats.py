"""The oracle pinned to the reference's own known-answer tests.

Each case below restates, against the oracle's exported primitives and its
simulation, a unit test the reference ships for this path; the docstrings name
the test and file. The reference is Rust and does not build here, so these
are the pins that the oracle (and, through it, the CUDA path) is held to:

* distance primitives: crates/vistio-contact/src/tests/distance_primitives_tests.rs
* CCD and the cubic solver: crates/vistio-contact/src/tests/ccd_tests.rs
* barrier and kappa: crates/vistio-contact/src/tests/barrier_tests.rs
* IPC contact set: crates/vistio-contact/src/tests/ipc_response_tests.rs
* polar decomposition and the sparse solver: crates/vistio-math/tests/math_tests.rs
* PD solver and bending: crates/vistio-solver/tests/solver_tests.rs
"""
import ctypes as C
import math

import numpy as np
import pytest

import oracle_api as O
from vistio_b200 import scenarios

DT_FACE, DT_EDGE0, DT_VERT0, DT_DEGEN = 0, 1, 4, 8
PI32 = float(np.float32(math.pi))


def v3(*xs):
    return O.vec3(xs)


def pt(p, a, b, c):
    t = C.c_int(-1)
    d = O.lib().orc_pt_dist2(v3(*p), v3(*a), v3(*b), v3(*c), C.byref(t))
    return float(d), t.value


def ee(a0, a1, b0, b1):
    t = C.c_int(-1)
    d = O.lib().orc_ee_dist2(v3(*a0), v3(*a1), v3(*b0), v3(*b1), C.byref(t))
    return float(d), t.value


def grad(fn, *pts):
    out = np.zeros(12, np.float32)
    fn(*[v3(*p) for p in pts], out.ctypes.data_as(C.POINTER(C.c_float)))
    return out.reshape(4, 3)


A, B, CC = (0.0, 0.0, 0.0), (1.0, 0.0, 0.0), (0.0, 1.0, 0.0)


# ---------------------------------------------------------------- distances
@pytest.mark.parametrize("p,d2,dtype", [
    ((0.25, 0.25, 0.0), 0.0, DT_FACE),     # distance_point_on_face
    ((0.25, 0.25, 0.5), 0.25, DT_FACE),    # distance_point_above_face
    ((-1.0, -1.0, 0.0), 2.0, DT_VERT0),    # distance_point_nearest_vertex
    ((0.5, -0.5, 0.0), 0.25, DT_EDGE0),    # distance_point_nearest_edge
])
def test_point_triangle_distance(p, d2, dtype):
    d, t = pt(p, A, B, CC)
    assert abs(d - d2) < (1e-10 if d2 == 0.0 else 1e-6), d
    assert t == dtype


def test_point_degenerate_triangle():
    """distance_degenerate_triangle: collinear triangle, d^2 = 1."""
    d, _ = pt((0.5, 1.0, 0.0), (0.0, 0.0, 0.0), (1.0, 0.0, 0.0), (0.5, 0.0, 0.0))
    assert abs(d - 1.0) < 1e-6


@pytest.mark.parametrize("edges,d2", [
    (((0, 0, -1), (0, 0, 1), (-1, 1, 0), (1, 1, 0)), 1.0),   # distance_edges_crossing
    (((0, 0, 0), (1, 0, 0), (0, 1, 0), (1, 1, 0)), 1.0),     # distance_edges_parallel
    (((0, 0, 0), (1, 0, 0), (0.5, 0, 0), (0.5, 1, 0)), 0.0),  # distance_edges_touching
])
def test_edge_edge_distance(edges, d2):
    d, _ = ee(*edges)
    assert abs(d - d2) < (1e-10 if d2 == 0.0 else 1e-6), d


def test_degenerate_edges():
    """distance_degenerate_edges: both segments are points, d^2 = 1, Degenerate."""
    d, t = ee((0, 0, 0), (0, 0, 0), (1, 0, 0), (1, 0, 0))
    assert abs(d - 1.0) < 1e-6 and t == DT_DEGEN


def test_point_triangle_gradient_finite_difference():
    """point_triangle_gradient_finite_difference: d(d^2)/dp.x against a forward difference."""
    p = (0.25, 0.25, 0.5)
    g = grad(O.lib().orc_pt_grad, p, A, B, CC)
    eps = 1e-4
    fd = (pt((p[0] + eps, p[1], p[2]), A, B, CC)[0] - pt(p, A, B, CC)[0]) / eps
    assert abs(g[0, 0] - fd) < 0.01


def test_edge_edge_gradient_finite_difference():
    """edge_edge_gradient_finite_difference: d(d^2)/da0.y against a forward difference."""
    e = [(0.0, 0.0, -0.5), (0.0, 0.0, 0.5), (-0.5, 1.0, 0.0), (0.5, 1.0, 0.0)]
    g = grad(O.lib().orc_ee_grad, *e)
    eps = 1e-4
    shifted = [(e[0][0], e[0][1] + eps, e[0][2])] + e[1:]
    fd = (ee(*shifted)[0] - ee(*e)[0]) / eps
    assert abs(g[0, 1] - fd) < 0.05


# ---------------------------------------------------------------------- CCD
def vt_ccd(p0, p1, tri0, tri1):
    toi = C.c_float(-1.0)
    hit = O.lib().orc_vt_ccd(v3(*p0), v3(*p1), v3(*tri0[0]), v3(*tri1[0]), v3(*tri0[1]), v3(*tri1[1]),
                             v3(*tri0[2]), v3(*tri1[2]), C.byref(toi))
    return bool(hit), toi.value


TRI = (A, B, CC)


def test_ccd_vertex_passes_through_triangle():
    """ccd_vertex_passes_through_triangle: TOI in (0, 1), near 0.5 x the 0.9 safety margin."""
    hit, t = vt_ccd((0.25, 0.25, 1.0), (0.25, 0.25, -1.0), TRI, TRI)
    assert hit and 0.0 < t < 1.0
    assert abs(t - 0.5 * 0.9) < 0.1


@pytest.mark.parametrize("p0,p1", [
    ((5.0, 5.0, 1.0), (5.0, 5.0, -1.0)),    # ccd_vertex_misses_triangle
    ((0.25, 0.25, 1.0), (0.25, 0.25, 2.0)),  # ccd_vertex_moves_away
])
def test_ccd_vertex_no_hit(p0, p1):
    assert not vt_ccd(p0, p1, TRI, TRI)[0]


def ee_ccd(a0, a1, b0, b1, c0, c1, d0, d1):
    toi = C.c_float(-1.0)
    hit = O.lib().orc_ee_ccd(*[v3(*x) for x in (a0, a1, b0, b1, c0, c1, d0, d1)], C.byref(toi))
    return bool(hit)


def test_ccd_edge_edge_crossing():
    """ccd_edge_edge_crossing."""
    assert ee_ccd((-1, 0, 0.5), (-1, 0, -0.5), (1, 0, 0.5), (1, 0, -0.5),
                  (0, -1, -0.5), (0, -1, 0.5), (0, 1, -0.5), (0, 1, 0.5))


def test_ccd_edge_edge_no_crossing():
    """ccd_edge_edge_no_crossing: parallel, stationary edges 5 apart."""
    assert not ee_ccd((0, 0, 0), (0, 0, 0), (1, 0, 0), (1, 0, 0), (0, 5, 0), (0, 5, 0), (1, 5, 0), (1, 5, 0))


def cubic(a, b, c, d):
    out = np.zeros(3, np.float32)
    n = O.lib().orc_cubic_roots(a, b, c, d, out.ctypes.data_as(C.POINTER(C.c_float)))
    return sorted(out[:n].tolist())


def test_cubic_triple_root():
    """cubic_solver_triple_root: (t - 0.5)^3."""
    r = cubic(1.0, -1.5, 0.75, -0.125)
    assert r and all(abs(x - 0.5) < 0.01 for x in r)


def test_cubic_three_roots():
    """cubic_solver_identity: (t-1)(t-2)(t-3)."""
    r = cubic(1.0, -6.0, 11.0, -6.0)
    assert len(r) == 3 and all(abs(x - y) < 0.01 for x, y in zip(r, (1.0, 2.0, 3.0)))


# ------------------------------------------------------------------ barrier
def test_barrier_zero_outside_threshold():
    """barrier_zero_outside_threshold."""
    L = O.lib()
    assert L.orc_barrier_energy(0.02, 0.01) == 0.0 and L.orc_barrier_energy(0.01, 0.01) == 0.0
    assert L.orc_barrier_gradient(0.02, 0.01) == 0.0 and L.orc_barrier_hessian(0.02, 0.01) == 0.0


def test_barrier_inside_threshold():
    """barrier_positive_inside_threshold, barrier_increases_near_zero,
    barrier_gradient_negative_repulsive, barrier_hessian_positive_definite,
    barrier_continuous_at_threshold."""
    L = O.lib()
    assert L.orc_barrier_energy(0.005, 0.01) > 0.0
    assert L.orc_barrier_energy(0.001, 0.01) > L.orc_barrier_energy(0.005, 0.01)
    assert L.orc_barrier_gradient(0.005, 0.01) < 0.0
    assert L.orc_barrier_hessian(0.005, 0.01) > 0.0
    assert L.orc_barrier_energy(0.01 - 1e-6, 0.01) < 1e-10


def test_scaled_barrier_and_nonpositive_distance():
    """scaled_barrier_scales_correctly (through the scaled gradient the step
    uses) and barrier_massive_at_nonpositive_d."""
    L = O.lib()
    g, sg = L.orc_barrier_gradient(0.005, 0.01), L.orc_scaled_barrier_gradient(0.005, 0.01, 1000.0)
    assert abs(sg - 1000.0 * g) <= 1e-5 * abs(sg)
    assert L.orc_barrier_energy(0.0, 0.01) == 0.0
    assert L.orc_barrier_gradient(0.0, 0.01) < -5.0


def test_adaptive_kappa():
    """adaptive_kappa_scales_with_mass and adaptive_kappa_respects_override."""
    L = O.lib()
    k1, k2 = L.orc_estimate_kappa(0.0, 0.001, 9.81, 1e-3), L.orc_estimate_kappa(0.0, 0.01, 9.81, 1e-3)
    assert k2 > k1 > 0.0 and k2 < 1e8
    assert L.orc_estimate_kappa(5000.0, 0.001, 9.81, 1e-3) == 5000.0


def test_barrier_with_thickness():
    """barrier_with_thickness_increases_min_distance and thickness_gradient_repulsive."""
    L = O.lib()
    d_hat, t = 0.01, 0.001
    t2 = float(np.float32(t) * np.float32(t))
    assert L.orc_barrier_energy_thick(t2, d_hat, t) > 1e5
    assert L.orc_barrier_energy_thick(t2 + d_hat + 0.001, d_hat, t) == 0.0
    assert L.orc_barrier_energy_thick(t2 + d_hat * 0.5, d_hat, t) > 0.0
    assert L.orc_barrier_gradient_thick(t2 + d_hat * 0.01, d_hat, t) < 0.0


# ---------------------------------------------------------- IPC contact set
def test_ipc_vertex_triangle_contact():
    """ipc_detect_close_vertex_triangle, ipc_barrier_energy_positive,
    ipc_gradient_nonzero, ipc_constraint_violation (d_hat 0.1, kappa 1e4):
    vertex (0.25, 0.25, 0.05) over the unit right triangle is one contact with
    positive energy, a gradient that pushes the vertex out (+z) and no
    violation; ipc_detect_far_vertex_triangle: (10, 10, 10) is none at 0.01."""
    L = O.lib()
    d, _ = pt((0.25, 0.25, 0.05), A, B, CC)
    assert d < 0.1
    assert 1e4 * L.orc_barrier_energy(d, 0.1) > 0.0
    g = grad(L.orc_pt_grad, (0.25, 0.25, 0.05), A, B, CC)
    force_z = -L.orc_scaled_barrier_gradient(d, 0.1, 1e4) * g[0, 2]
    assert force_z > 0.0 and float(np.sum(g[0] ** 2)) > 0.0
    assert d > 1e-12  # no violation
    assert not pt((10.0, 10.0, 10.0), A, B, CC)[0] < 0.01


# ------------------------------------------------------------------- math
def polar(f):
    f = np.asarray(f, np.float32)
    rot, st, sv = np.zeros(6, np.float32), np.zeros(4, np.float32), np.zeros(2, np.float32)
    O.lib().orc_polar(*[a.ctypes.data_as(C.POINTER(C.c_float)) for a in (f, rot, st, sv)])
    return rot, st, sv


def test_polar_decomposition():
    """polar_identity, polar_scaled, polar_degenerate_does_not_panic."""
    rot, st, _ = polar([1, 0, 0, 0, 1, 0])
    assert abs(rot[0] - 1) < 1e-4 and abs(rot[1]) < 1e-4 and abs(rot[4] - 1) < 1e-4
    assert abs(st[0] - 1) < 1e-4 and abs(st[3] - 1) < 1e-4
    _, st, _ = polar([2, 0, 0, 0, 2, 0])
    assert abs(st[0] - 2) < 1e-4 and abs(st[3] - 2) < 1e-4
    rot, st, _ = polar([0] * 6)
    assert np.isfinite(rot).all() and np.isfinite(st).all()


def test_sparse_solver_cases():
    """faer_identity_solve, faer_spd_matrix_solve, faer_factorize_then_multi_solve,
    faer_large_laplacian, faer_non_square_fails, faer_empty_matrix_fails."""
    st, x = O.sparse_solve(3, 3, [(0, 0, 1.0), (1, 1, 1.0), (2, 2, 1.0)], [3.0, 7.0, -2.0])
    assert st == 0 and np.abs(x - [3.0, 7.0, -2.0]).max() < 1e-5
    spd = [(0, 0, 4.0), (0, 1, 1.0), (1, 0, 1.0), (1, 1, 3.0), (1, 2, 1.0), (2, 1, 1.0), (2, 2, 2.0)]
    st, x = O.sparse_solve(3, 3, spd, [1.0, 2.0, 3.0])
    A3 = np.array([[4, 1, 0], [1, 3, 1], [0, 1, 2]], np.float64)
    assert st == 0 and np.abs(A3 @ x - [1, 2, 3]).max() < 1e-4
    diag = [(0, 0, 2.0), (1, 1, 3.0), (2, 2, 5.0)]
    assert np.abs(O.sparse_solve(3, 3, diag, [4.0, 9.0, 25.0])[1] - [2, 3, 5]).max() < 1e-5
    assert np.abs(O.sparse_solve(3, 3, diag, [1.0, 1.0, 1.0])[1] - [0.5, 1 / 3, 0.2]).max() < 1e-5
    n = 100
    lap = [(i, i, 2.1) for i in range(n)] + [(i, i - 1, -1.0) for i in range(1, n)] + \
          [(i, i + 1, -1.0) for i in range(n - 1)]
    st, x = O.sparse_solve(n, n, lap, np.ones(n))
    ax = 2.1 * x.astype(np.float64)
    ax[1:] -= x[:-1]
    ax[:-1] -= x[1:]
    assert st == 0 and np.abs(ax - 1.0).max() < 1e-3
    assert O.sparse_solve(2, 3, [(0, 0, 1.0)], [1.0, 1.0])[0] == 1
    assert O.sparse_solve(0, 0, [], [])[0] == 2


# -------------------------------------------------------------- PD solver
def grid_sim(cols, rows, pinned=(), **cfg):
    """SolverConfig::debug() (3 iterations, tolerance 1e-3) on init's defaults
    (pd_solver.rs:221-246): stiffness 1.0 x 1000, bending 0.5 x 100, 200 g/m^2."""
    px, py, pz, tris = scenarios.quad_grid(cols, rows, 1.0, 1.0)
    pin = np.zeros(px.shape[0], np.uint8)
    pin[list(pinned)] = 1
    mesh = scenarios.Mesh(px, py, pz, tris, pin)
    base = dict(max_iterations=3, tolerance=1e-3, rayleigh_mass_damping=2.0, damping=0.01)
    base.update(cfg)
    return O.OracleSim(mesh, O.init_params(stiffness=1000.0, bend_stiffness=50.0, density_gsm=200.0),
                       O.default_config(**base), precision=0), mesh


def test_pinned_vertices_stay():
    """pd_solver_pinned_vertices_stay (solver_tests.rs:418-451): 5 steps."""
    sim, mesh = grid_sim(4, 4, pinned=(0, 4))
    y0 = sim.state()[0][:, 1].copy()
    for _ in range(5):
        sim.step(1.0 / 60.0)
    y = sim.state()[0][:, 1]
    assert abs(y[0] - y0[0]) < 1e-6 and abs(y[4] - y0[4]) < 1e-6


def test_gravity_pulls_centroid_down():
    """pd_solver_gravity_pulls_down (solver_tests.rs:453-483): 10 steps."""
    sim, _ = grid_sim(3, 3)
    c0 = float(sim.state()[0][:, 1].mean())
    for _ in range(10):
        sim.step(1.0 / 60.0)
    assert float(sim.state()[0][:, 1].mean()) < c0


def test_rayleigh_damping_reduces_kinetic_energy():
    """solver_rayleigh_damping_reduces_ke (solver_tests.rs:720-766): 20 steps of
    3 iterations, Rayleigh 0 against 5; kinetic energy with the state's 0.01 kg."""
    ke = []
    for alpha in (0.0, 5.0):
        sim, _ = grid_sim(5, 5, max_iterations=3, tolerance=1e-6, rayleigh_mass_damping=alpha)
        for _ in range(20):
            sim.step(1.0 / 60.0)
        v = sim.state()[1].astype(np.float64)
        ke.append(0.5 * 0.01 * float(np.sum(v * v)))
    assert ke[1] < ke[0], ke


def test_bending_elements_and_flat_rest_angles():
    """bending_element_count_matches_interior_edges (4x4 grid: 40 interior
    edges), bending_rest_angle_flat_mesh and bending_flat_rest_angles_exactly_pi
    (5x5 grid: every rest angle is exactly the f32 pi)."""
    sim, _ = grid_sim(4, 4)
    assert len(sim.hinges()[1]) == 40
    sim, _ = grid_sim(5, 5)
    rest = sim.hinges()[1]
    assert len(rest) and np.all(rest == np.float32(PI32))
