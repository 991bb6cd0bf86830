"""CPU checks of the cylinder and box colliders of the oracle
(CylinderCollider / BoxCollider::detect_ipc_contacts, crates/vistio-contact/
src/cylinder.rs:121-198 and box_collider.rs:107-200) on single vertices whose
distances are known in closed form, and of the disc generator of the Cusick
drape (generators.rs:174-240). The GPU kernels are checked against this oracle
in tests/test_gpu_contact.py."""
import math

import numpy as np
import pytest

import oracle_api as O
from vistio_b200 import scenarios

D_HAT, KAPPA = 1e-3, 1e4


def one_vertex_sim():
    mesh = scenarios.hanging_sheet(1, 1.0)  # 4 vertices, 2 triangles
    return O.OracleSim(mesh, O.init_params(), O.default_config(), precision=1), mesh.nv


def detect_at(contact, point):
    sim, n = one_vertex_sim()
    pos = np.full((n, 3), 50.0, np.float32)  # the other vertices far from everything
    pos[0] = point
    g, nrm, inc, mv, act = sim.detect(contact, D_HAT, pos)
    return g[0].astype(np.float64), inc[0], mv, act


def barrier_force(dsq):
    """scaled_barrier_gradient(d^2) * 2 d, the gradient along the outward
    direction: negative (the energy falls as the distance grows)."""
    return float(O.lib().orc_scaled_barrier_gradient(dsq, D_HAT, KAPPA)) * 2.0 * math.sqrt(dsq)


def cylinder():
    c = O.Contact()
    c.has_cylinder = 1
    c.cylinder_center_x, c.cylinder_center_z, c.cylinder_top_y, c.cylinder_radius = 0.1, -0.2, 0.3, 0.09
    c.kappa = KAPPA
    return c


def box():
    c = O.Contact()
    c.has_box = 1
    c.box_min[:] = (-0.1, 0.0, -0.2)
    c.box_max[:] = (0.1, 0.499, 0.0)
    c.kappa = KAPPA
    return c


@pytest.mark.parametrize("point,direction,dist", [
    ((0.1, 0.32, -0.2), (0, 1, 0), 0.02),                           # over the top face
    ((0.1 + 0.09 + 0.015, 0.1, -0.2), (1, 0, 0), 0.015),           # beside the wall
    ((0.1, 0.1, -0.2 - 0.09 - 0.02), (0, 0, -1), 0.02),            # beside the wall, -z
])
def test_cylinder_barrier_face_and_wall(point, direction, dist):
    g, inc, mv, act = detect_at(cylinder(), point)
    assert act == 1 and mv == 0.0
    assert inc == 0  # the pipeline gives cylinder contacts no normal (collision_pipeline.rs:305-310)
    expect = barrier_force(dist * dist) * np.asarray(direction, np.float64)
    assert np.allclose(g, expect, rtol=1e-4, atol=1e-9), (g, expect)


def test_cylinder_rim_and_inside_and_far():
    # above and outside: the distance to the rim circle
    ds, dt = 0.01, 0.012
    g, _, mv, act = detect_at(cylinder(), (0.1 + 0.09 + ds, 0.3 + dt, -0.2))
    d = math.hypot(ds, dt)
    assert act == 1 and mv == 0.0
    assert np.allclose(g, barrier_force(d * d) * np.array([ds / d, dt / d, 0.0]), rtol=1e-4)
    # inside, nearer the wall than the top face: the way out is radial (+x here),
    # at the tiny distance 1e-12; the violation is the depth
    g, _, mv, act = detect_at(cylinder(), (0.1 + 0.08, 0.2, -0.2))
    assert act == 1 and abs(mv - 0.01) < 1e-6
    assert g[0] < 0 and abs(g[1]) < 1e-9 * abs(g[0]) and abs(g[2]) < 1e-9 * abs(g[0])
    # inside, nearer the top face: the way out is up
    g, _, mv, act = detect_at(cylinder(), (0.1, 0.295, -0.2))
    assert act == 1 and abs(mv - 0.005) < 1e-6 and g[1] < 0 and g[0] == 0 and g[2] == 0
    # farther than sqrt(d_hat) (d_hat is compared with the squared distance)
    g, _, mv, act = detect_at(cylinder(), (0.1, 0.3 + 0.04, -0.2))
    assert act == 0 and not g.any()


def test_box_faces_edges_corners_and_inside():
    c = box()
    # over the top face (the cantilever shelf's top at y = 0.499)
    g, inc, mv, act = detect_at(c, (0.0, 0.519, -0.1))
    assert act == 1 and inc == 0 and mv == 0.0
    assert np.allclose(g, barrier_force(0.02 ** 2) * np.array([0, 1.0, 0]), rtol=1e-4)
    # beyond an edge (x and z outside): distance to the edge, direction (1, 0, 1)/sqrt 2 scaled by q
    q = 0.01
    g, _, _, act = detect_at(c, (0.1 + q, 0.25, 0.0 + q))
    d = math.sqrt(2) * q
    assert act == 1
    assert np.allclose(g, barrier_force(d * d) * np.array([q / d, 0.0, q / d]), rtol=1e-4)
    # beyond a corner, on the -x, -y, -z side
    g, _, _, act = detect_at(c, (-0.1 - q, -q, -0.2 - q))
    d = math.sqrt(3) * q
    assert act == 1
    assert np.allclose(g, barrier_force(d * d) * np.array([-q / d, -q / d, -q / d]), rtol=1e-4)
    # inside, nearest the -z face: the way out is -z, violation = depth
    g, _, mv, act = detect_at(c, (0.0, 0.25, -0.19))
    assert act == 1 and abs(mv - 0.01) < 1e-6
    assert g[2] > 0 and g[0] == 0 and g[1] == 0
    # far
    g, _, _, act = detect_at(c, (0.5, 0.25, -0.1))
    assert act == 0 and not g.any()


def test_cusick_disc_mesh():
    """circular_grid(0.15, 64): a 32 x 32 grid of side 0.3 keeps the vertices
    within 1.01 r and the cells whose four corners it kept, two triangles each
    with the quad grid's checkerboard diagonals; the Cusick drape turns it into
    the XZ plane at y = 0.5."""
    px, py, pz, tris = scenarios.circular_grid(0.15, 64)
    r = np.sqrt(px.astype(np.float64) ** 2 + py.astype(np.float64) ** 2)
    assert r.max() <= 0.15 * 1.01 + 1e-6
    assert not pz.any()
    n = 32
    grid = {(round(float(x) * 1e6), round(float(y) * 1e6)): k for k, (x, y) in enumerate(zip(px, py))}
    assert len(grid) == px.shape[0]
    cells = 0
    for j in range(n):
        for i in range(n):
            x0, y0 = -0.15 + i * 0.3 / n, 0.15 - j * 0.3 / n
            corners = [(x0, y0), (x0 + 0.3 / n, y0), (x0, y0 - 0.3 / n), (x0 + 0.3 / n, y0 - 0.3 / n)]
            keys = [(round(x * 1e6), round(y * 1e6)) for x, y in corners]
            cells += all(k in grid for k in keys)
    assert tris.shape[0] == 2 * cells
    m = scenarios.cusick_drape()
    assert np.all(m.py == np.float32(0.5)) and np.array_equal(m.pz, py) and not m.pinned.any()
