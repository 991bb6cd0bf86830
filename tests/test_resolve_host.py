"""CPU checks of the oracle's collider projections, the runner's non-IPC
collision step (CollisionPipeline::step with thickness 0, crates/vistio-
contact/src/collision_pipeline.rs:117-199): the reference's own ground-plane
tests (crates/vistio-contact/tests/contact_tests.rs:246-298) and single
vertices whose projections follow by hand from ground_plane.rs:26-65,
sphere.rs:29-100, cylinder.rs:30-118 and box_collider.rs:26-99. The GPU
kernel is checked against this oracle in tests/test_gpu_resolve.py."""
import numpy as np
import pytest

import oracle_api as O
from vistio_b200 import scenarios

F = np.float32


def sim_at(rest_y=0.0, pinned=None, cols=4):
    """An oracle state on quad_grid(cols, cols, 1, 1); every vertex's previous
    position (the rest position before any step) at height rest_y."""
    px, py, pz, tris = scenarios.quad_grid(cols, cols, 1.0, 1.0)
    n = px.shape[0]
    pin = np.zeros(n, np.uint8) if pinned is None else pinned
    mesh = scenarios.Mesh(px, np.full(n, F(rest_y)), py.copy(), tris, pin)
    return O.OracleSim(mesh, O.init_params(), O.default_config(), precision=0), n


def contact(**kw):
    c = O.Contact()
    for k, v in kw.items():
        if isinstance(v, tuple):
            getattr(c, k)[:] = v
        else:
            setattr(c, k, v)
    return c


def place(sim, n, pos, vel):
    """Put the first len(pos) vertices at pos with vel; the rest far away at rest."""
    P = np.full((n, 3), 50.0, F)
    V = np.zeros((n, 3), F)
    P[: len(pos)] = pos
    V[: len(vel)] = vel
    sim.set_state(P, V)


def test_ground_plane_prevents_penetration():
    """contact_tests.rs:246-282: every vertex at y = -1 moving down at 5 m/s."""
    sim, n = sim_at()
    p, _ = sim.state()
    p[:, 1] = -1.0
    v = np.zeros_like(p)
    v[:, 1] = -5.0
    v[:, 0] = 2.0
    sim.set_state(p, v)
    r = sim.resolve(contact(has_ground=1, ground_height=0.0))
    assert r[0, 0] == n
    assert r[0, 1] > 0.0 and r[0, 2] == pytest.approx(n * 1.0)
    p, v = sim.state()
    assert (p[:, 1] >= 0.0).all() and (v[:, 1] >= 0.0).all()
    assert np.all(v[:, 0] == 1.0)  # tangential friction 0.5
    assert r[1:].sum() == 0


def test_ground_plane_no_correction_above():
    """contact_tests.rs:284-298."""
    sim, n = sim_at(cols=2)
    p, v = sim.state()
    p[:, 1] = 5.0
    sim.set_state(p, v)
    assert sim.resolve(contact(has_ground=1, ground_height=0.0))[0, 0] == 0


def test_sphere_surface_and_centre():
    sim, n = sim_at()
    c = contact(has_sphere=1, sphere_center=(0.0, 0.0, 0.0), sphere_radius=0.5)
    place(sim, n, [(0.25, 0.0, 0.0), (0.0, 0.0, 0.0), (0.0, 0.2, 0.0)], [(-1.0, 0.5, 0.0), (3.0, 1.0, 2.0),
                                                                          (0.0, 1.0, 0.0)])
    r = sim.resolve(c)
    p, v = sim.state()
    np.testing.assert_array_equal(p[0], F([0.5, 0.0, 0.0]))   # pushed out along +x
    np.testing.assert_array_equal(v[0], F([0.0, 0.25, 0.0]))  # inward part gone, the rest halved
    np.testing.assert_array_equal(p[1], F([0.0, 0.5, 0.0]))   # the centre: straight up
    np.testing.assert_array_equal(v[1], F([0.0, 0.0, 0.0]))
    np.testing.assert_array_equal(p[2], F([0.0, 0.5, 0.0]))
    np.testing.assert_array_equal(v[2], F([0.0, 1.0, 0.0]))   # moving out: velocity kept
    assert r[1, 0] == 3 and r[1, 1] == F(0.5)


def test_cylinder_top_side_and_previous_height():
    cyl = dict(has_cylinder=1, cylinder_center_x=0.0, cylinder_center_z=0.0, cylinder_top_y=0.3,
               cylinder_radius=0.1)
    # previous positions below the top: the shallower of the side and the top wins
    sim, n = sim_at(rest_y=-1.0)
    place(sim, n, [(0.08, 0.0, 0.0), (0.0, 0.29, 0.05), (0.05, 0.31, 0.0), (0.0, 0.1, 0.0)],
          [(-1.0, -1.0, 1.0), (1.0, -2.0, 1.0), (0.0, -1.0, 0.0), (1.0, 1.0, 1.0)])
    r = sim.resolve(contact(**cyl))
    p, v = sim.state()
    np.testing.assert_allclose(p[0], [0.1, 0.0, 0.0], atol=1e-7)   # out through the wall
    np.testing.assert_allclose(v[0], [0.0, -0.7, 1.0], atol=1e-7)  # radial inflow gone, vertical x 0.7
    np.testing.assert_array_equal(p[1], F([0.0, 0.3, 0.05]))       # up through the top
    np.testing.assert_allclose(v[1], [0.1, 0.0, 0.1], atol=1e-7)
    np.testing.assert_array_equal(p[2], F([0.05, 0.31, 0.0]))      # above the top: untouched
    np.testing.assert_array_equal(p[3], F([0.0, 0.3, 0.0]))        # on the axis: up
    assert r[2, 0] == 3
    # previous positions above the top: up even where the wall is closer
    sim, n = sim_at(rest_y=1.0)
    place(sim, n, [(0.08, 0.0, 0.0)], [(0.0, -1.0, 0.0)])
    sim.resolve(contact(**cyl))
    np.testing.assert_array_equal(sim.state()[0][0], F([0.08, 0.3, 0.0]))


@pytest.mark.parametrize("rest_y,point,expect,vel_expect", [
    (-1.0, (-0.95, 0.5, 0.2), (-1.0, 0.5, 0.2), (0.0, 0.7, 0.7)),   # -x face
    (-1.0, (0.9, 0.5, 0.2), (1.0, 0.5, 0.2), (1.0, 0.7, 0.7)),      # +x face
    (-1.0, (0.0, 0.95, 0.2), (0.0, 1.0, 0.2), (0.7, 1.0, 0.7)),     # +y face
    (-1.0, (0.0, 0.05, 0.2), (0.0, 0.0, 0.2), (0.7, 0.0, 0.7)),     # -y face
    (-1.0, (0.0, 0.5, 0.45), (0.0, 0.5, 0.5), (0.7, 0.7, 1.0)),     # +z face
    (-1.0, (0.0, 0.5, -0.45), (0.0, 0.5, -0.5), (0.7, 0.7, 0.0)),   # -z face
    (2.0, (-0.95, 0.5, 0.2), (-0.95, 1.0, 0.2), (0.7, 1.0, 0.7)),   # came from above: the top
    (-1.0, (-1.0, 0.5, 0.2), (-1.0, 0.5, 0.2), (0.0, 0.7, 0.7)),    # on the -x face: depth 0
])
def test_box_faces(rest_y, point, expect, vel_expect):
    sim, n = sim_at(rest_y=rest_y)
    place(sim, n, [point], [(1.0, 1.0, 1.0)])
    r = sim.resolve(contact(has_box=1, box_min=(-1.0, 0.0, -0.5), box_max=(1.0, 1.0, 0.5)))
    p, v = sim.state()
    np.testing.assert_allclose(p[0], expect, atol=1e-7)
    np.testing.assert_allclose(v[0], vel_expect, atol=1e-7)
    assert r[3, 0] == 1


def test_pinned_and_pipeline_order():
    """Pinned vertices stay; the ground runs before the sphere, so a vertex under
    the ground and inside the sphere is lifted and then pushed out."""
    pin = np.zeros(25, np.uint8)
    pin[1] = 1
    sim, n = sim_at(pinned=pin)
    place(sim, n, [(0.0, -0.2, 0.0), (0.0, -0.2, 0.0)], [(0.0, -1.0, 0.0), (0.0, -1.0, 0.0)])
    r = sim.resolve(contact(has_ground=1, ground_height=0.0, has_sphere=1, sphere_center=(0.0, -0.1, 0.0),
                            sphere_radius=0.3))
    p, v = sim.state()
    np.testing.assert_allclose(p[0], [0.0, 0.2, 0.0], atol=1e-7)  # ground to 0, then out of the sphere
    np.testing.assert_array_equal(p[1], F([0.0, -0.2, 0.0]))     # pinned
    assert r[0, 0] == 1 and r[1, 0] == 1
