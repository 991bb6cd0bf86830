"""GPU runs of the simulation I/O contract (vistio_b200.io.simulate): the
output's draped mesh equals stepping the same garment through the solver's
material path directly, the metrics are consistent with the run, and the
output survives a JSON round trip."""
import json

import numpy as np
import pytest

from vistio_b200 import api, scenarios
from vistio_b200 import io as vio

pytestmark = pytest.mark.gpu


def test_simulate_equals_the_material_path():
    mesh = scenarios.hanging_sheet(14, 0.6)
    inp = vio.SimulationInput(vio.TriangleMesh.from_mesh(mesh), None, [bool(p) for p in mesh.pinned],
                              vio.SimulationParams(duration=0.25, iterations=10, material_name="denim_14oz"))
    out = vio.simulate(inp)
    # the reference runner's path for an anisotropic fabric (runner.rs:100-140)
    props = vio.MATERIALS["denim_14oz"]
    cfg = api.SolverConfig(max_iterations=10)
    s = api.ProjectiveDynamicsSolver().init_with_material_tier3(
        mesh, cfg, props, api.MODEL_ANISOTROPIC, pinned=mesh.pinned,
        warp=props.stretch_stiffness_warp, weft=props.stretch_stiffness_weft)
    for _ in range(15):
        s.step(1.0 / 60.0)
    x = s.state()[0]
    d = out.draped_mesh
    assert np.array_equal(np.stack([d.pos_x, d.pos_y, d.pos_z], 1).astype(np.float32), x)
    m = out.metrics
    assert m.timestep_count == 15 and m.avg_iterations == 10.0 and m.max_penetration == 0.0
    assert np.isfinite(m.final_energy) and m.max_strain == max(out.vertex_metadata.strain)
    assert not any(out.vertex_metadata.contact_force)
    back = vio.SimulationOutput.from_json(out.to_json())
    assert back.metrics == out.metrics and back.draped_mesh == out.draped_mesh
    assert set(json.loads(out.to_json())) == {"draped_mesh", "vertex_metadata", "metrics"}


def test_simulate_with_contact():
    """A sheet dropped onto the sphere collider: contact forces are reported
    where the sheet touches, and the final penetration stays within the
    barrier's tolerance (bench_tests.rs:138-225: 2 cm)."""
    mesh = scenarios.sphere_drape(side=16, length=1.0, height=0.36)
    inp = vio.SimulationInput(vio.TriangleMesh.from_mesh(mesh), None, [False] * mesh.nv,
                              vio.SimulationParams(duration=0.5, iterations=15, material_name="cotton_twill"))
    sphere = api.Contact(has_ground=True, ground_height=-0.3, has_sphere=True, sphere_center=(0.0, 0.0, 0.0),
                         sphere_radius=0.3)
    out = vio.simulate(inp, sphere)
    f = np.asarray(out.vertex_metadata.contact_force)
    assert f.shape == (mesh.nv,) and (f > 0).any()
    assert out.metrics.max_penetration <= 0.02
    assert out.metrics.timestep_count == 30


def test_simulate_non_ipc_with_exporter(tmp_path):
    """ipc=False: a plain step then the colliders' projections each step (the
    runner's non-IPC branch), the same as driving the solver directly; the
    exporter receives every step's positions."""
    mesh = scenarios.sphere_drape(side=12, length=0.6, height=0.13)
    box = api.Contact(has_ground=True, ground_height=-0.3, has_box=True, box_min=(-0.2, -0.1, -0.2),
                      box_max=(0.2, 0.1, 0.2))
    inp = vio.SimulationInput(vio.TriangleMesh.from_mesh(mesh), None, [False] * mesh.nv,
                              vio.SimulationParams(duration=0.2, iterations=10, material_name="cotton_twill"))
    e = vio.JsonFrameExporter(str(tmp_path / "frames.json"))
    out = vio.simulate(inp, contact=box, ipc=False, exporter=e)
    props = vio.MATERIALS["cotton_twill"]
    s = api.ProjectiveDynamicsSolver().init_explicit(mesh, vio.solver_config(inp.params),
                                                     vio.setup_for(props, inp.params.dt), pinned=mesh.pinned)
    s.set_ground(-0.3)
    boxed = 0
    frames = []
    for _ in range(12):
        s.step(inp.params.dt)
        boxed += s.resolve_contacts(box).box.resolved_count
        frames.append(s.state()[0])
    d = out.draped_mesh
    assert np.array_equal(np.stack([d.pos_x, d.pos_y, d.pos_z], 1).astype(np.float32), frames[-1])
    assert boxed > 0 and out.metrics.timestep_count == 12
    assert not any(out.vertex_metadata.contact_force)
    assert e.frame_count() == 12
    e.finalize()
    got = json.loads((tmp_path / "frames.json").read_text())
    assert [f["timestep"] for f in got["frames"]] == list(range(12))
    for f, x in zip(got["frames"], frames):
        assert np.array_equal(np.array(f["positions"], np.float32), x.ravel())
