"""The simulation I/O contract (vistio_b200.io; crates/vistio-io/src/
contract.rs, validator.rs): JSON in the reference's serde shape, the
validator's checks and messages, the material database, and the material
set-up mapping. CPU only; the GPU run is in tests/test_gpu_io.py."""
import json

import numpy as np
import pytest

from vistio_b200 import _lib as L
from vistio_b200 import api, scenarios
from vistio_b200 import io as vio


def sample_input(side=6):
    mesh = scenarios.hanging_sheet(side, 0.5)
    return vio.SimulationInput(vio.TriangleMesh.from_mesh(mesh), None, [bool(p) for p in mesh.pinned],
                               vio.SimulationParams(duration=0.1))


def test_json_shape_and_round_trip():
    inp = sample_input()
    d = json.loads(inp.to_json())
    assert set(d) == {"garment", "body", "pinned", "params"}
    assert d["body"] is None
    assert set(d["garment"]) == {"pos_x", "pos_y", "pos_z", "normal_x", "normal_y", "normal_z", "uv_u", "uv_v",
                                 "indices", "material_ids"}
    assert all(isinstance(m, int) for m in d["garment"]["material_ids"])  # MaterialId(u16) serialises bare
    assert set(d["params"]) == {"duration", "dt", "iterations", "gravity", "gravity_direction",
                                "contact_thickness", "material_name"}
    back = vio.SimulationInput.from_json(inp.to_json())
    assert back == inp
    with pytest.raises(L.VistioError) as e:
        vio.SimulationInput.from_json('{"garment": {}}')
    assert e.value.status == 5


def test_defaults_match_reference_constants():
    p = vio.SimulationParams()
    assert (p.duration, p.iterations, p.gravity, p.gravity_direction, p.contact_thickness, p.material_name) == (
        2.0, 10, 9.81, (0.0, -1.0, 0.0), 0.005, "cotton_twill")
    assert abs(p.dt - 1.0 / 60.0) < 1e-12


@pytest.mark.parametrize("mutate,status,message", [
    (lambda i: i.garment.pos_y.pop(), 1, "Garment mesh: Position arrays have inconsistent lengths"),
    (lambda i: i.garment.uv_u.pop(), 1, "Garment mesh: UV arrays have inconsistent lengths"),
    (lambda i: i.garment.indices.pop(), 1, "Garment mesh: Index count is not divisible by 3"),
    (lambda i: i.garment.material_ids.pop(), 1, "Garment mesh: Material IDs count (49) != triangle count (50)"),
    (lambda i: i.garment.indices.__setitem__(4, 999), 1,
     "Garment mesh: Index 999 at position 4 is out of range (vertex count: 36)"),
    (lambda i: i.garment.indices.__setitem__(4, i.garment.indices[3]), 1, "Garment mesh: Triangle 1 has repeated"),
    (lambda i: i.pinned.pop(), 1, "Pinned array length (35) != garment vertex count (36)"),
    (lambda i: setattr(i.params, "dt", 0.0), 3, "Timestep dt must be positive"),
    (lambda i: setattr(i.params, "dt", 2.0), 3, "Timestep dt > 1.0 is unreasonably large"),
    (lambda i: setattr(i.params, "duration", 0.0), 3, "Duration must be positive"),
    (lambda i: setattr(i.params, "iterations", 0), 3, "Solver iterations must be >= 1"),
    (lambda i: setattr(i.params, "gravity", -1.0), 3, "Gravity magnitude must be non-negative"),
    (lambda i: setattr(i.params, "contact_thickness", -1.0), 3, "Contact thickness must be non-negative"),
    (lambda i: setattr(i.params, "gravity_direction", (0.0, -2.0, 0.0)), 3,
     "Gravity direction should be unit length, got magnitude 2"),
])
def test_validator_checks_and_messages(mutate, status, message):
    """validator.rs:17-90 and mesh.rs:118-172, message for message."""
    inp = sample_input(5)  # 36 vertices, 50 triangles
    vio.validate_input(inp)
    mutate(inp)
    with pytest.raises(L.VistioError) as e:
        vio.validate_input(inp)
    assert e.value.status == status
    assert message in str(e.value), str(e.value)


def test_material_database_and_setup():
    """database.rs:80-160: five presets by name; each maps to the set-up the
    runner's material path builds (anisotropic fabrics: the anisotropic
    co-rotational model with the warp / weft stretch stiffnesses and
    anisotropic Discrete Shells)."""
    assert sorted(vio.MATERIALS) == ["chiffon", "cotton_twill", "denim_14oz", "jersey_knit", "silk_charmeuse"]
    cot = vio.material("cotton_twill")
    assert (cot.density, cot.stretch_stiffness_warp, cot.bending_stiffness_weft) == (200.0, 0.90, 0.45)
    s = vio.setup_for(cot, 1.0 / 60.0)
    assert s.model == api.MODEL_ANISOTROPIC and s.bending == api.BENDING_DISCRETE_SHELLS_ANISOTROPIC
    assert s.stiffness == float(np.float32((np.float32(0.9) + np.float32(0.85)) / np.float32(2) * np.float32(10)))
    assert (s.warp_stiffness, s.weft_stiffness) == (0.90, 0.85)
    iso = api.FabricProperties(stretch_stiffness_warp=1.0, stretch_stiffness_weft=1.0)
    s = vio.setup_for(iso, 1.0 / 60.0)
    assert s.model == api.MODEL_COROTATIONAL and s.bending == api.BENDING_DIHEDRAL
    with pytest.raises(L.VistioError) as e:
        vio.material("tweed")
    assert e.value.status == 2


@pytest.mark.parametrize("value,text", [
    (0.1, "0.1"), (1.0, "1.0"), (100.0, "100.0"), (1234.5, "1234.5"), (-2.5, "-2.5"), (0.0, "0.0"),
    (-0.0, "-0.0"), (1e-7, "1e-7"), (1.5e20, "1.5e20"), (0.000123, "0.000123"), (1e-6, "0.000001"),
    (1e13, "1e13"), (9999e9, "9999000000000.0"), (123456789.0, "123456790.0"), (float("nan"), "null"),
    (float("inf"), "null"),
])
def test_json_f32_text(value, text):
    """An f32 in JSON: the shortest decimal that reads back as the same f32."""
    assert vio._json_f32(value) == text


def test_json_f32_round_trips():
    rng = np.random.default_rng(3)
    a = (10 ** rng.uniform(-9, 20, 20000)).astype(np.float32) * np.where(rng.random(20000) < 0.5, -1, 1)
    a = a.astype(np.float32)
    text = vio._json_f32_array(a)
    assert np.array_equal(np.array(json.loads(text), np.float32), a)
    assert text == "[" + ",".join(vio._json_f32(x) for x in a) + "]"


def test_json_frame_exporter(tmp_path):
    """json_exporter.rs:39-104: init from the mesh, one frame per submit, the
    whole animation written compactly on finalize, frames handed over."""
    mesh = scenarios.hanging_sheet(3, 1.0)
    path = tmp_path / "anim.json"
    e = vio.JsonFrameExporter(str(path))
    assert e.name() == "json_exporter" and e.frame_count() == 0
    e.init(vio.TriangleMesh.from_mesh(mesh))
    x = np.stack([mesh.px, mesh.py, mesh.pz], 1)
    for t in range(3):
        e.submit_frame(t, x + np.float32(0.1) * t)
    assert e.frame_count() == 3
    e.finalize()
    assert e.frame_count() == 0
    text = path.read_text()
    assert " " not in text and text.startswith('{"vertex_count":16,"triangle_count":18,"indices":[')
    d = json.loads(text)
    assert list(d) == ["vertex_count", "triangle_count", "indices", "frames"]
    assert d["indices"] == [int(i) for i in mesh.tris.ravel()]
    assert [f["timestep"] for f in d["frames"]] == [0, 1, 2]
    for t, f in enumerate(d["frames"]):
        assert list(f) == ["timestep", "positions"]
        np.testing.assert_array_equal(np.array(f["positions"], np.float32), (x + np.float32(0.1) * t).ravel())
    # a scenarios.Mesh initialises the same way
    e2 = vio.JsonFrameExporter(str(tmp_path / "b.json"))
    e2.init(mesh)
    assert (e2.vertex_count, e2.triangle_count, e2.indices) == (16, 18, d["indices"])


def test_json_frame_exporter_write_error(tmp_path):
    e = vio.JsonFrameExporter(str(tmp_path / "missing" / "a.json"))
    e.init(scenarios.hanging_sheet(2, 1.0))
    with pytest.raises(L.VistioError) as err:
        e.finalize()
    assert err.value.status == 4
