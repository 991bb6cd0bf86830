"""The simulation input/output contract as a wire format for the solver.

`SimulationInput`, `SimulationParams`, `SimulationOutput`, `VertexMetadata` and
`SimulationMetrics` follow the reference's contract types field for field
(crates/vistio-io/src/contract.rs:13-105), and their JSON is the one the
reference's serde derives write: a `TriangleMesh` is an object of its arrays
(crates/vistio-mesh/src/mesh.rs:20-48), a `MaterialId` its bare number, an
absent body `null`. `validate_input` gives the reference's checks and
messages (crates/vistio-io/src/validator.rs:17-90, mesh.rs:118-172).

`SimulationParams.material_name` names a fabric of the reference's material
database (crates/vistio-material/src/database.rs:80-160, the same five
presets). `simulate` runs an input on the GPU solver the way the reference's
runner sets a material up (runner.rs:100-140: anisotropic fabrics get the
anisotropic co-rotational model and Discrete Shells bending, the others the
co-rotational model and dihedral bending) and fills the output from the final
state. The reference ships the contract without a consumer; the metrics'
definitions are therefore this module's and are stated at each field.

A body mesh is not simulated: the solver's obstacles are the analytical
colliders of `api.Contact` (ground, sphere, cylinder, box).

`JsonFrameExporter` writes an animation in the layout of the reference's
JSON frame exporter (crates/vistio-render/src/json_exporter.rs:14-104), with
every position printed as the shortest decimal that reads back as the same
f32, the form serde_json gives an f32.
"""
from __future__ import annotations

import dataclasses
import json
import math
import time
from typing import List, Optional

import numpy as np

from . import _lib as L
from . import api
from .scenarios import Mesh

# crates/vistio-types/src/constants.rs
GRAVITY = 9.81
DEFAULT_DT = 1.0 / 60.0
DEFAULT_PD_ITERATIONS = 10
DEFAULT_CONTACT_THICKNESS = 0.005


def _preset(density, sw, sf, sh, bw, bf, th, fr, dm):
    return api.FabricProperties(density=density, stretch_stiffness_warp=sw, stretch_stiffness_weft=sf,
                                shear_stiffness=sh, bending_stiffness_warp=bw, bending_stiffness_weft=bf,
                                thickness=th, friction=fr, damping=dm)


# MaterialDatabase::with_defaults (database.rs:22-33, presets 80-160)
MATERIALS = {
    "cotton_twill": _preset(200.0, 0.90, 0.85, 0.50, 0.50, 0.45, 0.0008, 0.50, 0.02),
    "silk_charmeuse": _preset(80.0, 0.70, 0.65, 0.30, 0.10, 0.08, 0.0004, 0.30, 0.01),
    "denim_14oz": _preset(400.0, 0.98, 0.92, 0.70, 0.85, 0.75, 0.0014, 0.60, 0.03),
    "jersey_knit": _preset(180.0, 0.50, 0.60, 0.25, 0.20, 0.25, 0.0006, 0.40, 0.02),
    "chiffon": _preset(50.0, 0.60, 0.55, 0.20, 0.05, 0.04, 0.0003, 0.20, 0.005),
}


def _f32(v):
    return [float(np.float32(x)) for x in v]


@dataclasses.dataclass
class TriangleMesh:
    """TriangleMesh (mesh.rs:20-48): SoA vertex arrays, flat indices, one
    material id per triangle."""
    pos_x: List[float]
    pos_y: List[float]
    pos_z: List[float]
    normal_x: List[float]
    normal_y: List[float]
    normal_z: List[float]
    uv_u: List[float]
    uv_v: List[float]
    indices: List[int]
    material_ids: List[int]

    def vertex_count(self) -> int:
        return len(self.pos_x)

    def triangle_count(self) -> int:
        return len(self.indices) // 3

    def validate(self):
        """TriangleMesh::validate (mesh.rs:118-172)."""
        n = len(self.pos_x)
        if len(self.pos_y) != n or len(self.pos_z) != n:
            raise L.VistioError(1, "Position arrays have inconsistent lengths")
        if len(self.normal_x) != n or len(self.normal_y) != n or len(self.normal_z) != n:
            raise L.VistioError(1, "Normal arrays have inconsistent lengths")
        if len(self.uv_u) != n or len(self.uv_v) != n:
            raise L.VistioError(1, "UV arrays have inconsistent lengths")
        if len(self.indices) % 3 != 0:
            raise L.VistioError(1, "Index count is not divisible by 3")
        tc = self.triangle_count()
        if len(self.material_ids) != tc:
            raise L.VistioError(1, f"Material IDs count ({len(self.material_ids)}) != triangle count ({tc})")
        for i, idx in enumerate(self.indices):
            if idx >= n:
                raise L.VistioError(1, f"Index {idx} at position {i} is out of range (vertex count: {n})")
        for t in range(tc):
            a, b, c = self.indices[3 * t:3 * t + 3]
            if a == b or b == c or a == c:
                raise L.VistioError(1, f"Triangle {t} has repeated vertex indices: [{a}, {b}, {c}]")

    @staticmethod
    def from_mesh(mesh: Mesh) -> "TriangleMesh":
        """A scenario mesh as a TriangleMesh: normals of the triangles around
        each vertex (area-weighted), uv from the bounding rectangle of x and
        the second in-plane axis, material 0."""
        pos = np.stack([mesh.px, mesh.py, mesh.pz], 1).astype(np.float32)
        nrm = _vertex_normals(pos, mesh.tris)
        lo, hi = pos.min(0), pos.max(0)
        ax = [k for k in range(3) if hi[k] - lo[k] > 0][:2] or [0, 1]
        ax += [ax[-1]] * (2 - len(ax))
        uv = [(pos[:, k] - lo[k]) / max(float(hi[k] - lo[k]), 1e-12) for k in ax]
        return TriangleMesh(_f32(mesh.px), _f32(mesh.py), _f32(mesh.pz), _f32(nrm[:, 0]), _f32(nrm[:, 1]),
                            _f32(nrm[:, 2]), _f32(uv[0]), _f32(uv[1]), [int(i) for i in mesh.tris.reshape(-1)],
                            [0] * int(mesh.tris.shape[0]))

    def to_mesh(self, pinned=None) -> Mesh:
        n = self.vertex_count()
        pin = np.zeros(n, np.uint8) if pinned is None else np.asarray(pinned, np.uint8)
        return Mesh(np.asarray(self.pos_x, np.float32), np.asarray(self.pos_y, np.float32),
                    np.asarray(self.pos_z, np.float32), np.asarray(self.indices, np.uint32).reshape(-1, 3), pin)


def _vertex_normals(pos: np.ndarray, tris: np.ndarray) -> np.ndarray:
    t = np.asarray(tris, np.int64).reshape(-1, 3)
    fn = np.cross(pos[t[:, 1]] - pos[t[:, 0]], pos[t[:, 2]] - pos[t[:, 0]]).astype(np.float64)
    acc = np.zeros((pos.shape[0], 3))
    for k in range(3):
        np.add.at(acc, t[:, k], fn)
    ln = np.linalg.norm(acc, axis=1, keepdims=True)
    return np.where(ln > 1e-20, acc / np.maximum(ln, 1e-20), np.array([0.0, 0.0, 1.0]))


@dataclasses.dataclass
class SimulationParams:
    """SimulationParams (contract.rs:31-63) with the reference's defaults."""
    duration: float = 2.0
    dt: float = DEFAULT_DT
    iterations: int = DEFAULT_PD_ITERATIONS
    gravity: float = GRAVITY
    gravity_direction: tuple = (0.0, -1.0, 0.0)
    contact_thickness: float = DEFAULT_CONTACT_THICKNESS
    material_name: str = "cotton_twill"


@dataclasses.dataclass
class SimulationInput:
    """SimulationInput (contract.rs:13-28)."""
    garment: TriangleMesh
    body: Optional[TriangleMesh]
    pinned: List[bool]
    params: SimulationParams

    def to_json(self) -> str:
        d = dataclasses.asdict(self)
        d["params"]["gravity_direction"] = list(d["params"]["gravity_direction"])
        return json.dumps(d)

    @staticmethod
    def from_json(text: str) -> "SimulationInput":
        try:
            d = json.loads(text)
            body = TriangleMesh(**d["body"]) if d.get("body") is not None else None
            p = dict(d["params"])
            p["gravity_direction"] = tuple(p["gravity_direction"])
            return SimulationInput(TriangleMesh(**d["garment"]), body, [bool(x) for x in d["pinned"]],
                                   SimulationParams(**p))
        except (KeyError, TypeError, ValueError) as e:
            raise L.VistioError(5, f"SimulationInput: {e}") from None


@dataclasses.dataclass
class VertexMetadata:
    """VertexMetadata (contract.rs:79-88)."""
    strain: List[float]         # per triangle: largest principal stretch of the final state - 1
    contact_force: List[float]  # per vertex: magnitude of the last contact detect's barrier gradient (0: none)


@dataclasses.dataclass
class SimulationMetrics:
    """SimulationMetrics (contract.rs:90-105)."""
    wall_time_seconds: float = 0.0
    timestep_count: int = 0
    final_energy: float = 0.0   # kinetic + gravitational (height along -gravity_direction) + membrane
    max_penetration: float = 0.0  # deepest final penetration of a collider (m)
    max_strain: float = 0.0
    avg_iterations: float = 0.0


@dataclasses.dataclass
class SimulationOutput:
    """SimulationOutput (contract.rs:66-76)."""
    draped_mesh: TriangleMesh
    vertex_metadata: VertexMetadata
    metrics: SimulationMetrics

    def to_json(self) -> str:
        return json.dumps(dataclasses.asdict(self))

    @staticmethod
    def from_json(text: str) -> "SimulationOutput":
        d = json.loads(text)
        return SimulationOutput(TriangleMesh(**d["draped_mesh"]), VertexMetadata(**d["vertex_metadata"]),
                                SimulationMetrics(**d["metrics"]))


def _json_f32(v) -> str:
    """The JSON text of an f32: the shortest decimal that reads back as the same
    float, positional for 1e-6 <= |v| < 1e13 ("0.1", "100.0", "0.000123"),
    else d.ddde<k> ("1e-7", "1.5e20"); a non-finite value is null."""
    f = np.float32(v)
    if not np.isfinite(f):
        return "null"
    if f == 0:
        return "-0.0" if np.signbit(f) else "0.0"
    mant, exp = np.format_float_scientific(f, unique=True, trim="-").split("e")
    neg = mant.startswith("-")
    digits = mant.lstrip("-").replace(".", "")
    n = len(digits)
    kk = int(exp) + 1  # 10^(kk-1) <= |v| < 10^kk
    k = kk - n         # the power of ten of the last digit
    if 0 <= k and kk <= 13:
        out = digits + "0" * k + ".0"
    elif 0 < kk <= 13:
        out = digits[:kk] + "." + digits[kk:]
    elif -6 < kk <= 0:
        out = "0." + "0" * (-kk) + digits
    elif n == 1:
        out = f"{digits}e{kk - 1}"
    else:
        out = f"{digits[0]}.{digits[1:]}e{kk - 1}"
    return "-" + out if neg else out


def _json_f32_array(a) -> str:
    out = []
    for x in np.asarray(a, np.float32).ravel():
        t = str(x)  # numpy's shortest text: the same where it is positional
        out.append(t if np.isfinite(x) and "e" not in t else _json_f32(x))
    return "[" + ",".join(out) + "]"


class JsonFrameExporter:
    """JsonFrameExporter (json_exporter.rs:39-104): collects the positions of
    every submitted frame and writes the whole animation to one JSON file on
    finalize(): {"vertex_count", "triangle_count", "indices", "frames":
    [{"timestep", "positions": [x0, y0, z0, x1, ...]}]}, compact as
    serde_json::to_string writes it. The frames are handed over on finalize()
    (frame_count() is 0 afterwards)."""

    def __init__(self, output_path: str):
        self.output_path = str(output_path)
        self.indices: List[int] = []
        self.vertex_count = 0
        self.triangle_count = 0
        self.frames: List[tuple] = []

    def init(self, mesh):
        """From a TriangleMesh of the contract or a scenarios.Mesh."""
        if isinstance(mesh, TriangleMesh):
            self.vertex_count, self.triangle_count = mesh.vertex_count(), mesh.triangle_count()
            self.indices = [int(i) for i in mesh.indices]
        else:
            self.vertex_count, self.triangle_count = mesh.nv, mesh.nt
            self.indices = [int(i) for i in np.asarray(mesh.tris).ravel()]

    def submit_frame(self, timestep: int, positions):
        """positions: (V, 3) (or the three coordinate arrays stacked that way)."""
        self.frames.append((int(timestep), np.array(positions, np.float32).reshape(-1, 3)))

    def finalize(self):
        frames, self.frames = self.frames, []
        parts = [f'{{"vertex_count":{self.vertex_count},"triangle_count":{self.triangle_count},"indices":[',
                 ",".join(str(i) for i in self.indices), '],"frames":[']
        parts.append(",".join(f'{{"timestep":{t},"positions":{_json_f32_array(x)}}}' for t, x in frames))
        parts.append("]}")
        try:
            with open(self.output_path, "w") as f:
                f.write("".join(parts))
        except OSError as e:
            raise L.VistioError(4, f"{self.output_path}: {e}") from None

    def name(self) -> str:
        return "json_exporter"

    def frame_count(self) -> int:
        return len(self.frames)


def validate_input(inp: SimulationInput):
    """validate_input (validator.rs:17-90): raises VistioError with the
    reference's messages."""
    try:
        inp.garment.validate()
    except L.VistioError as e:
        raise L.VistioError(1, f"Garment mesh: {str(e).split(': ', 1)[1]}") from None
    if inp.body is not None:
        try:
            inp.body.validate()
        except L.VistioError as e:
            raise L.VistioError(1, f"Body mesh: {str(e).split(': ', 1)[1]}") from None
    n = inp.garment.vertex_count()
    if len(inp.pinned) != n:
        raise L.VistioError(1, f"Pinned array length ({len(inp.pinned)}) != garment vertex count ({n})")
    p = inp.params
    if p.dt <= 0.0:
        raise L.VistioError(3, "Timestep dt must be positive")
    if p.dt > 1.0:
        raise L.VistioError(3, "Timestep dt > 1.0 is unreasonably large")
    if p.duration <= 0.0:
        raise L.VistioError(3, "Duration must be positive")
    if p.iterations == 0:
        raise L.VistioError(3, "Solver iterations must be >= 1")
    if p.gravity < 0.0:
        raise L.VistioError(3, "Gravity magnitude must be non-negative")
    if p.contact_thickness < 0.0:
        raise L.VistioError(3, "Contact thickness must be non-negative")
    g = p.gravity_direction
    ln = math.sqrt(float(np.float32(g[0] * g[0] + g[1] * g[1] + g[2] * g[2])))
    if abs(ln - 1.0) > 0.01:
        raise L.VistioError(3, f"Gravity direction should be unit length, got magnitude {ln}")


def material(name: str) -> api.FabricProperties:
    if name not in MATERIALS:
        raise L.VistioError(2, f"Unknown material '{name}' (known: {', '.join(sorted(MATERIALS))})")
    return MATERIALS[name]


def setup_for(props: api.FabricProperties, dt: float) -> api.SetupDesc:
    """The explicit set-up the runner's material path reduces to
    (runner.rs:100-140 with init_with_material / _tier3, pd_solver.rs:106-193),
    in the same float32 arithmetic; the system matrix is built for `dt`."""
    f = np.float32
    aniso = props.is_anisotropic()
    return api.SetupDesc(
        model=api.MODEL_ANISOTROPIC if aniso else api.MODEL_COROTATIONAL,
        bending=api.BENDING_DISCRETE_SHELLS_ANISOTROPIC if aniso else api.BENDING_DIHEDRAL,
        stiffness=float((f(props.stretch_stiffness_warp) + f(props.stretch_stiffness_weft)) / f(2.0) * f(10.0)),
        bend_stiffness=float((f(props.bending_stiffness_warp) + f(props.bending_stiffness_weft)) / f(2.0) * f(100.0)),
        density_gsm=props.density,
        warp_stiffness=props.stretch_stiffness_warp if aniso else 0.0,
        weft_stiffness=props.stretch_stiffness_weft if aniso else 0.0,
        bend_warp=props.bending_stiffness_warp, bend_weft=props.bending_stiffness_weft, matrix_dt=dt)


def solver_config(p: SimulationParams, **kw) -> api.SolverConfig:
    g = [float(np.float32(p.gravity) * np.float32(c)) for c in p.gravity_direction]
    return api.SolverConfig(max_iterations=int(p.iterations), gravity=tuple(g), **kw)


def _penetration(x: np.ndarray, c: Optional[api.Contact]) -> float:
    if c is None:
        return 0.0
    depth = np.zeros(x.shape[0])
    if c.has_ground:
        depth = np.maximum(depth, c.ground_height - x[:, 1])
    if c.has_sphere:
        depth = np.maximum(depth, c.sphere_radius - np.linalg.norm(x - np.asarray(c.sphere_center), axis=1))
    if c.has_cylinder:
        cx, cz, top, r = c.cylinder
        side = r - np.hypot(x[:, 0] - cx, x[:, 2] - cz)
        depth = np.maximum(depth, np.where(x[:, 1] <= top, np.minimum(side, top - x[:, 1]), 0.0))
    if c.has_box:
        lo, hi = np.asarray(c.box_min), np.asarray(c.box_max)
        inside = np.min(np.minimum(x - lo, hi - x), axis=1)
        depth = np.maximum(depth, inside)
    return float(max(0.0, depth.max()))


def _membrane(rest: np.ndarray, x: np.ndarray, tris: np.ndarray, stiffness: float):
    """Per triangle the largest principal stretch - 1 and the co-rotational
    membrane energy stiffness * area / 2 * |F - R|^2, with F the deformation
    gradient of the rest triangle (in its own plane) to the final one."""
    t = np.asarray(tris, np.int64).reshape(-1, 3)
    r0, r1, r2 = (rest[t[:, k]].astype(np.float64) for k in range(3))
    e1, e2 = r1 - r0, r2 - r0
    u = e1 / np.maximum(np.linalg.norm(e1, axis=1, keepdims=True), 1e-20)
    nrm = np.cross(e1, e2)
    area = 0.5 * np.linalg.norm(nrm, axis=1)
    v = np.cross(nrm / np.maximum(2 * area[:, None], 1e-20), u)
    dm = np.stack([np.stack([np.sum(e1 * u, 1), np.sum(e1 * v, 1)], 1),
                   np.stack([np.sum(e2 * u, 1), np.sum(e2 * v, 1)], 1)], 2)  # columns: rest edges in 2D
    ds = np.stack([x[t[:, 1]] - x[t[:, 0]], x[t[:, 2]] - x[t[:, 0]]], 2).astype(np.float64)
    ok = np.abs(np.linalg.det(dm)) > 1e-20
    dmi = np.linalg.inv(np.where(ok[:, None, None], dm, np.eye(2)))
    F = ds @ dmi
    U, S, Vt = np.linalg.svd(F, full_matrices=False)
    R = U @ Vt
    strain = np.where(ok, S[:, 0] - 1.0, 0.0)
    energy = float(np.sum(np.where(ok, stiffness * area / 2 * np.sum((F - R) ** 2, axis=(1, 2)), 0.0)))
    return strain, energy


def simulate(inp: SimulationInput, contact: Optional[api.Contact] = None, ctx=None, ipc: bool = True,
             exporter: Optional[JsonFrameExporter] = None) -> SimulationOutput:
    """Runs `inp` on the GPU solver: round(duration / dt) steps, each a plain
    PD step, or a step with IPC contact against `contact`'s colliders (its
    self-contact thickness defaults to the input's contact_thickness). With
    ipc=False the colliders act as the runner's non-IPC branch has them: a
    plain step, then their resolve() projections (runner.rs:209-215).
    `exporter`, when given, is initialised with the garment and receives the
    positions after every step (timestep 0, 1, ...); finalize() is the
    caller's."""
    validate_input(inp)
    if inp.body is not None:
        raise L.VistioError(3, "A body mesh is not simulated: pass the obstacles as analytical colliders (Contact)")
    p = inp.params
    props = material(p.material_name)
    mesh = inp.garment.to_mesh(inp.pinned)
    setup = setup_for(props, p.dt)
    cfg = solver_config(p)
    if contact is not None and contact.self_collision and contact.thickness == 0.0:
        contact = dataclasses.replace(contact, thickness=p.contact_thickness)
    s = api.ProjectiveDynamicsSolver(ctx).init_explicit(mesh, cfg, setup, pinned=mesh.pinned)
    if contact is not None and not ipc and contact.has_ground:
        s.set_ground(contact.ground_height)  # runner.rs:152-157
    steps = max(1, int(round(p.duration / p.dt)))
    if exporter is not None:
        exporter.init(inp.garment)
    t0 = time.perf_counter()
    iters = 0
    for k in range(steps):
        if contact is not None and ipc:
            r = s.step_with_ipc(p.dt, contact)
        else:
            r = s.step(p.dt)
            if contact is not None:
                s.resolve_contacts(contact)
        iters += r.iterations
        if exporter is not None:
            exporter.submit_frame(k, s.state()[0])
    wall = time.perf_counter() - t0
    x, v = s.state()
    rest = np.stack([mesh.px, mesh.py, mesh.pz], 1)
    strain, membrane = _membrane(rest, x, mesh.tris, setup.stiffness)
    strain = strain.astype(np.float32)
    m = s.lumped_masses().astype(np.float64)
    free = ~mesh.pinned.astype(bool)
    gdir = np.asarray(p.gravity_direction, np.float64)
    kinetic = 0.5 * float(np.sum(m[free] * np.sum(v[free].astype(np.float64) ** 2, 1)))
    potential = float(np.sum(m[free] * p.gravity * -(x[free].astype(np.float64) @ gdir)))
    force = s.contact_force() if contact is not None and ipc else np.zeros(mesh.nv, np.float32)
    nrm = _vertex_normals(x, mesh.tris)
    g = inp.garment
    draped = TriangleMesh(_f32(x[:, 0]), _f32(x[:, 1]), _f32(x[:, 2]), _f32(nrm[:, 0]), _f32(nrm[:, 1]),
                          _f32(nrm[:, 2]), list(g.uv_u), list(g.uv_v), list(g.indices), list(g.material_ids))
    metrics = SimulationMetrics(wall_time_seconds=wall, timestep_count=steps,
                                final_energy=kinetic + potential + membrane,
                                max_penetration=_penetration(x.astype(np.float64), contact),
                                max_strain=float(strain.max()) if strain.size else 0.0,
                                avg_iterations=iters / steps)
    return SimulationOutput(draped, VertexMetadata(_f32(strain), _f32(force)), metrics)
