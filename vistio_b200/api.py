"""Python host interface mirroring the reference's solver API over the C ABI.

Names and argument meanings follow crates/vistio-solver (SolverConfig,
SimulationState, ProjectiveDynamicsSolver::init / init_with_material /
init_with_material_tier3 / step / step_with_ipc / lumped_masses) and
crates/vistio-material (FabricProperties, the ConstitutiveModel kinds). Every
call goes through libvistio_b200.so; errors raise VistioError.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import List, Optional, Sequence

import numpy as np

from . import _lib as L

MODEL_ARAP, MODEL_COROTATIONAL, MODEL_ORTHOTROPIC, MODEL_ANISOTROPIC, MODEL_ISOTROPIC_LINEAR = 0, 1, 2, 3, 4
BENDING_NONE, BENDING_DIHEDRAL, BENDING_DISCRETE_SHELLS, BENDING_DISCRETE_SHELLS_ANISOTROPIC = 0, 1, 2, 3


@dataclasses.dataclass
class SolverConfig:
    """SolverConfig (crates/vistio-solver/src/config.rs:10-166) live fields, reference defaults."""
    max_iterations: int = 10
    tolerance: float = 1e-6
    gravity: tuple = (0.0, -9.81, 0.0)
    damping: float = 0.01
    stretch_weight: float = 1.0
    bending_weight: float = 0.5
    rayleigh_mass_damping: float = 2.0
    barrier_d_hat: float = 1e-3
    barrier_kappa: float = 0.0
    al_max_iterations: int = 10
    al_mu_initial: float = 1.0
    al_mu_growth: float = 10.0
    al_tolerance: float = 1e-4
    friction_coefficient: float = 0.4
    contact_damping: float = 0.3
    compliant_contact: bool = True
    compliant_d_hat_scale: float = 2.0
    adaptive_contact_damping: bool = True
    contact_damping_max: float = 0.5
    contact_velocity_threshold: float = 0.1
    # FP64 refinement sweeps of the global solve (this library only; the
    # reference solves in FP64): 0, 1 or 2. Off by default: with the local
    # projections and barriers in FP64 the FP32 sweeps already keep a step
    # within 1e-5 of FP64 on the drape workloads, and a sweep costs ~7% there.
    refinement_sweeps: int = 0
    # False (default): the numeric FP64 Cholesky factorization runs on the GPU
    # when the garment is first packed; True: on the host (both produce the
    # same factor up to FP64 rounding).
    host_factorization: bool = False

    def to_c(self) -> L.SolverConfigC:
        c = L.SolverConfigC()
        c.max_iterations = int(self.max_iterations)
        c.al_max_iterations = int(self.al_max_iterations)
        c.tolerance = float(self.tolerance)
        c.gravity[:] = [float(g) for g in self.gravity]
        for f in ("damping", "stretch_weight", "bending_weight", "rayleigh_mass_damping", "barrier_d_hat",
                  "barrier_kappa", "al_mu_initial", "al_mu_growth", "al_tolerance", "friction_coefficient",
                  "contact_damping", "compliant_d_hat_scale", "contact_damping_max", "contact_velocity_threshold"):
            setattr(c, f, float(getattr(self, f)))
        c.compliant_contact = int(bool(self.compliant_contact))
        c.adaptive_contact_damping = int(bool(self.adaptive_contact_damping))
        c.refinement_sweeps = int(self.refinement_sweeps)
        c.host_factorization = int(bool(self.host_factorization))
        return c


def drape_config(**kw) -> SolverConfig:
    """The drape workloads' configuration: the reference defaults with a fixed
    iteration count (tolerance 0) and Rayleigh alpha 0.01."""
    base = dict(tolerance=0.0, rayleigh_mass_damping=0.01)
    base.update(kw)
    return SolverConfig(**base)


@dataclasses.dataclass
class FabricProperties:
    """FabricProperties (crates/vistio-material/src/properties.rs:23-58)."""
    density: float = 200.0
    stretch_stiffness_warp: float = 1.0
    stretch_stiffness_weft: float = 1.0
    shear_stiffness: float = 0.5
    bending_stiffness_warp: float = 0.5
    bending_stiffness_weft: float = 0.5
    thickness: float = 0.001
    friction: float = 0.4
    damping: float = 0.1

    def is_anisotropic(self) -> bool:  # properties.rs:80-88
        ratio = self.stretch_stiffness_warp / self.stretch_stiffness_weft if self.stretch_stiffness_weft > 1e-8 else 1.0
        return abs(ratio - 1.0) > 0.05

    def to_c(self) -> L.MaterialDesc:
        m = L.MaterialDesc()
        for f in dataclasses.fields(self):
            setattr(m, f.name, float(getattr(self, f.name)))
        return m


@dataclasses.dataclass
class SetupDesc:
    """The explicit set-up every init path reduces to."""
    model: int = MODEL_ARAP
    bending: int = BENDING_DIHEDRAL
    stiffness: float = 1000.0
    bend_stiffness: float = 1e-4
    density_gsm: float = 200.0
    warp_stiffness: float = 0.0
    weft_stiffness: float = 0.0
    bend_warp: float = 0.0
    bend_weft: float = 0.0
    matrix_dt: float = 1.0 / 60.0

    def to_c(self) -> L.SetupDesc:
        s = L.SetupDesc()
        for f in dataclasses.fields(self):
            setattr(s, f.name, (int if f.name in ("model", "bending") else float)(getattr(self, f.name)))
        return s


@dataclasses.dataclass
class Contact:
    """What the reference's runner wires into its CollisionPipeline (runner.rs:48-99)."""
    has_ground: bool = False
    ground_height: float = 0.0
    has_sphere: bool = False
    sphere_center: tuple = (0.0, 0.0, 0.0)
    sphere_radius: float = 0.0
    self_collision: bool = False
    kappa: float = 0.0
    thickness: float = 0.0
    # CylinderCollider (cylinder.rs): (center x, center z, top y, radius), endless downwards
    has_cylinder: bool = False
    cylinder: tuple = (0.0, 0.0, 0.0, 0.0)
    # BoxCollider (box_collider.rs): axis-aligned [box_min, box_max]
    has_box: bool = False
    box_min: tuple = (0.0, 0.0, 0.0)
    box_max: tuple = (0.0, 0.0, 0.0)

    def to_c(self) -> L.ContactDesc:
        c = L.ContactDesc()
        c.has_ground = int(self.has_ground)
        c.ground_height = float(self.ground_height)
        c.has_sphere = int(self.has_sphere)
        c.sphere_center[:] = [float(v) for v in self.sphere_center]
        c.sphere_radius = float(self.sphere_radius)
        c.self_collision = int(self.self_collision)
        c.kappa = float(self.kappa)
        c.thickness = float(self.thickness)
        c.has_cylinder = int(self.has_cylinder)
        (c.cylinder_center_x, c.cylinder_center_z, c.cylinder_top_y,
         c.cylinder_radius) = [float(v) for v in self.cylinder]
        c.has_box = int(self.has_box)
        c.box_min[:] = [float(v) for v in self.box_min]
        c.box_max[:] = [float(v) for v in self.box_max]
        return c


@dataclasses.dataclass
class StepResult:
    """StepResult (crates/vistio-solver/src/strategy.rs:15-24) plus contact diagnostics."""
    iterations: int
    final_residual: float
    converged: bool
    wall_time: float
    al_iterations: int = 0
    active_contacts: int = 0
    last_alpha: float = 1.0

    @classmethod
    def from_c(cls, r: L.StepResultC) -> "StepResult":
        return cls(r.iterations, r.final_residual, bool(r.converged), r.wall_time, r.al_iterations,
                   r.active_contacts, r.last_alpha)


@dataclasses.dataclass
class ContactResult:
    """ContactResult (crates/vistio-contact/src/response.rs:13-20)."""
    resolved_count: int
    max_residual_penetration: float
    total_force_magnitude: float


@dataclasses.dataclass
class ColliderResults:
    """The collider rows of CollisionStepResult (collision_pipeline.rs:405-420)."""
    ground: ContactResult
    sphere: ContactResult
    cylinder: ContactResult
    box: ContactResult

    @classmethod
    def from_c(cls, r: L.ColliderResultsC) -> "ColliderResults":
        def one(c):
            return ContactResult(c.resolved_count, c.max_residual_penetration, c.total_force_magnitude)
        return cls(one(r.ground), one(r.sphere), one(r.cylinder), one(r.box))


def _fp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _f32(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float32)


class Context:
    """One CUDA device and stream (vistio_ctx)."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        L.check(L.lib().vistio_ctx_create(device, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None) and L is not None and L._lib is not None:
            L.lib().vistio_ctx_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()

    def sync(self):
        L.check(L.lib().vistio_sync(self.h), self.h)


_default_ctx: Optional[Context] = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


class ProjectiveDynamicsSolver:
    """A CUDA drop-in for the reference's ProjectiveDynamicsSolver
    (crates/vistio-solver/src/pd_solver.rs:53): init*, step, step_with_ipc,
    lumped_masses, name. Device state lives in HBM; set_state / state copy."""

    def __init__(self, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.h = None
        self.nv = 0

    def _mesh(self, px, py, pz, tris):
        self._keep = [_f32(px), _f32(py), _f32(pz), np.ascontiguousarray(tris, dtype=np.uint32).reshape(-1)]
        m = L.MeshDesc()
        m.vertex_count = len(self._keep[0])
        m.triangle_count = len(self._keep[3]) // 3
        m.pos_x, m.pos_y, m.pos_z = (_fp(a) for a in self._keep[:3])
        m.indices = self._keep[3].ctypes.data_as(C.POINTER(C.c_uint32))
        self.nv = m.vertex_count
        return m

    def _pinned(self, pinned):
        p = np.zeros(self.nv, np.uint8) if pinned is None else np.ascontiguousarray(pinned, dtype=np.uint8)
        self._pin = p
        return p.ctypes.data_as(C.POINTER(C.c_uint8))

    def init(self, mesh, config: SolverConfig, pinned=None):
        """SolverStrategy::init (pd_solver.rs:221-257): ARAP + dihedral bending, 200 g/m^2."""
        h = C.c_void_p()
        md = self._mesh(mesh.px, mesh.py, mesh.pz, mesh.tris)
        cfg = config.to_c()
        L.check(L.lib().vistio_solver_init(self.ctx.h, C.byref(md), C.byref(cfg), self._pinned(pinned), C.byref(h)),
                self.ctx.h)
        self.h = h
        return self

    def init_with_material(self, mesh, config: SolverConfig, properties: FabricProperties, model_kind: int,
                           pinned=None, warp: float = 0.0, weft: float = 0.0, bending: int = BENDING_DIHEDRAL):
        """init_with_material (pd_solver.rs:106-143) with a ConstitutiveModel kind."""
        h = C.c_void_p()
        md = self._mesh(mesh.px, mesh.py, mesh.pz, mesh.tris)
        cfg = config.to_c()
        mat = properties.to_c()
        mod = L.ModelDesc()
        mod.kind, mod.warp_stiffness, mod.weft_stiffness = int(model_kind), float(warp), float(weft)
        L.check(L.lib().vistio_solver_init_with_material(self.ctx.h, C.byref(md), C.byref(cfg), C.byref(mat),
                                                         C.byref(mod), int(bending), self._pinned(pinned),
                                                         C.byref(h)), self.ctx.h)
        self.h = h
        return self

    def init_with_material_tier3(self, mesh, config, properties: FabricProperties, model_kind: int, pinned=None,
                                 warp: float = 0.0, weft: float = 0.0):
        """init_with_material_tier3 (pd_solver.rs:152-193): Discrete Shells bending."""
        bend = BENDING_DISCRETE_SHELLS_ANISOTROPIC if properties.is_anisotropic() else BENDING_DISCRETE_SHELLS
        return self.init_with_material(mesh, config, properties, model_kind, pinned, warp, weft, bend)

    def init_explicit(self, mesh, config: SolverConfig, setup: SetupDesc, pinned=None):
        h = C.c_void_p()
        md = self._mesh(mesh.px, mesh.py, mesh.pz, mesh.tris)
        cfg = config.to_c()
        sd = setup.to_c()
        L.check(L.lib().vistio_solver_init_explicit(self.ctx.h, C.byref(md), C.byref(cfg), C.byref(sd),
                                                    self._pinned(pinned), C.byref(h)), self.ctx.h)
        self.h = h
        return self

    def close(self):
        if getattr(self, "h", None) and L is not None and L._lib is not None:
            L.lib().vistio_solver_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()

    def name(self) -> str:
        return L.lib().vistio_solver_name(self.h).decode()

    def info(self) -> dict:
        vals = [C.c_uint32(), C.c_uint32(), C.c_uint32(), C.c_uint64(), C.c_uint64(), C.c_uint32(), C.c_uint32()]
        L.check(L.lib().vistio_solver_info(self.h, *[C.byref(v) for v in vals]), self.ctx.h)
        keys = ("nv", "nt", "nh", "nnz_a", "nnz_l", "supernodes", "levels")
        return {k: v.value for k, v in zip(keys, vals)}

    def lumped_masses(self) -> np.ndarray:
        out = np.zeros(self.nv, np.float32)
        L.check(L.lib().vistio_solver_lumped_masses(self.h, _fp(out)), self.ctx.h)
        return out

    def contact_force(self) -> np.ndarray:
        """Per vertex |contact barrier gradient| of the last contact detect (vistio_solver_contact_force)."""
        out = np.zeros(self.nv, np.float32)
        L.check(L.lib().vistio_solver_contact_force(self.h, _fp(out)), self.ctx.h)
        return out

    def set_ground(self, height: Optional[float]):
        L.check(L.lib().vistio_solver_set_ground(self.h, int(height is not None), float(height or 0.0)), self.ctx.h)

    def set_state(self, pos: np.ndarray, vel: Optional[np.ndarray] = None):
        pos = _f32(pos)
        vel = np.zeros_like(pos) if vel is None else _f32(vel)
        cols = [np.ascontiguousarray(pos[:, k]) for k in range(3)] + [np.ascontiguousarray(vel[:, k]) for k in range(3)]
        L.check(L.lib().vistio_solver_set_state(self.h, *[_fp(c) for c in cols]), self.ctx.h)

    def state(self):
        cols = [np.zeros(self.nv, np.float32) for _ in range(6)]
        L.check(L.lib().vistio_solver_get_state(self.h, *[_fp(c) for c in cols]), self.ctx.h)
        return np.stack(cols[:3], 1), np.stack(cols[3:], 1)

    def step(self, dt: float) -> StepResult:
        r = L.StepResultC()
        L.check(L.lib().vistio_step(self.h, float(dt), C.byref(r)), self.ctx.h)
        return StepResult.from_c(r)

    def step_with_ipc(self, dt: float, contact: Contact) -> StepResult:
        r = L.StepResultC()
        c = contact.to_c()
        L.check(L.lib().vistio_step_with_ipc(self.h, float(dt), C.byref(c), C.byref(r)), self.ctx.h)
        return StepResult.from_c(r)

    def resolve_contacts(self, contact: Contact) -> ColliderResults:
        """The runner's non-IPC collision step after step() (runner.rs:209-215): ground twice, then the
        sphere, cylinder and box colliders project the vertices inside them onto their surfaces."""
        r = L.ColliderResultsC()
        c = contact.to_c()
        L.check(L.lib().vistio_resolve_contacts(self.h, C.byref(c), C.byref(r)), self.ctx.h)
        return ColliderResults.from_c(r)


class Batch:
    """Many garments in one ragged SoA set of HBM buffers, stepped by one CUDA graph."""

    def __init__(self, solvers: Sequence[ProjectiveDynamicsSolver], ctx: Optional[Context] = None):
        self.ctx = ctx or solvers[0].ctx
        self.solvers = list(solvers)
        arr = (C.c_void_p * len(solvers))(*[s.h for s in solvers])
        h = C.c_void_p()
        L.check(L.lib().vistio_batch_create(self.ctx.h, arr, len(solvers), C.byref(h)), self.ctx.h)
        self.h = h
        self.nverts = [s.nv for s in solvers]

    def close(self):
        if getattr(self, "h", None) and L is not None and L._lib is not None:
            L.lib().vistio_batch_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()

    def step(self, dt: float, nsteps: int = 1, contact: Optional[Contact] = None):
        c = contact.to_c() if contact is not None else None
        L.check(L.lib().vistio_batch_step(self.h, float(dt), int(nsteps), C.byref(c) if c is not None else None),
                self.ctx.h)

    def resolve_contacts(self, contact: Contact) -> List[ColliderResults]:
        """ProjectiveDynamicsSolver.resolve_contacts on every garment with the same colliders."""
        r = (L.ColliderResultsC * len(self.solvers))()
        c = contact.to_c()
        L.check(L.lib().vistio_batch_resolve_contacts(self.h, C.byref(c), r), self.ctx.h)
        return [ColliderResults.from_c(x) for x in r]

    def state(self, k: int):
        nv = self.nverts[k]
        cols = [np.zeros(nv, np.float32) for _ in range(6)]
        L.check(L.lib().vistio_batch_get_state(self.h, k, *[_fp(c) for c in cols]), self.ctx.h)
        return np.stack(cols[:3], 1), np.stack(cols[3:], 1)

    def set_state(self, k: int, pos, vel=None):
        pos = _f32(pos)
        vel = np.zeros_like(pos) if vel is None else _f32(vel)
        cols = [np.ascontiguousarray(pos[:, j]) for j in range(3)] + [np.ascontiguousarray(vel[:, j]) for j in range(3)]
        L.check(L.lib().vistio_batch_set_state(self.h, k, *[_fp(c) for c in cols]), self.ctx.h)

    def upload_positions(self, xyz: np.ndarray):
        xyz = _f32(xyz)
        L.check(L.lib().vistio_batch_upload_positions(self.h, _fp(xyz)), self.ctx.h)

    def download_positions(self, out: Optional[np.ndarray] = None) -> np.ndarray:
        if out is None:
            out = np.zeros((sum(self.nverts), 3), np.float32)
        L.check(L.lib().vistio_batch_download_positions(self.h, _fp(out)), self.ctx.h)
        return out

    def info(self) -> dict:
        vals = [C.c_uint32(), C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint64()]
        L.check(L.lib().vistio_batch_info(self.h, *[C.byref(v) for v in vals]), self.ctx.h)
        keys = ("instances", "vertices", "triangles", "hinges", "factor_bytes", "device_bytes")
        return {k: v.value for k, v in zip(keys, vals)}

    def factor_stats(self) -> dict:
        """The device factorization done when the batch was created: kernel
        launches and device milliseconds (0, 0 if every garment was factorized
        on the host)."""
        n, ms = C.c_uint32(), C.c_float()
        L.check(L.lib().vistio_batch_factor_stats(self.h, C.byref(n), C.byref(ms)), self.ctx.h)
        return {"launches": n.value, "device_ms": ms.value}

    def launches_per_step(self) -> int:
        v = C.c_uint32()
        L.check(L.lib().vistio_batch_launches_per_step(self.h, C.byref(v)), self.ctx.h)
        return v.value

    def stream(self) -> int:
        return L.lib().vistio_batch_stream(self.h) or 0

    PHASES = {"predict": 0, "membrane": 1, "bending": 2, "gather": 3, "solve": 4, "finalize": 5, "refine": 6}

    TUNE_LIMITS = (0, 1024, 2048, 4096, 6144, 12288, 1 << 30)

    SWEEP_MODES = ("levels", "dataflow", "grouped")

    GROUP_LIMITS = (0, 64, 128, 256, 512, 1024, 6144)

    def tune(self) -> dict:
        """Autotunes the sweeps on this batch (vistio_batch_tune): returns the
        chosen sweep kind and warp-item limit, and the sweep time of every
        candidate (per kind, per limit)."""
        chosen = C.c_uint32()
        ms = (C.c_float * 21)()
        L.check(L.lib().vistio_batch_tune(self.h, C.byref(chosen), ms), self.ctx.h)
        tri, hinge = C.c_uint32(), C.c_uint32()
        lms = (C.c_float * 4)()
        L.check(L.lib().vistio_batch_tune_local(self.h, C.byref(tri), C.byref(hinge), lms), self.ctx.h)
        sweep_ms = {mode: {str(lim): float(ms[7 * m + i]) for i, lim in enumerate(self.TUNE_LIMITS)}
                    for m, mode in enumerate(self.SWEEP_MODES[:2])}
        grouped = {str(lim): float(ms[14 + i]) for i, lim in enumerate(self.GROUP_LIMITS) if ms[14 + i] >= 0}
        if grouped:
            sweep_ms["grouped"] = grouped
        blocks, occ = self.sweep_blocks()
        return {"sweep_mode": self.sweep_mode()[0], "warp_item_limit": chosen.value,
                "sweep_blocks_per_sm": blocks, "sweep_blocks_ms": occ,
                "group_limit": self.group_limit() if grouped else None,
                "sweep_ms": sweep_ms,
                "triangles_per_thread": tri.value, "hinges_per_thread": hinge.value,
                "local_ms": {"membrane": {"1": float(lms[0]), "2": float(lms[1])},
                             "bending": {"1": float(lms[2]), "2": float(lms[3])}}}

    def set_group_limit(self, limit: int):
        """Largest s (s + m) of a supernode above the bottom subtrees that the
        garment groups sweep one lane per garment (sweep kind "grouped")."""
        L.check(L.lib().vistio_batch_set_group_limit(self.h, int(limit)), self.ctx.h)

    def group_limit(self) -> int:
        v = C.c_uint32()
        L.check(L.lib().vistio_batch_get_group_limit(self.h, C.byref(v)), self.ctx.h)
        return v.value

    def set_local_shape(self, triangles_per_thread: int, hinges_per_thread: int):
        """Elements per thread of the membrane and bending steps (1 or 2 each)."""
        L.check(L.lib().vistio_batch_set_local_shape(self.h, int(triangles_per_thread), int(hinges_per_thread)),
                self.ctx.h)

    def set_self_ccd_dedup(self, on: bool):
        """Self-contact CCD over each vertex-triangle test once (True, the
        default) or over every test of every candidate pair (False); the step
        is bit-identical either way."""
        L.check(L.lib().vistio_batch_set_self_ccd_dedup(self.h, 1 if on else 0), self.ctx.h)

    def set_warp_limit(self, limit: int):
        L.check(L.lib().vistio_batch_set_warp_limit(self.h, int(limit)), self.ctx.h)

    def set_sweep_mode(self, mode: str):
        """"levels": one launch per level; "dataflow": one dependency-driven
        launch for both directions; "grouped" (batches with garment groups:
        8 or more garments of one mesh topology): the groups' tree bottoms
        one lane per garment, the rest dependency-driven."""
        L.check(L.lib().vistio_batch_set_sweep_mode(self.h, self.SWEEP_MODES.index(mode)), self.ctx.h)

    def set_sweep_blocks(self, blocks_per_sm: int):
        """Compiled form of the dependency-driven sweep kernel, by resident
        blocks per SM: 5 or 4 (eight-warp blocks) or 2 (sixteen-warp blocks);
        bit-identical results."""
        L.check(L.lib().vistio_batch_set_sweep_blocks(self.h, int(blocks_per_sm)), self.ctx.h)

    def sweep_blocks(self) -> tuple:
        """(blocks per SM of the form in use, {form: the tuner's ms per solve})."""
        v, ms = C.c_uint32(), (C.c_float * 3)()
        L.check(L.lib().vistio_batch_get_sweep_blocks(self.h, C.byref(v), ms), self.ctx.h)
        return v.value, {"5": float(ms[0]), "4": float(ms[1]), "2": float(ms[2])}

    def sweep_mode(self) -> tuple:
        """(sweep kind, warp-item limit) in use."""
        m, lim = C.c_uint32(), C.c_uint32()
        L.check(L.lib().vistio_batch_get_sweep_mode(self.h, C.byref(m), C.byref(lim)), self.ctx.h)
        return self.SWEEP_MODES[m.value], lim.value

    def launch_phase(self, phase: str):
        L.check(L.lib().vistio_batch_launch_phase(self.h, self.PHASES[phase]), self.ctx.h)

    def phase_bytes(self, phase: str) -> int:
        v = C.c_uint64()
        L.check(L.lib().vistio_batch_phase_bytes(self.h, self.PHASES[phase], C.byref(v)), self.ctx.h)
        return v.value


def symbolic_cache_info() -> dict:
    """The host's cache of symbolic factorizations (vistio_symbolic_cache_info)."""
    vals = [C.c_uint64() for _ in range(4)]
    L.check(L.lib().vistio_symbolic_cache_info(*[C.byref(v) for v in vals]))
    return dict(zip(("hits", "misses", "bytes", "entries"), (v.value for v in vals)))


def set_symbolic_cache_limit(nbytes: int):
    """Bound the symbolic cache's bytes (0 empties and disables it)."""
    L.check(L.lib().vistio_symbolic_cache_set_limit(int(nbytes)))


class SparseSolver:
    """SparseSolver / FaerSolver mirror (crates/vistio-math/src/sparse.rs:110-120)."""

    def __init__(self, ctx: Optional[Context] = None):
        self.ctx = ctx or default_context()
        self.h = None
        self.n = 0

    def factorize(self, row_ptr, col_idx, values, n: int):
        rp = np.ascontiguousarray(row_ptr, np.uint32)
        ci = np.ascontiguousarray(col_idx, np.uint32)
        va = _f32(values)
        h = C.c_void_p()
        L.check(L.lib().vistio_sparse_factorize(self.ctx.h, int(n), rp.ctypes.data_as(C.POINTER(C.c_uint32)),
                                                ci.ctypes.data_as(C.POINTER(C.c_uint32)), _fp(va), C.byref(h)),
                self.ctx.h)
        self.h = h
        self.n = n

    def is_factorized(self) -> bool:
        return self.h is not None

    def solve(self, rhs) -> np.ndarray:
        if self.h is None:
            raise L.VistioError(3, "Solver not factorized. Call factorize() first.")
        b = _f32(rhs)
        if b.shape[0] != self.n:
            raise L.VistioError(3, f"RHS length ({b.shape[0]}) != matrix dimension ({self.n})")
        x = np.zeros_like(b)
        L.check(L.lib().vistio_sparse_solve(self.h, _fp(b), _fp(x)), self.ctx.h)
        return x

    def __del__(self):
        if getattr(self, "h", None) and L is not None and L._lib is not None:
            L.lib().vistio_sparse_destroy(self.h)
        self.h = None


def broadphase_pairs(pos: np.ndarray, tris: np.ndarray, margin: float, ctx: Optional[Context] = None) -> np.ndarray:
    """Sorted candidate triangle pairs (ta < tb) with overlapping inflated AABBs (GPU)."""
    ctx = ctx or default_context()
    pos = _f32(pos)
    tris = np.ascontiguousarray(tris, np.uint32)
    cols = [np.ascontiguousarray(pos[:, k]) for k in range(3)]
    cnt = C.c_uint64()
    u32 = C.POINTER(C.c_uint32)
    L.check(L.lib().vistio_broadphase_pairs(ctx.h, pos.shape[0], *[_fp(c) for c in cols], tris.shape[0],
                                            tris.ctypes.data_as(u32), float(margin), None, 0, C.byref(cnt)), ctx.h)
    out = np.zeros((max(cnt.value, 1), 2), np.uint32)
    L.check(L.lib().vistio_broadphase_pairs(ctx.h, pos.shape[0], *[_fp(c) for c in cols], tris.shape[0],
                                            tris.ctypes.data_as(u32), float(margin), out.ctypes.data_as(u32),
                                            cnt.value, C.byref(cnt)), ctx.h)
    return out[: cnt.value]


NOALLOC_MAX_PAIRS = 1 << 20  # VISTIO_NOALLOC_MAX_PAIRS
_noalloc_host = None  # one reusable host buffer of NOALLOC_MAX_PAIRS pairs


def broadphase_pairs_noalloc(pos: np.ndarray, tris: np.ndarray, margin: float,
                             ctx: Optional[Context] = None) -> np.ndarray:
    """broadphase_pairs through the allocation-free entry point: the library
    allocates no device memory for the call (meshes up to 65536 triangles and
    65536 vertices, up to 1048576 pairs; larger inputs raise VistioError with
    status CAPACITY). Calls on one device must not overlap. One call per
    query: the pairs land in a host buffer sized for the maximum pair count,
    allocated once and reused, and the result is a copy of its first rows."""
    global _noalloc_host
    ctx = ctx or default_context()
    pos = _f32(pos)
    tris = np.ascontiguousarray(tris, np.uint32)
    cols = [np.ascontiguousarray(pos[:, k]) for k in range(3)]
    if _noalloc_host is None:
        _noalloc_host = np.zeros((NOALLOC_MAX_PAIRS, 2), np.uint32)
    cnt = C.c_uint64()
    u32 = C.POINTER(C.c_uint32)
    L.check(L.lib().vistio_broadphase_pairs_noalloc(ctx.h, pos.shape[0], *[_fp(c) for c in cols], tris.shape[0],
                                                    tris.ctypes.data_as(u32), float(margin),
                                                    _noalloc_host.ctypes.data_as(u32), NOALLOC_MAX_PAIRS,
                                                    C.byref(cnt)), ctx.h)
    return _noalloc_host[: cnt.value].copy()


def ccd_hits(p0: np.ndarray, p1: np.ndarray, tris: np.ndarray, pairs: np.ndarray, ctx: Optional[Context] = None):
    """Sorted unique (vertex, triangle) vertex-triangle CCD hits and the min TOI (GPU, FP64)."""
    ctx = ctx or default_context()
    p0 = _f32(p0).reshape(-1)
    p1 = _f32(p1).reshape(-1)
    tris = np.ascontiguousarray(tris, np.uint32)
    pairs = np.ascontiguousarray(pairs, np.uint32)
    u32 = C.POINTER(C.c_uint32)
    cap = 6 * max(len(pairs), 1)
    hits = np.zeros((cap, 2), np.uint32)
    nh = C.c_uint64()
    mt = C.c_float()
    L.check(L.lib().vistio_ccd_hits(ctx.h, p0.shape[0] // 3, _fp(p0), _fp(p1), tris.shape[0],
                                    tris.ctypes.data_as(u32), len(pairs), pairs.ctypes.data_as(u32),
                                    hits.ctypes.data_as(u32), cap, C.byref(nh), C.byref(mt)), ctx.h)
    return hits[: nh.value], mt.value


def barrier_grad(d2, d_hat: float, kappa: float, thickness: float = 0.0, ctx: Optional[Context] = None) -> np.ndarray:
    """The device's kappa-scaled barrier gradient at squared distances d2 (FP64; C-IPC form when thickness > 0)."""
    ctx = ctx or default_context()
    d = np.ascontiguousarray(d2, np.float64).reshape(-1)
    out = np.zeros_like(d)
    dp = C.POINTER(C.c_double)
    L.check(L.lib().vistio_barrier_grad(ctx.h, d.shape[0], d.ctypes.data_as(dp), float(d_hat), float(kappa),
                                        float(thickness), out.ctypes.data_as(dp)), ctx.h)
    return out


REQUEST_STATES = {0: "queued", 1: "setup", 2: "ready", 3: "running", 4: "done", 5: "failed"}


class Server:
    """Continuous batching of drape requests (vistio_server_*): each request
    carries its own mesh, material, contact set-up, dt and step count; requests
    that arrive while others run are admitted at the next tick as memory
    allows and share the GPU with them. Results are read back per request."""

    def __init__(self, hbm_budget_bytes: int = 8 << 30, max_cohort: int = 64, setup_threads: int = 4,
                 steps_per_slice: int = 10, cache_bytes: int = 1 << 30, device: int = 0,
                 gpu_factorization: bool = False, sweep_mode: str = "levels", admit_wait_ms: int = 0):
        """gpu_factorization False: the set-up threads factorize on the host,
        beside the GPU's work; True: each request's own host_factorization.
        sweep_mode: the sweep kind of every cohort (Batch.SWEEP_MODES).
        admit_wait_ms: while cohorts run, how long ready requests of one step
        configuration may wait for others to form a larger cohort."""
        cfg = L.ServerConfig(device, int(hbm_budget_bytes), int(max_cohort), int(setup_threads), int(steps_per_slice),
                             int(cache_bytes), int(bool(gpu_factorization)), Batch.SWEEP_MODES.index(sweep_mode),
                             int(admit_wait_ms))
        h = C.c_void_p()
        st = L.lib().vistio_server_create(C.byref(cfg), C.byref(h))
        if st != L.OK:
            raise L.VistioError(st, "server creation failed")
        self.h = h
        self._nv = {}

    def close(self):
        if getattr(self, "h", None) and L is not None and L._lib is not None:
            L.lib().vistio_server_destroy(self.h)
        self.h = None

    def __del__(self):
        self.close()

    def _check(self, st: int):
        if st != L.OK:
            raise L.VistioError(st, L.lib().vistio_server_last_error(self.h).decode())

    def submit(self, mesh, config: SolverConfig, setup: SetupDesc, steps: int, dt: float,
               contact: Optional[Contact] = None, ipc: bool = False, pinned=None) -> int:
        """Queues a request; with ipc the steps are step_with_ipc(contact),
        else plain steps (contact.has_ground adds the ground clamp)."""
        px, py, pz = _f32(mesh.px), _f32(mesh.py), _f32(mesh.pz)
        tris = np.ascontiguousarray(mesh.tris, dtype=np.uint32).reshape(-1)
        pin = None if pinned is None else np.ascontiguousarray(pinned, dtype=np.uint8)
        r = L.RequestC()
        r.mesh.vertex_count = len(px)
        r.mesh.triangle_count = len(tris) // 3
        r.mesh.pos_x, r.mesh.pos_y, r.mesh.pos_z = _fp(px), _fp(py), _fp(pz)
        r.mesh.indices = tris.ctypes.data_as(C.POINTER(C.c_uint32))
        r.pinned = pin.ctypes.data_as(C.POINTER(C.c_uint8)) if pin is not None else None
        r.config = config.to_c()
        r.setup = setup.to_c()
        r.has_contact = int(bool(ipc))
        r.contact = (contact or Contact()).to_c()
        r.dt = float(dt)
        r.steps = int(steps)
        rid = C.c_uint64()
        self._check(L.lib().vistio_server_submit(self.h, C.byref(r), C.byref(rid)))
        self._nv[rid.value] = len(px)
        return rid.value

    def tick(self) -> int:
        n = C.c_uint32()
        self._check(L.lib().vistio_server_tick(self.h, C.byref(n)))
        return n.value

    def drain(self, timeout_s: float = 600.0):
        self._check(L.lib().vistio_server_drain(self.h, float(timeout_s)))

    def query(self, rid: int) -> dict:
        i = L.RequestInfo()
        self._check(L.lib().vistio_server_query(self.h, int(rid), C.byref(i)))
        return {"state": REQUEST_STATES[i.state], "status": i.status, "vertex_count": i.vertex_count,
                "cohort": i.cohort, "cache_hit": bool(i.cache_hit), "submit_s": i.submit_s, "ready_s": i.ready_s,
                "start_s": i.start_s, "done_s": i.done_s}

    def result(self, rid: int):
        nv = self._nv[rid]
        cols = [np.zeros(nv, np.float32) for _ in range(6)]
        self._check(L.lib().vistio_server_result(self.h, int(rid), *[_fp(c) for c in cols]))
        return np.stack(cols[:3], 1), np.stack(cols[3:], 1)

    def release(self, rid: int):
        self._check(L.lib().vistio_server_release(self.h, int(rid)))
        self._nv.pop(rid, None)

    def stats(self) -> dict:
        s = L.ServerStats()
        self._check(L.lib().vistio_server_get_stats(self.h, C.byref(s)))
        return {name: getattr(s, name) for name, _ in L.ServerStats._fields_}
