"""ctypes binding of the CPU oracle (oracle/liboracle.so).

Test infrastructure: only tests/, __graft_entry__.smoke() and bench.py's
CPU-baseline leg import this module, and only as the checker.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB_PATH = os.path.join(ROOT, "oracle", "liboracle.so")

MODEL_ARAP, MODEL_COROT, MODEL_ORTHO, MODEL_ANISO, MODEL_ISO_LINEAR = 0, 1, 2, 3, 4
BEND_NONE, BEND_DIHEDRAL, BEND_DS, BEND_DS_ANISO = 0, 1, 2, 3


class Params(C.Structure):
    _fields_ = [("model", C.c_int32), ("bending", C.c_int32), ("stiffness", C.c_float),
                ("bend_stiffness", C.c_float), ("density_gsm", C.c_float), ("warp", C.c_float),
                ("weft", C.c_float), ("bend_warp", C.c_float), ("bend_weft", C.c_float),
                ("matrix_dt", C.c_float)]


class Config(C.Structure):
    _fields_ = [("max_iterations", C.c_uint32), ("al_max_iterations", C.c_uint32),
                ("tolerance", C.c_double), ("gravity", C.c_float * 3), ("damping", C.c_float),
                ("rayleigh_mass_damping", C.c_float), ("barrier_d_hat", C.c_float),
                ("al_mu_initial", C.c_float), ("al_mu_growth", C.c_float), ("al_tolerance", C.c_float),
                ("friction_coefficient", C.c_float), ("contact_damping", C.c_float),
                ("compliant_d_hat_scale", C.c_float), ("contact_damping_max", C.c_float),
                ("contact_velocity_threshold", C.c_float), ("compliant_contact", C.c_int32),
                ("adaptive_contact_damping", C.c_int32)]


class Contact(C.Structure):
    _fields_ = [("has_ground", C.c_int32), ("ground_height", C.c_float), ("has_sphere", C.c_int32),
                ("sphere_center", C.c_float * 3), ("sphere_radius", C.c_float),
                ("self_collision", C.c_int32), ("bvh_faithful", C.c_int32), ("kappa", C.c_float),
                ("thickness", C.c_float), ("has_cylinder", C.c_int32), ("cylinder_center_x", C.c_float),
                ("cylinder_center_z", C.c_float), ("cylinder_top_y", C.c_float), ("cylinder_radius", C.c_float),
                ("has_box", C.c_int32), ("box_min", C.c_float * 3), ("box_max", C.c_float * 3)]


class StepResult(C.Structure):
    _fields_ = [("iterations", C.c_uint32), ("converged", C.c_int32), ("final_residual", C.c_double),
                ("status", C.c_int32), ("al_iterations", C.c_uint32), ("active_contacts", C.c_uint32),
                ("last_alpha", C.c_float)]


def default_config(**kw) -> Config:
    """SolverConfig::default() (config.rs:131-166) with the drape mapping:
    tolerance 0 (fixed iteration count) and Rayleigh alpha 0.01."""
    c = Config()
    c.max_iterations = 10
    c.al_max_iterations = 10
    c.tolerance = 0.0
    c.gravity[:] = (0.0, -9.81, 0.0)
    c.damping = 0.01
    c.rayleigh_mass_damping = 0.01
    c.barrier_d_hat = 1e-3
    c.al_mu_initial = 1.0
    c.al_mu_growth = 10.0
    c.al_tolerance = 1e-4
    c.friction_coefficient = 0.4
    c.contact_damping = 0.3
    c.compliant_d_hat_scale = 2.0
    c.contact_damping_max = 0.5
    c.contact_velocity_threshold = 0.1
    c.compliant_contact = 1
    c.adaptive_contact_damping = 1
    for k, v in kw.items():
        setattr(c, k, v)
    return c


def init_params(stiffness=1e3, bend_stiffness=1e-4, density_gsm=150.0, model=MODEL_ARAP,
                bending=BEND_DIHEDRAL, warp=0.0, weft=0.0, bend_warp=0.0, bend_weft=0.0,
                matrix_dt=1.0 / 60.0) -> Params:
    p = Params()
    p.model, p.bending = model, bending
    p.stiffness, p.bend_stiffness, p.density_gsm = stiffness, bend_stiffness, density_gsm
    p.warp, p.weft, p.bend_warp, p.bend_weft = warp, weft, bend_warp, bend_weft
    p.matrix_dt = matrix_dt
    return p


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            subprocess.check_call(["make", "-s", "-C", os.path.join(ROOT, "oracle")])
        L = C.CDLL(LIB_PATH)
        fp = C.POINTER(C.c_float)
        L.orc_create.restype = C.c_void_p
        L.orc_create.argtypes = [C.c_int, C.c_uint32, fp, fp, fp, C.c_uint32, C.POINTER(C.c_uint32),
                                 C.POINTER(C.c_uint8), C.POINTER(Params), C.POINTER(Config),
                                 C.POINTER(C.c_int32)]
        L.orc_destroy.argtypes = [C.c_void_p]
        L.orc_step.argtypes = [C.c_void_p, C.c_float, C.POINTER(StepResult)]
        L.orc_step_ipc.argtypes = [C.c_void_p, C.c_float, C.POINTER(Contact), C.POINTER(StepResult)]
        L.orc_set_ground.argtypes = [C.c_void_p, C.c_int, C.c_float]
        L.orc_resolve.argtypes = [C.c_void_p, C.POINTER(Contact), C.POINTER(C.c_float)]
        L.orc_sparse_solve.argtypes = [C.c_uint32, C.c_uint32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                                       C.POINTER(C.c_float), C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.orc_get_state.argtypes = [C.c_void_p] + [fp] * 6
        L.orc_set_state.argtypes = [C.c_void_p] + [fp] * 6
        dp = C.POINTER(C.c_double)
        L.orc_get_state64.argtypes = [C.c_void_p, dp, dp, dp]
        L.orc_hinge_count.restype = C.c_uint32
        L.orc_hinge_count.argtypes = [C.c_void_p]
        L.orc_get_hinges.argtypes = [C.c_void_p, C.POINTER(C.c_uint32), fp, fp, fp]
        L.orc_get_masses.argtypes = [C.c_void_p, fp]
        L.orc_matrix_nnz.restype = C.c_uint32
        L.orc_matrix_nnz.argtypes = [C.c_void_p]
        L.orc_get_matrix.argtypes = [C.c_void_p, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32), dp]
        L.orc_factor_nnz.restype = C.c_uint64
        L.orc_factor_nnz.argtypes = [C.c_void_p]
        L.orc_assemble_rhs.argtypes = [C.c_void_p, C.c_float, fp, fp, fp]
        L.orc_solve.argtypes = [C.c_void_p, fp, fp]
        L.orc_quad_grid.argtypes = [C.c_uint32, C.c_uint32, C.c_float, C.c_float, fp, fp, fp,
                                    C.POINTER(C.c_uint32)]
        f3 = fp
        L.orc_pt_dist2.restype = C.c_float
        L.orc_pt_dist2.argtypes = [f3, f3, f3, f3, C.POINTER(C.c_int)]
        L.orc_ee_dist2.restype = C.c_float
        L.orc_ee_dist2.argtypes = [f3, f3, f3, f3, C.POINTER(C.c_int)]
        L.orc_pt_grad.argtypes = [f3, f3, f3, f3, fp]
        L.orc_ee_grad.argtypes = [f3, f3, f3, f3, fp]
        L.orc_vt_ccd.restype = C.c_int
        L.orc_vt_ccd.argtypes = [f3] * 8 + [fp]
        L.orc_ee_ccd.restype = C.c_int
        L.orc_ee_ccd.argtypes = [f3] * 8 + [fp]
        L.orc_cubic_roots.restype = C.c_int
        L.orc_cubic_roots.argtypes = [C.c_float] * 4 + [fp]
        for name in ("orc_barrier_energy", "orc_barrier_gradient", "orc_barrier_hessian"):
            getattr(L, name).restype = C.c_float
            getattr(L, name).argtypes = [C.c_float, C.c_float]
        for name in ("orc_scaled_barrier_gradient", "orc_barrier_energy_thick", "orc_barrier_gradient_thick"):
            getattr(L, name).restype = C.c_float
            getattr(L, name).argtypes = [C.c_float, C.c_float, C.c_float]
        L.orc_estimate_kappa.restype = C.c_float
        L.orc_estimate_kappa.argtypes = [C.c_float] * 4
        L.orc_polar.argtypes = [fp, fp, fp, fp]
        u32p = C.POINTER(C.c_uint32)
        L.orc_tri_pairs.restype = C.c_uint64
        L.orc_tri_pairs.argtypes = [C.c_uint32, fp, fp, fp, C.c_uint32, u32p, C.c_float, C.c_int, u32p, C.c_uint64]
        L.orc_ccd_hits.restype = C.c_float
        L.orc_ccd_hits.argtypes = [C.c_uint32] + [fp] * 6 + [C.c_uint32, u32p, C.c_uint64, u32p, u32p,
                                                             C.c_uint64, C.POINTER(C.c_uint64)]
        L.orc_detect.argtypes = [C.c_void_p, C.POINTER(Contact), C.c_float, fp, fp, fp] + [fp] * 6 + [
            C.POINTER(C.c_uint8), fp, u32p]
        _lib = L
    return _lib


def _f(a):
    return np.ascontiguousarray(a, dtype=np.float32).ctypes.data_as(C.POINTER(C.c_float))


def vec3(v):
    return (C.c_float * 3)(*[float(x) for x in v])


class OracleSim:
    """One oracle simulation (ProjectiveDynamicsSolver + SimulationState)."""

    def __init__(self, mesh, params: Params, config: Config, precision: int = 0):
        L = lib()
        self.nv = mesh.nv
        self._keep = [np.ascontiguousarray(a) for a in (mesh.px, mesh.py, mesh.pz)]
        tris = np.ascontiguousarray(mesh.tris, dtype=np.uint32)
        pin = np.ascontiguousarray(mesh.pinned, dtype=np.uint8)
        st = C.c_int32(0)
        self.params, self.config = params, config
        self.h = L.orc_create(precision, mesh.nv, _f(mesh.px), _f(mesh.py), _f(mesh.pz), mesh.nt,
                              tris.ctypes.data_as(C.POINTER(C.c_uint32)),
                              pin.ctypes.data_as(C.POINTER(C.c_uint8)), C.byref(params),
                              C.byref(config), C.byref(st))
        self.status = st.value

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def step(self, dt):
        r = StepResult()
        lib().orc_step(self.h, dt, C.byref(r))
        return r

    def step_ipc(self, dt, contact: Contact):
        r = StepResult()
        lib().orc_step_ipc(self.h, dt, C.byref(contact), C.byref(r))
        return r

    def set_ground(self, has, h=0.0):
        lib().orc_set_ground(self.h, int(has), float(h))

    def resolve(self, contact: Contact) -> np.ndarray:
        """The colliders' resolve() after a plain step; rows ground, sphere, cylinder, box of
        (resolved count, max penetration, depth sum)."""
        out = np.zeros(12, np.float32)
        lib().orc_resolve(self.h, C.byref(contact), out.ctypes.data_as(C.POINTER(C.c_float)))
        return out.reshape(4, 3)

    def state(self):
        out = [np.zeros(self.nv, np.float32) for _ in range(6)]
        lib().orc_get_state(self.h, *[_f(a) if False else a.ctypes.data_as(C.POINTER(C.c_float)) for a in out])
        return np.stack(out[:3], 1), np.stack(out[3:], 1)

    def set_state(self, pos, vel):
        pos = np.ascontiguousarray(pos, np.float32)
        vel = np.ascontiguousarray(vel, np.float32)
        cols = [np.ascontiguousarray(pos[:, k]) for k in range(3)] + [np.ascontiguousarray(vel[:, k]) for k in range(3)]
        lib().orc_set_state(self.h, *[c.ctypes.data_as(C.POINTER(C.c_float)) for c in cols])

    def masses(self):
        m = np.zeros(self.nv, np.float32)
        lib().orc_get_masses(self.h, m.ctypes.data_as(C.POINTER(C.c_float)))
        return m

    def hinges(self):
        nh = lib().orc_hinge_count(self.h)
        v = np.zeros((nh, 4), np.uint32)
        rest = np.zeros(nh, np.float32)
        w = np.zeros(nh, np.float32)
        st = np.zeros((nh, 4), np.float32)
        lib().orc_get_hinges(self.h, v.ctypes.data_as(C.POINTER(C.c_uint32)), rest.ctypes.data_as(C.POINTER(C.c_float)),
                             w.ctypes.data_as(C.POINTER(C.c_float)), st.ctypes.data_as(C.POINTER(C.c_float)))
        return v, rest, w, st

    def matrix(self):
        L = lib()
        nnz = L.orc_matrix_nnz(self.h)
        rp = np.zeros(self.nv + 1, np.uint32)
        ci = np.zeros(nnz, np.uint32)
        va = np.zeros(nnz, np.float64)
        L.orc_get_matrix(self.h, rp.ctypes.data_as(C.POINTER(C.c_uint32)), ci.ctypes.data_as(C.POINTER(C.c_uint32)),
                         va.ctypes.data_as(C.POINTER(C.c_double)))
        return rp, ci, va

    def factor_nnz(self):
        return int(lib().orc_factor_nnz(self.h))

    def solve(self, b):
        b = np.ascontiguousarray(b, np.float32)
        x = np.zeros_like(b)
        lib().orc_solve(self.h, b.ctypes.data_as(C.POINTER(C.c_float)), x.ctypes.data_as(C.POINTER(C.c_float)))
        return x

    def detect(self, contact: Contact, d_hat, pos):
        n = self.nv
        pos = np.ascontiguousarray(pos, np.float32)
        cols = [np.ascontiguousarray(pos[:, k]) for k in range(3)]
        outs = [np.zeros(n, np.float32) for _ in range(6)]
        inc = np.zeros(n, np.uint8)
        mv = C.c_float(0)
        act = C.c_uint32(0)
        lib().orc_detect(self.h, C.byref(contact), d_hat, *[c.ctypes.data_as(C.POINTER(C.c_float)) for c in cols],
                         *[o.ctypes.data_as(C.POINTER(C.c_float)) for o in outs],
                         inc.ctypes.data_as(C.POINTER(C.c_uint8)), C.byref(mv), C.byref(act))
        return np.stack(outs[:3], 1), np.stack(outs[3:], 1), inc, mv.value, act.value


def tri_pairs(pos, tris, margin, mode=0):
    L = lib()
    pos = np.ascontiguousarray(pos, np.float32)
    tris = np.ascontiguousarray(tris, np.uint32)
    cols = [np.ascontiguousarray(pos[:, k]) for k in range(3)]
    u32p = C.POINTER(C.c_uint32)
    cnt = L.orc_tri_pairs(pos.shape[0], *[c.ctypes.data_as(C.POINTER(C.c_float)) for c in cols], tris.shape[0],
                          tris.ctypes.data_as(u32p), margin, mode, None, 0)
    out = np.zeros((max(cnt, 1), 2), np.uint32)
    L.orc_tri_pairs(pos.shape[0], *[c.ctypes.data_as(C.POINTER(C.c_float)) for c in cols], tris.shape[0],
                    tris.ctypes.data_as(u32p), margin, mode, out.ctypes.data_as(u32p), cnt)
    return out[:cnt]


def ccd_hits(p0, p1, tris, pairs):
    L = lib()
    p0 = np.ascontiguousarray(p0, np.float32)
    p1 = np.ascontiguousarray(p1, np.float32)
    tris = np.ascontiguousarray(tris, np.uint32)
    pairs = np.ascontiguousarray(pairs, np.uint32)
    u32p = C.POINTER(C.c_uint32)
    cols = [np.ascontiguousarray(p[:, k]) for p in (p0, p1) for k in range(3)]
    cap = 6 * max(len(pairs), 1)
    hits = np.zeros((cap, 2), np.uint32)
    nh = C.c_uint64(0)
    mt = L.orc_ccd_hits(p0.shape[0], *[c.ctypes.data_as(C.POINTER(C.c_float)) for c in cols], tris.shape[0],
                        tris.ctypes.data_as(u32p), len(pairs), pairs.ctypes.data_as(u32p),
                        hits.ctypes.data_as(u32p), cap, C.byref(nh))
    return hits[: nh.value], mt


def sparse_solve(rows, cols, triplets, rhs):
    """orc_sparse_solve on a CSR built from (row, col, value) triplets, rows
    sorted by column (CsrMatrix::from_triplets, crates/vistio-math/src/sparse.rs).
    Returns (status, solution)."""
    by_row = [[] for _ in range(rows)]
    for r, c, v in triplets:
        by_row[r].append((c, v))
    ptr, col, val = [0], [], []
    for r in range(rows):
        for c, v in sorted(by_row[r], key=lambda e: e[0]):
            col.append(c)
            val.append(v)
        ptr.append(len(col))
    ptr = np.asarray(ptr, np.uint32)
    col = np.asarray(col if col else [0], np.uint32)
    val = np.asarray(val if val else [0.0], np.float32)
    b = np.ascontiguousarray(rhs, np.float32)
    x = np.zeros(max(rows, 1), np.float32)
    st = lib().orc_sparse_solve(rows, cols, ptr.ctypes.data_as(C.POINTER(C.c_uint32)),
                                col.ctypes.data_as(C.POINTER(C.c_uint32)), val.ctypes.data_as(C.POINTER(C.c_float)),
                                b.ctypes.data_as(C.POINTER(C.c_float)), x.ctypes.data_as(C.POINTER(C.c_float)))
    return st, x[:rows]
