"""Procedural inputs for the drape workloads (host-side set-up, numpy).

`quad_grid` restates the reference's generator
(crates/vistio-mesh/src/generators.rs:28-100) in float32 with the same
operation order, so meshes are bit-identical to the reference's.  The
scenario builders follow crates/vistio-bench/src/scenarios.rs:84-147 with the
parameter mapping of the drape workloads:

* hanging_sheet: 1 m x 1 m, 20x20 cells, rotated into XZ at y = 1.0, the
  first 21 vertices pinned, no contact.
* sphere_drape: 1.5 m x 1.5 m, 64x64 cells, sheet plane y = 0.5, sphere at the
  origin r = 0.3, ground y = -0.3 (runner.rs:77-81).
* cusick_drape: a disc of radius 0.15 m (`circular_grid`, generators.rs:174)
  at y = 0.5 over a pedestal cylinder (top y = 0.3, r = 0.09) and the ground.
* cantilever_bending: a 0.1 m x 0.4 m strip at y = 0.5, three rows pinned, the
  free end over a box shelf, stepped without IPC (scenarios.rs:176-201,
  runner.rs:87-90).
* self_fold: 0.2 m x 2.0 m, 40x400 cells, rotated 45 degrees about x with the
  lowest point at y = 0.5, ground y = 0, self contact.
* batched sheets: hanging sheets of random side / size / material.

The reference is Y-up (gravity (0, -9.81, 0)); a "z" in the workload text
means the reference's y.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

SEED = 20261203


def quad_grid(cols: int, rows: int, width: float, height: float):
    """Flat grid in the XY plane with checkerboard diagonals (generators.rs:28)."""
    f32 = np.float32
    vx, vy = cols + 1, rows + 1
    hw, hh = f32(width) / f32(2.0), f32(height) / f32(2.0)
    i = np.arange(vx, dtype=np.float32)
    j = np.arange(vy, dtype=np.float32)
    u = (i / f32(cols)).astype(np.float32)
    v = (j / f32(rows)).astype(np.float32)
    x = (-hw + u * f32(width)).astype(np.float32)
    y = (hh - v * f32(height)).astype(np.float32)
    px = np.tile(x, vy).astype(np.float32)
    py = np.repeat(y, vx).astype(np.float32)
    pz = np.zeros(vx * vy, dtype=np.float32)
    jj, ii = np.meshgrid(np.arange(rows, dtype=np.int64), np.arange(cols, dtype=np.int64), indexing="ij")
    tl = (jj * vx + ii).ravel()
    tr, bl = tl + 1, tl + vx
    br = bl + 1
    even = ((ii + jj) % 2 == 0).ravel()
    t_even = np.stack([tl, bl, tr, tr, bl, br], axis=1)
    t_odd = np.stack([tl, bl, br, tl, br, tr], axis=1)
    tris = np.where(even[:, None], t_even, t_odd).reshape(-1, 3).astype(np.uint32)
    return px, py, pz, tris


def circular_grid(radius: float, segments: int):
    """Disc in the XY plane (generators.rs:174-240): a (segments // 2)^2 grid of
    side 2 radius keeps the vertices within 1.01 radius and the cells whose
    four corners it kept, with the quad grid's checkerboard diagonals; float32
    with the same operation order."""
    f32 = np.float32
    n = segments // 2
    w = f32(radius) * f32(2.0)
    hw = w / f32(2.0)
    i = np.arange(n + 1, dtype=np.float32)
    u = (i / f32(n)).astype(np.float32)
    x = (-hw + u * w).astype(np.float32)  # along columns
    y = (hw - u * w).astype(np.float32)   # along rows
    gx = np.tile(x, n + 1).astype(np.float32)
    gy = np.repeat(y, n + 1).astype(np.float32)
    keep = np.sqrt((gx * gx + gy * gy).astype(np.float32)).astype(np.float32) <= f32(radius) * f32(1.01)
    vmap = np.full((n + 1) * (n + 1), -1, dtype=np.int64)
    vmap[keep] = np.arange(int(keep.sum()))
    tris = []
    for j in range(n):
        for c in range(n):
            tl = j * (n + 1) + c
            tr, bl = tl + 1, tl + n + 1
            br = bl + 1
            q = [vmap[tl], vmap[tr], vmap[bl], vmap[br]]
            if min(q) < 0:
                continue
            a, b, cc, d = q
            tris += [a, cc, b, b, cc, d] if (c + j) % 2 == 0 else [a, cc, d, a, d, b]
    return (gx[keep].copy(), gy[keep].copy(), np.zeros(int(keep.sum()), dtype=np.float32),
            np.asarray(tris, dtype=np.uint32).reshape(-1, 3))


@dataclasses.dataclass
class Mesh:
    px: np.ndarray
    py: np.ndarray
    pz: np.ndarray
    tris: np.ndarray  # (T, 3) uint32
    pinned: np.ndarray  # (V,) uint8

    @property
    def nv(self) -> int:
        return int(self.px.shape[0])

    @property
    def nt(self) -> int:
        return int(self.tris.shape[0])


def hanging_sheet(side: int = 20, length: float = 1.0, height: float = 1.0) -> Mesh:
    """scenarios.rs:84-114: rotate into XZ at y = height, pin the first row."""
    px, py, pz, tris = quad_grid(side, side, length, length)
    pz = py.copy()
    py = np.full_like(px, np.float32(height))
    pinned = np.zeros(px.shape[0], dtype=np.uint8)
    pinned[: side + 1] = 1
    return Mesh(px, py, pz, tris, pinned)


def sphere_drape(side: int = 64, length: float = 1.5, height: float = 0.5) -> Mesh:
    """scenarios.rs:120-147 with the sheet plane at y = 0.5; nothing pinned."""
    px, py, pz, tris = quad_grid(side, side, length, length)
    pz = py.copy()
    py = np.full_like(px, np.float32(height))
    return Mesh(px, py, pz, tris, np.zeros(px.shape[0], dtype=np.uint8))


def cusick_drape(height: float = 0.5, radius: float = 0.15, segments: int = 64) -> Mesh:
    """scenarios.rs:151-174: a disc of radius 0.15 m (circular_grid(0.15, 64)),
    turned into the XZ plane at y = `height` (0.5 in the reference), nothing
    pinned; the runner adds a pedestal cylinder (axis at the origin, top y =
    0.3, radius 0.09) and the ground at y = -0.3 (runner.rs:83-86)."""
    px, py, pz, tris = circular_grid(radius, segments)
    pz = py.copy()
    py = np.full_like(px, np.float32(height))
    return Mesh(px, py, pz, tris, np.zeros(px.shape[0], dtype=np.uint8))


def cantilever_bending(cols: int = 10, rows: int = 40, width: float = 0.10, length: float = 0.40) -> Mesh:
    """scenarios.rs:176-201: a 0.1 m x 0.4 m strip at y = 0.5, its first three
    rows (z = 0.4 down to 0.38) pinned, its last row at z = 0 over the edge of
    the box x in [-0.1, 0.1], y in [0, 0.499], z in [-0.2, 0] that the runner
    adds (runner.rs:87-90); the runner steps it without IPC and resolves the
    box after every step."""
    px, py, pz, tris = quad_grid(cols, rows, width, length)
    pz = (py + np.float32(0.20)).astype(np.float32)
    py = np.full_like(px, np.float32(0.5))
    pinned = np.zeros(px.shape[0], dtype=np.uint8)
    pinned[: 3 * (cols + 1)] = 1
    return Mesh(px, py, pz, tris, pinned)


CANTILEVER_BOX = ((-0.1, 0.0, -0.2), (0.1, 0.499, 0.0))  # (min, max) of the shelf, runner.rs:87-90


def self_fold(cols: int = 40, rows: int = 400, width: float = 0.2, height: float = 2.0,
              lowest: float = 0.5) -> Mesh:
    """Ribbon rotated 45 degrees about x, lowest point at y = `lowest`."""
    px, py, pz, tris = quad_grid(cols, rows, width, height)
    c = np.float32(math.cos(math.pi / 4))
    s = np.float32(math.sin(math.pi / 4))
    ny = (py * c - pz * s).astype(np.float32)
    nz = (py * s + pz * c).astype(np.float32)
    ny = (ny + (np.float32(lowest) - ny.min())).astype(np.float32)
    return Mesh(px, ny, nz, tris, np.zeros(px.shape[0], dtype=np.uint8))


@dataclasses.dataclass
class SheetSpec:
    side: int
    length: float
    stretch: float   # element stiffness k (N/m): weight = k * area
    bending: float   # hinge stiffness k_b (N m): weight = k_b * edge length
    density_gsm: float


def batched_specs(n_instances: int = 512, n_topologies: int = 8, side_lo: int = 16, side_hi: int = 128,
                  seed: int = SEED):
    """The batched workload: 8 grid sides drawn once and assigned round-robin;
    per instance a side length in [0.5, 2] m, stretch log-uniform in
    [2e2, 5e3] N/m, bending log-uniform in [1e-5, 1e-3] N m and density
    uniform in [0.08, 0.30] kg/m^2."""
    rng = np.random.default_rng(seed)
    sides = rng.integers(side_lo, side_hi + 1, size=n_topologies)
    specs = []
    for k in range(n_instances):
        specs.append(SheetSpec(
            side=int(sides[k % n_topologies]),
            length=float(rng.uniform(0.5, 2.0)),
            stretch=float(math.exp(rng.uniform(math.log(2e2), math.log(5e3)))),
            bending=float(math.exp(rng.uniform(math.log(1e-5), math.log(1e-3)))),
            density_gsm=float(rng.uniform(0.08, 0.30) * 1000.0),
        ))
    return specs
