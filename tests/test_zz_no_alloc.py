"""GPU test of vistio_broadphase_pairs_noalloc, the broad phase that allocates
no device memory on the call (its buffers live in a fixed region built into
the library). Its pair lists must equal those of vistio_broadphase_pairs on
the same inputs, call after call: the second and third calls reuse the region
a previous, differently sized call left behind. The cases include a mesh whose
triangles are stored in random order (this entry point builds its tree over
mesh order, without the Morton sort) and one of 64,800 triangles, near the
65,536-triangle limit. Across several calls the device's free memory and the
default memory pool's reserved and used bytes must not change. The module
sorts last so it also runs after every other GPU test in the same process."""
import numpy as np
import pytest

import oracle_api as O
from vistio_b200 import _lib, api, scenarios

pytestmark = pytest.mark.gpu

CAPACITY = 12  # VISTIO_ERR_CAPACITY


def folded_sheet(cols, rows, width, height, gap, seed):
    """A quad-grid strip folded over itself with its layers `gap` apart,
    jittered so that many triangle pairs are close."""
    px, py, pz, tris = scenarios.quad_grid(cols, rows, width, height)
    s = (py - py.min()) / (py.max() - py.min()) * height
    half = height / 2
    y = np.where(s < half, s, height - s)
    z = np.where(s < half, 0.0, gap)
    z = np.where(np.abs(s - half) < height / rows, gap / 2, z)
    rng = np.random.default_rng(seed)
    z = z + rng.uniform(-gap / 8, gap / 8, size=z.shape)
    return np.stack([px, y + 0.5, z], 1).astype(np.float32), tris


def permuted(pos, tris, seed):
    """The same surface with its triangles stored in a random order."""
    order = np.random.default_rng(seed).permutation(len(tris))
    return pos, np.ascontiguousarray(tris[order])


def flat_sheet(side, length, seed):
    """A jittered flat quad-grid sheet (2 side^2 triangles)."""
    px, py, pz, tris = scenarios.quad_grid(side, side, length, length)
    rng = np.random.default_rng(seed)
    pos = np.stack([px, rng.uniform(-2e-4, 2e-4, px.shape).astype(np.float32) + 0.5, py], 1)
    return pos.astype(np.float32), tris


CASES = [
    folded_sheet(8, 60, 0.1, 0.6, 0.004, 0) + (7.5e-4,),
    folded_sheet(20, 140, 0.2, 1.4, 0.003, 1) + (1.5e-3,),  # 5600 triangles, a larger tree
    folded_sheet(3, 5, 0.05, 0.1, 0.002, 2) + (1e-3,),
    permuted(*folded_sheet(20, 140, 0.2, 1.4, 0.003, 1), 4) + (1.5e-3,),  # triangles out of spatial order
    flat_sheet(180, 1.8, 3) + (1e-3,),  # 64,800 triangles, about 546k pairs
]


def test_noalloc_matches_allocating_entry_point_call_after_call():
    for round_ in range(2):
        for pos, tris, margin in CASES:
            ref = api.broadphase_pairs(pos, tris, margin)
            got = api.broadphase_pairs_noalloc(pos, tris, margin)
            assert got.shape == ref.shape, (round_, got.shape, ref.shape)
            assert np.array_equal(got, ref), round_
    # and both equal the oracle's complete overlap set
    pos, tris, margin = CASES[0]
    assert np.array_equal(api.broadphase_pairs_noalloc(pos, tris, margin), O.tri_pairs(pos, tris, margin, mode=0))


def test_noalloc_empty_and_limits():
    pos = np.zeros((3, 3), np.float32)
    assert len(api.broadphase_pairs_noalloc(pos, np.array([[0, 1, 2]], np.uint32), 1e-3)) == 0
    # more triangles than the fixed region holds: rejected with CAPACITY
    px, py, pz, tris = scenarios.quad_grid(190, 190, 1.0, 1.0)  # 72200 triangles
    big = np.stack([px, py, pz], 1)
    with pytest.raises(_lib.VistioError) as e:
        api.broadphase_pairs_noalloc(big, tris, 1e-3)
    assert e.value.status == CAPACITY and "65536" in str(e.value)
    # a caller buffer smaller than the pair count: CAPACITY, count reported
    pos, tris, margin = CASES[0]
    n = len(api.broadphase_pairs(pos, tris, margin))
    import ctypes as C
    ctx = api.default_context()
    cols = [np.ascontiguousarray(pos[:, k]) for k in range(3)]
    out = np.zeros((n - 1, 2), np.uint32)
    cnt = C.c_uint64()
    u32 = C.POINTER(C.c_uint32)
    fp = C.POINTER(C.c_float)
    st = _lib.lib().vistio_broadphase_pairs_noalloc(ctx.h, len(pos), *[c.ctypes.data_as(fp) for c in cols],
                                                    len(tris), np.ascontiguousarray(tris, np.uint32).ctypes.data_as(u32),
                                                    margin, out.ctypes.data_as(u32), n - 1, C.byref(cnt))
    assert st == CAPACITY and cnt.value == n


def _device_memory():
    """(free bytes of the device, reserved and used bytes of its default pool)."""
    import torch
    from cuda.bindings import runtime as rt
    torch.cuda.synchronize()
    free, _ = torch.cuda.mem_get_info()
    err, pool = rt.cudaDeviceGetDefaultMemPool(torch.cuda.current_device())
    assert err == rt.cudaError_t.cudaSuccess
    out = [free]
    for attr in (rt.cudaMemPoolAttr.cudaMemPoolAttrReservedMemCurrent, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent):
        err, v = rt.cudaMemPoolGetAttribute(pool, attr)
        assert err == rt.cudaError_t.cudaSuccess
        out.append(int(v))
    return tuple(out)


def test_noalloc_calls_allocate_no_device_memory():
    """After one warm-up call (which may load the library's module), calls of
    four different sizes leave the device's free memory and the default pool's
    reserved and used bytes exactly as they were."""
    got = [len(api.broadphase_pairs_noalloc(p, t, m)) for p, t, m in CASES[:1]]
    before = _device_memory()
    for p, t, m in (CASES[4], CASES[1], CASES[2], CASES[3]):
        got.append(len(api.broadphase_pairs_noalloc(p, t, m)))
    after = _device_memory()
    assert before == after, (before, after)
    assert min(got[1:]) > 0
