"""CPU tests of the C-ABI boundary and the host-side set-up (no GPU calls)."""
import ctypes as C
import json
import os
import re
import subprocess

import numpy as np
import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "vistio_cuda.h")


def declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(vistio_[a-z0-9_]+)\s*\(", src)))


def test_library_loads_and_exports_every_declared_symbol():
    from vistio_b200 import _lib

    L = _lib.lib()
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # the Python binding declares a signature for every header entry point
    assert set(names) == set(_lib.SIGNATURES), set(names) ^ set(_lib.SIGNATURES)


def test_status_strings():
    from vistio_b200 import _lib

    L = _lib.lib()
    assert L.vistio_status_string(0) == b"ok"
    assert L.vistio_status_string(11) == b"matrix not positive definite"


def test_no_device_reports_gpu_error_not_fallback():
    """Without a GPU the context fails loudly (VISTIO_ERR_GPU); there is no CPU path."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from vistio_b200 import _lib

    h = C.c_void_p()
    assert _lib.lib().vistio_ctx_create(0, C.byref(h)) == 6


@pytest.fixture(scope="module")
def factor_check_bin(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("fc") / "factor_check")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-o", out, os.path.join(ROOT, "tests", "cpp", "factor_check.cpp"),
                           os.path.join(ROOT, "vistio_b200", "csrc", "setup.cpp")])
    return out


@pytest.mark.parametrize("grid", [(20, 20, 1.0), (64, 64, 1.5), (40, 400, 0.2), (16, 16, 0.5), (3, 1, 1.0)])
def test_supernodal_layout_replays_exactly(factor_check_bin, grid):
    """The level-scheduled supernodal sweeps over the packed factor solve A x = b
    (FP64 replay ~1e-14, FP32 replay ~1e-5 relative residual). One FP64
    refinement with the permuted f64 matrix, formed as the GPU forms it, brings
    the FP32 solution to within FP32 rounding (~3e-8) of the FP64 solution.
    The symbolic-only set-up (numeric factorization on the device) has the same
    structure, and a CPU replay of the device's multifrontal factorization
    (fronts, extend-add through the child-row maps, partial Cholesky, inverted
    diagonal blocks) reproduces the host factor to FP64 rounding."""
    out = subprocess.check_output([factor_check_bin] + [str(g) for g in grid])
    r = json.loads(out)
    assert r["resid64"] < 1e-11, r
    assert r["resid32"] < 1e-4, r
    assert r["resid32_refined"] < r["resid32"], r
    assert r["err32_refined"] < min(6e-8, r["err32"] / 3), r
    assert r["levels"] <= 32
    assert r["symbolic_same"] == 1, r
    assert r["multifrontal_diff"] < 1e-12, r


def test_hanging_sheet_sizes_and_hinges():
    """bench_tests.rs:14-31: hanging_sheet has 441 vertices and 800 triangles;
    a 20x20 grid has 1160 interior edges."""
    from vistio_b200 import scenarios
    import oracle_api as O

    m = scenarios.hanging_sheet(20)
    assert (m.nv, m.nt) == (441, 800)
    assert int(m.pinned.sum()) == 21
    sim = O.OracleSim(m, O.init_params(), O.default_config())
    assert len(sim.hinges()[1]) == 1160
    rp, ci, va = sim.matrix()
    assert len(ci) == 4517  # summed nonzeros of A for the 441-vertex sheet


def test_quad_grid_matches_reference_generator():
    """The product's numpy quad_grid is bit-identical to the oracle's restatement."""
    from vistio_b200 import scenarios
    import oracle_api as O

    for cols, rows, w, h in [(20, 20, 1.0, 1.0), (7, 3, 0.3, 1.7), (64, 64, 1.5, 1.5)]:
        px, py, pz, tris = scenarios.quad_grid(cols, rows, w, h)
        n = (cols + 1) * (rows + 1)
        a = [np.zeros(n, np.float32) for _ in range(3)]
        t = np.zeros(cols * rows * 6, np.uint32)
        O.lib().orc_quad_grid(cols, rows, w, h, *[x.ctypes.data_as(C.POINTER(C.c_float)) for x in a],
                              t.ctypes.data_as(C.POINTER(C.c_uint32)))
        assert np.array_equal(px, a[0]) and np.array_equal(py, a[1]) and np.array_equal(pz, a[2])
        assert np.array_equal(tris.reshape(-1), t)


def test_symbolic_cache_hits_equal_fresh_analyses(tmp_path):
    """The host's symbolic-analysis cache (factorize_csr, numeric = false): a hit
    is the Factor a fresh analysis gives, field for field (grids with pins, DS
    bending, perturbed geometry); uniformly scaled copies of a grid share one
    entry; concurrent set-ups of one mesh run one analysis; the byte bound
    evicts, and 0 empties it."""
    out = str(tmp_path / "scc")
    subprocess.check_call(["g++", "-O2", "-std=c++17", "-o", out,
                           os.path.join(ROOT, "tests", "cpp", "symbolic_cache_check.cpp"),
                           os.path.join(ROOT, "vistio_b200", "csrc", "setup.cpp"), "-lpthread"])
    r = json.loads(subprocess.check_output([out]))
    assert r["identical"] == r["cases"] and r["scaled_same"] == r["scales"], r
    assert r["scaled_ok"] and r["concurrent_ok"] and r["evict_ok"] and r["zero_ok"], r


def test_symbolic_cache_entry_points_without_a_device():
    from vistio_b200 import api
    info = api.symbolic_cache_info()
    assert set(info) == {"hits", "misses", "bytes", "entries"}
    api.set_symbolic_cache_limit(0)
    assert api.symbolic_cache_info()["entries"] == 0
    api.set_symbolic_cache_limit(1 << 30)
