"""The allocation-free dense solve against the regular factor-only entry
point.

sdfgpu_dense_ldlt_solve_noalloc serves callers that cannot allocate device
memory when they solve (a host framework's caching allocator already holds
the free memory, or a real-time loop allows no allocation after start-up): it
keeps its work in a fixed file-scope device array instead. This file is
collected last so that a failure here comes after every other test has run;
it passes alone in a fresh process and after the rest of the suite.
"""
import ctypes

import numpy as np
import pytest

import sdf_slam_b200 as P

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the factor-only LDL^T tolerance of the parity tests


def _spd(n, seed):
    rng = np.random.default_rng(seed)
    m = rng.uniform(-1.0, 1.0, (n, n))
    return m @ m.T + n * np.eye(n), rng.uniform(-1.0, 1.0, n)


def _noalloc(a, b):
    n = len(b)
    a = np.asfortranarray(a, dtype=np.float64)
    b = np.ascontiguousarray(b, dtype=np.float64)
    x = np.zeros(n)
    rc = P.lib().sdfgpu_dense_ldlt_solve_noalloc(
        n, a.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), b.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
        x.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    P._check(rc)
    return x


def _existing(a, b):
    n = len(b)
    outer = np.arange(0, n * n + 1, n, dtype=np.int32)
    inner = np.tile(np.arange(n, dtype=np.int32), n)
    solver = P.LdltSolver(n, outer, inner)
    solver.factorize(np.asfortranarray(a).reshape(-1, order="F"))
    x = solver.solve(b)
    solver.close()
    return x


def test_noalloc_matches_existing_entry_point_on_two_calls_in_a_row():
    for n, seed in [(700, 1), (333, 2)]:
        a, b = _spd(n, seed)
        x = _noalloc(a, b)
        ref = _existing(a, b)
        assert np.linalg.norm(x - ref) / np.linalg.norm(ref) <= TOL
        assert np.linalg.norm(a @ x - b) / np.linalg.norm(b) <= 1e-12


def test_noalloc_rejects_sizes_beyond_the_maximum():
    n = 1025
    a = np.eye(n)
    with pytest.raises(ValueError, match="outside 1..1024"):
        _noalloc(a, np.ones(n))


def test_noalloc_zero_pivot_fails_then_next_call_succeeds():
    """A zero pivot gives SDFGPU_ERR_NUMERICAL with the reference's message
    (lm_solver.cpp:354-362); the next call clears the shared status word and
    solves normally."""
    n = 200
    d = np.full(n, 2.0)
    d[n // 2] = 0.0
    with pytest.raises(RuntimeError, match="factorization failed"):
        _noalloc(np.diag(d), np.ones(n))
    a, b = _spd(150, 3)
    x = _noalloc(a, b)
    ref = _existing(a, b)
    assert np.linalg.norm(x - ref) / np.linalg.norm(ref) <= TOL
