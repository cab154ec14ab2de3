"""g2oc_solve_block_system_static: the PCG block solve for callers that cannot
allocate device memory (a GPU process with capped or pre-partitioned memory,
a caller-owned allocator, a plugin that must not grow the device footprint).
Its scratch is a file-scope device array, so it must give the same answer as
g2oc_solve_block_system, which allocates, on consecutive calls that reuse the
scratch. Collected last on purpose (file name), and independent of the other
test files' state.
"""
import ctypes as C

import numpy as np
import pytest

from g2o_b200.abi import LINEAR_PCG

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative; the two entry points run the same kernels in the same order


def _p(a, t=C.c_double):
    return a.ctypes.data_as(C.POINTER(t))


def static_solve(L, offs, rc, vals, b, tol, maxit):
    bs = int(offs[1] - offs[0])
    x = np.zeros_like(b)
    it = C.c_int32()
    rc = np.ascontiguousarray(rc, np.int32)
    vals = np.ascontiguousarray(vals, np.float64)
    st = L.g2oc_solve_block_system_static(0, len(offs) - 1, bs, len(rc), _p(rc, C.c_int32), _p(vals), _p(b), _p(x),
                                          tol, maxit, C.byref(it))
    return st, x, it.value


def random_spd_system(nb, bs, density, seed):
    rng = np.random.default_rng(seed)
    pattern = [(r, c) for c in range(nb) for r in range(c + 1) if r == c or rng.random() < density]
    n = nb * bs
    A = np.zeros((n, n))
    vals = []
    for r, c in pattern:
        M = rng.normal(size=(bs, bs))
        if r == c:
            M = M @ M.T + 4 * nb * np.eye(bs)
        vals.append(M)
        A[r * bs:(r + 1) * bs, c * bs:(c + 1) * bs] = M
        if r != c:
            A[c * bs:(c + 1) * bs, r * bs:(r + 1) * bs] = M.T
    offs = np.arange(nb + 1, dtype=np.int32) * bs
    return offs, np.array(pattern, np.int32), np.concatenate([v.ravel() for v in vals]), rng.normal(size=n), A


def cases():
    from tests.test_oracle_pinning import load_sparse_system
    offs, rc, vals, b, _, _ = load_sparse_system()
    yield "reference_36x36", offs, rc, vals, b
    o, rc2, v2, b2, _ = random_spd_system(150, 6, 0.2, seed=3)
    yield "random_150x6", o, rc2, v2, b2
    # a full upper pattern of 130 block rows has nnzb = 8515 >= 64 * nb: the
    # 256-thread (wide) row and column passes
    o3, rc3, v3, b3, _ = random_spd_system(130, 6, 1.0, seed=5)
    assert len(rc3) >= 64 * 130
    yield "dense_130x6", o3, rc3, v3, b3


@pytest.mark.parametrize("tol,maxit", [(1e-6, -1), (1e-20, 200)])
def test_static_entry_point_matches_allocating_one(tol, maxit):
    from g2o_b200 import backend
    L = backend.library()
    prm = backend.default_params(pcg_tolerance=tol, pcg_max_iterations=maxit)
    for name, offs, rc, vals, b in cases():
        st_ref, x_ref, it_ref = backend.solve_block_system(LINEAR_PCG, offs, rc, vals, b, prm)
        assert st_ref == 0, name
        for call in range(2):  # the second call reuses the scratch the first left behind
            st, x, it = static_solve(L, offs, rc, vals, b, tol, maxit)
            assert st == 0, (name, call, L.g2oc_last_error())
            assert it == it_ref, (name, call, it, it_ref)
            assert np.linalg.norm(x - x_ref) <= TOL * np.linalg.norm(x_ref), (name, call)


def test_static_entry_point_solves_reference_fixture():
    # the reference's 36x36 system: the solution within its test's
    # isApprox(1e-6) (unit_test/solver/linear_solver_test.cpp:84-101), twice
    from g2o_b200 import backend
    from tests.test_oracle_pinning import is_approx, load_sparse_system
    L = backend.library()
    offs, rc, vals, b, x_ref, _ = load_sparse_system()
    for call in range(2):
        st, x, it = static_solve(L, offs, rc, vals, b, 1e-20, 200)
        assert st == 0 and it > 0, (call, L.g2oc_last_error())
        assert is_approx(x, x_ref, 1e-6), call


def test_static_entry_point_keeps_the_callers_device():
    import torch
    from g2o_b200 import backend
    L = backend.library()
    torch.cuda.set_device(0)
    offs, rc, vals, b, _ = random_spd_system(20, 3, 0.3, seed=9)[:5]
    st, _, _ = static_solve(L, offs, rc, vals, b, 1e-6, -1)
    assert st == 0
    assert torch.cuda.current_device() == 0


def test_static_entry_point_rejects_oversized_systems():
    from g2o_b200 import backend
    L = backend.library()
    nb, bs = 4000, 6
    offs = np.arange(nb + 1, dtype=np.int32) * bs
    rc = np.array([(i, i) for i in range(nb)], np.int32)
    vals = np.tile(np.eye(bs).ravel(), nb)
    b = np.ones(nb * bs)
    # 4000 diagonal 6x6 blocks fit; a dense upper pattern of 4000 rows does not
    st, x, _ = static_solve(L, offs, rc, vals, b, 1e-6, -1)
    assert st == 0 and np.allclose(x, 1.0)
    nb2 = 400
    offs2 = np.arange(nb2 + 1, dtype=np.int32) * bs
    rc2 = np.array([(r, c) for c in range(nb2) for r in range(c + 1)], np.int32)
    vals2 = np.zeros(len(rc2) * bs * bs)
    st2, _, _ = static_solve(L, offs2, rc2, vals2, np.ones(nb2 * bs), 1e-6, -1)
    assert st2 == 1  # G2OC_ERR_INVALID_ARGUMENT
    assert b"static" in L.g2oc_last_error()
