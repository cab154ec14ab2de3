"""The C-ABI boundary: header/ctypes layouts agree, the library loads and
exports every declared entry point, and the factory behaves like g2o's
OptimizationAlgorithmFactory (unit_test/solver/allocate_algorithm_test.cpp:48-127).
No GPU compute here."""
import ctypes as C
import os
import subprocess
import tempfile

import pytest

from g2o_b200 import abi, backend

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _c_layout():
    src = r"""
#include <stdio.h>
#include <stddef.h>
#include "g2o_cuda.h"
#define F(T, m) printf(#T "." #m " %zu\n", offsetof(T, m));
int main(void) {
  printf("g2oc_graph %zu\n", sizeof(g2oc_graph));
  F(g2oc_graph, pose_estimate) F(g2oc_graph, num_points) F(g2oc_graph, edge_vertex)
  F(g2oc_graph, robust_delta) F(g2oc_graph, focal_length) F(g2oc_graph, principal_point)
  F(g2oc_graph, focal_length_y)
  printf("g2oc_params %zu\n", sizeof(g2oc_params));
  F(g2oc_params, pcg_tolerance) F(g2oc_params, initial_lambda) F(g2oc_params, refine_tolerance)
  F(g2oc_params, initial_delta) F(g2oc_params, lambda_factor)
  printf("g2oc_iteration_stats %zu\n", sizeof(g2oc_iteration_stats));
  F(g2oc_iteration_stats, chi2) F(g2oc_iteration_stats, time_iteration)
  F(g2oc_iteration_stats, trust_radius) F(g2oc_iteration_stats, dogleg_step)
  printf("g2oc_hessian_info %zu\n", sizeof(g2oc_hessian_info));
  F(g2oc_hessian_info, vector_size) F(g2oc_hessian_info, schur_pairs)
  return 0;
}
"""
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        exe = os.path.join(d, "t")
        open(c, "w").write(src)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), c, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    return dict(line.split() for line in out.strip().splitlines())


def test_struct_layouts_match_header():
    lay = _c_layout()
    structs = {"g2oc_graph": abi.G2ocGraph, "g2oc_params": abi.G2ocParams,
               "g2oc_iteration_stats": abi.G2ocIterationStats, "g2oc_hessian_info": abi.G2ocHessianInfo}
    for name, cls in structs.items():
        assert int(lay[name]) == C.sizeof(cls), name
    for key, val in lay.items():
        if "." in key:
            s, m = key.split(".")
            cls = structs[s]
            field = "lambda_" if m == "lambda" else m
            assert getattr(cls, field).offset == int(val), key


def test_library_exports_every_declared_symbol(cuda_lib):
    names = backend.header_symbols()
    assert len(names) >= 20
    for n in names:
        assert hasattr(cuda_lib, n), n
    assert cuda_lib.g2oc_abi_version() == 5


def test_factory_lists_and_constructs():
    fac = backend.OptimizationAlgorithmFactory.instance()
    names = fac.list_solvers()
    for n in ["gn_cuda", "lm_cuda", "lm_cuda_pcg6_3", "gn_cuda_pcg3_3", "lm_cuda_chol", "lm_cuda_mixed",
              "lm_cuda_mixed_fast"]:
        assert n in names
    for n in names:
        p = fac.construct(n)
        assert p is not None, n
        want = {"gn": abi.ALGO_GAUSS_NEWTON, "lm": abi.ALGO_LEVENBERG, "dl": abi.ALGO_DOGLEG,
                "st": abi.ALGO_STRUCTURE_ONLY}[n[:2]]
        assert p.algorithm == want, n
    assert fac.construct("lm_cuda_mixed").precision == abi.PREC_MIXED
    assert fac.construct("lm_cuda_mixed").refine_max_iterations == 2
    fast = fac.construct("lm_cuda_mixed_fast")
    assert fast.precision == abi.PREC_MIXED and fast.refine_max_iterations == -1
    assert fac.construct("gn_cuda_chol").linear_solver == abi.LINEAR_CHOLESKY
    assert fac.construct("gn_cuda_pcg6_3").linear_solver == abi.LINEAR_PCG
    dl = fac.construct("dl_cuda_chol")
    # OptimizationAlgorithmDogleg's property defaults (optimization_algorithm_dogleg.cpp:44-51)
    assert dl.linear_solver == abi.LINEAR_CHOLESKY and dl.max_trials_after_failure == 100
    assert dl.initial_lambda == 1e-7 and dl.initial_delta == 1e4 and dl.lambda_factor == 10.0
    assert fac.construct("non_existing_solver") is None
    assert fac.construct("") is None


def test_default_params_are_the_reference_defaults():
    p = backend.default_params()
    assert p.pcg_tolerance == 1e-6 and p.pcg_max_iterations == -1 and p.pcg_absolute_tolerance == 1
    assert p.max_trials_after_failure == 10 and p.tau == 1e-5 and p.initial_lambda == 0.0


def test_create_without_device_reports_no_device(cuda_lib):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("a CUDA device is present")
    except ImportError:
        pass
    h = C.c_void_p()
    st = cuda_lib.g2oc_create(0, C.byref(h))
    assert st == abi.G2OC_ERR_NO_DEVICE
    assert not h.value


def test_static_block_solve_rejects_argument_errors_before_the_device(cuda_lib):
    # g2oc_solve_block_system_static checks its arguments and the host-scratch
    # bound before it touches a device, so these run without a GPU
    import numpy as np

    def call(nb, bs, rc, vals, b, device=0):
        x = np.zeros_like(b)
        it = C.c_int32()
        rc = np.ascontiguousarray(rc, np.int32)
        return cuda_lib.g2oc_solve_block_system_static(
            device, nb, bs, len(rc), rc.ctypes.data_as(C.POINTER(C.c_int32)),
            vals.ctypes.data_as(C.POINTER(C.c_double)), b.ctypes.data_as(C.POINTER(C.c_double)),
            x.ctypes.data_as(C.POINTER(C.c_double)), 1e-6, -1, C.byref(it))

    # a full upper pattern of 1300 block rows: 845,650 blocks, past the host
    # list bound (5 * nnzb + 4 * nb + 8 ints of 4 Mi)
    nb = 1300
    cols = np.repeat(np.arange(nb), np.arange(1, nb + 1))
    rows = np.concatenate([np.arange(c + 1) for c in range(nb)])
    rc = np.stack([rows, cols], axis=1)
    vals = np.zeros(len(rc) * 9)
    b = np.ones(nb * 3)
    assert call(nb, 3, rc, vals, b) == abi.G2OC_ERR_INVALID_ARGUMENT
    assert b"static scratch" in cuda_lib.g2oc_last_error()
    # lower-triangle block, unsupported block size, bad device
    small = np.array([[1, 0]], np.int32)
    assert call(2, 3, small, np.zeros(9), np.ones(6)) == abi.G2OC_ERR_INVALID_ARGUMENT
    assert call(1, 4, np.array([[0, 0]]), np.zeros(16), np.ones(4)) == abi.G2OC_ERR_INVALID_ARGUMENT
    assert call(1, 3, np.array([[0, 0]]), np.eye(3).ravel(), np.ones(3), device=-1) == abi.G2OC_ERR_INVALID_ARGUMENT
