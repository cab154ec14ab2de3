// lm_kernels.cuh -- Levenberg-Marquardt control on the device
// (OptimizationAlgorithmLevenberg::solve / computeLambdaInit / computeScale,
// g2o/core/optimization_algorithm_levenberg.cpp:60-176) and small vector
// kernels shared by the paths.
#pragma once

#include "g2oc_internal.h"
#include "pcg_kernels.cuh"
#include "reduce.cuh"

namespace g2oc {

// lambda_0 = initialLambda if set, else tau * max diag(H); ni = 2
static __global__ void lm_init_lambda(DevScalars* sc, double user_lambda, double tau) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    sc->lambda = user_lambda > 0.0 ? user_lambda : tau * sc->max_diag;
    sc->ni = 2.0;
  }
}

// One trial's decision. rho = (chi_current - chi_temp) / (scale + 1e-3);
// accept: lambda *= max(1/3, min(2/3, 1 - (2 rho - 1)^3)), ni = 2;
// reject: lambda *= ni, ni *= 2 (estimates restored by the host).
static __global__ void lm_decide(DevScalars* sc) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  const bool ok2 = sc->solve_ok != 0;
  double tempChi = sc->chi2_temp;
  if (!ok2) tempChi = 1.79769313486231570815e+308;
  double rho = sc->chi2_current - tempChi;
  const double scale = ok2 ? sc->scale : 1.0;  // sc->scale already holds computeScale() + 1e-3
  rho /= scale;
  if (rho > 0 && isfinite(tempChi) && ok2) {
    double alpha = 1. - pow((2 * rho - 1), 3);
    alpha = fmin(alpha, 2. / 3.);
    const double scaleFactor = fmax(1. / 3., alpha);
    sc->lambda *= scaleFactor;
    sc->ni = 2;
    sc->chi2_current = tempChi;
    sc->chi2_plain = sc->chi2_temp_plain;  // the accepted state's errors are the current ones
    sc->accept = 1;
  } else {
    sc->lambda *= sc->ni;
    sc->ni *= 2;
    sc->accept = 0;
  }
  sc->rho = rho;
}

static __global__ void set_solve_ok(DevScalars* sc, int ok) {
  if (threadIdx.x == 0 && blockIdx.x == 0) sc->solve_ok = ok;
}

// partial sums of x (lambda x + b) (computeScale)
// lam_from: first entry the lambda term applies to (0; a sharded bundle
// adjustment's ranks other than 0 leave the replicated camera entries' term
// to rank 0)
static __global__ void lm_scale_partials(const double* x, const double* b, int n, const DevScalars* sc, double* partials,
                                         int lam_from = 0) {
  const double lambda = sc->lambda;
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
    s += x[i] * ((i >= lam_from ? lambda : 0.0) * x[i] + b[i]);
  s = block_sum1(s);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// sum of squares partials (refinement residual norms)
static __global__ void sumsq_partials(const double* a, int n, double* partials) {
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += a[i] * a[i];
  s = block_sum1(s);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// partial sums of a . b
static __global__ void dot_partials(const double* a, const double* b, int n, double* partials) {
  double s = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) s += a[i] * b[i];
  s = block_sum1(s);
  if (threadIdx.x == 0) partials[blockIdx.x] = s;
}

// y = x + a * y
static __global__ void xpay_kernel(double* y, const double* x, double a, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] = x[i] + a * y[i];
}

static __global__ void axpy_kernel(double* y, const double* x, double a, int n) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) y[i] += a * x[i];
}

template <typename Real, int BS>
__global__ void damp_diag(const int* diag, int nb, double lambda, Real* dst) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nb * BS) return;
  const int i = t / BS, d = t % BS;
  Real* v = dst + (size_t)diag[i] * BS * BS + d * (BS + 1);
  *v = (Real)((double)*v + lambda);
}

// ---------------------------------------------------------------- Dogleg
// out = a x + b y (x or y NULL: that term is absent), the vector
// combinations of OptimizationAlgorithmDogleg::solve
// (g2o/core/optimization_algorithm_dogleg.cpp:99-157)
static __global__ void dl_axpby(int n, double a, const double* x, double b, const double* y, double* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  double v = 0.0;
  if (x) v = a * x[i];
  if (y) v = x ? v + b * y[i] : b * y[i];
  out[i] = v;
}

// y = Hpp x for a pose graph: BlockSolver::multiplyHessian
// (g2o/core/block_solver.h:96) = SparseBlockMatrix::multiplySymmetricUpperTriangle
// over the upper blocks, listed by the system's row and column lists, values
// in the column-major pattern order (perm). One thread per block row; the
// row's blocks, then the transposed strictly-upper blocks of its column.
template <typename Real, int BS>
__global__ void hpp_mult_sym(SysDev<Real> A, const Real* hv, const double* x, double* y) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= A.nb) return;
  double acc[BS];
#pragma unroll
  for (int a = 0; a < BS; ++a) acc[a] = 0.0;
  for (int k = A.rptr[r]; k < A.rptr[r + 1]; ++k) {
    const int c = A.rcol[k];
    const Real* B = hv + (size_t)A.perm[k] * BS * BS;
#pragma unroll
    for (int i = 0; i < BS; ++i)
#pragma unroll
      for (int b = 0; b < BS; ++b) acc[i] += (double)B[i * BS + b] * x[(size_t)c * BS + b];
  }
  for (int p = A.cptr[r]; p < A.cptr[r + 1]; ++p) {
    const int k = A.cblk[p];
    const int row = A.brow[k];
    const Real* B = hv + (size_t)A.perm[k] * BS * BS;
#pragma unroll
    for (int i = 0; i < BS; ++i)
#pragma unroll
      for (int b = 0; b < BS; ++b) acc[b] += (double)B[i * BS + b] * x[(size_t)row * BS + i];
  }
#pragma unroll
  for (int a = 0; a < BS; ++a) y[(size_t)r * BS + a] = acc[a];
}

// y = Hpp x for bundle adjustment: Hpp is the cameras' 6x6 diagonal blocks
// (no pose-pose edges); the landmark part of y is zero, as multiplyHessian
// touches only the pose part of the vector
template <typename Real>
__global__ void hpp_mult_diag6(int nb, const Real* hv, const double* x, double* y, int n) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  if (t >= nb * 6) {
    y[t] = 0.0;
    return;
  }
  const int h = t / 6, i = t % 6;
  const Real* B = hv + (size_t)h * 36 + i * 6;
  double acc = 0.0;
#pragma unroll
  for (int b = 0; b < 6; ++b) acc += (double)B[b] * x[(size_t)h * 6 + b];
  y[t] = acc;
}

// y += the pose-pose blocks' part of Hpp x (a pose edge set): per camera row
// h its pair blocks in order, pp_ptr / pp_ent (storage block, other camera,
// transposed: the block is (other, h), read as its transpose)
template <typename Real>
__global__ void hpp_mult_pairs6(int Cf, const int* pp_ptr, const int4* pp_ent, const Real* hv, const double* x,
                                double* y) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= Cf * 6) return;
  const int h = t / 6, i = t % 6;
  double acc = 0.0;
  for (int q = pp_ptr[h]; q < pp_ptr[h + 1]; ++q) {
    const int4 en = pp_ent[q];
    const Real* B = hv + (size_t)en.x * 36;
    const double* xo = x + (size_t)en.y * 6;
#pragma unroll
    for (int b = 0; b < 6; ++b) acc += (double)(en.z ? B[b * 6 + i] : B[i * 6 + b]) * xo[b];
  }
  y[t] += acc;
}

}  // namespace g2oc
