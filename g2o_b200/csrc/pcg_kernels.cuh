// pcg_kernels.cuh -- block-Jacobi preconditioned conjugate gradients on a
// symmetric block matrix stored as upper-triangular blocks in column-major
// order, the device form of LinearSolverPCG::solve / mult / multDiag
// (g2o/solvers/pcg/linear_solver_pcg.hpp:87-205). Real is the matrix and
// Krylov-vector type, BS the block size (3 or 6). The solution x and all
// dot products are FP64.
//
// One iteration is two kernels: pcg_spmv (direction update d = s + beta d
// fused into q = A d, partial d.q) and pcg_update (x, r, s = M^-1 r, partial
// r.s). Scalars live in PcgState on the device; the last block of each kernel
// (atomic ticket, no waiting) sums the partials in index order and advances
// the state, so the host only polls `done`.
#pragma once

#include "g2o_math.cuh"
#include "reduce.cuh"

namespace g2oc {

template <typename Real>
struct SysDev {
  int nb;
  const int* col_ptr;   // nb + 1, column-major ranges, diagonal last
  const int* row;       // per block
  const int* diag;      // per row: block of the diagonal
  const int* rowu_ptr;  // nb + 1, strictly-upper blocks listed by row
  const int* rowu_blk;
  const int* rowu_col;
  const Real* val;      // BS*BS row-major per block
};

struct PcgState {
  double dn;              // r^T M^-1 r of the current iterate
  double d0;              // stopping threshold
  double alpha;
  double beta;
  double residual_carry;  // LinearSolverPCG::_residual (0.5 * final dn of the previous solve)
  double tolerance;
  unsigned int counter;   // last-block ticket
  int k;                  // completed iterations
  int done;
  int iterations;
  int max_iter;
  int absolute_tolerance;
  int relative_only;      // refinement solves: ignore the carried residual
  int pad;
};

// M^-1: inverse of each diagonal block (computed in FP64)
template <typename Real, int BS>
__global__ void pcg_diag_inv(SysDev<Real> A, Real* minv, int* nonfinite) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.nb) return;
  const Real* D = A.val + (size_t)A.diag[i] * BS * BS;
  double M[BS * BS], I[BS * BS];
#pragma unroll
  for (int k = 0; k < BS * BS; ++k) M[k] = (double)D[k];
  bool ok;
  if (BS == 3) ok = inverse3(M, I);
  else ok = inverse_gj<double, BS>(M, I);
  if (!ok) *nonfinite = 1;
#pragma unroll
  for (int k = 0; k < BS * BS; ++k) minv[(size_t)i * BS * BS + k] = (Real)I[k];
}

__device__ __forceinline__ bool last_block_ticket(unsigned int* counter) {
  __shared__ bool last;
  __syncthreads();
  if (threadIdx.x == 0) {
    __threadfence();
    const unsigned int t = atomicAdd(counter, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  return last;
}

__device__ __forceinline__ double sum_partials(const double* p, int n) {
  double a = 0.0;
  for (int j = threadIdx.x; j < n; j += blockDim.x) a += __ldcg(p + j);
  return block_sum1(a);
}

// r = b, x = 0, s = M^-1 r, dn = r.s, d0 = tol * dn (raised to the carried
// residual when absolute tolerance is on), linear_solver_pcg.hpp:117-137
template <typename Real, int BS>
__global__ void pcg_init(int nb, const double* b, const Real* minv, Real* r, Real* s, double* x, double* partials,
                         PcgState* st) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double dot = 0.0;
  if (i < nb) {
    Real rb[BS];
#pragma unroll
    for (int k = 0; k < BS; ++k) {
      rb[k] = (Real)b[(size_t)i * BS + k];
      r[(size_t)i * BS + k] = rb[k];
      x[(size_t)i * BS + k] = 0.0;
    }
    const Real* M = minv + (size_t)i * BS * BS;
#pragma unroll
    for (int a = 0; a < BS; ++a) {
      Real v = Real(0);
#pragma unroll
      for (int c = 0; c < BS; ++c) v += M[a * BS + c] * rb[c];
      s[(size_t)i * BS + a] = v;
      dot += (double)rb[a] * (double)v;
    }
  }
  dot = block_sum1(dot);
  if (threadIdx.x == 0) partials[blockIdx.x] = dot;
  if (last_block_ticket(&st->counter)) {
    const double dn = sum_partials(partials, gridDim.x);
    if (threadIdx.x == 0) {
      st->counter = 0;
      double d0 = st->tolerance * dn;
      if (st->absolute_tolerance && !st->relative_only) {
        if (st->residual_carry > 0.0 && st->residual_carry > d0) d0 = st->residual_carry;
      }
      st->d0 = d0;
      st->dn = dn;
      st->beta = 0.0;
      st->k = 0;
      st->done = (dn <= d0 || st->max_iter <= 0) ? 1 : 0;
      if (st->done) {
        st->iterations = 0;
        if (!st->relative_only) st->residual_carry = 0.5 * dn;
      }
    }
  }
}

// d_k = s + beta d_{k-1} (ping-pong by parity of k), q = A d_k (both the
// upper blocks and their transposes, as LinearSolverPCG::mult), partial d.q.
// One warp per block row.
template <typename Real, int BS, int THREADS>
__global__ void __launch_bounds__(THREADS) pcg_spmv(SysDev<Real> A, const Real* s, Real* d0buf, Real* d1buf, Real* q,
                                                    double* partials, PcgState* st) {
  if (st->done) return;
  const int k = st->k;
  const double beta = st->beta;
  Real* dcur = (k & 1) ? d1buf : d0buf;
  const Real* dprev = (k & 1) ? d0buf : d1buf;
  const Real rb = (Real)beta;
  const bool use_prev = beta != 0.0;
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * (THREADS / 32) + (threadIdx.x >> 5);
  double dot = 0.0;
  if (i < A.nb) {
    Real acc[BS];
#pragma unroll
    for (int a = 0; a < BS; ++a) acc[a] = Real(0);
    auto dval = [&](int j, Real* out) {
#pragma unroll
      for (int c = 0; c < BS; ++c) {
        Real v = s[(size_t)j * BS + c];
        if (use_prev) v += rb * dprev[(size_t)j * BS + c];
        out[c] = v;
      }
    };
    // column i: blocks (rj, i) with rj <= i contribute A(rj,i)^T d_rj
    const int c1 = A.col_ptr[i + 1];
    for (int p = A.col_ptr[i] + lane; p < c1; p += 32) {
      const int rj = A.row[p];
      Real dj[BS];
      dval(rj, dj);
      const Real* M = A.val + (size_t)p * BS * BS;
#pragma unroll
      for (int r = 0; r < BS; ++r)
#pragma unroll
        for (int c = 0; c < BS; ++c) acc[c] += M[r * BS + c] * dj[r];
    }
    // row i: strictly-upper blocks (i, cj) contribute A(i,cj) d_cj
    const int r1 = A.rowu_ptr[i + 1];
    for (int p = A.rowu_ptr[i] + lane; p < r1; p += 32) {
      const int cj = A.rowu_col[p];
      Real dj[BS];
      dval(cj, dj);
      const Real* M = A.val + (size_t)A.rowu_blk[p] * BS * BS;
#pragma unroll
      for (int r = 0; r < BS; ++r)
#pragma unroll
        for (int c = 0; c < BS; ++c) acc[r] += M[r * BS + c] * dj[c];
    }
#pragma unroll
    for (int a = 0; a < BS; ++a) acc[a] = warp_sum(acc[a]);
    Real di[BS];
    dval(i, di);
    if (lane < BS) {
      Real qa = acc[0], da = di[0];
#pragma unroll
      for (int a = 1; a < BS; ++a)
        if (lane == a) {
          qa = acc[a];
          da = di[a];
        }
      q[(size_t)i * BS + lane] = qa;
      dcur[(size_t)i * BS + lane] = da;
      dot = (double)da * (double)qa;
    }
  }
  dot = block_sum1(dot);
  if (threadIdx.x == 0) partials[blockIdx.x] = dot;
  if (last_block_ticket(&st->counter)) {
    const double dq = sum_partials(partials, gridDim.x);
    if (threadIdx.x == 0) {
      st->counter = 0;
      st->alpha = st->dn / dq;
    }
  }
}

// x += alpha d, r -= alpha q, s = M^-1 r, dn = r.s, beta = dn / dn_old;
// stop when dn <= d0 or after max_iter iterations (linear_solver_pcg.hpp:139-158)
template <typename Real, int BS>
__global__ void pcg_update(int nb, const Real* minv, const Real* d0buf, const Real* d1buf, const Real* q, Real* r,
                           Real* s, double* x, double* partials, PcgState* st) {
  if (st->done) return;
  const int k = st->k;
  const double alpha = st->alpha;
  const Real* d = (k & 1) ? d1buf : d0buf;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double dot = 0.0;
  if (i < nb) {
    Real rb[BS];
    const Real ra = (Real)alpha;
#pragma unroll
    for (int c = 0; c < BS; ++c) {
      const size_t o = (size_t)i * BS + c;
      x[o] += alpha * (double)d[o];
      rb[c] = r[o] - ra * q[o];
      r[o] = rb[c];
    }
    const Real* M = minv + (size_t)i * BS * BS;
#pragma unroll
    for (int a = 0; a < BS; ++a) {
      Real v = Real(0);
#pragma unroll
      for (int c = 0; c < BS; ++c) v += M[a * BS + c] * rb[c];
      s[(size_t)i * BS + a] = v;
      dot += (double)rb[a] * (double)v;
    }
  }
  dot = block_sum1(dot);
  if (threadIdx.x == 0) partials[blockIdx.x] = dot;
  if (last_block_ticket(&st->counter)) {
    const double dn = sum_partials(partials, gridDim.x);
    if (threadIdx.x == 0) {
      st->counter = 0;
      st->beta = dn / st->dn;
      st->dn = dn;
      st->k = k + 1;
      if (dn <= st->d0 || k + 1 >= st->max_iter) {
        st->done = 1;
        st->iterations = k + 1;
        if (!st->relative_only) st->residual_carry = 0.5 * dn;
      }
    }
  }
}

}  // namespace g2oc
