// pcg_kernels.cuh -- block-Jacobi preconditioned conjugate gradients on a
// symmetric block matrix, the device form of LinearSolverPCG::solve / mult /
// multDiag (g2o/solvers/pcg/linear_solver_pcg.hpp:87-205). Real is the
// storage type of the matrix blocks (double, or float on the mixed path,
// where the matrix is the dominant traffic), BS the block size (3 or 6). The
// Krylov vectors, the preconditioner, the solution and all dot products are
// FP64.
//
// Storage: only the upper blocks, row by row (each row's blocks contiguous,
// diagonal first), so the product reads the matrix once: the row pass forms
// sum_c A(r,c) d_c for its row and writes the transposed contributions
// A(r,c)^T d_r per block; the column pass sums those per column in row order.
// One PCG iteration is three kernels: row pass (with the direction update
// d = s + beta d fused in), column pass (q, partial d.q, alpha), update (x, r,
// s = M^-1 r, partial r.s, beta, stop test). Scalars live in PcgState on the
// device; the last block of a kernel (atomic ticket, no waiting) sums the
// partials in index order and advances the state, so the host only polls
// `done`. All sums are in a fixed order: results are bit-reproducible.
#pragma once

#include "g2o_math.cuh"
#include "reduce.cuh"

namespace g2oc {

template <typename Real>
struct SysDev {
  int nb;
  int nnzb;
  const int* rptr;   // nb + 1: blocks of row r (upper, diagonal first)
  const int* rcol;   // per block: column
  const int* brow;   // per block: row
  const int* diag;   // per row: block of the diagonal
  const int* cptr;   // nb + 1: strictly-upper blocks of column c
  const int* cblk;   //         (block indices, rows ascending)
  const int* perm;   // per block: index in the column-major pattern (diagonal
                     // last in each column), where the transposed
                     // contribution of the block is stored
  const Real* val;   // block values, row-SoA layout (sys_offset)
};

// Storage of the block values: the blocks of row r occupy the contiguous
// range [rptr[r] * BS*BS, rptr[r+1] * BS*BS); inside it entry e (row-major
// within the block) of the row's j-th block sits at e * nblk_r + j, so the
// same entry of consecutive blocks is contiguous (coalesced when one lane
// handles one block).
template <int BS>
__host__ __device__ __forceinline__ size_t sys_offset(int rbase, int nblk, int j, int e) {
  return (size_t)rbase * BS * BS + (size_t)e * nblk + j;
}

struct PcgState {
  double dn;              // r^T M^-1 r of the current iterate
  double d0;              // stopping threshold
  double alpha;
  double beta;
  double residual_carry;  // LinearSolverPCG::_residual (0.5 * final dn of the previous solve)
  double tolerance;
  double check_dn;        // M-norm of a given residual (refinement check)
  unsigned int counter;   // last-block ticket
  int k;                  // completed iterations
  int done;
  int iterations;
  int max_iter;
  int absolute_tolerance;
  int fixed_d0;           // correction solves: keep d0 of the first solve, leave the carry
  int breakdown;          // d.q <= 0 met (the matrix is not positive definite along d)
  // grid barrier of the persistent solve (the count returns to zero after
  // every barrier; any generation value works)
  unsigned int sync_count;
  unsigned int sync_gen;
  int sync_error;         // a barrier wait ran out of its spin limit
  int pad;
  long long total_iterations;  // iterations of all solves since the state was reset
};

// Gauss-Jordan inverse with partial pivoting of an N x N matrix held one row
// per lane by N consecutive lanes (g0: the group's first lane, i: this lane's
// row): the operations of inverse_gj in the same order, with the rows in
// registers and the pivot row and swaps by shuffles instead of serial loops
// over a local array. Every lane of the warp takes part in the shuffles.
template <int N>
__device__ __forceinline__ bool inverse_gj_lanes(double (&m)[N], double (&inv)[N], int i, int g0) {
  constexpr unsigned FULL = 0xffffffffu;
#pragma unroll
  for (int k = 0; k < N; ++k) inv[k] = (k == i) ? 1.0 : 0.0;
  bool ok = true;
#pragma unroll
  for (int c = 0; c < N; ++c) {
    // pivot: the first row r >= c with the largest |m(r, c)|
    int p = c;
    double best = fabs(__shfl_sync(FULL, m[c], g0 + c));
#pragma unroll
    for (int r = c + 1; r < N; ++r) {
      const double v = fabs(__shfl_sync(FULL, m[c], g0 + r));
      if (v > best) {
        best = v;
        p = r;
      }
    }
    if (best == 0.0) ok = false;
#pragma unroll
    for (int k = 0; k < N; ++k) {  // swap rows p and c
      const double mp = __shfl_sync(FULL, m[k], g0 + p), mc = __shfl_sync(FULL, m[k], g0 + c);
      const double ip = __shfl_sync(FULL, inv[k], g0 + p), ic = __shfl_sync(FULL, inv[k], g0 + c);
      if (i == c) {
        m[k] = mp;
        inv[k] = ip;
      } else if (i == p) {
        m[k] = mc;
        inv[k] = ic;
      }
    }
    const double iv = 1.0 / __shfl_sync(FULL, m[c], g0 + c);
    if (i == c) {
#pragma unroll
      for (int k = 0; k < N; ++k) {
        m[k] *= iv;
        inv[k] *= iv;
      }
    }
    const double f = m[c];
#pragma unroll
    for (int k = 0; k < N; ++k) {
      const double mck = __shfl_sync(FULL, m[k], g0 + c), ick = __shfl_sync(FULL, inv[k], g0 + c);
      if (i != c) {
        m[k] -= f * mck;
        inv[k] -= f * ick;
      }
    }
  }
  return ok;
}

// M^-1 of BS x BS diagonal blocks, 32 / BS blocks per warp (BS lanes each,
// one row per lane; the lanes past the last group idle): the inverses of
// pcg_diag_inv<Real, BS> without its per-thread local arrays. Launch with
// ceil(nb / (32 / BS)) warps or more.
template <typename Real, int BS>
__global__ void pcg_diag_inv_lanes(SysDev<Real> A, double* minv, int* nonfinite) {
  constexpr int G = 32 / BS;
  const int lane = threadIdx.x & 31;
  const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int grp = lane / BS, i = lane - BS * grp;
  const int blk = gw * G + grp;
  const bool act = grp < G && blk < A.nb;
  double m[BS], inv[BS];
  if (act) {
    const int rb = A.rptr[blk], nblk = A.rptr[blk + 1] - rb, j = A.diag[blk] - rb;
#pragma unroll
    for (int c = 0; c < BS; ++c) m[c] = (double)A.val[sys_offset<BS>(rb, nblk, j, i * BS + c)];
  } else {
#pragma unroll
    for (int c = 0; c < BS; ++c) m[c] = (c == i) ? 1.0 : 0.0;
  }
  const bool ok = inverse_gj_lanes<BS>(m, inv, i, lane - i);
  if (act) {
    if (!ok && i == 0) *nonfinite = 1;
#pragma unroll
    for (int c = 0; c < BS; ++c) minv[(size_t)blk * BS * BS + i * BS + c] = inv[c];
  }
}

// M^-1 of 6x6 diagonal blocks, five blocks per warp (six lanes each, one
// row per lane; lanes 30 and 31 idle): the inverses of pcg_diag_inv<Real, 6>
// without its per-thread local arrays. Launch with nb * 32 / 5 threads or more.
template <typename Real>
__global__ void pcg_diag_inv6_lanes(SysDev<Real> A, double* minv, int* nonfinite) {
  const int lane = threadIdx.x & 31;
  const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int grp = lane / 6, i = lane - 6 * grp;
  const int blk = gw * 5 + grp;
  const bool act = grp < 5 && blk < A.nb;
  double m[6], inv[6];
  if (act) {
    const int rb = A.rptr[blk], nblk = A.rptr[blk + 1] - rb, j = A.diag[blk] - rb;
#pragma unroll
    for (int c = 0; c < 6; ++c) m[c] = (double)A.val[sys_offset<6>(rb, nblk, j, i * 6 + c)];
  } else {
#pragma unroll
    for (int c = 0; c < 6; ++c) m[c] = (c == i) ? 1.0 : 0.0;
  }
  const bool ok = inverse_gj_lanes<6>(m, inv, i, lane - i);
  if (act) {
    if (!ok && i == 0) *nonfinite = 1;
#pragma unroll
    for (int c = 0; c < 6; ++c) minv[(size_t)blk * 36 + i * 6 + c] = inv[c];
  }
}

// M^-1: inverse of each diagonal block (computed in FP64)
template <typename Real, int BS>
__global__ void pcg_diag_inv(SysDev<Real> A, double* minv, int* nonfinite) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= A.nb) return;
  const int rb = A.rptr[i], nblk = A.rptr[i + 1] - rb, j = A.diag[i] - rb;
  double M[BS * BS], I[BS * BS];
#pragma unroll
  for (int k = 0; k < BS * BS; ++k) M[k] = (double)A.val[sys_offset<BS>(rb, nblk, j, k)];
  bool ok;
  if (BS == 3) ok = inverse3(M, I);
  else ok = inverse_gj<double, BS>(M, I);
  if (!ok) *nonfinite = 1;
#pragma unroll
  for (int k = 0; k < BS * BS; ++k) minv[(size_t)i * BS * BS + k] = I[k];
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
template <int BS>
__global__ void pcg_init(int nb, const double* b, const double* minv, double* r, double* s, double* x,
                         double* partials, PcgState* st) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double dot = 0.0;
  if (i < nb) {
    double rb[BS];
#pragma unroll
    for (int k = 0; k < BS; ++k) {
      rb[k] = b[(size_t)i * BS + k];
      r[(size_t)i * BS + k] = rb[k];
      x[(size_t)i * BS + k] = 0.0;
    }
    const double* M = minv + (size_t)i * BS * BS;
#pragma unroll
    for (int a = 0; a < BS; ++a) {
      double v = 0.0;
#pragma unroll
      for (int c = 0; c < BS; ++c) v += M[a * BS + c] * rb[c];
      s[(size_t)i * BS + a] = v;
      dot += rb[a] * v;
    }
  }
  dot = block_sum1(dot);
  if (threadIdx.x == 0) partials[blockIdx.x] = dot;
  if (last_block_ticket(&st->counter)) {
    const double dn = sum_partials(partials, gridDim.x);
    if (threadIdx.x == 0) {
      st->counter = 0;
      double d0 = st->d0;
      if (!st->fixed_d0) {
        d0 = st->tolerance * dn;
        if (st->absolute_tolerance) {
          if (st->residual_carry > 0.0 && st->residual_carry > d0) d0 = st->residual_carry;
        }
      }
      st->d0 = d0;
      st->dn = dn;
      st->beta = 0.0;
      st->k = 0;
      st->breakdown = 0;
      st->done = (dn <= d0 || st->max_iter <= 0) ? 1 : 0;
      if (st->done) {
        st->iterations = 0;
        if (!st->fixed_d0) st->residual_carry = 0.5 * dn;
      }
    }
  }
}

// Row pass: d_k = s + beta d_{k-1} (ping-pong by parity of k), for row r
// qrow_r = sum_c A(r,c) d_c, and per strictly-upper block T_b = A(r,c)^T d_r.
// One CTA per block row; thread t takes blocks t, t + THREADS, ... of the row
// (with the row-SoA layout each entry load is coalesced across the warp),
// then a fixed-order CTA reduction.
template <typename Real, int BS, int THREADS>
__global__ void __launch_bounds__(THREADS) pcg_rowpass(SysDev<Real> A, const double* s, double* d0buf,
                                                       double* d1buf, double* qrow, double* tbuf,
                                                       const PcgState* st) {
  if (st->done) return;
  __shared__ double red[THREADS / 32][BS];
  const int k = st->k;
  const double beta = st->beta;
  double* dcur = (k & 1) ? d1buf : d0buf;
  const double* dprev = (k & 1) ? d0buf : d1buf;
  const bool use_prev = beta != 0.0;
  const int r = blockIdx.x;
  auto dval = [&](int j, double* out) {
#pragma unroll
    for (int c = 0; c < BS; ++c) {
      double v = s[(size_t)j * BS + c];
      if (use_prev) v += beta * dprev[(size_t)j * BS + c];
      out[c] = v;
    }
  };
  double dr[BS];
  dval(r, dr);
  double acc[BS];
#pragma unroll
  for (int a = 0; a < BS; ++a) acc[a] = 0.0;
  const int rb = A.rptr[r], nblk = A.rptr[r + 1] - rb;
  const Real* base = A.val + (size_t)rb * BS * BS;
  for (int j = threadIdx.x; j < nblk; j += THREADS) {
    const int c = A.rcol[rb + j];
    double dc[BS];
    dval(c, dc);
    double tj[BS];
#pragma unroll
    for (int b = 0; b < BS; ++b) tj[b] = 0.0;
#pragma unroll
    for (int i = 0; i < BS; ++i)
#pragma unroll
      for (int b = 0; b < BS; ++b) {
        const double m = (double)base[(size_t)(i * BS + b) * nblk + j];
        acc[i] += m * dc[b];
        tj[b] += m * dr[i];
      }
    if (c != r) {
      double* t = tbuf + (size_t)A.perm[rb + j] * BS;
#pragma unroll
      for (int b = 0; b < BS; ++b) t[b] = tj[b];
    }
  }
  block_sum_array<double, BS, THREADS>(acc, &red[0][0]);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int a = 0; a < BS; ++a) {
      qrow[(size_t)r * BS + a] = acc[a];
      dcur[(size_t)r * BS + a] = dr[a];
    }
  }
}

// Column pass: q_c = qrow_c + sum over strictly-upper blocks (r, c) of T_b,
// rows in a fixed thread assignment; partial d.q; the last block sets
// alpha = dn / d.q. One CTA per column.
template <typename Real, int BS, int THREADS>
__global__ void __launch_bounds__(THREADS) pcg_colpass(SysDev<Real> A, const double* d0buf, const double* d1buf,
                                                       const double* qrow, const double* tbuf, double* q,
                                                       double* partials, PcgState* st) {
  if (st->done) return;
  __shared__ double red[THREADS / 32][BS];
  const int k = st->k;
  const double* dcur = (k & 1) ? d1buf : d0buf;
  const int c = blockIdx.x;
  double acc[BS];
#pragma unroll
  for (int a = 0; a < BS; ++a) acc[a] = 0.0;
  // column c's strictly-upper blocks sit contiguously at column-major
  // positions [cptr[c] + c, cptr[c + 1] + c) (one diagonal per earlier column)
  const int p0 = A.cptr[c] + c, p1 = A.cptr[c + 1] + c;
  for (int p = p0 + threadIdx.x; p < p1; p += THREADS) {
    const double* t = tbuf + (size_t)p * BS;
#pragma unroll
    for (int a = 0; a < BS; ++a) acc[a] += t[a];
  }
  block_sum_array<double, BS, THREADS>(acc, &red[0][0]);
  double dot = 0.0;
  if (threadIdx.x == 0) {
#pragma unroll
    for (int a = 0; a < BS; ++a) {
      const double qa = acc[a] + qrow[(size_t)c * BS + a];
      q[(size_t)c * BS + a] = qa;
      dot += dcur[(size_t)c * BS + a] * qa;
    }
    partials[blockIdx.x] = dot;
  }
  if (last_block_ticket(&st->counter)) {
    const double dq = sum_partials(partials, gridDim.x);
    if (threadIdx.x == 0) {
      st->counter = 0;
      st->alpha = st->dn / dq;
      if (!(dq > 0.0)) st->breakdown = 1;
    }
  }
}

// x += alpha d, r -= alpha q, s = M^-1 r, dn = r.s, beta = dn / dn_old;
// stop when dn <= d0 or after max_iter iterations (linear_solver_pcg.hpp:139-158)
template <int BS>
__global__ void pcg_update(int nb, const double* minv, const double* d0buf, const double* d1buf, const double* q,
                           double* r, double* s, double* x, double* partials, PcgState* st) {
  if (st->done) return;
  const int k = st->k;
  if (st->breakdown) {
    // d.q <= 0: the (rounded) matrix is not positive definite along d; stop
    // with the current iterate instead of stepping along a non-descent
    // direction (cannot occur for an SPD FP64 system, where d.q > 0 whenever
    // dn > d0)
    if (blockIdx.x == 0 && threadIdx.x == 0) {
      st->done = 1;
      st->iterations = k;
      if (!st->fixed_d0) st->residual_carry = 0.5 * st->dn;
    }
    return;
  }
  const double alpha = st->alpha;
  const double* d = (k & 1) ? d1buf : d0buf;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double dot = 0.0;
  if (i < nb) {
    double rb[BS];
#pragma unroll
    for (int c = 0; c < BS; ++c) {
      const size_t o = (size_t)i * BS + c;
      x[o] += alpha * d[o];
      rb[c] = r[o] - alpha * q[o];
      r[o] = rb[c];
    }
    const double* M = minv + (size_t)i * BS * BS;
#pragma unroll
    for (int a = 0; a < BS; ++a) {
      double v = 0.0;
#pragma unroll
      for (int c = 0; c < BS; ++c) v += M[a * BS + c] * rb[c];
      s[(size_t)i * BS + a] = v;
      dot += rb[a] * v;
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
        if (!st->fixed_d0) st->residual_carry = 0.5 * dn;
      }
    }
  }
}

// iterations of a solve driven from the host, added to the running total
static __global__ void pcg_add_total(PcgState* st) {
  if (threadIdx.x == 0 && blockIdx.x == 0) st->total_iterations += st->iterations;
}

// M-norm r^T M^-1 r of a residual in FP64 -> st->check_dn (refinement check)
template <int BS>
__global__ void pcg_check_dn(int nb, const double* minv, const double* r, double* partials, PcgState* st) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  double dot = 0.0;
  if (i < nb) {
    const double* M = minv + (size_t)i * BS * BS;
    const double* rb = r + (size_t)i * BS;
#pragma unroll
    for (int a = 0; a < BS; ++a) {
      double v = 0.0;
#pragma unroll
      for (int c = 0; c < BS; ++c) v += M[a * BS + c] * rb[c];
      dot += rb[a] * v;
    }
  }
  dot = block_sum1(dot);
  if (threadIdx.x == 0) partials[blockIdx.x] = dot;
  if (last_block_ticket(&st->counter)) {
    const double dn = sum_partials(partials, gridDim.x);
    if (threadIdx.x == 0) {
      st->counter = 0;
      st->check_dn = dn;
    }
  }
}

// internal (row-SoA) system from a column-major pattern matrix (blocks
// row-major inside), with lambda added to the diagonal
template <typename Real, int BS>
__global__ void sys_gather_damped(const Real* src, const int* perm, const int* brow, const int* rptr, const int* rcol,
                                  int nnzb, double lambda, Real* dst) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nnzb * BS * BS) return;
  const int k = (int)(t / (BS * BS)), e = (int)(t % (BS * BS));
  double v = (double)src[(size_t)perm[k] * BS * BS + e];
  const int r = brow[k];
  if (r == rcol[k] && e / BS == e % BS) v += lambda;
  const int rb = rptr[r];
  dst[sys_offset<BS>(rb, rptr[r + 1] - rb, k - rb, e)] = (Real)v;
}

}  // namespace g2oc
