// pcg_persistent.cuh -- the whole block-Jacobi PCG solve of
// LinearSolverPCG::solve / pcg (g2o/solvers/pcg/linear_solver_pcg.hpp:87-158)
// as one cooperative launch: every CTA stays resident for the solve and the
// phases of an iteration are separated by a grid barrier (bounded waits).
// This is the form for a sparse block matrix; pcg_tiles.cuh has the one for
// a nearly full matrix.
//
// Per iteration (the matrix A is stored as its upper blocks, row-SoA):
//   A  row chunks (<= 32 blocks of one row, one warp, one lane per block,
//      grid-stride over the chunks): chunk partial of q_r = sum_c A(r,c) d_c,
//      transposed contribution T_b = A(r,c)^T d_r of each strictly-upper
//      block, and d.q, summed block by block as d_r.A(r,c) d_c (twice for an
//      off-diagonal block);
//   -- barrier; alpha = dn / d.q (every CTA sums the per-CTA partials in the
//      same order, so all CTAs hold the same value)
//   B  one warp per row c: q_c = its row's chunk partials + its column's T,
//      x_c += alpha d_c, r_c -= alpha q_c, s_c = M_c^-1 r_c, partial r.s;
//   -- barrier; dn = r.s, beta = dn / dn_old, stop test (identical in all CTAs)
//   D  d_c = s_c + beta d_c for the warp's rows;
//   -- barrier.
// Data another CTA wrote during the launch is read with ld.global.cg (L2),
// never through L1. All sums run in a fixed order for a given grid size, so
// results are bit-reproducible on a device.
#pragma once

#include "pcg_kernels.cuh"

namespace g2oc {

constexpr int kPcgThreads = 256;
constexpr int kPcgWarps = kPcgThreads / 32;
// well under a second of polling at a barrier before the solve gives up
// with an error (a phase of a large solve takes milliseconds)
constexpr unsigned int kGridSyncSpinLimit = 1u << 21;

// Grid-wide barrier over the co-resident CTAs of a cooperative launch:
// arrival counter plus generation number. gen (meaningful in thread 0 only)
// is the generation the barrier completes from: read once per launch by
// grid_gen_start (no barrier can complete before every CTA has read it) and
// counted locally after that, so an arrival costs one atomic and no read of
// the shared generation. Returns false (in every thread of the CTA) once any
// CTA's wait has run out; the caller then returns. extra: arrivals expected
// beyond the grid (0; a context created with G2OC_TEST_BARRIER_EXTRA set
// passes 1, so that no barrier completes and every wait runs out: the test
// of the bounded wait and of the status the host reads back).
__device__ __forceinline__ unsigned grid_gen_start(const PcgState* st) {
  return threadIdx.x == 0 ? *reinterpret_cast<const volatile unsigned int*>(&st->sync_gen) : 0u;
}
__device__ __forceinline__ bool grid_barrier(PcgState* st, unsigned& gen, unsigned extra) {
  __shared__ int s_ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    volatile unsigned int* vgen = &st->sync_gen;
    volatile int* verr = &st->sync_error;
    __threadfence();
    if (atomicAdd(&st->sync_count, 1u) == gridDim.x - 1 + extra) {
      atomicExch(&st->sync_count, 0u);
      __threadfence();
      atomicAdd(&st->sync_gen, 1u);
    } else {
      unsigned int spins = 0;
      while (*vgen == gen && *verr == 0) {
        if (++spins > kGridSyncSpinLimit) {
          atomicExch(&st->sync_error, 1);
          break;
        }
        __nanosleep(32);
      }
    }
    __threadfence();
    gen += 1;
    s_ok = (*verr == 0);
  }
  __syncthreads();
  return s_ok != 0;
}

// CTA partial: sum of a per-thread value in a fixed order -> out[blockIdx.x]
template <int WARPS = kPcgWarps>
__device__ __forceinline__ void cta_partial(double v, double* out, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  v = warp_sum(v);
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    double a = 0.0;
#pragma unroll
    for (int w = 0; w < WARPS; ++w) a += red[w];
    out[blockIdx.x] = a;
  }
  __syncthreads();
}

// sum of all CTAs' partials, same order (and so same value) in every CTA
template <int WARPS = kPcgWarps>
__device__ __forceinline__ double cta_sum_all(const double* part, double* red) {
  double a = 0.0;
  for (int j = threadIdx.x; j < (int)gridDim.x; j += blockDim.x) a += __ldcg(part + j);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  a = warp_sum(a);
  __syncthreads();
  if (lane == 0) red[warp] = a;
  __syncthreads();
  double t = 0.0;
#pragma unroll
  for (int w = 0; w < WARPS; ++w) t += red[w];
  __syncthreads();
  return t;
}

template <int BS>
__device__ __forceinline__ double pick(const double (&v)[BS], int a) {
  double out = 0.0;
#pragma unroll
  for (int i = 0; i < BS; ++i)
    if (a == i) out = v[i];
  return out;
}

// r_c, s_c = M^-1 r_c and the lane's share of r.s, lanes a < BS own entry a
template <int BS>
__device__ __forceinline__ double row_precondition(const double* minv, int c, const double (&rc)[BS], int lane,
                                                   double* s) {
  if (lane >= BS) return 0.0;
  const double* M = minv + (size_t)c * BS * BS + (size_t)lane * BS;
  double v = 0.0;
#pragma unroll
  for (int b = 0; b < BS; ++b) v += M[b] * rc[b];
  s[(size_t)c * BS + lane] = v;
  return pick<BS>(rc, lane) * v;
}

// Solve A x = b from x = 0. Configuration in the arguments (nothing is
// written to the state before the launch); state in: d0 (fixed_d0 solves)
// and residual_carry; out: dn, d0, iterations, breakdown, done,
// residual_carry, total_iterations.
template <typename Real, int BS>
__global__ void __launch_bounds__(kPcgThreads, 2)
    pcg_solve_persistent(SysDev<Real> A, const int* chunk_ptr, const int* chunk_row, int nchunks, const double* minv,
                         const double* b, double* x, double* r, double* s, double* d, double* tbuf, double* cpart,
                         double* part_dq, double* part_rs, PcgState* st, double tol, int max_iter, int abs_tol,
                         int fixed_d0, unsigned barrier_extra) {
  __shared__ double red[kPcgWarps];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int gw = blockIdx.x * kPcgWarps + warp, GW = gridDim.x * kPcgWarps;
  const bool fixed = fixed_d0 != 0;
  const double d0_in = st->d0;
  const double carry = st->residual_carry;
  unsigned gen = grid_gen_start(st);

  // r = b, x = 0, s = M^-1 r, d = s, dn = r.s (linear_solver_pcg.hpp:117-137)
  double rs = 0.0;
  for (int c = gw; c < A.nb; c += GW) {
    double rc[BS];
#pragma unroll
    for (int a = 0; a < BS; ++a) rc[a] = b[(size_t)c * BS + a];
    rs += row_precondition<BS>(minv, c, rc, lane, s);
    if (lane < BS) {
      const size_t o = (size_t)c * BS + lane;
      r[o] = pick<BS>(rc, lane);
      x[o] = 0.0;
      d[o] = s[o];
    }
  }
  cta_partial(rs, part_rs, red);
  if (!grid_barrier(st, gen, barrier_extra)) return;
  double dn = cta_sum_all(part_rs, red);
  double d0 = d0_in;
  if (!fixed) {
    d0 = tol * dn;
    if (abs_tol && carry > 0.0 && carry > d0) d0 = carry;
  }
  int k = 0;
  bool breakdown = false;
  bool stop = dn <= d0 || max_iter <= 0;
  while (!stop) {
    // ---- A: row chunks
    double dq = 0.0;
    for (int ch = gw; ch < nchunks; ch += GW) {
      const int row = chunk_row[ch];
      const int rb = A.rptr[row], nblk = A.rptr[row + 1] - rb;
      const int j = (ch - chunk_ptr[row]) * kSysChunk + lane;
      double acc[BS];
#pragma unroll
      for (int a = 0; a < BS; ++a) acc[a] = 0.0;
      if (j < nblk) {
        const int c = A.rcol[rb + j];
        double dr[BS], dc[BS], tj[BS];
#pragma unroll
        for (int a = 0; a < BS; ++a) {
          dr[a] = __ldcg(d + (size_t)row * BS + a);
          dc[a] = __ldcg(d + (size_t)c * BS + a);
          tj[a] = 0.0;
        }
        const Real* base = A.val + (size_t)rb * BS * BS + j;
#pragma unroll
        for (int i = 0; i < BS; ++i)
#pragma unroll
          for (int q = 0; q < BS; ++q) {
            const double m = (double)__ldg(base + (size_t)(i * BS + q) * nblk);
            acc[i] += m * dc[q];
            tj[q] += m * dr[i];
          }
        double v = 0.0;
#pragma unroll
        for (int a = 0; a < BS; ++a) v += dr[a] * acc[a];
        if (c != row) {
          double* t = tbuf + (size_t)A.perm[rb + j] * BS;
#pragma unroll
          for (int q = 0; q < BS; ++q) t[q] = tj[q];
          dq += 2.0 * v;
        } else {
          dq += v;
        }
      }
#pragma unroll
      for (int a = 0; a < BS; ++a) acc[a] = warp_sum(acc[a]);
      if (lane < BS) cpart[(size_t)ch * BS + lane] = pick<BS>(acc, lane);
    }
    cta_partial(dq, part_dq, red);
    if (!grid_barrier(st, gen, barrier_extra)) return;
    const double dqs = cta_sum_all(part_dq, red);
    if (!(dqs > 0.0)) {
      // the (rounded) matrix is not positive definite along d: stop with the
      // current iterate (cannot occur for an SPD FP64 system while dn > d0)
      breakdown = true;
      break;
    }
    const double alpha = dn / dqs;
    // ---- B: rows
    rs = 0.0;
    for (int c = gw; c < A.nb; c += GW) {
      double q[BS];
#pragma unroll
      for (int a = 0; a < BS; ++a) q[a] = 0.0;
      const int p0 = A.cptr[c] + c, p1 = A.cptr[c + 1] + c;
#pragma unroll 4
      for (int p = p0 + lane; p < p1; p += 32) {
        const double* t = tbuf + (size_t)p * BS;
#pragma unroll
        for (int a = 0; a < BS; ++a) q[a] += __ldcg(t + a);
      }
      for (int ch = chunk_ptr[c] + lane; ch < chunk_ptr[c + 1]; ch += 32) {
        const double* t = cpart + (size_t)ch * BS;
#pragma unroll
        for (int a = 0; a < BS; ++a) q[a] += __ldcg(t + a);
      }
      double rc[BS];
#pragma unroll
      for (int a = 0; a < BS; ++a) {
        q[a] = warp_sum(q[a]);
        rc[a] = __ldcg(r + (size_t)c * BS + a) - alpha * q[a];
      }
      __syncwarp();  // every lane has read r_c before its owner lane rewrites it
      rs += row_precondition<BS>(minv, c, rc, lane, s);
      if (lane < BS) {
        const size_t o = (size_t)c * BS + lane;
        x[o] += alpha * __ldcg(d + o);
        r[o] = pick<BS>(rc, lane);
      }
    }
    cta_partial(rs, part_rs, red);
    if (!grid_barrier(st, gen, barrier_extra)) return;
    const double dn_new = cta_sum_all(part_rs, red);
    const double beta = dn_new / dn;
    dn = dn_new;
    ++k;
    if (dn <= d0 || k >= max_iter) break;
    // ---- D: direction
    for (int c = gw; c < A.nb; c += GW)
      if (lane < BS) {
        const size_t o = (size_t)c * BS + lane;
        d[o] = __ldcg(s + o) + beta * __ldcg(d + o);
      }
    if (!grid_barrier(st, gen, barrier_extra)) return;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) {
    st->dn = dn;
    st->d0 = d0;
    st->k = k;
    st->iterations = k;
    st->breakdown = breakdown ? 1 : 0;
    st->done = 1;
    st->total_iterations += k;
    if (!fixed) st->residual_carry = 0.5 * dn;
  }
}

}  // namespace g2oc
