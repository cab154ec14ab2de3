// tile_potrf.cuh -- Cholesky factorization and inverse of one dense N x N
// diagonal tile in FP64, by one CTA, for the tiled Cholesky solvers
// (cholesky.cuh: 64 x 64 tiles; tc_chol.cuh: 128 x 128 tiles).
//
// The CTA is a TR x TC grid of threads; thread (tr, tc) holds the elements
// (tr + TR * a, tc + TC * b) of the tile in registers (an interleaved
// sub-block, so every thread has work until the last columns).
//
// Factorization, right-looking, one barrier per column j: the column's
// values (final after step j - 1) are published in a double-buffered
// shared vector by the threads that hold them; every thread forms
// rs = rsqrt(a_jj), y_r = a_rj rs for its rows and columns and updates its
// elements a_rc -= y_r y_c (c > j); the holders of column j keep
// L(r, j) = y_r and L(j, j) = a_jj rs, then publish column j + 1. The pivot
// chain of a column is one reciprocal square root (no square root and
// division in sequence), and the update is branch-free: y_c is zero for the
// finished columns c <= j and y_r for the rows r <= j, so an element above
// the diagonal takes only the mirror of its transpose's trailing update (it
// is never read as part of L).
//
// Inverse W = L^-1 (lower), forward substitution by rows, one barrier per
// row k: the holders of row k scale it by the kept reciprocal 1 / L(k, k)
// and publish it; every thread subtracts L(i, k) W(k, c) from its rows i > k.
//
// Every element is updated by one thread in a fixed order: the results are
// bit-reproducible. A non-positive pivot sets *info and is replaced by 1.
#pragma once

namespace g2oc {

// T: the tile in shared memory, T[i * ld + j] = element (i, j); on entry the
// lower triangle holds A, on return the lower triangle holds L. buf: 3 * N
// doubles of shared memory (two column vectors and the pivots' reciprocals).
// W (optional, may be nullptr): W = L^-1 written as W[j * ldw + i] = W(i, j)
// (column-major), zero above the diagonal, in the precision of OutT.
// blockDim.x must be TR * TC. Ends with a barrier: on return T and a
// shared-memory W are complete for the whole CTA.
template <int N, int TR, int TC, typename OutT>
__device__ __forceinline__ void tile_potrf_inv(double* T, int ld, double* buf, int* info, OutT* W, int ldw) {
  static_assert(N % TR == 0 && N % TC == 0, "the thread grid divides the tile");
  constexpr int RA = N / TR, CB = N / TC;
  const int tr = (int)threadIdx.x % TR, tc = (int)threadIdx.x / TR;
  double* rdiag = buf + 2 * N;
  double a[RA][CB];
#pragma unroll
  for (int i = 0; i < RA; ++i)
#pragma unroll
    for (int k = 0; k < CB; ++k) {
      const int r = tr + TR * i, c = tc + TC * k;
      a[i][k] = r >= c ? T[r * ld + c] : 0.0;
    }
  // publish column 0
  if (tc == 0) {
#pragma unroll
    for (int i = 0; i < RA; ++i) buf[tr + TR * i] = a[i][0];
  }
  __syncthreads();
  for (int j = 0; j < N; ++j) {
    const double* cj = buf + (j & 1) * N;
    double d = cj[j];
    if (!(d > 0.0)) {
      if (threadIdx.x == 0) *info = 1;
      d = 1.0;
    }
    const double rs = rsqrt(d);
    double yr[RA], yc[CB];
#pragma unroll
    for (int i = 0; i < RA; ++i) yr[i] = tr + TR * i > j ? cj[tr + TR * i] * rs : 0.0;
#pragma unroll
    for (int k = 0; k < CB; ++k) yc[k] = tc + TC * k > j ? cj[tc + TC * k] * rs : 0.0;
#pragma unroll
    for (int i = 0; i < RA; ++i)
#pragma unroll
      for (int k = 0; k < CB; ++k) a[i][k] -= yr[i] * yc[k];
    // column j itself (register indices stay compile-time constants: a
    // predicated sweep over this thread's columns instead of a computed index)
#pragma unroll
    for (int k = 0; k < CB; ++k)
      if (tc + TC * k == j) {
#pragma unroll
        for (int i = 0; i < RA; ++i) {
          const int r = tr + TR * i;
          if (r > j) a[i][k] = yr[i];
          else if (r == j) a[i][k] = d * rs;
        }
      }
    if (threadIdx.x == 0) rdiag[j] = rs;
    double* nxt = buf + ((j + 1) & 1) * N;
#pragma unroll
    for (int k = 0; k < CB; ++k)
      if (tc + TC * k == j + 1) {
#pragma unroll
        for (int i = 0; i < RA; ++i) nxt[tr + TR * i] = a[i][k];
      }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < RA; ++i)
#pragma unroll
    for (int k = 0; k < CB; ++k) {
      const int r = tr + TR * i, c = tc + TC * k;
      if (r >= c) T[r * ld + c] = a[i][k];
    }
  __syncthreads();  // L complete in T
  if (!W) return;
  // W = L^-1: a holds rows of W, starting from the identity
#pragma unroll
  for (int i = 0; i < RA; ++i)
#pragma unroll
    for (int k = 0; k < CB; ++k) a[i][k] = (tr + TR * i == tc + TC * k) ? 1.0 : 0.0;
  // row 0 final: W(0, c) = e_0 / L(0, 0)
  if (tr == 0) {
    const double rl = rdiag[0];
#pragma unroll
    for (int k = 0; k < CB; ++k) {
      a[0][k] *= rl;
      buf[tc + TC * k] = a[0][k];
    }
  }
  __syncthreads();
  for (int kk = 0; kk < N; ++kk) {
    const double* wk = buf + (kk & 1) * N;
    double w[CB];
#pragma unroll
    for (int k = 0; k < CB; ++k) w[k] = wk[tc + TC * k];
#pragma unroll
    for (int i = 0; i < RA; ++i) {
      const int r = tr + TR * i;
      const double l = r > kk ? T[r * ld + kk] : 0.0;
#pragma unroll
      for (int k = 0; k < CB; ++k) a[i][k] -= l * w[k];
    }
    double* nxt = buf + ((kk + 1) & 1) * N;
#pragma unroll
    for (int i = 0; i < RA; ++i)
      if (tr + TR * i == kk + 1) {
        const double rl = rdiag[kk + 1];
#pragma unroll
        for (int k = 0; k < CB; ++k) {
          a[i][k] *= rl;
          nxt[tc + TC * k] = a[i][k];
        }
      }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < RA; ++i)
#pragma unroll
    for (int k = 0; k < CB; ++k) {
      const int r = tr + TR * i, c = tc + TC * k;
      W[(size_t)c * ldw + r] = (OutT)(r >= c ? a[i][k] : 0.0);
    }
  __syncthreads();
}

}  // namespace g2oc
