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
// s = sqrt(a_jj), y_r = a_rj / s for its rows and columns and updates its
// elements a_rc -= y_r y_c (c > j, r >= c); the holders of column j keep
// L(r, j) = y_r and L(j, j) = s, then publish column j + 1.
//
// Inverse W = L^-1 (lower), forward substitution by rows, one barrier per
// row k: the holders of row k scale it by 1 / L(k, k) and publish it; every
// thread subtracts L(i, k) W(k, c) from its rows i > k.
//
// Every element is updated by one thread in a fixed order: the results are
// bit-reproducible. A non-positive pivot sets *info and is replaced by 1.
#pragma once

namespace g2oc {

// T: the tile in shared memory, T[i * ld + j] = element (i, j); on entry the
// lower triangle holds A, on return the lower triangle holds L. buf: 2 * N
// doubles of shared memory. W (optional, may be nullptr): W = L^-1 written
// as W[j * ldw + i] = W(i, j) (column-major), zero above the diagonal, in the
// precision of OutT.
template <int N, int TR, int TC, typename OutT>
__device__ __forceinline__ void tile_potrf_inv(double* T, int ld, double* buf, int* info, OutT* W, int ldw) {
  static_assert(N % TR == 0 && N % TC == 0, "the thread grid divides the tile");
  constexpr int RA = N / TR, CB = N / TC;
  const int tr = (int)threadIdx.x % TR, tc = (int)threadIdx.x / TR;
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
    const double s = sqrt(d);
    const double rs = 1.0 / s;
    double yr[RA], yc[CB];
#pragma unroll
    for (int i = 0; i < RA; ++i) yr[i] = cj[tr + TR * i] * rs;
#pragma unroll
    for (int k = 0; k < CB; ++k) yc[k] = cj[tc + TC * k] * rs;
#pragma unroll
    for (int i = 0; i < RA; ++i)
#pragma unroll
      for (int k = 0; k < CB; ++k) {
        const int r = tr + TR * i, c = tc + TC * k;
        if (c > j && r >= c) a[i][k] -= yr[i] * yc[k];
        else if (c == j && r > j) a[i][k] = yr[i];
        else if (c == j && r == j) a[i][k] = s;
      }
    // (register indices stay compile-time constants: a predicated sweep over
    // this thread's columns instead of a computed index)
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
    const double rl = 1.0 / T[0];
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
      if (r > kk) {
        const double l = T[r * ld + kk];
#pragma unroll
        for (int k = 0; k < CB; ++k) a[i][k] -= l * w[k];
      }
    }
    double* nxt = buf + ((kk + 1) & 1) * N;
#pragma unroll
    for (int i = 0; i < RA; ++i)
      if (tr + TR * i == kk + 1) {
        const double rl = 1.0 / T[(kk + 1) * ld + kk + 1];
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
