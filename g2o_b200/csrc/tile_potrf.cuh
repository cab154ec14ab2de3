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

namespace g2oc {

// Blocked form for a 64 x 64 tile and 256 threads, the same results to
// rounding (every reduction in a fixed order), with 4 x 4 + 9 barriers
// instead of one per column and row. T (shared memory, leading dimension
// ld): lower triangle A in, L out; Wsm (shared memory, FP64, column-major
// with leading dimension ldw): W = L^-1 out, zero above the diagonal. Per
// block column of 16 (offset o):
//   1. warp 0 factors the 16 x 16 diagonal block in registers (lane r holds
//      row r; the pivot and the column values pass by shuffles, pivots by
//      rsqrt) and inverts it (W_oo, rows by forward substitution);
//   2. the panel below: L(p, o + c) = sum_{t <= c} A(p, o + t) W_oo(c, t),
//      four threads per row, four columns each;
//   3. the trailing lower triangle takes A(p, q) -= sum_t L(p, o + t)
//      L(q, o + t) in 4 x 4 patches, one per thread.
// Then W's blocks below the diagonal by block rows i = 1..3:
//   W_ij = -W_ii sum_{k=j}^{i-1} L_ik W_kj, the sums staged in W's (zero)
//   upper blocks and cleared afterwards.
// A non-positive pivot sets *info and is replaced by 1. blockDim.x must be
// 256. Ends with a barrier.
__device__ __forceinline__ void tile_potrf_inv_blk64(double* T, int ld, double* Wsm, int ldw, int* info) {
  constexpr unsigned FULL = 0xffffffffu;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  for (int kb = 0; kb < 4; ++kb) {
    const int o = 16 * kb;
    if (warp == 0) {
      const int r = lane;  // lanes 16..31 shadow the shuffles; their values are discarded
      double a[16];
#pragma unroll
      for (int c = 0; c < 16; ++c) a[c] = (r < 16 && c <= r) ? T[(o + r) * ld + o + c] : 0.0;
      double rsj[16];
#pragma unroll
      for (int j = 0; j < 16; ++j) {
        double d = __shfl_sync(FULL, a[j], j);
        if (!(d > 0.0)) {
          if (lane == 0) *info = 1;
          d = 1.0;
        }
        const double rs = rsqrt(d);
        rsj[j] = rs;
        const double l = (r > j && r < 16) ? a[j] * rs : 0.0;
        if (r == j) a[j] = d * rs;
        else if (r > j) a[j] = l;
#pragma unroll
        for (int c = j + 1; c < 16; ++c) {
          const double lc = __shfl_sync(FULL, l, c);
          a[c] -= l * lc;
        }
      }
      if (r < 16) {
#pragma unroll
        for (int c = 0; c < 16; ++c)
          if (c <= r) T[(o + r) * ld + o + c] = a[c];
      }
      // W_oo: lane r holds row r
      double w[16];
#pragma unroll
      for (int c = 0; c < 16; ++c) w[c] = c == r ? 1.0 : 0.0;
#pragma unroll
      for (int t = 0; t < 16; ++t) {
        if (r == t) {
#pragma unroll
          for (int c = 0; c <= t; ++c) w[c] *= rsj[t];
        }
#pragma unroll
        for (int c = 0; c <= t; ++c) {
          const double wt = __shfl_sync(FULL, w[c], t);
          if (r > t) w[c] -= a[t] * wt;
        }
      }
      if (r < 16) {
#pragma unroll
        for (int c = 0; c < 16; ++c) Wsm[(o + c) * ldw + o + r] = c <= r ? w[c] : 0.0;
      }
    }
    __syncthreads();
    const int m = 48 - o;  // rows below the block
    if (m > 0) {
      // panel
      double out[4] = {0.0, 0.0, 0.0, 0.0};
      const int p = o + 16 + (tid >> 2), c4 = tid & 3;
      if (tid < 4 * m) {
        double x[16];
#pragma unroll
        for (int t = 0; t < 16; ++t) x[t] = T[p * ld + o + t];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int c = 4 * c4 + q;
          double s = 0.0;
#pragma unroll
          for (int t = 0; t < 16; ++t)
            if (t <= c) s += x[t] * Wsm[(o + t) * ldw + o + c];
          out[q] = s;
        }
      }
      __syncthreads();
      if (tid < 4 * m) {
#pragma unroll
        for (int q = 0; q < 4; ++q) T[p * ld + o + 4 * c4 + q] = out[q];
      }
      __syncthreads();
      // trailing lower triangle in 4 x 4 patches (pi >= qj)
      const int np4 = m / 4, npat = np4 * (np4 + 1) / 2;
      for (int pp = tid; pp < npat; pp += blockDim.x) {
        int pi = 0;
        while ((pi + 1) * (pi + 2) / 2 <= pp) ++pi;
        const int qj = pp - pi * (pi + 1) / 2;
        const int p0 = o + 16 + 4 * pi, q0 = o + 16 + 4 * qj;
        double acc[4][4];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int k = 0; k < 4; ++k) acc[i][k] = 0.0;
#pragma unroll 4
        for (int t = 0; t < 16; ++t) {
          double lp[4], lq[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            lp[i] = T[(p0 + i) * ld + o + t];
            lq[i] = T[(q0 + i) * ld + o + t];
          }
#pragma unroll
          for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int k = 0; k < 4; ++k) acc[i][k] += lp[i] * lq[k];
        }
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int k = 0; k < 4; ++k)
            if (p0 + i >= q0 + k) T[(p0 + i) * ld + q0 + k] -= acc[i][k];
      }
      __syncthreads();
    }
  }
  // W below the diagonal, block rows 1..3; S_ij staged in W's upper block
  // (j, i), i.e. S_ij(r, c) at Wsm[(16 i + r) * ldw + 16 j + c]
  for (int i = 1; i < 4; ++i) {
    for (int e = tid; e < 256 * i; e += blockDim.x) {
      const int j = e >> 8, rr = (e >> 4) & 15, cc = e & 15;
      double s = 0.0;
      for (int k = j; k < i; ++k)
#pragma unroll
        for (int t = 0; t < 16; ++t)
          s += T[(16 * i + rr) * ld + 16 * k + t] * Wsm[(16 * j + cc) * ldw + 16 * k + t];
      Wsm[(16 * i + rr) * ldw + 16 * j + cc] = s;
    }
    __syncthreads();
    // (256 threads: element e = tid + 256 q of the i blocks, q < i)
    double v[3];
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const int e = tid + 256 * q;
      v[q] = 0.0;
      if (q < i) {
        const int j = e >> 8, rr = (e >> 4) & 15, cc = e & 15;
        double s = 0.0;
#pragma unroll
        for (int t = 0; t < 16; ++t)
          if (t <= rr) s += Wsm[(16 * i + t) * ldw + 16 * i + rr] * Wsm[(16 * i + t) * ldw + 16 * j + cc];
        v[q] = -s;
      }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const int e = tid + 256 * q;
      if (q < i) {
        const int j = e >> 8, rr = (e >> 4) & 15, cc = e & 15;
        Wsm[(16 * j + cc) * ldw + 16 * i + rr] = v[q];
        Wsm[(16 * i + rr) * ldw + 16 * j + cc] = 0.0;
      }
    }
    __syncthreads();
  }
}

}  // namespace g2oc
