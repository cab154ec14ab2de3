// tile_potrf.cuh -- Cholesky factorization and inverse of one dense 64 x 64
// diagonal tile in FP64 by one CTA of 256 threads, and the FP64
// tensor-core product of 64 x 64 blocks, for the tiled Cholesky solvers
// (cholesky.cuh: 64 x 64 tiles; tc_chol.cuh: 128 x 128 tiles as 2 x 2
// blocks).
#pragma once

namespace g2oc {

// Factorization and inverse of a 64 x 64 tile, blocked by 16, with 4 x 4 + 9
// barriers (every reduction in a fixed order: bit-reproducible). T (shared memory, leading dimension
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
// A pivot at or below floor (a small multiple of the matrix's largest
// diagonal entry: a rank-deficient matrix leaves rounding-sized pivots of
// either sign) sets *info and is replaced by 1. blockDim.x must be 256.
// Ends with a barrier.
__device__ __forceinline__ void tile_potrf_inv_blk64(double* T, int ld, double* Wsm, int ldw, int* info,
                                                     double floor) {
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
        if (!(d > floor)) {
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


// P = X Y^T over k = 0..63 on the FP64 tensor cores (mma.sync m8n8k4, 256
// threads): warp w owns rows 16 (w % 4) .. + 16 and columns 32 (w / 4) .. + 32
// of P as 2 x 4 fragments of 8 x 8; lane (g, t) = (lane / 4, lane % 4) holds
// P(i0 + 8u + g, j0 + 8v + 2t + e) in acc[u][v][e]. X(i, k) is at
// Xs[i * ld + k] (row-major) or, with XK, at Xs[k * ld + i]; likewise
// Y(j, k) with YK. With ld = 68 (mod 32 = 4 pairs of banks) the fragment
// loads (eight rows x four k per warp instruction) fall in distinct bank
// pairs. The k sums run in a fixed order: bit-reproducible.
template <bool XK, bool YK>
__device__ __forceinline__ void tile_dmma64(const double* Xs, const double* Ys, int ld, double (&acc)[2][4][2]) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int i0 = 16 * (w & 3), j0 = 32 * (w >> 2);
#pragma unroll
  for (int u = 0; u < 2; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v) acc[u][v][0] = acc[u][v][1] = 0.0;
#pragma unroll 4
  for (int k0 = 0; k0 < 64; k0 += 4) {
    double fa[2], fb[4];
#pragma unroll
    for (int u = 0; u < 2; ++u) fa[u] = XK ? Xs[(k0 + t) * ld + i0 + 8 * u + g] : Xs[(i0 + 8 * u + g) * ld + k0 + t];
#pragma unroll
    for (int v = 0; v < 4; ++v) fb[v] = YK ? Ys[(k0 + t) * ld + j0 + 8 * v + g] : Ys[(j0 + 8 * v + g) * ld + k0 + t];
#pragma unroll
    for (int u = 0; u < 2; ++u)
#pragma unroll
      for (int v = 0; v < 4; ++v)
        asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                     : "+d"(acc[u][v][0]), "+d"(acc[u][v][1])
                     : "d"(fa[u]), "d"(fb[v]));
  }
}

// the element of P that acc[u][v][e] of this thread holds (tile_dmma64)
__device__ __forceinline__ int tile_dmma64_row(int u) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  return 16 * (w & 3) + 8 * u + (lane >> 2);
}
__device__ __forceinline__ int tile_dmma64_col(int v, int e) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  return 32 * (w >> 2) + 8 * v + 2 * (lane & 3) + e;
}

}  // namespace g2oc
