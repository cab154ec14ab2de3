// tile_potrf.cuh -- Cholesky factorization and inverse of one dense 64 x 64
// diagonal tile in FP64 by one CTA of 256 threads, and the FP64
// tensor-core product of 64 x 64 blocks, for the tiled Cholesky solvers
// (cholesky.cuh: 64 x 64 tiles; tc_chol.cuh: 128 x 128 tiles as 2 x 2
// blocks).
#pragma once

namespace g2oc {

// One FP64 tensor-core product of 8 x 8 fragments (mma.sync m8n8k4):
// lane (g, t) = (lane / 4, lane % 4) holds P(8 fi + g, 8 fj + 2 t + e) in
// c[e], P = sum_k X(i, k) Y(j, k) over k < K (a multiple of 4). X(i, k) is at
// X[i * ldx + k] (row-major) or, with XK, at X[k * ldx + i]; likewise Y.
template <bool XK, bool YK>
__device__ __forceinline__ void dmma_frag(const double* X, int ldx, const double* Y, int ldy, int fi, int fj, int K,
                                          double (&c)[2]) {
  const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
  c[0] = c[1] = 0.0;
  for (int k0 = 0; k0 < K; k0 += 4) {
    const double a = XK ? X[(k0 + t) * ldx + 8 * fi + g] : X[(8 * fi + g) * ldx + k0 + t];
    const double b = YK ? Y[(k0 + t) * ldy + 8 * fj + g] : Y[(8 * fj + g) * ldy + k0 + t];
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(c[0]), "+d"(c[1])
                 : "d"(a), "d"(b));
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

// Factorization and inverse of a 64 x 64 tile, blocked by 16 (every
// reduction in a fixed order: bit-reproducible). T (shared memory, leading
// dimension ld): lower triangle A in, L out; Wsm (shared memory, FP64,
// column-major with leading dimension ldw): W = L^-1 out, zero above the
// diagonal; scratch: 768 doubles of shared memory. Per block column of 16
// (offset o):
//   1. warp 0 factors the 16 x 16 diagonal block in registers (lane r holds
//      row r; the pivot and the column values pass by shuffles, pivots by
//      rsqrt) and inverts it (W_oo, rows by forward substitution);
//   2. the panel below: L(p, o + c) = sum_t A(p, o + t) W_oo(c, t);
//   3. the trailing lower triangle: A(p, q) -= sum_t L(p, o + t) L(q, o + t);
// both as FP64 tensor-core products of 8 x 8 fragments dealt to the warps.
// Then W's blocks below the diagonal by block rows i = 1..3:
//   W_ij = -W_ii (sum_{k=j}^{i-1} L_ik W_kj), the sums staged in scratch.
// A pivot at or below floor (a small multiple of the matrix's largest
// diagonal entry: a rank-deficient matrix leaves rounding-sized pivots of
// either sign) sets *info and is replaced by 1. blockDim.x must be 256.
// Ends with a barrier.
__device__ __forceinline__ void tile_potrf_inv_blk64(double* T, int ld, double* Wsm, int ldw, int* info,
                                                     double floor, double* scratch) {
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
      const int lane2 = lane >> 2, t2 = lane & 3;
      // panel into scratch (m x 16, row-major), then over A's panel
      const int npan = (m / 8) * 2;
      for (int f = warp; f < npan; f += 8) {
        const int fi = f >> 1, fj = f & 1;
        double c[2];
        dmma_frag<false, true>(T + (o + 16) * ld + o, ld, Wsm + o * ldw + o, ldw, fi, fj, 16, c);
        scratch[(8 * fi + lane2) * 16 + 8 * fj + 2 * t2] = c[0];
        scratch[(8 * fi + lane2) * 16 + 8 * fj + 2 * t2 + 1] = c[1];
      }
      __syncthreads();
      for (int e = tid; e < m * 16; e += blockDim.x) T[(o + 16 + (e >> 4)) * ld + o + (e & 15)] = scratch[e];
      __syncthreads();
      // trailing lower triangle: fragments (fi >= fj) of the m x m block
      const int nf = m / 8, ntri = nf * (nf + 1) / 2;
      for (int f = warp; f < ntri; f += 8) {
        int fi = 0;
        while ((fi + 1) * (fi + 2) / 2 <= f) ++fi;
        const int fj = f - fi * (fi + 1) / 2;
        double c[2];
        const double* P = T + (o + 16) * ld + o;
        dmma_frag<false, false>(P, ld, P, ld, fi, fj, 16, c);
        const int r = 8 * fi + lane2, q = 8 * fj + 2 * t2;
        if (r >= q) T[(o + 16 + r) * ld + o + 16 + q] -= c[0];
        if (r >= q + 1) T[(o + 16 + r) * ld + o + 16 + q + 1] -= c[1];
      }
      __syncthreads();
    }
  }
  // W's blocks above the diagonal are zero
  for (int e = tid; e < 6 * 256; e += blockDim.x) {
    const int b = e >> 8, rr = (e >> 4) & 15, cc = e & 15;
    const int bi = b < 1 ? 1 : b < 3 ? 2 : 3, bj = b < 1 ? 0 : b < 3 ? b - 1 : b - 3;  // (1,0) (2,0) (2,1) (3,0..2)
    Wsm[(16 * bi + cc) * ldw + 16 * bj + rr] = 0.0;
  }
  // W below the diagonal, block rows 1..3: S_ij = sum_{k=j}^{i-1} L_ik W_kj
  // into scratch (16 x 16 row-major per j), then W_ij = -W_ii S_ij
  const int lane2 = lane >> 2, t2 = lane & 3;
  for (int i = 1; i < 4; ++i) {
    for (int f = warp; f < 4 * i; f += 8) {
      const int j = f >> 2, fi = (f >> 1) & 1, fj = f & 1;
      double c[2];
      // X(r, kk) = L(16 i + r, 16 j + kk); Y(cc, kk) = W(16 j + kk, 16 j + cc)
      dmma_frag<false, false>(T + 16 * i * ld + 16 * j, ld, Wsm + 16 * j * ldw + 16 * j, ldw, fi, fj, 16 * (i - j), c);
      scratch[j * 256 + (8 * fi + lane2) * 16 + 8 * fj + 2 * t2] = c[0];
      scratch[j * 256 + (8 * fi + lane2) * 16 + 8 * fj + 2 * t2 + 1] = c[1];
    }
    __syncthreads();
    for (int f = warp; f < 4 * i; f += 8) {
      const int j = f >> 2, fi = (f >> 1) & 1, fj = f & 1;
      double c[2];
      // X(r, kk) = W_ii(r, kk) at Wsm[(16 i + kk) ldw + 16 i + r]; Y(cc, kk) = S_ij(kk, cc)
      dmma_frag<true, true>(Wsm + 16 * i * ldw + 16 * i, ldw, scratch + j * 256, 16, fi, fj, 16, c);
      const int r = 8 * fi + lane2, q = 8 * fj + 2 * t2;
      Wsm[(16 * j + q) * ldw + 16 * i + r] = -c[0];
      Wsm[(16 * j + q + 1) * ldw + 16 * i + r] = -c[1];
    }
    __syncthreads();
  }
}


}  // namespace g2oc
