// pcg_tiles.cuh -- the PCG solve of pcg_persistent.cuh for a nearly full
// matrix of 6x6 blocks (the reduced camera system of a bundle adjustment
// whose cameras co-observe most of the points): the upper blocks are copied
// into dense tiles of 16 x 16 blocks (96 x 96 scalars, row-major; diagonal
// tiles hold both triangles, blocks outside the pattern are zero), and the
// product A d is a dense pass over the tiles with no index loads and no
// scattered writes.
//
// Per iteration k (d_k = s_k + beta_k d_{k-1} formed where it is read):
//   A  one CTA per tile (I, J) in turn: rows(I) += Tile d(J) and, for I < J,
//      cols(J) += Tile^T d(I), per tile; d.q as d(I).Tile d(J) (twice for an
//      off-diagonal tile);
//   -- barrier; alpha = dn / d.q
//   C  one warp per block row r: q_r = the sum of its partials, d_k stored,
//      x_r += alpha d_k, r_r -= alpha q_r, s_r = M_r^-1 r_r, partial r.s.
//      The partials of block row r are contiguous, one slot per tile index:
//      slot J holds the row sum of tile (I(r), J), slot I' < I(r) the column
//      sum of tile (I', I(r)); slots of tiles outside the pattern stay zero;
//
//   -- barrier; dn, beta, stop test.
// The arithmetic is FP64 whatever the storage type of the tiles. Sums run in
// a fixed order for a given grid size (bit-reproducible on a device).
#pragma once

#include "pcg_persistent.cuh"

namespace g2oc {

constexpr int kTileScalars = kTileBlocks * 6;              // 96
constexpr int kTileSize = kTileScalars * kTileScalars;     // 9216
constexpr int kTileThreads = 192;                          // 8 row groups x 24 column groups
constexpr int kTileWarps = kTileThreads / 32;

// Upper blocks (row-SoA, sys_offset) -> tiles. Thread per (block row a, block
// k), k fastest: reads are coalesced over the blocks of a row, each thread
// writes the 6 contiguous entries of one scalar row of its block. Blocks of a
// diagonal tile also write their transpose into its lower triangle.
template <typename Real>
__global__ void sys_to_tiles(SysDev<Real> A, const int* tile_off, Real* tiles) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)A.nnzb * 6) return;
  const int k = (int)(t % A.nnzb), a = (int)(t / A.nnzb);
  const int r = A.brow[k], c = A.rcol[k];
  const int rb = A.rptr[r], nblk = A.rptr[r + 1] - rb, j = k - rb;
  Real v[6];
#pragma unroll
  for (int b = 0; b < 6; ++b) v[b] = A.val[sys_offset<6>(rb, nblk, j, a * 6 + b)];
  const int off = tile_off[k];
  Real* dst = tiles + off + a * kTileScalars;
#pragma unroll
  for (int b = 0; b < 6; ++b) dst[b] = v[b];
  if (r != c && r / kTileBlocks == c / kTileBlocks) {
    Real* base = tiles + (off / kTileSize) * kTileSize;
    const int lr = (r % kTileBlocks) * 6, lc = (c % kTileBlocks) * 6;
#pragma unroll
    for (int b = 0; b < 6; ++b) base[(lc + b) * kTileScalars + lr + a] = v[b];
  }
}

// Block-Jacobi preconditioner read from the tiles (the Schur rows wrote the
// system there directly): the same values as the row-SoA diagonal blocks and
// the same inverses as pcg_diag_inv, five blocks per warp, one row per lane
// (inverse_gj_lanes). Launch with nb * 32 / 5 threads or more.
template <typename Real>
__global__ void pcg_diag_inv_tiles(const Real* tiles, const int* tile_off, const int* diag, int nb, double* minv,
                                   int* nonfinite) {
  const int lane = threadIdx.x & 31;
  const int gw = (int)((blockIdx.x * blockDim.x + threadIdx.x) >> 5);
  const int grp = lane / 6, i = lane - 6 * grp;
  const int blk = gw * 5 + grp;
  const bool act = grp < 5 && blk < nb;
  double m[6], inv[6];
  if (act) {
    const Real* T = tiles + tile_off[diag[blk]] + (size_t)i * kTileScalars;
#pragma unroll
    for (int c = 0; c < 6; ++c) m[c] = (double)T[c];
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

// four consecutive entries of a tile row (16-byte aligned), kept in the
// storage type until they are used
__device__ __forceinline__ void load4(const float* p, float (&m)[4]) {
  const float4 v = __ldg(reinterpret_cast<const float4*>(p));
  m[0] = v.x;
  m[1] = v.y;
  m[2] = v.z;
  m[3] = v.w;
}
__device__ __forceinline__ void load4(const double* p, double (&m)[4]) {
  const double2 u = __ldg(reinterpret_cast<const double2*>(p));
  const double2 w = __ldg(reinterpret_cast<const double2*>(p) + 1);
  m[0] = u.x;
  m[1] = u.y;
  m[2] = w.x;
  m[3] = w.y;
}

template <typename Real>
__global__ void __launch_bounds__(kTileThreads, sizeof(Real) == 4 ? 3 : 2)
    pcg_solve_tiles(const Real* tiles, const int2* tile_ij, int ntiles, int nbt, int nb, const double* minv,
                    const double* b, double* x, double* r, double* s, double* dbuf0, double* dbuf1, double* part,
                    double* part_dq, double* part_rs, PcgState* st, double tol, int max_iter, int abs_tol,
                    int fixed_d0, unsigned barrier_extra) {
  constexpr int BS = 6;
  __shared__ double red[kTileWarps];
  __shared__ double drow[kTileScalars], dcol[kTileScalars];
  __shared__ double red_row[kTileScalars][25];
  __shared__ double red_col[8][kTileScalars];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int gw = blockIdx.x * kTileWarps + warp, GW = gridDim.x * kTileWarps;
  const int h = tid / 24, g = tid % 24;  // row group (12 rows), column group (4 columns)
  const int n = nb * BS;
  const bool fixed = fixed_d0 != 0;
  const double d0_in = st->d0;
  const double carry = st->residual_carry;
  unsigned gen = grid_gen_start(st);

  // r = b, x = 0, s = M^-1 r, d_{-1} = 0, dn = r.s (linear_solver_pcg.hpp:117-137)
  double rs = 0.0;
  for (int c = gw; c < nb; c += GW) {
    double rc[BS];
#pragma unroll
    for (int a = 0; a < BS; ++a) rc[a] = b[(size_t)c * BS + a];
    rs += row_precondition<BS>(minv, c, rc, lane, s);
    if (lane < BS) {
      const size_t o = (size_t)c * BS + lane;
      r[o] = pick<BS>(rc, lane);
      x[o] = 0.0;
      dbuf1[o] = 0.0;
    }
  }
  cta_partial<kTileWarps>(rs, part_rs, red);
  if (!grid_barrier(st, gen, barrier_extra)) return;
  double dn = cta_sum_all<kTileWarps>(part_rs, red);
  double d0 = d0_in;
  if (!fixed) {
    d0 = tol * dn;
    if (abs_tol && carry > 0.0 && carry > d0) d0 = carry;
  }
  int k = 0;
  double beta = 0.0;
  bool breakdown = false;
  bool stop = dn <= d0 || max_iter <= 0;
  while (!stop) {
    const double* dprev = (k & 1) ? dbuf0 : dbuf1;  // d_{k-1}
    double* dcur = (k & 1) ? dbuf1 : dbuf0;         // d_k
    // ---- A: tiles
    double dq = 0.0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
      const int2 ij = __ldg(tile_ij + t);
      {
        const int which = tid < kTileScalars ? 0 : 1;
        const int i = tid - which * kTileScalars;
        const int gi = (which ? ij.y : ij.x) * kTileScalars + i;
        const double v = gi < n ? __ldcg(s + gi) + beta * __ldcg(dprev + gi) : 0.0;
        if (which) dcol[i] = v;
        else drow[i] = v;
      }
      __syncthreads();
      const Real* T = tiles + (size_t)t * kTileSize + (size_t)(12 * h) * kTileScalars + 4 * g;
      Real m[12][4];
#pragma unroll
      for (int i = 0; i < 12; ++i) load4(T + i * kTileScalars, m[i]);
      double dc[4], colacc[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        dc[q] = dcol[4 * g + q];
        colacc[q] = 0.0;
      }
#pragma unroll
      for (int i = 0; i < 12; ++i) {
        double ra = 0.0;
        const double dri = drow[12 * h + i];
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const double mv = (double)m[i][q];
          ra += mv * dc[q];
          colacc[q] += mv * dri;
        }
        red_row[12 * h + i][g] = ra;
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) red_col[h][4 * g + q] = colacc[q];
      __syncthreads();
      if (tid < kTileScalars) {
        double v = 0.0;
#pragma unroll
        for (int q = 0; q < 24; ++q) v += red_row[tid][q];
        const int rr = ij.x * kTileBlocks + tid / BS;
        if (rr < nb) part[((size_t)rr * nbt + ij.y) * BS + tid % BS] = v;
        dq += (ij.x == ij.y ? 1.0 : 2.0) * drow[tid] * v;
      } else if (ij.x != ij.y) {
        const int cc = tid - kTileScalars;
        double v = 0.0;
#pragma unroll
        for (int q = 0; q < 8; ++q) v += red_col[q][cc];
        const int rr = ij.y * kTileBlocks + cc / BS;
        if (rr < nb) part[((size_t)rr * nbt + ij.x) * BS + cc % BS] = v;
      }
      __syncthreads();
    }
    // the first block row of this warp in phase C: its s, d_{k-1}, r, x and
    // M^-1 row, loaded while the CTAs meet at the barrier (they do not
    // depend on alpha)
    double sa = 0.0, da = 0.0, ra = 0.0, xa = 0.0, mrow[BS];
    auto load_row = [&](int c) {
      if (lane < BS) {
        const size_t o = (size_t)c * BS + lane;
        sa = __ldcg(s + o);
        da = __ldcg(dprev + o);
        ra = __ldcg(r + o);
        xa = __ldcg(x + o);
        const double* M = minv + (size_t)c * BS * BS + (size_t)lane * BS;
#pragma unroll
        for (int b2 = 0; b2 < BS; ++b2) mrow[b2] = M[b2];
      }
    };
#pragma unroll
    for (int b2 = 0; b2 < BS; ++b2) mrow[b2] = 0.0;
    if (gw < nb) load_row(gw);
    cta_partial<kTileWarps>(dq, part_dq, red);
    if (!grid_barrier(st, gen, barrier_extra)) return;
    const double dqs = cta_sum_all<kTileWarps>(part_dq, red);
    if (!(dqs > 0.0)) {
      breakdown = true;  // not positive definite along d (see pcg_solve_persistent)
      break;
    }
    const double alpha = dn / dqs;
    // ---- C: block rows
    rs = 0.0;
    for (int c = gw; c < nb; c += GW) {
      if (c != gw) load_row(c);
      double q[BS];
#pragma unroll
      for (int a = 0; a < BS; ++a) q[a] = 0.0;
      const double* pr = part + (size_t)c * nbt * BS;
      for (int e = lane; e < nbt; e += 32) {
#pragma unroll
        for (int a = 0; a < BS; ++a) q[a] += __ldcg(pr + (size_t)e * BS + a);
      }
#pragma unroll
      for (int a = 0; a < BS; ++a) q[a] = warp_sum(q[a]);
      const double qa = pick<BS>(q, lane);
      const double dka = sa + beta * da;
      const double rca = ra - alpha * qa;
      double rc[BS];
#pragma unroll
      for (int a = 0; a < BS; ++a) rc[a] = __shfl_sync(0xffffffffu, rca, a);
      if (lane < BS) {
        double v = 0.0;
#pragma unroll
        for (int b2 = 0; b2 < BS; ++b2) v += mrow[b2] * rc[b2];
        const size_t o = (size_t)c * BS + lane;
        s[o] = v;
        rs += rca * v;
        x[o] = xa + alpha * dka;
        dcur[o] = dka;
        r[o] = rca;
      }
    }
    cta_partial<kTileWarps>(rs, part_rs, red);
    if (!grid_barrier(st, gen, barrier_extra)) return;
    const double dn_new = cta_sum_all<kTileWarps>(part_rs, red);
    beta = dn_new / dn;
    dn = dn_new;
    ++k;
    stop = dn <= d0 || k >= max_iter;
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
