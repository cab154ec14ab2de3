// cholesky.cuh -- LinearSolverCudaCholesky: FP64 tiled Cholesky of the
// (reduced) block system, the role of LinearSolverEigen's SimplicialLLT and
// LinearSolverDense's LDLT (g2o/solvers/eigen/linear_solver_eigen.h:94-191,
// g2o/solvers/dense/linear_solver_dense.h:57-105).
//
// Plan (once per pattern, on the host): reverse Cuthill-McKee block ordering
// for sparse systems, then a symbolic factorization at the level of 64x64
// tiles, giving per step k the list of nonzero panel tiles and the list of
// trailing tile pairs to update. Numeric (every solve, on the device): the
// permuted matrix is expanded into a dense column-major buffer, and only the
// structurally nonzero tiles are factored (potrf of the diagonal tile, trsm
// of the panel, gemm/syrk of the trailing tiles), followed by blocked
// forward / backward substitution. A non-positive pivot sets the info flag
// (G2OC_ERR_NOT_PD at the boundary); nothing traps.
#pragma once

#include <algorithm>
#include <queue>
#include <vector>

#include "g2oc_internal.h"
#include "pcg_kernels.cuh"
#include "tile_potrf.cuh"

namespace g2oc {

constexpr int kTile = 64;

struct CholPlan {
  int nb = 0, bs = 0, n = 0, np = 0, nt = 0;
  const void* key = nullptr;  // pattern identity
  std::vector<int> perm;      // block i -> position
  std::vector<int> pnl_ptr, pnl;     // per k: tiles i > k with L(i,k) != 0
  std::vector<int> upd_ptr;          // per k: range into upd
  std::vector<int2> upd;             // trailing pairs (i, j), i >= j > k
  std::vector<int> bwd_ptr, bwd;     // per k: tiles i < k with L(k,i) != 0
  DBuf<int> d_perm, d_pnl, d_bwd;
  DBuf<int2> d_upd;
  DBuf<int> d_pnl_ptr, d_upd_ptr, d_bwd_ptr;
  DBuf<double> A, y;
  DBuf<double> W;  // W(k) = L(k,k)^-1 per diagonal tile
  DBuf<double> floor;  // pivot floor of the current factorization
  DBuf<int> info;
  // every step has at most kCholSingleWidth panel tiles plus trailing
  // updates: the whole plan runs in one CTA (chol_factor_single)
  bool single = false;
};

constexpr int kCholSingleWidth = 24;

// reverse Cuthill-McKee on the block graph
static void rcm_order(int nb, const std::vector<int32_t>& rc, std::vector<int>& perm) {
  std::vector<std::vector<int>> adj(nb);
  for (size_t k = 0; k < rc.size() / 2; ++k) {
    const int r = rc[2 * k], c = rc[2 * k + 1];
    if (r != c) {
      adj[r].push_back(c);
      adj[c].push_back(r);
    }
  }
  std::vector<int> order;
  order.reserve(nb);
  std::vector<char> seen(nb, 0);
  while ((int)order.size() < nb) {
    int start = -1;
    size_t best = SIZE_MAX;
    for (int i = 0; i < nb; ++i)
      if (!seen[i] && adj[i].size() < best) {
        best = adj[i].size();
        start = i;
      }
    std::queue<int> q;
    q.push(start);
    seen[start] = 1;
    while (!q.empty()) {
      const int u = q.front();
      q.pop();
      order.push_back(u);
      std::vector<int> nbr;
      for (int v : adj[u])
        if (!seen[v]) {
          seen[v] = 1;
          nbr.push_back(v);
        }
      std::sort(nbr.begin(), nbr.end(), [&](int a, int b) {
        return adj[a].size() < adj[b].size() || (adj[a].size() == adj[b].size() && a < b);
      });
      for (int v : nbr) q.push(v);
    }
  }
  perm.assign(nb, 0);
  for (int i = 0; i < nb; ++i) perm[order[nb - 1 - i]] = i;
}

// extra: further (row, col) block pairs whose entries the plan must hold
// (the blocks a selected inverse is asked for), treated as structural
// nonzeros of the matrix so that the symbolic fill covers them
static int chol_plan_build(CholPlan& P, int nb, int bs, const std::vector<int32_t>& rc, bool reorder,
                           cudaStream_t st, const std::vector<int32_t>* extra = nullptr) {
  P.nb = nb;
  P.bs = bs;
  P.n = nb * bs;
  P.nt = (P.n + kTile - 1) / kTile;
  P.np = P.nt * kTile;
  if (reorder) rcm_order(nb, rc, P.perm);
  else {
    P.perm.resize(nb);
    for (int i = 0; i < nb; ++i) P.perm[i] = i;
  }
  const int nt = P.nt;
  std::vector<char> nz((size_t)nt * nt, 0);
  auto mark = [&](int r, int c) {
    const int a0 = P.perm[r] * bs, b0 = P.perm[c] * bs;
    for (int ti = a0 / kTile; ti <= (a0 + bs - 1) / kTile; ++ti)
      for (int tj = b0 / kTile; tj <= (b0 + bs - 1) / kTile; ++tj) {
        const int i = std::max(ti, tj), j = std::min(ti, tj);
        nz[(size_t)i * nt + j] = 1;
      }
  };
  for (size_t k = 0; k < rc.size() / 2; ++k) mark(rc[2 * k], rc[2 * k + 1]);
  if (extra)
    for (size_t k = 0; k < extra->size() / 2; ++k) mark((*extra)[2 * k], (*extra)[2 * k + 1]);
  for (int t = 0; t < nt; ++t) nz[(size_t)t * nt + t] = 1;
  P.pnl_ptr.assign(nt + 1, 0);
  P.upd_ptr.assign(nt + 1, 0);
  P.pnl.clear();
  P.upd.clear();
  std::vector<int> cols;
  for (int k = 0; k < nt; ++k) {
    cols.clear();
    for (int i = k + 1; i < nt; ++i)
      if (nz[(size_t)i * nt + k]) cols.push_back(i);
    for (size_t a = 0; a < cols.size(); ++a)
      for (size_t b = 0; b <= a; ++b) {
        nz[(size_t)cols[a] * nt + cols[b]] = 1;
        P.upd.push_back(make_int2(cols[a], cols[b]));
      }
    P.pnl.insert(P.pnl.end(), cols.begin(), cols.end());
    P.pnl_ptr[k + 1] = (int)P.pnl.size();
    P.upd_ptr[k + 1] = (int)P.upd.size();
  }
  // backward lists: for k, tiles i < k with L(k, i) != 0
  P.bwd_ptr.assign(nt + 1, 0);
  P.bwd.clear();
  for (int k = 0; k < nt; ++k) {
    for (int i = 0; i < k; ++i)
      if (nz[(size_t)k * nt + i]) P.bwd.push_back(i);
    P.bwd_ptr[k + 1] = (int)P.bwd.size();
  }
  int width = 0;
  for (int k = 0; k < nt; ++k)
    width = std::max(width, P.pnl_ptr[k + 1] - P.pnl_ptr[k] + P.upd_ptr[k + 1] - P.upd_ptr[k]);
  P.single = width <= kCholSingleWidth;
  G2OC_TRY(P.d_pnl_ptr.upload(P.pnl_ptr, st));
  G2OC_TRY(P.d_upd_ptr.upload(P.upd_ptr, st));
  G2OC_TRY(P.d_bwd_ptr.upload(P.bwd_ptr, st));
  G2OC_TRY(P.d_perm.upload(P.perm, st));
  G2OC_TRY(P.d_pnl.upload(P.pnl.empty() ? std::vector<int>{0} : P.pnl, st));
  G2OC_TRY(P.d_upd.upload(P.upd.empty() ? std::vector<int2>{make_int2(0, 0)} : P.upd, st));
  G2OC_TRY(P.d_bwd.upload(P.bwd.empty() ? std::vector<int>{0} : P.bwd, st));
  G2OC_TRY(P.A.alloc((size_t)P.np * P.np));
  G2OC_TRY(P.y.alloc(P.np));
  G2OC_TRY(P.W.alloc((size_t)nt * kTile * kTile));
  G2OC_TRY(P.floor.alloc(1));
  G2OC_TRY(P.info.alloc(1));
  return G2OC_OK;
}

// dense column-major A(np x np): permuted blocks and their transposes,
// identity on the padding
template <typename Real>
__global__ void chol_densify(SysDev<Real> S, int bs, const int* perm, int n, int np, double* A) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long per = (long long)bs * bs;
  const int nnzb = S.nnzb;
  if (t < (long long)nnzb * per) {
    const int p = (int)(t / per), e = (int)(t % per);
    const int r = S.brow[p], c = S.rcol[p];
    const int i = e / bs, j = e % bs;
    const int gi = perm[r] * bs + i, gj = perm[c] * bs + j;
    const int rb = S.rptr[r], nblk = S.rptr[r + 1] - rb;
    const double v = (double)S.val[(size_t)rb * per + (size_t)e * nblk + (p - rb)];
    A[(size_t)gj * np + gi] = v;
    A[(size_t)gi * np + gj] = v;
  } else {
    const long long pad = t - (long long)nnzb * per;
    if (pad < np - n) {
      const int g = n + (int)pad;
      A[(size_t)g * np + g] = 1.0;
    }
  }
}

// the pivot floor of a factorization: 4 n eps times the largest diagonal
// entry of the (densified) matrix, one CTA of 1024 threads (fixed tree)
template <typename Elem>
static __global__ void __launch_bounds__(1024) chol_pivot_floor(const Elem* A, int np, int n, double* floor) {
  __shared__ double red[32];
  double m = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) m = fmax(m, fabs((double)A[(size_t)i * np + i]));
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = fmax(r, red[w]);
    *floor = 4.0 * (double)n * 2.220446049250313e-16 * r;
  }
}

// asynchronous 8-byte global -> shared copies (every load of a tile in
// flight at once, instead of one round trip per loop step)
__device__ __forceinline__ void cp_async8(void* dst, const void* src) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"((unsigned)__cvta_generic_to_shared(dst)), "l"(src)
               : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Operand tiles of the tile products in shared memory: 64 rows of kLd
// doubles (row-major, (row, k) at [row * kLd + k]). With kLd = 68 the
// fragment loads of the FP64 tensor-core products (eight rows x four k per
// warp instruction) fall in distinct bank pairs.
constexpr int kLd = kTile + 4;
constexpr int kTileBuf = kTile * kLd;  // doubles per operand tile

// factor the diagonal tile k in shared memory (lower; T: a tile buffer, used
// with leading dimension kTile + 1) and form W = L(k,k)^-1 in Wsm (FP64
// shared memory, column-major, leading dimension ldw; scratch: 768 doubles of
// shared memory); 256 threads
__device__ __forceinline__ void chol_potrf_tile(double* A, int np, int k, double* T, double* Wsm, int ldw, int* info,
                                                double floor, double* scratch) {
  constexpr int ld = kTile + 1;
  const size_t base = (size_t)k * kTile;
  for (int e = threadIdx.x; e < kTile * kTile; e += blockDim.x) {
    const int i = e % kTile, j = e / kTile;
    if (i >= j) cp_async8(T + i * ld + j, A + (base + j) * np + base + i);
  }
  cp_async_wait_all();
  __syncthreads();
  tile_potrf_inv_blk64(T, ld, Wsm, ldw, info, floor, scratch);
  for (int e = threadIdx.x; e < kTile * kTile; e += blockDim.x) {
    const int i = e % kTile, j = e / kTile;
    if (i >= j) A[(base + j) * np + base + i] = T[i * ld + j];
  }
}

// W(k) of every diagonal tile, kTile x kTile column-major, at W + k kTile^2
constexpr int kPotrfSmem = (2 * kTile * (kTile + 1) + 768) * (int)sizeof(double);
static __global__ void __launch_bounds__(256) chol_potrf(double* A, int np, int k, double* W, const double* floor,
                                                         int* info) {
  extern __shared__ double sm_potrf[];
  double* T = sm_potrf;
  double* Wsm = sm_potrf + kTile * (kTile + 1);
  chol_potrf_tile(A, np, k, T, Wsm, kTile + 1, info, *floor, sm_potrf + 2 * kTile * (kTile + 1));
  double* Wk = W + (size_t)k * kTile * kTile;
  for (int e = threadIdx.x; e < kTile * kTile; e += blockDim.x) Wk[e] = Wsm[(e / kTile) * (kTile + 1) + e % kTile];
}

constexpr int kTileSmem = 2 * kTileBuf * (int)sizeof(double);
// chol_factor_single: two operand tiles and W
constexpr int kTileSmemSingle = 3 * kTileBuf * (int)sizeof(double);

// an operand tile (row, k) from the column-major tile of A at rows rb,
// columns cb (k = column)
__device__ __forceinline__ void chol_load_operand(const double* A, int np, size_t rb, size_t cb, double* Xs) {
  for (int e = threadIdx.x; e < kTile * kTile; e += blockDim.x) {
    const int r = e % kTile, c = e / kTile;
    cp_async8(Xs + r * kLd + c, A + (cb + c) * np + rb + r);
  }
}

// panel: L(i,k) = A(i,k) L(k,k)^-T = A(i,k) W^T for the tile i, with
// W(r, c) at Ws[c * kLd + r] in shared memory (256 threads)
__device__ __forceinline__ void chol_trsm_tile(double* A, int np, int k, int ti, const double* Ws, double* Xs) {
  const size_t kb = (size_t)k * kTile, ib = (size_t)ti * kTile;
  chol_load_operand(A, np, ib, kb, Xs);
  cp_async_wait_all();
  __syncthreads();
  double acc[2][4][2];
  tile_dmma64<false, true>(Xs, Ws, kLd, acc);  // Y(j, t) = W(j, t) at Ws[t * kLd + j]
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int i0 = 16 * (w & 3), j0 = 32 * (w >> 2);
#pragma unroll
  for (int u = 0; u < 2; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
      for (int e = 0; e < 2; ++e)
        A[(kb + j0 + 8 * v + 2 * t + e) * np + ib + i0 + 8 * u + g] = acc[u][v][e];
}

static __global__ void __launch_bounds__(256) chol_trsm(double* A, int np, int k, const int* tiles, const double* W) {
  extern __shared__ double sm_trsm[];
  double* Ws = sm_trsm;
  double* Xs = sm_trsm + kTileBuf;
  const double* Wk = W + (size_t)k * kTile * kTile;
  for (int e = threadIdx.x; e < kTile * kTile; e += blockDim.x) Ws[(e / kTile) * kLd + e % kTile] = Wk[e];
  chol_trsm_tile(A, np, k, tiles[blockIdx.x], Ws, Xs);
}

// trailing update: A(i,j) -= L(i,k) L(j,k)^T (256 threads)
__device__ __forceinline__ void chol_gemm_tile(double* A, int np, int k, int2 ij, double* Li, double* Lj) {
  const size_t kb = (size_t)k * kTile, ib = (size_t)ij.x * kTile, jb = (size_t)ij.y * kTile;
  chol_load_operand(A, np, ib, kb, Li);
  chol_load_operand(A, np, jb, kb, Lj);
  cp_async_wait_all();
  __syncthreads();
  double acc[2][4][2];
  tile_dmma64<false, false>(Li, Lj, kLd, acc);
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int i0 = 16 * (w & 3), j0 = 32 * (w >> 2);
  const bool diag = ij.x == ij.y;
#pragma unroll
  for (int u = 0; u < 2; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int r = i0 + 8 * u + g, c = j0 + 8 * v + 2 * t + e;
        if (diag && r < c) continue;
        A[(jb + c) * np + ib + r] -= acc[u][v][e];
      }
}

static __global__ void __launch_bounds__(256) chol_gemm(double* A, int np, int k, const int2* pairs) {
  extern __shared__ double sm_gemm[];
  chol_gemm_tile(A, np, k, pairs[blockIdx.x], sm_gemm, sm_gemm + kTileBuf);
}

// The whole factorization in one CTA of 256 threads, for plans whose steps
// are narrow (the pose graphs after reverse Cuthill-McKee: a banded tile
// pattern, a few panel tiles and trailing updates per step). The
// multi-launch form spends such a plan in the launch latency of its n / 64
// strictly sequential steps; here the steps run back to back with the same
// tile algorithms (same arithmetic, same order), the tiles passing through
// shared memory, W(k) staying in shared memory and the factor in the dense
// buffer.
static __global__ void __launch_bounds__(256) chol_factor_single(double* A, int np, int nt, const int* pnl_ptr,
                                                                 const int* pnl, const int* upd_ptr,
                                                                 const int2* upd, double* W, const double* floor,
                                                                 int* info) {
  extern __shared__ double sm_single[];
  double* B0 = sm_single;
  double* B1 = sm_single + kTileBuf;
  double* Ws = sm_single + 2 * kTileBuf;
  const double fl = *floor;
  for (int k = 0; k < nt; ++k) {
    chol_potrf_tile(A, np, k, B0, Ws, kLd, info, fl, B1);  // B1 is free until the panel
    // W(k) kept for the substitutions (chol_solve_single)
    for (int e = threadIdx.x; e < kTile * kTile; e += blockDim.x)
      W[(size_t)k * kTile * kTile + e] = Ws[(e / kTile) * kLd + e % kTile];
    __syncthreads();
    for (int p = pnl_ptr[k]; p < pnl_ptr[k + 1]; ++p) {
      chol_trsm_tile(A, np, k, pnl[p], Ws, B1);
      __syncthreads();
    }
    for (int p = upd_ptr[k]; p < upd_ptr[k + 1]; ++p) {
      chol_gemm_tile(A, np, k, upd[p], B0, B1);
      __syncthreads();
    }
  }
}

// permuted right-hand side y(perm) = b
static __global__ void chol_load_rhs(const double* b, const int* perm, int nb, int bs, int n, int np, double* y) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) y[perm[t / bs] * bs + t % bs] = b[t];
  else if (t < np) y[t] = 0.0;
}

static __global__ void chol_store_x(const double* y, const int* perm, int bs, int n, double* x) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n) x[t] = y[perm[t / bs] * bs + t % bs];
}

// The substitutions take 64-long dot products with four threads per row
// (16 terms each, all loads in flight, then a fixed xor tree over the four
// lanes): 256 threads per 64 x 64 tile.
__device__ __forceinline__ double chol_dot4(double s) {
  s += __shfl_xor_sync(0xffffffffu, s, 1);
  s += __shfl_xor_sync(0xffffffffu, s, 2);
  return s;
}

// s = sum over this thread's 16 columns of M(row, c) v[c], M column-major
// with leading dimension ld (M(row, c) at M[c * ld + row]), summed over the
// row's four threads
__device__ __forceinline__ double chol_rowdot(const double* M, size_t ld, const double* v) {
  const int q = threadIdx.x & 3, row = threadIdx.x >> 2;
  double t[16];
#pragma unroll
  for (int c = 0; c < 16; ++c) t[c] = M[(size_t)(q * 16 + c) * ld + row];
  double s = 0.0;
#pragma unroll
  for (int c = 0; c < 16; ++c) s += t[c] * v[q * 16 + c];
  return chol_dot4(s);
}

// s = sum over this thread's 16 rows of M(r, col) v[r] (a column of M times
// v), M column-major with leading dimension ld, col = the thread's row index
__device__ __forceinline__ double chol_coldot(const double* M, size_t ld, const double* v) {
  const int q = threadIdx.x & 3, col = threadIdx.x >> 2;
  double t[16];
#pragma unroll
  for (int r = 0; r < 16; ++r) t[r] = M[(size_t)col * ld + q * 16 + r];
  double s = 0.0;
#pragma unroll
  for (int r = 0; r < 16; ++r) s += t[r] * v[q * 16 + r];
  return chol_dot4(s);
}

// L(k,k) y_k = y_k as y_k = W(k) y_k (256 threads)
static __global__ void __launch_bounds__(256) chol_fwd_diag(const double* W, int k, double* y) {
  __shared__ double v[kTile];
  const size_t kb = (size_t)k * kTile;
  if (threadIdx.x < kTile) v[threadIdx.x] = y[kb + threadIdx.x];
  __syncthreads();
  const double s = chol_rowdot(W + kb * kTile, kTile, v);
  if ((threadIdx.x & 3) == 0) y[kb + (threadIdx.x >> 2)] = s;
}

// y_i -= L(i,k) y_k for the listed tiles i > k (CTA per tile, 256 threads)
static __global__ void __launch_bounds__(256) chol_fwd_update(const double* A, int np, int k, const int* tiles,
                                                              double* y) {
  __shared__ double v[kTile];
  const size_t kb = (size_t)k * kTile, ib = (size_t)tiles[blockIdx.x] * kTile;
  if (threadIdx.x < kTile) v[threadIdx.x] = y[kb + threadIdx.x];
  __syncthreads();
  const double s = chol_rowdot(A + kb * np + ib, np, v);
  if ((threadIdx.x & 3) == 0) y[ib + (threadIdx.x >> 2)] -= s;
}

// L(k,k)^T x_k = y_k as y_k = W(k)^T y_k (256 threads)
static __global__ void __launch_bounds__(256) chol_bwd_diag(const double* W, int k, double* y) {
  __shared__ double v[kTile];
  const size_t kb = (size_t)k * kTile;
  if (threadIdx.x < kTile) v[threadIdx.x] = y[kb + threadIdx.x];
  __syncthreads();
  const double s = chol_coldot(W + kb * kTile, kTile, v);
  if ((threadIdx.x & 3) == 0) y[kb + (threadIdx.x >> 2)] = s;
}

// y_i -= L(k,i)^T y_k for the listed tiles i < k (CTA per tile, 256 threads)
static __global__ void __launch_bounds__(256) chol_bwd_update(const double* A, int np, int k, const int* tiles,
                                                              double* y) {
  __shared__ double v[kTile];
  const size_t kb = (size_t)k * kTile, ib = (size_t)tiles[blockIdx.x] * kTile;
  if (threadIdx.x < kTile) v[threadIdx.x] = y[kb + threadIdx.x];
  __syncthreads();
  const double s = chol_coldot(A + ib * np + kb, np, v);
  if ((threadIdx.x & 3) == 0) y[ib + (threadIdx.x >> 2)] -= s;
}

// Both substitutions of a single-CTA plan in one CTA of 256 threads: per
// diagonal tile the product with W(k) (kept by chol_factor_single), then
// the products of the tiles the step updates, one tile at a time, with the
// four-thread dot products above.
static __global__ void __launch_bounds__(256) chol_solve_single(const double* A, const double* W, int np, int nt,
                                                                const int* pnl_ptr, const int* pnl,
                                                                const int* bwd_ptr, const int* bwd, double* y) {
  __shared__ double v[kTile], x[kTile];
  const bool lead = (threadIdx.x & 3) == 0;
  const int row = threadIdx.x >> 2;
  for (int k = 0; k < nt; ++k) {
    const size_t kb = (size_t)k * kTile;
    if (threadIdx.x < kTile) v[threadIdx.x] = y[kb + threadIdx.x];
    __syncthreads();
    const double s = chol_rowdot(W + kb * kTile, kTile, v);
    if (lead) {
      x[row] = s;
      y[kb + row] = s;
    }
    __syncthreads();
    for (int p = pnl_ptr[k]; p < pnl_ptr[k + 1]; ++p) {
      const size_t ib = (size_t)pnl[p] * kTile;
      const double t = chol_rowdot(A + kb * np + ib, np, x);
      if (lead) y[ib + row] -= t;
    }
    __syncthreads();
  }
  for (int k = nt - 1; k >= 0; --k) {
    const size_t kb = (size_t)k * kTile;
    if (threadIdx.x < kTile) v[threadIdx.x] = y[kb + threadIdx.x];
    __syncthreads();
    const double s = chol_coldot(W + kb * kTile, kTile, v);
    if (lead) {
      x[row] = s;
      y[kb + row] = s;
    }
    __syncthreads();
    for (int p = bwd_ptr[k]; p < bwd_ptr[k + 1]; ++p) {
      const size_t ib = (size_t)bwd[p] * kTile;
      const double t = chol_coldot(A + ib * np + kb, np, x);
      if (lead) y[ib + row] -= t;
    }
    __syncthreads();
  }
}

// densify and factor: P.A holds L (lower tiles of the pattern), P.info the pivot flag
template <typename Real>
static int chol_factor(CholPlan& P, cudaStream_t st, const SysDev<Real>& S, long long* nl) {
  const int nnzb = S.nnzb;
  const int np = P.np, nt = P.nt;
  G2OC_CUDA_TRY(cudaFuncSetAttribute(chol_potrf, cudaFuncAttributeMaxDynamicSharedMemorySize, kPotrfSmem));
  G2OC_CUDA_TRY(cudaFuncSetAttribute(chol_trsm, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmem));
  G2OC_CUDA_TRY(cudaFuncSetAttribute(chol_gemm, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmem));
  G2OC_CUDA_TRY(cudaMemsetAsync(P.A.p, 0, P.A.bytes(), st));
  G2OC_CUDA_TRY(cudaMemsetAsync(P.info.p, 0, sizeof(int), st));
  const long long work = (long long)nnzb * P.bs * P.bs + (np - P.n);
  chol_densify<Real><<<(int)((work + 255) / 256), 256, 0, st>>>(S, P.bs, P.d_perm.p, P.n, np, P.A.p);
  chol_pivot_floor<double><<<1, 1024, 0, st>>>(P.A.p, np, P.n, P.floor.p);
  *nl += 1;
  if (P.single) {
    G2OC_CUDA_TRY(
        cudaFuncSetAttribute(chol_factor_single, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmemSingle));
    chol_factor_single<<<1, 256, kTileSmemSingle, st>>>(P.A.p, np, nt, P.d_pnl_ptr.p, P.d_pnl.p, P.d_upd_ptr.p,
                                                        P.d_upd.p, P.W.p, P.floor.p, P.info.p);
    *nl += 1;
  }
  for (int k = 0; k < (P.single ? 0 : nt); ++k) {
    chol_potrf<<<1, 256, kPotrfSmem, st>>>(P.A.p, np, k, P.W.p, P.floor.p, P.info.p);
    const int np_k = P.pnl_ptr[k + 1] - P.pnl_ptr[k];
    if (np_k > 0) chol_trsm<<<np_k, 256, kTileSmem, st>>>(P.A.p, np, k, P.d_pnl.p + P.pnl_ptr[k], P.W.p);
    const int nu = P.upd_ptr[k + 1] - P.upd_ptr[k];
    if (nu > 0) chol_gemm<<<nu, 256, kTileSmem, st>>>(P.A.p, np, k, P.d_upd.p + P.upd_ptr[k]);
    *nl += 1 + (np_k > 0) + (nu > 0);
  }
  const cudaError_t e1 = cudaGetLastError();
  if (e1 != cudaSuccess) {
    set_error("cholesky launch: %s", cudaGetErrorString(e1));
    return G2OC_ERR_CUDA;
  }
  return G2OC_OK;
}

// forward and backward substitution with the factor chol_factor left in P.A
// (a refinement's correction solve reuses it)
static int chol_resolve(CholPlan& P, cudaStream_t st, const double* rhs, double* xout, long long* nlaunch) {
  long long nl = 2;  // load_rhs, store_x
  const int np = P.np, nt = P.nt;
  chol_load_rhs<<<(np + 255) / 256, 256, 0, st>>>(rhs, P.d_perm.p, P.nb, P.bs, P.n, np, P.y.p);
  if (P.single) {
    chol_solve_single<<<1, 256, 0, st>>>(P.A.p, P.W.p, np, nt, P.d_pnl_ptr.p, P.d_pnl.p, P.d_bwd_ptr.p, P.d_bwd.p,
                                         P.y.p);
    nl += 1;
  }
  for (int k = 0; k < (P.single ? 0 : nt); ++k) {
    chol_fwd_diag<<<1, 256, 0, st>>>(P.W.p, k, P.y.p);
    const int np_k = P.pnl_ptr[k + 1] - P.pnl_ptr[k];
    if (np_k > 0) chol_fwd_update<<<np_k, 256, 0, st>>>(P.A.p, np, k, P.d_pnl.p + P.pnl_ptr[k], P.y.p);
    nl += 1 + (np_k > 0);
  }
  for (int k = (P.single ? -1 : nt - 1); k >= 0; --k) {
    chol_bwd_diag<<<1, 256, 0, st>>>(P.W.p, k, P.y.p);
    const int nbk = P.bwd_ptr[k + 1] - P.bwd_ptr[k];
    if (nbk > 0) chol_bwd_update<<<nbk, 256, 0, st>>>(P.A.p, np, k, P.d_bwd.p + P.bwd_ptr[k], P.y.p);
    nl += 1 + (nbk > 0);
  }
  chol_store_x<<<(P.n + 255) / 256, 256, 0, st>>>(P.y.p, P.d_perm.p, P.bs, P.n, xout);
  const cudaError_t e2 = cudaGetLastError();
  if (e2 != cudaSuccess) {
    set_error("cholesky solve launch: %s", cudaGetErrorString(e2));
    return G2OC_ERR_CUDA;
  }
  if (nlaunch) *nlaunch += nl;
  return G2OC_OK;
}

template <typename Real>
static int chol_solve(CholPlan& P, cudaStream_t st, const SysDev<Real>& S, const double* rhs, double* xout, int* ok,
                      long long* nlaunch) {
  long long nl = 2;  // densify + memsets
  G2OC_TRY(chol_factor<Real>(P, st, S, &nl));
  G2OC_TRY(chol_resolve(P, st, rhs, xout, &nl));
  if (nlaunch) *nlaunch += nl - 1;
  int info = 0;
  G2OC_CUDA_TRY(cudaMemcpyAsync(&info, P.info.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  G2OC_CUDA_TRY(cudaStreamSynchronize(st));
  *ok = info == 0;
  return G2OC_OK;
}

// ------------------------------------------------------------------------
// Selected inverse (the marginal covariances of
// LinearSolver::solvePattern, g2o/core/linear_solver.h:78-90, which g2o's
// Cholesky solvers compute with MarginalCovarianceCholesky,
// g2o/core/linear_solver.h:165-173 and g2o/core/marginal_covariance_cholesky.h:42-106). From H = L L^T
// and L^T Sigma = L^-1 (upper-triangular right side), for tile column J
// taken from last to first with S_J = {I > J : L(I,J) != 0} and
// Lh(I,J) = L(I,J) L(J,J)^-1:
//   Sigma(K,J) = - sum_{I in S_J} Sigma(K,I) Lh(I,J)          (K in S_J)
//   Sigma(J,J) = L(J,J)^-T L(J,J)^-1 - sum_{I in S_J} Lh(I,J)^T Sigma(I,J)
// Every Sigma(K,I) needed lies in the filled tile pattern (S_J is a clique
// of it), so only the pattern's tiles are computed: the tile form of the
// Takahashi recurrences. Sigma is kept in a dense column-major np x np
// buffer: lower tiles and full diagonal tiles. L's panel tiles are
// overwritten by Lh.

// W = L(J,J)^-1 (lower), column c by thread c: forward substitution of e_c
static __global__ void __launch_bounds__(256) selinv_tri_inv(const double* A, int np, int J, double* W) {
  extern __shared__ double sm_ti[];
  double (*L)[kTile + 1] = reinterpret_cast<double (*)[kTile + 1]>(sm_ti);
  double (*X)[kTile + 1] = reinterpret_cast<double (*)[kTile + 1]>(sm_ti + kTile * (kTile + 1));
  const size_t jb = (size_t)J * kTile;
  for (int e = threadIdx.x; e < kTile * kTile; e += blockDim.x) {
    const int r = e % kTile, c = e / kTile;
    L[r][c] = r >= c ? A[(jb + c) * np + jb + r] : 0.0;
  }
  __syncthreads();
  const int c = threadIdx.x;
  if (c < kTile) {
    for (int r = 0; r < c; ++r) X[r][c] = 0.0;
    for (int r = c; r < kTile; ++r) {
      double v = r == c ? 1.0 : 0.0;
      for (int t = c; t < r; ++t) v -= L[r][t] * X[t][c];
      X[r][c] = v / L[r][r];
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < kTile * kTile; e += blockDim.x) {
    const int r = e % kTile, cc = e / kTile;
    W[cc * kTile + r] = X[r][cc];
  }
}

// Lh(I,J) = L(I,J) W for the listed tiles I, in place
static __global__ void __launch_bounds__(256) selinv_panel(double* A, int np, int J, const int* tiles,
                                                           const double* W) {
  extern __shared__ double sm_sp[];
  double (*X)[kTile + 1] = reinterpret_cast<double (*)[kTile + 1]>(sm_sp);
  double (*Wt)[kTile + 1] = reinterpret_cast<double (*)[kTile + 1]>(sm_sp + kTile * (kTile + 1));
  const size_t jb = (size_t)J * kTile, ib = (size_t)tiles[blockIdx.x] * kTile;
  for (int e = threadIdx.x; e < kTile * kTile; e += blockDim.x) {
    const int r = e % kTile, c = e / kTile;
    X[r][c] = A[(jb + c) * np + ib + r];
    Wt[r][c] = W[c * kTile + r];
  }
  __syncthreads();
  const int tr = threadIdx.x % 16, tc = threadIdx.x / 16;
  double acc[4][4] = {};
  for (int t = 0; t < kTile; ++t) {
    double x[4], y[4];
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      x[a] = X[tr + 16 * a][t];
      y[a] = Wt[t][tc + 16 * a];
    }
#pragma unroll
    for (int a = 0; a < 4; ++a)
#pragma unroll
      for (int b = 0; b < 4; ++b) acc[a][b] += x[a] * y[b];
  }
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) A[(jb + tc + 16 * b) * np + ib + tr + 16 * a] = acc[a][b];
}

// Sigma tile (K, I) of the stored lower/diagonal tiles, into smem as T[r][c]
__device__ __forceinline__ void selinv_load_sigma(const double* Sg, int np, int K, int I,
                                                  double (*T)[kTile + 1]) {
  const size_t kb = (size_t)K * kTile, ib = (size_t)I * kTile;
  if (K >= I) {
    for (int e = threadIdx.x; e < kTile * kTile; e += blockDim.x) {
      const int r = e % kTile, c = e / kTile;
      T[r][c] = Sg[(ib + c) * np + kb + r];
    }
  } else {  // Sigma(K,I) = Sigma(I,K)^T
    for (int e = threadIdx.x; e < kTile * kTile; e += blockDim.x) {
      const int c = e % kTile, r = e / kTile;
      T[r][c] = Sg[(kb + r) * np + ib + c];
    }
  }
}

// Sigma(K,J) = - sum_I Sigma(K,I) Lh(I,J), one CTA per K in S_J
static __global__ void __launch_bounds__(256) selinv_offdiag(const double* A, double* Sg, int np, int J,
                                                             const int* tiles, int ntiles) {
  extern __shared__ double sm_so[];
  double (*Sk)[kTile + 1] = reinterpret_cast<double (*)[kTile + 1]>(sm_so);
  double (*Lh)[kTile + 1] = reinterpret_cast<double (*)[kTile + 1]>(sm_so + kTile * (kTile + 1));
  const int K = tiles[blockIdx.x];
  const size_t jb = (size_t)J * kTile;
  const int tr = threadIdx.x % 16, tc = threadIdx.x / 16;
  double acc[4][4] = {};
  for (int q = 0; q < ntiles; ++q) {
    const int I = tiles[q];
    const size_t ib = (size_t)I * kTile;
    __syncthreads();
    selinv_load_sigma(Sg, np, K, I, Sk);
    for (int e = threadIdx.x; e < kTile * kTile; e += blockDim.x) {
      const int r = e % kTile, c = e / kTile;
      Lh[r][c] = A[(jb + c) * np + ib + r];
    }
    __syncthreads();
    for (int t = 0; t < kTile; ++t) {
      double x[4], y[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        x[a] = Sk[tr + 16 * a][t];
        y[a] = Lh[t][tc + 16 * a];
      }
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] += x[a] * y[b];
    }
  }
  const size_t kb = (size_t)K * kTile;
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) Sg[(jb + tc + 16 * b) * np + kb + tr + 16 * a] = -acc[a][b];
}

// Sigma(J,J) = W^T W - sum_I Lh(I,J)^T Sigma(I,J), symmetrized
static __global__ void __launch_bounds__(256) selinv_diag(const double* A, double* Sg, int np, int J,
                                                          const int* tiles, int ntiles, const double* W) {
  extern __shared__ double sm_sd[];
  double (*P0)[kTile + 1] = reinterpret_cast<double (*)[kTile + 1]>(sm_sd);
  double (*P1)[kTile + 1] = reinterpret_cast<double (*)[kTile + 1]>(sm_sd + kTile * (kTile + 1));
  const size_t jb = (size_t)J * kTile;
  const int tr = threadIdx.x % 16, tc = threadIdx.x / 16;
  double acc[4][4] = {};
  for (int q = -1; q < ntiles; ++q) {
    __syncthreads();
    if (q < 0) {
      for (int e = threadIdx.x; e < kTile * kTile; e += blockDim.x) {
        const int r = e % kTile, c = e / kTile;
        P0[r][c] = W[c * kTile + r];
        P1[r][c] = -W[c * kTile + r];
      }
    } else {
      const size_t ib = (size_t)tiles[q] * kTile;
      for (int e = threadIdx.x; e < kTile * kTile; e += blockDim.x) {
        const int r = e % kTile, c = e / kTile;
        P0[r][c] = A[(jb + c) * np + ib + r];   // Lh(I,J)
        P1[r][c] = Sg[(jb + c) * np + ib + r];  // Sigma(I,J)
      }
    }
    __syncthreads();
    // acc -= P0^T P1
    for (int t = 0; t < kTile; ++t) {
      double x[4], y[4];
#pragma unroll
      for (int a = 0; a < 4; ++a) {
        x[a] = P0[t][tr + 16 * a];
        y[a] = P1[t][tc + 16 * a];
      }
#pragma unroll
      for (int a = 0; a < 4; ++a)
#pragma unroll
        for (int b = 0; b < 4; ++b) acc[a][b] -= x[a] * y[b];
    }
  }
  __syncthreads();
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int b = 0; b < 4; ++b) P0[tr + 16 * a][tc + 16 * b] = acc[a][b];
  __syncthreads();
  for (int e = threadIdx.x; e < kTile * kTile; e += blockDim.x) {
    const int r = e % kTile, c = e / kTile;
    Sg[(jb + c) * np + jb + r] = 0.5 * (P0[r][c] + P0[c][r]);
  }
}

// requested blocks (row, col) of H^-1, row-major bs x bs each
static __global__ void selinv_gather(const double* Sg, int np, const int* perm, int bs, const int2* req, int nreq,
                                     double* out) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const int per = bs * bs;
  if (t >= (long long)nreq * per) return;
  const int q = (int)(t / per), e = (int)(t % per);
  const int i = perm[req[q].x] * bs + e / bs, j = perm[req[q].y] * bs + e % bs;
  out[t] = (i / kTile >= j / kTile) ? Sg[(size_t)j * np + i] : Sg[(size_t)i * np + j];
}

// the requested blocks of S^-1 (pairs (row, col) of block indices, covered by
// the plan's extra pairs) into out (device, nreq * bs * bs)
template <typename Real>
static int chol_selected_inverse(CholPlan& P, cudaStream_t st, const SysDev<Real>& S, const int2* d_req, int nreq,
                                 double* d_out, int* ok, long long* nlaunch) {
  long long nl = 2;
  const int np = P.np, nt = P.nt;
  G2OC_TRY(chol_factor<Real>(P, st, S, &nl));
  int info = 0;
  G2OC_CUDA_TRY(cudaMemcpyAsync(&info, P.info.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  G2OC_CUDA_TRY(cudaStreamSynchronize(st));
  *ok = info == 0;
  if (!*ok) return G2OC_OK;
  DBuf<double> Sg, W;
  G2OC_TRY(Sg.alloc((size_t)np * np));
  G2OC_TRY(W.alloc((size_t)kTile * kTile));
  G2OC_CUDA_TRY(cudaMemsetAsync(Sg.p, 0, Sg.bytes(), st));
  G2OC_CUDA_TRY(cudaFuncSetAttribute(selinv_tri_inv, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmem));
  G2OC_CUDA_TRY(cudaFuncSetAttribute(selinv_panel, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmem));
  G2OC_CUDA_TRY(cudaFuncSetAttribute(selinv_offdiag, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmem));
  G2OC_CUDA_TRY(cudaFuncSetAttribute(selinv_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, kTileSmem));
  for (int J = nt - 1; J >= 0; --J) {
    const int nj = P.pnl_ptr[J + 1] - P.pnl_ptr[J];
    const int* tl = P.d_pnl.p + P.pnl_ptr[J];
    selinv_tri_inv<<<1, 256, kTileSmem, st>>>(P.A.p, np, J, W.p);
    if (nj > 0) {
      selinv_panel<<<nj, 256, kTileSmem, st>>>(P.A.p, np, J, tl, W.p);
      selinv_offdiag<<<nj, 256, kTileSmem, st>>>(P.A.p, Sg.p, np, J, tl, nj);
    }
    selinv_diag<<<1, 256, kTileSmem, st>>>(P.A.p, Sg.p, np, J, tl, nj, W.p);
    nl += 2 + 2 * (nj > 0);
  }
  const long long work = (long long)nreq * P.bs * P.bs;
  if (work > 0) selinv_gather<<<(int)((work + 255) / 256), 256, 0, st>>>(Sg.p, np, P.d_perm.p, P.bs, d_req, nreq, d_out);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("selected inverse launch: %s", cudaGetErrorString(e));
    return G2OC_ERR_CUDA;
  }
  G2OC_CUDA_TRY(cudaStreamSynchronize(st));
  if (nlaunch) *nlaunch += nl;
  return G2OC_OK;
}

}  // namespace g2oc
