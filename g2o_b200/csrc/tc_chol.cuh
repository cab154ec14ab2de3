// tc_chol.cuh -- dense Cholesky of a nearly full reduced camera system on the
// 5th-generation tensor cores: the role of LinearSolverDense
// (g2o/solvers/dense/linear_solver_dense.h:57-105) when the Schur complement
// of a bundle adjustment is dense enough that a direct factorization is
// GEMM-shaped.
//
// Storage: the system is expanded into a dense FP32 column-major np x np
// matrix (np a multiple of 128; the padding is the identity), lower triangle.
// Right-looking blocked factorization in 128 x 128 tiles; per step k:
//   tc_potrf:  the diagonal tile is factored in FP64 in shared memory (one
//              CTA) and W(k) = L(k,k)^-1 is formed; L(k,k) and W(k) are
//              stored in FP32;
//   tc_tiles:  panel L(i,k) = A(i,k) W(k)^T and trailing update
//              A(i,j) -= L(i,k) L(j,k)^T, one CTA per 128 x 128 output tile,
//              as tcgen05.mma kind::tf32 products (M = N = 128, K = 8 per
//              instruction) issued by one thread, operands in shared memory,
//              the FP32 accumulator in tensor memory (128 lanes x 128
//              columns), read back with tcgen05.ld for the epilogue.
// Each operand value x is split into hi = tf32(x) and lo = tf32(x - hi) and
// a product is formed as hi*hi + hi*lo + lo*hi (three MMAs per K step), which
// gives FP32-level accuracy; accumulation is FP32 in tensor memory.
// Solves use the factor in FP64 arithmetic: y(k) = W(k) (y(k)) then the
// updates of the other tiles, forward and backward. The caller refines the
// solution on its true FP64 residual.
//
// Shared-memory operand layout (no swizzle, K-major canonical form of the
// UMMA descriptor): element (i, j) of a 128 (M or N) x 64 (K) FP32 tile at
// byte (i % 8) * 16 + (j % 4) * 4 + (i / 8) * 128 + (j / 4) * 2048: core
// matrices of 8 rows x 4 K values (16 bytes per row, 128 bytes), row groups
// 128 bytes apart (stride byte offset), K groups 2048 bytes apart (leading
// byte offset); one MMA (K = 8) spans two K groups. (The MN-major form of
// the descriptor gave a zero product for kind::tf32 on this hardware, so the
// operands are transposed into K-major order while they are staged.)
#pragma once

#include <cstdint>
#include <vector>

#include "g2oc_internal.h"
#include "pcg_persistent.cuh"
#include "tile_potrf.cuh"

namespace g2oc {

constexpr int kTc = 128;           // tile edge
constexpr int kTcK = 64;           // K per staged chunk
constexpr int kTcOpBytes = kTc * kTcK * 4;        // one operand tile (hi or lo): 32 KB
constexpr int kTcSmem = 4 * kTcOpBytes + 1024;    // A hi/lo, B hi/lo, barrier and TMEM address
constexpr long long kTcSpinLimit = 1ll << 26;     // bounded waits (tens of ms at worst)

// ------------------------------------------------------------ PTX helpers
__device__ __forceinline__ uint32_t tc_smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ float tc_tf32(float x) {
  uint32_t r;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
  return __uint_as_float(r);
}

// UMMA shared-memory descriptor: start address, leading / stride byte
// offsets (16-byte units), version 1, no swizzle
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)((lbo >> 4) & 0x3FFFu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// instruction descriptor: kind::tf32, D in FP32, A and B TF32, both K-major,
// N = 128 (bits 17-22: N >> 3), M = 128 (bits 24-28: M >> 4)
constexpr uint32_t kTcIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(kTc >> 3) << 17) |
                              ((uint32_t)(kTc >> 4) << 24);

__device__ __forceinline__ void tc_mma(uint32_t tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n" ::"r"(tmem),
      "l"(a), "l"(b), "r"(kTcIdesc), "r"(accumulate));
}

__device__ __forceinline__ void tc_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar) : "memory");
}

__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }

// wait for phase `parity` of the barrier, at most kTcSpinLimit polls; false
// when the limit ran out
__device__ __forceinline__ bool tc_wait(uint32_t mbar, uint32_t parity) {
  for (long long it = 0; it < kTcSpinLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 16 consecutive FP32 accumulator columns of this thread's TMEM lane
__device__ __forceinline__ void tc_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
        "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int t = 0; t < 16; ++t) v[t] = __uint_as_float(r[t]);
}

// stage the two 128 (MN) x 64 (K) FP32 operand sub-tiles of a tile product
// (column j of a sub-tile at G + j * ld) as hi / lo TF32 parts in the K-major
// layout above. One core matrix (8 rows x 4 K values, 32 consecutive words
// of shared memory) per warp instruction: lane l takes row 8 mg + l / 4 and
// K value 4 kg + l % 4, so each store covers the 32 banks once and each load
// reads four 32-byte column runs. Each warp takes 64 core matrices of each
// operand, 32 of each per round with all 64 loads in flight (the loads are
// what the staging waits on).
__device__ __forceinline__ void tc_stage_cm(const float* G, size_t ld, int cm, int lane, float& x) {
  const int mg = cm & 15, kg = cm >> 4;
  x = G[(size_t)(4 * kg + (lane & 3)) * ld + 8 * mg + (lane >> 2)];
}
__device__ __forceinline__ void tc_store_cm(unsigned char* hi, unsigned char* lo, int cm, int lane, float x) {
  const int mg = cm & 15, kg = cm >> 4;
  const uint32_t off = (uint32_t)mg * 128 + (uint32_t)kg * 2048 + (uint32_t)lane * 4;
  const float h = tc_tf32(x);
  *reinterpret_cast<float*>(hi + off) = h;
  *reinterpret_cast<float*>(lo + off) = tc_tf32(x - h);
}
__device__ __forceinline__ void tc_stage2(const float* GA, size_t lda, const float* GB, size_t ldb, unsigned char* a_hi,
                                          unsigned char* a_lo, unsigned char* b_hi, unsigned char* b_lo) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;  // 4 warps
#pragma unroll 1
  for (int rnd = 0; rnd < 2; ++rnd) {
    const int cm0 = warp * 64 + rnd * 32;
    float xa[32], xb[32];
#pragma unroll
    for (int u = 0; u < 32; ++u) {
      tc_stage_cm(GA, lda, cm0 + u, lane, xa[u]);
      tc_stage_cm(GB, ldb, cm0 + u, lane, xb[u]);
    }
#pragma unroll
    for (int u = 0; u < 32; ++u) {
      tc_store_cm(a_hi, a_lo, cm0 + u, lane, xa[u]);
      tc_store_cm(b_hi, b_lo, cm0 + u, lane, xb[u]);
    }
  }
}

// ------------------------------------------------------------ tile products
// One CTA (128 threads, one warpgroup) per output tile:
//   panel  (ij.y < 0):  L(i,k) = A(i,k) W(k)^T          (ij.x = i)
//   update (ij.y >= 0): A(i,j) -= L(i,k) L(j,k)^T       (i = ij.x, j = ij.y)
// P = X Y^T with X the 128 x 128 left operand and Y the right one (both
// column-major, leading dimension ldx / ldy), formed over two K chunks of 64.
// *err is set when a bounded wait gives up (the tile is then left unchanged).
static __global__ void __launch_bounds__(128, 1)
    tc_tiles(float* A, int np, int k, const int2* list, const float* Wk, int* err) {
  extern __shared__ __align__(1024) unsigned char tc_smem[];
  unsigned char* a_hi = tc_smem;
  unsigned char* a_lo = tc_smem + kTcOpBytes;
  unsigned char* b_hi = tc_smem + 2 * kTcOpBytes;
  unsigned char* b_lo = tc_smem + 3 * kTcOpBytes;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(tc_smem + 4 * kTcOpBytes);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(tc_smem + 4 * kTcOpBytes + 64);
  const int2 ij = list[blockIdx.x];
  const bool panel = ij.y < 0;
  const size_t kb = (size_t)k * kTc;
  const float* X = A + kb * np + (size_t)ij.x * kTc;           // A(i,k) or L(i,k)
  const float* Y = panel ? Wk : A + kb * np + (size_t)ij.y * kTc;  // W(k) or L(j,k)
  const size_t ldy = panel ? (size_t)kTc : (size_t)np;
  float* D = A + (panel ? kb : (size_t)ij.y * kTc) * np + (size_t)ij.x * kTc;
  const int warp = threadIdx.x >> 5;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(tc_smem_addr(tmem_slot)),
                 "r"(kTc));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(tc_smem_addr(mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = *tmem_slot;
  const uint32_t mb = tc_smem_addr(mbar);
  bool ok = true;
  for (int ch = 0; ch < kTc / kTcK && ok; ++ch) {
    tc_stage2(X + (size_t)ch * kTcK * np, np, Y + (size_t)ch * kTcK * ldy, ldy, a_hi, a_lo, b_hi, b_lo);
    // the generic-proxy stores must be visible to the tensor core's reads
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (threadIdx.x == 0) {
      tc_fence_after();
      const uint32_t ah = tc_smem_addr(a_hi), al = tc_smem_addr(a_lo);
      const uint32_t bh = tc_smem_addr(b_hi), bl = tc_smem_addr(b_lo);
#pragma unroll
      for (int kg = 0; kg < kTcK / 8; ++kg) {
        const uint32_t o = (uint32_t)kg * 4096;
        tc_mma(tmem, tc_desc(ah + o, 2048, 128), tc_desc(bh + o, 2048, 128), (ch > 0 || kg > 0) ? 1u : 0u);
        tc_mma(tmem, tc_desc(ah + o, 2048, 128), tc_desc(bl + o, 2048, 128), 1u);
        tc_mma(tmem, tc_desc(al + o, 2048, 128), tc_desc(bh + o, 2048, 128), 1u);
      }
      tc_commit(mb);
    }
    // every thread waits for the products of this chunk before the operand
    // tiles are overwritten (or the accumulator is read); the outcome is
    // made uniform over the CTA so every thread takes the same path
    ok = __syncthreads_and(tc_wait(mb, (uint32_t)(ch & 1)) ? 1 : 0) != 0;
  }
  tc_fence_after();
  if (!ok) {
    if (threadIdx.x == 0) atomicExch(err, 1);
  } else {
    // epilogue: thread (warp w, lane t) holds row m = 32 w + t of P; the
    // trailing update's old values of the row are loaded 64 at a time, all
    // in flight together
    const int m = threadIdx.x;
    const uint32_t lane_base = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll 1
    for (int h = 0; h < kTc; h += 64) {
      float dold[64];
      if (!panel) {
#pragma unroll
        for (int c = 0; c < 64; ++c) dold[c] = D[(size_t)(h + c) * np + m];
      }
#pragma unroll
      for (int c0 = 0; c0 < 64; c0 += 16) {
        float v[16];
        tc_ld16(lane_base + (uint32_t)(h + c0), v);
#pragma unroll
        for (int t = 0; t < 16; ++t) {
          float* d = D + (size_t)(h + c0 + t) * np + m;
          *d = panel ? v[t] : dold[c0 + t] - v[t];
        }
      }
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(kTc));
  }
}

// ------------------------------------------------------------ diagonal tile
// Factor the diagonal tile k in FP64 (lower), write L(k,k) back in FP32 and
// W(k) = L(k,k)^-1 (FP32, column-major 128 x 128, zero above the diagonal)
// to Wk. The 128 x 128 tile is taken as 2 x 2 blocks of 64 (256 threads):
//   L11 W11 = chol(A11)                    tile_potrf_inv_blk64
//   L21 = A21 W11^T                        FP64 tensor-core product
//   L22 W22 = chol(A22 - L21 L21^T)        product, then tile_potrf_inv_blk64
//   W21 = -W22 (L21 W11)                   two products
// A non-positive pivot sets *info (the pivot is replaced by 1 so the
// arithmetic stays finite).
constexpr int kTcLd = 68;                    // operand blocks, as tile_dmma64 reads them
constexpr int kTcBlk = 64 * kTcLd;           // doubles per operand block
constexpr int kTcTri = 64 * 65;              // doubles per diagonal block (leading dimension 65)
constexpr size_t kTcPotrfSmem = (size_t)(2 * kTcTri + 3 * kTcBlk + 768) * sizeof(double);

static __global__ void __launch_bounds__(256, 1) tc_potrf(float* A, int np, int k, float* Wk, const double* floor,
                                                           int* info) {
  extern __shared__ double tcp_smem[];
  double* T1 = tcp_smem;                // A11 -> L11 (ld 65)
  double* T2 = T1 + kTcTri;             // A22 -> L22
  double* X = T2 + kTcTri;              // A21 -> L21 -> L21 W11 (ld kTcLd)
  double* W1 = X + kTcBlk;              // W11 (column-major, ld kTcLd)
  double* W2 = W1 + kTcBlk;             // W22
  double* scratch = W2 + kTcBlk;        // the blocked factorization's staging (768 doubles)
  const size_t kb = (size_t)k * kTc;
  for (int e = threadIdx.x; e < 64 * 64; e += blockDim.x) {
    const int i = e % 64, j = e / 64;
    if (i >= j) {
      T1[i * 65 + j] = (double)A[(kb + j) * np + kb + i];
      T2[i * 65 + j] = (double)A[(kb + 64 + j) * np + kb + 64 + i];
    }
    X[i * kTcLd + j] = (double)A[(kb + j) * np + kb + 64 + i];
  }
  __syncthreads();
  int bad = 0;
  const double fl = *floor;
  tile_potrf_inv_blk64(T1, 65, W1, kTcLd, &bad, fl, scratch);
  double acc[2][4][2];
  // L21 = A21 W11^T (Y(j, t) = W11(j, t) at W1[t * ld + j])
  tile_dmma64<false, true>(X, W1, kTcLd, acc);
  __syncthreads();
#pragma unroll
  for (int u = 0; u < 2; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int r = tile_dmma64_row(u), c = tile_dmma64_col(v, e);
        X[r * kTcLd + c] = acc[u][v][e];
        A[(kb + c) * np + kb + 64 + r] = (float)acc[u][v][e];
      }
  __syncthreads();
  // A22 -= L21 L21^T
  tile_dmma64<false, false>(X, X, kTcLd, acc);
#pragma unroll
  for (int u = 0; u < 2; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int r = tile_dmma64_row(u), c = tile_dmma64_col(v, e);
        if (r >= c) T2[r * 65 + c] -= acc[u][v][e];
      }
  __syncthreads();
  tile_potrf_inv_blk64(T2, 65, W2, kTcLd, &bad, fl, scratch);
  // M = L21 W11 (Y(c, t) = W11(t, c) at W1[c * ld + t]), into X
  tile_dmma64<false, false>(X, W1, kTcLd, acc);
  __syncthreads();
#pragma unroll
  for (int u = 0; u < 2; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
      for (int e = 0; e < 2; ++e) X[tile_dmma64_row(u) * kTcLd + tile_dmma64_col(v, e)] = acc[u][v][e];
  __syncthreads();
  // W21 = -W22 M (X(r, t) = W22(r, t) at W2[t * ld + r]; Y(c, t) = M(t, c) at X[t * ld + c])
  tile_dmma64<true, true>(W2, X, kTcLd, acc);
#pragma unroll
  for (int u = 0; u < 2; ++u)
#pragma unroll
    for (int v = 0; v < 4; ++v)
#pragma unroll
      for (int e = 0; e < 2; ++e) {
        const int r = tile_dmma64_row(u), c = tile_dmma64_col(v, e);
        Wk[(size_t)c * kTc + 64 + r] = (float)(-acc[u][v][e]);
      }
  if (threadIdx.x == 0 && bad) atomicExch(info, 1);
  for (int e = threadIdx.x; e < 64 * 64; e += blockDim.x) {
    const int i = e % 64, j = e / 64;
    if (i >= j) {
      A[(kb + j) * np + kb + i] = (float)T1[i * 65 + j];
      A[(kb + 64 + j) * np + kb + 64 + i] = (float)T2[i * 65 + j];
    }
    Wk[(size_t)j * kTc + i] = (float)W1[j * kTcLd + i];
    Wk[(size_t)(64 + j) * kTc + 64 + i] = (float)W2[j * kTcLd + i];
    Wk[(size_t)(64 + j) * kTc + i] = 0.0f;
  }
}

// ------------------------------------------------------------ solves
// y(k) = W(k) y(k) (128 threads, FP64)
static __global__ void tc_apply_w(const float* Wk, double* y, int k, bool transpose) {
  __shared__ double v[kTc];
  const int r = threadIdx.x;
  v[r] = y[(size_t)k * kTc + r];
  __syncthreads();
  double acc = 0.0;
  if (!transpose) {
    for (int c = 0; c <= r; ++c) acc += (double)Wk[(size_t)c * kTc + r] * v[c];
  } else {
    for (int c = r; c < kTc; ++c) acc += (double)Wk[(size_t)r * kTc + c] * v[c];
  }
  y[(size_t)k * kTc + r] = acc;
}

// forward update: y(i) -= L(i,k) y(k) for the tiles i > k (CTA per tile,
// thread per row, columns in order)
static __global__ void tc_fwd_update(const float* A, int np, int k, double* y) {
  __shared__ double v[kTc];
  const int i = k + 1 + blockIdx.x, r = threadIdx.x;
  v[r] = y[(size_t)k * kTc + r];
  __syncthreads();
  const float* L = A + (size_t)k * kTc * np + (size_t)i * kTc + r;
  double acc = 0.0;
  for (int c = 0; c < kTc; ++c) acc += (double)L[(size_t)c * np] * v[c];
  y[(size_t)i * kTc + r] -= acc;
}

// backward update: y(l) -= L(k,l)^T x(k) for the tiles l < k (CTA per tile;
// warp per group of columns, lanes over the rows, fixed-order shuffle sums)
static __global__ void tc_bwd_update(const float* A, int np, int k, double* y) {
  __shared__ double v[kTc];
  const int l = blockIdx.x;
  v[threadIdx.x] = y[(size_t)k * kTc + threadIdx.x];
  __syncthreads();
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int c = warp; c < kTc; c += blockDim.x >> 5) {
    const float* col = A + ((size_t)l * kTc + c) * np + (size_t)k * kTc;
    double acc = 0.0;
    for (int r = lane; r < kTc; r += 32) acc += (double)col[r] * v[r];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) y[(size_t)l * kTc + c] -= acc;
  }
}

// Both substitutions as one cooperative launch each (dir 0: y = L^-1 y,
// dir 1: y = L^-T y), one grid barrier per tile step instead of two launches:
// every CTA with work in step k stages W(k) in shared memory (FP32, columns
// 129 floats apart: conflict-free in both orientations), forms
// v = W(k) y_k (or W(k)^T y_k) in FP64 (thread per row, columns in order), CTA
// 0 stores it as the new y_k after the step's barrier, and the CTAs take the
// step's updates in units
// of 32 rows of one tile: y_i -= L(i,k) v for the tiles i > k (dir 0), or
// 32 columns of one tile: y_l -= L(k,l)^T v for l < k (dir 1), four threads
// per 128-long dot product (32 terms each, a fixed xor tree). A barrier
// that runs out of its spin limit sets the state's error flag and the
// kernel returns (the host reports a timeout).
constexpr int kTcSolveThreads = 128;
constexpr size_t kTcSolveSmem = (size_t)kTc * (kTc + 1) * sizeof(float);

static __global__ void __launch_bounds__(kTcSolveThreads) tc_solve_coop(const float* A, const float* W, int np, int nt,
                                                                        double* y, PcgState* st, unsigned barrier_extra,
                                                                        int dir) {
  extern __shared__ float tcs_smem[];
  float* Ws = tcs_smem;  // W(k)(r, c) at Ws[c * 129 + r]
  __shared__ double vin[kTc], v[kTc];
  unsigned gen = grid_gen_start(st);
  const int tid = threadIdx.x;
  for (int s = 0; s < nt; ++s) {
    const int k = dir == 0 ? s : nt - 1 - s;
    const size_t kb = (size_t)k * kTc;
    const int nunits = 4 * (dir == 0 ? nt - 1 - k : k);
    // the previous step's tile, stored only now: every CTA has read its old
    // value (before the barrier), and no later step of this direction reads it
    if (s > 0 && blockIdx.x == 0) y[(size_t)(dir == 0 ? k - 1 : k + 1) * kTc + tid] = v[tid];
    if (blockIdx.x == 0 || (int)blockIdx.x < nunits) {
      const float* Wk = W + kb * kTc;
      for (int q = tid; q < kTc * kTc / 4; q += kTcSolveThreads) {
        const int c = q >> 5, r4 = (q & 31) * 4;
        const float4 w4 = *reinterpret_cast<const float4*>(Wk + (size_t)c * kTc + r4);
        Ws[c * 129 + r4] = w4.x;
        Ws[c * 129 + r4 + 1] = w4.y;
        Ws[c * 129 + r4 + 2] = w4.z;
        Ws[c * 129 + r4 + 3] = w4.w;
      }
      vin[tid] = y[kb + tid];
      __syncthreads();
      double acc = 0.0;
      if (dir == 0) {
        for (int c = 0; c <= tid; ++c) acc += (double)Ws[c * 129 + tid] * vin[c];
      } else {
        for (int c = tid; c < kTc; ++c) acc += (double)Ws[tid * 129 + c] * vin[c];
      }
      v[tid] = acc;
      __syncthreads();
      const int q4 = tid & 3, rr = tid >> 2;
      for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        const int slab = u & 3, idx = u >> 2;
        double t = 0.0;
        if (dir == 0) {
          const size_t ib = (size_t)(k + 1 + idx) * kTc + slab * 32 + rr;  // row of y and of L(i,k)
          const float* L = A + kb * np + ib;                                 // L(i,k)(row, c) at L[c * np]
          float x[32];
#pragma unroll
          for (int c = 0; c < 32; ++c) x[c] = L[(size_t)(q4 * 32 + c) * np];
#pragma unroll
          for (int c = 0; c < 32; ++c) t += (double)x[c] * v[q4 * 32 + c];
          t += __shfl_xor_sync(0xffffffffu, t, 1);
          t += __shfl_xor_sync(0xffffffffu, t, 2);
          if (q4 == 0) y[ib] -= t;
        } else {
          const size_t lc = (size_t)idx * kTc + slab * 32 + rr;  // column of L(k,l), row of y
          const float* L = A + lc * np + kb;                       // L(k,l)(t, col) at L[t]
          float x[32];
#pragma unroll
          for (int c = 0; c < 32; ++c) x[c] = L[q4 * 32 + c];
#pragma unroll
          for (int c = 0; c < 32; ++c) t += (double)x[c] * v[q4 * 32 + c];
          t += __shfl_xor_sync(0xffffffffu, t, 1);
          t += __shfl_xor_sync(0xffffffffu, t, 2);
          if (q4 == 0) y[lc] -= t;
        }
      }
    }
    if (!grid_barrier(st, gen, barrier_extra)) return;
  }
  if (blockIdx.x == 0) y[(size_t)(dir == 0 ? nt - 1 : 0) * kTc + tid] = v[tid];
}

// ------------------------------------------------------------ expansion
// dense FP32 column-major lower triangle of the system held in the dense
// 96 x 96 tiles of the tile PCG (kTileBlocks 6x6 blocks per tile edge; tile
// (R, C), R <= C, row-major; tile_index[R * nbt + C] = its index or -1),
// identity on the padding (rows n .. np-1)
static __global__ void tc_expand_tiles(const float* tiles, const int* tile_index, int nbt, int n, int np, float* A) {
  constexpr int TS = kTileBlocks * 6;
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)np * np) return;
  const int j = (int)(t / np), i = (int)(t % np);  // column j, row i; only i >= j is written and read
  if (i < j) return;
  float v = 0.0f;
  if (i < n) {
    // S(i, j) = S(j, i): row j, column i of the upper storage
    const int R = j / TS, C = i / TS;
    const int ti = tile_index[R * nbt + C];
    if (ti >= 0) v = tiles[(size_t)ti * TS * TS + (size_t)(j % TS) * TS + (i % TS)];
  } else if (i == j) {
    v = 1.0f;
  }
  A[t] = v;
}

static __global__ void tc_load_rhs(const double* b, int n, int np, double* y) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < np) y[t] = t < n ? b[t] : 0.0;
}

// ------------------------------------------------------------ host driver
struct TcChol {
  int n = 0, np = 0, nt = 0, nbt = 0;
  DBuf<float> A, W;
  DBuf<double> y;
  DBuf<int> info, err, tile_index;
  DBuf<double> floor;  // pivot floor of the current factorization
  DBuf<PcgState> sync;  // grid barrier of the cooperative substitutions
  DBuf<int2> lists;                 // per step: panel tiles then update pairs
  std::vector<int> list_ptr;        // per step: [panel start, update start, end)
};

static int tc_chol_plan(TcChol& P, int n, int nbt_tiles, const std::vector<int32_t>& tile_ij, cudaStream_t st) {
  P.n = n;
  P.nt = (n + kTc - 1) / kTc;
  P.np = P.nt * kTc;
  P.nbt = nbt_tiles;
  std::vector<int> index((size_t)nbt_tiles * nbt_tiles, -1);
  for (size_t t = 0; t < tile_ij.size() / 2; ++t) index[(size_t)tile_ij[2 * t] * nbt_tiles + tile_ij[2 * t + 1]] = (int)t;
  G2OC_TRY(P.tile_index.upload(index, st));
  std::vector<int2> L;
  P.list_ptr.assign(2 * P.nt + 1, 0);
  for (int k = 0; k < P.nt; ++k) {
    P.list_ptr[2 * k] = (int)L.size();
    for (int i = k + 1; i < P.nt; ++i) L.push_back(make_int2(i, -1));
    P.list_ptr[2 * k + 1] = (int)L.size();
    for (int j = k + 1; j < P.nt; ++j)
      for (int i = j; i < P.nt; ++i) L.push_back(make_int2(i, j));
  }
  P.list_ptr[2 * P.nt] = (int)L.size();
  if (L.empty()) L.push_back(make_int2(0, 0));
  G2OC_TRY(P.lists.upload(L, st));
  G2OC_TRY(P.A.alloc((size_t)P.np * P.np));
  G2OC_TRY(P.W.alloc((size_t)P.nt * kTc * kTc));
  G2OC_TRY(P.y.alloc(P.np));
  G2OC_TRY(P.info.alloc(1));
  G2OC_TRY(P.err.alloc(1));
  G2OC_TRY(P.floor.alloc(1));
  G2OC_TRY(P.sync.alloc(1));
  return G2OC_OK;
}

}  // namespace g2oc
