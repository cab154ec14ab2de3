// batch_kernels.cuh -- many independent local bundle adjustments (windows)
// in one packed graph: the linearization, Schur complement and
// back-substitution kernels run over all windows at once (the packed Hessian
// is block-diagonal by window), while the Levenberg-Marquardt control of
// OptimizationAlgorithmLevenberg::solve (g2o/core/optimization_algorithm_levenberg.cpp:60-153)
// runs per window on the device: each round every unfinished window makes one
// trial with its own lambda, accepts or rejects it (restoring only its own
// vertices) and advances its own iteration count. Each window's reduced
// camera system is solved by a dense FP64 Cholesky (LinearSolverDense,
// g2o/solvers/dense/linear_solver_dense.h:57-105), one CTA per window.
#pragma once

#include "../../include/g2o_cuda.h"
#include "ba_kernels.cuh"
#include "pcg_kernels.cuh"
#include "reduce.cuh"

namespace g2oc {

struct WinState {
  double chi2_init;   // robust chi2 before the first iteration
  double chi2_cur;    // currentChi of the window's iteration
  double chi2_temp;   // tempChi after the trial
  double lambda;
  double ni;
  double scale;       // computeScale() + 1e-3
  double rho;
  double max_diag;
  int iteration;      // completed iterations
  int qmax;           // trials in the current iteration
  int trials;         // trials in all
  int done;           // finished (iteration limit or Terminate)
  int accept;         // the last trial was accepted
  int result;         // G2OC_RESULT_* of the last iteration
  int solve_ok;       // the last factorization succeeded
  int pad;
};

// ranges of window w: free cameras [cam[w], cam[w+1]) and landmarks
// [lm[w], lm[w+1]) in Hessian order, device edges [edge[w], edge[w+1]),
// vertices (caller order) poses [pose[w], pose[w+1]) and points
// [point[w], point[w+1])
struct WinDev {
  int nw;
  const int* cam;
  const int* lm;
  const int* edge;
  const int* pose;
  const int* point;
  const long long* mat;  // offset of the window's dense n x n matrix in the scratch
};

// robust chi2 per window (activeRobustChi2) into chi2_cur (which = 0, windows
// at the start of an iteration) or chi2_temp (which = 1), over edge chunks of
// at most kWinChi2Chunk edges so that the largest windows do not set the
// launch's tail: per chunk a CTA's sum, then per window the chunk sums in
// chunk order (win_chi2_finish).
constexpr int kWinChi2Chunk = 2048;
template <int THREADS>
__global__ void __launch_bounds__(THREADS) win_chi2_chunks(BAEdges E, BAVertices V, WinDev W, const int* chunk_w,
                                                          const int* chunk_e0, const WinState* ws, int which,
                                                          double* partial) {
  const int ch = blockIdx.x, w = chunk_w[ch];
  const WinState& s = ws[w];
  if (s.done || (which == 0 && s.qmax != 0)) return;
  const int k1 = min(chunk_e0[ch] + kWinChi2Chunk, W.edge[w + 1]);
  double r = 0.0;
  for (int k = chunk_e0[ch] + threadIdx.x; k < k1; k += THREADS) {
    double e[2], Xc[3], chi2, wt;
    const double4 om = ba_om(E, k);
    ba_edge_error(V, E.v[k], E.z[k], om, e, Xc, chi2, wt);
    if (om.w > 0.0) {
      double rho[3];
      huber(chi2, om.w, rho);
      r += rho[0];
    } else {
      r += chi2;
    }
  }
  r = block_sum1(r);
  if (threadIdx.x == 0) partial[ch] = r;
}

static __global__ void win_chi2_finish(const int* win_chunk_ptr, int nw, const double* partial, WinState* ws,
                                       int which) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nw) return;
  WinState& s = ws[w];
  if (s.done || (which == 0 && s.qmax != 0)) return;
  double r = 0.0;
  for (int c = win_chunk_ptr[w]; c < win_chunk_ptr[w + 1]; ++c) r += partial[c];
  if (which == 0) {
    s.chi2_cur = r;
    if (s.iteration == 0) s.chi2_init = r;
  } else {
    s.chi2_temp = r;
  }
}

// computeLambdaInit for windows starting their first iteration: lambda =
// tau * max |diag H| over the window's free cameras and landmarks, ni = 2
template <typename Real, int THREADS>
__global__ void __launch_bounds__(THREADS) win_lambda_init(const Real* hpp, const Real* hll, WinDev W, WinState* ws,
                                                            double user_lambda, double tau) {
  const int w = blockIdx.x;
  WinState& s = ws[w];
  if (s.done || s.iteration != 0 || s.qmax != 0) return;
  double m = 0.0;
  const int c0 = W.cam[w], nc = (W.cam[w + 1] - c0) * 6;
  for (int t = threadIdx.x; t < nc; t += THREADS) {
    const int h = c0 + t / 6, d = t % 6;
    m = fmax(m, fabs((double)hpp[(size_t)h * 36 + d * 7]));  // BA: Hpp block h is camera h's diagonal
  }
  const int l0 = W.lm[w], nl = (W.lm[w + 1] - l0) * 3;
  for (int t = threadIdx.x; t < nl; t += THREADS) {
    const int l = l0 + t / 3, d = t % 3;
    m = fmax(m, fabs((double)hll[(size_t)l * 6 + (d == 0 ? 0 : d == 1 ? 3 : 5)]));
  }
  __shared__ double sm[THREADS / 32];
  m = warp_max(m);
  if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double x = 0.0;
    for (int i = 0; i < THREADS / 32; ++i) x = fmax(x, sm[i]);
    s.max_diag = x;
    s.lambda = user_lambda > 0.0 ? user_lambda : tau * x;
    s.ni = 2.0;
  }
}

// the window's lambda on each of its free cameras and landmarks
static __global__ void win_spread_lambda(const int* win_of_cam, int Cf, const int* win_of_lm, int Pf,
                                         const WinState* ws, double* lam_c, double* lam_l) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < Cf) lam_c[t] = ws[win_of_cam[t]].lambda;
  else if (t < Cf + Pf) lam_l[t - Cf] = ws[win_of_lm[t - Cf]].lambda;
}

constexpr int kWinNB = 32;      // panel width of the window Cholesky (one warp)
constexpr int kWinGroups = 16;  // fixed partial-sum groups of the backward solve

// shared memory of win_chol_solve for windows of at most nmax unknowns: the
// panel (kWinNB x win_ldt(nmax), column-major), x (nmax), the group sums and
// the reciprocal pivots (nmax)
__host__ __device__ inline int win_ldt(int n) { return (n + 2) & ~1; }
inline size_t win_chol_smem(int nmax) {
  return ((size_t)kWinNB * win_ldt(nmax) + 2 * nmax + kWinGroups * kWinNB) * sizeof(double);
}

// Dense Cholesky solve of one window's reduced camera system, one CTA per
// window from the list (LinearSolverDense: LLT of the damped Schur complement,
// then the two triangular solves). The matrix is the window's (n + 1) x n
// block of the scratch, written by the Schur rows (lower triangle; row n =
// the right-hand side), factored in place, right-looking, by panels of
// kWinNB columns:
//   - the panel (rows p0..n, the right-hand side row included) is staged in
//     shared memory column-major;
//   - warp 0 factors its diagonal block with the block's rows in registers
//     (lane i = row i; L_jk broadcast by shuffles, no CTA barrier per column);
//   - every thread solves one panel row against the diagonal block (the
//     right-hand-side row gives y = L^-1 b on the way);
//   - the trailing lower triangle takes the panel's update in 16 x 16 tiles,
//     one warp each, as FP64 tensor-core products (mma.sync m8n8k4) fed from
//     the column-major panel.
// Then x = L^-T y backwards by blocks of kWinNB: the sums over the rows below
// a block in kWinGroups fixed row groups, the block's triangle on warp 0.
// Every sum runs in an order fixed by n alone (not by the CTA size). The
// pivots' reciprocals 1/L_kk = rsqrt(d_k) are kept, so the long dependent
// chains (the diagonal block, each panel row, the backward block solves)
// multiply instead of divide. A non-positive pivot sets solve_ok = 0 for the
// window and x = 0.
template <int THREADS>
__global__ void __launch_bounds__(THREADS, 512 / THREADS) win_chol_solve(const int* wlist, int nlist, WinDev W, const double* bs,
                                                           double* xp, double* scratch, WinState* ws) {
  constexpr int WARPS = THREADS / 32;
  constexpr unsigned FULL = 0xffffffffu;
  extern __shared__ __align__(16) double sm[];
  __shared__ int s_ok;
  if ((int)blockIdx.x >= nlist) return;
  const int w = wlist[blockIdx.x];
  const int h0 = W.cam[w], n = 6 * (W.cam[w + 1] - h0);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (ws[w].done || n == 0) {
    for (int i = tid; i < n; i += THREADS) xp[(size_t)h0 * 6 + i] = 0.0;
    return;
  }
  const int ldt = win_ldt(n);
  double* PT = sm;                          // PT[k * ldt + i]: panel column k, row p0 + i
  double* vec = sm + (size_t)kWinNB * ldt;  // x
  double* grp = vec + n;                    // kWinGroups x kWinNB
  double* invd = grp + kWinGroups * kWinNB; // 1 / L_kk
  double* M = scratch + W.mat[w];
  for (int i = tid; i < n; i += THREADS) M[(size_t)n * n + i] = bs[(size_t)h0 * 6 + i];
  if (tid == 0) s_ok = 1;
  __syncthreads();
  for (int p0 = 0; p0 < n; p0 += kWinNB) {
    const int pb = min(kWinNB, n - p0);  // panel width
    const int m = n + 1 - p0;            // panel rows, the right-hand side row last
    // stage: row-major global reads (coalesced), entries above the diagonal
    // and columns past pb as zeros
    for (int t = tid; t < m * kWinNB; t += THREADS) {
      const int i = t / kWinNB, k = t % kWinNB;
      PT[k * ldt + i] = (k < pb && k <= i) ? M[(size_t)(p0 + i) * n + p0 + k] : 0.0;
    }
    __syncthreads();
    // diagonal block on warp 0
    if (warp == 0) {
      double a[kWinNB];
#pragma unroll
      for (int j = 0; j < kWinNB; ++j) a[j] = PT[j * ldt + lane];
      bool ok = true;
#pragma unroll
      for (int k = 0; k < kWinNB; ++k) {
        if (k < pb && ok) {
          const double d = __shfl_sync(FULL, a[k], k);
          if (!(d > 0.0)) {
            ok = false;  // uniform: every lane read the same pivot
          } else {
            const double inv = rsqrt(d);
            if (lane == k) {
              a[k] = d * inv;
              invd[p0 + k] = inv;
            } else if (lane > k) {
              a[k] *= inv;
            }
#pragma unroll
            for (int j = k + 1; j < kWinNB; ++j) {
              const double ljk = __shfl_sync(FULL, a[k], j);
              if (lane >= j) a[j] -= a[k] * ljk;
            }
          }
        }
      }
      if (lane < pb) {
#pragma unroll
        for (int j = 0; j < kWinNB; ++j)
          if (j <= lane) PT[j * ldt + lane] = a[j];
      }
      if (!ok && lane == 0) s_ok = 0;
    }
    __syncthreads();
    if (!s_ok) break;  // uniform
    // panel rows below the diagonal block: x L_JJ^T = a
    for (int i = pb + tid; i < m; i += THREADS) {
      double x[kWinNB];
#pragma unroll
      for (int j = 0; j < kWinNB; ++j) x[j] = PT[j * ldt + i];
#pragma unroll
      for (int k = 0; k < kWinNB; ++k) {
        if (k < pb) {
          x[k] *= invd[p0 + k];
#pragma unroll
          for (int j = k + 1; j < kWinNB; ++j) x[j] -= x[k] * PT[k * ldt + j];
        }
      }
#pragma unroll
      for (int j = 0; j < kWinNB; ++j) PT[j * ldt + i] = x[j];
    }
    __syncthreads();
    // the factored panel back (lower part and the right-hand side row)
    for (int t = tid; t < m * kWinNB; t += THREADS) {
      const int i = t / kWinNB, k = t % kWinNB;
      if (k < pb && k <= i) M[(size_t)(p0 + i) * n + p0 + k] = PT[k * ldt + i];
    }
    // trailing update: rows pb..m-1 (local), columns pb..m-2, lower part, in
    // 16 x 16 tiles (a, b), b <= a, numbered row-block by row-block, one warp
    // per tile: 2 x 2 FP64 tensor-core products (mma m8n8k4) per 4 columns of
    // the panel, operands straight from the column-major panel
    const int nc = m - 1 - pb;
    if (nc > 0) {
      const int nbc = (nc + 15) / 16, nbr = (m - pb + 15) / 16;
      const int tri = nbc * (nbc + 1) / 2;
      const int ntile = tri + (nbr > nbc ? nbc : 0);  // the last row block holds the right-hand side row only
      const int gi = lane >> 2, ti = lane & 3;
      for (int t = warp; t < ntile; t += WARPS) {
        int a, b;
        if (t < tri) {
          a = (int)((sqrtf(8.0f * (float)t + 1.0f) - 1.0f) * 0.5f);
          while ((a + 1) * (a + 2) / 2 <= t) ++a;
          while (a * (a + 1) / 2 > t) --a;
          b = t - a * (a + 1) / 2;
        } else {
          a = nbc;
          b = t - tri;
        }
        const int i0 = pb + 16 * a, j0 = pb + 16 * b;
        double acc[2][2][2];
#pragma unroll
        for (int u = 0; u < 2; ++u)
#pragma unroll
          for (int v = 0; v < 2; ++v) acc[u][v][0] = acc[u][v][1] = 0.0;
        for (int k0 = 0; k0 < pb; k0 += 4) {
          const double* col = PT + (k0 + ti) * ldt;
          const double fa0 = col[i0 + gi], fa1 = col[i0 + 8 + gi];
          const double fb0 = col[j0 + gi], fb1 = col[j0 + 8 + gi];
          const double fa[2] = {fa0, fa1}, fb[2] = {fb0, fb1};
#pragma unroll
          for (int u = 0; u < 2; ++u)
#pragma unroll
            for (int v = 0; v < 2; ++v)
              asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                           : "+d"(acc[u][v][0]), "+d"(acc[u][v][1])
                           : "d"(fa[u]), "d"(fb[v]));
        }
#pragma unroll
        for (int u = 0; u < 2; ++u)
#pragma unroll
          for (int v = 0; v < 2; ++v)
#pragma unroll
            for (int e = 0; e < 2; ++e) {
              const int i = i0 + 8 * u + gi, j = j0 + 8 * v + 2 * ti + e;
              if (i < m && j <= m - 2 && j <= i) {
                double* pm = M + (size_t)(p0 + i) * n + p0 + j;
                *pm = *pm - acc[u][v][e];
              }
            }
      }
    }
    __syncthreads();
  }
  if (!s_ok) {
    if (tid == 0) ws[w].solve_ok = 0;
    for (int i = tid; i < n; i += THREADS) xp[(size_t)h0 * 6 + i] = 0.0;
    return;
  }
  // x = L^-T y, y = row n; blocks from the last
  const double* y = M + (size_t)n * n;
  const int nblk = (n + kWinNB - 1) / kWinNB;
  for (int J = nblk - 1; J >= 0; --J) {
    const int q0 = J * kWinNB, qb = min(kWinNB, n - q0), r0 = q0 + qb;
    // group sums: g covers rows r0 + g, r0 + g + kWinGroups, ...
    for (int g = warp; g < kWinGroups; g += WARPS) {
      double acc = 0.0;
      if (lane < qb)
        for (int i = r0 + g; i < n; i += kWinGroups) acc += M[(size_t)i * n + q0 + lane] * vec[i];
      grp[g * kWinNB + lane] = acc;
    }
    __syncthreads();
    if (warp == 0) {
      double sj = 0.0;
      if (lane < qb) {
        sj = y[q0 + lane];
        for (int g = 0; g < kWinGroups; ++g) sj -= grp[g * kWinNB + lane];
      }
      double lc[kWinNB];  // column lane of the block: lc[k] = L(q0 + k, q0 + lane)
#pragma unroll
      for (int k = 0; k < kWinNB; ++k)
        lc[k] = (k < qb && lane <= k) ? M[(size_t)(q0 + k) * n + q0 + lane] : 0.0;
#pragma unroll
      for (int k = kWinNB - 1; k >= 0; --k) {
        if (k < qb) {
          const double xk = __shfl_sync(FULL, sj * invd[q0 + k], k);  // lane k: s_k / L_kk
          if (lane == k) sj = xk;
          else if (lane < k) sj -= lc[k] * xk;
        }
      }
      if (lane < qb) vec[q0 + lane] = sj;
    }
    __syncthreads();
  }
  for (int i = tid; i < n; i += THREADS) xp[(size_t)h0 * 6 + i] = vec[i];
  if (tid == 0) ws[w].solve_ok = 1;
}

// zero the step of finished windows (their vertices stay as they are)
static __global__ void win_mask_step(const int* win_of_cam, int Cf, const int* win_of_lm, int Pf, const WinState* ws,
                                     double* x) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < Cf * 6) {
    if (ws[win_of_cam[t / 6]].done) x[t] = 0.0;
  } else if (t < Cf * 6 + Pf * 3) {
    if (ws[win_of_lm[(t - Cf * 6) / 3]].done) x[t] = 0.0;
  }
}

// computeScale per window: x . (lambda x + b) over its Hessian range, + 1e-3
template <int THREADS>
__global__ void __launch_bounds__(THREADS) win_scale(const double* x, const double* b, int Cf, WinDev W,
                                                      WinState* ws) {
  const int w = blockIdx.x;
  WinState& s = ws[w];
  if (s.done) return;
  const double lambda = s.lambda;
  double acc = 0.0;
  const int c0 = W.cam[w] * 6, c1 = W.cam[w + 1] * 6;
  for (int i = c0 + threadIdx.x; i < c1; i += THREADS) acc += x[i] * (lambda * x[i] + b[i]);
  const int l0 = Cf * 6 + W.lm[w] * 3, l1 = Cf * 6 + W.lm[w + 1] * 3;
  for (int i = l0 + threadIdx.x; i < l1; i += THREADS) acc += x[i] * (lambda * x[i] + b[i]);
  acc = block_sum1(acc);
  if (threadIdx.x == 0) s.scale = acc + 1e-3;
}

// One trial's decision per window (lm_decide), then the trial loop and
// iteration bookkeeping of OptimizationAlgorithmLevenberg::solve and
// SparseOptimizer::optimize: the trial loop continues while rho < 0 and
// fewer than max_trials trials were made; it ends in Terminate when
// max_trials is reached, rho == 0 or lambda is not finite.
static __global__ void win_decide(WinState* ws, int nw, int max_trials, int max_iterations, int* active) {
  const int w = blockIdx.x * blockDim.x + threadIdx.x;
  if (w >= nw) return;
  WinState& s = ws[w];
  if (s.done) return;
  const bool ok2 = s.solve_ok != 0;
  double tempChi = s.chi2_temp;
  if (!ok2) tempChi = 1.79769313486231570815e+308;
  double rho = s.chi2_cur - tempChi;
  rho /= ok2 ? s.scale : 1.0;
  if (rho > 0 && isfinite(tempChi) && ok2) {
    double alpha = 1. - pow((2 * rho - 1), 3);
    alpha = fmin(alpha, 2. / 3.);
    s.lambda *= fmax(1. / 3., alpha);
    s.ni = 2;
    s.chi2_cur = tempChi;
    s.accept = 1;
  } else {
    s.lambda *= s.ni;
    s.ni *= 2;
    s.accept = 0;
  }
  s.rho = rho;
  s.qmax++;
  s.trials++;
  const bool more = rho < 0 && s.qmax < max_trials && isfinite(s.lambda);
  if (more) {
    atomicAdd(active, 1);
    return;
  }
  // the iteration is over
  if (s.qmax == max_trials || rho == 0 || !isfinite(s.lambda)) {
    s.result = G2OC_RESULT_TERMINATE;
    s.done = 1;
  } else {
    s.result = G2OC_RESULT_OK;
  }
  s.iteration++;
  s.qmax = 0;
  if (s.iteration >= max_iterations) s.done = 1;
  if (!s.done) atomicAdd(active, 1);
}

// restore the vertices of windows whose trial was rejected (pop), one thread
// per vertex record
static __global__ void win_pop(const int* win_of_pose, int C, const int* win_of_point, int P, const WinState* ws,
                               const double* pose_bak, double* pose, const double* point_bak, double* point) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < C * 8) {
    const WinState& s = ws[win_of_pose[t / 8]];
    if (!s.accept) pose[t] = pose_bak[t];
  } else if (t < C * 8 + P * 4) {
    const int u = t - C * 8;
    const WinState& s = ws[win_of_point[u / 4]];
    if (!s.accept) point[u] = point_bak[u];
  }
}

}  // namespace g2oc
