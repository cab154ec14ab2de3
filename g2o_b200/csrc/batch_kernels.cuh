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

// robust chi2 per window (activeRobustChi2), one CTA per window; into
// chi2_cur (which = 0, windows at the start of an iteration) or chi2_temp
// (which = 1)
template <int THREADS>
__global__ void __launch_bounds__(THREADS) win_chi2(BAEdges E, BAVertices V, WinDev W, WinState* ws, int which) {
  const int w = blockIdx.x;
  WinState& s = ws[w];
  if (s.done || (which == 0 && s.qmax != 0)) return;
  double r = 0.0;
  for (int k = W.edge[w] + threadIdx.x; k < W.edge[w + 1]; k += THREADS) {
    double e[2], Xc[3], chi2, wt;
    const double4 om = E.om[k];
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
  if (threadIdx.x == 0) {
    if (which == 0) {
      s.chi2_cur = r;
      if (s.iteration == 0) s.chi2_init = r;
    } else {
      s.chi2_temp = r;
    }
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

constexpr int kWinPanel = 16;  // columns per panel of the window Cholesky

// Dense Cholesky solve of one window's reduced camera system (upper blocks in
// the row-SoA store, right-hand side bs) into x_p, one CTA per window from the
// list. The full symmetric matrix is gathered in FP64 into the window's
// scratch and factored in place, right-looking by panels of kWinPanel
// columns: the panel is factored in shared memory (one column per step), then
// the trailing lower triangle takes the panel's rank-kWinPanel update (a warp
// per row, one read-modify-write per element per panel). The forward and
// backward substitutions run on one warp. A non-positive pivot sets
// solve_ok = 0 for the window. Dynamic shared memory: (nmax + 1) * (kWinPanel + 1)
// doubles.
template <typename Real, int THREADS>
__global__ void __launch_bounds__(THREADS) win_chol_solve(const int* wlist, int nlist, WinDev W, SysDev<Real> A,
                                                           const double* bs, double* xp, double* scratch,
                                                           WinState* ws) {
  constexpr int WARPS = THREADS / 32;
  constexpr int PS = kWinPanel + 1;  // panel row stride (padded against bank conflicts)
  extern __shared__ double sm[];     // panel: n x PS, then the vector (n)
  __shared__ int s_ok;
  if ((int)blockIdx.x >= nlist) return;
  const int w = wlist[blockIdx.x];
  const int h0 = W.cam[w], nb = W.cam[w + 1] - h0, n = nb * 6;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  if (ws[w].done || n == 0) {
    for (int i = tid; i < n; i += THREADS) xp[(size_t)h0 * 6 + i] = 0.0;
    return;
  }
  double* P = sm;
  double* vec = sm + (size_t)n * PS;
  double* M = scratch + W.mat[w];
  // gather: block k of row r (internal order) -> M rows (r-h0)*6.., cols (c-h0)*6..
  const int k0 = A.rptr[h0], k1 = A.rptr[h0 + nb];
  for (long long t = tid; t < (long long)(k1 - k0) * 36; t += THREADS) {
    const int k = k0 + (int)(t / 36), e = (int)(t % 36);
    const int r = A.brow[k], c = A.rcol[k];
    const int rb = A.rptr[r], nblk = A.rptr[r + 1] - rb;
    const double v = (double)A.val[sys_offset<6>(rb, nblk, k - rb, e)];
    const int i = (r - h0) * 6 + e / 6, j = (c - h0) * 6 + e % 6;
    M[(size_t)i * n + j] = v;
    if (r != c) M[(size_t)j * n + i] = v;  // a diagonal block writes each of its entries once
  }
  if (tid == 0) s_ok = 1;
  __syncthreads();
  for (int p0 = 0; p0 < n && s_ok; p0 += kWinPanel) {
    const int pb = min(kWinPanel, n - p0), m = n - p0;  // panel width, panel rows
    // the panel (rows p0.., columns p0..p0+pb) into shared memory
    for (int t = tid; t < m * pb; t += THREADS) {
      const int i = t / pb, cc = t % pb;
      P[i * PS + cc] = M[(size_t)(p0 + i) * n + p0 + cc];
    }
    __syncthreads();
    for (int cc = 0; cc < pb; ++cc) {
      const double d = P[cc * PS + cc];
      if (!(d > 0.0)) {
        if (tid == 0) s_ok = 0;
        break;  // uniform: every thread read the same pivot
      }
      const double piv = sqrt(d);
      for (int i = cc + 1 + tid; i < m; i += THREADS) P[i * PS + cc] /= piv;
      __syncthreads();
      if (tid == 0) P[cc * PS + cc] = piv;
      // the panel's later columns
      const int rest = pb - cc - 1;
      for (int t = tid; t < (m - cc - 1) * rest; t += THREADS) {
        const int i = cc + 1 + t / rest, c2 = cc + 1 + t % rest;
        if (i >= c2) P[i * PS + c2] -= P[i * PS + cc] * P[c2 * PS + cc];
      }
      __syncthreads();
    }
    __syncthreads();  // every thread (also one that left the loop at a bad pivot) sees s_ok
    if (!s_ok) break;
    // write the factored panel back, then the trailing update
    for (int t = tid; t < m * pb; t += THREADS) {
      const int i = t / pb, cc = t % pb;
      if (i >= cc) M[(size_t)(p0 + i) * n + p0 + cc] = P[i * PS + cc];
    }
    for (int i = pb + warp; i < m; i += WARPS) {
      double li[kWinPanel];
#pragma unroll
      for (int cc = 0; cc < kWinPanel; ++cc) li[cc] = cc < pb ? P[i * PS + cc] : 0.0;
      double* Mi = M + (size_t)(p0 + i) * n + p0;
      for (int j = pb + lane; j <= i; j += 32) {
        double acc = 0.0;
#pragma unroll
        for (int cc = 0; cc < kWinPanel; ++cc)
          if (cc < pb) acc += li[cc] * P[j * PS + cc];
        Mi[j] -= acc;
      }
    }
    __syncthreads();
  }
  __syncthreads();
  if (!s_ok) {
    if (tid == 0) ws[w].solve_ok = 0;
    for (int i = tid; i < n; i += THREADS) xp[(size_t)h0 * 6 + i] = 0.0;
    return;
  }
  // L y = b, then L^T x = y, on warp 0
  for (int i = tid; i < n; i += THREADS) vec[i] = bs[(size_t)h0 * 6 + i];
  __syncthreads();
  if (warp == 0) {
    for (int k = 0; k < n; ++k) {
      const double yk = vec[k] / M[(size_t)k * n + k];
      for (int i = k + 1 + lane; i < n; i += 32) vec[i] -= M[(size_t)i * n + k] * yk;
      __syncwarp();
      if (lane == 0) vec[k] = yk;
      __syncwarp();
    }
    for (int k = n - 1; k >= 0; --k) {
      double sacc = 0.0;
      for (int i = k + 1 + lane; i < n; i += 32) sacc += M[(size_t)i * n + k] * vec[i];
      sacc = warp_sum(sacc);
      if (lane == 0) vec[k] = (vec[k] - sacc) / M[(size_t)k * n + k];
      __syncwarp();
    }
  }
  __syncthreads();
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
