// bal_kernels.cuh -- device kernels of the BAL path: VertexCameraBAL (9
// parameters: angle-axis rotation, translation, focal length, two radial
// distortion terms; additive update), VertexPointBAL (marginalized) and
// EdgeObservationBAL (g2o/examples/bal/bal_example.cpp:67-203) under
// BlockSolver<9,3> with LinearSolverPCG or a Cholesky
// (bal_example.cpp:227-250). FP64 throughout.
//
// The edge records are those of the other projection edges (BAEdges /
// BACamEdges: point-major device order, camera-major copy, information and
// Huber record); the cameras are 9 doubles each, the points 4 (x y z pad).
// Hessian storage: H_ll 6 unique entries per landmark, Hpl 9 x 3 row-major
// per (camera, landmark) block, Hpp 9 x 9 per camera, the Schur complement
// 9 x 9 blocks in the row-SoA layout of SysDev (sys_offset<9>).
//
// Every sum is in a fixed order (per-thread loops, fixed shuffle trees,
// warps summed in index order): results are bit-identical run to run.
#pragma once

#include "ba_kernels.cuh"
#include "pcg_kernels.cuh"

namespace g2oc {

constexpr int kBalCam = 9;

// EdgeObservationBAL's prediction f r(p) p (bal_example.cpp:160-200) and,
// with JAC, its derivatives: Jc = d pred / d camera (2 x 9, row-major), Jp =
// d pred / d point (2 x 3). The rotation is Rodrigues' formula
// P = X cos t + (v x X) sin t + v (v.X)(1 - cos t) with t = |w|, v = w / t
// (P = X + w x X when t == 0), written in the reference's order. Its
// derivative in w is the chain rule through t and v (dt/dw = v, dv/dw =
// (I - v v^T) / t), the quantity forward-mode differentiation of that
// expression yields:
//   dP_i/dw_j = v_j g_i + A (e_j x X)_i + B (v.X) delta_ij + B v_i X_j,
//   g = -sin t X + (cos t - A)(v x X) + (v.X)(sin t - 2B) v,
//   A = sin t / t, B = (1 - cos t) / t.
template <bool JAC>
__device__ __forceinline__ void bal_eval(const double* cam, const double* X, double pred[2], double Jc[18],
                                         double Jp[6]) {
  const double w0 = cam[0], w1 = cam[1], w2 = cam[2];
  const double th2 = w0 * w0 + w1 * w1 + w2 * w2;
  double P[3], R[9], Jw[9];
  if (th2 > 0.0) {
    const double th = sqrt(th2);
    const double v[3] = {w0 / th, w1 / th, w2 / th};
    double sth, cth;
    sincos(th, &sth, &cth);
    const double q[3] = {v[1] * X[2] - v[2] * X[1], v[2] * X[0] - v[0] * X[2], v[0] * X[1] - v[1] * X[0]};
    const double d = v[0] * X[0] + v[1] * X[1] + v[2] * X[2];
    const double omc = 1.0 - cth;
#pragma unroll
    for (int i = 0; i < 3; ++i) P[i] = X[i] * cth + q[i] * sth + v[i] * d * omc;
    if (JAC) {
      const double A = sth / th, B = omc / th;
      const double gs = d * (sth - 2.0 * B);
#pragma unroll
      for (int i = 0; i < 3; ++i) {
        const double g = -sth * X[i] + (cth - A) * q[i] + gs * v[i];
#pragma unroll
        for (int j = 0; j < 3; ++j) Jw[i * 3 + j] = v[j] * g + B * v[i] * X[j] + (i == j ? B * d : 0.0);
      }
      // + A (e_j x X): e_0 x X = (0, -X2, X1), e_1 x X = (X2, 0, -X0), e_2 x X = (-X1, X0, 0)
      Jw[1 * 3 + 0] -= A * X[2];
      Jw[2 * 3 + 0] += A * X[1];
      Jw[0 * 3 + 1] += A * X[2];
      Jw[2 * 3 + 1] -= A * X[0];
      Jw[0 * 3 + 2] -= A * X[1];
      Jw[1 * 3 + 2] += A * X[0];
      // R = cos t I + sin t [v]x + (1 - cos t) v v^T
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int j = 0; j < 3; ++j) R[i * 3 + j] = omc * v[i] * v[j] + (i == j ? cth : 0.0);
      R[0 * 3 + 1] -= sth * v[2];
      R[0 * 3 + 2] += sth * v[1];
      R[1 * 3 + 0] += sth * v[2];
      R[1 * 3 + 2] -= sth * v[0];
      R[2 * 3 + 0] -= sth * v[1];
      R[2 * 3 + 1] += sth * v[0];
    }
  } else {
    P[0] = X[0] + (w1 * X[2] - w2 * X[1]);
    P[1] = X[1] + (w2 * X[0] - w0 * X[2]);
    P[2] = X[2] + (w0 * X[1] - w1 * X[0]);
    if (JAC) {
      // d (w x X) / dw = -[X]x ; d P / dX = I + [w]x
      Jw[0] = 0.0;   Jw[1] = X[2];  Jw[2] = -X[1];
      Jw[3] = -X[2]; Jw[4] = 0.0;   Jw[5] = X[0];
      Jw[6] = X[1];  Jw[7] = -X[0]; Jw[8] = 0.0;
      R[0] = 1.0; R[1] = -w2; R[2] = w1;
      R[3] = w2;  R[4] = 1.0; R[5] = -w0;
      R[6] = -w1; R[7] = w0;  R[8] = 1.0;
    }
  }
  P[0] += cam[3];
  P[1] += cam[4];
  P[2] += cam[5];
  const double p0 = -P[0] / P[2], p1 = -P[1] / P[2];
  const double r2 = p0 * p0 + p1 * p1;
  const double f = cam[6], k1 = cam[7], k2 = cam[8];
  const double rp = 1.0 + k1 * r2 + k2 * r2 * r2;
  const double fr = f * rp;
  pred[0] = fr * p0;
  pred[1] = fr * p1;
  if (JAC) {
    // d pred / d p = f (rp I + 2 (k1 + 2 k2 r2) p p^T); d p_k / d P = -(1/P2) (e_k, p_k)
    const double rd2 = 2.0 * (k1 + 2.0 * k2 * r2);
    const double D00 = f * (rp + rd2 * p0 * p0), D01 = f * rd2 * p0 * p1, D11 = f * (rp + rd2 * p1 * p1);
    const double iz = 1.0 / P[2];
    double G[6];  // d pred / d P
    G[0] = -iz * D00;
    G[1] = -iz * D01;
    G[2] = -iz * (D00 * p0 + D01 * p1);
    G[3] = -iz * D01;
    G[4] = -iz * D11;
    G[5] = -iz * (D01 * p0 + D11 * p1);
#pragma unroll
    for (int r = 0; r < 2; ++r) {
      const double* g = G + 3 * r;
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        Jc[r * 9 + j] = g[0] * Jw[j] + g[1] * Jw[3 + j] + g[2] * Jw[6 + j];
        Jc[r * 9 + 3 + j] = g[j];
        Jp[r * 3 + j] = g[0] * R[j] + g[1] * R[3 + j] + g[2] * R[6 + j];
      }
    }
    Jc[6] = rp * p0;
    Jc[15] = rp * p1;
    Jc[7] = f * r2 * p0;
    Jc[16] = f * r2 * p1;
    Jc[8] = f * r2 * r2 * p0;
    Jc[17] = f * r2 * r2 * p1;
  }
}

// error = prediction - measurement, chi2 = e^T Omega e and the robust weight
// rho'(chi2) (BaseEdge::robustInformation, g2o/core/base_edge.h:156-162)
template <bool JAC>
__device__ __forceinline__ void bal_edge(const BAVertices& V, int2 v, double2 z, double4 om, double e[2],
                                         double& chi2, double& w, double Jc[18], double Jp[6]) {
  double pred[2];
  bal_eval<JAC>(V.cam + (size_t)v.y * kBalCam, V.pt + (size_t)v.x * 4, pred, Jc, Jp);
  e[0] = pred[0] - z.x;
  e[1] = pred[1] - z.y;
  const double t0 = om.x * e[0] + om.y * e[1];
  const double t1 = om.y * e[0] + om.z * e[1];
  chi2 = e[0] * t0 + e[1] * t1;
  w = 1.0;
  if (om.w > 0.0) {
    double rho[3];
    huber(chi2, om.w, rho);
    w = rho[1];
  }
}

// computeActiveErrors + activeChi2 / activeRobustChi2
// (g2o/core/sparse_optimizer.cpp:78-130): partials[2*block] = (chi2, robust)
static __global__ void bal_chi2_kernel(BAEdges E, BAVertices V, double* partials) {
  double c = 0.0, r = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < E.n; k += gridDim.x * blockDim.x) {
    double e[2], chi2, w;
    const double4 om = ba_om(E, k);
    bal_edge<false>(V, E.v[k], E.z[k], om, e, chi2, w, nullptr, nullptr);
    c += chi2;
    if (om.w > 0.0) {
      double rho[3];
      huber(chi2, om.w, rho);
      r += rho[0];
    } else {
      r += chi2;
    }
  }
  block_sum2(c, r, partials + 2 * blockIdx.x);
}

// per-edge errors (parity hook)
static __global__ void bal_errors_kernel(BAEdges E, BAVertices V, double* err) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= E.n) return;
  double e[2], chi2, w;
  bal_edge<false>(V, E.v[k], E.z[k], ba_om(E, k), e, chi2, w, nullptr, nullptr);
  err[2 * k] = e[0];
  err[2 * k + 1] = e[1];
}

// per-edge Jacobians (parity hook): Jp 2 x 3, Jc 2 x 9
static __global__ void bal_jacobians_kernel(BAEdges E, BAVertices V, double* jp, double* jc) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= E.n) return;
  const int2 v = E.v[k];
  double pred[2], Jc[18], Jp[6];
  bal_eval<true>(V.cam + (size_t)v.y * kBalCam, V.pt + (size_t)v.x * 4, pred, Jc, Jp);
  for (int i = 0; i < 6; ++i) jp[6 * k + i] = Jp[i];
  for (int i = 0; i < 18; ++i) jc[18 * k + i] = Jc[i];
}

// Landmark side of BlockSolver::buildSystem (g2o/core/block_solver.hpp:492-565):
// one thread per free landmark over its (contiguous) edges: H_ll = sum Jp^T
// Om' Jp, b_l = sum Jp^T we (we = -rho' Omega e), and each Hpl block Jc^T Om'
// Jp (9 x 3; edges of one (camera, landmark) block are adjacent, summed in order).
static __global__ void bal_landmark_pass(BAEdges E, BAVertices V, const int* l_ptr, int Pf, double* hll,
                                         double* hpl, double* b_l) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= Pf) return;
  double H[6] = {0, 0, 0, 0, 0, 0};
  double bl[3] = {0, 0, 0};
  double B[27];
  int cur = -1;
  const int k1 = l_ptr[l + 1];
  for (int k = l_ptr[l]; k < k1; ++k) {
    const int2 v = E.v[k];
    const double4 om = ba_om(E, k);
    double e[2], chi2, w, Jc[18], Jp[6];
    bal_edge<true>(V, v, E.z[k], om, e, chi2, w, Jc, Jp);
    const double we0 = -w * (om.x * e[0] + om.y * e[1]);
    const double we1 = -w * (om.y * e[0] + om.z * e[1]);
    const double o00 = w * om.x, o01 = w * om.y, o11 = w * om.z;
    double A0[3], A1[3];  // (Om' Jp) rows, as columns of Jp^T Om'
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      A0[i] = Jp[i] * o00 + Jp[3 + i] * o01;
      A1[i] = Jp[i] * o01 + Jp[3 + i] * o11;
    }
    H[0] += A0[0] * Jp[0] + A1[0] * Jp[3];
    H[1] += A0[0] * Jp[1] + A1[0] * Jp[4];
    H[2] += A0[0] * Jp[2] + A1[0] * Jp[5];
    H[3] += A0[1] * Jp[1] + A1[1] * Jp[4];
    H[4] += A0[1] * Jp[2] + A1[1] * Jp[5];
    H[5] += A0[2] * Jp[2] + A1[2] * Jp[5];
#pragma unroll
    for (int i = 0; i < 3; ++i) bl[i] += Jp[i] * we0 + Jp[3 + i] * we1;
    const int blk = E.hpl[k];
    if (blk >= 0) {
      if (blk != cur) {
        if (cur >= 0) {
#pragma unroll
          for (int i = 0; i < 27; ++i) hpl[(size_t)cur * 27 + i] = B[i];
        }
#pragma unroll
        for (int i = 0; i < 27; ++i) B[i] = 0.0;
        cur = blk;
      }
#pragma unroll
      for (int r = 0; r < 9; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) B[r * 3 + c] += Jc[r] * A0[c] + Jc[9 + r] * A1[c];
    }
  }
  if (cur >= 0) {
#pragma unroll
    for (int i = 0; i < 27; ++i) hpl[(size_t)cur * 27 + i] = B[i];
  }
#pragma unroll
  for (int i = 0; i < 6; ++i) hll[(size_t)l * 6 + i] = H[i];
#pragma unroll
  for (int i = 0; i < 3; ++i) b_l[(size_t)l * 3 + i] = bl[i];
}

// upper-triangle index of (i, j), i <= j, of a 9 x 9 block
__host__ __device__ constexpr int bal_ut(int i, int j) { return i * 9 - i * (i - 1) / 2 + (j - i); }

// Camera side of buildSystem: one CTA per free camera sums H_pp = sum Jc^T
// Om' Jc (45 unique entries) and b_p = sum Jc^T we over the camera's edges
// (thread-strided, then a fixed shuffle tree per warp and the warps in
// order), and writes the full 9 x 9 block and b_p.
template <int THREADS>
__global__ void __launch_bounds__(THREADS) bal_camera_pass(BACamEdges CE, BAVertices V, double* hpp, double* b_p) {
  constexpr int WARPS = THREADS / 32;
  __shared__ double red[WARPS][54];
  const int h = blockIdx.x;
  double H[45], bp[9];
#pragma unroll
  for (int i = 0; i < 45; ++i) H[i] = 0.0;
#pragma unroll
  for (int i = 0; i < 9; ++i) bp[i] = 0.0;
  const int j1 = CE.ptr[h + 1];
  for (int j = CE.ptr[h] + threadIdx.x; j < j1; j += THREADS) {
    const int2 v = CE.v[j];
    const double4 om = ba_om(CE, j);
    double e[2], chi2, w, Jc[18], Jp[6];
    bal_edge<true>(V, v, CE.z[j], om, e, chi2, w, Jc, Jp);
    const double we0 = -w * (om.x * e[0] + om.y * e[1]);
    const double we1 = -w * (om.y * e[0] + om.z * e[1]);
    const double o00 = w * om.x, o01 = w * om.y, o11 = w * om.z;
    double A0[9], A1[9];
#pragma unroll
    for (int i = 0; i < 9; ++i) {
      A0[i] = Jc[i] * o00 + Jc[9 + i] * o01;
      A1[i] = Jc[i] * o01 + Jc[9 + i] * o11;
    }
#pragma unroll
    for (int i = 0; i < 9; ++i) {
#pragma unroll
      for (int k = i; k < 9; ++k) H[bal_ut(i, k)] += A0[i] * Jc[k] + A1[i] * Jc[9 + k];
      bp[i] += Jc[i] * we0 + Jc[9 + i] * we1;
    }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int i = 0; i < 45; ++i) {
    const double s = warp_sum(H[i]);
    if (lane == 0) red[wid][i] = s;
  }
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    const double s = warp_sum(bp[i]);
    if (lane == 0) red[wid][45 + i] = s;
  }
  __syncthreads();
  if (threadIdx.x < 54) {
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < WARPS; ++q) s += red[q][threadIdx.x];
    if (threadIdx.x < 45) {
      int i = 0, t = threadIdx.x;
      while (t >= 9 - i) {
        t -= 9 - i;
        ++i;
      }
      const int k = i + t;
      hpp[(size_t)h * 81 + i * 9 + k] = s;
      hpp[(size_t)h * 81 + k * 9 + i] = s;
    } else {
      b_p[(size_t)h * 9 + threadIdx.x - 45] = s;
    }
  }
}

// max |diag H| over Hpp and H_ll (computeLambdaInit,
// optimization_algorithm_levenberg.cpp:155-167): partial maxima per block
static __global__ void bal_max_diag(const double* hpp, int Cf, const double* hll, int Pf, double* partials) {
  double m = 0.0;
  const int n = Cf * 9 + Pf * 3;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    double v;
    if (t < Cf * 9) {
      v = fabs(hpp[(size_t)(t / 9) * 81 + (t % 9) * 10]);
    } else {
      const int l = (t - Cf * 9) / 3, d = (t - Cf * 9) % 3;
      v = fabs(hll[(size_t)l * 6 + (d == 0 ? 0 : d == 1 ? 3 : 5)]);
    }
    m = fmax(m, v);
  }
  block_max(m, partials + blockIdx.x);
}

// Per landmark: Dinv = (H_ll + lambda I)^-1 and, for each of its Hpl blocks,
// Y = Hpl Dinv (9 x 3), the factor every Schur product of the block uses
// (block_solver.hpp:372-386)
static __global__ void bal_schur_landmark(const double* hll, const double* hpl, const int* hb_ptr, int Pf,
                                          double lambda, double* dinv, double* Y, int* nonfinite) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= Pf) return;
  const double* h = hll + (size_t)l * 6;
  double A[9] = {h[0] + lambda, h[1], h[2], h[1], h[3] + lambda, h[4], h[2], h[4], h[5] + lambda};
  double D[9];
  if (!inverse3(A, D)) *nonfinite = 1;
#pragma unroll
  for (int i = 0; i < 9; ++i) dinv[(size_t)l * 9 + i] = D[i];
  if (!Y) return;
  const int b1 = hb_ptr[l + 1];
  for (int a = hb_ptr[l]; a < b1; ++a) {
    const double* B = hpl + (size_t)a * 27;
    double* o = Y + (size_t)a * 27;
#pragma unroll
    for (int r = 0; r < 9; ++r) {
      const double b0 = B[r * 3], b1v = B[r * 3 + 1], b2 = B[r * 3 + 2];
#pragma unroll
      for (int c = 0; c < 3; ++c) o[r * 3 + c] = b0 * D[c] + b1v * D[3 + c] + b2 * D[6 + c];
    }
  }
}

// Schur complement S = Hpp + lambda I - sum Hpl (H_ll + lambda I)^-1 Hpl^T
// (the Schur part of BlockSolver::solve, block_solver.hpp:346-433), one warp
// per 9 x 9 block of S in the internal row-major order. A diagonal block
// subtracts Y_a Hpl_a^T over its camera's Hpl blocks and also forms the
// reduced right-hand side b_p - sum Y_a b_l(a); an off-diagonal block (r, c)
// subtracts Y_a Hpl_b^T over its co-observation pairs (a of camera r, b of
// camera c, same landmark) in landmark order. The products' operands are
// staged four blocks at a time in shared memory (coalesced 216-byte rows);
// lane t owns entries t, t + 32, t + 64 of the block.
constexpr int kBalSchurWarps = 8;
constexpr int kBalStage = 4;

__global__ void __launch_bounds__(kBalSchurWarps * 32)
    bal_schur_blocks(int nnzb, const int* brow, const int* rptr, const int* rcol, const int* pair_ptr,
                     const int2* pairs, const int* hc_ptr, const int* hc_blk, const int* hpl_col, const double* hpp,
                     const double* hpl, const double* Y, double lambda, const double* b_p, const double* b_l,
                     double* S, double* bs) {
  __shared__ double stage[kBalSchurWarps][kBalStage][54];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int k = blockIdx.x * kBalSchurWarps + wid;
  if (k >= nnzb) return;
  const int r = brow[k], rb = rptr[r], nblk = rptr[r + 1] - rb, j = k - rb;
  const bool diag = rcol[k] == r;
  double (*st)[54] = stage[wid];
  double acc[3] = {0.0, 0.0, 0.0};
  int ei[3], ej[3];
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const int e = lane + 32 * q;
    ei[q] = e < 81 ? e / 9 : 0;
    ej[q] = e < 81 ? e % 9 : 0;
  }
  double rhs = 0.0;  // lanes < 9 of a diagonal block: the reduced right-hand side
  int n0, n1;
  if (diag) {
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      const int e = lane + 32 * q;
      if (e < 81) acc[q] = hpp[(size_t)r * 81 + e] + (ei[q] == ej[q] ? lambda : 0.0);
    }
    if (lane < 9) rhs = b_p[(size_t)r * 9 + lane];
    n0 = hc_ptr[r];
    n1 = hc_ptr[r + 1];
  } else {
    n0 = pair_ptr[k];
    n1 = pair_ptr[k + 1];
  }
  const int cam0 = hc_ptr[r];
  for (int p0 = n0; p0 < n1; p0 += kBalStage) {
    const int np = min(kBalStage, n1 - p0);
    __syncwarp();
    for (int t = lane; t < np * 54; t += 32) {
      const int it = t / 54, w = t % 54;
      int a, b;
      if (diag) {
        a = hc_blk[p0 + it];
        b = a;
      } else {
        const int2 pr = pairs[p0 + it];
        a = hc_blk[cam0 + pr.x];
        b = pr.y;
      }
      st[it][w] = w < 27 ? __ldg(Y + (size_t)a * 27 + w) : __ldg(hpl + (size_t)b * 27 + (w - 27));
    }
    __syncwarp();
    for (int it = 0; it < np; ++it) {
      const double* Ys = st[it];
      const double* Hs = st[it] + 27;
#pragma unroll
      for (int q = 0; q < 3; ++q) {
        const int i = ei[q], jj = ej[q];
        acc[q] -= Ys[i * 3] * Hs[jj * 3] + Ys[i * 3 + 1] * Hs[jj * 3 + 1] + Ys[i * 3 + 2] * Hs[jj * 3 + 2];
      }
      if (diag && lane < 9) {
        const double* bl = b_l + (size_t)hpl_col[hc_blk[p0 + it]] * 3;
        rhs -= Ys[lane * 3] * bl[0] + Ys[lane * 3 + 1] * bl[1] + Ys[lane * 3 + 2] * bl[2];
      }
    }
  }
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const int e = lane + 32 * q;
    if (e < 81) S[sys_offset<9>(rb, nblk, j, e)] = acc[q];
  }
  if (diag && lane < 9 && bs) bs[(size_t)r * 9 + lane] = rhs;
}

// Landmark back-substitution (block_solver.hpp:449-474):
// x_l = Dinv (r_l - sum_a Hpl_a^T x_p(row a))
static __global__ void bal_backsub(const int* hb_ptr, const int* hpl_row, int Pf, const double* hpl,
                                   const double* dinv, const double* r_l, const double* x_p, double* x_l) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= Pf) return;
  double cl[3] = {r_l[(size_t)l * 3], r_l[(size_t)l * 3 + 1], r_l[(size_t)l * 3 + 2]};
  const int b1 = hb_ptr[l + 1];
  for (int a = hb_ptr[l]; a < b1; ++a) {
    const double* B = hpl + (size_t)a * 27;
    const double* xp = x_p + (size_t)hpl_row[a] * 9;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double s = 0.0;
#pragma unroll
      for (int r = 0; r < 9; ++r) s += B[r * 3 + c] * xp[r];
      cl[c] -= s;
    }
  }
  const double* D = dinv + (size_t)l * 9;
#pragma unroll
  for (int i = 0; i < 3; ++i) x_l[(size_t)l * 3 + i] = D[i * 3] * cl[0] + D[i * 3 + 1] * cl[1] + D[i * 3 + 2] * cl[2];
}

// VertexCameraBAL::oplusImpl / VertexPointBAL::oplusImpl
// (bal_example.cpp:88-91, 116-119): estimate += update
static __global__ void bal_oplus(BAVertices V, int Cf, int Pf, const double* x, int* nonfinite) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < Cf * 9) {
    const int h = t / 9, d = t % 9;
    const double u = x[t];
    if (!isfinite(u)) *nonfinite = 1;
    V.cam[(size_t)V.free_pose[h] * kBalCam + d] += u;
  } else if (t < Cf * 9 + Pf * 3) {
    const int q = t - Cf * 9, l = q / 3, d = q % 3;
    const double u = x[t];
    if (!isfinite(u)) *nonfinite = 1;
    V.pt[(size_t)V.free_point[l] * 4 + d] += u;
  }
}

// dst = Hpp src over the camera part (block diagonal), zero landmark part
// (BlockSolverBase::multiplyHessian, g2o/core/block_solver.h:96)
static __global__ void bal_hpp_mult(int Cf, const double* hpp, const double* src, double* dst, int n) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  if (t >= Cf * 9) {
    dst[t] = 0.0;
    return;
  }
  const int h = t / 9, i = t % 9;
  const double* H = hpp + (size_t)h * 81 + i * 9;
  const double* s = src + (size_t)h * 9;
  double v = 0.0;
#pragma unroll
  for (int k = 0; k < 9; ++k) v += H[k] * s[k];
  dst[t] = v;
}

}  // namespace g2oc
