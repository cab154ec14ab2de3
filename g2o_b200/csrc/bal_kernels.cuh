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
// Hessian storage: H_ll 6 unique entries per landmark, Hpl 9 x 3 per
// (camera, landmark) block in the padded-triple layout (bal_bt), Hpp 9 x 9 per camera, the Schur complement
// 9 x 9 blocks in the row-SoA layout of SysDev (sys_offset<9>).
//
// Every sum is in a fixed order (per-thread loops, fixed shuffle trees,
// warps summed in index order): results are bit-identical run to run.
#pragma once

#include "ba_kernels.cuh"
#include "pcg_kernels.cuh"

namespace g2oc {

constexpr int kBalCam = 9;

// A 9 x 3 block (Hpl, Y = Hpl Dinv) is stored as three 3 x 3 row triples,
// each padded to 10 doubles (kBalBlk = 30 per block, the pads zero): element
// (r, c) at bal_bt(r, c). Every triple starts on a 16-byte boundary, so a
// block is 15 aligned 16-byte pieces and a triple's 9 values are four
// 16-byte loads and one 8-byte load.
constexpr int kBalBlk = 30;
__host__ __device__ constexpr int bal_bt(int r, int c) { return (r / 3) * 10 + (r % 3) * 3 + c; }

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

// a row-major 9 x 3 block into the padded-triple layout
__device__ __forceinline__ void bal_store_blk(double* o, const double (&B)[27]) {
#pragma unroll
  for (int r = 0; r < 9; ++r)
#pragma unroll
    for (int c = 0; c < 3; ++c) o[bal_bt(r, c)] = B[r * 3 + c];
  o[9] = 0.0;
  o[19] = 0.0;
  o[29] = 0.0;
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
        if (cur >= 0) bal_store_blk(hpl + (size_t)cur * kBalBlk, B);
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
  if (cur >= 0) bal_store_blk(hpl + (size_t)cur * kBalBlk, B);
#pragma unroll
  for (int i = 0; i < 6; ++i) hll[(size_t)l * 6 + i] = H[i];
#pragma unroll
  for (int i = 0; i < 3; ++i) b_l[(size_t)l * 3 + i] = bl[i];
}

// Landmark pass, edge-parallel form (landmarks of at most 32 edges, unique
// (camera, landmark) pairs; the chunks of whole landmarks packed on the host):
// one warp per chunk, one lane per edge with coalesced edge loads. Each
// lane's Hpl block goes to shared memory and the warp stores the chunk's
// contiguous block range coalesced; H_ll and b_l are summed by a segmented
// warp scan keyed by landmark (fixed shuffle order) and written by the
// segment's last lane. Four warps per CTA (27 KB of staging).
constexpr int kBalLmWarps = 4;

__global__ void __launch_bounds__(kBalLmWarps * 32)
    bal_landmark_warp(BAEdges E, BAVertices V, const int* chunk_ptr, int nchunks, const int* e_lm, double* hll,
                      double* hpl, double* b_l) {
  __shared__ double stage[kBalLmWarps][32 * kBalBlk];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int ch = blockIdx.x * kBalLmWarps + wid;
  if (ch >= nchunks) return;
  const int e0 = chunk_ptr[ch], e1 = chunk_ptr[ch + 1];
  const int k = e0 + lane;
  const bool act = k < e1;
  double H[6] = {0, 0, 0, 0, 0, 0};
  double bl[3] = {0, 0, 0};
  int key = -1 - lane;  // distinct for idle lanes
  const int blk = act ? E.hpl[k] : -1;
  const unsigned has = __ballot_sync(0xffffffffu, blk >= 0);
  const int blk0 = (int)__reduce_min_sync(0xffffffffu, blk >= 0 ? (unsigned)blk : 0x7fffffffu);
  if (act) {
    key = e_lm[k];
    const int2 v = E.v[k];
    const double4 om = ba_om(E, k);
    double e[2], chi2, w, Jc[18], Jp[6];
    bal_edge<true>(V, v, E.z[k], om, e, chi2, w, Jc, Jp);
    const double we0 = -w * (om.x * e[0] + om.y * e[1]);
    const double we1 = -w * (om.y * e[0] + om.z * e[1]);
    const double o00 = w * om.x, o01 = w * om.y, o11 = w * om.z;
    double A0[3], A1[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
      A0[i] = Jp[i] * o00 + Jp[3 + i] * o01;
      A1[i] = Jp[i] * o01 + Jp[3 + i] * o11;
    }
    H[0] = A0[0] * Jp[0] + A1[0] * Jp[3];
    H[1] = A0[0] * Jp[1] + A1[0] * Jp[4];
    H[2] = A0[0] * Jp[2] + A1[0] * Jp[5];
    H[3] = A0[1] * Jp[1] + A1[1] * Jp[4];
    H[4] = A0[1] * Jp[2] + A1[1] * Jp[5];
    H[5] = A0[2] * Jp[2] + A1[2] * Jp[5];
#pragma unroll
    for (int i = 0; i < 3; ++i) bl[i] = Jp[i] * we0 + Jp[3 + i] * we1;
    if (blk >= 0) {
      double hb[27];
#pragma unroll
      for (int r = 0; r < 9; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) hb[r * 3 + c] = Jc[r] * A0[c] + Jc[9 + r] * A1[c];
      bal_store_blk(&stage[wid][(blk - blk0) * kBalBlk], hb);
    }
  }
  // segmented inclusive scan by landmark
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int ko = __shfl_up_sync(0xffffffffu, key, off);
    double Ho[6], bo[3];
#pragma unroll
    for (int i = 0; i < 6; ++i) Ho[i] = __shfl_up_sync(0xffffffffu, H[i], off);
#pragma unroll
    for (int i = 0; i < 3; ++i) bo[i] = __shfl_up_sync(0xffffffffu, bl[i], off);
    if (lane >= off && ko == key) {
#pragma unroll
      for (int i = 0; i < 6; ++i) H[i] += Ho[i];
#pragma unroll
      for (int i = 0; i < 3; ++i) bl[i] += bo[i];
    }
  }
  const int knext = __shfl_down_sync(0xffffffffu, key, 1);
  if (act && (lane == 31 || knext != key)) {
#pragma unroll
    for (int i = 0; i < 6; ++i) hll[(size_t)key * 6 + i] = H[i];
#pragma unroll
    for (int i = 0; i < 3; ++i) b_l[(size_t)key * 3 + i] = bl[i];
  }
  __syncwarp();
  const int n = __popc(has) * kBalBlk;
  double* out = hpl + (size_t)blk0 * kBalBlk;
  for (int i = lane; i < n; i += 32) out[i] = stage[wid][i];
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

// Camera side in chunks: the camera-major edge list cut into chunks of at
// most kBalCamChunk edges of one camera (host plan: camera, first edge, end),
// a CTA per chunk summing its 45 + 9 values as bal_camera_pass does into
// `cpart`; bal_camera_reduce adds each camera's chunk sums in chunk order and
// writes the full 9 x 9 block and b_p. More CTAs than cameras keep the SMs
// busy (a 356-camera problem has ~3,600 edges per camera). Bounded to three
// CTAs per SM (168 registers, a few spilled): 97 us against 113 us at two.
constexpr int kBalCamChunk = 512;

template <int THREADS>
__global__ void __launch_bounds__(THREADS, 3)
    bal_camera_chunks(BACamEdges CE, BAVertices V, const int4* cch, double* cpart) {
  constexpr int WARPS = THREADS / 32;
  __shared__ double red[WARPS][54];
  const int4 cd = cch[blockIdx.x];
  double H[45], bp[9];
#pragma unroll
  for (int i = 0; i < 45; ++i) H[i] = 0.0;
#pragma unroll
  for (int i = 0; i < 9; ++i) bp[i] = 0.0;
  for (int j = cd.y + threadIdx.x; j < cd.z; j += THREADS) {
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
    cpart[(size_t)blockIdx.x * 54 + threadIdx.x] = s;
  }
}

// thread per (camera, value): the camera's chunk sums in order -> Hpp (both
// triangles) and b_p
static __global__ void bal_camera_reduce(int Cf, const int* cch_ptr, const double* cpart, double* hpp,
                                         double* b_p) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= Cf * 54) return;
  const int h = t / 54, q = t % 54;
  double s = 0.0;
  for (int c = cch_ptr[h]; c < cch_ptr[h + 1]; ++c) s += cpart[(size_t)c * 54 + q];
  if (q < 45) {
    int i = 0, u = q;
    while (u >= 9 - i) {
      u -= 9 - i;
      ++i;
    }
    const int k = i + u;
    hpp[(size_t)h * 81 + i * 9 + k] = s;
    hpp[(size_t)h * 81 + k * 9 + i] = s;
  } else {
    b_p[(size_t)h * 9 + q - 45] = s;
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

// Per landmark: Dinv = (H_ll + lambda I)^-1 (block_solver.hpp:372-386)
static __global__ void bal_schur_landmark(const double* hll, int Pf, double lambda, double* dinv, int* nonfinite) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= Pf) return;
  const double* h = hll + (size_t)l * 6;
  double A[9] = {h[0] + lambda, h[1], h[2], h[1], h[3] + lambda, h[4], h[2], h[4], h[5] + lambda};
  double D[9];
  if (!inverse3(A, D)) *nonfinite = 1;
#pragma unroll
  for (int i = 0; i < 9; ++i) dinv[(size_t)l * 9 + i] = D[i];
}

// Y_a = Hpl_a Dinv_l(a) for every Hpl block, the factor every Schur product
// of the block uses: a CTA per kBalYBlocks consecutive blocks loads them into
// shared memory coalesced, each thread forms its block's product in place,
// and the CTA stores the range coalesced. The three pads of a Y block carry
// b_l(a), so the diagonal Schur chunks that stage Y_a also form the reduced
// right-hand side's products Y_a b_l.
constexpr int kBalYBlocks = 128;

static __global__ void __launch_bounds__(kBalYBlocks)
    bal_schur_y(int nh, const int* hpl_col, const double* hpl, const double* dinv, const double* b_l, double* Y) {
  __shared__ __align__(16) double sm[kBalYBlocks * kBalBlk];
  const int a0 = blockIdx.x * kBalYBlocks;
  const int n = min(kBalYBlocks, nh - a0);
  // 16-byte pieces (a block is 15), all of a thread's loads issued before its stores
  const double2* src = reinterpret_cast<const double2*>(hpl + (size_t)a0 * kBalBlk);
  double2* sm2 = reinterpret_cast<double2*>(sm);
  constexpr int kPer = kBalYBlocks * kBalBlk / 2 / kBalYBlocks;  // 15 pieces per thread
  const int npc = n * kBalBlk / 2;
  double2 v[kPer];
#pragma unroll
  for (int u = 0; u < kPer; ++u) {
    const int t = u * kBalYBlocks + threadIdx.x;
    if (t < npc) v[u] = __ldg(src + t);
  }
#pragma unroll
  for (int u = 0; u < kPer; ++u) {
    const int t = u * kBalYBlocks + threadIdx.x;
    if (t < npc) sm2[t] = v[u];
  }
  __syncthreads();
  if ((int)threadIdx.x < n) {
    const int l = hpl_col[a0 + threadIdx.x];
    const double* D = dinv + (size_t)l * 9;
    double d[9];
#pragma unroll
    for (int q = 0; q < 9; ++q) d[q] = D[q];
    double* B = sm + threadIdx.x * kBalBlk;
#pragma unroll
    for (int r = 0; r < 9; ++r) {
      double* row = B + bal_bt(r, 0);
      const double b0 = row[0], b1 = row[1], b2 = row[2];
#pragma unroll
      for (int c = 0; c < 3; ++c) row[c] = b0 * d[c] + b1 * d[3 + c] + b2 * d[6 + c];
    }
    B[9] = b_l[(size_t)l * 3];
    B[19] = b_l[(size_t)l * 3 + 1];
    B[29] = b_l[(size_t)l * 3 + 2];
  }
  __syncthreads();
  double2* dst = reinterpret_cast<double2*>(Y + (size_t)a0 * kBalBlk);
#pragma unroll
  for (int u = 0; u < kPer; ++u) {
    const int t = u * kBalYBlocks + threadIdx.x;
    if (t < npc) dst[t] = sm2[t];
  }
}

// Schur complement S = Hpp + lambda I - sum Hpl (H_ll + lambda I)^-1 Hpl^T
// (the Schur part of BlockSolver::solve, block_solver.hpp:346-433). The
// products of a 9 x 9 block of S in the internal row-major order are its
// items: a diagonal block (r, r) has one per Hpl block a of camera r
// (Y_a Hpl_a^T), an off-diagonal block (r, c) one per co-observation pair (a
// of camera r, b of camera c, same landmark; Y_a Hpl_b^T), in landmark order.
// The items are cut into chunks of at most kBalChunk (host plan, fixed), one
// warp per chunk. The operands of kBalStage items (Y_a and Hpl_b, 15 aligned
// 16-byte pieces each) are copied into shared memory by asynchronous copies,
// double-buffered: the next stage's copies are in flight while this stage is
// multiplied, and the item indices are fetched one stage further ahead. The
// warp's first 27 lanes form three groups of nine, group G taking the items
// G, G + 3, ... of a stage and lane (bi, bj) of a group a 3 x 3 patch of the
// block (row triple bi of Y_a against row triple bj of Hpl_b: ten shared
// loads, 27 fused multiply-adds), two items at a time into two accumulator
// sets; at the end the sets and then the three groups' sums are added in
// order. A block of one chunk is written straight into S (diagonal:
// Hpp + lambda I minus the sum); the chunks of a longer block leave their
// sums in `part` and bal_schur_reduce adds them in chunk order, so every
// block's sum has a fixed order whatever the launch shape. Items: a diagonal
// block's are its camera's Hpl blocks (hc_blk), an off-diagonal block's its
// pairs (a, b) of absolute Hpl block indices. An item occupies kBalItem
// doubles of shared memory (Y at 0, Hpl_b at 30): 62 puts the two items a
// quarter-warp of 16-byte loads can touch in distinct banks.
constexpr int kBalChunk = 120;
constexpr int kBalStage = 12;
constexpr int kBalChunkWarps = 4;
constexpr int kBalItem = 62;
constexpr int kBalStageCopies = (kBalStage * 30 + 31) / 32;  // 16-byte copies per lane per stage

__device__ __forceinline__ void bal_cp16(double* dst, const double* src) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"((unsigned)__cvta_generic_to_shared(dst)),
               "l"(src)
               : "memory");
}
__device__ __forceinline__ void bal_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void bal_cp_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// the item indices of the stage starting at item p (lanes < np)
__device__ __forceinline__ void bal_item(bool diag, const int* hc_blk, const int2* pairs, int p, int np, int lane,
                                         int& a, int& b) {
  a = 0;
  b = 0;
  if (lane < np) {
    if (diag) {
      a = __ldg(hc_blk + p + lane);
      b = a;
    } else {
      const int2 pr = __ldg(pairs + p + lane);
      a = pr.x;
      b = pr.y;
    }
  }
}

// asynchronous copies of a stage's operands (every lane runs the same loop:
// the shuffles see the whole warp); piece w < 15 of an item is Y_a's, the
// rest Hpl_b's, both landing at 2 w in the item's slot
__device__ __forceinline__ void bal_stage_copy(double* st, int np, int a, int b, const double* Y, const double* hpl,
                                               int lane) {
  const int tot = np * 30;
#pragma unroll
  for (int u = 0; u < kBalStageCopies; ++u) {
    const int t = u * 32 + lane;
    const int it = min(t / 30, max(np - 1, 0));
    const int w = t - it * 30;
    const int ai = __shfl_sync(0xffffffffu, a, it);
    const int bi = __shfl_sync(0xffffffffu, b, it);
    if (t < tot)
      bal_cp16(st + it * kBalItem + 2 * w,
               w < 15 ? Y + (size_t)ai * kBalBlk + 2 * w : hpl + (size_t)bi * kBalBlk + 2 * (w - 15));
  }
  bal_cp_commit();
}

// a row triple (9 doubles, 16-byte aligned) from shared memory
__device__ __forceinline__ void bal_ld_triple(const double* p, double (&v)[9]) {
#pragma unroll
  for (int q = 0; q < 4; ++q) {
    const double2 t = *reinterpret_cast<const double2*>(p + 2 * q);
    v[2 * q] = t.x;
    v[2 * q + 1] = t.y;
  }
  v[8] = p[8];
}

__global__ void __launch_bounds__(kBalChunkWarps * 32)
    bal_schur_chunks(int nchunks, const int4* chunks, const int* brow, const int* rptr, const int* rcol,
                     const int2* pairs, const int* hc_blk, const double* hpp, const double* hpl, const double* Y,
                     double lambda, double* S, double* part, const double* b_p, double* bs, double* rpart) {
  __shared__ __align__(16) double stage[kBalChunkWarps][2][kBalStage * kBalItem];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int ch = blockIdx.x * kBalChunkWarps + wid;
  if (ch >= nchunks) return;
  const int4 cd = chunks[ch];
  const int k = cd.x, q0 = cd.y, q1 = cd.z, slot = cd.w;
  const int r = brow[k];
  const bool diag = rcol[k] == r;
  const int grp = lane / 9, sub = lane % 9, bi = sub / 3, bj = sub % 3;
  double acc[9], acc2[9];
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    acc[q] = 0.0;
    acc2[q] = 0.0;
  }
  // diagonal blocks: the lanes with bj == 0 also sum Y_a b_l(a) for their
  // rows 3bi .. 3bi + 2 (b_l rides in Y_a's pads)
  double rv[3] = {0.0, 0.0, 0.0};
  const bool rhs = diag && bj == 0;
  // stage s covers items q0 + s kBalStage ..; prologue: copies of stage 0,
  // indices of stage 1
  int a, b;
  int np = min(kBalStage, q1 - q0);
  bal_item(diag, hc_blk, pairs, q0, np, lane, a, b);
  if (np > 0) bal_stage_copy(stage[wid][0], np, a, b, Y, hpl, lane);
  int p1 = q0 + kBalStage;
  int np1 = max(0, min(kBalStage, q1 - p1));
  bal_item(diag, hc_blk, pairs, p1, np1, lane, a, b);
  for (int s = 0; np > 0; ++s) {
    if (np1 > 0) {
      bal_stage_copy(stage[wid][(s + 1) & 1], np1, a, b, Y, hpl, lane);
      const int p2 = p1 + kBalStage;
      const int np2 = max(0, min(kBalStage, q1 - p2));
      bal_item(diag, hc_blk, pairs, p2, np2, lane, a, b);
      bal_cp_wait<1>();  // this stage's copies have landed; the next stage's may still be in flight
      p1 = p2;
      np1 = np2;
    } else {
      bal_cp_wait<0>();
    }
    __syncwarp();
    const double* st = stage[wid][s & 1];
    if (lane < 27) {
      // two items at a time into two accumulator sets (independent chains)
      int it = grp;
      for (; it + 3 < np; it += 6) {
        double y[9], h[9], y2[9], h2[9];
        bal_ld_triple(st + it * kBalItem + bi * 10, y);  // Y rows 3bi .. 3bi + 2
        bal_ld_triple(st + it * kBalItem + 30 + bj * 10, h);  // Hpl_b rows 3bj .. 3bj + 2
        bal_ld_triple(st + (it + 3) * kBalItem + bi * 10, y2);
        bal_ld_triple(st + (it + 3) * kBalItem + 30 + bj * 10, h2);
#pragma unroll
        for (int m = 0; m < 3; ++m)
#pragma unroll
          for (int u = 0; u < 3; ++u)
#pragma unroll
            for (int v = 0; v < 3; ++v) {
              acc[u * 3 + v] = fma(y[u * 3 + m], h[v * 3 + m], acc[u * 3 + v]);
              acc2[u * 3 + v] = fma(y2[u * 3 + m], h2[v * 3 + m], acc2[u * 3 + v]);
            }
        if (rhs) {
          const double* p1 = st + it * kBalItem;
          const double* p2 = st + (it + 3) * kBalItem;
#pragma unroll
          for (int u = 0; u < 3; ++u) {
            rv[u] = fma(y[u * 3], p1[9], rv[u]);
            rv[u] = fma(y[u * 3 + 1], p1[19], rv[u]);
            rv[u] = fma(y[u * 3 + 2], p1[29], rv[u]);
            rv[u] = fma(y2[u * 3], p2[9], rv[u]);
            rv[u] = fma(y2[u * 3 + 1], p2[19], rv[u]);
            rv[u] = fma(y2[u * 3 + 2], p2[29], rv[u]);
          }
        }
      }
      if (it < np) {
        double y[9], h[9];
        bal_ld_triple(st + it * kBalItem + bi * 10, y);
        bal_ld_triple(st + it * kBalItem + 30 + bj * 10, h);
#pragma unroll
        for (int m = 0; m < 3; ++m)
#pragma unroll
          for (int u = 0; u < 3; ++u)
#pragma unroll
            for (int v = 0; v < 3; ++v) acc[u * 3 + v] = fma(y[u * 3 + m], h[v * 3 + m], acc[u * 3 + v]);
        if (rhs) {
          const double* p1 = st + it * kBalItem;
#pragma unroll
          for (int u = 0; u < 3; ++u) {
            rv[u] = fma(y[u * 3], p1[9], rv[u]);
            rv[u] = fma(y[u * 3 + 1], p1[19], rv[u]);
            rv[u] = fma(y[u * 3 + 2], p1[29], rv[u]);
          }
        }
      }
    }
    __syncwarp();  // the buffer is read before the copies of stage s + 2 overwrite it
    np = min(kBalStage, q1 - (q0 + (s + 1) * kBalStage));
  }
  // the two sets, then the three groups' sums in group order, on lanes 0..8
#pragma unroll
  for (int q = 0; q < 9; ++q) {
    acc[q] += acc2[q];
    const double g1 = __shfl_sync(0xffffffffu, acc[q], lane + 9 < 32 ? lane + 9 : lane);
    const double g2 = __shfl_sync(0xffffffffu, acc[q], lane + 18 < 32 ? lane + 18 : lane);
    acc[q] = (acc[q] + g1) + g2;
  }
#pragma unroll
  for (int u = 0; u < 3; ++u) {
    const double g1 = __shfl_sync(0xffffffffu, rv[u], lane + 9 < 32 ? lane + 9 : lane);
    const double g2 = __shfl_sync(0xffffffffu, rv[u], lane + 18 < 32 ? lane + 18 : lane);
    rv[u] = (rv[u] + g1) + g2;
  }
  if (lane >= 9) return;
  if (slot >= 0) {
#pragma unroll
    for (int u = 0; u < 3; ++u)
#pragma unroll
      for (int v = 0; v < 3; ++v) part[(size_t)slot * 81 + (3 * bi + u) * 9 + 3 * bj + v] = acc[u * 3 + v];
    if (rhs) {
#pragma unroll
      for (int u = 0; u < 3; ++u) rpart[(size_t)slot * 9 + 3 * bi + u] = rv[u];
    }
    return;
  }
  if (rhs && bs) {
#pragma unroll
    for (int u = 0; u < 3; ++u) bs[(size_t)r * 9 + 3 * bi + u] = b_p[(size_t)r * 9 + 3 * bi + u] - rv[u];
  }
  const int rb = rptr[r], nblk = rptr[r + 1] - rb, j = k - rb;
#pragma unroll
  for (int u = 0; u < 3; ++u)
#pragma unroll
    for (int v = 0; v < 3; ++v) {
      const int ii = 3 * bi + u, jj = 3 * bj + v, e = ii * 9 + jj;
      const double base = diag ? hpp[(size_t)r * 81 + e] + (ii == jj ? lambda : 0.0) : 0.0;
      S[sys_offset<9>(rb, nblk, j, e)] = base - acc[u * 3 + v];
    }
}

// the blocks cut into several chunks: (block, first slot, slots), thread per entry
static __global__ void bal_schur_reduce(int nred, const int4* red, const int* brow, const int* rptr,
                                        const int* rcol, const double* hpp, double lambda, const double* part,
                                        double* S, const double* rpart, const double* b_p, double* bs) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= nred * 81) return;
  const int q = t / 81, e = t % 81;
  const int4 rd = red[q];
  double s = 0.0;
  for (int n = 0; n < rd.z; ++n) s += part[(size_t)(rd.y + n) * 81 + e];
  const int k = rd.x, r = brow[k];
  if (e < 9 && bs && rcol[k] == r) {  // a diagonal block: the reduced right-hand side's entry e
    double sr = 0.0;
    for (int n = 0; n < rd.z; ++n) sr += rpart[(size_t)(rd.y + n) * 9 + e];
    bs[(size_t)r * 9 + e] = b_p[(size_t)r * 9 + e] - sr;
  }
  const int i = e / 9, jj = e % 9;
  const double base = rcol[k] == r ? hpp[(size_t)r * 81 + e] + (i == jj ? lambda : 0.0) : 0.0;
  const int rb = rptr[r], nblk = rptr[r + 1] - rb;
  S[sys_offset<9>(rb, nblk, k - rb, e)] = base - s;
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
    const double* B = hpl + (size_t)a * kBalBlk;
    const double* xp = x_p + (size_t)hpl_row[a] * 9;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double s = 0.0;
#pragma unroll
      for (int r = 0; r < 9; ++r) s += B[bal_bt(r, c)] * xp[r];
      cl[c] -= s;
    }
  }
  const double* D = dinv + (size_t)l * 9;
#pragma unroll
  for (int i = 0; i < 3; ++i) x_l[(size_t)l * 3 + i] = D[i * 3] * cl[0] + D[i * 3 + 1] * cl[1] + D[i * 3 + 2] * cl[2];
}

// Back-substitution, one warp per chunk of whole landmarks (the chunks of
// bal_landmark_warp), lane per edge: Hpl_a^T x_p(row a) per edge, summed per
// landmark by a segmented warp scan (fixed shuffle order), x_l = Dinv (r_l -
// sum) by the segment's last lane
static __global__ void bal_backsub_warp(const int* e_hpl, const int* hpl_row, const int* chunk_ptr, int nchunks,
                                        const int* e_lm, const double* hpl, const double* dinv, const double* r_l,
                                        const double* x_p, double* x_l) {
  const int lane = threadIdx.x & 31;
  const int ch = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (ch >= nchunks) return;
  const int e0 = chunk_ptr[ch], e1 = chunk_ptr[ch + 1];
  const int k = e0 + lane;
  const bool act = k < e1;
  double acc[3] = {0, 0, 0};
  int key = -1 - lane;
  if (act) {
    key = e_lm[k];
    const int blk = e_hpl[k];
    if (blk >= 0) {
      const double* B = hpl + (size_t)blk * kBalBlk;
      const double* xp = x_p + (size_t)hpl_row[blk] * 9;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double t = 0.0;
#pragma unroll
        for (int r = 0; r < 9; ++r) t += B[bal_bt(r, c)] * xp[r];
        acc[c] = t;
      }
    }
  }
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int ko = __shfl_up_sync(0xffffffffu, key, off);
    double ao[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) ao[i] = __shfl_up_sync(0xffffffffu, acc[i], off);
    if (lane >= off && ko == key) {
#pragma unroll
      for (int i = 0; i < 3; ++i) acc[i] += ao[i];
    }
  }
  const int knext = __shfl_down_sync(0xffffffffu, key, 1);
  if (act && (lane == 31 || knext != key)) {
    const double cl[3] = {r_l[(size_t)key * 3] - acc[0], r_l[(size_t)key * 3 + 1] - acc[1],
                          r_l[(size_t)key * 3 + 2] - acc[2]};
    const double* D = dinv + (size_t)key * 9;
#pragma unroll
    for (int i = 0; i < 3; ++i) x_l[(size_t)key * 3 + i] = D[i * 3] * cl[0] + D[i * 3 + 1] * cl[1] + D[i * 3 + 2] * cl[2];
  }
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
