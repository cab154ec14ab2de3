// ba_kernels.cuh -- device kernels of the bundle-adjustment path
// (EdgeProjectXYZ2UV between VertexPointXYZ landmarks, marginalized, and
// VertexSE3Expmap cameras). Real is the storage/accumulation type of the
// Jacobians, Hessian blocks and Schur products (double: FP64 path; float:
// mixed path). Errors, chi2, the gradient b and the solution x are FP64 in
// both paths.
//
// Every sum is a fixed-order reduction (per-thread loop, fixed shuffle tree,
// fixed shared-memory tree, partials summed in index order), so results are
// bit-identical run to run; no floating-point atomics.
#pragma once

#include "g2o_math.cuh"
#include "g2oc_internal.h"
#include "reduce.cuh"

namespace g2oc {

// two entries of the storage type in one access
template <typename Real>
struct Vec2;
template <>
struct Vec2<double> {
  using T = double2;
};
template <>
struct Vec2<float> {
  using T = float2;
};

struct BAEdges {
  int n;                  // active edges
  const int2* v;          // (point index, pose index), point-major device order
  const double2* z;       // measurement
  const double4* om;      // (Omega00, Omega01, Omega11, Huber delta; <= 0: none)
  const int* hpl;         // Hpl block per edge or -1
  // om == nullptr: every edge has the information and Huber delta om_const
  // (a uniform graph reads no per-edge record)
  double4 om_const = {0.0, 0.0, 0.0, 0.0};
  // stereo edges (stereo_kernels.cuh) instead of z / om: (u, v, u_right,
  // Huber delta), (O00, O01, O02, O11), (O12, O22)
  const double4* z3 = nullptr;
  const double4* oa3 = nullptr;
  const double2* ob3 = nullptr;
};

struct BACamEdges {       // camera-major copy of the edges of free cameras
  const int* ptr;         // Cf + 1
  const int2* v;
  const double2* z;
  const double4* om;
  const double4* z3 = nullptr;  // stereo, as BAEdges
  double4 om_const = {0.0, 0.0, 0.0, 0.0};  // om == nullptr: as BAEdges
  const double4* oa3 = nullptr;
  const double2* ob3 = nullptr;
};

struct BAVertices {
  double* cam;            // C x 8: qx qy qz qw tx ty tz pad (SE3Quat)
  double* pt;             // P x 4: x y z pad
  const int* free_pose;   // Cf: pose index of Hessian row h
  const int* free_point;  // Pf: point index of landmark l
  double fx, fy, cx, cy;  // EdgeProjectXYZ2UV: fx = fy = focal_length
  double bf = 0.0;        // EdgeStereoSE3ProjectXYZ::bf
};

// the information record of edge k (per edge, or the graph's uniform one)
__device__ __forceinline__ double4 ba_om(const BAEdges& E, int k) { return E.om ? E.om[k] : E.om_const; }
__device__ __forceinline__ double4 ba_om(const BACamEdges& E, int k) { return E.om ? E.om[k] : E.om_const; }

// Per-edge residual, robust weight and weighted error in FP64.
// robust weight = rho'(e^T Omega e) (BaseEdge::robustInformation keeps rho'
// only, g2o/core/base_edge.h:156-162); we = -rho' Omega e
// (BaseFixedSizedEdge::constructQuadraticForm, base_fixed_sized_edge.hpp:48-63).
__device__ __forceinline__ void ba_edge_error(const BAVertices& V, int2 v, double2 z, double4 om,
                                              double e[2], double Xc[3], double& chi2, double& w) {
  const double* cam = V.cam + (size_t)v.y * 8;
  const double* X = V.pt + (size_t)v.x * 4;
  ba_transform(cam, X, Xc);
  e[0] = z.x - (Xc[0] / Xc[2] * V.fx + V.cx);
  e[1] = z.y - (Xc[1] / Xc[2] * V.fy + V.cy);
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
static __global__ void ba_chi2_kernel(BAEdges E, BAVertices V, double* partials) {
  double c = 0.0, r = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < E.n; k += gridDim.x * blockDim.x) {
    double e[2], Xc[3], chi2, w;
    const double4 om = ba_om(E, k);
    ba_edge_error(V, E.v[k], E.z[k], om, e, Xc, chi2, w);
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

// ------------------------------------------------------- structure only
// StructureOnlySolver<3>::calc (g2o/solvers/structure_only/structure_only_solver.h:66-215)
// for every free landmark, the cameras held fixed: each landmark runs its own
// small Levenberg-Marquardt on its 3x3 system (mu = 0.01, nu = 2; stop when
// |b| < 0.001 or after num_max_trials rejected steps), with robust chi2
// rho[0] and the rho'-weighted quadratic form. Landmarks are independent: one
// thread each, its edges the landmark's contiguous device range.
__device__ __forceinline__ double so_robust_chi2(const BAEdges& E, const BAVertices& V, int k0, int k1) {
  double s = 0.0;
  for (int k = k0; k < k1; ++k) {
    double e[2], Xc[3], chi2, w;
    const double4 om = ba_om(E, k);
    ba_edge_error(V, E.v[k], E.z[k], om, e, Xc, chi2, w);
    if (om.w > 0.0) {
      double rho[3];
      huber(chi2, om.w, rho);
      s += rho[0];
    } else {
      s += chi2;
    }
  }
  return s;
}

static __global__ void ba_structure_only(BAEdges E, BAVertices V, const int* l_ptr, int Pf, int num_iters,
                                         int num_max_trials) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= Pf) return;
  double* X = V.pt + (size_t)V.free_point[l] * 4;
  const int k0 = l_ptr[l], k1 = l_ptr[l + 1];
  double chi2 = so_robust_chi2(E, V, k0, k1);
  double mu = 0.01, nu = 2.0;
  bool stop = false;
  for (int ig = 0; ig < num_iters; ++ig) {
    double H[6] = {0, 0, 0, 0, 0, 0};  // 00 01 02 11 12 22
    double b[3] = {0, 0, 0};
    for (int k = k0; k < k1; ++k) {
      double e[2], Xc[3], c2, w;
      const int2 v = E.v[k];
      const double4 om = ba_om(E, k);
      ba_edge_error(V, v, E.z[k], om, e, Xc, c2, w);
      double Jp[6], Jc[12];
      ba_jacobians_from_xc(V.cam + (size_t)v.y * 8, Xc, V.fx, V.fy, Jp, Jc);
      // weightedOmega = rho' Omega, omega_r = -rho' Omega e (constructQuadraticForm)
      const double w00 = w * om.x, w01 = w * om.y, w11 = w * om.z;
      const double r0 = -(om.x * e[0] + om.y * e[1]) * w, r1 = -(om.y * e[0] + om.z * e[1]) * w;
      double WJ[6];  // (rho' Omega) Jp, 2x3
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        WJ[c] = w00 * Jp[c] + w01 * Jp[3 + c];
        WJ[3 + c] = w01 * Jp[c] + w11 * Jp[3 + c];
      }
      H[0] += Jp[0] * WJ[0] + Jp[3] * WJ[3];
      H[1] += Jp[0] * WJ[1] + Jp[3] * WJ[4];
      H[2] += Jp[0] * WJ[2] + Jp[3] * WJ[5];
      H[3] += Jp[1] * WJ[1] + Jp[4] * WJ[4];
      H[4] += Jp[1] * WJ[2] + Jp[4] * WJ[5];
      H[5] += Jp[2] * WJ[2] + Jp[5] * WJ[5];
#pragma unroll
      for (int c = 0; c < 3; ++c) b[c] += Jp[c] * r0 + Jp[3 + c] * r1;
    }
    if (sqrt(b[0] * b[0] + b[1] * b[1] + b[2] * b[2]) < 0.001) break;
    int trial = 0;
    do {
      // LDL^T of H + mu I
      const double a00 = H[0] + mu, a11 = H[3] + mu, a22 = H[5] + mu;
      const double d0 = a00;
      const double l10 = H[1] / d0, l20 = H[2] / d0;
      const double d1 = a11 - l10 * l10 * d0;
      const double l21 = (H[4] - l20 * l10 * d0) / d1;
      const double d2 = a22 - l20 * l20 * d0 - l21 * l21 * d1;
      bool good = false;
      if (d0 > 0.0 && d1 > 0.0 && d2 > 0.0) {
        const double y0 = b[0], y1 = b[1] - l10 * y0, y2 = b[2] - l20 * y0 - l21 * y1;
        const double z2 = y2 / d2, z1 = y1 / d1 - l21 * z2, z0 = y0 / d0 - l10 * z1 - l20 * z2;
        const double old[3] = {X[0], X[1], X[2]};
        X[0] += z0;
        X[1] += z1;
        X[2] += z2;
        const double new_chi2 = so_robust_chi2(E, V, k0, k1);
        if (chi2 - new_chi2 > 0.0 && isfinite(new_chi2)) {
          good = true;
          chi2 = new_chi2;
        } else {
          X[0] = old[0];
          X[1] = old[1];
          X[2] = old[2];
        }
      }
      if (good) {
        mu *= 1.0 / 3.0;
        nu = 2.0;
        break;
      }
      mu *= nu;
      nu *= 2.0;
      if (++trial >= num_max_trials) stop = true;
    } while (!stop);
    if (stop) break;
  }
}

// per-edge errors (parity hook)
static __global__ void ba_errors_kernel(BAEdges E, BAVertices V, double* err) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= E.n) return;
  double e[2], Xc[3], chi2, w;
  ba_edge_error(V, E.v[k], E.z[k], ba_om(E, k), e, Xc, chi2, w);
  err[2 * k] = e[0];
  err[2 * k + 1] = e[1];
}

// per-edge Jacobians in FP64 (parity hook): Jp 2x3, Jc 2x6
static __global__ void ba_jacobians_kernel(BAEdges E, BAVertices V, double* jp, double* jc) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= E.n) return;
  const int2 v = E.v[k];
  const double* cam = V.cam + (size_t)v.y * 8;
  double Xc[3];
  ba_transform(cam, V.pt + (size_t)v.x * 4, Xc);
  double Jp[6], Jc[12];
  ba_jacobians_from_xc(cam, Xc, V.fx, V.fy, Jp, Jc);
  for (int i = 0; i < 6; ++i) jp[6 * k + i] = Jp[i];
  for (int i = 0; i < 12; ++i) jc[12 * k + i] = Jc[i];
}

// Landmark pass of BlockSolver::buildSystem (block_solver.hpp:492-565) for the
// landmark side: one thread per free landmark walks its edges (contiguous in
// the point-major order), accumulates H_ll = sum Jp^T Om' Jp and
// b_l = sum Jp^T we, and writes each Hpl block Jc^T Om' Jp (the transposed
// mapping of block_solver.hpp:210-216). Edges sharing a (camera, landmark)
// block are adjacent and summed in order.
template <typename Real>
__global__ void ba_landmark_pass(BAEdges E, BAVertices V, const int* l_ptr, int Pf, Real* hll, Real* hpl,
                                 double* b_l) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= Pf) return;
  Real H[6] = {0, 0, 0, 0, 0, 0};
  double bl[3] = {0, 0, 0};
  Real B[18];
  int cur = -1;
  const int k1 = l_ptr[l + 1];
  for (int k = l_ptr[l]; k < k1; ++k) {
    const int2 v = E.v[k];
    const double4 om = ba_om(E, k);
    double e[2], Xc[3], chi2, w;
    ba_edge_error(V, v, E.z[k], om, e, Xc, chi2, w);
    const double* cam = V.cam + (size_t)v.y * 8;
    double Jpd[6], Jcd[12];
    ba_jacobians_from_xc(cam, Xc, V.fx, V.fy, Jpd, Jcd);
    Real Jp[6], Jc[12];
#pragma unroll
    for (int i = 0; i < 6; ++i) Jp[i] = (Real)Jpd[i];
#pragma unroll
    for (int i = 0; i < 12; ++i) Jc[i] = (Real)Jcd[i];
    const double we0 = -w * (om.x * e[0] + om.y * e[1]);
    const double we1 = -w * (om.y * e[0] + om.z * e[1]);
    const Real o00 = (Real)(w * om.x), o01 = (Real)(w * om.y), o11 = (Real)(w * om.z);
    // AtO = Jp^T Om' (3x2)
    Real A0[3], A1[3];
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
    for (int i = 0; i < 3; ++i) bl[i] += Jpd[i] * we0 + Jpd[3 + i] * we1;
    const int blk = E.hpl[k];
    if (blk >= 0) {
      if (blk != cur) {
        if (cur >= 0) {
#pragma unroll
          for (int i = 0; i < 18; ++i) hpl[(size_t)cur * 18 + i] = B[i];
        }
#pragma unroll
        for (int i = 0; i < 18; ++i) B[i] = Real(0);
        cur = blk;
      }
      // B(6x3) += Jc^T (Om' Jp) = Jc^T (AtO)^T
#pragma unroll
      for (int r = 0; r < 6; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) B[r * 3 + c] += Jc[r] * A0[c] + Jc[6 + r] * A1[c];
    }
  }
  if (cur >= 0) {
#pragma unroll
    for (int i = 0; i < 18; ++i) hpl[(size_t)cur * 18 + i] = B[i];
  }
#pragma unroll
  for (int i = 0; i < 6; ++i) hll[(size_t)l * 6 + i] = H[i];
#pragma unroll
  for (int i = 0; i < 3; ++i) b_l[(size_t)l * 3 + i] = bl[i];
}

// Landmark pass, edge-parallel form (graphs whose landmarks have at most 32
// edges and whose (camera, landmark) pairs are unique): one warp per chunk of
// whole landmarks (at most 32 edges, packed on the host), one lane per edge.
// Edge loads are coalesced. The Hpl blocks of a chunk's edges are one
// contiguous range (one block per edge of a free camera, numbered in edge
// order): each lane puts its block in shared memory and the warp stores the
// range with coalesced pair stores. H_ll and b_l are summed by a segmented
// warp scan keyed by landmark (fixed shuffle order), written by the segment's
// last lane. Launched with 256 threads (8 warps).
template <typename Real>
__global__ void __launch_bounds__(256) ba_landmark_warp(BAEdges E, BAVertices V, const int* chunk_ptr, int nchunks, const int* e_lm,
                                 Real* hll, Real* hpl, double* b_l) {
  using R2 = typename Vec2<Real>::T;
  __shared__ R2 stage[8][32 * 9];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int ch = blockIdx.x * (blockDim.x >> 5) + wid;
  if (ch >= nchunks) return;
  const int e0 = chunk_ptr[ch], e1 = chunk_ptr[ch + 1];
  const int k = e0 + lane;
  const bool act = k < e1;
  Real H[6] = {0, 0, 0, 0, 0, 0};
  double bl[3] = {0, 0, 0};
  int key = -1 - lane;  // distinct for idle lanes
  const int blk = act ? E.hpl[k] : -1;
  const unsigned has = __ballot_sync(0xffffffffu, blk >= 0);
  const int blk0 = (int)__reduce_min_sync(0xffffffffu, blk >= 0 ? (unsigned)blk : 0x7fffffffu);
  if (act) {
    key = e_lm[k];
    const int2 v = E.v[k];
    const double4 om = ba_om(E, k);
    double e[2], Xc[3], chi2, w;
    ba_edge_error(V, v, E.z[k], om, e, Xc, chi2, w);
    double Jpd[6], Jcd[12];
    ba_jacobians_from_xc(V.cam + (size_t)v.y * 8, Xc, V.fx, V.fy, Jpd, Jcd);
    Real Jp[6], Jc[12];
#pragma unroll
    for (int i = 0; i < 6; ++i) Jp[i] = (Real)Jpd[i];
#pragma unroll
    for (int i = 0; i < 12; ++i) Jc[i] = (Real)Jcd[i];
    const double we0 = -w * (om.x * e[0] + om.y * e[1]);
    const double we1 = -w * (om.y * e[0] + om.z * e[1]);
    const Real o00 = (Real)(w * om.x), o01 = (Real)(w * om.y), o11 = (Real)(w * om.z);
    Real A0[3], A1[3];
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
    for (int i = 0; i < 3; ++i) bl[i] = Jpd[i] * we0 + Jpd[3 + i] * we1;
    if (blk >= 0) {
      Real hb[18];
#pragma unroll
      for (int r = 0; r < 6; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c) hb[r * 3 + c] = Jc[r] * A0[c] + Jc[6 + r] * A1[c];
      R2* o = &stage[wid][(blk - blk0) * 9];
#pragma unroll
      for (int q = 0; q < 9; ++q) {
        R2 t;
        t.x = hb[2 * q];
        t.y = hb[2 * q + 1];
        o[q] = t;
      }
    }
  }
  // segmented inclusive scan by landmark
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const int ko = __shfl_up_sync(0xffffffffu, key, off);
    Real Ho[6];
    double bo[3];
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
  // the chunk's Hpl range (8-byte aligned in FP32, 16 in FP64), coalesced
  __syncwarp();
  const int npair = __popc(has) * 9;
  if (npair > 0) {
    R2* out = reinterpret_cast<R2*>(hpl + (size_t)blk0 * 18);
    for (int i = lane; i < npair; i += 32) out[i] = stage[wid][i];
  }
}

// Camera pass: one CTA per free camera sums H_pp = sum Jc^T Om' Jc (21 unique)
// and b_p = sum Jc^T we over the camera's edges with a fixed-order block
// reduction, and writes the full 6x6 block.
template <typename Real, int THREADS>
__global__ void __launch_bounds__(THREADS) ba_camera_pass(BACamEdges CE, BAVertices V, Real* hpp, double* b_p) {
  const int h = blockIdx.x;
  Real H[21];
  double bp[6];
#pragma unroll
  for (int i = 0; i < 21; ++i) H[i] = Real(0);
#pragma unroll
  for (int i = 0; i < 6; ++i) bp[i] = 0.0;
  const int j1 = CE.ptr[h + 1];
  // the next edge's record is loaded while this one's point is
  int j = CE.ptr[h] + threadIdx.x;
  int2 vn = make_int2(0, 0);
  double2 zn = make_double2(0.0, 0.0);
  double4 omn = make_double4(0.0, 0.0, 0.0, 0.0);
  if (j < j1) {
    vn = CE.v[j];
    zn = CE.z[j];
    omn = ba_om(CE, j);
  }
  for (; j < j1; j += THREADS) {
    const int2 v = vn;
    const double2 z = zn;
    const double4 om = omn;
    if (j + THREADS < j1) {
      vn = CE.v[j + THREADS];
      zn = CE.z[j + THREADS];
      omn = ba_om(CE, j + THREADS);
    }
    double e[2], Xc[3], chi2, w;
    ba_edge_error(V, v, z, om, e, Xc, chi2, w);
    const double* cam = V.cam + (size_t)v.y * 8;
    double Jpd[6], Jcd[12];
    ba_jacobians_from_xc(cam, Xc, V.fx, V.fy, Jpd, Jcd);
    Real Jc[12];
#pragma unroll
    for (int i = 0; i < 12; ++i) Jc[i] = (Real)Jcd[i];
    const double we0 = -w * (om.x * e[0] + om.y * e[1]);
    const double we1 = -w * (om.y * e[0] + om.z * e[1]);
    const Real o00 = (Real)(w * om.x), o01 = (Real)(w * om.y), o11 = (Real)(w * om.z);
    Real A0[6], A1[6];
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      A0[i] = Jc[i] * o00 + Jc[6 + i] * o01;
      A1[i] = Jc[i] * o01 + Jc[6 + i] * o11;
    }
    int t = 0;
#pragma unroll
    for (int r = 0; r < 6; ++r)
#pragma unroll
      for (int c = r; c < 6; ++c) H[t++] += A0[r] * Jc[c] + A1[r] * Jc[6 + c];
#pragma unroll
    for (int i = 0; i < 6; ++i) bp[i] += Jcd[i] * we0 + Jcd[6 + i] * we1;
  }
  __shared__ double red[THREADS / 32][27];
  block_sum_array<Real, 21, THREADS>(H, &red[0][0]);
  block_sum_array<double, 6, THREADS>(bp, &red[0][0]);
  if (threadIdx.x == 0) {
    Real* out = hpp + (size_t)h * 36;
    int t = 0;
    for (int r = 0; r < 6; ++r)
      for (int c = r; c < 6; ++c) {
        out[r * 6 + c] = H[t];
        out[c * 6 + r] = H[t];
        ++t;
      }
    for (int i = 0; i < 6; ++i) b_p[(size_t)h * 6 + i] = bp[i];
  }
}

// ---------------------------------------------------------------- Schur
// Landmark step of the Schur loop (block_solver.hpp:359-378):
// Dinv = (H_ll + lambda I)^-1 and BD_a = B_a Dinv for every Hpl block a of
// the landmark, written in camera-major order (bdc[hc_index[a]]) so a camera
// row's blocks are contiguous for the Schur row kernel.
template <typename Real>
__global__ void schur_landmark(const Real* hll, const Real* hpl, const int* hb_ptr, const int* hc_index, int Pf,
                               double lambda_all, const double* lambda_of, Real* dinv, Real* bdc, int* nonfinite) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= Pf) return;
  const double lambda = lambda_of ? lambda_of[l] : lambda_all;  // per landmark (batched windows)
  const Real* h = hll + (size_t)l * 6;
  double A[9] = {(double)h[0] + lambda, (double)h[1], (double)h[2],
                 (double)h[1], (double)h[3] + lambda, (double)h[4],
                 (double)h[2], (double)h[4], (double)h[5] + lambda};
  double Di[9];
  if (!inverse3(A, Di)) *nonfinite = 1;
  Real D[9];
#pragma unroll
  for (int i = 0; i < 9; ++i) {
    D[i] = (Real)Di[i];
    dinv[(size_t)l * 9 + i] = D[i];
  }
  if (!bdc) return;
  const int b1 = hb_ptr[l + 1];
  for (int a = hb_ptr[l]; a < b1; ++a) {
    const Real* B = hpl + (size_t)a * 18;
    Real* o = bdc + (size_t)hc_index[a] * 18;
#pragma unroll
    for (int r = 0; r < 6; ++r)
#pragma unroll
      for (int c = 0; c < 3; ++c) o[r * 3 + c] = B[r * 3] * D[c] + B[r * 3 + 1] * D[3 + c] + B[r * 3 + 2] * D[6 + c];
  }
}

// One 6 x 3 Hpl block (18 values, row-major) into registers. FP32 blocks are
// 72 bytes at a 72-byte stride: a block starts on a 16-byte boundary when its
// index is even (four 16-byte loads, then 8 bytes) and on an 8-byte one when
// odd (8 bytes, then four 16-byte loads): five loads instead of nine. FP64
// blocks (144 bytes) are nine 16-byte loads.
template <bool VEC>
__device__ __forceinline__ void ldg_block18(const float* hpl, int blk, float (&b)[18]) {
  const float* base = hpl + (size_t)blk * 18;
  if (VEC) {
    const bool odd = blk & 1;
    const int o4 = odd ? 2 : 0;
    const float4 u0 = __ldg(reinterpret_cast<const float4*>(base + o4));
    const float4 u1 = __ldg(reinterpret_cast<const float4*>(base + o4 + 4));
    const float4 u2 = __ldg(reinterpret_cast<const float4*>(base + o4 + 8));
    const float4 u3 = __ldg(reinterpret_cast<const float4*>(base + o4 + 12));
    const float2 w = __ldg(reinterpret_cast<const float2*>(base + (odd ? 0 : 16)));
    const float q[18] = {u0.x, u0.y, u0.z, u0.w, u1.x, u1.y, u1.z, u1.w, u2.x,
                         u2.y, u2.z, u2.w, u3.x, u3.y, u3.z, u3.w, w.x,  w.y};
#pragma unroll
    for (int t = 0; t < 18; ++t) b[t] = odd ? (t < 2 ? q[16 + t] : q[t - 2]) : q[t];
  } else {
    const float2* B2 = reinterpret_cast<const float2*>(base);
#pragma unroll
    for (int t = 0; t < 9; ++t) {
      const float2 v = __ldg(B2 + t);
      b[2 * t] = v.x;
      b[2 * t + 1] = v.y;
    }
  }
}
template <bool VEC>
__device__ __forceinline__ void ldg_block18(const double* hpl, int blk, double (&b)[18]) {
  const double2* B2 = reinterpret_cast<const double2*>(hpl + (size_t)blk * 18);
#pragma unroll
  for (int t = 0; t < 9; ++t) {
    const double2 v = __ldg(B2 + t);
    b[2 * t] = v.x;
    b[2 * t + 1] = v.y;
  }
}

// Dense output of the Schur rows for batched windows: each camera row belongs
// to one window, whose reduced system is a dense FP64 matrix (n + 1 rows of
// n, row-major, at M + mat[w]; the last row holds the right-hand side). Only
// the lower triangle is written: the diagonal blocks whole, each upper block
// (r, c) transposed into block (c, r).
struct DenseOut {
  const int* win_of_cam;  // window of each camera row
  const int* cam;         // first camera row of each window (nw + 1)
  const long long* mat;   // offset of each window's matrix in M
  double* M;              // nullptr: no dense output
};


// Schur complement by camera rows (block_solver.hpp:343-433): one CTA per
// free camera r stages the camera's BD_a blocks (contiguous in bdc) in shared
// memory with coalesced loads. The diagonal block S(r, r) = Hpp(r) + lambda I
// - sum_a BD_a B_a^T over all of the camera's landmarks is reduced by the
// whole CTA (fixed assignment and tree); each off-diagonal block (r, c) is
// summed by two lanes (lane parity = rows 0-2 or 3-5, 18 FP64 accumulators
// each) over its co-observing pairs in landmark order, with B_b from L1/L2.
// With bs != nullptr the reduced right-hand side bs_r = b_r - sum_a BD_a
// b_l(a) is formed from the same staged blocks. S is written in the row-SoA
// layout of sys_offset.
// G = lanes per off-diagonal block: lane pairs split the block's 6 rows in two
// halves and the G / 2 pairs of a group split its pair list (partial sums
// combined by a fixed xor tree). rows: the camera rows of this launch (or
// nullptr: row = blockIdx.x); the row's G is chosen from its pair-list lengths.
// tiles != nullptr: S is written straight into the dense tiles of the tile PCG
// (block k at tile_off[k], scalar rows 96 apart; an off-diagonal block inside
// a diagonal tile also into its transposed place) instead of the row-SoA;
// dn.M != nullptr: into the windows' dense matrices (DenseOut) instead.
// block_order (or nullptr: storage order): per row, the off-diagonal block j
// that the q-th lane group of a round takes, block_order[rptr[r] + q].
template <typename Real, int THREADS, bool STAGE, int G = 2, bool VEC = false>
__global__ void __launch_bounds__(THREADS, sizeof(Real) == 4 ? 2 : 1)
    schur_rows(const int* rows, const int* hc_ptr, const int* hc_blk, const int* hc_col, const Real* hpl,
               const Real* dinv, const Real* bdc, const int* rptr, const int* rcol, const int* pair_ptr,
               const int2* pairs, const int* block_order, const int* s_hpp, const Real* hpp, double lambda_all, const double* lambda_of, Real* S,
               Real* tiles, const int* tile_off, DenseOut dn, const double* b_p, const double* b_l, double* bs,
               int bds) {
  constexpr int TS = kTileBlocks * 6;  // scalar row stride of a tile
  static_assert(G >= 2 && G <= 32 && (G & (G - 1)) == 0, "lanes per block: a power of two in [2, 32]");
  using R2 = typename Vec2<Real>::T;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  __shared__ double red[THREADS / 32][27];
  const int r = rows ? rows[blockIdx.x] : blockIdx.x;
  const double lambda = lambda_of ? lambda_of[r] : lambda_all;  // per camera row (batched windows)
  const int a0 = hc_ptr[r], na = hc_ptr[r + 1] - a0;
  const int rb = rptr[r], nblk = rptr[r + 1] - rb;
  Real* Sr = S + (size_t)rb * 36;
  // dense output: the window's matrix, its row length and this row's first index
  double* Md = nullptr;
  int dn_n = 0, dn_h0 = 0;
  if (dn.M) {
    const int w = dn.win_of_cam[r];
    dn_h0 = dn.cam[w];
    dn_n = 6 * (dn.cam[w + 1] - dn_h0);
    Md = dn.M + dn.mat[w];
  }
  // One pass over the camera's Hpl blocks B_a, one thread per block: BD_a =
  // B_a Dinv_l, staged in shared memory (or, for cameras with more blocks
  // than shared memory holds, written to the camera-major scratch bdc and read
  // back in place); with B_a still in registers, its diagonal-block term
  // BD_a B_a^T (upper 21 entries) and its right-hand-side term BD_a b_l.
  // staged BD blocks: bds entries apart, rows 0-2 at 0 and rows 3-5 at bds / 2
  // (bds = 24 in FP32: each half starts on a 16-byte boundary, read with two
  // 16-byte loads and one 4-byte load; else 18, packed)
  if (!STAGE) bds = 18;
  const int bhalf = bds / 2;
  Real* BDw = STAGE ? reinterpret_cast<Real*>(smem_raw) : const_cast<Real*>(bdc) + (size_t)a0 * 18;
  Real dacc[21];
  double racc[6] = {0, 0, 0, 0, 0, 0};
#pragma unroll
  for (int u = 0; u < 21; ++u) dacc[u] = 0;
  // the next block's indices are loaded while this one's Hpl and Dinv are
  int a_next = 0, l_next = 0;
  if ((int)threadIdx.x < na) {
    a_next = hc_blk[a0 + threadIdx.x];
    l_next = hc_col[a0 + threadIdx.x];
  }
  for (int t = threadIdx.x; t < na; t += THREADS) {
    const int a = a_next, l = l_next;
    if (t + THREADS < na) {
      a_next = hc_blk[a0 + t + THREADS];
      l_next = hc_col[a0 + t + THREADS];
    }
    const Real* Dl = dinv + (size_t)l * 9;
    Real b[18], D[9], bd[18];
    ldg_block18<VEC>(hpl, a, b);
#pragma unroll
    for (int q = 0; q < 9; ++q) D[q] = Dl[q];
    Real* o = BDw + (size_t)t * bds;
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        bd[i * 3 + c] = b[i * 3] * D[c] + b[i * 3 + 1] * D[3 + c] + b[i * 3 + 2] * D[6 + c];
        o[(i / 3) * bhalf + (i % 3) * 3 + c] = bd[i * 3 + c];
      }
    int u = 0;
#pragma unroll
    for (int i = 0; i < 6; ++i)
#pragma unroll
      for (int c = i; c < 6; ++c, ++u)
        dacc[u] += bd[i * 3] * b[c * 3] + bd[i * 3 + 1] * b[c * 3 + 1] + bd[i * 3 + 2] * b[c * 3 + 2];
    if (bs) {
      const double* bl = b_l + (size_t)l * 3;
#pragma unroll
      for (int q = 0; q < 6; ++q)
        racc[q] += (double)bd[q * 3] * bl[0] + (double)bd[q * 3 + 1] * bl[1] + (double)bd[q * 3 + 2] * bl[2];
    }
  }
  if (!STAGE) __threadfence_block();
  // fixed-order CTA sum of the 21 diagonal-block and 6 right-hand-side terms:
  // warp sums, then term u summed over the warps in order by thread u, which
  // writes its entry (and its mirror) of the diagonal block or of bs. The
  // barrier also publishes the staged BD.
  {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double acc[27];
#pragma unroll
    for (int u = 0; u < 21; ++u) acc[u] = (double)dacc[u];
#pragma unroll
    for (int q = 0; q < 6; ++q) acc[21 + q] = racc[q];
#pragma unroll
    for (int u = 0; u < 27; ++u) acc[u] = warp_sum(acc[u]);
    if (lane == 0) {
#pragma unroll
      for (int u = 0; u < 27; ++u) red[warp][u] = acc[u];
    }
    __syncthreads();
    const int u = threadIdx.x;
    if (u < 27) {
      double sum = red[0][u];
#pragma unroll
      for (int w = 1; w < THREADS / 32; ++w) sum += red[w][u];
      if (u < 21) {
        int i = 0, c = u;  // u -> (i, c), i <= c, row by row
        while (c >= 6 - i) {
          c -= 6 - i;
          ++i;
        }
        c += i;
        const int hb = s_hpp[rb];
        Real* Td = tiles ? tiles + tile_off[rb] : nullptr;
        double* Dd = Md ? Md + (size_t)(r - dn_h0) * 6 * dn_n + (r - dn_h0) * 6 : nullptr;
        double v = -sum + (i == c ? lambda : 0.0);
        if (hb >= 0) v += (double)hpp[(size_t)hb * 36 + i * 6 + c];
        if (Td) Td[i * TS + c] = (Real)v;
        else if (Dd) Dd[(size_t)i * dn_n + c] = (double)(Real)v;
        else Sr[(size_t)(i * 6 + c) * nblk] = (Real)v;
        if (c != i) {
          double w = -sum;
          if (hb >= 0) w += (double)hpp[(size_t)hb * 36 + c * 6 + i];
          if (Td) Td[c * TS + i] = (Real)w;
          else if (Dd) Dd[(size_t)c * dn_n + i] = (double)(Real)w;
          else Sr[(size_t)(c * 6 + i) * nblk] = (Real)w;
        }
      } else if (bs) {
        bs[(size_t)r * 6 + (u - 21)] = b_p[(size_t)r * 6 + (u - 21)] - sum;
      }
    }
  }
  const Real* BDa = BDw;
  // off-diagonal blocks (the row's diagonal is its first block); the loop
  // runs the same number of times in every lane, so the group reduction's
  // shuffles see full warps
  const int half = threadIdx.x & 1, sub = (threadIdx.x % G) >> 1;
  for (int j0 = 1; j0 < nblk; j0 += THREADS / G) {
    const int q = j0 + (int)threadIdx.x / G;
    const bool valid = q < nblk;
    const int j = (valid && block_order) ? block_order[rb + q] : q;
    const int k = rb + j;
    // pair products summed in the storage type (FP64 on the FP64 path; FP32
    // on the mixed path, whose S is stored in FP32), added to Hpp in FP64
    Real acc[18];
#pragma unroll
    for (int t = 0; t < 18; ++t) acc[t] = 0;
    // two pairs per step: their index and Hpl loads are independent, so two
    // gathers are in flight per thread; accumulation stays in pair order.
    // The pair list and S are touched once per pass: streamed (evict-first
    // loads and stores), so the L2 lines go to the Hpl blocks gathered again
    auto load_b = [&](int blk, Real (&b)[18]) { ldg_block18<VEC>(hpl, blk, b); };
    auto accum = [&](int a, const Real (&b)[18]) {
      const Real* D = BDa + (size_t)a * bds + half * bhalf;
      Real d[9];
      if (sizeof(Real) == 4 && bds == 24) {
        const float4 d0 = *reinterpret_cast<const float4*>(D);
        const float4 d1 = *reinterpret_cast<const float4*>(D + 4);
        d[0] = d0.x; d[1] = d0.y; d[2] = d0.z; d[3] = d0.w;
        d[4] = d1.x; d[5] = d1.y; d[6] = d1.z; d[7] = d1.w;
        d[8] = D[8];
      } else {
#pragma unroll
        for (int t = 0; t < 9; ++t) d[t] = D[t];
      }
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int c = 0; c < 6; ++c)
          acc[i * 6 + c] += d[i * 3] * b[c * 3] + d[i * 3 + 1] * b[c * 3 + 1] + d[i * 3 + 2] * b[c * 3 + 2];
    };
    constexpr int STEP = G / 2;  // this lane's pairs: p0 + sub, p0 + sub + STEP, ...
    int p = valid ? pair_ptr[k] + sub : 0;
    const int p1 = valid ? pair_ptr[k + 1] : 0;
    // the next step's pair indices are loaded while this step's blocks are
    int2 na2 = make_int2(0, 0), nb2 = make_int2(0, 0);
    if (p < p1) na2 = __ldcs(pairs + p);
    if (p + STEP < p1) nb2 = __ldcs(pairs + p + STEP);
    for (; p + STEP < p1; p += 2 * STEP) {
      const int2 pa = na2, pb = nb2;
      if (p + 2 * STEP < p1) na2 = __ldcs(pairs + p + 2 * STEP);
      if (p + 3 * STEP < p1) nb2 = __ldcs(pairs + p + 3 * STEP);
      Real ba[18], bb[18];
      load_b(pa.y, ba);
      load_b(pb.y, bb);
      accum(pa.x, ba);
      accum(pb.x, bb);
    }
    if (p < p1) {
      const int2 pa = na2;
      Real ba[18];
      load_b(pa.y, ba);
      accum(pa.x, ba);
    }
#pragma unroll
    for (int off = 2; off < G; off <<= 1)
#pragma unroll
      for (int t = 0; t < 18; ++t) acc[t] += __shfl_xor_sync(0xffffffffu, acc[t], off);
    if (valid && sub == 0) {
      const int hb = s_hpp[k];
      Real v[18];
#pragma unroll
      for (int i = 0; i < 3; ++i)
#pragma unroll
        for (int c = 0; c < 6; ++c) {
          const int e = (half * 3 + i) * 6 + c;
          double w = -(double)acc[i * 6 + c];
          if (hb >= 0) w += (double)hpp[(size_t)hb * 36 + e];
          v[i * 6 + c] = (Real)w;
        }
      if (tiles) {
        // this lane's three scalar rows of the block: six contiguous entries each
        const int off = tile_off[k];
        Real* T = tiles + off + half * 3 * TS;
        // (six entries of a row start on an 8-byte boundary in FP32: pairs)
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int c = 0; c < 6; c += 2) {
            R2 pr;
            pr.x = v[i * 6 + c];
            pr.y = v[i * 6 + c + 1];
            __stcs(reinterpret_cast<R2*>(T + i * TS + c), pr);
          }
        const int cc = rcol[k];
        if (r / kTileBlocks == cc / kTileBlocks) {
          Real* base = tiles + (size_t)(off / (TS * TS)) * (TS * TS);
          const int lr = (r % kTileBlocks) * 6 + half * 3, lc = (cc % kTileBlocks) * 6;
#pragma unroll
          for (int i = 0; i < 3; ++i)
#pragma unroll
            for (int c = 0; c < 6; ++c) __stcs(base + (lc + c) * TS + lr + i, v[i * 6 + c]);
        }
      } else if (Md) {
        // block (r, cc) transposed into the lower triangle: entry (3h + i, c)
        // at row (cc - h0) * 6 + c, column (r - h0) * 6 + 3h + i
        const int cc = rcol[k];
        double* D = Md + (size_t)(cc - dn_h0) * 6 * dn_n + (r - dn_h0) * 6 + half * 3;
#pragma unroll
        for (int c = 0; c < 6; ++c)
#pragma unroll
          for (int i = 0; i < 3; ++i) D[(size_t)c * dn_n + i] = (double)v[i * 6 + c];
      } else {
#pragma unroll
        for (int i = 0; i < 3; ++i)
#pragma unroll
          for (int c = 0; c < 6; ++c) __stcs(Sr + (size_t)((half * 3 + i) * 6 + c) * nblk + j, v[i * 6 + c]);
      }
    }
  }
}

// db_l = Dinv_l r_l
template <typename Real>
__global__ void schur_db(const Real* dinv, const double* r_l, int Pf, double* db) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= Pf) return;
  const Real* D = dinv + (size_t)l * 9;
  const double* rl = r_l + (size_t)l * 3;
#pragma unroll
  for (int i = 0; i < 3; ++i)
    db[(size_t)l * 3 + i] = (double)D[i * 3] * rl[0] + (double)D[i * 3 + 1] * rl[1] + (double)D[i * 3 + 2] * rl[2];
}

// Reduced right-hand side for a given (r_p, r_l) (block_solver.hpp:366-392,
// 429-433): one CTA per free camera, bs = r_p - sum_a B_a db_l(a), threads
// over the camera's Hpl blocks (camera-major lists), fixed-order reduction.
template <typename Real, int THREADS>
__global__ void __launch_bounds__(THREADS) schur_rhs(const int* hc_ptr, const int* hc_blk, const int* hc_col,
                                                     const Real* hpl, const double* db, const double* r_p,
                                                     double* bs) {
  const int h = blockIdx.x;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  const int e1 = hc_ptr[h + 1];
  for (int p = hc_ptr[h] + threadIdx.x; p < e1; p += THREADS) {
    const int a = hc_blk[p];
    const double* d = db + (size_t)hc_col[p] * 3;
    const Real* B = hpl + (size_t)a * 18;
#pragma unroll
    for (int q = 0; q < 6; ++q) acc[q] += (double)B[q * 3] * d[0] + (double)B[q * 3 + 1] * d[1] + (double)B[q * 3 + 2] * d[2];
  }
  __shared__ double red[THREADS / 32][6];
  block_sum_array<double, 6, THREADS>(acc, &red[0][0]);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < 6; ++q) bs[(size_t)h * 6 + q] = r_p[(size_t)h * 6 + q] - acc[q];
  }
}

// Landmark back-substitution (block_solver.hpp:449-474):
// x_l = Dinv (r_l - sum_a B_a^T x_p(row a))
template <typename Real>
__global__ void ba_backsub(const int* hb_ptr, const int* hpl_row, int Pf, const Real* hpl, const Real* dinv,
                           const double* r_l, const double* x_p, double* x_l) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= Pf) return;
  double cl[3] = {r_l[(size_t)l * 3], r_l[(size_t)l * 3 + 1], r_l[(size_t)l * 3 + 2]};
  const int b1 = hb_ptr[l + 1];
  for (int a = hb_ptr[l]; a < b1; ++a) {
    const Real* B = hpl + (size_t)a * 18;
    const double* xp = x_p + (size_t)hpl_row[a] * 6;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      double s = 0.0;
#pragma unroll
      for (int r = 0; r < 6; ++r) s += (double)B[r * 3 + c] * xp[r];
      cl[c] -= s;
    }
  }
  const Real* D = dinv + (size_t)l * 9;
#pragma unroll
  for (int i = 0; i < 3; ++i)
    x_l[(size_t)l * 3 + i] = (double)D[i * 3] * cl[0] + (double)D[i * 3 + 1] * cl[1] + (double)D[i * 3 + 2] * cl[2];
}

// Back-substitution, one warp per chunk of whole landmarks (lane per edge,
// each edge of a free camera owns one Hpl block when the chunks exist),
// segmented warp scan by landmark.
template <typename Real>
__global__ void ba_backsub_warp(const int* e_hpl, const int* hpl_row, const int* chunk_ptr, int nchunks,
                                const int* e_lm, const Real* hpl, const Real* dinv, const double* r_l,
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
      const Real* B = hpl + (size_t)blk * 18;
      const double* xp = x_p + (size_t)hpl_row[blk] * 6;
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        double t = 0.0;
#pragma unroll
        for (int r = 0; r < 6; ++r) t += (double)B[r * 3 + c] * xp[r];
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
    const Real* D = dinv + (size_t)key * 9;
#pragma unroll
    for (int i = 0; i < 3; ++i)
      x_l[(size_t)key * 3 + i] = (double)D[i * 3] * cl[0] + (double)D[i * 3 + 1] * cl[1] + (double)D[i * 3 + 2] * cl[2];
  }
}

// Matrix-free FP64 residual of the damped normal equations for the
// mixed-precision refinement, r = b - (J^T Om' J + lambda I) x, with the
// Jacobians recomputed in FP64 from the edges (no FP32 Hessian involved).
// Landmark side: one thread per free landmark over its edges.
static __global__ void ba_resid64_landmark(BAEdges E, BAVertices V, const int* l_ptr, int Pf, const int* pose_h,
                                    double lambda, const double* b_l, const double* x_p, const double* x_l,
                                    double* r_l) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= Pf) return;
  const double* xl = x_l + (size_t)l * 3;
  double acc[3] = {lambda * xl[0], lambda * xl[1], lambda * xl[2]};
  const int k1 = l_ptr[l + 1];
  for (int k = l_ptr[l]; k < k1; ++k) {
    const int2 v = E.v[k];
    const double4 om = ba_om(E, k);
    double e[2], Xc[3], chi2, w;
    ba_edge_error(V, v, E.z[k], om, e, Xc, chi2, w);
    double Jp[6], Jc[12];
    ba_jacobians_from_xc(V.cam + (size_t)v.y * 8, Xc, V.fx, V.fy, Jp, Jc);
    double u0 = Jp[0] * xl[0] + Jp[1] * xl[1] + Jp[2] * xl[2];
    double u1 = Jp[3] * xl[0] + Jp[4] * xl[1] + Jp[5] * xl[2];
    const int h = pose_h[v.y];
    if (h >= 0) {
      const double* xp = x_p + (size_t)h * 6;
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        u0 += Jc[q] * xp[q];
        u1 += Jc[6 + q] * xp[q];
      }
    }
    const double o0 = w * (om.x * u0 + om.y * u1), o1 = w * (om.y * u0 + om.z * u1);
#pragma unroll
    for (int i = 0; i < 3; ++i) acc[i] += Jp[i] * o0 + Jp[3 + i] * o1;
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) r_l[(size_t)l * 3 + i] = b_l[(size_t)l * 3 + i] - acc[i];
}

// Landmark side, one warp per chunk of whole landmarks (<= 32 edges, lane
// per edge) with a segmented warp scan, as ba_landmark_warp.
static __global__ void ba_resid64_landmark_warp(BAEdges E, BAVertices V, const int* chunk_ptr, int nchunks,
                                                const int* e_lm, const int* pose_h, double lambda, const double* b_l,
                                                const double* x_p, const double* x_l, double* r_l) {
  const int lane = threadIdx.x & 31;
  const int ch = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (ch >= nchunks) return;
  const int e0 = chunk_ptr[ch], e1 = chunk_ptr[ch + 1];
  const int k = e0 + lane;
  const bool act = k < e1;
  double acc[3] = {0, 0, 0};
  int key = -1 - lane;  // distinct for idle lanes
  if (act) {
    key = e_lm[k];
    const double* xl = x_l + (size_t)key * 3;
    const int2 v = E.v[k];
    const double4 om = ba_om(E, k);
    double e[2], Xc[3], chi2, w;
    ba_edge_error(V, v, E.z[k], om, e, Xc, chi2, w);
    double Jp[6], Jc[12];
    ba_jacobians_from_xc(V.cam + (size_t)v.y * 8, Xc, V.fx, V.fy, Jp, Jc);
    double u0 = Jp[0] * xl[0] + Jp[1] * xl[1] + Jp[2] * xl[2];
    double u1 = Jp[3] * xl[0] + Jp[4] * xl[1] + Jp[5] * xl[2];
    const int h = pose_h[v.y];
    if (h >= 0) {
      const double* xp = x_p + (size_t)h * 6;
#pragma unroll
      for (int q = 0; q < 6; ++q) {
        u0 += Jc[q] * xp[q];
        u1 += Jc[6 + q] * xp[q];
      }
    }
    const double o0 = w * (om.x * u0 + om.y * u1), o1 = w * (om.y * u0 + om.z * u1);
#pragma unroll
    for (int i = 0; i < 3; ++i) acc[i] = Jp[i] * o0 + Jp[3 + i] * o1;
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
    const double* xl = x_l + (size_t)key * 3;
#pragma unroll
    for (int i = 0; i < 3; ++i) r_l[(size_t)key * 3 + i] = b_l[(size_t)key * 3 + i] - lambda * xl[i] - acc[i];
  }
}

// Camera side: one CTA per free camera over its edges, fixed-order reduction.
template <int THREADS>
__global__ void __launch_bounds__(THREADS) ba_resid64_camera(BACamEdges CE, BAVertices V, const int* point_l,
                                                             double lambda, const double* b_p, const double* x_p,
                                                             const double* x_l, double* r_p) {
  const int h = blockIdx.x;
  const double* xp = x_p + (size_t)h * 6;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  const int j1 = CE.ptr[h + 1];
  for (int j = CE.ptr[h] + threadIdx.x; j < j1; j += THREADS) {
    const int2 v = CE.v[j];
    const double4 om = ba_om(CE, j);
    double e[2], Xc[3], chi2, w;
    ba_edge_error(V, v, CE.z[j], om, e, Xc, chi2, w);
    double Jp[6], Jc[12];
    ba_jacobians_from_xc(V.cam + (size_t)v.y * 8, Xc, V.fx, V.fy, Jp, Jc);
    double u0 = 0.0, u1 = 0.0;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      u0 += Jc[q] * xp[q];
      u1 += Jc[6 + q] * xp[q];
    }
    const int l = point_l[v.x];
    if (l >= 0) {
      const double* xl = x_l + (size_t)l * 3;
      u0 += Jp[0] * xl[0] + Jp[1] * xl[1] + Jp[2] * xl[2];
      u1 += Jp[3] * xl[0] + Jp[4] * xl[1] + Jp[5] * xl[2];
    }
    const double o0 = w * (om.x * u0 + om.y * u1), o1 = w * (om.y * u0 + om.z * u1);
#pragma unroll
    for (int q = 0; q < 6; ++q) acc[q] += Jc[q] * o0 + Jc[6 + q] * o1;
  }
  __shared__ double red[THREADS / 32][6];
  block_sum_array<double, 6, THREADS>(acc, &red[0][0]);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < 6; ++q) r_p[(size_t)h * 6 + q] = b_p[(size_t)h * 6 + q] - lambda * xp[q] - acc[q];
  }
}

// SparseOptimizer::update (sparse_optimizer.cpp:457-468) with
// VertexSE3Expmap::oplusImpl (g2o/types/sba/vertex_se3_expmap.cpp:48-51):
// T <- exp(dx) * T; VertexPointXYZ: p <- p + dx (vertex_pointxyz.h:47-50)
static __global__ void ba_oplus(BAVertices V, int Cf, int Pf, const double* x, int* nonfinite) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < Cf) {
    double u[6];
    bool bad = false;
#pragma unroll
    for (int i = 0; i < 6; ++i) {
      u[i] = x[(size_t)t * 6 + i];
      bad |= !isfinite(u[i]);
    }
    if (bad) *nonfinite = 1;
    double* cam = V.cam + (size_t)V.free_pose[t] * 8;
    SE3Q<double> T;
    T.q = Q4<double>{cam[0], cam[1], cam[2], cam[3]};
    T.t[0] = cam[4]; T.t[1] = cam[5]; T.t[2] = cam[6];
    SE3Q<double> R = se3q_mul(se3q_exp(u), T);
    cam[0] = R.q.x; cam[1] = R.q.y; cam[2] = R.q.z; cam[3] = R.q.w;
    cam[4] = R.t[0]; cam[5] = R.t[1]; cam[6] = R.t[2];
  } else if (t < Cf + Pf) {
    const int l = t - Cf;
    double* p = V.pt + (size_t)V.free_point[l] * 4;
    const double* u = x + (size_t)Cf * 6 + (size_t)l * 3;
    if (!isfinite(u[0]) || !isfinite(u[1]) || !isfinite(u[2])) *nonfinite = 1;
    p[0] += u[0];
    p[1] += u[1];
    p[2] += u[2];
  }
}

// max |diag| over Hpp and H_ll (computeLambdaInit,
// optimization_algorithm_levenberg.cpp:155-167): partial maxima per block
// sharded bundle adjustment: the diagonal of this rank's part of Hpp
template <typename Real>
__global__ void ba_hpp_diag(const Real* hpp, int Cf, double* out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < Cf * 6) out[t] = (double)hpp[(size_t)(t / 6) * 36 + (t % 6) * 7];
}

// max |diag H| from the summed Hpp diagonal (all ranks) and this rank's Hll
template <typename Real>
__global__ void ba_max_diag_summed(const double* pdiag, int Cf, const Real* hll, int Pf, double* partials) {
  double m = 0.0;
  const int n = Cf * 6 + Pf * 3;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    double v;
    if (t < Cf * 6) {
      v = fabs(pdiag[t]);
    } else {
      const int l = (t - Cf * 6) / 3, d = (t - Cf * 6) % 3;
      const int idx = d == 0 ? 0 : d == 1 ? 3 : 5;
      v = fabs((double)hll[(size_t)l * 6 + idx]);
    }
    m = fmax(m, v);
  }
  block_max(m, partials + blockIdx.x);
}

template <typename Real>
__global__ void ba_max_diag(const Real* hpp, int Cf, const Real* hll, int Pf, double* partials) {
  double m = 0.0;
  const int n = Cf * 6 + Pf * 3;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    double v;
    if (t < Cf * 6) {
      const int h = t / 6, d = t % 6;
      v = fabs((double)hpp[(size_t)h * 36 + d * 7]);
    } else {
      const int l = (t - Cf * 6) / 3, d = (t - Cf * 6) % 3;
      const int idx = d == 0 ? 0 : d == 1 ? 3 : 5;
      v = fabs((double)hll[(size_t)l * 6 + idx]);
    }
    m = fmax(m, v);
  }
  block_max(m, partials + blockIdx.x);
}

}  // namespace g2oc
