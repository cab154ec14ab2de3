// pg_kernels.cuh -- device kernels of the pose-graph paths: EdgeSE2 between
// VertexSE2, EdgeSE3 between VertexSE3 and EdgeSE3Expmap between
// VertexSE3Expmap. The Hessian is assembled in two
// deterministic passes: one thread per edge writes its contributions
// (H_00, H_11, H_01 and b_0, b_1 of BaseFixedSizedEdge::constructQuadraticForm,
// g2o/core/base_fixed_sized_edge.hpp:48-130) to scratch, then one thread per
// (Hpp block, row) and per (pose, row) sums them in insertion order.
#pragma once

#include "g2o_math.cuh"
#include "reduce.cuh"

namespace g2oc {

template <int PT>
struct PGTraits;
template <>
struct PGTraits<G2OC_POSE_SE2> {
  static constexpr int PD = 3;   // tangent dimension
  static constexpr int EST = 3;  // stored estimate doubles
  static constexpr int ZD = 3;   // stored inverse measurement doubles
};
template <>
struct PGTraits<G2OC_POSE_SE3> {
  static constexpr int PD = 6;
  static constexpr int EST = 12;
  static constexpr int ZD = 12;
};
template <>
struct PGTraits<G2OC_POSE_SE3EXPMAP> {  // EdgeSE3Expmap between VertexSE3Expmap
  static constexpr int PD = 6;
  static constexpr int EST = 7;   // SE3Quat::toVector
  static constexpr int ZD = 7;    // the measurement C itself (the error uses C, not C^-1)
};

struct PGEdges {
  int n;
  const int2* v;
  const double* zinv;   // inverse measurement per edge
  const double* info;   // D x D row-major per edge
  const double* delta;  // Huber delta per edge (<= 0: none)
};

template <int PT>
__device__ __forceinline__ void pg_error(const double* est, const PGEdges& E, int k, double* e) {
  constexpr int EST = PGTraits<PT>::EST, ZD = PGTraits<PT>::ZD;
  const int2 v = E.v[k];
  const double* xi = est + (size_t)v.x * EST;
  const double* xj = est + (size_t)v.y * EST;
  const double* zi = E.zinv + (size_t)k * ZD;
  if (PT == G2OC_POSE_SE2) se2_error(xi, xj, zi, e);
  else if (PT == G2OC_POSE_SE3EXPMAP) se3exp_error(xi, xj, zi, e);
  else se3_error(xi, xj, zi, e);
}

template <int PT>
__device__ __forceinline__ double pg_chi2_of(const PGEdges& E, int k, const double* e) {
  constexpr int D = PGTraits<PT>::PD;
  const double* Om = E.info + (size_t)k * D * D;
  double s = 0.0;
#pragma unroll
  for (int i = 0; i < D; ++i) {
    double t = 0.0;
#pragma unroll
    for (int j = 0; j < D; ++j) t += Om[i * D + j] * e[j];
    s += e[i] * t;
  }
  return s;
}

template <int PT>
__global__ void pg_chi2_kernel(const double* est, PGEdges E, double* partials) {
  double c = 0.0, r = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < E.n; k += gridDim.x * blockDim.x) {
    double e[6];
    pg_error<PT>(est, E, k, e);
    const double chi = pg_chi2_of<PT>(E, k, e);
    c += chi;
    const double dl = E.delta ? E.delta[k] : 0.0;
    if (dl > 0.0) {
      double rho[3];
      huber(chi, dl, rho);
      r += rho[0];
    } else {
      r += chi;
    }
  }
  block_sum2(c, r, partials + 2 * blockIdx.x);
}

template <int PT>
__global__ void pg_errors_kernel(const double* est, PGEdges E, double* out) {
  constexpr int D = PGTraits<PT>::PD;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= E.n) return;
  double e[6];
  pg_error<PT>(est, E, k, e);
#pragma unroll
  for (int i = 0; i < D; ++i) out[(size_t)k * D + i] = e[i];
}

template <int PT>
__device__ __forceinline__ void pg_jac(const double* est, const PGEdges& E, int k, double* J0, double* J1) {
  constexpr int EST = PGTraits<PT>::EST, ZD = PGTraits<PT>::ZD;
  const int2 v = E.v[k];
  const double* xi = est + (size_t)v.x * EST;
  const double* xj = est + (size_t)v.y * EST;
  const double* zi = E.zinv + (size_t)k * ZD;
  if (PT == G2OC_POSE_SE2) se2_jacobians(xi, xj, zi, J0, J1);
  else if (PT == G2OC_POSE_SE3EXPMAP) se3exp_jacobians(xi, xj, zi, J0, J1);
  else se3_jacobians(xi, xj, zi, J0, J1);
}

template <int PT>
__global__ void pg_jacobians_kernel(const double* est, PGEdges E, double* j0, double* j1) {
  constexpr int D = PGTraits<PT>::PD;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= E.n) return;
  double J0[36], J1[36];
  pg_jac<PT>(est, E, k, J0, J1);
  for (int i = 0; i < D * D; ++i) {
    j0[(size_t)k * D * D + i] = J0[i];
    j1[(size_t)k * D * D + i] = J1[i];
  }
}

// per-edge contributions: slot 0 = J0^T Om' J0, 1 = J1^T Om' J1,
// 2 = J0^T Om' J1 (or its transpose when the block is stored transposed),
// b0 = J0^T we, b1 = J1^T we
template <typename Real, int PT>
__global__ void pg_linearize(const double* est, PGEdges E, const uint8_t* trans, Real* hcontrib, double* bcontrib) {
  constexpr int D = PGTraits<PT>::PD;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= E.n) return;
  double e[6], J0[36], J1[36];
  pg_error<PT>(est, E, k, e);
  pg_jac<PT>(est, E, k, J0, J1);
  const double* I = E.info + (size_t)k * D * D;
  double w = 1.0;
  const double dl = E.delta ? E.delta[k] : 0.0;
  if (dl > 0.0) {
    double rho[3];
    huber(pg_chi2_of<PT>(E, k, e), dl, rho);
    w = rho[1];
  }
  double we[6];
#pragma unroll
  for (int i = 0; i < D; ++i) {
    double t = 0.0;
#pragma unroll
    for (int j = 0; j < D; ++j) t += I[i * D + j] * e[j];
    we[i] = -w * t;
  }
  // AtO_a = J_a^T Om'  (D x D)
  double A0[36], A1[36];
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) {
      double s0 = 0.0, s1 = 0.0;
#pragma unroll
      for (int q = 0; q < D; ++q) {
        s0 += J0[q * D + i] * I[q * D + j];
        s1 += J1[q * D + i] * I[q * D + j];
      }
      A0[i * D + j] = w * s0;
      A1[i * D + j] = w * s1;
    }
  Real* h = hcontrib + (size_t)k * 3 * D * D;
  const bool tr = trans[k];
#pragma unroll
  for (int i = 0; i < D; ++i)
#pragma unroll
    for (int j = 0; j < D; ++j) {
      double s00 = 0.0, s11 = 0.0, s01 = 0.0;
#pragma unroll
      for (int q = 0; q < D; ++q) {
        s00 += A0[i * D + q] * J0[q * D + j];
        s11 += A1[i * D + q] * J1[q * D + j];
        s01 += A0[i * D + q] * J1[q * D + j];
      }
      h[i * D + j] = (Real)s00;
      h[D * D + i * D + j] = (Real)s11;
      if (tr) h[2 * D * D + j * D + i] = (Real)s01;
      else h[2 * D * D + i * D + j] = (Real)s01;
    }
  double* b = bcontrib + (size_t)k * 2 * D;
#pragma unroll
  for (int i = 0; i < D; ++i) {
    double s0 = 0.0, s1 = 0.0;
#pragma unroll
    for (int q = 0; q < D; ++q) {
      s0 += J0[q * D + i] * we[q];
      s1 += J1[q * D + i] * we[q];
    }
    b[i] = s0;
    b[D + i] = s1;
  }
}

// Mixed-precision refinement of the pose graphs: the Gauss-Newton Hessian
// times a vector, matrix-free and in FP64 from the edges (FP64 Jacobians at
// the current estimates, the same robust weight rho' as pg_linearize). Per
// edge, with u = J0 x_i + J1 x_j (a fixed vertex contributes 0) and
// g = rho' Om u: slot 0 = J0^T g, slot 1 = J1^T g, summed per pose by
// pg_assemble_b in the gradient's order.
template <int PT>
__global__ void pg_hx_contrib(const double* est, PGEdges E, const int* pose_h, const double* x, double* out) {
  constexpr int D = PGTraits<PT>::PD;
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= E.n) return;
  double e[6], J0[36], J1[36];
  pg_error<PT>(est, E, k, e);
  pg_jac<PT>(est, E, k, J0, J1);
  const double* I = E.info + (size_t)k * D * D;
  double w = 1.0;
  const double dl = E.delta ? E.delta[k] : 0.0;
  if (dl > 0.0) {
    double rho[3];
    huber(pg_chi2_of<PT>(E, k, e), dl, rho);
    w = rho[1];
  }
  const int2 v = E.v[k];
  const int h0 = pose_h[v.x], h1 = pose_h[v.y];
  double xi[6], xj[6];
#pragma unroll
  for (int q = 0; q < D; ++q) {
    xi[q] = h0 >= 0 ? x[(size_t)h0 * D + q] : 0.0;
    xj[q] = h1 >= 0 ? x[(size_t)h1 * D + q] : 0.0;
  }
  double u[6], g[6];
#pragma unroll
  for (int i = 0; i < D; ++i) {
    double t = 0.0;
#pragma unroll
    for (int q = 0; q < D; ++q) t += J0[i * D + q] * xi[q] + J1[i * D + q] * xj[q];
    u[i] = t;
  }
#pragma unroll
  for (int i = 0; i < D; ++i) {
    double t = 0.0;
#pragma unroll
    for (int q = 0; q < D; ++q) t += I[i * D + q] * u[q];
    g[i] = w * t;
  }
  double* o = out + (size_t)k * 2 * D;
#pragma unroll
  for (int i = 0; i < D; ++i) {
    double s0 = 0.0, s1 = 0.0;
#pragma unroll
    for (int q = 0; q < D; ++q) {
      s0 += J0[q * D + i] * g[q];
      s1 += J1[q * D + i] * g[q];
    }
    o[i] = s0;
    o[D + i] = s1;
  }
}

// r = b - (H x + lambda x); per-CTA partial sums of |r|^2 and |b|^2 at
// partials[2 * block], partials[2 * block + 1]
__global__ void pg_resid_finish(int n, const double* b, const double* hx, const double* x, double lambda, double* r,
                                double* partials) {
  double rr = 0.0, bb = 0.0;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = b[i] - hx[i] - lambda * x[i];
    r[i] = v;
    rr += v * v;
    bb += b[i] * b[i];
  }
  block_sum2(rr, bb, partials + 2 * blockIdx.x);
}

// Hpp block (row r of block blk) = sum of its contributions in edge order
template <typename Real, int D>
__global__ void pg_assemble_h(int nnzb, const int* src_ptr, const int* src, const Real* hcontrib, Real* hpp) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int blk = t / D, r = t % D;
  if (blk >= nnzb) return;
  double acc[D];
#pragma unroll
  for (int c = 0; c < D; ++c) acc[c] = 0.0;
  for (int p = src_ptr[blk]; p < src_ptr[blk + 1]; ++p) {
    const int code = src[p];
    const Real* h = hcontrib + (size_t)(code / 3) * 3 * D * D + (size_t)(code % 3) * D * D + r * D;
#pragma unroll
    for (int c = 0; c < D; ++c) acc[c] += (double)h[c];
  }
#pragma unroll
  for (int c = 0; c < D; ++c) hpp[(size_t)blk * D * D + r * D + c] = (Real)acc[c];
}

template <int D>
__global__ void pg_assemble_b(int Cf, const int* src_ptr, const int* src, const double* bcontrib, double* b) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int h = t / D, r = t % D;
  if (h >= Cf) return;
  double acc = 0.0;
  for (int p = src_ptr[h]; p < src_ptr[h + 1]; ++p) {
    const int code = src[p];
    acc += bcontrib[(size_t)(code / 2) * 2 * D + (size_t)(code % 2) * D + r];
  }
  b[(size_t)h * D + r] = acc;
}

// The pose edge set of a projection graph joins the camera system: its
// assembled blocks (pg_assemble_h over the storage blocks: the Cf diagonal
// blocks, then the pose-pose blocks) are added to the camera pass's diagonal
// blocks and become the pose-pose blocks; its gradient is added to b_p
template <typename Real>
__global__ void ba_add_pose_system(int Cf, int npp, const Real* phpp, Real* hpp, const double* pb, double* b) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long nd = (long long)Cf * 36, nh = (long long)(Cf + npp) * 36;
  if (t < nd) hpp[t] = (Real)((double)hpp[t] + (double)phpp[t]);
  else if (t < nh) hpp[t] = phpp[t];
  else if (t < nh + (long long)Cf * 6) b[t - nh] += pb[t - nh];
}

// VertexSE2::oplusImpl (g2o/types/slam2d/vertex_se2.h:48-54) and
// VertexSE3::oplusImpl with orthogonalization after 1000 updates
// (g2o/types/slam3d/vertex_se3.h:99-108, isometry3d_mappings.h:81-85)
template <int PT>
__global__ void pg_oplus(double* est, const int* free_pose, int Cf, const double* x, int* oplus_count,
                         int* nonfinite) {
  constexpr int PD = PGTraits<PT>::PD, EST = PGTraits<PT>::EST;
  const int h = blockIdx.x * blockDim.x + threadIdx.x;
  if (h >= Cf) return;
  const double* u = x + (size_t)h * PD;
  bool bad = false;
#pragma unroll
  for (int i = 0; i < PD; ++i) bad |= !isfinite(u[i]);
  if (bad) *nonfinite = 1;
  const int pi = free_pose[h];
  double* X = est + (size_t)pi * EST;
  if (PT == G2OC_POSE_SE2) {
    X[0] += u[0];
    X[1] += u[1];
    X[2] = normalize_theta(X[2] + u[2]);
  } else if (PT == G2OC_POSE_SE3EXPMAP) {
    // VertexSE3Expmap::oplusImpl (g2o/types/sba/vertex_se3_expmap.cpp:48-51): T <- exp(u) T
    se3q_to7(se3q_mul(se3q_exp(u), se3q_from7(X)), X);
  } else {
    double inc[12], Y[12];
    from_compact_quat(u + 3, inc);
    inc[9] = u[0]; inc[10] = u[1]; inc[11] = u[2];
    iso_mul(X, inc, Y);
    if (++oplus_count[pi] > 1000) {
      oplus_count[pi] = 0;
      double E[9], RE[9];
      for (int r = 0; r < 3; ++r)
        for (int c = 0; c < 3; ++c)
          E[r * 3 + c] = Y[r] * Y[c] + Y[3 + r] * Y[3 + c] + Y[6 + r] * Y[6 + c] - (r == c ? 1.0 : 0.0);
      matmul3(Y, E, RE);
      for (int q = 0; q < 9; ++q) Y[q] -= 0.5 * RE[q];
    }
#pragma unroll
    for (int i = 0; i < 12; ++i) X[i] = Y[i];
  }
}

template <typename Real, int D>
__global__ void pg_max_diag(const Real* hpp, const int* diag, int Cf, double* partials) {
  double m = 0.0;
  for (int t = blockIdx.x * blockDim.x + threadIdx.x; t < Cf * D; t += gridDim.x * blockDim.x) {
    const int h = t / D, d = t % D;
    m = fmax(m, fabs((double)hpp[(size_t)diag[h] * D * D + d * (D + 1)]));
  }
  block_max(m, partials + blockIdx.x);
}

}  // namespace g2oc
