// stereo_kernels.cuh -- the bundle-adjustment passes for EdgeStereoSE3ProjectXYZ
// (g2o/types/sba/edge_project_stereo_xyz.h:38-77, edge_project_stereo_xyz.cpp:34-106):
// vertex0 = VertexPointXYZ, vertex1 = VertexSE3Expmap, D = 3, measurement
// (u_left, v_left, u_right), error z - (u, v, u - bf / z) with
// u = x / z fx + cx, v = y / z fy + cy in the camera frame. The two-row
// projection edges keep the kernels of ba_kernels.cuh; these are the same
// passes (errors and chi2, landmark pass with H_ll, Hpl and b_l, camera pass
// with H_pp and b_p, the matrix-free FP64 residual of the mixed refinement)
// for three rows, one thread per landmark and one CTA per camera, with every
// sum in a fixed order. The Schur complement, PCG, Cholesky, back-substitution
// and update are the edge type's own blocks (6 x 6, 6 x 3, 3 x 3) and are
// shared with the two-row edges.
#pragma once

#include "ba_kernels.cuh"

namespace g2oc {

// one stereo observation: z (3), the information matrix's upper triangle
// O00 O01 O02 O11 O12 O22 and the Huber delta (<= 0: none)
struct StereoObs {
  double z[3];
  double O[6];
  double delta;
};

__device__ __forceinline__ StereoObs st_load(const double4* z3, const double4* oa, const double2* ob, int k) {
  StereoObs o;
  const double4 a = z3[k], b = oa[k];
  const double2 c = ob[k];
  o.z[0] = a.x; o.z[1] = a.y; o.z[2] = a.z; o.delta = a.w;
  o.O[0] = b.x; o.O[1] = b.y; o.O[2] = b.z; o.O[3] = b.w;
  o.O[4] = c.x; o.O[5] = c.y;
  return o;
}

// y = O x for the symmetric 3 x 3 O of an observation
__device__ __forceinline__ void st_omega(const double O[6], const double x[3], double y[3]) {
  y[0] = O[0] * x[0] + O[1] * x[1] + O[2] * x[2];
  y[1] = O[1] * x[0] + O[3] * x[1] + O[4] * x[2];
  y[2] = O[2] * x[0] + O[4] * x[1] + O[5] * x[2];
}

// error, camera-frame point, chi2 = e^T O e and robust weight rho'(chi2).
// cam_project takes bf as a float reference (edge_project_stereo_xyz.cpp:34),
// so the right image coordinate uses bf rounded to single precision.
__device__ __forceinline__ void st_edge_error(const BAVertices& V, int2 v, const StereoObs& o, double e[3],
                                              double Xc[3], double& chi2, double& w) {
  ba_transform(V.cam + (size_t)v.y * 8, V.pt + (size_t)v.x * 4, Xc);
  const double invz = 1.0 / Xc[2];
  const double u = Xc[0] * invz * V.fx + V.cx;
  const double vv = Xc[1] * invz * V.fy + V.cy;
  const double ur = u - (double)(float)V.bf * invz;
  e[0] = o.z[0] - u;
  e[1] = o.z[1] - vv;
  e[2] = o.z[2] - ur;
  double t[3];
  st_omega(o.O, e, t);
  chi2 = e[0] * t[0] + e[1] * t[1] + e[2] * t[2];
  w = 1.0;
  if (o.delta > 0.0) {
    double rho[3];
    huber(chi2, o.delta, rho);
    w = rho[1];
  }
}

// Jp (3 x 3, row-major) and Jc (3 x 6, columns omega then upsilon) of
// EdgeStereoSE3ProjectXYZ::linearizeOplus (edge_project_stereo_xyz.cpp:58-106)
__device__ __forceinline__ void st_jacobians(const double* cam, const double Xc[3], double fx, double fy, double bf,
                                             double Jp[9], double Jc[18]) {
  const double x = Xc[0], y = Xc[1], z = Xc[2], z2 = z * z;
  double R[9];
  quat_to_rot(Q4<double>{cam[0], cam[1], cam[2], cam[3]}, R);
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    Jp[c] = -fx * R[c] / z + fx * x * R[6 + c] / z2;
    Jp[3 + c] = -fy * R[3 + c] / z + fy * y * R[6 + c] / z2;
    Jp[6 + c] = Jp[c] - bf * R[6 + c] / z2;
  }
  Jc[0] = x * y / z2 * fx;
  Jc[1] = -(1.0 + (x * x / z2)) * fx;
  Jc[2] = y / z * fx;
  Jc[3] = -1.0 / z * fx;
  Jc[4] = 0.0;
  Jc[5] = x / z2 * fx;
  Jc[6] = (1.0 + y * y / z2) * fy;
  Jc[7] = -x * y / z2 * fy;
  Jc[8] = -x / z * fy;
  Jc[9] = 0.0;
  Jc[10] = -1.0 / z * fy;
  Jc[11] = y / z2 * fy;
  Jc[12] = Jc[0] - bf * y / z2;
  Jc[13] = Jc[1] + bf * x / z2;
  Jc[14] = Jc[2];
  Jc[15] = Jc[3];
  Jc[16] = 0.0;
  Jc[17] = Jc[5] - bf / z2;
}

// computeActiveErrors + activeChi2 / activeRobustChi2
static __global__ void st_chi2_kernel(BAEdges E, BAVertices V, double* partials) {
  double c = 0.0, r = 0.0;
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < E.n; k += gridDim.x * blockDim.x) {
    const StereoObs o = st_load(E.z3, E.oa3, E.ob3, k);
    double e[3], Xc[3], chi2, w;
    st_edge_error(V, E.v[k], o, e, Xc, chi2, w);
    c += chi2;
    if (o.delta > 0.0) {
      double rho[3];
      huber(chi2, o.delta, rho);
      r += rho[0];
    } else {
      r += chi2;
    }
  }
  block_sum2(c, r, partials + 2 * blockIdx.x);
}

// per-edge errors and Jacobians in FP64 (parity hooks)
static __global__ void st_errors_kernel(BAEdges E, BAVertices V, double* err) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= E.n) return;
  double e[3], Xc[3], chi2, w;
  st_edge_error(V, E.v[k], st_load(E.z3, E.oa3, E.ob3, k), e, Xc, chi2, w);
#pragma unroll
  for (int i = 0; i < 3; ++i) err[3 * (size_t)k + i] = e[i];
}

static __global__ void st_jacobians_kernel(BAEdges E, BAVertices V, double* jp, double* jc) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= E.n) return;
  const int2 v = E.v[k];
  const double* cam = V.cam + (size_t)v.y * 8;
  double Xc[3];
  ba_transform(cam, V.pt + (size_t)v.x * 4, Xc);
  double Jp[9], Jc[18];
  st_jacobians(cam, Xc, V.fx, V.fy, V.bf, Jp, Jc);
  for (int i = 0; i < 9; ++i) jp[9 * (size_t)k + i] = Jp[i];
  for (int i = 0; i < 18; ++i) jc[18 * (size_t)k + i] = Jc[i];
}

// the per-edge quantities of the quadratic form
// (BaseFixedSizedEdge::constructQuadraticForm, base_fixed_sized_edge.hpp:48-130):
// Jp, Jc, A = (rho' O) Jp (3 x 3), we = -rho' O e
struct StereoLin {
  double Jp[9], Jc[18], A[9], we[3], w;
};

__device__ __forceinline__ void st_linearize(const BAVertices& V, int2 v, const StereoObs& o, StereoLin& L) {
  double e[3], Xc[3], chi2;
  st_edge_error(V, v, o, e, Xc, chi2, L.w);
  st_jacobians(V.cam + (size_t)v.y * 8, Xc, V.fx, V.fy, V.bf, L.Jp, L.Jc);
  double t[3];
  st_omega(o.O, e, t);
#pragma unroll
  for (int d = 0; d < 3; ++d) L.we[d] = -L.w * t[d];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const double x[3] = {L.Jp[c], L.Jp[3 + c], L.Jp[6 + c]};
    double y[3];
    st_omega(o.O, x, y);
#pragma unroll
    for (int d = 0; d < 3; ++d) L.A[d * 3 + c] = L.w * y[d];
  }
}

// Landmark pass: one thread per free landmark over its edges (point-major,
// edges sharing an Hpl block adjacent): H_ll = sum Jp^T A (upper 6),
// b_l = sum Jp^T we, Hpl block (6 x 3) = sum Jc^T A.
template <typename Real>
__global__ void st_landmark_pass(BAEdges E, BAVertices V, const int* l_ptr, int Pf, Real* hll, Real* hpl,
                                 double* b_l) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= Pf) return;
  double H[6] = {0, 0, 0, 0, 0, 0}, bl[3] = {0, 0, 0};
  double B[18];
  int cur = -1;
  const int k1 = l_ptr[l + 1];
  for (int k = l_ptr[l]; k < k1; ++k) {
    StereoLin L;
    st_linearize(V, E.v[k], st_load(E.z3, E.oa3, E.ob3, k), L);
    int u = 0;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int c = i; c < 3; ++c, ++u)
        H[u] += L.Jp[i] * L.A[c] + L.Jp[3 + i] * L.A[3 + c] + L.Jp[6 + i] * L.A[6 + c];
#pragma unroll
    for (int i = 0; i < 3; ++i) bl[i] += L.Jp[i] * L.we[0] + L.Jp[3 + i] * L.we[1] + L.Jp[6 + i] * L.we[2];
    const int blk = E.hpl[k];
    if (blk >= 0) {
      if (blk != cur) {
        if (cur >= 0) {
#pragma unroll
          for (int i = 0; i < 18; ++i) hpl[(size_t)cur * 18 + i] = (Real)B[i];
        }
#pragma unroll
        for (int i = 0; i < 18; ++i) B[i] = 0.0;
        cur = blk;
      }
#pragma unroll
      for (int r = 0; r < 6; ++r)
#pragma unroll
        for (int c = 0; c < 3; ++c)
          B[r * 3 + c] += L.Jc[r] * L.A[c] + L.Jc[6 + r] * L.A[3 + c] + L.Jc[12 + r] * L.A[6 + c];
    }
  }
  if (cur >= 0) {
#pragma unroll
    for (int i = 0; i < 18; ++i) hpl[(size_t)cur * 18 + i] = (Real)B[i];
  }
#pragma unroll
  for (int i = 0; i < 6; ++i) hll[(size_t)l * 6 + i] = (Real)H[i];
#pragma unroll
  for (int i = 0; i < 3; ++i) b_l[(size_t)l * 3 + i] = bl[i];
}

// Camera pass: one CTA per free camera, H_pp = sum Jc^T (rho' O) Jc (21
// unique) and b_p = sum Jc^T we with a fixed-order block reduction
template <typename Real, int THREADS>
__global__ void __launch_bounds__(THREADS) st_camera_pass(BACamEdges CE, BAVertices V, Real* hpp, double* b_p) {
  const int h = blockIdx.x;
  double H[21], bp[6];
#pragma unroll
  for (int i = 0; i < 21; ++i) H[i] = 0.0;
#pragma unroll
  for (int i = 0; i < 6; ++i) bp[i] = 0.0;
  const int j1 = CE.ptr[h + 1];
  for (int j = CE.ptr[h] + threadIdx.x; j < j1; j += THREADS) {
    const StereoObs o = st_load(CE.z3, CE.oa3, CE.ob3, j);
    double e[3], Xc[3], chi2, w;
    const int2 v = CE.v[j];
    st_edge_error(V, v, o, e, Xc, chi2, w);
    double Jp[9], Jc[18];
    st_jacobians(V.cam + (size_t)v.y * 8, Xc, V.fx, V.fy, V.bf, Jp, Jc);
    double t[3];
    st_omega(o.O, e, t);
    // G = (rho' O) Jc (3 x 6)
    double G[18];
#pragma unroll
    for (int c = 0; c < 6; ++c) {
      const double x[3] = {Jc[c], Jc[6 + c], Jc[12 + c]};
      double y[3];
      st_omega(o.O, x, y);
#pragma unroll
      for (int d = 0; d < 3; ++d) G[d * 6 + c] = w * y[d];
    }
    int u = 0;
#pragma unroll
    for (int r = 0; r < 6; ++r)
#pragma unroll
      for (int c = r; c < 6; ++c, ++u) H[u] += Jc[r] * G[c] + Jc[6 + r] * G[6 + c] + Jc[12 + r] * G[12 + c];
#pragma unroll
    for (int i = 0; i < 6; ++i) bp[i] += -w * (Jc[i] * t[0] + Jc[6 + i] * t[1] + Jc[12 + i] * t[2]);
  }
  __shared__ double red[THREADS / 32][27];
  block_sum_array<double, 21, THREADS>(H, &red[0][0]);
  block_sum_array<double, 6, THREADS>(bp, &red[0][0]);
  if (threadIdx.x == 0) {
    Real* out = hpp + (size_t)h * 36;
    int t = 0;
    for (int r = 0; r < 6; ++r)
      for (int c = r; c < 6; ++c) {
        out[r * 6 + c] = (Real)H[t];
        out[c * 6 + r] = (Real)H[t];
        ++t;
      }
    for (int i = 0; i < 6; ++i) b_p[(size_t)h * 6 + i] = bp[i];
  }
}

// Matrix-free FP64 residual r = b - (J^T rho' O J + lambda I) x of the mixed
// refinement, landmark side (thread per landmark) and camera side (CTA per
// camera), as ba_resid64_landmark / ba_resid64_camera for three rows.
static __global__ void st_resid64_landmark(BAEdges E, BAVertices V, const int* l_ptr, int Pf, const int* pose_h,
                                           double lambda, const double* b_l, const double* x_p, const double* x_l,
                                           double* r_l) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= Pf) return;
  const double* xl = x_l + (size_t)l * 3;
  double acc[3] = {lambda * xl[0], lambda * xl[1], lambda * xl[2]};
  const int k1 = l_ptr[l + 1];
  for (int k = l_ptr[l]; k < k1; ++k) {
    const int2 v = E.v[k];
    const StereoObs o = st_load(E.z3, E.oa3, E.ob3, k);
    double e[3], Xc[3], chi2, w;
    st_edge_error(V, v, o, e, Xc, chi2, w);
    double Jp[9], Jc[18];
    st_jacobians(V.cam + (size_t)v.y * 8, Xc, V.fx, V.fy, V.bf, Jp, Jc);
    double u[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) u[d] = Jp[d * 3] * xl[0] + Jp[d * 3 + 1] * xl[1] + Jp[d * 3 + 2] * xl[2];
    const int h = pose_h[v.y];
    if (h >= 0) {
      const double* xp = x_p + (size_t)h * 6;
#pragma unroll
      for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int q = 0; q < 6; ++q) u[d] += Jc[d * 6 + q] * xp[q];
    }
    double t[3];
    st_omega(o.O, u, t);
#pragma unroll
    for (int i = 0; i < 3; ++i) acc[i] += w * (Jp[i] * t[0] + Jp[3 + i] * t[1] + Jp[6 + i] * t[2]);
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) r_l[(size_t)l * 3 + i] = b_l[(size_t)l * 3 + i] - acc[i];
}

template <int THREADS>
__global__ void __launch_bounds__(THREADS) st_resid64_camera(BACamEdges CE, BAVertices V, const int* point_l,
                                                             double lambda, const double* b_p, const double* x_p,
                                                             const double* x_l, double* r_p) {
  const int h = blockIdx.x;
  const double* xp = x_p + (size_t)h * 6;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  const int j1 = CE.ptr[h + 1];
  for (int j = CE.ptr[h] + threadIdx.x; j < j1; j += THREADS) {
    const int2 v = CE.v[j];
    const StereoObs o = st_load(CE.z3, CE.oa3, CE.ob3, j);
    double e[3], Xc[3], chi2, w;
    st_edge_error(V, v, o, e, Xc, chi2, w);
    double Jp[9], Jc[18];
    st_jacobians(V.cam + (size_t)v.y * 8, Xc, V.fx, V.fy, V.bf, Jp, Jc);
    double u[3] = {0.0, 0.0, 0.0};
#pragma unroll
    for (int d = 0; d < 3; ++d)
#pragma unroll
      for (int q = 0; q < 6; ++q) u[d] += Jc[d * 6 + q] * xp[q];
    const int l = point_l[v.x];
    if (l >= 0) {
      const double* xl = x_l + (size_t)l * 3;
#pragma unroll
      for (int d = 0; d < 3; ++d) u[d] += Jp[d * 3] * xl[0] + Jp[d * 3 + 1] * xl[1] + Jp[d * 3 + 2] * xl[2];
    }
    double t[3];
    st_omega(o.O, u, t);
#pragma unroll
    for (int q = 0; q < 6; ++q) acc[q] += w * (Jc[q] * t[0] + Jc[6 + q] * t[1] + Jc[12 + q] * t[2]);
  }
  __shared__ double red[THREADS / 32][6];
  block_sum_array<double, 6, THREADS>(acc, &red[0][0]);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < 6; ++q) r_p[(size_t)h * 6 + q] = b_p[(size_t)h * 6 + q] - lambda * xp[q] - acc[q];
  }
}

// Rows [0, na) of the point-major stereo arrays from input edge src_dev[row],
// rows [0, nc) of the camera-major copies from src_cam[row]: z3 = (u, v,
// u_right, Huber delta), oa = (O00, O01, O02, O11), ob = (O12, O22) from the
// row-major 3 x 3 information matrix.
static __global__ void st_gather_edges(int na, int nc, const int* src_dev, const int* src_cam, const double* meas,
                                       const double* info, const double* delta, double4* e_z3, double4* e_oa,
                                       double2* e_ob, double4* c_z3, double4* c_oa, double2* c_ob) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= na + nc) return;
  const bool cam = t >= na;
  const int row = cam ? t - na : t;
  const int e = cam ? src_cam[row] : src_dev[row];
  const double* z = meas + (size_t)e * 3;
  const double* I = info + (size_t)e * 9;
  const double4 z3 = make_double4(z[0], z[1], z[2], delta ? delta[e] : 0.0);
  const double4 oa = make_double4(I[0], I[1], I[2], I[4]);
  const double2 ob = make_double2(I[5], I[8]);
  if (cam) {
    c_z3[row] = z3;
    c_oa[row] = oa;
    c_ob[row] = ob;
  } else {
    e_z3[row] = z3;
    e_oa[row] = oa;
    e_ob[row] = ob;
  }
}

}  // namespace g2oc
