// adjoint_kernels.cuh -- device kernels of g2oc_backward, the implicit-
// function-theorem adjoint of a converged bundle adjustment (no counterpart in
// the reference, which has no differentiation).
//
// F(x) = 1/2 sum_e rho(e^T Om e), e = z - pi(x) (EdgeProjectXYZ2UV), G = grad F
// = sum_e rho' J^T Om e in the vertices' update charts (VertexSE3Expmap:
// T <- exp([omega, upsilon]) T; VertexPointXYZ: X <- X + dX).
//
// Exact Hessian-vector products H p = d/dt G(x [+] t p) at t = 0 are taken in
// forward mode with dual numbers through the projection: with the left update,
// d Xc / dt = omega x Xc + R dX + upsilon and d R / dt = [omega]x R, and the
// Jacobians, the error, chi2 and the Huber weight rho' are evaluated on dual
// numbers; the derivative parts of rho' J^T Om e are H p. This is the true
// Hessian (Gauss-Newton term, the error's second derivatives and the robust
// kernel's rho''), without the cancellation of a difference quotient.
#pragma once

#include "ba_kernels.cuh"

namespace g2oc {

// value + derivative along one direction
struct Dual {
  double v, d;
  __host__ __device__ Dual(double a = 0.0, double b = 0.0) : v(a), d(b) {}
};
__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
__device__ __forceinline__ Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
  const double q = a.v / b.v;
  return Dual(q, (a.d - q * b.d) / b.v);
}
__device__ __forceinline__ Dual dsqrt(Dual a) {
  const double s = sqrt(a.v);
  return Dual(s, 0.5 * a.d / s);
}

// EdgeProjectXYZ2UV::linearizeOplus (g2o/types/sba/edge_project_xyz2uv.cpp:58-97)
// on dual numbers, with the camera rotation given as a matrix
__device__ __forceinline__ void ba_jacobians_dual(const Dual R[9], const Dual Xc[3], double fxs, double fys,
                                                  Dual Jp[6], Dual Jc[12]) {
  const Dual fx(fxs), fy(fys);
  const Dual x = Xc[0], y = Xc[1], z = Xc[2], z2 = z * z;
  const Dual a02 = -x / z * fx, a12 = -y / z * fy;
  const Dual iz = Dual(-1.0) / z;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    Jp[c] = iz * (fx * R[c] + a02 * R[6 + c]);
    Jp[3 + c] = iz * (fy * R[3 + c] + a12 * R[6 + c]);
  }
  Jc[0] = x * y / z2 * fx;
  Jc[1] = -(Dual(1.0) + (x * x / z2)) * fx;
  Jc[2] = y / z * fx;
  Jc[3] = Dual(-1.0) / z * fx;
  Jc[4] = Dual(0.0);
  Jc[5] = x / z2 * fx;
  Jc[6] = (Dual(1.0) + y * y / z2) * fy;
  Jc[7] = -x * y / z2 * fy;
  Jc[8] = -x / z * fy;
  Jc[9] = Dual(0.0);
  Jc[10] = Dual(-1.0) / z * fy;
  Jc[11] = y / z2 * fy;
}

// Derivative along p of one edge's gradient terms: gp = d/dt (rho' Jp^T Om e)
// (the landmark's 3) and gc = d/dt (rho' Jc^T Om e) (the camera's 6).
// pc: the camera's direction (omega, upsilon) or nullptr (fixed camera);
// px: the landmark's direction or nullptr (fixed point).
__device__ __forceinline__ void ba_edge_hvp(const BAVertices& V, int2 v, double2 z, double4 om, const double* pc,
                                            const double* px, double gp[3], double gc[6]) {
  const double* cam = V.cam + (size_t)v.y * 8;
  const double* X = V.pt + (size_t)v.x * 4;
  double R[9];
  quat_to_rot(Q4<double>{cam[0], cam[1], cam[2], cam[3]}, R);
  double Xc[3];
#pragma unroll
  for (int i = 0; i < 3; ++i) Xc[i] = R[3 * i] * X[0] + R[3 * i + 1] * X[1] + R[3 * i + 2] * X[2] + cam[4 + i];
  const double w0 = pc ? pc[0] : 0.0, w1 = pc ? pc[1] : 0.0, w2 = pc ? pc[2] : 0.0;
  double dXc[3] = {w1 * Xc[2] - w2 * Xc[1], w2 * Xc[0] - w0 * Xc[2], w0 * Xc[1] - w1 * Xc[0]};
  if (pc) {
    dXc[0] += pc[3];
    dXc[1] += pc[4];
    dXc[2] += pc[5];
  }
  if (px) {
#pragma unroll
    for (int i = 0; i < 3; ++i) dXc[i] += R[3 * i] * px[0] + R[3 * i + 1] * px[1] + R[3 * i + 2] * px[2];
  }
  Dual Xd[3], Rd[9];
#pragma unroll
  for (int i = 0; i < 3; ++i) Xd[i] = Dual(Xc[i], dXc[i]);
  // d R = [omega]x R
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    Rd[c] = Dual(R[c], w1 * R[6 + c] - w2 * R[3 + c]);
    Rd[3 + c] = Dual(R[3 + c], w2 * R[c] - w0 * R[6 + c]);
    Rd[6 + c] = Dual(R[6 + c], w0 * R[3 + c] - w1 * R[c]);
  }
  const Dual e0 = Dual(z.x) - (Xd[0] / Xd[2] * Dual(V.fx) + Dual(V.cx));
  const Dual e1 = Dual(z.y) - (Xd[1] / Xd[2] * Dual(V.fy) + Dual(V.cy));
  const Dual oe0 = Dual(om.x) * e0 + Dual(om.y) * e1;
  const Dual oe1 = Dual(om.y) * e0 + Dual(om.z) * e1;
  Dual rho1(1.0);
  if (om.w > 0.0) {
    // RobustKernelHuber (g2o/core/robust_kernel_impl.cpp:60-74): rho' = 1 inside, delta / sqrt(chi2) outside
    const Dual chi2 = e0 * oe0 + e1 * oe1;
    if (chi2.v > om.w * om.w) rho1 = Dual(om.w) / dsqrt(chi2);
  }
  const Dual g0 = rho1 * oe0, g1 = rho1 * oe1;
  Dual Jp[6], Jc[12];
  ba_jacobians_dual(Rd, Xd, V.fx, V.fy, Jp, Jc);
#pragma unroll
  for (int i = 0; i < 3; ++i) gp[i] = (Jp[i] * g0 + Jp[3 + i] * g1).d;
#pragma unroll
  for (int i = 0; i < 6; ++i) gc[i] = (Jc[i] * g0 + Jc[6 + i] * g1).d;
}

// (H p) for the free landmarks: one warp per chunk of whole landmarks (lane
// per edge), segmented warp scan by landmark, as ba_landmark_warp
static __global__ void ba_hvp_landmark_warp(BAEdges E, BAVertices V, const int* chunk_ptr, int nchunks,
                                            const int* e_lm, const int* pose_h, int Cf, const double* p,
                                            double* hp) {
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
    const int2 v = E.v[k];
    const int h = pose_h[v.y];
    double gc[6];
    ba_edge_hvp(V, v, E.z[k], ba_om(E, k), h >= 0 ? p + (size_t)h * 6 : nullptr, p + (size_t)Cf * 6 + (size_t)key * 3,
                acc, gc);
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
#pragma unroll
    for (int i = 0; i < 3; ++i) hp[(size_t)Cf * 6 + (size_t)key * 3 + i] = acc[i];
  }
}

// (H p) for the free landmarks, one thread per landmark (landmarks with more
// than 32 edges or repeated observations)
static __global__ void ba_hvp_landmark(BAEdges E, BAVertices V, const int* l_ptr, int Pf, const int* pose_h, int Cf,
                                       const double* p, double* hp) {
  const int l = blockIdx.x * blockDim.x + threadIdx.x;
  if (l >= Pf) return;
  double acc[3] = {0, 0, 0};
  for (int k = l_ptr[l]; k < l_ptr[l + 1]; ++k) {
    const int2 v = E.v[k];
    const int h = pose_h[v.y];
    double gp[3], gc[6];
    ba_edge_hvp(V, v, E.z[k], ba_om(E, k), h >= 0 ? p + (size_t)h * 6 : nullptr, p + (size_t)Cf * 6 + (size_t)l * 3,
                gp, gc);
#pragma unroll
    for (int i = 0; i < 3; ++i) acc[i] += gp[i];
  }
#pragma unroll
  for (int i = 0; i < 3; ++i) hp[(size_t)Cf * 6 + (size_t)l * 3 + i] = acc[i];
}

// (H p) for the free cameras: one CTA per camera over its edges, fixed-order
// reduction
template <int THREADS>
__global__ void __launch_bounds__(THREADS) ba_hvp_camera(BACamEdges CE, BAVertices V, const int* point_l, int Cf,
                                                         const double* p, double* hp) {
  const int h = blockIdx.x;
  double acc[6] = {0, 0, 0, 0, 0, 0};
  for (int j = CE.ptr[h] + threadIdx.x; j < CE.ptr[h + 1]; j += THREADS) {
    const int2 v = CE.v[j];
    const int l = point_l[v.x];
    double gp[3], gc[6];
    ba_edge_hvp(V, v, CE.z[j], ba_om(CE, j), p + (size_t)h * 6, l >= 0 ? p + (size_t)Cf * 6 + (size_t)l * 3 : nullptr,
                gp, gc);
#pragma unroll
    for (int i = 0; i < 6; ++i) acc[i] += gc[i];
  }
  __shared__ double red[THREADS / 32][6];
  block_sum_array<double, 6, THREADS>(acc, &red[0][0]);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < 6; ++i) hp[(size_t)h * 6 + i] = acc[i];
  }
}

// Per-edge gradients of the loss. With G = grad_x F, F = 1/2 sum rho(e^T Om e), e = z - pi(x),
// the implicit-function theorem gives dL/dtheta = -(dG/dtheta)^T v for
// v = H^-1 dL/dx (H the exact Hessian of F in the vertices' tangent charts).
// For edge e with u = J_e v (J = de/dx as in linearizeOplus), Huber weights
// rho' and rho'' at chi2 = e^T Om e:
//   dG_e/dz_e = J^T (rho' Om + 2 rho'' Om e e^T Om)  ->  dL/dz_e = -(rho' Om u + 2 rho'' (Om e)(e^T Om u))
//   Om_e = exp(s_e) Om:  dG_e/ds_e = (rho' + rho'' chi2) J^T Om e  ->  dL/ds_e = -(rho' + rho'' chi2) e^T Om u
// Outputs in the caller's edge order (src_dev: device edge -> input edge).
static __global__ void ba_backward_edges(BAEdges E, BAVertices V, const int* pose_h, const int* point_l, int Cf,
                                         const double* v, const int* src_dev, double* dmeas, double* dlogw) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= E.n) return;
  const int2 vv = E.v[k];
  const double4 om = ba_om(E, k);
  double e[2], Xc[3], chi2, w;
  ba_edge_error(V, vv, E.z[k], om, e, Xc, chi2, w);
  double Jp[6], Jc[12];
  ba_jacobians_from_xc(V.cam + (size_t)vv.y * 8, Xc, V.fx, V.fy, Jp, Jc);
  double u0 = 0.0, u1 = 0.0;
  const int h = pose_h[vv.y], l = point_l[vv.x];
  if (h >= 0) {
    const double* vp = v + (size_t)h * 6;
#pragma unroll
    for (int q = 0; q < 6; ++q) {
      u0 += Jc[q] * vp[q];
      u1 += Jc[6 + q] * vp[q];
    }
  }
  if (l >= 0) {
    const double* vl = v + (size_t)Cf * 6 + (size_t)l * 3;
#pragma unroll
    for (int q = 0; q < 3; ++q) {
      u0 += Jp[q] * vl[q];
      u1 += Jp[3 + q] * vl[q];
    }
  }
  double r1 = 1.0, r2 = 0.0;
  if (om.w > 0.0) {
    double rho[3];
    huber(chi2, om.w, rho);
    r1 = rho[1];
    r2 = rho[2];
  }
  const double oe0 = om.x * e[0] + om.y * e[1], oe1 = om.y * e[0] + om.z * e[1];
  const double ou0 = om.x * u0 + om.y * u1, ou1 = om.y * u0 + om.z * u1;
  const double eou = e[0] * ou0 + e[1] * ou1;
  const int id = src_dev[k];
  dmeas[2 * (size_t)id] = -(r1 * ou0 + 2.0 * r2 * oe0 * eou);
  dmeas[2 * (size_t)id + 1] = -(r1 * ou1 + 2.0 * r2 * oe1 * eou);
  dlogw[id] = -(r1 + r2 * chi2) * eou;
}

}  // namespace g2oc
