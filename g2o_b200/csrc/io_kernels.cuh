// io_kernels.cuh -- host-layout <-> device-layout conversion on the device.
// The C-ABI takes the graph in the layout of g2oc_graph (edge insertion
// order, VertexSE3Expmap as (t, q) with 7 doubles, VertexPointXYZ as 3
// doubles). Those arrays are copied to the device unchanged, straight from the
// caller's buffers, and reordered here: edges into the point-major and
// camera-major orders the bundle-adjustment kernels read, poses into the
// (q, t) 8-double records of the device, points into 4-double records.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace g2oc {

// Rows [0, na) of the point-major edge arrays come from input edge
// src_dev[row]; rows [0, nc) of the camera-major copies from src_cam[row].
// e_om / c_om hold (Omega_00, Omega_01, Omega_11, Huber delta).
static __global__ void ba_gather_edges(int na, int nc, const int* src_dev, const int* src_cam, const double* meas,
                                       const double* info, const double* delta, double2* e_z, double4* e_om,
                                       double2* c_z, double4* c_om) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= na + nc) return;
  const bool cam = t >= na;
  const int row = cam ? t - na : t;
  const int e = cam ? src_cam[row] : src_dev[row];
  const double2 z = reinterpret_cast<const double2*>(meas)[e];
  const double4 I = reinterpret_cast<const double4*>(info)[e];
  const double4 om = make_double4(I.x, I.y, I.w, delta ? delta[e] : 0.0);
  if (cam) {
    c_z[row] = z;
    c_om[row] = om;
  } else {
    e_z[row] = z;
    e_om[row] = om;
  }
}

// VertexSE3Expmap estimate (tx, ty, tz, qx, qy, qz, qw) -> (qx, qy, qz, qw, tx, ty, tz, 0)
static __global__ void ba_pack_poses(int C, const double* in7, double* out8) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= C * 8) return;
  const int i = t >> 3, k = t & 7;
  const double* v = in7 + (size_t)i * 7;
  out8[t] = k < 4 ? v[3 + k] : (k < 7 ? v[k - 4] : 0.0);
}

static __global__ void ba_unpack_poses(int C, const double* in8, double* out7) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= C * 7) return;
  const int i = t / 7, k = t % 7;
  const double* o = in8 + (size_t)i * 8;
  out7[t] = k < 3 ? o[4 + k] : o[k - 3];
}

static __global__ void ba_pack_points(int P, const double* in3, double* out4) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= P * 4) return;
  const int i = t >> 2, k = t & 3;
  out4[t] = k < 3 ? in3[(size_t)i * 3 + k] : 0.0;
}

static __global__ void ba_unpack_points(int P, const double* in4, double* out3) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= P * 3) return;
  const int i = t / 3, k = t % 3;
  out3[t] = in4[(size_t)i * 4 + k];
}

}  // namespace g2oc
