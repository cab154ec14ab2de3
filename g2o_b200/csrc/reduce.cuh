// reduce.cuh -- fixed-order reductions (xor-shuffle trees, shared-memory
// trees over warps in warp order, partials summed in index order). The
// results are bit-identical run to run; no floating-point atomics.
#pragma once

#include <cuda_runtime.h>

namespace g2oc {

template <typename T>
__device__ __forceinline__ T warp_sum(T v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// Sum N per-thread values over the block; thread 0 ends with the totals.
// smem: at least (THREADS/32) * N doubles.
template <typename T, int N, int THREADS>
__device__ __forceinline__ void block_sum_array(T (&v)[N], double* smem) {
  constexpr int W = THREADS / 32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
#pragma unroll
  for (int i = 0; i < N; ++i) v[i] = warp_sum(v[i]);
  if (lane == 0) {
#pragma unroll
    for (int i = 0; i < N; ++i) smem[warp * N + i] = (double)v[i];
  }
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int i = 0; i < N; ++i) {
      double s = smem[i];
      for (int w = 1; w < W; ++w) s += smem[w * N + i];
      v[i] = (T)s;
    }
  }
  __syncthreads();
}

// block sum of two doubles, written by thread 0 to out[0..1]
__device__ __forceinline__ void block_sum2(double a, double b, double* out) {
  __shared__ double sa[32], sb[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  a = warp_sum(a);
  b = warp_sum(b);
  if (lane == 0) {
    sa[warp] = a;
    sb[warp] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int W = (blockDim.x + 31) >> 5;
    double x = 0.0, y = 0.0;
    for (int w = 0; w < W; ++w) {
      x += sa[w];
      y += sb[w];
    }
    out[0] = x;
    out[1] = y;
  }
}

__device__ __forceinline__ double block_sum1(double a) {
  __shared__ double sa[32];
  __shared__ double total;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  a = warp_sum(a);
  __syncthreads();
  if (lane == 0) sa[warp] = a;
  __syncthreads();
  if (threadIdx.x == 0) {
    const int W = (blockDim.x + 31) >> 5;
    double x = 0.0;
    for (int w = 0; w < W; ++w) x += sa[w];
    total = x;
  }
  __syncthreads();
  return total;
}

__device__ __forceinline__ void block_max(double m, double* out) {
  __shared__ double sm[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  m = warp_max(m);
  if (lane == 0) sm[warp] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    const int W = (blockDim.x + 31) >> 5;
    double x = 0.0;
    for (int w = 0; w < W; ++w) x = fmax(x, sm[w]);
    *out = x;
  }
}

// one block: out[i] = sum_j partials[j * stride + i] for i < stride, in a fixed order
static __global__ void finalize_sum_kernel(const double* partials, int n, int stride, double* out0, double* out1,
                                    double add0) {
  double a = 0.0, b = 0.0;
  for (int j = threadIdx.x; j < n; j += blockDim.x) {
    a += partials[(size_t)j * stride];
    if (stride > 1) b += partials[(size_t)j * stride + 1];
  }
  const double sa = block_sum1(a);
  const double sb = block_sum1(b);
  if (threadIdx.x == 0) {
    if (out0) *out0 = sa + add0;
    if (out1) *out1 = sb;
  }
}

static __global__ void finalize_max_kernel(const double* partials, int n, double* out) {
  double m = 0.0;
  for (int j = threadIdx.x; j < n; j += blockDim.x) m = fmax(m, partials[j]);
  block_max(m, out);
}

}  // namespace g2oc
