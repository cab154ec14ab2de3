// noalloc.cu -- g2oc_solve_block_system_static: the block-Jacobi PCG solve of
// g2oc_solve_block_system for callers that cannot allocate device memory
// (code running where cudaMalloc is not allowed or not wanted: inside a
// memory-capped or pre-partitioned GPU process, under a caller-owned
// allocator, or in a plugin that must not grow the device footprint).
//
// All device scratch lives in one file-scope __device__ array of
// G2OC_STATIC_SCRATCH_BYTES; every GPU that loads this library holds it until
// the process exits. Host-side scratch is a file-scope array as well: the
// entry point calls no cudaMalloc, cudaFree, malloc or allocating library
// routine. Calls share the arrays (a mutex serializes host callers); calls
// that overlap on the GPU from different processes or unsynchronized streams
// of one device are not possible through this entry point, since each call
// runs to completion before returning.
#include <cstring>
#include <mutex>

#include "g2oc_internal.h"
#include "pcg_kernels.cuh"

namespace g2oc {

static __device__ __align__(256) unsigned char g_static_scratch[G2OC_STATIC_SCRATCH_BYTES];

namespace {

constexpr int kMaxDevices = 64;
void* g_scratch_ptr[kMaxDevices] = {};
std::mutex g_static_mutex;

// host-side scratch for the block lists (ints), sized to the largest system
// the device scratch can hold
constexpr size_t kHostInts = 4u << 20;
int g_host_ints[kHostInts];

size_t align_up(size_t v) { return (v + 255) & ~(size_t)255; }

// scatter the caller's column-major block values into the row-SoA layout
template <int BS>
__global__ void static_gather_values(const double* src, const int* perm, const int* brow, const int* rptr, int nnzb,
                                     double* dst) {
  const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= (long long)nnzb * BS * BS) return;
  const int k = (int)(t / (BS * BS)), e = (int)(t % (BS * BS));
  const int r = brow[k], rb = rptr[r];
  dst[sys_offset<BS>(rb, rptr[r + 1] - rb, k - rb, e)] = src[(size_t)perm[k] * BS * BS + e];
}

template <int BS>
int static_solve(cudaStream_t st, unsigned char* arena, int nb, int nnzb, const int32_t* rc, const double* values,
                 const double* b, double* x, double tolerance, int max_iterations, int32_t* iterations) {
  // host lists: internal order = (row, col) as build_sym_lists
  int* rptr = g_host_ints;
  int* rcol = rptr + (nb + 1);
  int* brow = rcol + nnzb;
  int* diag = brow + nnzb;
  int* cptr = diag + nb;
  int* cblk = cptr + (nb + 1);
  int* perm = cblk + nnzb;
  int* tmp = perm + nnzb;  // nb + 1
  for (int i = 0; i <= nb; ++i) rptr[i] = 0;
  for (int k = 0; k < nnzb; ++k) rptr[rc[2 * k] + 1]++;
  for (int i = 0; i < nb; ++i) rptr[i + 1] += rptr[i];
  for (int i = 0; i < nb; ++i) {
    tmp[i] = rptr[i];
    diag[i] = -1;
  }
  for (int k = 0; k < nnzb; ++k) {
    const int r = rc[2 * k], c = rc[2 * k + 1];
    const int q = tmp[r]++;
    perm[q] = k;
    rcol[q] = c;
    brow[q] = r;
    if (r == c) diag[r] = q;
  }
  for (int i = 0; i < nb; ++i)
    if (diag[i] < 0) {
      set_error("diagonal block %d missing", i);
      return G2OC_ERR_INVALID_ARGUMENT;
    }
  for (int i = 0; i <= nb; ++i) cptr[i] = 0;
  for (int q = 0; q < nnzb; ++q)
    if (brow[q] != rcol[q]) cptr[rcol[q] + 1]++;
  for (int i = 0; i < nb; ++i) cptr[i + 1] += cptr[i];
  for (int i = 0; i < nb; ++i) tmp[i] = cptr[i];
  for (int q = 0; q < nnzb; ++q)
    if (brow[q] != rcol[q]) cblk[tmp[rcol[q]]++] = q;
  // the transposed contribution of internal block q is stored at its index in
  // the caller's column-major list, perm[q]

  // device arena layout
  const int n = nb * BS;
  const size_t per = (size_t)BS * BS;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    const size_t o = off;
    off = align_up(off + bytes);
    return arena + o;
  };
  int* d_rptr = (int*)take(sizeof(int) * (nb + 1));
  int* d_rcol = (int*)take(sizeof(int) * nnzb);
  int* d_brow = (int*)take(sizeof(int) * nnzb);
  int* d_diag = (int*)take(sizeof(int) * nb);
  int* d_cptr = (int*)take(sizeof(int) * (nb + 1));
  int* d_cblk = (int*)take(sizeof(int) * (nnzb > 0 ? nnzb : 1));
  int* d_perm = (int*)take(sizeof(int) * nnzb);
  double* d_vin = (double*)take(sizeof(double) * per * nnzb);
  double* d_val = (double*)take(sizeof(double) * per * nnzb);
  double* d_rhs = (double*)take(sizeof(double) * n);
  double* d_x = (double*)take(sizeof(double) * n);
  double* d_r = (double*)take(sizeof(double) * n);
  double* d_s = (double*)take(sizeof(double) * n);
  double* d_d0 = (double*)take(sizeof(double) * n);
  double* d_d1 = (double*)take(sizeof(double) * n);
  double* d_q = (double*)take(sizeof(double) * n);
  double* d_qrow = (double*)take(sizeof(double) * n);
  double* d_t = (double*)take(sizeof(double) * BS * (size_t)nnzb);
  double* d_minv = (double*)take(sizeof(double) * per * nb);
  double* d_part = (double*)take(sizeof(double) * (nb > 1024 ? nb : 1024));
  PcgState* d_st = (PcgState*)take(sizeof(PcgState));
  int* d_flag = (int*)take(sizeof(int));
  if (off > (size_t)G2OC_STATIC_SCRATCH_BYTES) {
    set_error("block system needs %zu bytes of device scratch, more than the static %u bytes", off,
              (unsigned)G2OC_STATIC_SCRATCH_BYTES);
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  G2OC_CUDA_TRY(cudaMemcpyAsync(d_rptr, rptr, sizeof(int) * (nb + 1), cudaMemcpyHostToDevice, st));
  G2OC_CUDA_TRY(cudaMemcpyAsync(d_rcol, rcol, sizeof(int) * nnzb, cudaMemcpyHostToDevice, st));
  G2OC_CUDA_TRY(cudaMemcpyAsync(d_brow, brow, sizeof(int) * nnzb, cudaMemcpyHostToDevice, st));
  G2OC_CUDA_TRY(cudaMemcpyAsync(d_diag, diag, sizeof(int) * nb, cudaMemcpyHostToDevice, st));
  G2OC_CUDA_TRY(cudaMemcpyAsync(d_cptr, cptr, sizeof(int) * (nb + 1), cudaMemcpyHostToDevice, st));
  if (cptr[nb] > 0) G2OC_CUDA_TRY(cudaMemcpyAsync(d_cblk, cblk, sizeof(int) * cptr[nb], cudaMemcpyHostToDevice, st));
  G2OC_CUDA_TRY(cudaMemcpyAsync(d_perm, perm, sizeof(int) * nnzb, cudaMemcpyHostToDevice, st));
  G2OC_CUDA_TRY(cudaMemcpyAsync(d_vin, values, sizeof(double) * per * nnzb, cudaMemcpyHostToDevice, st));
  G2OC_CUDA_TRY(cudaMemcpyAsync(d_rhs, b, sizeof(double) * n, cudaMemcpyHostToDevice, st));
  // the arena keeps the previous call's contents: clear what must start at zero
  G2OC_CUDA_TRY(cudaMemsetAsync(d_flag, 0, sizeof(int), st));
  G2OC_CUDA_TRY(cudaMemsetAsync(d_x, 0, sizeof(double) * n, st));
  G2OC_CUDA_TRY(cudaMemsetAsync(d_t, 0, sizeof(double) * BS * (size_t)nnzb, st));
  const long long nel = (long long)nnzb * per;
  static_gather_values<BS><<<(int)((nel + 255) / 256), 256, 0, st>>>(d_vin, d_perm, d_brow, d_rptr, nnzb, d_val);
  SysDev<double> A{nb, nnzb, d_rptr, d_rcol, d_brow, d_diag, d_cptr, d_cblk, d_perm, d_val};
  const int nbv = (nb + 127) / 128;
  pcg_diag_inv<double, BS><<<nbv, 128, 0, st>>>(A, d_minv, d_flag);
  PcgState cfg;
  std::memset(&cfg, 0, sizeof(cfg));
  cfg.residual_carry = -1.0;
  cfg.tolerance = tolerance;
  cfg.max_iter = max_iterations < 0 ? n : max_iterations;
  cfg.absolute_tolerance = 1;
  G2OC_CUDA_TRY(cudaMemcpyAsync(d_st, &cfg, sizeof(PcgState), cudaMemcpyHostToDevice, st));
  pcg_init<BS><<<nbv, 128, 0, st>>>(nb, d_rhs, d_minv, d_r, d_s, d_x, d_part, d_st);
  const bool wide = nnzb >= 64 * nb;
  PcgState host;
  int chunk = 4, launched = 0;
  for (;;) {
    for (int k = 0; k < chunk; ++k) {
      if (wide) {
        pcg_rowpass<double, BS, 256><<<nb, 256, 0, st>>>(A, d_s, d_d0, d_d1, d_qrow, d_t, d_st);
        pcg_colpass<double, BS, 256><<<nb, 256, 0, st>>>(A, d_d0, d_d1, d_qrow, d_t, d_q, d_part, d_st);
      } else {
        pcg_rowpass<double, BS, 32><<<nb, 32, 0, st>>>(A, d_s, d_d0, d_d1, d_qrow, d_t, d_st);
        pcg_colpass<double, BS, 32><<<nb, 32, 0, st>>>(A, d_d0, d_d1, d_qrow, d_t, d_q, d_part, d_st);
      }
      pcg_update<BS><<<nbv, 128, 0, st>>>(nb, d_minv, d_d0, d_d1, d_q, d_r, d_s, d_x, d_part, d_st);
    }
    const cudaError_t le = cudaGetLastError();
    if (le != cudaSuccess) {
      set_error("kernel launch: %s", cudaGetErrorString(le));
      return G2OC_ERR_CUDA;
    }
    launched += chunk;
    G2OC_CUDA_TRY(cudaMemcpyAsync(&host, d_st, sizeof(PcgState), cudaMemcpyDeviceToHost, st));
    G2OC_CUDA_TRY(cudaStreamSynchronize(st));
    if (host.done) break;
    if (launched > cfg.max_iter + 2) {
      set_error("PCG did not report completion after %d iterations", launched);
      return G2OC_ERR_TIMEOUT;
    }
    chunk = chunk * 2 > 64 ? 64 : chunk * 2;
  }
  G2OC_CUDA_TRY(cudaMemcpyAsync(x, d_x, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
  G2OC_CUDA_TRY(cudaStreamSynchronize(st));
  if (iterations) *iterations = host.iterations;
  return G2OC_OK;
}

}  // namespace
}  // namespace g2oc

using namespace g2oc;

extern "C" int g2oc_solve_block_system_static(int device, int32_t num_block_rows, int32_t block_size, int32_t nnzb,
                                              const int32_t* block_rc, const double* values, const double* b,
                                              double* x, double pcg_tolerance, int32_t pcg_max_iterations,
                                              int32_t* iterations) {
  const int nb = num_block_rows;
  if (nb <= 0 || nnzb <= 0 || !block_rc || !values || !b || !x || (block_size != 3 && block_size != 6)) {
    set_error("invalid block system arguments (block size must be 3 or 6)");
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  for (int k = 0; k < nnzb; ++k) {
    const int r = block_rc[2 * k], c = block_rc[2 * k + 1];
    if (r < 0 || c < 0 || r >= nb || c >= nb || r > c ||
        (k > 0 && (block_rc[2 * k - 1] > c || (block_rc[2 * k - 1] == c && block_rc[2 * k - 2] >= r)))) {
      set_error("blocks must be upper-triangular and listed column-major");
      return G2OC_ERR_INVALID_ARGUMENT;
    }
  }
  if ((size_t)5 * nnzb + (size_t)4 * nb + 8 > kHostInts) {
    set_error("block system too large for the static scratch (%d blocks)", nnzb);
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  if (device < 0 || device >= kMaxDevices) {
    set_error("device %d out of range", device);
    return G2OC_ERR_INVALID_ARGUMENT;
  }
  std::lock_guard<std::mutex> lock(g_static_mutex);
  // the caller's current device is put back on every return
  int caller_device = -1;
  G2OC_CUDA_TRY(cudaGetDevice(&caller_device));
  struct RestoreDevice {
    int d;
    ~RestoreDevice() { cudaSetDevice(d); }
  } restore{caller_device};
  G2OC_CUDA_TRY(cudaSetDevice(device));
  if (!g_scratch_ptr[device]) {
    // once per device, with the device current: the device address of the
    // file-scope array (its name is only a host-side stand-in)
    void* p = nullptr;
    G2OC_CUDA_TRY(cudaGetSymbolAddress(&p, g_static_scratch));
    g_scratch_ptr[device] = p;
  }
  unsigned char* arena = (unsigned char*)g_scratch_ptr[device];
  const cudaStream_t st = cudaStreamPerThread;
  const int rc =
      block_size == 3
          ? static_solve<3>(st, arena, nb, nnzb, block_rc, values, b, x, pcg_tolerance, pcg_max_iterations, iterations)
          : static_solve<6>(st, arena, nb, nnzb, block_rc, values, b, x, pcg_tolerance, pcg_max_iterations, iterations);
  // a failed call may have left kernels queued that still use the shared
  // arena: drain them before the lock lets the next caller in
  if (rc != G2OC_OK) cudaStreamSynchronize(st);
  return rc;
}
