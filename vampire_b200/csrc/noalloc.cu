// Masked magnetisation reduction that allocates no device memory.
//
// Some callers cannot call cudaMalloc: a plugin running inside another
// framework whose caching allocator owns the device memory (a cudaMalloc of
// its own would fragment that pool or fail under the framework's memory cap),
// or a time-critical loop that must not stall on the implicit device
// synchronisation that cudaMalloc and cudaFree can bring.
// vgpu_magnetization_noalloc serves them: the caller passes device pointers to
// its inputs and outputs, and the block partial sums go to a fixed-size
// scratch array compiled into this library (a file-scope __device__ array,
// held by every GPU that loads the library until the process exits).
//
// The arithmetic is that of the statistics module's magnetisation pass
// (reference: magnetization_statistic_t::calculate_magnetization,
// src/statistics/magnetization.cpp:134-180): per mask bin sum(mu s) and
// sum(mu) in FP64, then m_hat and |m|/m_sat, empty bins zero.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>

#include "vgpu.h"
#include "vgpu_ctx.cuh"

namespace {

constexpr int kMaxBlocks = VGPU_NOALLOC_MAX_BLOCKS;
constexpr int kMaxBins = VGPU_NOALLOC_MAX_BINS;

// [kMaxBlocks][kMaxBins][4] partial sums: 256 * 64 * 4 * 8 B = 512 KiB per GPU.
static __device__ __align__(256) double g_noalloc_scratch[kMaxBlocks * kMaxBins * 4];

// Host code may not use g_noalloc_scratch as a device address (on the host it
// names a host-side stand-in); its device address is looked up once per
// device with that device current and cached here.  A cudaDeviceReset
// destroys the array with the context, and the cached address would then be
// stale: a process that resets a device does not call this entry point on it
// again.
std::mutex g_scratch_mutex;
double* g_scratch_ptr[128] = {nullptr};

// Each thread keeps its running sums in registers while its atoms stay in
// one bin and adds them to the block's shared sums when the bin changes; at
// the end a warp whose lanes all hold the same bin adds its sums by shuffles
// first, so a one-bin (system) mask costs four shared atomics per warp.
__global__ void noalloc_partial_kernel(const float* __restrict__ sx, const float* __restrict__ sy,
                                       const float* __restrict__ sz, const float* __restrict__ mu,
                                       const int32_t* __restrict__ mask, int n, int size,
                                       double* __restrict__ scratch) {
   __shared__ double acc[kMaxBins * 4];
   for (int k = threadIdx.x; k < size * 4; k += blockDim.x) acc[k] = 0.0;
   __syncthreads();
   const int per = (n + gridDim.x - 1) / gridDim.x;
   const int begin = blockIdx.x * per;
   const int end = min(n, begin + per);
   int cur = -1;  // bin of the running sums (-1: none)
   double r[4] = {0.0, 0.0, 0.0, 0.0};
   for (int i = begin + threadIdx.x; i < end; i += blockDim.x) {
      const int b = mask[i];
      if (b < 0 || b >= size) continue;  // out-of-range bins are skipped
      if (b != cur) {
         if (cur >= 0)
            for (int q = 0; q < 4; ++q) atomicAdd(&acc[4 * cur + q], r[q]);
         cur = b;
         r[0] = r[1] = r[2] = r[3] = 0.0;
      }
      const double m = (double)mu[i];
      r[0] += (double)sx[i] * m;
      r[1] += (double)sy[i] * m;
      r[2] += (double)sz[i] * m;
      r[3] += m;
   }
   const unsigned full = 0xffffffffu;
   const int lane = threadIdx.x & 31;
   const int cur0 = __shfl_sync(full, cur, 0);
   if (__all_sync(full, cur == cur0)) {
      for (int q = 0; q < 4; ++q)
         for (int o = 16; o > 0; o >>= 1) r[q] += __shfl_down_sync(full, r[q], o);
      if (lane == 0 && cur >= 0)
         for (int q = 0; q < 4; ++q) atomicAdd(&acc[4 * cur + q], r[q]);
   } else if (cur >= 0) {
      for (int q = 0; q < 4; ++q) atomicAdd(&acc[4 * cur + q], r[q]);
   }
   __syncthreads();
   // every block writes its whole row, so the scratch needs no clearing
   double* row = scratch + (size_t)blockIdx.x * kMaxBins * 4;
   for (int k = threadIdx.x; k < size * 4; k += blockDim.x) row[k] = acc[k];
}

__global__ void noalloc_final_kernel(const double* __restrict__ scratch, int nblocks, int size,
                                     double* __restrict__ out) {
   const int bin = blockIdx.x * blockDim.x + threadIdx.x;
   if (bin >= size) return;
   double v[4];
   for (int q = 0; q < 4; ++q) {
      double s = 0.0, c = 0.0;  // Neumaier-compensated sum over blocks
      for (int b = 0; b < nblocks; ++b) {
         const double x = scratch[((size_t)b * kMaxBins + bin) * 4 + q];
         const double t = s + x;
         c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
         s = t;
      }
      v[q] = s + c;
   }
   const double magm = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
   if (v[3] == 0.0) {
      out[4 * bin + 0] = out[4 * bin + 1] = out[4 * bin + 2] = out[4 * bin + 3] = 0.0;
   } else {
      out[4 * bin + 0] = v[0] / magm;
      out[4 * bin + 1] = v[1] / magm;
      out[4 * bin + 2] = v[2] / magm;
      out[4 * bin + 3] = magm / v[3];
   }
}

int scratch_for_current_device(double** out) {
   int dev = 0;
   cudaError_t e = cudaGetDevice(&dev);
   if (e != cudaSuccess) return vgpu::cuda_err(nullptr, e, "cudaGetDevice");
   if (dev < 0 || dev >= 128) return vgpu::set_err(nullptr, VGPU_ERR_ARG, "device index %d unsupported", dev);
   std::lock_guard<std::mutex> g(g_scratch_mutex);
   if (!g_scratch_ptr[dev]) {
      void* p = nullptr;
      e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
      if (e != cudaSuccess) return vgpu::cuda_err(nullptr, e, "cudaGetSymbolAddress(no-alloc scratch)");
      g_scratch_ptr[dev] = (double*)p;
   }
   *out = g_scratch_ptr[dev];
   return VGPU_OK;
}

}  // namespace

extern "C" int vgpu_magnetization_noalloc(const float* sx, const float* sy, const float* sz, const float* mu_muB,
                                          const int32_t* mask, int32_t num_atoms, int32_t mask_size, double* m_out,
                                          void* stream) {
   if (!sx || !sy || !sz || !mu_muB || !mask || !m_out)
      return vgpu::set_err(nullptr, VGPU_ERR_ARG, "null device pointer");
   if (num_atoms <= 0) return vgpu::set_err(nullptr, VGPU_ERR_ARG, "num_atoms must be positive");
   if (mask_size <= 0 || mask_size > kMaxBins)
      return vgpu::set_err(nullptr, VGPU_ERR_ARG, "mask_size %d outside 1..%d (the fixed scratch holds %d bins)",
                           mask_size, kMaxBins, kMaxBins);
   double* scratch = nullptr;
   int rc = scratch_for_current_device(&scratch);
   if (rc) return rc;
   // an error left pending by earlier work is reported as such, not as this call's
   cudaError_t e = cudaPeekAtLastError();
   if (e != cudaSuccess) return vgpu::cuda_err(nullptr, e, "CUDA error pending before the no-alloc call");
   cudaStream_t st = (cudaStream_t)stream;
   const int nblocks = std::max(1, std::min(kMaxBlocks, (num_atoms + 255) / 256));
   noalloc_partial_kernel<<<nblocks, 256, 0, st>>>(sx, sy, sz, mu_muB, mask, num_atoms, mask_size, scratch);
   e = cudaGetLastError();
   if (e != cudaSuccess) return vgpu::cuda_err(nullptr, e, "no-alloc magnetisation launch");
   noalloc_final_kernel<<<(mask_size + 63) / 64, 64, 0, st>>>(scratch, nblocks, mask_size, m_out);
   e = cudaGetLastError();
   if (e != cudaSuccess) return vgpu::cuda_err(nullptr, e, "no-alloc magnetisation launch");
   return VGPU_OK;
}
