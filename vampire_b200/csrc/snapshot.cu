// Device-side spin snapshots for the configuration output.
//
// The reference writes a snapshot of the spins of its output atoms every
// config output step (src/config/atoms_spins.cpp): copy_data_to_buffer
// (src/config/buffer.cpp:28-50) gathers x, y, z of the atoms in
// local_output_atom_list into one FP64 buffer, interleaved per atom, and
// write_data_binary (src/config/write.cpp:107-140) writes a uint64 count and
// that buffer.  Here the gather runs on the device over the resident state, so
// a snapshot moves exactly the 24 bytes per output atom that the file holds
// across PCIe, already in the file's layout; the host writes the file
// (vampire_b200/config.py) or hands the buffer to the reference's own writer.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "vgpu.h"
#include "vgpu_ctx.cuh"

using namespace vgpu;

namespace {

template <typename R>
__global__ void snapshot_gather_kernel(const R* __restrict__ sx, const R* __restrict__ sy, const R* __restrict__ sz,
                                       const int32_t* __restrict__ idx, int64_t count, double* __restrict__ out) {
   for (int64_t k = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; k < count; k += (int64_t)gridDim.x * blockDim.x) {
      const int i = idx[k];
      out[3 * k + 0] = (double)sx[i];
      out[3 * k + 1] = (double)sy[i];
      out[3 * k + 2] = (double)sz[i];
   }
}

}  // namespace

extern "C" int vgpu_snapshot_setup(vgpu_handle h, const int64_t* atoms, int64_t count) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   SysDev& S = h->sys;
   if (!S.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   if (count < 0 || count > (int64_t)S.n || (count > 0 && !atoms))
      return set_err(h, VGPU_ERR_ARG, "snapshot list: count %lld outside 0..%d", (long long)count, S.n);
   std::vector<int32_t> idx((size_t)count);
   for (int64_t k = 0; k < count; ++k) {
      if (atoms[k] < 0 || atoms[k] >= S.n)
         return set_err(h, VGPU_ERR_ARG, "snapshot list entry %lld is atom %lld, outside 0..%d", (long long)k,
                        (long long)atoms[k], S.n - 1);
      idx[(size_t)k] = (int32_t)atoms[k];
   }
   cudaSetDevice(h->device);
   h->release(S.snap_idx);
   h->release(S.snap_buf);
   S.snap_idx = S.snap_buf = nullptr;
   S.snap_n = -1;
   S.snap_idx = h->alloc(sizeof(int32_t) * (size_t)count);
   S.snap_buf = h->alloc(3 * sizeof(double) * (size_t)count);
   if (!S.snap_idx || !S.snap_buf) return set_err(h, VGPU_ERR_OOM, "cudaMalloc failed for the snapshot buffers");
   if (count) {
      const int rc = cuda_err(h, cudaMemcpyAsync(S.snap_idx, idx.data(), sizeof(int32_t) * (size_t)count,
                                                 cudaMemcpyHostToDevice, h->stream),
                              "snapshot list");
      if (rc) return rc;
      // the host vector is released on return: the copy must have read it
      if (const int rc2 = cuda_err(h, cudaStreamSynchronize(h->stream), "snapshot list")) return rc2;
   }
   S.snap_n = count;
   return VGPU_OK;
}

extern "C" int vgpu_snapshot(vgpu_handle h, double* out) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   SysDev& S = h->sys;
   if (!S.uploaded || S.snap_n < 0) return set_err(h, VGPU_ERR_STATE, "vgpu_snapshot_setup not called");
   if (S.snap_n == 0) return VGPU_OK;
   if (!out) return set_err(h, VGPU_ERR_ARG, "null output buffer");
   cudaSetDevice(h->device);
   const int64_t n = S.snap_n;
   const int grid = (int)std::min<int64_t>((n + 255) / 256, 148 * 16);
   if (h->prec == VGPU_PREC_FP64)
      snapshot_gather_kernel<double><<<grid, 256, 0, h->stream>>>((const double*)S.s[0], (const double*)S.s[1],
                                                                  (const double*)S.s[2], (const int32_t*)S.snap_idx,
                                                                  n, (double*)S.snap_buf);
   else
      snapshot_gather_kernel<float><<<grid, 256, 0, h->stream>>>((const float*)S.s[0], (const float*)S.s[1],
                                                                 (const float*)S.s[2], (const int32_t*)S.snap_idx, n,
                                                                 (double*)S.snap_buf);
   int rc = cuda_err(h, cudaGetLastError(), "snapshot gather");
   if (rc) return rc;
   h->kernel_launches += 1;
   return cuda_err(h, cudaMemcpyAsync(out, S.snap_buf, 3 * sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost,
                                      h->stream),
                   "snapshot copy");
}
