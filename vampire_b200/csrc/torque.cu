// Torque statistics on the device.
//
// Reference: stats::system_torque (src/utility/statistics.cpp:271-325) and
// stats::max_torque (:221-260).  From the current spins and the total field
// on every atom -- the spin fields (exchange, anisotropy) plus the external
// fields (applied, thermal, dipole), exactly the field the passes integrate
// (calculate_spin_fields + calculate_external_fields in the reference) --
//
//   T        = sum_i mu_s,i S_i x H_i   [J]   (system, and per material)
//   max_torq = max_i |S_i x H_i|        [T]
//
// The reference accumulates T into running sums (total_mean_system_torque,
// sublattice_mean_torque_*_array) divided by torque_data_counter on output
// (vio/outputfunctions.cpp, functions 15 and 20); here the sums stay on the
// device and only the finished values cross to the host when asked for.
//
//   pass 0  the field-only pass writes H_i (the same kernel as vgpu_get_fields);
//   pass 1  each block sums mu_s S x H per material in FP64 (warp shuffles per
//           distinct material of a warp, then shared-memory adds) and keeps the
//           block's largest |S x H|; one partial row per block;
//   pass 2  one block merges the rows with compensated sums, writes the current
//           values and adds them to the running sums.
// Shards sum their owned atoms only; the host adds the sums over ranks.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "llg_device.cuh"
#include "vgpu_ctx.cuh"

namespace vgpu {

constexpr double kMuB = 9.27400915e-24;  // Bohr magneton [J/T], as the material upload

struct TorqueState {
   int M = 0, nblocks = 0;
   double* partial = nullptr;  // [nblocks][3M + 1]: per-material torque, then the block max
   double* cur = nullptr;      // [3 + 3M + 1]: total, per material, max |S x H|
   double* sum = nullptr;      // [3 + 3M]: running sums of total and per material
   long long counter = 0;
};

static TorqueState* torque_of(vgpu_ctx* h) { return (TorqueState*)h->extras[4]; }

__device__ __forceinline__ double warp_max(double v) {
   for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
   return v;
}

__device__ __forceinline__ double warp_add(double v) {
   for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
   return v;
}

template <typename R>
__global__ void __launch_bounds__(256) torque_partial_kernel(const LLGArgs<R> a, int M,
                                                               double* __restrict__ partial) {
   extern __shared__ double tacc[];  // [3M] per material, then [8] warp maxima
   double* wmax = tacc + 3 * M;
   const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
   for (int k = threadIdx.x; k < 3 * M; k += blockDim.x) tacc[k] = 0.0;
   __syncthreads();
   const int per = (a.n_upd + gridDim.x - 1) / gridDim.x;  // owned atoms only
   const int begin = blockIdx.x * per;
   const int end = min(a.n_upd, begin + per);
   double tmax = 0.0;
   // block-uniform trip count: every lane of a warp takes part in the shuffles
   for (int base = begin; base < end; base += blockDim.x) {
      const int i = base + threadIdx.x;
      const bool on = i < end;
      double t[3] = {0.0, 0.0, 0.0};
      int mi = -1;
      if (on) {
         mi = a.mat ? __ldg(a.mat + i) : 0;
         const double S[3] = {(double)a.ax[i], (double)a.ay[i], (double)a.az[i]};
         const double H[3] = {(double)a.fx[i], (double)a.fy[i], (double)a.fz[i]};
         const double c[3] = {S[1] * H[2] - S[2] * H[1], S[2] * H[0] - S[0] * H[2], S[0] * H[1] - S[1] * H[0]};
         tmax = fmax(tmax, sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]));
         const double mu = (double)a.mp[mi].mu_s_muB * kMuB;
         t[0] = c[0] * mu; t[1] = c[1] * mu; t[2] = c[2] * mu;
      }
      // one shuffle reduction per distinct material of the warp (a warp of an
      // alloy holds a few); past four, the remaining lanes add one by one
      unsigned left = __ballot_sync(0xffffffffu, on);
      for (int round = 0; left; ++round) {
         if (round == 4) {
            if (on && ((left >> lane) & 1u))
               for (int q = 0; q < 3; ++q) atomicAdd(tacc + 3 * mi + q, t[q]);
            break;
         }
         const int src = __ffs(left) - 1;
         const int m = __shfl_sync(0xffffffffu, mi, src);
         const bool mine = on && mi == m;
         left &= ~__ballot_sync(0xffffffffu, mine);
         for (int q = 0; q < 3; ++q) {
            const double v = warp_add(mine ? t[q] : 0.0);
            if (lane == src) atomicAdd(tacc + 3 * m + q, v);
         }
      }
   }
   tmax = warp_max(tmax);
   if (lane == 0) wmax[warp] = tmax;
   __syncthreads();
   double* out = partial + (size_t)blockIdx.x * (3 * M + 1);
   for (int k = threadIdx.x; k < 3 * M; k += blockDim.x) out[k] = tacc[k];
   if (threadIdx.x == 0) {
      double m = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) m = fmax(m, wmax[w]);
      out[3 * M] = m;
   }
}

// one thread per (material, component): Neumaier sum over the block rows;
// thread 3M takes the maximum; then the system total and the running sums
__global__ void torque_final_kernel(const double* __restrict__ partial, int nblocks, int M,
                                    double* __restrict__ cur, double* __restrict__ sum) {
   const int k = threadIdx.x;
   const int w = 3 * M + 1;
   if (k < 3 * M) {
      double s = 0.0, c = 0.0;
      for (int b = 0; b < nblocks; ++b) {
         const double x = partial[(size_t)b * w + k];
         const double t = s + x;
         c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
         s = t;
      }
      cur[3 + k] = s + c;
   } else if (k == 3 * M) {
      double m = 0.0;
      for (int b = 0; b < nblocks; ++b) m = fmax(m, partial[(size_t)b * w + 3 * M]);
      cur[3 + 3 * M] = m;
   }
   __syncthreads();
   if (k < 3) {
      double s = 0.0;
      for (int mi = 0; mi < M; ++mi) s += cur[3 + 3 * mi + k];
      cur[k] = s;
   }
   __syncthreads();
   if (k < 3 + 3 * M) sum[k] += cur[k];
}

template <typename R>
static int torque_update_typed(vgpu_ctx* h) {
   SysDev& S = h->sys;
   TorqueState* t = torque_of(h);
   if (!S.f[0]) {
      for (int q = 0; q < 3; ++q) {
         S.f[q] = h->alloc(S.n_alloc * sizeof(R));
         if (!S.f[q]) return set_err(h, VGPU_ERR_OOM, "cudaMalloc failed for field buffer");
      }
   }
   LLGArgs<R> a = make_args<R>(h);
   cudaError_t e = launch_llg_pass<R>(a, S.fmt, PASS_FIELD, S.nslices, h->stream);
   if (e != cudaSuccess) return cuda_err(h, e, "torque field launch");
   h->kernel_launches++;
   const size_t smem = (size_t)(3 * t->M + 8) * sizeof(double);
   torque_partial_kernel<R><<<t->nblocks, 256, smem, h->stream>>>(a, t->M, t->partial);
   e = cudaGetLastError();
   if (e != cudaSuccess) return cuda_err(h, e, "torque launch");
   torque_final_kernel<<<1, ((3 * t->M + 3 + 31) / 32) * 32, 0, h->stream>>>(t->partial, t->nblocks, t->M, t->cur,
                                                                             t->sum);
   e = cudaGetLastError();
   if (e != cudaSuccess) return cuda_err(h, e, "torque launch");
   h->kernel_launches += 2;
   t->counter++;
   return VGPU_OK;
}

void torque_destroy(vgpu_ctx* h) {
   TorqueState* t = torque_of(h);
   if (!t) return;
   h->release(t->partial);
   h->release(t->cur);
   h->release(t->sum);
   delete t;
   h->extras[4] = nullptr;
}

int torque_reset(vgpu_ctx* h) {
   TorqueState* t = torque_of(h);
   if (!t) return VGPU_OK;
   t->counter = 0;
   return cuda_err(h, cudaMemsetAsync(t->sum, 0, (size_t)(3 + 3 * t->M) * sizeof(double), h->stream),
                   "torque reset");
}

}  // namespace vgpu

using namespace vgpu;

extern "C" int vgpu_torque_update(vgpu_handle h) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   if (int rc = h->fields_ready()) return rc;
   cudaSetDevice(h->device);
   const int M = h->sys.M;
   if (3 * M + 3 > 1024) return set_err(h, VGPU_ERR_ARG, "torque statistics support at most 340 materials");
   TorqueState* t = torque_of(h);
   if (!t) {
      t = new TorqueState();
      t->M = M;
      int dev_sms = 148;
      cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, h->device);
      t->nblocks = std::max(1, std::min(4 * dev_sms, (h->sys.n + 255) / 256));
      t->partial = (double*)h->alloc((size_t)t->nblocks * (3 * M + 1) * sizeof(double));
      t->cur = (double*)h->alloc((size_t)(4 + 3 * M) * sizeof(double));
      t->sum = (double*)h->alloc((size_t)(3 + 3 * M) * sizeof(double));
      h->extras[4] = t;
      if (!t->partial || !t->cur || !t->sum) {
         torque_destroy(h);
         return set_err(h, VGPU_ERR_OOM, "cudaMalloc failed for torque statistics");
      }
      if (int rc = torque_reset(h)) return rc;
   }
   return h->prec == VGPU_PREC_FP64 ? torque_update_typed<double>(h) : torque_update_typed<float>(h);
}

extern "C" int vgpu_torque_get(vgpu_handle h, double* total, double* mean, double* material, double* material_mean,
                               double* max_torque, int64_t* counter) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   TorqueState* t = torque_of(h);
   const int M = h->sys.M;
   std::vector<double> cur(4 + 3 * M, 0.0), sum(3 + 3 * M, 0.0);
   if (t) {
      int rc = cuda_err(h, cudaMemcpyAsync(cur.data(), t->cur, cur.size() * sizeof(double), cudaMemcpyDeviceToHost,
                                           h->stream), "torque download");
      if (!rc) rc = cuda_err(h, cudaMemcpyAsync(sum.data(), t->sum, sum.size() * sizeof(double),
                                                cudaMemcpyDeviceToHost, h->stream), "torque download");
      if (!rc) rc = cuda_err(h, cudaStreamSynchronize(h->stream), "torque download");
      if (rc) return rc;
   }
   const long long n = t ? t->counter : 0;
   const double inv = n > 0 ? 1.0 / (double)n : 0.0;
   for (int q = 0; q < 3; ++q) {
      if (total) total[q] = cur[q];
      if (mean) mean[q] = sum[q] * inv;
   }
   for (int k = 0; k < 3 * M; ++k) {
      if (material) material[k] = cur[3 + k];
      if (material_mean) material_mean[k] = sum[3 + k] * inv;
   }
   if (max_torque) *max_torque = cur[3 + 3 * M];
   if (counter) *counter = n;
   return VGPU_OK;
}

extern "C" int vgpu_torque_reset(vgpu_handle h) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   return torque_reset(h);
}
