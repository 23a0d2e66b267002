// Masked magnetisation and energy reductions (K4), FP64 accumulation.
//
// Reference: stats::update (src/statistics/statistics.cpp:26-63) ->
// magnetization_statistic_t::calculate_magnetization
// (src/statistics/magnetization.cpp:134-180) and energy_statistic_t::calculate
// (src/statistics/energy.cpp:141-258).  The reference's GPU path computes the
// magnetisation only (src/cuda/statistics.cu:303-464, by default by copying all
// spins to the host) and silently skips energies (statistics.cpp:35-37); here
// both run on the device in one pass per mask:
//
//   pass 1  each block accumulates, per mask bin, sum(mu s), sum(mu) and the
//           four energy terms into shared memory (FP64) and writes one
//           partial row per block;
//   pass 2  one thread per (bin, quantity) sums the block partials with
//           Neumaier compensation, then bins are normalised exactly as the
//           reference does (unit vector and |m|/m_sat; exchange and
//           magnetostatic energies halved) and added to the running means.
//
// Only the final bins cross to the host, and only when the caller asks.
#include <cuda_runtime.h>

#include <cstring>
#include <vector>

#include "llg_device.cuh"
#include "vgpu_ctx.cuh"

namespace vgpu {

enum { ST_MX, ST_MY, ST_MZ, ST_MU, ST_EEX, ST_EAN, ST_EAP, ST_EMS, ST_NQ };
// finalised row per bin: m_hat(3), |m|/m_sat, E_total, E_exchange, E_anisotropy, E_applied, E_magnetostatic
constexpr int ST_W = 9;

struct StatsMask {
   int size = 0;
   int* mask = nullptr;        // [n]
   double* partial = nullptr;  // [nblocks][size][ST_NQ]
   double* cur = nullptr;      // [size][ST_W] finalised rows
   double* mean = nullptr;     // [size][ST_W] running sums of the finalised rows
   long long counter_mag = 0, counter_en = 0;
};

struct StatsState {
   std::vector<StatsMask> masks;
   int nblocks = 0;
};

static StatsState* stats_of(vgpu_ctx* h) { return (StatsState*)h->extras[0]; }

template <typename R, int FMT>
__global__ void stats_partial_kernel(const LLGArgs<R> a, const int* __restrict__ mask, int size, int do_energy,
                                     const R* __restrict__ hm, double* __restrict__ partial) {
   extern __shared__ double acc[];
   const int nq = ST_NQ;
   for (int k = threadIdx.x; k < size * nq; k += blockDim.x) acc[k] = 0.0;
   __syncthreads();
   const int per = (a.n + gridDim.x - 1) / gridDim.x;
   const int begin = blockIdx.x * per;
   const int end = min(a.n, begin + per);
   for (int i = begin + threadIdx.x; i < end; i += blockDim.x) {
      const int mi = a.mat ? __ldg(a.mat + i) : 0;
      const MatParams<R> m = a.mp[mi];
      const double mu = (double)m.mu_s_muB;
      const R S[3] = {a.ax[i], a.ay[i], a.az[i]};
      double* b = acc + (size_t)__ldg(mask + i) * nq;
      atomicAdd(b + ST_MX, (double)S[0] * mu);
      atomicAdd(b + ST_MY, (double)S[1] * mu);
      atomicAdd(b + ST_MZ, (double)S[2] * mu);
      atomicAdd(b + ST_MU, mu);
      if (do_energy) {
         R hx = 0, hy = 0, hz = 0;
         exchange_gather<R, FMT>(a, i, mi, a.ax, a.ay, a.az, hx, hy, hz);
         const double eex = -((double)S[0] * hx + (double)S[1] * hy + (double)S[2] * hz);
         double ean = 0.0;
         if (a.uniaxial) {
            const double sd = (double)S[0] * m.kux + (double)S[1] * m.kuy + (double)S[2] * m.kuz;
            ean += -(double)m.ku2 * (sd * sd);
         }
         if (a.cubic) {
            const double x2 = (double)S[0] * S[0], y2 = (double)S[1] * S[1], z2 = (double)S[2] * S[2];
            ean += -0.5 * (double)m.kc4 * (x2 * x2 + y2 * y2 + z2 * z2);
         }
         const double eap = -((double)a.hx * S[0] + (double)a.hy * S[1] + (double)a.hz * S[2]);
         double ems = 0.0;
         if (a.cell) {
            const int c = __ldg(a.cell + i);
            ems = -((double)a.cell_hd[c] * S[0] + (double)a.cell_hd[a.ncells + c] * S[1] +
                    (double)a.cell_hd[2 * a.ncells + c] * S[2]);
         } else if (hm) {
            ems = -((double)hm[i] * S[0] + (double)hm[a.n + i] * S[1] + (double)hm[2 * a.n + i] * S[2]);
         }
         atomicAdd(b + ST_EEX, eex * mu);
         atomicAdd(b + ST_EAN, ean * mu);
         atomicAdd(b + ST_EAP, eap * mu);
         atomicAdd(b + ST_EMS, ems * mu);
      }
   }
   __syncthreads();
   double* out = partial + (size_t)blockIdx.x * size * nq;
   for (int k = threadIdx.x; k < size * nq; k += blockDim.x) out[k] = acc[k];
}

// Neumaier-compensated sum of block partials, then reference normalisation.
__global__ void stats_final_kernel(const double* __restrict__ partial, int nblocks, int size, int do_mag,
                                   int do_energy, double* __restrict__ cur, double* __restrict__ mean) {
   const int bin = blockIdx.x * blockDim.x + threadIdx.x;
   if (bin >= size) return;
   double v[ST_NQ];
   for (int q = 0; q < ST_NQ; ++q) {
      double s = 0.0, c = 0.0;
      for (int b = 0; b < nblocks; ++b) {
         const double x = partial[((size_t)b * size + bin) * ST_NQ + q];
         const double t = s + x;
         c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
         s = t;
      }
      v[q] = s + c;
   }
   double* o = cur + (size_t)bin * ST_W;
   double* mn = mean + (size_t)bin * ST_W;
   if (do_mag) {
      const double msat = v[ST_MU];
      const double magm = sqrt(v[ST_MX] * v[ST_MX] + v[ST_MY] * v[ST_MY] + v[ST_MZ] * v[ST_MZ]);
      if (msat == 0.0) {
         o[0] = o[1] = o[2] = o[3] = 0.0;
      } else {
         o[0] = v[ST_MX] / magm;
         o[1] = v[ST_MY] / magm;
         o[2] = v[ST_MZ] / magm;
         o[3] = magm / msat;
      }
      for (int q = 0; q < 4; ++q) mn[q] += o[q];
   }
   if (do_energy) {
      const double ex = 0.5 * v[ST_EEX], an = v[ST_EAN], ap = v[ST_EAP], ms = 0.5 * v[ST_EMS];
      o[4] = ex + an + ap + ms;
      o[5] = ex; o[6] = an; o[7] = ap; o[8] = ms;
      for (int q = 4; q < 9; ++q) mn[q] += o[q];
   }
}

template <typename R, int FMT>
static cudaError_t launch_stats(const LLGArgs<R>& a, StatsMask& m, int nblocks, int do_mag, int do_energy,
                                const R* hm, cudaStream_t st) {
   const size_t smem = (size_t)m.size * ST_NQ * sizeof(double);
   if (smem > 48 * 1024) {
      cudaError_t e = cudaFuncSetAttribute(stats_partial_kernel<R, FMT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)smem);
      if (e != cudaSuccess) return e;
   }
   stats_partial_kernel<R, FMT><<<nblocks, 256, smem, st>>>(a, m.mask, m.size, do_energy, hm, m.partial);
   cudaError_t e = cudaGetLastError();
   if (e != cudaSuccess) return e;
   stats_final_kernel<<<(m.size + 127) / 128, 128, 0, st>>>(m.partial, nblocks, m.size, do_mag, do_energy, m.cur,
                                                           m.mean);
   return cudaGetLastError();
}

template <typename R>
static cudaError_t stats_dispatch(const LLGArgs<R>& a, int fmt, StatsMask& m, int nblocks, int do_mag, int do_en,
                                  const R* hm, cudaStream_t st) {
   switch (fmt) {
      case FMT_ISO_TAB: return launch_stats<R, FMT_ISO_TAB>(a, m, nblocks, do_mag, do_en, hm, st);
      case FMT_ISO_BOND: return launch_stats<R, FMT_ISO_BOND>(a, m, nblocks, do_mag, do_en, hm, st);
      case FMT_VEC_TAB: return launch_stats<R, FMT_VEC_TAB>(a, m, nblocks, do_mag, do_en, hm, st);
      case FMT_VEC_BOND: return launch_stats<R, FMT_VEC_BOND>(a, m, nblocks, do_mag, do_en, hm, st);
      case FMT_DMI_TAB: return launch_stats<R, FMT_DMI_TAB>(a, m, nblocks, do_mag, do_en, hm, st);
      default: return launch_stats<R, FMT_TENSOR_BOND>(a, m, nblocks, do_mag, do_en, hm, st);
   }
}

void stats_destroy(vgpu_ctx* h) {
   StatsState* s = stats_of(h);
   if (!s) return;
   for (StatsMask& m : s->masks) {
      cudaFree(m.mask); cudaFree(m.partial); cudaFree(m.cur); cudaFree(m.mean);
   }
   delete s;
   h->extras[0] = nullptr;
}

}  // namespace vgpu

using namespace vgpu;

extern "C" int vgpu_stats_add_mask(vgpu_handle h, const int32_t* mask, int32_t mask_size, int32_t* id_out) {
   if (!h || !mask || !id_out) return set_err(h, VGPU_ERR_ARG, "null argument");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   if (mask_size <= 0 || mask_size > 2048) return set_err(h, VGPU_ERR_ARG, "mask_size must be in 1..2048");
   const int n = h->sys.n;
   for (int i = 0; i < n; ++i)
      if (mask[i] < 0 || mask[i] >= mask_size)
         return set_err(h, VGPU_ERR_ARG, "mask[%d] = %d outside 0..%d", i, mask[i], mask_size - 1);
   cudaSetDevice(h->device);
   if (!h->extras[0]) h->extras[0] = new StatsState();
   StatsState* s = stats_of(h);
   int dev_sms = 148;
   cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, h->device);
   s->nblocks = std::max(1, std::min(4 * dev_sms, (n + 255) / 256));
   StatsMask m;
   m.size = mask_size;
   cudaError_t e;
   if ((e = cudaMalloc(&m.mask, sizeof(int) * n)) != cudaSuccess) return cuda_err(h, e, "stats mask");
   if ((e = cudaMalloc(&m.partial, sizeof(double) * (size_t)s->nblocks * mask_size * ST_NQ)) != cudaSuccess)
      return cuda_err(h, e, "stats partials");
   if ((e = cudaMalloc(&m.cur, sizeof(double) * mask_size * ST_W)) != cudaSuccess) return cuda_err(h, e, "stats");
   if ((e = cudaMalloc(&m.mean, sizeof(double) * mask_size * ST_W)) != cudaSuccess)
      return cuda_err(h, e, "stats");
   cudaMemcpyAsync(m.mask, mask, sizeof(int) * n, cudaMemcpyHostToDevice, h->stream);
   cudaMemsetAsync(m.cur, 0, sizeof(double) * mask_size * ST_W, h->stream);
   cudaMemsetAsync(m.mean, 0, sizeof(double) * mask_size * ST_W, h->stream);
   if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return cuda_err(h, e, "stats mask upload");
   s->masks.push_back(m);
   *id_out = (int32_t)s->masks.size() - 1;
   return VGPU_OK;
}

template <typename R>
static int stats_update_typed(vgpu_handle h, int flags) {
   StatsState* s = stats_of(h);
   LLGArgs<R> a = make_args<R>(h);
   for (StatsMask& m : s->masks) {
      cudaError_t e = stats_dispatch<R>(a, h->sys.fmt, m, s->nblocks, flags & 1, (flags >> 1) & 1,
                                        (const R*)h->sys.hm_atom, h->stream);
      if (e != cudaSuccess) return cuda_err(h, e, "stats launch");
      h->kernel_launches += 2;
      if (flags & 1) m.counter_mag++;
      if (flags & 2) m.counter_en++;
   }
   return VGPU_OK;
}

/* flags: bit 0 magnetisation, bit 1 energy */
extern "C" int vgpu_stats_update(vgpu_handle h, int32_t flags) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   if (!stats_of(h) || stats_of(h)->masks.empty()) return set_err(h, VGPU_ERR_STATE, "no statistics mask registered");
   cudaSetDevice(h->device);
   h->prof_begin(PROF_STATS);
   int rc = h->prec == VGPU_PREC_FP64 ? stats_update_typed<double>(h, flags) : stats_update_typed<float>(h, flags);
   h->prof_end(PROF_STATS);
   return rc;
}

static int stats_get(vgpu_handle h, int32_t id, int offset, int count, double* cur, double* mean, int64_t* counter,
                     bool energy) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   StatsState* s = stats_of(h);
   if (!s || id < 0 || id >= (int)s->masks.size()) return set_err(h, VGPU_ERR_ARG, "unknown statistics mask %d", id);
   StatsMask& m = s->masks[id];
   cudaSetDevice(h->device);
   std::vector<double> c((size_t)m.size * ST_W), mn((size_t)m.size * ST_W);
   cudaError_t e = cudaMemcpyAsync(c.data(), m.cur, c.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
   if (e == cudaSuccess)
      e = cudaMemcpyAsync(mn.data(), m.mean, mn.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
   if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
   if (e != cudaSuccess) return cuda_err(h, e, "statistics download");
   for (int b = 0; b < m.size; ++b)
      for (int q = 0; q < count; ++q) {
         // magnetisation layout: 4 per bin interleaved (reference magnetization[4*id+k]);
         // energy layout: 5 blocks of size bins (total | exchange | anisotropy | applied | magnetostatic)
         const size_t dst = energy ? (size_t)q * m.size + b : (size_t)b * count + q;
         if (cur) cur[dst] = c[(size_t)b * ST_W + offset + q];
         if (mean) mean[dst] = mn[(size_t)b * ST_W + offset + q];
      }
   if (counter) *counter = energy ? m.counter_en : m.counter_mag;
   return VGPU_OK;
}

extern "C" int vgpu_stats_get_magnetization(vgpu_handle h, int32_t id, double* m, double* mean, int64_t* counter) {
   return stats_get(h, id, 0, 4, m, mean, counter, false);
}

extern "C" int vgpu_stats_get_energy(vgpu_handle h, int32_t id, double* e, double* mean, int64_t* counter) {
   return stats_get(h, id, 4, 5, e, mean, counter, true);
}

extern "C" int vgpu_stats_reset(vgpu_handle h) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   StatsState* s = stats_of(h);
   if (!s) return VGPU_OK;
   cudaSetDevice(h->device);
   for (StatsMask& m : s->masks) {
      cudaMemsetAsync(m.mean, 0, sizeof(double) * m.size * ST_W, h->stream);
      m.counter_mag = m.counter_en = 0;
   }
   return cuda_err(h, cudaStreamSynchronize(h->stream), "statistics reset");
}
