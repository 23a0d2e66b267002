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
//   pass 2  one warp per (bin, quantity) sums the block partials with
//           compensated two-sums, then bins are normalised exactly as the
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
// derived-statistic sums per bin: susceptibility (statistics/susceptibility.cpp:40-66)
// sum m_k|m| (4), sum (m_k|m|)^2 (4), the same of absolute values (8); specific
// heat (specific_heat.cpp:37-44) sum E, sum E^2; standard deviation
// (standard_deviation.cpp:37-50) running mean (4) and residual sum (4)
enum { DV_SUS = 0, DV_SUS2 = 4, DV_ASUS = 8, DV_ASUS2 = 12, DV_E = 16, DV_E2 = 17, DV_MEAN = 18, DV_RES = 22,
       ST_DV = 26 };

struct StatsMask {
   int size = 0;
   int* mask = nullptr;        // [n]
   double* partial = nullptr;  // [nblocks][size][ST_NQ]
   double* cur = nullptr;      // [size][ST_W] finalised rows
   double* mean = nullptr;     // [size][ST_W] running sums of the finalised rows
   double* raw = nullptr;      // [size][ST_NQ] raw sums of the last update (combined across shards)
   double* derived = nullptr;  // [size][ST_DV] running sums behind the derived statistics
   int* ticket = nullptr;      // blocks finished in the running small-mask update (0 between updates)
   std::vector<double> saturation;     // [size] sum of mu_s (mu_B) per bin (magnetization set_mask)
   std::vector<double> normalisation;  // [size] atoms per bin (energy set_mask)
   long long counter_mag = 0, counter_en = 0;
};

struct StatsState {
   std::vector<StatsMask> masks;
   int nblocks = 0;
};

static StatsState* stats_of(vgpu_ctx* h) { return (StatsState*)h->extras[0]; }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
   for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
   return v;
}

__device__ __forceinline__ void two_sum_acc(double& s, double& c, double x) {
   const double t = s + x;
   c += fabs(s) >= fabs(x) ? (s - t) + x : (x - t) + s;
   s = t;
}

// Merge of the block partial rows of one bin and the finalised row, running
// means and derived sums: warp q of the calling block merges quantity q with
// compensated sums (32 * ST_NQ threads take part), thread 0 finalises.  The
// partial rows are read through L2 (written by other blocks of the same
// launch when called from the last block of stats_mag_small_kernel).
__device__ void stats_finalize_bin(const double* __restrict__ partial, int nblocks, int size, int bin, int do_mag,
                                   int do_energy, double* __restrict__ cur, double* __restrict__ mean,
                                   double* __restrict__ raw, double* __restrict__ derived, double mag_count,
                                   double* vq) {
   const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
   double s = 0.0, c = 0.0;
   if (q < ST_NQ) {
      // eight partial rows per lane in flight at a time, then their compensated adds
      for (int b0 = lane; b0 < nblocks; b0 += 32 * 8) {
         double v[8];
#pragma unroll
         for (int u = 0; u < 8; ++u) {
            const int b = b0 + 32 * u;
            v[u] = b < nblocks ? __ldcg(partial + ((size_t)b * size + bin) * ST_NQ + q) : 0.0;
         }
#pragma unroll
         for (int u = 0; u < 8; ++u) two_sum_acc(s, c, v[u]);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
         const double s2 = __shfl_down_sync(0xffffffffu, s, o);
         const double c2 = __shfl_down_sync(0xffffffffu, c, o);
         if (lane < o) {
            two_sum_acc(s, c, s2);
            c += c2;
         }
      }
      if (lane == 0) {
         vq[q] = s + c;
         raw[(size_t)bin * ST_NQ + q] = s + c;
      }
   }
   __syncthreads();
   if (threadIdx.x != 0) return;
   const double* v = vq;
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
      for (int k = 0; k < 4; ++k) mn[k] += o[k];
      double* dv = derived + (size_t)bin * ST_DV;
      const double mm = o[3];
      for (int k = 0; k < 3; ++k) {
         dv[DV_SUS + k] += o[k] * mm;
         dv[DV_SUS2 + k] += o[k] * o[k] * mm * mm;
         dv[DV_ASUS + k] += fabs(o[k] * mm);
         dv[DV_ASUS2 + k] += fabs(o[k] * o[k] * mm * mm);
      }
      dv[DV_SUS + 3] += mm;
      dv[DV_SUS2 + 3] += mm * mm;
      dv[DV_ASUS + 3] += mm;
      dv[DV_ASUS2 + 3] += mm * mm;
      for (int k = 0; k < 4; ++k) {  // Welford update, mag_count includes this update
         const double r1 = o[k] - dv[DV_MEAN + k];
         dv[DV_MEAN + k] += r1 / mag_count;
         const double r2 = o[k] - dv[DV_MEAN + k];
         dv[DV_RES + k] += r1 * r2;
      }
   }
   if (do_energy) {
      const double ex = 0.5 * v[ST_EEX], an = v[ST_EAN], ap = v[ST_EAP], ms = 0.5 * v[ST_EMS];
      o[4] = ex + an + ap + ms;
      o[5] = ex; o[6] = an; o[7] = ap; o[8] = ms;
      for (int k = 4; k < 9; ++k) mn[k] += o[k];
      double* dv = derived + (size_t)bin * ST_DV;
      dv[DV_E] += o[4];
      dv[DV_E2] += o[4] * o[4];
   }
}


// Magnetisation only, masks of at most NB bins (system, material of a few
// materials): per-thread register sums over a grid-stride loop (no
// reductions inside the loop), one warp reduction and shared-memory add per
// block at the end.  FP32 state is read four atoms at a time (16-byte loads of
// x, y, z, material and mask ids), the moments per material come from shared
// memory (no dependent global load per atom).  Writes the same block partial
// rows as stats_partial_kernel (energy quantities zero).
constexpr int kStatsMuShared = 64;  // materials whose moments the kernel keeps in shared memory

// The last block to finish (atomic ticket after a fence) merges every block's
// row and finalises the bins (stats_finalize_bin), so one launch does the
// whole update; it resets the ticket for the next launch.
struct StatsOut {
   int* ticket;
   double* cur;
   double* mean;
   double* raw;
   double* derived;
   double mag_count;
};

template <typename R, int NB>
__global__ void __launch_bounds__(256) stats_mag_small_kernel(const LLGArgs<R> a, const int* __restrict__ mask,
                                                              int size, double* __restrict__ partial,
                                                              const StatsOut so) {
   __shared__ double acc[NB * ST_NQ];
   __shared__ double smu[kStatsMuShared];
   // launched with programmatic stream serialisation (launch_pdl): the
   // previous kernel of the stream (the corrector) has completed after this
   asm volatile("griddepcontrol.wait;" ::: "memory");
   const bool mu_shared = a.M <= kStatsMuShared;
   for (int k = threadIdx.x; k < NB * ST_NQ; k += blockDim.x) acc[k] = 0.0;
   if (mu_shared)
      for (int k = threadIdx.x; k < a.M; k += blockDim.x) smu[k] = (double)a.mp[k].mu_s_muB;
   __syncthreads();
   double s[NB][4];
#pragma unroll
   for (int b = 0; b < NB; ++b) s[b][0] = s[b][1] = s[b][2] = s[b][3] = 0.0;
   auto add = [&](int mi, int bin, R sx, R sy, R sz) {
      const double mu = mu_shared ? smu[mi] : (double)a.mp[mi].mu_s_muB;
      const double x = (double)sx * mu, y = (double)sy * mu, z = (double)sz * mu;
#pragma unroll
      for (int b = 0; b < NB; ++b) {
         const bool on = NB == 1 || bin == b;
         s[b][0] += on ? x : 0.0;
         s[b][1] += on ? y : 0.0;
         s[b][2] += on ? z : 0.0;
         s[b][3] += on ? mu : 0.0;
      }
   };
   const int tid = blockIdx.x * blockDim.x + threadIdx.x;
   const int stride = gridDim.x * blockDim.x;
   int i0 = 0;  // first atom of the scalar loop
   if (sizeof(R) == 4) {
      const int ng = a.n_upd >> 2;
      const float4* X = reinterpret_cast<const float4*>(a.ax);
      const float4* Y = reinterpret_cast<const float4*>(a.ay);
      const float4* Z = reinterpret_cast<const float4*>(a.az);
#pragma unroll 2
      for (int g = tid; g < ng; g += stride) {
         const float4 x = __ldg(X + g), y = __ldg(Y + g), z = __ldg(Z + g);
         const int4 m = a.mat ? __ldg(reinterpret_cast<const int4*>(a.mat) + g) : make_int4(0, 0, 0, 0);
         const int4 bn = NB == 1 ? make_int4(0, 0, 0, 0) : __ldg(reinterpret_cast<const int4*>(mask) + g);
         add(m.x, bn.x, x.x, y.x, z.x);
         add(m.y, bn.y, x.y, y.y, z.y);
         add(m.z, bn.z, x.z, y.z, z.z);
         add(m.w, bn.w, x.w, y.w, z.w);
      }
      i0 = ng << 2;
   }
   for (int i = i0 + tid; i < a.n_upd; i += stride)
      add(a.mat ? __ldg(a.mat + i) : 0, NB == 1 ? 0 : __ldg(mask + i), a.ax[i], a.ay[i], a.az[i]);
   const int lane = threadIdx.x & 31;
#pragma unroll
   for (int b = 0; b < NB; ++b)
#pragma unroll
      for (int q = 0; q < 4; ++q) {
         const double v = warp_sum(s[b][q]);
         if (lane == 0) atomicAdd(acc + b * ST_NQ + q, v);
      }
   __syncthreads();
   double* out = partial + (size_t)blockIdx.x * size * ST_NQ;  // size <= NB bins
   for (int k = threadIdx.x; k < size * ST_NQ; k += blockDim.x) out[k] = acc[k];
   __shared__ int last;
   __threadfence();  // this block's row is visible before its ticket
   __syncthreads();
   if (threadIdx.x == 0) last = atomicAdd(so.ticket, 1) == (int)gridDim.x - 1;
   __syncthreads();
   if (!last) return;
   __threadfence();
   __shared__ double vq[ST_NQ];
   for (int bin = 0; bin < size; ++bin) {
      stats_finalize_bin(partial, gridDim.x, size, bin, 1, 0, so.cur, so.mean, so.raw, so.derived, so.mag_count, vq);
      __syncthreads();  // vq is reused by the next bin
   }
   if (threadIdx.x == 0) *so.ticket = 0;
}

template <typename R, int FMT>
__global__ void stats_partial_kernel(const LLGArgs<R> a, const int* __restrict__ mask, int size, int do_energy,
                                     const R* __restrict__ hm, double* __restrict__ partial) {
   extern __shared__ double acc[];
   const int nq = ST_NQ;
   const int nq_used = do_energy ? ST_NQ : ST_MU + 1;
   const int lane = threadIdx.x & 31;
   for (int k = threadIdx.x; k < size * nq; k += blockDim.x) acc[k] = 0.0;
   __syncthreads();
   const int per = (a.n_upd + gridDim.x - 1) / gridDim.x;  // owned atoms only
   const int begin = blockIdx.x * per;
   const int end = min(a.n_upd, begin + per);
   // block-uniform trip count: every lane of a warp runs the aggregation below
   for (int base = begin; base < end; base += blockDim.x) {
      const int i = base + threadIdx.x;
      const bool on = i < end;
      double q[ST_NQ];
#pragma unroll
      for (int k = 0; k < ST_NQ; ++k) q[k] = 0.0;
      int bin = -1;
      if (on) {
         const int mi = a.mat ? __ldg(a.mat + i) : 0;
         const MatParams<R> m = a.mp[mi];
         const double mu = (double)m.mu_s_muB;
         const R S[3] = {a.ax[i], a.ay[i], a.az[i]};
         bin = __ldg(mask + i);
         q[ST_MX] = (double)S[0] * mu;
         q[ST_MY] = (double)S[1] * mu;
         q[ST_MZ] = (double)S[2] * mu;
         q[ST_MU] = mu;
         if (do_energy) {
            R hx = 0, hy = 0, hz = 0;
            exchange_gather<R, FMT>(a, i, mi, a.ax, a.ay, a.az, hx, hy, hz);
            double eex = -((double)S[0] * hx + (double)S[1] * hy + (double)S[2] * hz);
            if (a.bq_off) {
               const double Sb[3] = {(double)S[0], (double)S[1], (double)S[2]};
               eex += biquadratic_energy<double, R>(a, i, Sb);
            }
            const double Sd[3] = {(double)S[0], (double)S[1], (double)S[2]};
            const double ean = anisotropy_energy<double, R>(a, i, m, Sd);
            const double eap = -((double)a.hx * S[0] + (double)a.hy * S[1] + (double)a.hz * S[2]);
            double ems = 0.0;
            if (a.cell) {
               const int c = __ldg(a.cell + i);
               ems = -((double)a.cell_hd[c] * S[0] + (double)a.cell_hd[a.ncells + c] * S[1] +
                       (double)a.cell_hd[2 * a.ncells + c] * S[2]);
            } else if (hm) {
               ems = -((double)hm[i] * S[0] + (double)hm[a.n + i] * S[1] + (double)hm[2 * a.n + i] * S[2]);
            }
            q[ST_EEX] = eex * mu;
            q[ST_EAN] = ean * mu;
            q[ST_EAP] = eap * mu;
            q[ST_EMS] = ems * mu;
         }
      }
      // warp aggregation: one shuffle reduction per distinct bin in the warp
      // (masks are mostly uniform over 32 consecutive atoms), so the shared
      // accumulators see one atomic per bin and quantity instead of 32; a warp
      // holding more than 4 bins adds the rest lane by lane
      unsigned left = __ballot_sync(0xffffffffu, on);
      for (int round = 0; left; ++round) {
         if (round == 4) {
            if (on && ((left >> lane) & 1u)) {
#pragma unroll
               for (int k = 0; k < ST_NQ; ++k)
                  if (k < nq_used) atomicAdd(acc + (size_t)bin * nq + k, q[k]);
            }
            break;
         }
         const int src = __ffs(left) - 1;
         const int b = __shfl_sync(0xffffffffu, bin, src);
         const bool mine = on && bin == b;
         left &= ~__ballot_sync(0xffffffffu, mine);
#pragma unroll
         for (int k = 0; k < ST_NQ; ++k) {
            if (k < nq_used) {
               const double v = warp_sum(mine ? q[k] : 0.0);
               if (lane == src) atomicAdd(acc + (size_t)b * nq + k, v);
            }
         }
      }
   }
   __syncthreads();
   double* out = partial + (size_t)blockIdx.x * size * nq;
   for (int k = threadIdx.x; k < size * nq; k += blockDim.x) out[k] = acc[k];
}

// Compensated sum of block partials, then reference normalisation.  One
// block per bin, one warp per quantity: each lane keeps a Neumaier sum over a
// strided share of the partials, and the 32 (sum, compensation) pairs are
// merged by error-free two-sums in a fixed tree order (deterministic).
__global__ void __launch_bounds__(32 * ST_NQ) stats_final_kernel(const double* __restrict__ partial, int nblocks,
                                                                  int size, int do_mag, int do_energy,
                                                                  double* __restrict__ cur,
                                                                  double* __restrict__ mean,
                                                                  double* __restrict__ raw,
                                                                  double* __restrict__ derived, double mag_count) {
   __shared__ double vq[ST_NQ];
   stats_finalize_bin(partial, nblocks, size, blockIdx.x, do_mag, do_energy, cur, mean, raw, derived, mag_count, vq);
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
   if (do_mag && !do_energy && m.size <= 4) {
      nblocks = std::max(1, nblocks / 2);  // 4 blocks per SM: measured best for this streaming kernel
      // the per-step magnetisation of small masks: one launch, merged and
      // finalised by its last block
      const StatsOut so{m.ticket, m.cur, m.mean, m.raw, m.derived, (double)(m.counter_mag + 1)};
      const dim3 g(nblocks), b(256);
      const int* mk = m.mask;
      double* pt = m.partial;
      if (m.size == 1) return launch_pdl(stats_mag_small_kernel<R, 1>, g, b, 0, st, a, mk, m.size, pt, so);
      if (m.size == 2) return launch_pdl(stats_mag_small_kernel<R, 2>, g, b, 0, st, a, mk, m.size, pt, so);
      return launch_pdl(stats_mag_small_kernel<R, 4>, g, b, 0, st, a, mk, m.size, pt, so);
   }
   stats_partial_kernel<R, FMT><<<nblocks, 256, smem, st>>>(a, m.mask, m.size, do_energy, hm, m.partial);
   cudaError_t e = cudaGetLastError();
   if (e != cudaSuccess) return e;
   stats_final_kernel<<<m.size, 32 * ST_NQ, 0, st>>>(m.partial, nblocks, m.size, do_mag, do_energy, m.cur, m.mean,
                                                     m.raw, m.derived, (double)(m.counter_mag + 1));
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

// the rows of one mask into device-addressable host memory (vgpu_stats_copy_rows)
__global__ void stats_rows_copy_kernel(const double* __restrict__ src, double* __restrict__ dst, int n) {
   asm volatile("griddepcontrol.wait;" ::: "memory");
   for (int k = threadIdx.x; k < n; k += blockDim.x) dst[k] = src[k];
}

void stats_destroy(vgpu_ctx* h) {
   StatsState* s = stats_of(h);
   if (!s) return;
   for (StatsMask& m : s->masks) {
      cudaFree(m.mask); cudaFree(m.partial); cudaFree(m.cur); cudaFree(m.mean); cudaFree(m.raw); cudaFree(m.derived);
      cudaFree(m.ticket);
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
   s->nblocks = std::max(1, std::min(8 * dev_sms, (n + 255) / 256));  // a full SM of 256-thread blocks
   StatsMask m;
   m.size = mask_size;
   cudaError_t e;
   if ((e = cudaMalloc(&m.mask, sizeof(int) * n)) != cudaSuccess) return cuda_err(h, e, "stats mask");
   if ((e = cudaMalloc(&m.partial, sizeof(double) * (size_t)s->nblocks * mask_size * ST_NQ)) != cudaSuccess)
      return cuda_err(h, e, "stats partials");
   if ((e = cudaMalloc(&m.cur, sizeof(double) * mask_size * ST_W)) != cudaSuccess) return cuda_err(h, e, "stats");
   if ((e = cudaMalloc(&m.mean, sizeof(double) * mask_size * ST_W)) != cudaSuccess)
      return cuda_err(h, e, "stats");
   if ((e = cudaMalloc(&m.raw, sizeof(double) * mask_size * ST_NQ)) != cudaSuccess) return cuda_err(h, e, "stats");
   cudaMemsetAsync(m.raw, 0, sizeof(double) * mask_size * ST_NQ, h->stream);
   if ((e = cudaMalloc(&m.derived, sizeof(double) * mask_size * ST_DV)) != cudaSuccess) return cuda_err(h, e, "stats");
   cudaMemsetAsync(m.derived, 0, sizeof(double) * mask_size * ST_DV, h->stream);
   if ((e = cudaMalloc(&m.ticket, sizeof(int))) != cudaSuccess) return cuda_err(h, e, "stats");
   cudaMemsetAsync(m.ticket, 0, sizeof(int), h->stream);
   // bin saturation and atom counts, summed in atom order as set_mask does
   // (statistics/magnetization.cpp:54-116 with mm = mu_s/mu_B, energy.cpp:84-89)
   m.saturation.assign(mask_size, 0.0);
   m.normalisation.assign(mask_size, 0.0);
   for (int i = 0; i < n; ++i) {
      const vgpu_material& q = h->sys.materials[h->sys.type_host.empty() ? 0 : h->sys.type_host[i]];
      m.saturation[mask[i]] += q.mu_s_SI / 9.27400915e-24;
      m.normalisation[mask[i]] += 1.0;
   }
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
      h->kernel_launches += ((flags & 3) == 1 && m.size <= 4) ? 1 : 2;  // small masks: one launch
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
   if (int rc = h->fields_ready()) return rc;
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

/* enqueue-only copy of the latest rows of mask `id` (see vgpu.h) */
extern "C" int vgpu_stats_copy_rows(vgpu_handle h, int32_t id, double* out) {
   if (!h || !out) return set_err(h, VGPU_ERR_ARG, "null argument");
   StatsState* s = stats_of(h);
   if (!s || id < 0 || id >= (int)s->masks.size()) return set_err(h, VGPU_ERR_ARG, "unknown statistics mask %d", id);
   StatsMask& m = s->masks[id];
   cudaSetDevice(h->device);
   const int n = m.size * ST_W;
   // pinned host memory the device can address (any cudaHostAlloc /
   // cudaMallocHost buffer under unified addressing): a small kernel writes
   // the rows there, so the copy joins the stream's chain of programmatically
   // serialised kernels instead of waiting for a copy-engine transfer
   cudaPointerAttributes pa;
   if (cudaPointerGetAttributes(&pa, out) == cudaSuccess && pa.type == cudaMemoryTypeHost && pa.devicePointer) {
      const double* src = m.cur;
      double* dst = static_cast<double*>(pa.devicePointer);
      return cuda_err(h, launch_pdl(stats_rows_copy_kernel, dim3(1), dim3(32 * ((n + 31) / 32 < 8 ? (n + 31) / 32 : 8)),
                                    0, h->stream, src, dst, n),
                      "statistics rows");
   }
   cudaGetLastError();  // a failed attribute query leaves no error behind
   return cuda_err(h, cudaMemcpyAsync(out, m.cur, sizeof(double) * n, cudaMemcpyDefault, h->stream),
                   "statistics rows");
}

extern "C" int vgpu_stats_get_magnetization(vgpu_handle h, int32_t id, double* m, double* mean, int64_t* counter) {
   return stats_get(h, id, 0, 4, m, mean, counter, false);
}

extern "C" int vgpu_stats_get_energy(vgpu_handle h, int32_t id, double* e, double* mean, int64_t* counter) {
   return stats_get(h, id, 4, 5, e, mean, counter, true);
}

extern "C" int vgpu_stats_reset(vgpu_handle h) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   cudaSetDevice(h->device);
   // the torque means too, as the reference's mag_m_reset (utility/statistics.cpp)
   if (int rc = torque_reset(h)) return rc;
   StatsState* s = stats_of(h);
   if (!s) return VGPU_OK;
   for (StatsMask& m : s->masks) {
      cudaMemsetAsync(m.mean, 0, sizeof(double) * m.size * ST_W, h->stream);
      cudaMemsetAsync(m.derived, 0, sizeof(double) * m.size * ST_DV, h->stream);
      m.counter_mag = m.counter_en = 0;
   }
   return cuda_err(h, cudaStreamSynchronize(h->stream), "statistics reset");
}

/* raw per-bin sums of the last update: [bin][8] = sum mu s_x, sum mu s_y,
 * sum mu s_z, sum mu (mu_B), then the four energy sums (exchange and
 * magnetostatic not yet halved); shards add these across ranks */
extern "C" int vgpu_stats_get_sums(vgpu_handle h, int32_t id, double* sums) {
   if (!h || !sums) return set_err(h, VGPU_ERR_ARG, "null argument");
   StatsState* s = stats_of(h);
   if (!s || id < 0 || id >= (int)s->masks.size()) return set_err(h, VGPU_ERR_ARG, "unknown statistics mask %d", id);
   StatsMask& m = s->masks[id];
   cudaSetDevice(h->device);
   cudaError_t e = cudaMemcpyAsync(sums, m.raw, sizeof(double) * m.size * ST_NQ, cudaMemcpyDeviceToHost, h->stream);
   if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
   return cuda_err(h, e, "statistics sums");
}

/* Derived statistics of mask `id` over the updates since the last reset, as
 * the reference's output functions compute them at temperature T:
 * susceptibility[4*bin + k] (statistics/susceptibility.cpp:70-88: the
 * 9.274e-24 / (1.3806503e-23 T) prefactor times the bin saturation),
 * specific_heat[bin] (specific_heat.cpp:50-66: muB / (kB T^2) per atom, with
 * constants::muB = 9.27400999e-24, kB = 1.3806503e-23) and
 * std_dev[4*bin + k] (standard_deviation.cpp:60-70).  Any output may be NULL.
 * The reference evaluates these on the host only, never in GPU mode. */
extern "C" int vgpu_stats_get_derived(vgpu_handle h, int32_t id, double temperature, double* susceptibility,
                                      double* specific_heat, double* std_dev) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   StatsState* s = stats_of(h);
   if (!s || id < 0 || id >= (int)s->masks.size()) return set_err(h, VGPU_ERR_ARG, "unknown statistics mask %d", id);
   StatsMask& m = s->masks[id];
   cudaSetDevice(h->device);
   std::vector<double> dv((size_t)m.size * ST_DV);
   cudaError_t e = cudaMemcpyAsync(dv.data(), m.derived, dv.size() * sizeof(double), cudaMemcpyDeviceToHost, h->stream);
   if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
   if (e != cudaSuccess) return cuda_err(h, e, "derived statistics");
   const double T = temperature;
   const double cm = (double)m.counter_mag, ce = (double)m.counter_en;
   for (int b = 0; b < m.size; ++b) {
      const double* v = dv.data() + (size_t)b * ST_DV;
      if (susceptibility) {
         const double itemp = T < 1.e-300 ? 0.0 : 9.274e-24 / (1.3806503e-23 * T);
         const double imc = 1.0 / cm, imc2 = 1.0 / (cm * cm);
         const double pre = itemp * m.saturation[b];
         for (int k = 0; k < 4; ++k)
            susceptibility[4 * b + k] = pre * (v[DV_SUS2 + k] * imc - v[DV_SUS + k] * v[DV_SUS + k] * imc2);
      }
      if (specific_heat) {
         const double itemp2 = T < 1.e-300 ? +0.0 : 9.27400999e-24 / (1.3806503e-23 * T * T);
         const double imc = 1.0 / ce, imc2 = 1.0 / (ce * ce);
         const double pre = itemp2 / m.normalisation[b];
         specific_heat[b] = pre * ((v[DV_E2] * imc) - (v[DV_E] * v[DV_E] * imc2));
      }
      if (std_dev) {
         const double imc = 1.0 / cm;
         for (int k = 0; k < 4; ++k) std_dev[4 * b + k] = sqrt(v[DV_RES + k] * imc);
      }
   }
   return VGPU_OK;
}
