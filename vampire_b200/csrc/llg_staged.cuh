// Fused LLG-Heun passes with bulk-staged bond records (FP32, FMT_DMI_TAB).
//
// The per-bond records are the bulk of the HBM stream: {neighbour, d_x, d_y,
// d_z} (12 x 16 B per atom per pass) or, with compact records (CREC), one
// 4-byte word per bond, neighbour | coupling index, whose couplings come from
// a dictionary that every block copies into its shared memory.  In the plain
// pass every thread loads its own twelve; here a block walks tiles of 32 SL
// atoms and thread 0 issues one cp.async.bulk (1-D bulk copy, global -> this
// CTA's shared memory, no multicast) for the whole contiguous record range of
// a tile, plus one per own-atom array of the tile, completing on an mbarrier
// with the byte count given by expect_tx.  Threads read their records and
// own-atom data from shared memory; neighbour spins are gathered through
// L1/L2.  The arithmetic is the plain pass's (spin_field, external_field and
// the llg_*_finish tails of llg_kernels.cuh), so results are identical.
//
// Waits on the mbarriers are bounded (1 s of wall time, and a poll count): if
// a copy has not landed by then the block records status bit 2
// (VGPU_ERR_TIMEOUT on the host), waits -- bounded again -- for its copies
// still in flight, and returns.  a.stage_extra_tx > 0 makes every tile expect
// that many bytes more than its copy delivers, so the wait runs out: the test
// of this path.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "llg_kernels.cuh"

namespace vgpu {

constexpr long long kStagePolls = 1ll << 26;
constexpr uint64_t kStageWaitNs = 1000000000ull;  // 1 s

__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* m, uint32_t count) {
   asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(m)), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* m, uint32_t bytes) {
   asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(m)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_copy_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* m) {
   asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    smem_addr(dst)),
                "l"(src), "r"(bytes), "r"(smem_addr(m))
                : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* m, uint32_t parity) {
   uint32_t ok;
   asm volatile(
       "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
       : "=r"(ok)
       : "r"(smem_addr(m)), "r"(parity)
       : "memory");
   return ok != 0;
}

__device__ __forceinline__ uint64_t global_ns() {
   uint64_t t;
   asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
   return t;
}

// wait for phase `parity` of m: at most kStageWaitNs of wall time (checked every
// 256 polls) and at most kStagePolls polls
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* m, uint32_t parity) {
   const uint64_t t0 = global_ns();
   for (long long it = 0; it < kStagePolls; ++it) {
      if (mbar_try_wait(m, parity)) return true;
      if ((it & 255) == 255 && global_ns() - t0 > kStageWaitNs) return false;
   }
   return false;
}

// Compile-time facts of a staged pass.  FEAT_FIXED: the common production
// case -- no field ramp, no per-material applied field, no per-atom
// demagnetising field, no stored predictor increment, one system per handle,
// Philox noise, no biquadratic or higher-order anisotropy terms, no padding of
// the expected bytes -- with the thermal, uniaxial, cubic and scalar-table
// flags given by the other bits.  Without FEAT_FIXED nothing is folded.
enum StageFeat : int { FEAT_FIXED = 1, FEAT_THERMAL = 2, FEAT_UNIAXIAL = 4, FEAT_CUBIC = 8, FEAT_TABSCALAR = 16 };

// the bits that hold for a (0 when a is not the FEAT_FIXED case)
inline int stage_features(const LLGArgs<float>& a) {
   if (a.ramp_n || a.local_field || a.hd_atom || a.ex || a.sys_off || a.noise_mode != VGPU_NOISE_PHILOX || a.bq_off ||
       a.aniso_ext || a.stage_extra_tx)
      return 0;
   return FEAT_FIXED | (a.thermal ? FEAT_THERMAL : 0) | (a.uniaxial ? FEAT_UNIAXIAL : 0) |
          (a.cubic ? FEAT_CUBIC : 0) | (a.tab_scalar ? FEAT_TABSCALAR : 0);
}

// a with the facts of FEAT written in as constants (equal to what a holds
// whenever stage_features(a) == FEAT)
template <int FEAT>
__device__ __forceinline__ LLGArgs<float> fold_features(const LLGArgs<float>& in) {
   LLGArgs<float> a = in;
   if (FEAT & FEAT_FIXED) {
      a.ramp_n = 0;
      a.local_field = 0;
      a.hd_atom = nullptr;
      a.ex = a.ey = a.ez = nullptr;
      a.sys_off = nullptr;
      a.noise_mode = VGPU_NOISE_PHILOX;
      a.bq_off = 0;
      a.aniso_ext = 0;
      a.stage_extra_tx = 0;
      a.thermal = (FEAT & FEAT_THERMAL) ? 1 : 0;
      a.uniaxial = (FEAT & FEAT_UNIAXIAL) ? 1 : 0;
      a.cubic = (FEAT & FEAT_CUBIC) ? 1 : 0;
      a.tab_scalar = (FEAT & FEAT_TABSCALAR) ? 1 : 0;
   }
   return a;
}

// SL slices (32 SL atoms) per tile, NBUF = 1 (one tile per block, the other
// resident blocks hide the copy) or 2 (persistent, next tile's copy in flight
// while this one is computed).  Each buffer holds the tile's bond records
// (buf_bytes) and its own-atom arrays (kStageOwnArrays x 32 SL words: s0 x|y|z,
// s' x|y|z for the corrector, material ids, cell ids (predictor), and for the
// corrector the step's external field that the predictor stored), all brought by bulk
// copies completing on the buffer's barrier; after the buffers come the
// coupling dictionary (compact records, copied with the block's first tile)
// and the material table (read into shared memory once per block when it has
// at most kStageMaxMat rows).  The predictor generates the Philox Gaussians of
// the tile's atoms while the copy is in flight (they need no data) and stores
// the atoms' external field of the step (thermal, applied and macrocell
// dipole; a.gx); the corrector, which needs the same field (nothing it depends
// on changes between the two passes of a step), copies it in with the tile
// instead of computing it again.
// Registers are capped for 768 resident threads per SM (85 a thread): the
// compact-record corrector otherwise takes 92 and fits 5 blocks of 128
// (measured 12 % slower); a cap at 64 spills and was slower again.
// FEAT: facts about the pass known when it is compiled (StageFeat bits; 0 =
// every flag read at run time).  The launcher picks the specialisation whose
// facts hold for the arguments (stage_features), so a specialised pass
// computes exactly what the generic one does -- its branches on the folded
// flags and their parameter loads are gone (0.288 -> 0.256-0.260 ms per
// step at FCC 100^3 in a timing probe, identical spins).
template <int MODE, int SL, int NBUF, bool CREC, int FEAT = 0>
__global__ void __launch_bounds__(32 * SL, 24 / SL) llg_staged_kernel(const LLGArgs<float> a_in, int nslices,
                                                                       int ntiles, int buf_bytes) {
   const LLGArgs<float> a = fold_features<FEAT>(a_in);
   constexpr int TS = 32 * SL;
   extern __shared__ __align__(128) unsigned char stage_smem[];
   __shared__ __align__(8) uint64_t mbar[2];
   // launched with programmatic stream serialisation: the previous kernel of
   // the stream has completed and its writes are visible after this
   asm volatile("griddepcontrol.wait;" ::: "memory");
   const int tid = threadIdx.x;
   const int stride = buf_bytes + kStageOwnArrays * TS * 4;
   float4* sdict = reinterpret_cast<float4*>(stage_smem + NBUF * stride);
   const uint32_t dict_bytes = CREC ? 16u * (uint32_t)(a.tab_scalar ? a.cdict_n : 2 * a.cdict_n) : 0u;
   MatParams<float>* smp = reinterpret_cast<MatParams<float>*>(stage_smem + NBUF * stride + dict_bytes);
   const bool mp_shared = a.M <= kStageMaxMat;
   // thread 0: expect the tile's bytes and start its bulk copies: records,
   // own-atom arrays (and, with the first tile, the dictionary)
   auto issue = [&](int t, int b, bool first) {
      const int s0 = a.slice_first + t * SL;
      const int s1 = min(s0 + SL, nslices);
      const int o0 = __ldg(a.slice_off + s0), o1 = __ldg(a.slice_off + s1);
      const uint32_t bytes = (uint32_t)(o1 - o0) * (CREC ? 4u : 16u);
      const void* src = CREC ? (const void*)(a.crec + o0) : (const void*)(a.rec + o0);
      const uint32_t db = first ? dict_bytes : 0u;
      const uint32_t nb = 128u * (uint32_t)(s1 - s0);  // own-array bytes: 32 atoms x 4 B per slice
      // the corrector with the predictor's stored field needs no cell ids
      const bool gin = MODE == PASS_CORRECTOR && a.gx, cin = a.cell && !gin;
      const int na = 3 + (MODE == PASS_CORRECTOR ? 3 : 0) + (a.mat ? 1 : 0) + (cin ? 1 : 0) + (gin ? 3 : 0);
      unsigned char* buf = stage_smem + b * stride;
      float* own = reinterpret_cast<float*>(buf + buf_bytes);
      const size_t a0 = (size_t)s0 * 32;
      fence_proxy_async();
      mbar_arrive_expect_tx(&mbar[b], bytes + db + nb * (uint32_t)na + (uint32_t)a.stage_extra_tx);
      if (bytes) bulk_copy_g2s(buf, src, bytes, &mbar[b]);
      if (db) bulk_copy_g2s(sdict, a.cdict, db, &mbar[b]);
      bulk_copy_g2s(own, a.ax + a0, nb, &mbar[b]);
      bulk_copy_g2s(own + TS, a.ay + a0, nb, &mbar[b]);
      bulk_copy_g2s(own + 2 * TS, a.az + a0, nb, &mbar[b]);
      if (MODE == PASS_CORRECTOR) {
         bulk_copy_g2s(own + 3 * TS, a.bx + a0, nb, &mbar[b]);
         bulk_copy_g2s(own + 4 * TS, a.by + a0, nb, &mbar[b]);
         bulk_copy_g2s(own + 5 * TS, a.bz + a0, nb, &mbar[b]);
      }
      if (a.mat) bulk_copy_g2s(own + 6 * TS, a.mat + a0, nb, &mbar[b]);
      if (cin) bulk_copy_g2s(own + 7 * TS, a.cell + a0, nb, &mbar[b]);
      if (gin) {
         bulk_copy_g2s(own + 8 * TS, a.gx + a0, nb, &mbar[b]);
         bulk_copy_g2s(own + 9 * TS, a.gy + a0, nb, &mbar[b]);
         bulk_copy_g2s(own + 10 * TS, a.gz + a0, nb, &mbar[b]);
      }
   };
   uint32_t phase = 0;  // bit b: parity of the phase of mbar[b] to wait for next
   int t = blockIdx.x, k = 0, b = 0;
   bool failed = false;
   if (tid == 0) {
      mbar_init(&mbar[0], 1);
      mbar_init(&mbar[1], 1);
      fence_mbar_init();
      if (t < ntiles) issue(t, 0, true);
   }
   if (mp_shared) {
      const int nw = a.M * (int)(sizeof(MatParams<float>) / 4);
      const float* g = reinterpret_cast<const float*>(a.mp);
      float* d = reinterpret_cast<float*>(smp);
      for (int q = tid; q < nw; q += TS) d[q] = __ldg(g + q);
   }
   __syncthreads();  // barriers initialised, material table in place
   const MatParams<float>* mpt = mp_shared ? smp : a.mp;
   for (; t < ntiles; t += gridDim.x, ++k) {
      b = NBUF == 1 ? 0 : (k & 1);
      if (tid == 0 && k > 0 && NBUF == 1) issue(t, 0, false);
      if (tid == 0 && NBUF == 2 && t + (int)gridDim.x < ntiles) issue(t + gridDim.x, b ^ 1, false);
      const int i = (a.slice_first + t * SL) * 32 + tid;
      const bool act = i < a.n_upd;
      // the tile's Gaussians (the Philox noise needs no data) while the copy
      // lands; a corrector with the predictor's stored field needs none
      float g[3] = {0.f, 0.f, 0.f};
      if (a.thermal && (MODE == PASS_PREDICTOR || !a.gx)) thermal_xi(a, act ? i : 0, g[0], g[1], g[2]);
      const int tile_off = __ldg(a.slice_off + a.slice_first + t * SL);
      const bool done = mbar_wait_bounded(&mbar[b], (phase >> b) & 1u);
      if (__syncthreads_or(!done)) {  // every thread takes the same branch
         failed = true;
         break;
      }
      phase ^= 1u << b;
      const unsigned char* buf = stage_smem + b * stride;
      const float* own = reinterpret_cast<const float*>(buf + buf_bytes);
      if (act) {
         const int mi = a.mat ? reinterpret_cast<const int*>(own)[6 * TS + tid] : 0;
         const MatParams<float> m = mpt[mi];
         const float S0[3] = {own[tid], own[TS + tid], own[2 * TS + tid]};
         float E[3];
         if (MODE == PASS_CORRECTOR && a.gx) {  // the predictor's field of this step
            E[0] = own[8 * TS + tid]; E[1] = own[9 * TS + tid]; E[2] = own[10 * TS + tid];
         } else {
            external_field_g<float>(a, i, m, g, a.cell ? reinterpret_cast<const int*>(own)[7 * TS + tid] : -1, E);
            if (MODE == PASS_PREDICTOR && a.gx) { a.gx[i] = E[0]; a.gy[i] = E[1]; a.gz[i] = E[2]; }
         }
         const int4* sb = reinterpret_cast<const int4*>(buf);
         float H[3];
         if (MODE == PASS_PREDICTOR) {
            spin_field<float, FMT_DMI_TAB, 0, true, false, CREC ? REC_COMPACT : REC_WIDE>(a, i, mi, m, a.ax, a.ay,
                                                                                           a.az, S0, H, sb,
                                                                                           tile_off, sdict);
            H[0] += E[0]; H[1] += E[1]; H[2] += E[2];
            llg_predict_finish<float>(a, i, m, S0, H);
         } else {
            const float S1[3] = {own[3 * TS + tid], own[4 * TS + tid], own[5 * TS + tid]};
            spin_field<float, FMT_DMI_TAB, 0, true, false, CREC ? REC_COMPACT : REC_WIDE>(a, i, mi, m, a.bx, a.by,
                                                                                           a.bz, S1, H, sb,
                                                                                           tile_off, sdict);
            H[0] += E[0]; H[1] += E[1]; H[2] += E[2];
            llg_correct_finish<float>(a, i, m, S0, S1, H);
         }
      }
      // buffer b fully read before it is refilled (one tile per block: never)
      if (NBUF == 2 || t + (int)gridDim.x < ntiles) __syncthreads();
   }
   if (failed) {
      if (tid == 0) {
         atomicOr(a.status, 2);
         // copies still in flight: the one waited for and, double-buffered, the next tile's
         mbar_wait_bounded(&mbar[b], (phase >> b) & 1u);
         if (NBUF == 2 && t + (int)gridDim.x < ntiles) mbar_wait_bounded(&mbar[b ^ 1], (phase >> (b ^ 1)) & 1u);
      }
      __syncthreads();
   }
}

// Per-warp pipelined passes (FP32 compact records): every warp of a
// persistent block walks its own tiles of one slice (32 atoms) with two
// buffers and two mbarriers of its own -- lane 0 starts the bulk copies of the
// warp's next slice (bond words and own-atom arrays) while the warp computes
// the current one -- so no block-wide barrier is taken after the start (the
// dictionary and the material table are read into shared memory once per
// block).  The arithmetic is the staged pass's, so results are identical.
// Shared memory: dictionary (dict_bytes), material table (mp_bytes), then per
// warp two buffers of buf_bytes words + kStageOwnArrays x 128 bytes.
template <int MODE>
__global__ void __launch_bounds__(128, 6) llg_warp_kernel(const LLGArgs<float> a, int nslices, int ntiles,
                                                          int buf_bytes, int dict_bytes, int mp_bytes) {
   extern __shared__ __align__(128) unsigned char stage_smem[];
   __shared__ __align__(8) uint64_t wbar[2 * 4];
   asm volatile("griddepcontrol.wait;" ::: "memory");
   const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
   const int wpb = blockDim.x >> 5;
   float4* sdict = reinterpret_cast<float4*>(stage_smem);
   MatParams<float>* smp = reinterpret_cast<MatParams<float>*>(stage_smem + dict_bytes);
   const bool mp_shared = mp_bytes > 0;
   const int stride = buf_bytes + kStageOwnArrays * 128;
   unsigned char* wbuf = stage_smem + dict_bytes + mp_bytes + warp * 2 * stride;
   uint64_t* mb = wbar + 2 * warp;
   const int tstride = gridDim.x * wpb;
   int t = blockIdx.x * wpb + warp;
   // lane 0: expect the slice's bytes and start its copies into buffer b
   auto issue = [&](int tt, int b) {
      const int s0 = a.slice_first + tt;
      const int o0 = __ldg(a.slice_off + s0), o1 = __ldg(a.slice_off + s0 + 1);
      const uint32_t bytes = (uint32_t)(o1 - o0) * 4u;
      const bool gin = MODE == PASS_CORRECTOR && a.gx, cin = a.cell && !gin;
      const int na = 3 + (MODE == PASS_CORRECTOR ? 3 : 0) + (a.mat ? 1 : 0) + (cin ? 1 : 0) + (gin ? 3 : 0);
      unsigned char* buf = wbuf + b * stride;
      float* own = reinterpret_cast<float*>(buf + buf_bytes);
      const size_t a0 = (size_t)s0 * 32;
      fence_proxy_async();
      mbar_arrive_expect_tx(&mb[b], bytes + 128u * (uint32_t)na + (uint32_t)a.stage_extra_tx);
      if (bytes) bulk_copy_g2s(buf, a.crec + o0, bytes, &mb[b]);
      bulk_copy_g2s(own, a.ax + a0, 128, &mb[b]);
      bulk_copy_g2s(own + 32, a.ay + a0, 128, &mb[b]);
      bulk_copy_g2s(own + 64, a.az + a0, 128, &mb[b]);
      if (MODE == PASS_CORRECTOR) {
         bulk_copy_g2s(own + 96, a.bx + a0, 128, &mb[b]);
         bulk_copy_g2s(own + 128, a.by + a0, 128, &mb[b]);
         bulk_copy_g2s(own + 160, a.bz + a0, 128, &mb[b]);
      }
      if (a.mat) bulk_copy_g2s(own + 192, a.mat + a0, 128, &mb[b]);
      if (cin) bulk_copy_g2s(own + 224, a.cell + a0, 128, &mb[b]);
      if (gin) {
         bulk_copy_g2s(own + 256, a.gx + a0, 128, &mb[b]);
         bulk_copy_g2s(own + 288, a.gy + a0, 128, &mb[b]);
         bulk_copy_g2s(own + 320, a.gz + a0, 128, &mb[b]);
      }
   };
   if (lane == 0) {
      mbar_init(&mb[0], 1);
      mbar_init(&mb[1], 1);
      fence_mbar_init();
      if (t < ntiles) issue(t, 0);
   }
   {  // dictionary and material table, once per block
      const int nd = dict_bytes / 16;
      for (int q = tid; q < nd; q += blockDim.x) sdict[q] = __ldg(a.cdict + q);
      if (mp_shared) {
         const int nw = a.M * (int)(sizeof(MatParams<float>) / 4);
         const float* g = reinterpret_cast<const float*>(a.mp);
         float* d = reinterpret_cast<float*>(smp);
         for (int q = tid; q < nw; q += blockDim.x) d[q] = __ldg(g + q);
      }
   }
   __syncthreads();  // barriers initialised, dictionary and table in place
   const MatParams<float>* mpt = mp_shared ? smp : a.mp;
   uint32_t phase = 0;
   int k = 0, b = 0;
   bool failed = false;
   for (; t < ntiles; t += tstride, ++k) {
      b = k & 1;
      // buffer b ^ 1 was last read in the previous iteration, closed by __syncwarp
      if (lane == 0 && t + tstride < ntiles) issue(t + tstride, b ^ 1);
      const int i = (a.slice_first + t) * 32 + lane;
      const bool act = i < a.n_upd;
      float g[3] = {0.f, 0.f, 0.f};
      if (a.thermal && (MODE == PASS_PREDICTOR || !a.gx)) thermal_xi(a, act ? i : 0, g[0], g[1], g[2]);
      const int tile_off = __ldg(a.slice_off + a.slice_first + t);
      const bool done = mbar_wait_bounded(&mb[b], (phase >> b) & 1u);
      if (__any_sync(0xffffffffu, !done)) {  // every lane takes the same branch
         failed = true;
         break;
      }
      phase ^= 1u << b;
      const unsigned char* buf = wbuf + b * stride;
      const float* own = reinterpret_cast<const float*>(buf + buf_bytes);
      if (act) {
         const int mi = a.mat ? reinterpret_cast<const int*>(own)[192 + lane] : 0;
         const MatParams<float> m = mpt[mi];
         const float S0[3] = {own[lane], own[32 + lane], own[64 + lane]};
         float E[3];
         if (MODE == PASS_CORRECTOR && a.gx) {  // the predictor's field of this step
            E[0] = own[256 + lane]; E[1] = own[288 + lane]; E[2] = own[320 + lane];
         } else {
            external_field_g<float>(a, i, m, g, a.cell ? reinterpret_cast<const int*>(own)[224 + lane] : -1, E);
            if (MODE == PASS_PREDICTOR && a.gx) { a.gx[i] = E[0]; a.gy[i] = E[1]; a.gz[i] = E[2]; }
         }
         const int4* sb = reinterpret_cast<const int4*>(buf);
         float H[3];
         if (MODE == PASS_PREDICTOR) {
            spin_field<float, FMT_DMI_TAB, 0, true, false, REC_COMPACT>(a, i, mi, m, a.ax, a.ay, a.az, S0, H, sb,
                                                                        tile_off, sdict);
            H[0] += E[0]; H[1] += E[1]; H[2] += E[2];
            llg_predict_finish<float>(a, i, m, S0, H);
         } else {
            const float S1[3] = {own[96 + lane], own[128 + lane], own[160 + lane]};
            spin_field<float, FMT_DMI_TAB, 0, true, false, REC_COMPACT>(a, i, mi, m, a.bx, a.by, a.bz, S1, H, sb,
                                                                        tile_off, sdict);
            H[0] += E[0]; H[1] += E[1]; H[2] += E[2];
            llg_correct_finish<float>(a, i, m, S0, S1, H);
         }
      }
      __syncwarp();  // buffer b fully read before lane 0 refills it
   }
   if (failed && lane == 0) {
      atomicOr(a.status, 2);
      // copies still in flight: the one waited for and the next slice's
      mbar_wait_bounded(&mb[b], (phase >> b) & 1u);
      if (t + tstride < ntiles) mbar_wait_bounded(&mb[b ^ 1], (phase >> (b ^ 1)) & 1u);
   }
   __syncwarp();
}

// Window-staged passes (FP32 compact records): besides the tile's bond words,
// the neighbour spins the tile reads are bulk-copied into shared memory too,
// as the tile's "window": the few contiguous atom ranges (segments) that hold
// every neighbour of the tile's atoms (for a lattice numbered cell by cell,
// the neighbouring rows of cells), planned on the host, each word naming its
// neighbour by window slot.  Warp 0 sets the expected bytes and issues one
// bulk copy per segment and spin component plus one for the words; the
// gathers then read shared memory only.  One tile per block.  Shared memory:
// words (rec_bytes), three components of wmax slots, the dictionary.
template <int MODE, int SL>
__global__ void __launch_bounds__(32 * SL, 24 / SL) llg_window_kernel(const LLGArgs<float> a, int nslices,
                                                                       int rec_bytes, int wmax) {
   extern __shared__ __align__(128) unsigned char stage_smem[];
   __shared__ __align__(8) uint64_t mbar;
   const int tid = threadIdx.x;
   const int t = blockIdx.x;
   const uint32_t* swords = reinterpret_cast<const uint32_t*>(stage_smem);
   float* wx = reinterpret_cast<float*>(stage_smem + rec_bytes);
   float4* sdict = reinterpret_cast<float4*>(wx + 3 * wmax);
   const int s0 = t * SL;
   const int tile_off = __ldg(a.slice_off + s0);
   // warp 0 initialises the barrier and issues every copy at once (words,
   // dictionary, window segments); the other warps see the initialised
   // barrier after the block barrier below, before they wait on it
   if (tid < 32) {
      if (tid == 0) {
         mbar_init(&mbar, 1);
         fence_mbar_init();
      }
      __syncwarp();
      const int o1 = __ldg(a.slice_off + min(s0 + SL, nslices));
      const int sb = __ldg(a.wtile_seg + t), se = __ldg(a.wtile_seg + t + 1);
      const uint32_t rb = (uint32_t)(o1 - tile_off) * 4u;
      const uint32_t db = 16u * (uint32_t)(a.tab_scalar ? a.cdict_n : 2 * a.cdict_n);
      if (tid == 0) {
         fence_proxy_async();
         mbar_arrive_expect_tx(&mbar, rb + db + 12u * (uint32_t)__ldg(a.wtile_w + t) + (uint32_t)a.stage_extra_tx);
         if (rb) bulk_copy_g2s(stage_smem, a.lrec + tile_off, rb, &mbar);
         bulk_copy_g2s(sdict, a.cdict, db, &mbar);
      }
      __syncwarp();
      const float* gx = MODE == PASS_PREDICTOR ? a.ax : a.bx;
      const float* gy = MODE == PASS_PREDICTOR ? a.ay : a.by;
      const float* gz = MODE == PASS_PREDICTOR ? a.az : a.bz;
      for (int q = sb + tid; q < se; q += 32) {
         const int4 g = __ldg(a.wseg + q);  // {first atom, atoms, first slot, 0}
         const uint32_t nb = 4u * (uint32_t)g.y;
         bulk_copy_g2s(wx + g.z, gx + g.x, nb, &mbar);
         bulk_copy_g2s(wx + wmax + g.z, gy + g.x, nb, &mbar);
         bulk_copy_g2s(wx + 2 * wmax + g.z, gz + g.x, nb, &mbar);
      }
   }
   // own-atom work overlapping the copies: state, material, external field
   const int i = s0 * 32 + tid;
   const bool act = i < a.n_upd;
   const int ii = act ? i : a.n_upd - 1;
   const int mi = a.mat ? __ldg(a.mat + ii) : 0;
   const MatParams<float> m = a.mp[mi];
   float S0[3] = {a.ax[ii], a.ay[ii], a.az[ii]};
   float S1[3];
   if (MODE == PASS_CORRECTOR) { S1[0] = a.bx[ii]; S1[1] = a.by[ii]; S1[2] = a.bz[ii]; }
   float E[3];
   external_field<float>(a, ii, m, true, E);
   __syncthreads();  // the barrier's initialisation is visible to every thread
   const bool done = mbar_wait_bounded(&mbar, 0);
   if (__syncthreads_or(!done)) {
      if (tid == 0) {
         atomicOr(a.status, 2);
         mbar_wait_bounded(&mbar, 0);  // copies still in flight
      }
      __syncthreads();
      return;
   }
   if (!act) return;
   const int4* sb = reinterpret_cast<const int4*>(swords);
   float H[3];
   if (MODE == PASS_PREDICTOR) {
      spin_field<float, FMT_DMI_TAB, 0, true, false, REC_WINDOW>(a, i, mi, m, a.ax, a.ay, a.az, S0, H, sb, tile_off,
                                                                 sdict, wx, wmax);
      H[0] += E[0]; H[1] += E[1]; H[2] += E[2];
      llg_predict_finish<float>(a, i, m, S0, H);
   } else {
      spin_field<float, FMT_DMI_TAB, 0, true, false, REC_WINDOW>(a, i, mi, m, a.bx, a.by, a.bz, S1, H, sb, tile_off,
                                                                 sdict, wx, wmax);
      H[0] += E[0]; H[1] += E[1]; H[2] += E[2];
      llg_correct_finish<float>(a, i, m, S0, S1, H);
   }
}

// bytes of the largest tile's 16-byte record range (buffer size) for the
// host; compact records take a quarter of it
inline int staged_tile_bytes(const std::vector<int>& slice_off, int sl) {
   const int nsl = (int)slice_off.size() - 1;
   int mx = 0;
   for (int s0 = 0; s0 < nsl; s0 += sl) {
      const int s1 = std::min(s0 + sl, nsl);
      mx = std::max(mx, (slice_off[s1] - slice_off[s0]) * 16);
   }
   return mx;
}

}  // namespace vgpu
