// Device helpers shared by the fused LLG, statistics, Monte Carlo and adjoint
// kernels: the SELL-32 exchange gather, anisotropy and external fields, the
// LLG right-hand side, and in-register Philox thermal noise.
#pragma once
#include <cuda_runtime.h>

#include "philox.cuh"
#include "vgpu_internal.cuh"

namespace vgpu {

template <typename R> __device__ __forceinline__ R rsqrt_(R x);
template <> __device__ __forceinline__ float rsqrt_<float>(float x) { return rsqrtf(x); }
template <> __device__ __forceinline__ double rsqrt_<double>(double x) { return 1.0 / sqrt(x); }

template <typename R>
__device__ __forceinline__ void thermal_xi(const LLGArgs<R>& a, int i, R& gx, R& gy, R& gz) {
   if (a.noise_mode == VGPU_NOISE_REPLAY) {
      gx = a.xi[i];
      gy = a.xi[a.n + i];
      gz = a.xi[2 * a.n + i];
      return;
   }
   // batched systems: system k's atoms draw the stream of a single system
   // seeded seed + k, with their own local index (same numbers as a plain run)
   uint32_t li = (uint32_t)i + a.noise_base, klo = a.seed_lo, khi = a.seed_hi;
   if (a.sys_off) {
      const int k = (a.mat ? __ldg(a.mat + i) : 0) / a.m_per_sys;
      li = (uint32_t)(i - __ldg(a.sys_off + k));
      const uint64_t s = (((uint64_t)a.seed_hi << 32) | a.seed_lo) + (uint64_t)k;
      klo = (uint32_t)s;
      khi = (uint32_t)(s >> 32);
   }
   u32x4 c = {li, (uint32_t)a.step, (uint32_t)(a.step >> 32), RNG_THERMAL};
   u32x4 r = philox4x32_10(c, klo, khi);
   if (sizeof(R) == 4) {
      // fast approximations: each Gaussian within 1e-5 of the exact transform
      float s1, c1;
      const float r1 = bm_radius_fast(r.x);
      bm_angle_fast(r.y, c1, s1);
      gx = (R)(r1 * c1);
      gy = (R)(r1 * s1);
      gz = (R)(bm_radius_fast(r.z) * bm_cos_fast(r.w));
   } else {
      double s1, c1, s2, c2;
      const double r1 = sqrt(-2.0 * log(u01d(r.x)));
      const double r2 = sqrt(-2.0 * log(u01d(r.z)));
      sincospi(2.0 * u01d(r.y), &s1, &c1);
      sincospi(2.0 * u01d(r.w), &s2, &c2);
      gx = (R)(r1 * c1);
      gy = (R)(r1 * s1);
      gz = (R)(r2 * c2);
   }
}

// One bond of the diagonal-plus-DMI exchange: h += J s_j + d x s_j, with J
// the diagonal (jx, jy, jz) and d the antisymmetric part.  FP32: three fused
// multiply-adds per component chained through the field (one instruction per
// component fewer than the products summed first); FP64: the products summed
// first, then added.  Every FP32 record layout uses this one form, so their
// fields stay identical.
template <typename R>
__device__ __forceinline__ void dmi_bond(R jx, R jy, R jz, R dx, R dy, R dz, R x, R y, R z, R& hx, R& hy, R& hz);
template <>
__device__ __forceinline__ void dmi_bond<float>(float jx, float jy, float jz, float dx, float dy, float dz, float x,
                                                float y, float z, float& hx, float& hy, float& hz) {
   hx = fmaf(-dz, y, fmaf(dy, z, fmaf(jx, x, hx)));
   hy = fmaf(-dx, z, fmaf(dz, x, fmaf(jy, y, hy)));
   hz = fmaf(-dy, x, fmaf(dx, y, fmaf(jz, z, hz)));
}
template <>
__device__ __forceinline__ void dmi_bond<double>(double jx, double jy, double jz, double dx, double dy, double dz,
                                                 double x, double y, double z, double& hx, double& hy, double& hz) {
   hx += jx * x + (dy * z - dz * y);
   hy += jy * y + (dz * x - dx * z);
   hz += jz * z + (dx * y - dy * x);
}

// exchange gather of atom i over its SELL row, sources (sx,sy,sz)
template <typename R> __device__ __forceinline__ R ld_src(const R* p, int coherent) {
   return coherent ? __ldcg(p) : __ldg(p);
}

// The row is given by its first entry (base) and width (w); exchange_gather
// below finds them from the slice offsets of atom i.
// LOAD = 1: source spins were written earlier in the same launch by other
// blocks (persistent batched kernel) and are read through L2 (ld.global.cg)
template <typename R, int FMT, int LOAD = 0>
__device__ __forceinline__ void exchange_gather_row(const LLGArgs<R>& a, int base, int w, int mi,
                                                    const R* __restrict__ sx, const R* __restrict__ sy,
                                                    const R* __restrict__ sz, R& hx, R& hy, R& hz) {
   const R* __restrict__ tab = a.jtab;
#pragma unroll 4
   for (int k = 0; k < w; ++k) {
      const int e = base + 32 * k;
      const int c = __ldg(a.col + e);
      const int j = c & a.idx_mask;
      const R x = ld_src(sx + j, LOAD), y = ld_src(sy + j, LOAD), z = ld_src(sz + j, LOAD);
      if (FMT == FMT_ISO_TAB) {
         const int mj = a.mat_shift ? (c >> a.mat_shift) : 0;
         const R J = __ldg(tab + mi * a.M + mj);
         hx += J * x; hy += J * y; hz += J * z;
      } else if (FMT == FMT_ISO_BOND) {
         const R J = __ldg(a.jb[0] + e);
         hx += J * x; hy += J * y; hz += J * z;
      } else if (FMT == FMT_VEC_TAB) {
         const int mj = a.mat_shift ? (c >> a.mat_shift) : 0;
         const R* t = tab + 3 * (mi * a.M + mj);
         hx += __ldg(t) * x; hy += __ldg(t + 1) * y; hz += __ldg(t + 2) * z;
      } else if (FMT == FMT_VEC_BOND) {
         hx += __ldg(a.jb[0] + e) * x; hy += __ldg(a.jb[1] + e) * y; hz += __ldg(a.jb[2] + e) * z;
      } else if (FMT == FMT_DMI_TAB) {
         const int mj = a.mat_shift ? (c >> a.mat_shift) : 0;
         const R* t = tab + 3 * (mi * a.M + mj);
         const R dx = __ldg(a.jb[0] + e), dy = __ldg(a.jb[1] + e), dz = __ldg(a.jb[2] + e);
         // diag part plus the antisymmetric part written as d x s_j
         dmi_bond<R>(__ldg(t), __ldg(t + 1), __ldg(t + 2), dx, dy, dz, x, y, z, hx, hy, hz);
      } else {  // FMT_TENSOR_BOND
         const R t0 = __ldg(a.jb[0] + e), t1 = __ldg(a.jb[1] + e), t2 = __ldg(a.jb[2] + e);
         const R t3 = __ldg(a.jb[3] + e), t4 = __ldg(a.jb[4] + e), t5 = __ldg(a.jb[5] + e);
         const R t6 = __ldg(a.jb[6] + e), t7 = __ldg(a.jb[7] + e), t8 = __ldg(a.jb[8] + e);
         hx += (t0 * x + t1 * y + t2 * z);
         hy += (t3 * x + t4 * y + t5 * z);
         hz += (t6 * x + t7 * y + t8 * z);
      }
   }
}

template <typename R, int FMT, int LOAD = 0>
__device__ __forceinline__ void exchange_gather(const LLGArgs<R>& a, int i, int mi, const R* __restrict__ sx,
                                                const R* __restrict__ sy, const R* __restrict__ sz, R& hx,
                                                R& hy, R& hz) {
   const int sl = i >> 5;
   const int off = __ldg(a.slice_off + sl);
   const int w = (__ldg(a.slice_off + sl + 1) - off) >> 5;
   exchange_gather_row<R, FMT, LOAD>(a, off + (i & 31), w, mi, sx, sy, sz, hx, hy, hz);
}

// Row of compile-time width W read from packed 16-byte bond records
// {neighbour | material bits, d_x, d_y, d_z} (FMT_DMI_TAB) or from the
// neighbour index alone (FMT_ISO_TAB), fully unrolled so that all W record
// loads and 3W neighbour-spin loads of a thread are in flight together.
// Same arithmetic, in the same bond order, as exchange_gather.
// STAGED: the records of this row were bulk-copied to shared memory; srec
// points at the thread's first record there (stride 32 records per bond).
template <typename R, int FMT, int W, int LOAD, bool STAGED>
__device__ __forceinline__ void exchange_gather_w(const LLGArgs<R>& a, int base, int mi, const R* __restrict__ sx,
                                                  const R* __restrict__ sy, const R* __restrict__ sz, R& hx, R& hy,
                                                  R& hz, const int4* srec) {
   const R* __restrict__ tab = a.jtab;
   if (FMT == FMT_DMI_TAB && STAGED) {
      // records in shared memory: take only the neighbour words first so that
      // the registers hold the 3W gathered spins (all in flight together), and
      // re-read each bond's d vector from shared memory where it is used
      const int* sw = reinterpret_cast<const int*>(srec);
      int c[W];
#pragma unroll
      for (int k = 0; k < W; ++k) c[k] = sw[128 * k];
      R x[W], y[W], z[W];
#pragma unroll
      for (int k = 0; k < W; ++k) {
         const int j = c[k] & a.idx_mask;
         x[k] = ld_src(sx + j, LOAD); y[k] = ld_src(sy + j, LOAD); z[k] = ld_src(sz + j, LOAD);
      }
#pragma unroll
      for (int k = 0; k < W; ++k) {
         const int mj = a.mat_shift ? (c[k] >> a.mat_shift) : 0;
         const R dx = __int_as_float(sw[128 * k + 1]), dy = __int_as_float(sw[128 * k + 2]),
                 dz = __int_as_float(sw[128 * k + 3]);
         if (a.tab_scalar) {
            const R J = __ldg(a.jtab_s + mi * a.M + mj);
            dmi_bond<R>(J, J, J, dx, dy, dz, x[k], y[k], z[k], hx, hy, hz);
         } else {
            const R* t = tab + 3 * (mi * a.M + mj);
            dmi_bond<R>(__ldg(t), __ldg(t + 1), __ldg(t + 2), dx, dy, dz, x[k], y[k], z[k], hx, hy, hz);
         }
      }
   } else if (FMT == FMT_DMI_TAB) {
      int4 rec[W];
#pragma unroll
      for (int k = 0; k < W; ++k) rec[k] = STAGED ? srec[32 * k] : __ldg(a.rec + base + 32 * k);
      R x[W], y[W], z[W];
#pragma unroll
      for (int k = 0; k < W; ++k) {
         const int j = rec[k].x & a.idx_mask;
         x[k] = ld_src(sx + j, LOAD); y[k] = ld_src(sy + j, LOAD); z[k] = ld_src(sz + j, LOAD);
      }
#pragma unroll
      for (int k = 0; k < W; ++k) {
         const int mj = a.mat_shift ? (rec[k].x >> a.mat_shift) : 0;
         const R dx = __int_as_float(rec[k].y), dy = __int_as_float(rec[k].z), dz = __int_as_float(rec[k].w);
         if (a.tab_scalar) {
            // isotropic diagonal: one coupling per material pair (scalar table)
            const R J = __ldg(a.jtab_s + mi * a.M + mj);
            dmi_bond<R>(J, J, J, dx, dy, dz, x[k], y[k], z[k], hx, hy, hz);
         } else {
            const R* t = tab + 3 * (mi * a.M + mj);
            dmi_bond<R>(__ldg(t), __ldg(t + 1), __ldg(t + 2), dx, dy, dz, x[k], y[k], z[k], hx, hy, hz);
         }
      }
   } else {  // FMT_ISO_TAB
      int c[W];
#pragma unroll
      for (int k = 0; k < W; ++k) c[k] = __ldg(a.col + base + 32 * k);
      R x[W], y[W], z[W];
#pragma unroll
      for (int k = 0; k < W; ++k) {
         const int j = c[k] & a.idx_mask;
         x[k] = ld_src(sx + j, LOAD); y[k] = ld_src(sy + j, LOAD); z[k] = ld_src(sz + j, LOAD);
      }
#pragma unroll
      for (int k = 0; k < W; ++k) {
         const int mj = a.mat_shift ? (c[k] >> a.mat_shift) : 0;
         const R J = __ldg(tab + mi * a.M + mj);
         hx += J * x[k]; hy += J * y[k]; hz += J * z[k];
      }
   }
}

// Row of compile-time width W read from compact records: one word per bond,
// neighbour | coupling index << crec_shift, the coupling {J, d} taken from the
// dictionary (shared memory in the staged passes, global otherwise).  Same
// arithmetic, in the same bond order, as the FMT_DMI_TAB branch above, on the
// same coupling values, so the two record layouts give identical fields.
// STAGED: sw points at the thread's first word in shared memory (stride 32).
template <typename R, int W, int LOAD, bool STAGED>
__device__ __forceinline__ void exchange_gather_c(const LLGArgs<R>& a, int base, const R* __restrict__ sx,
                                                  const R* __restrict__ sy, const R* __restrict__ sz, R& hx, R& hy,
                                                  R& hz, const uint32_t* sw, const float4* dict) {
   const uint32_t jmask = (1u << a.crec_shift) - 1u;
   uint32_t c[W];
#pragma unroll
   for (int k = 0; k < W; ++k) c[k] = STAGED ? sw[32 * k] : __ldg(a.crec + base + 32 * k);
   R x[W], y[W], z[W];
#pragma unroll
   for (int k = 0; k < W; ++k) {
      const int j = (int)(c[k] & jmask);
      x[k] = ld_src(sx + j, LOAD); y[k] = ld_src(sy + j, LOAD); z[k] = ld_src(sz + j, LOAD);
   }
#pragma unroll
   for (int k = 0; k < W; ++k) {
      const uint32_t q = c[k] >> a.crec_shift;
      const float4 e = dict[q];
      const R dx = e.y, dy = e.z, dz = e.w;
      if (a.tab_scalar) {
         const R J = e.x;
         dmi_bond<R>(J, J, J, dx, dy, dz, x[k], y[k], z[k], hx, hy, hz);
      } else {
         const float4 e2 = dict[a.cdict_n + q];
         dmi_bond<R>((R)e.x, (R)e2.x, (R)e2.y, dx, dy, dz, x[k], y[k], z[k], hx, hy, hz);
      }
   }
}

// Row read from window-staged records: per bond the word slot | coupling
// index << 16, the neighbour spin taken from the tile's window of spins in
// shared memory (wx, wx + wmax, wx + 2 wmax) and the coupling from the
// dictionary.  W > 0: compile-time width (all loads of the row first); W = 0:
// width w_rt.  Same arithmetic, in the same bond order, on the same values as
// exchange_gather_c, so the results are identical.
template <typename R, int W>
__device__ __forceinline__ void exchange_gather_win(const LLGArgs<R>& a, int w_rt, R& hx, R& hy, R& hz,
                                                    const uint32_t* sw, const float4* dict, const float* wx,
                                                    int wmax) {
   const float* wy = wx + wmax;
   const float* wz = wy + wmax;
   auto bond = [&](uint32_t c, R x, R y, R z) {
      const float4 e = dict[c >> 16];
      const R dx = e.y, dy = e.z, dz = e.w;
      if (a.tab_scalar) {
         const R J = e.x;
         dmi_bond<R>(J, J, J, dx, dy, dz, x, y, z, hx, hy, hz);
      } else {
         const float4 e2 = dict[a.cdict_n + (c >> 16)];
         dmi_bond<R>((R)e.x, (R)e2.x, (R)e2.y, dx, dy, dz, x, y, z, hx, hy, hz);
      }
   };
   if (W > 0) {
      uint32_t c[W > 0 ? W : 1];
      R x[W > 0 ? W : 1], y[W > 0 ? W : 1], z[W > 0 ? W : 1];
#pragma unroll
      for (int k = 0; k < W; ++k) c[k] = sw[32 * k];
#pragma unroll
      for (int k = 0; k < W; ++k) {
         const int s = (int)(c[k] & 0xffffu);
         x[k] = wx[s]; y[k] = wy[s]; z[k] = wz[s];
      }
#pragma unroll
      for (int k = 0; k < W; ++k) bond(c[k], x[k], y[k], z[k]);
   } else {
      for (int k = 0; k < w_rt; ++k) {
         const uint32_t c = sw[32 * k];
         const int s = (int)(c & 0xffffu);
         bond(c, wx[s], wy[s], wz[s]);
      }
   }
}

// biquadratic exchange field of atom i at own spin S over its SELL-32 list:
// sum_j 2 J_bq (S.s_j) s_j (src/exchange/biquadratic_fields.cpp:60-76)
template <typename R, int LOAD = 0>
__device__ __forceinline__ void biquadratic_field(const LLGArgs<R>& a, int i, const R* __restrict__ sx,
                                                  const R* __restrict__ sy, const R* __restrict__ sz, const R S[3],
                                                  R& hx, R& hy, R& hz) {
   hx = hy = hz = 0;
   const int sl = i >> 5;
   const int off = __ldg(a.bq_off + sl);
   const int w = (__ldg(a.bq_off + sl + 1) - off) >> 5;
   const int base = off + (i & 31);
   for (int k = 0; k < w; ++k) {
      const int e = base + 32 * k;
      const int j = __ldg(a.bq_col + e);
      const R twoJbq = (R)2 * __ldg(a.bq_j + e);
      const R x = ld_src(sx + j, LOAD), y = ld_src(sy + j, LOAD), z = ld_src(sz + j, LOAD);
      const R d = S[0] * x + S[1] * y + S[2] * z;
      hx += twoJbq * x * d;
      hy += twoJbq * y * d;
      hz += twoJbq * z * d;
   }
}

// biquadratic energy of atom i at spin S: -sum_j J_bq (S.s_j)^2
// (src/exchange/biquadratic_energy.cpp:24-37)
template <typename E, typename R>
__device__ __forceinline__ E biquadratic_energy(const LLGArgs<R>& a, int i, const E S[3]) {
   E en = 0;
   const int sl = i >> 5;
   const int off = __ldg(a.bq_off + sl);
   const int w = (__ldg(a.bq_off + sl + 1) - off) >> 5;
   const int base = off + (i & 31);
   for (int k = 0; k < w; ++k) {
      const int e = base + 32 * k;
      const int j = __ldg(a.bq_col + e);
      const E J = (E)__ldg(a.bq_j + e);
      const E d = S[0] * (E)a.ax[j] + S[1] * (E)a.ay[j] + S[2] * (E)a.az[j];
      en -= J * d * d;
   }
   return en;
}

// exchange field with the fixed-width fast paths (FP32, packed records).
// STAGED (FMT_DMI_TAB only): srec_tile is the shared-memory copy of the
// records of the tile starting at slice_off[tile_slice0] (16-byte records, or
// compact words when a.crec is set, with the dictionary copied to sdict).
// REC: which FP32 DMI record layout the caller was compiled for (REC_ANY:
// compact when a.crec is set, else 16-byte; the staged passes fix one).
template <typename R, int FMT, int LOAD, bool STAGED = false, int REC = REC_ANY>
__device__ __forceinline__ void exchange_field(const LLGArgs<R>& a, int i, int mi, const R* __restrict__ sx,
                                               const R* __restrict__ sy, const R* __restrict__ sz, R& hx, R& hy,
                                               R& hz, const int4* srec_tile = nullptr, int tile_off = 0,
                                               const float4* sdict = nullptr, const float* swin = nullptr,
                                               int wmax = 0) {
   if (REC == REC_WINDOW) {  // staged window passes (FP32 FMT_DMI_TAB): every width from shared memory
      const int sl = i >> 5;
      const int off = __ldg(a.slice_off + sl);
      const int w = (__ldg(a.slice_off + sl + 1) - off) >> 5;
      const uint32_t* sw = reinterpret_cast<const uint32_t*>(srec_tile) + (off + (i & 31) - tile_off);
      if (w == 12) exchange_gather_win<R, 12>(a, w, hx, hy, hz, sw, sdict, swin, wmax);
      else if (w == 6) exchange_gather_win<R, 6>(a, w, hx, hy, hz, sw, sdict, swin, wmax);
      else exchange_gather_win<R, 0>(a, w, hx, hy, hz, sw, sdict, swin, wmax);
      return;
   }
   if (sizeof(R) == 4 && FMT == FMT_DMI_TAB && REC != REC_WIDE && (REC == REC_COMPACT || a.crec)) {
      const int sl = i >> 5;
      const int off = __ldg(a.slice_off + sl);
      const int w = (__ldg(a.slice_off + sl + 1) - off) >> 5;
      const int base = off + (i & 31);
      const uint32_t* sw = STAGED ? reinterpret_cast<const uint32_t*>(srec_tile) + (base - tile_off) : nullptr;
      const float4* dict = STAGED ? sdict : a.cdict;
      if (w == 12) { exchange_gather_c<R, 12, LOAD, STAGED>(a, base, sx, sy, sz, hx, hy, hz, sw, dict); return; }
      if (w == 6) { exchange_gather_c<R, 6, LOAD, STAGED>(a, base, sx, sy, sz, hx, hy, hz, sw, dict); return; }
   } else if (sizeof(R) == 4 && (FMT == FMT_DMI_TAB || FMT == FMT_ISO_TAB) && REC != REC_COMPACT &&
              (FMT == FMT_ISO_TAB || a.rec)) {
      const int sl = i >> 5;
      const int off = __ldg(a.slice_off + sl);
      const int w = (__ldg(a.slice_off + sl + 1) - off) >> 5;
      const int base = off + (i & 31);
      const int4* sr = STAGED ? srec_tile + (base - tile_off) : nullptr;
      if (w == 12) { exchange_gather_w<R, FMT, 12, LOAD, STAGED>(a, base, mi, sx, sy, sz, hx, hy, hz, sr); return; }
      if (w == 6) { exchange_gather_w<R, FMT, 6, LOAD, STAGED>(a, base, mi, sx, sy, sz, hx, hy, hz, sr); return; }
   }
   exchange_gather<R, FMT, LOAD>(a, i, mi, sx, sy, sz, hx, hy, hz);
}

// spin-dependent field of atom i at spin S: exchange + anisotropy
// (calculate_spin_fields, src/simulate/fields.cpp:67-118)
// EXT = false compiles the passes without the higher-order anisotropy terms
// (register budget of the common case); launchers pick EXT from a.aniso_ext.
template <typename R, int FMT, int LOAD = 0, bool STAGED = false, bool EXT = true, int REC = REC_ANY>
__device__ __forceinline__ void spin_field(const LLGArgs<R>& a, int i, int mi, const MatParams<R>& m,
                                           const R* sx, const R* sy, const R* sz, const R S[3], R H[3],
                                           const int4* srec_tile = nullptr, int tile_off = 0,
                                           const float4* sdict = nullptr, const float* swin = nullptr,
                                           int wmax = 0) {
   R hx = 0, hy = 0, hz = 0;
   exchange_field<R, FMT, LOAD, STAGED, REC>(a, i, mi, sx, sy, sz, hx, hy, hz, srec_tile, tile_off, sdict, swin,
                                             wmax);
   if (EXT && a.bq_off) {
      // biquadratic exchange (exchange/biquadratic_fields.cpp): its own sum,
      // added to the bilinear field as exchange::fields does
      R bx, by, bz;
      biquadratic_field<R, LOAD>(a, i, sx, sy, sz, S, bx, by, bz);
      hx += bx; hy += by; hz += bz;
   }
   // anisotropy terms in the order of anisotropy::fields (src/anisotropy/fields.cpp:42-63)
   if (a.uniaxial) {
      const R sdote = S[0] * m.kux + S[1] * m.kuy + S[2] * m.kuz;
      const R k2 = (R)2 * m.ku2 * sdote;
      hx += m.kux * k2; hy += m.kuy * k2; hz += m.kuz * k2;
   }
   if (EXT && (a.aniso_ext & (ANI_U4 | ANI_U6))) {
      const R sdote = S[0] * m.kux + S[1] * m.kuy + S[2] * m.kuz;
      const R sdote3 = sdote * sdote * sdote;
      if (a.aniso_ext & ANI_U4) {  // uniaxial_fourth_order.cpp: (2/3)(1/8) ku4 (140 (s.e)^3 - 60 s.e) e
         const R k4 = (R)(1.0 / 8.0 * 2.0 / 3.0) * m.ku4 * ((R)140 * sdote3 - (R)60 * sdote);
         hx += m.kux * k4; hy += m.kuy * k4; hz += m.kuz * k4;
      }
      if (a.aniso_ext & ANI_U6) {  // uniaxial_sixth_order.cpp: (2/3)(1/16) ku6 (1386 s^5 - 1260 s^3 + 210 s) e
         const R sdote5 = sdote3 * sdote * sdote;
         const R k6 = (R)(1.0 / 16.0 * 2.0 / 3.0) * m.ku6 * ((R)1386 * sdote5 - (R)1260 * sdote3 + (R)210 * sdote);
         hx += m.kux * k6; hy += m.kuy * k6; hz += m.kuz * k6;
      }
   }
   if (a.cubic) {
      const R k4 = (R)2 * m.kc4;
      hx += S[0] * S[0] * S[0] * k4;
      hy += S[1] * S[1] * S[1] * k4;
      hz += S[2] * S[2] * S[2] * k4;
   }
   if (EXT && (a.aniso_ext & (ANI_CROT | ANI_C6 | ANI_NEEL))) {
      if (a.aniso_ext & ANI_CROT) {  // cubic_fourth_order_rotation.cpp: 2 kc4 sum_k (s.e_k)^3 e_k
         const R* e = m.kcb;
         const R k4 = (R)2 * m.kc4;
         const R d1 = S[0] * e[0] + S[1] * e[1] + S[2] * e[2];
         const R d2 = S[0] * e[3] + S[1] * e[4] + S[2] * e[5];
         const R d3 = S[0] * e[6] + S[1] * e[7] + S[2] * e[8];
         const R d13 = d1 * d1 * d1, d23 = d2 * d2 * d2, d33 = d3 * d3 * d3;
         hx += k4 * (d13 * e[0] + d23 * e[3] + d33 * e[6]);
         hy += k4 * (d13 * e[1] + d23 * e[4] + d33 * e[7]);
         hz += k4 * (d13 * e[2] + d23 * e[5] + d33 * e[8]);
      }
      if (a.aniso_ext & ANI_C6) {  // cubic_sixth_order.cpp: H_x = -2 kc6 s_x s_y^2 s_z^2 (cyclic)
         const R k6 = (R)(-2) * m.kc6;
         const R x2 = S[0] * S[0], y2 = S[1] * S[1], z2 = S[2] * S[2];
         hx += S[0] * y2 * z2 * k6;
         hy += S[1] * z2 * x2 * k6;
         hz += S[2] * x2 * y2 * k6;
      }
      if (a.aniso_ext & ANI_NEEL) {  // neel.cpp: H += 2 T s with the atom's surface tensor T
         const size_t st = (size_t)a.n_alloc;
         const R* t = a.neel + i;
         const R t0 = __ldg(t), t1 = __ldg(t + st), t2 = __ldg(t + 2 * st), t3 = __ldg(t + 3 * st),
                 t4 = __ldg(t + 4 * st), t5 = __ldg(t + 5 * st), t6 = __ldg(t + 6 * st), t7 = __ldg(t + 7 * st),
                 t8 = __ldg(t + 8 * st);
         hx += (R)2 * (t0 * S[0] + t1 * S[1] + t2 * S[2]);
         hy += (R)2 * (t3 * S[0] + t4 * S[1] + t5 * S[2]);
         hz += (R)2 * (t6 * S[0] + t7 * S[1] + t8 * S[2]);
      }
   }
   H[0] = hx; H[1] = hy; H[2] = hz;
}

// anisotropy energy of atom i at spin S in the order of
// anisotropy::single_spin_energy (src/anisotropy/energy.cpp:27-36), E in T
// (uniaxial_second_order.cpp, ..._fourth_order.cpp, ..._sixth_order.cpp,
// cubic_fourth_order.cpp, cubic_fourth_order_rotation.cpp,
// cubic_sixth_order.cpp, neel.cpp energy functions; the reference's decimal
// 1/12 and 1/24 literals kept)
// EXT_ONLY: the higher-order terms alone (callers that add the second-order
// uniaxial and fourth-order cubic terms themselves).
template <typename E, typename R, bool EXT_ONLY = false>
__device__ __forceinline__ E anisotropy_energy(const LLGArgs<R>& a, int i, const MatParams<R>& m, const E S[3]) {
   E an = 0;
   const E kux = (E)m.kux, kuy = (E)m.kuy, kuz = (E)m.kuz;
   if (!EXT_ONLY && a.uniaxial) {
      const E sd = S[0] * kux + S[1] * kuy + S[2] * kuz;
      an += -(E)m.ku2 * (sd * sd);
   }
   if (a.aniso_ext & ANI_U4) {
      const E sd = S[0] * kux + S[1] * kuy + S[2] * kuz;
      const E sd2 = sd * sd;
      an += (E)(-0.08333333333) * (E)m.ku4 * ((E)35 * sd2 * sd2 - (E)30 * sd2);
   }
   if (a.aniso_ext & ANI_U6) {
      const E sd = S[0] * kux + S[1] * kuy + S[2] * kuz;
      const E sd2 = sd * sd;
      an += (E)(-0.04166666666) * (E)m.ku6 * ((E)231 * sd2 * sd2 * sd2 - (E)315 * sd2 * sd2 + (E)105 * sd2);
   }
   if (!EXT_ONLY && a.cubic) {
      const E x4 = S[0] * S[0] * S[0] * S[0], y4 = S[1] * S[1] * S[1] * S[1], z4 = S[2] * S[2] * S[2] * S[2];
      an += (E)(-0.5) * (E)m.kc4 * (x4 + y4 + z4);
   }
   if (a.aniso_ext & ANI_CROT) {
      const R* e = m.kcb;
      const E d1 = S[0] * (E)e[0] + S[1] * (E)e[1] + S[2] * (E)e[2];
      const E d2 = S[0] * (E)e[3] + S[1] * (E)e[4] + S[2] * (E)e[5];
      const E d3 = S[0] * (E)e[6] + S[1] * (E)e[7] + S[2] * (E)e[8];
      const E x4 = d1 * d1 * d1 * d1, y4 = d2 * d2 * d2 * d2, z4 = d3 * d3 * d3 * d3;
      an += (E)(-0.5) * (E)m.kc4 * (x4 + y4 + z4);
   }
   if (a.aniso_ext & ANI_C6) an += (E)m.kc6 * S[0] * S[0] * S[1] * S[1] * S[2] * S[2];
   if (a.aniso_ext & ANI_NEEL) {
      const size_t st = (size_t)a.n_alloc;
      const R* t = a.neel + i;
      const E t0 = (E)__ldg(t), t1 = (E)__ldg(t + st), t2 = (E)__ldg(t + 2 * st), t3 = (E)__ldg(t + 3 * st),
              t4 = (E)__ldg(t + 4 * st), t5 = (E)__ldg(t + 5 * st), t6 = (E)__ldg(t + 6 * st),
              t7 = (E)__ldg(t + 7 * st), t8 = (E)__ldg(t + 8 * st);
      const E en = S[0] * t0 * S[0] + S[0] * t1 * S[1] + S[0] * t2 * S[2] + S[1] * t3 * S[0] + S[1] * t4 * S[1] +
                   S[1] * t5 * S[2] + S[2] * t6 * S[0] + S[2] * t7 * S[1] + S[2] * t8 * S[2];
      an += (E)(-1) * en;
   }
   return an;
}

// external field (calculate_external_fields, fields.cpp:120-169)
template <typename R>
__device__ __forceinline__ void external_field_g(const LLGArgs<R>& a, int i, const MatParams<R>& m, const R g[3],
                                                 int cell_id, R E[3]);

template <typename R>
__device__ __forceinline__ void external_field(const LLGArgs<R>& a, int i, const MatParams<R>& m, bool with_noise,
                                               R E[3]) {
   R g[3] = {0, 0, 0};
   if (a.thermal && with_noise) thermal_xi(a, i, g[0], g[1], g[2]);
   external_field_g<R>(a, i, m, g, -1, E);
}

// the same with the atom's Gaussians g (used when a.thermal) given, and its
// macrocell id (cell_id >= 0) when the caller has it already
template <typename R>
__device__ __forceinline__ void external_field_g(const LLGArgs<R>& a, int i, const MatParams<R>& m, const R g[3],
                                                 int cell_id, R E[3]) {
   R ex = 0, ey = 0, ez = 0;
   if (a.thermal) { ex = g[0] * m.sigma; ey = g[1] * m.sigma; ez = g[2] * m.sigma; }
   if (a.ramp_n) {
      const R f = (R)(a.step < a.ramp_n ? a.step : a.ramp_n) / (R)a.ramp_n;
      ex += a.hx + (m.hlx + m.dhx * f); ey += a.hy + (m.hly + m.dhy * f); ez += a.hz + (m.hlz + m.dhz * f);
   } else if (a.local_field) { ex += a.hx + m.hlx; ey += a.hy + m.hly; ez += a.hz + m.hlz; }
   else { ex += a.hx; ey += a.hy; ez += a.hz; }
   if (a.cell) {
      const int c = cell_id >= 0 ? cell_id : __ldg(a.cell + i);
      ex += __ldg(a.cell_field + c);
      ey += __ldg(a.cell_field + a.ncells + c);
      ez += __ldg(a.cell_field + 2 * a.ncells + c);
   } else if (a.hd_atom) {
      ex += __ldg(a.hd_atom + i); ey += __ldg(a.hd_atom + a.n + i); ez += __ldg(a.hd_atom + 2 * a.n + i);
   }
   E[0] = ex; E[1] = ey; E[2] = ez;
}

// LLG right-hand side exactly as LLGHeun.cpp:201-203
template <typename R>
__device__ __forceinline__ void llg_rhs(R A, R B, const R S[3], const R H[3], R d[3]) {
   d[0] = A * (S[1] * H[2] - S[2] * H[1]) + B * (S[1] * (S[0] * H[1] - S[1] * H[0]) - S[2] * (S[2] * H[0] - S[0] * H[2]));
   d[1] = A * (S[2] * H[0] - S[0] * H[2]) + B * (S[2] * (S[1] * H[2] - S[2] * H[1]) - S[0] * (S[0] * H[1] - S[1] * H[0]));
   d[2] = A * (S[0] * H[1] - S[1] * H[0]) + B * (S[0] * (S[2] * H[0] - S[0] * H[2]) - S[1] * (S[1] * H[2] - S[2] * H[1]));
}

}  // namespace vgpu
