// Fused stochastic LLG-Heun passes (sm_100a).
//
// The reference step (src/simulate/LLGHeun.cpp:160-282) makes two full field
// evaluations and four streaming loops over 12 SoA arrays per step; its CUDA
// backend (src/cuda/llg_heun.cu:121-208) makes 11 launches and 3 copies.
// Here a step is two launches, each one HBM pass:
//
//   predictor  s'  = n(s0 + dt * f(s0, H(s0) + H_ext))          reads s0, writes s'
//   corrector  s1  = n(s0 + dt/2 (f(s0,..) + f(s', H(s') + H_ext)))
//                                                 reads s0 and s', writes s1 over s0
//
// H(s) is the exchange gather over a sliced-ELL (SELL-32) copy of the CSR
// list (a warp = 32 consecutive atoms; bond k of lane l sits at
// slice_off + 32 k + l, so every index/coupling load of a warp is one 128-byte
// line) plus uniaxial and cubic anisotropy; H_ext is thermal noise
// regenerated in-register from Philox (no noise buffer), applied field and the
// macrocell dipole field looked up by cell id.  The predictor's
// f(s0, ...) dt is not stored: since f is perpendicular to s0 and
// s' = (s0 + f dt)/|s0 + f dt|, the corrector recovers
// f dt = s' |s0|^2 / (s'.s0) - s0 exactly from the two states it reads anyway.
#pragma once
#include <cuda_runtime.h>

#include "llg_device.cuh"

namespace vgpu {

// Predictor tail of atom i, given s0 and its total field H:
// s' = n(s0 + dt f(s0, H)) (LLGHeun.cpp:195-222).
template <typename R>
__device__ __forceinline__ void llg_predict_finish(const LLGArgs<R>& a, int i, const MatParams<R>& m, const R S0[3],
                                                   const R H[3]) {
   R d[3];
   llg_rhs<R>(m.A, m.B, S0, H, d);
   if (a.ex) { a.ex[i] = d[0]; a.ey[i] = d[1]; a.ez[i] = d[2]; }
   R Sn[3] = {S0[0] + d[0] * a.dt, S0[1] + d[1] * a.dt, S0[2] + d[2] * a.dt};
   const R r = rsqrt_<R>(Sn[0] * Sn[0] + Sn[1] * Sn[1] + Sn[2] * Sn[2]);
   a.bx[i] = Sn[0] * r; a.by[i] = Sn[1] * r; a.bz[i] = Sn[2] * r;
}

// Corrector tail of atom i, given s0, s' and the total field H' of s':
// s1 = n(s0 + dt/2 (f0 + f(s', H'))) (LLGHeun.cpp:238-279), written over s0.
template <typename R>
__device__ __forceinline__ void llg_correct_finish(const LLGArgs<R>& a, int i, const MatParams<R>& m, const R S0[3],
                                                   const R S1[3], const R H[3]) {
   R d[3];
   llg_rhs<R>(m.A, m.B, S1, H, d);
   R Sn[3];
   if (a.ex) {
      // stored predictor increment: s0 + dt/2 (f0 + f1) as LLGHeun.cpp:264-266
      const R e0[3] = {a.ex[i], a.ey[i], a.ez[i]};
#pragma unroll
      for (int k = 0; k < 3; ++k) Sn[k] = S0[k] + a.half_dt * (e0[k] + d[k]);
   } else {
      // recover the predictor increment f(s0) dt from s0 and s'
      const R s00 = S0[0] * S0[0] + S0[1] * S0[1] + S0[2] * S0[2];
      const R c = s00 / (S1[0] * S0[0] + S1[1] * S0[1] + S1[2] * S0[2]);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
         const R e = S1[k] * c - S0[k];
         Sn[k] = S0[k] + ((R)0.5 * e + a.half_dt * d[k]);
      }
   }
   const R n2 = Sn[0] * Sn[0] + Sn[1] * Sn[1] + Sn[2] * Sn[2];
   const R r = rsqrt_<R>(n2);
   if (!(n2 > (R)0.25 && n2 < (R)4)) atomicOr(a.status, 1);  // non-finite or runaway
   a.ax[i] = Sn[0] * r; a.ay[i] = Sn[1] * r; a.az[i] = Sn[2] * r;
}

// Cayley-transform rotation of sim::LLG_Midpoint (src/simulate/LLGMidpoint.cpp:
// 70-105, 117-150): F = H + alpha M x H, b2 = beta^2,
// out = (S (1 - b2 F.F) + 2 (beta F x S + F b2 F.S)) / (1 + b2 F.F).
template <typename R>
__device__ __forceinline__ void midpoint_rotate(R alpha, R beta, const R M[3], const R S[3], const R H[3],
                                                R out[3]) {
   const R beta2 = beta * beta;
   const R F[3] = {H[0] + alpha * (M[1] * H[2] - M[2] * H[1]), H[1] + alpha * (M[2] * H[0] - M[0] * H[2]),
                   H[2] + alpha * (M[0] * H[1] - M[1] * H[0])};
   const R FdotF = F[0] * F[0] + F[1] * F[1] + F[2] * F[2];
   const R beta2FdotS = beta2 * (F[0] * S[0] + F[1] * S[1] + F[2] * S[2]);
   const R c1 = (R)1 / ((R)1 + beta2 * FdotF);
   const R c2 = (R)1 - beta2 * FdotF;
   out[0] = c1 * (S[0] * c2 + (R)2 * (beta * (F[1] * S[2] - F[2] * S[1]) + F[0] * beta2FdotS));
   out[1] = c1 * (S[1] * c2 + (R)2 * (beta * (F[2] * S[0] - F[0] * S[2]) + F[1] * beta2FdotS));
   out[2] = c1 * (S[2] * c2 + (R)2 * (beta * (F[0] * S[1] - F[1] * S[0]) + F[2] * beta2FdotS));
}

// midpoint first half: M = (S0 + R(S0; F(S0, H))) / 2, not renormalised
template <typename R>
__device__ __forceinline__ void mid_predict_finish(const LLGArgs<R>& a, int i, const MatParams<R>& m, const R S0[3],
                                                   const R H[3]) {
   R r[3];
   midpoint_rotate<R>(m.alpha, m.beta_mid, S0, S0, H, r);
   a.bx[i] = (S0[0] + r[0]) * (R)0.5;
   a.by[i] = (S0[1] + r[1]) * (R)0.5;
   a.bz[i] = (S0[2] + r[2]) * (R)0.5;
}

// midpoint second half: S1 = R(S0; F(M, H(M))), written over S0
template <typename R>
__device__ __forceinline__ void mid_correct_finish(const LLGArgs<R>& a, int i, const MatParams<R>& m, const R S0[3],
                                                   const R M[3], const R H[3]) {
   R r[3];
   midpoint_rotate<R>(m.alpha, m.beta_mid, M, S0, H, r);
   const R n2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
   if (!(n2 > (R)0.25 && n2 < (R)4)) atomicOr(a.status, 1);  // non-finite or runaway
   a.ax[i] = r[0]; a.ay[i] = r[1]; a.az[i] = r[2];
}

// Predictor of atom i: s' = n(s0 + dt f(s0, H)) (Heun) or the midpoint M.
// LOAD = 1 reads neighbour spins through L2 (they may have been written
// earlier in the same launch).
template <typename R, int FMT, int LOAD, int VAR = VAR_HEUN_EXT>
__device__ __forceinline__ void llg_predict_atom(const LLGArgs<R>& a, int i) {
   const int mi = a.mat ? __ldg(a.mat + i) : 0;
   const MatParams<R> m = a.mp[mi];
   const R S0[3] = {a.ax[i], a.ay[i], a.az[i]};
   R H[3], E[3];
   spin_field<R, FMT, LOAD, false, VAR != VAR_HEUN>(a, i, mi, m, a.ax, a.ay, a.az, S0, H);
   external_field<R>(a, i, m, true, E);
   H[0] += E[0]; H[1] += E[1]; H[2] += E[2];
   if (VAR == VAR_MIDPOINT) mid_predict_finish<R>(a, i, m, S0, H);
   else llg_predict_finish<R>(a, i, m, S0, H);
}

// Corrector of atom i: s1 = n(s0 + dt/2 (f0 + f(s', H'))) (Heun) or the
// midpoint's second half, written over s0.
template <typename R, int FMT, int LOAD, int VAR = VAR_HEUN_EXT>
__device__ __forceinline__ void llg_correct_atom(const LLGArgs<R>& a, int i) {
   const int mi = a.mat ? __ldg(a.mat + i) : 0;
   const MatParams<R> m = a.mp[mi];
   const R S0[3] = {a.ax[i], a.ay[i], a.az[i]};
   const R S1[3] = {a.bx[i], a.by[i], a.bz[i]};
   R H[3], E[3];
   spin_field<R, FMT, LOAD, false, VAR != VAR_HEUN>(a, i, mi, m, a.bx, a.by, a.bz, S1, H);
   external_field<R>(a, i, m, true, E);
   H[0] += E[0]; H[1] += E[1]; H[2] += E[2];
   if (VAR == VAR_MIDPOINT) mid_correct_finish<R>(a, i, m, S0, S1, H);
   else llg_correct_finish<R>(a, i, m, S0, S1, H);
}

template <typename R, int FMT, int MODE, int VAR>
__global__ void __launch_bounds__(256) llg_pass_kernel(const LLGArgs<R> a) {
   // launched with programmatic stream serialisation (launch_pdl): the
   // previous kernel of the stream has completed and its writes are visible
   asm volatile("griddepcontrol.wait;" ::: "memory");
   const int i = (MODE == PASS_FIELD ? 0 : 32 * a.slice_first) + blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= (MODE == PASS_FIELD ? a.n : a.n_upd)) return;
   if (MODE == PASS_PREDICTOR) {
      llg_predict_atom<R, FMT, 0, VAR>(a, i);
   } else if (MODE == PASS_CORRECTOR) {
      llg_correct_atom<R, FMT, 0, VAR>(a, i);
   } else {
      // field of s0: exchange, anisotropy, applied and dipole terms (no thermal term)
      const int mi = a.mat ? __ldg(a.mat + i) : 0;
      const MatParams<R> m = a.mp[mi];
      const R S0[3] = {a.ax[i], a.ay[i], a.az[i]};
      R H[3], E[3];
      spin_field<R, FMT, 0, false, VAR != VAR_HEUN>(a, i, mi, m, a.ax, a.ay, a.az, S0, H);
      external_field<R>(a, i, m, false, E);
      a.fx[i] = H[0] + E[0]; a.fy[i] = H[1] + E[1]; a.fz[i] = H[2] + E[2];
   }
}

template <typename R, int FMT, int VAR>
inline cudaError_t launch_mode(const LLGArgs<R>& a, int mode, int grid, int bs, cudaStream_t st) {
   const dim3 g(grid), b(bs);
   if (mode == PASS_PREDICTOR) return launch_pdl(llg_pass_kernel<R, FMT, PASS_PREDICTOR, VAR>, g, b, 0, st, a);
   if (mode == PASS_CORRECTOR) return launch_pdl(llg_pass_kernel<R, FMT, PASS_CORRECTOR, VAR>, g, b, 0, st, a);
   return launch_pdl(llg_pass_kernel<R, FMT, PASS_FIELD, VAR>, g, b, 0, st, a);
}

template <typename R, int FMT>
inline cudaError_t launch_fmt(const LLGArgs<R>& a, int mode, cudaStream_t st) {
   const int bs = 256;
   const int grid = ((mode == PASS_FIELD ? a.n : a.n_upd - 32 * a.slice_first) + bs - 1) / bs;
   if (grid <= 0) return cudaSuccess;
   if (a.integrator == INTEG_MIDPOINT && mode != PASS_FIELD) return launch_mode<R, FMT, VAR_MIDPOINT>(a, mode, grid, bs, st);
   if (a.aniso_ext || a.bq_off) return launch_mode<R, FMT, VAR_HEUN_EXT>(a, mode, grid, bs, st);
   return launch_mode<R, FMT, VAR_HEUN>(a, mode, grid, bs, st);
}

template <typename R>
cudaError_t launch_llg_pass(const LLGArgs<R>& a, int fmt, int mode, int nslices, cudaStream_t st) {
   (void)nslices;
   switch (fmt) {
      case FMT_ISO_TAB: return launch_fmt<R, FMT_ISO_TAB>(a, mode, st);
      case FMT_ISO_BOND: return launch_fmt<R, FMT_ISO_BOND>(a, mode, st);
      case FMT_VEC_TAB: return launch_fmt<R, FMT_VEC_TAB>(a, mode, st);
      case FMT_VEC_BOND: return launch_fmt<R, FMT_VEC_BOND>(a, mode, st);
      case FMT_DMI_TAB: return launch_fmt<R, FMT_DMI_TAB>(a, mode, st);
      default: return launch_fmt<R, FMT_TENSOR_BOND>(a, mode, st);
   }
}

template <typename R>
__global__ void thermal_noise_kernel(const LLGArgs<R> a) {
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= a.n) return;
   R gx, gy, gz;
   thermal_xi(a, i, gx, gy, gz);
   a.fx[i] = gx; a.fy[i] = gy; a.fz[i] = gz;
}

template <typename R>
cudaError_t launch_thermal_noise(const LLGArgs<R>& a, cudaStream_t st) {
   thermal_noise_kernel<R><<<(a.n + 255) / 256, 256, 0, st>>>(a);
   return cudaGetLastError();
}
}  // namespace vgpu
