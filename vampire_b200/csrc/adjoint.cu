// Adjoint of the deterministic LLG-Heun trajectory (K8).
//
// No counterpart in the reference (which computes no derivatives).  For the
// loss L = sum_{t=1..N} w (m_z(t) - target_t)^2 (m_z: moment-weighted mean of
// s_z after step t) the reverse pass runs the step
//
//   s' = n(v),  v = s + dt f(s, H(s)),   s1 = n(u),  u = s + dt/2 (f(s,H(s)) + f(s',H(s')))
//   f(s,H) = A s x H + B s x (s x H),   H(s)_i = sum_j J_ij s_j + anisotropy(s_i) + H_app
//
// backwards with four fused per-atom kernels per step: (1) recompute H(s), f,
// s'; (2) recompute H(s'), f', s1 and push lambda through n(u), f' and H(s');
// (3) the transposed exchange gather of H(s')-bar, through n(v), f and H(s);
// (4) the transposed gather of H(s)-bar plus dL_t/ds_t gives lambda_t.
//
// Transposed gather.  The reference normalises every coupling by the moment of
// its own atom (J_ij [T] = J_SI,ij / mu_s,i, exchange/unroll_normalised.cpp),
// and its couplings are reciprocal in SI units (J_SI,ji = J_SI,ij^T: a
// symmetric exchange matrix; the three-site DMI vector changes sign with the
// bond).  So J_ji^T = (mu_s,i / mu_s,j) J_ij and the adjoint's
// sum_j J_ji^T Hbar_j = mu_s,i sum_j J_ij (Hbar_j / mu_s,j): the forward SELL
// gather of Hbar / mu_s, in every exchange format (isotropic, vectorial,
// diagonal + DMI, full tensor).  A device check before the run refuses
// couplings that are not reciprocal.
//
// Parameter gradients, block-reduced and accumulated in FP64: every coupling
// scaled together, Ku, H_app; and per pair of materials (a, b) the scale of
// the couplings of the bonds from atoms of a to atoms of b (the diagonal,
// exchange-matrix part for the diagonal + DMI format), plus the common scale
// of the DMI vectors.  States are checkpointed every ceil(sqrt(N)) steps and
// recomputed segment by segment with the forward passes.
//
// Precision: the state, the recomputed steps and the adjoint vectors are in
// the handle's precision (FP32 in production, FP64 in the debug build); the
// parameter gradients, m_z and the loss are FP64 sums.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <vector>

#include "llg_kernels.cuh"
#include "vgpu_ctx.cuh"

namespace vgpu {

template <typename R>
struct AdjBufs {
   R* S;                        // [3n] state s_t (segment slot)
   R *sp, *ex0, *ex1, *f0, *ub, *spb, *sb, *Hb0, *Hb1, *lam;   // [3n] each, x|y|z blocks
   R* nv;                       // [n] |v|
   double* g;                   // [5] dL/d(J scale), dL/dKu, dL/dH
   double* gp;                  // [1 + M*M] dL/d(DMI scale), dL/d(scale of the a->b couplings), or nullptr
   const double* mz;            // [N+1]
   const double* target;        // [N]
   double w, musum;
   int n, stride;               // stride = n_alloc (component offset)
};

template <typename R>
__device__ __forceinline__ void f_vjp(R A, R B, const R s[3], const R H[3], const R a[3], R sb[3], R Hb[3]) {
   const R sH = s[0] * H[0] + s[1] * H[1] + s[2] * H[2];
   const R as = a[0] * s[0] + a[1] * s[1] + a[2] * s[2];
   const R aH = a[0] * H[0] + a[1] * H[1] + a[2] * H[2];
   const R ss = s[0] * s[0] + s[1] * s[1] + s[2] * s[2];
   sb[0] = A * (H[1] * a[2] - H[2] * a[1]);
   sb[1] = A * (H[2] * a[0] - H[0] * a[2]);
   sb[2] = A * (H[0] * a[1] - H[1] * a[0]);
   Hb[0] = A * (a[1] * s[2] - a[2] * s[1]);
   Hb[1] = A * (a[2] * s[0] - a[0] * s[2]);
   Hb[2] = A * (a[0] * s[1] - a[1] * s[0]);
#pragma unroll
   for (int k = 0; k < 3; ++k) {
      sb[k] += B * (a[k] * sH + as * H[k] - (R)2 * aH * s[k]);
      Hb[k] += B * (as * s[k] - a[k] * ss);
   }
}

template <typename R>
__device__ __forceinline__ void aniso_h(const LLGArgs<R>& a, const MatParams<R>& m, const R S[3], R H[3]) {
   H[0] = H[1] = H[2] = (R)0;
   if (a.uniaxial) {
      const R k2 = (R)2 * m.ku2 * (S[0] * m.kux + S[1] * m.kuy + S[2] * m.kuz);
      H[0] += m.kux * k2; H[1] += m.kuy * k2; H[2] += m.kuz * k2;
   }
   if (a.cubic) {
      const R k4 = (R)2 * m.kc4;
      H[0] += S[0] * S[0] * S[0] * k4; H[1] += S[1] * S[1] * S[1] * k4; H[2] += S[2] * S[2] * S[2] * k4;
   }
}

// VJP of the anisotropy field with respect to s (added to sbar)
template <typename R>
__device__ __forceinline__ void aniso_vjp(const LLGArgs<R>& a, const MatParams<R>& m, const R S[3], const R hb[3],
                                          R sb[3]) {
   if (a.uniaxial) {
      const R he = hb[0] * m.kux + hb[1] * m.kuy + hb[2] * m.kuz;
      sb[0] += (R)2 * m.ku2 * he * m.kux; sb[1] += (R)2 * m.ku2 * he * m.kuy; sb[2] += (R)2 * m.ku2 * he * m.kuz;
   }
   if (a.cubic) {
      for (int k = 0; k < 3; ++k) sb[k] += (R)6 * m.kc4 * S[k] * S[k] * hb[k];
   }
}

// block-reduce 5 gradient partials and add them to g
__device__ __forceinline__ void grad_add(double v[5], double* g) {
#pragma unroll
   for (int q = 0; q < 5; ++q)
      for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
   __shared__ double red[5][8];
   const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
   if (l == 0)
      for (int q = 0; q < 5; ++q) red[q][w] = v[q];
   __syncthreads();
   if (threadIdx.x < 5) {
      double s = 0.0;
      for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += red[threadIdx.x][k];
      atomicAdd(g + threadIdx.x, s);
   }
}

// coupling of SELL entry e (row atom material mi, neighbour material mj) as
// a 3x3 matrix, row-major, in the generic (non-compact) formats
template <typename R, int FMT>
__device__ __forceinline__ void bond_tensor(const LLGArgs<R>& a, int e, int mi, int mj, R T[9]) {
#pragma unroll
   for (int k = 0; k < 9; ++k) T[k] = (R)0;
   if (FMT == FMT_ISO_TAB) {
      T[0] = T[4] = T[8] = a.jtab[mi * a.M + mj];
   } else if (FMT == FMT_ISO_BOND) {
      T[0] = T[4] = T[8] = a.jb[0][e];
   } else if (FMT == FMT_VEC_TAB || FMT == FMT_DMI_TAB) {
      const R* t = a.jtab + 3 * (mi * a.M + mj);
      T[0] = t[0]; T[4] = t[1]; T[8] = t[2];
      if (FMT == FMT_DMI_TAB) {  // d x s: [[0, -dz, dy], [dz, 0, -dx], [-dy, dx, 0]]
         const R dx = a.jb[0][e], dy = a.jb[1][e], dz = a.jb[2][e];
         T[1] = -dz; T[2] = dy; T[3] = dz; T[5] = -dx; T[6] = -dy; T[7] = dx;
      }
   } else if (FMT == FMT_VEC_BOND) {
      T[0] = a.jb[0][e]; T[4] = a.jb[1][e]; T[8] = a.jb[2][e];
   } else {
#pragma unroll
      for (int k = 0; k < 9; ++k) T[k] = a.jb[k][e];
   }
}

template <typename R>
__device__ __forceinline__ int nb_material(const LLGArgs<R>& a, int c, int j) {
   return a.mat_shift ? (c >> a.mat_shift) : (a.mat ? a.mat[j] : 0);
}

// Parameter gradients of one atom's exchange field: hb . (J_ij s_j) summed
// per material pair (diagonal part for the DMI format) into sp[1 + mi*M + mj]
// and hb . (d_ij x s_j) into sp[0] (shared memory, this block's sums)
template <typename R, int FMT>
__device__ __forceinline__ void pair_grads(const LLGArgs<R>& a, int i, int mi, const R* sx, const R* sy, const R* sz,
                                           const R hb[3], double* sp) {
   const int sl = i >> 5, lane = i & 31;
   const int off = a.slice_off[sl];
   const int w = (a.slice_off[sl + 1] - off) >> 5;
   double dm = 0.0;
   for (int k = 0; k < w; ++k) {
      const int e = off + lane + 32 * k;
      const int c = a.col[e];
      const int j = c & a.idx_mask;
      if (j >= a.n) continue;  // padding entry
      const int mj = nb_material(a, c, j);
      const R s[3] = {sx[j], sy[j], sz[j]};
      R T[9];
      bond_tensor<R, FMT>(a, e, mi, mj, T);
      const double diag = (double)(hb[0] * T[0] * s[0] + hb[1] * T[4] * s[1] + hb[2] * T[8] * s[2]);
      const double off_d = (double)(hb[0] * (T[1] * s[1] + T[2] * s[2]) + hb[1] * (T[3] * s[0] + T[5] * s[2]) +
                                    hb[2] * (T[6] * s[0] + T[7] * s[1]));
      if (FMT == FMT_DMI_TAB) {
         atomicAdd(sp + 1 + mi * a.M + mj, diag);
         dm += off_d;
      } else {
         atomicAdd(sp + 1 + mi * a.M + mj, diag + off_d);
      }
   }
   if (FMT == FMT_DMI_TAB) atomicAdd(sp, dm);
}

// Reciprocity of the couplings in SI units: for every bond i -> j, the sum of
// mu_s,i J_ij over the bonds of row i to j equals the transpose of the sum of
// mu_s,j J_ji over the bonds of row j to i (to 1e-10 of its largest entry in
// FP64, 1e-5 for couplings held in FP32).  Sets *bad = 1 + i at a failing atom.
template <typename R, int FMT>
__global__ void adj_reciprocal_kernel(const LLGArgs<R> a, int* bad) {
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= a.n) return;
   const int mi = a.mat ? a.mat[i] : 0;
   const double mui = a.mp[mi].mu_s_muB;
   const int off = a.slice_off[i >> 5], w = (a.slice_off[(i >> 5) + 1] - off) >> 5;
   for (int k = 0; k < w; ++k) {
      const int c = a.col[off + (i & 31) + 32 * k];
      const int j = c & a.idx_mask;
      if (j >= a.n) continue;
      const int mj = a.mat ? a.mat[j] : 0;
      const double muj = a.mp[mj].mu_s_muB;
      double Sij[9] = {0}, Sji[9] = {0};
      R T[9];
      for (int q = 0; q < w; ++q) {
         const int e = off + (i & 31) + 32 * q;
         const int cq = a.col[e];
         if ((cq & a.idx_mask) != j) continue;
         bond_tensor<R, FMT>(a, e, mi, nb_material(a, cq, j), T);
         for (int r = 0; r < 9; ++r) Sij[r] += mui * (double)T[r];
      }
      const int offj = a.slice_off[j >> 5], wj = (a.slice_off[(j >> 5) + 1] - offj) >> 5;
      for (int q = 0; q < wj; ++q) {
         const int e = offj + (j & 31) + 32 * q;
         const int cq = a.col[e];
         if ((cq & a.idx_mask) != i) continue;
         bond_tensor<R, FMT>(a, e, mj, nb_material(a, cq, i), T);
         for (int r = 0; r < 9; ++r) Sji[r] += muj * (double)T[r];
      }
      double mx = 0.0, dv = 0.0;
      for (int r = 0; r < 3; ++r)
         for (int s = 0; s < 3; ++s) {
            mx = fmax(mx, fabs(Sij[3 * r + s]));
            dv = fmax(dv, fabs(Sij[3 * r + s] - Sji[3 * s + r]));
         }
      if (dv > (sizeof(R) == 4 ? 1e-5 : 1e-10) * mx) {
         atomicCAS(bad, 0, 1 + i);
         return;
      }
   }
}

template <typename R, int FMT>
__global__ void __launch_bounds__(256) adj_k1(const LLGArgs<R> a, AdjBufs<R> b) {
   asm volatile("griddepcontrol.wait;" ::: "memory");  // launched by launch_pdl
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= b.n) return;
   const int st = b.stride;
   const int mi = a.mat ? a.mat[i] : 0;
   const MatParams<R> m = a.mp[mi];
   const R S[3] = {b.S[i], b.S[st + i], b.S[2 * st + i]};
   R ex[3] = {0, 0, 0}, Ha[3];
   exchange_gather<R, FMT>(a, i, mi, b.S, b.S + st, b.S + 2 * st, ex[0], ex[1], ex[2]);
   aniso_h(a, m, S, Ha);
   const R H[3] = {ex[0] + Ha[0] + a.hx, ex[1] + Ha[1] + a.hy, ex[2] + Ha[2] + a.hz};
   R d[3];
   llg_rhs<R>(m.A, m.B, S, H, d);
   R v[3];
   for (int k = 0; k < 3; ++k) {
      b.ex0[k * st + i] = ex[k];
      b.f0[k * st + i] = d[k];
      v[k] = S[k] + d[k] * a.dt;
   }
   const R L = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
   b.nv[i] = L;
   for (int k = 0; k < 3; ++k) b.sp[k * st + i] = v[k] / L;
}

// shared sums of the pair gradients: [1 + M*M] (M <= kAdjMaxPairMat)
constexpr int kAdjMaxPairMat = 8;

template <typename R>
__device__ __forceinline__ void pair_init(double* sp, const AdjBufs<R>& b, int M) {
   if (b.gp)
      for (int k = threadIdx.x; k < 1 + M * M; k += blockDim.x) sp[k] = 0.0;
   __syncthreads();
}

template <typename R>
__device__ __forceinline__ void pair_flush(const double* sp, const AdjBufs<R>& b, int M) {
   if (!b.gp) return;
   __syncthreads();
   for (int k = threadIdx.x; k < 1 + M * M; k += blockDim.x)
      if (sp[k] != 0.0) atomicAdd(b.gp + k, sp[k]);
}

// dL/dKu of one atom from its field adjoint hb at spin s (uniaxial term)
template <typename R>
__device__ __forceinline__ double ku_grad(const MatParams<R>& m, const R hb[3], const R s[3]) {
   const double he = (double)(hb[0] * m.kux + hb[1] * m.kuy + hb[2] * m.kuz);
   const double se = (double)(s[0] * m.kux + s[1] * m.kuy + s[2] * m.kuz);
   return 2.0 * he * se / ((double)m.mu_s_muB * 9.27400915e-24);
}

template <typename R, int FMT>
__global__ void __launch_bounds__(256) adj_k2(const LLGArgs<R> a, AdjBufs<R> b) {
   asm volatile("griddepcontrol.wait;" ::: "memory");  // launched by launch_pdl
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   const int st = b.stride;
   double gv[5] = {0, 0, 0, 0, 0};
   __shared__ double sp[1 + kAdjMaxPairMat * kAdjMaxPairMat];
   pair_init(sp, b, a.M);
   if (i < b.n) {
      const int mi = a.mat ? a.mat[i] : 0;
      const MatParams<R> m = a.mp[mi];
      const R S[3] = {b.S[i], b.S[st + i], b.S[2 * st + i]};
      const R Sp[3] = {b.sp[i], b.sp[st + i], b.sp[2 * st + i]};
      R ex[3] = {0, 0, 0}, Ha[3];
      exchange_gather<R, FMT>(a, i, mi, b.sp, b.sp + st, b.sp + 2 * st, ex[0], ex[1], ex[2]);
      aniso_h(a, m, Sp, Ha);
      const R H1[3] = {ex[0] + Ha[0] + a.hx, ex[1] + Ha[1] + a.hy, ex[2] + Ha[2] + a.hz};
      R f1[3], u[3];
      llg_rhs<R>(m.A, m.B, Sp, H1, f1);
      for (int k = 0; k < 3; ++k) u[k] = S[k] + (R)0.5 * a.dt * (b.f0[k * st + i] + f1[k]);
      const R L = sqrt(u[0] * u[0] + u[1] * u[1] + u[2] * u[2]);
      const R s1[3] = {u[0] / L, u[1] / L, u[2] / L};
      const R l[3] = {b.lam[i], b.lam[st + i], b.lam[2 * st + i]};
      const R ls = l[0] * s1[0] + l[1] * s1[1] + l[2] * s1[2];
      R u_b[3], a1[3], sdir[3], hb[3];
      for (int k = 0; k < 3; ++k) { u_b[k] = (l[k] - ls * s1[k]) / L; a1[k] = (R)0.5 * a.dt * u_b[k]; }
      f_vjp(m.A, m.B, Sp, H1, a1, sdir, hb);
      const R imu = (R)1 / m.mu_s_muB;  // Hbar / mu_s for the transposed gather
      for (int k = 0; k < 3; ++k) {
         b.ub[k * st + i] = u_b[k];
         b.spb[k * st + i] = sdir[k];
         b.Hb1[k * st + i] = hb[k] * imu;
         b.ex1[k * st + i] = ex[k];
         gv[0] += (double)hb[k] * (double)ex[k];
         gv[2 + k] += (double)hb[k];
      }
      if (b.gp) pair_grads<R, FMT>(a, i, mi, b.sp, b.sp + st, b.sp + 2 * st, hb, sp);
      if (a.uniaxial) gv[1] += ku_grad(m, hb, Sp);
   }
   pair_flush(sp, b, a.M);
   grad_add(gv, b.g);
}

template <typename R, int FMT>
__global__ void __launch_bounds__(256) adj_k3(const LLGArgs<R> a, AdjBufs<R> b) {
   asm volatile("griddepcontrol.wait;" ::: "memory");  // launched by launch_pdl
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   const int st = b.stride;
   double gv[5] = {0, 0, 0, 0, 0};
   __shared__ double sp[1 + kAdjMaxPairMat * kAdjMaxPairMat];
   pair_init(sp, b, a.M);
   if (i < b.n) {
      const int mi = a.mat ? a.mat[i] : 0;
      const MatParams<R> m = a.mp[mi];
      const R mu = m.mu_s_muB;
      const R S[3] = {b.S[i], b.S[st + i], b.S[2 * st + i]};
      const R Sp[3] = {b.sp[i], b.sp[st + i], b.sp[2 * st + i]};
      R t[3] = {0, 0, 0};
      exchange_gather<R, FMT>(a, i, mi, b.Hb1, b.Hb1 + st, b.Hb1 + 2 * st, t[0], t[1], t[2]);
      const R hb1[3] = {b.Hb1[i] * mu, b.Hb1[st + i] * mu, b.Hb1[2 * st + i] * mu};
      R spbar[3];
      for (int k = 0; k < 3; ++k) spbar[k] = b.spb[k * st + i] + t[k] * mu;
      aniso_vjp(a, m, Sp, hb1, spbar);
      const R sps = spbar[0] * Sp[0] + spbar[1] * Sp[1] + spbar[2] * Sp[2];
      R vb[3], a0[3];
      for (int k = 0; k < 3; ++k) {
         vb[k] = (spbar[k] - sps * Sp[k]) / b.nv[i];
         a0[k] = (R)0.5 * a.dt * b.ub[k * st + i] + a.dt * vb[k];
      }
      R Ha[3];
      aniso_h(a, m, S, Ha);
      R H0[3], ex[3];
      for (int k = 0; k < 3; ++k) {
         ex[k] = b.ex0[k * st + i];
         H0[k] = ex[k] + Ha[k] + (k == 0 ? a.hx : k == 1 ? a.hy : a.hz);
      }
      R sdir[3], hb[3];
      f_vjp(m.A, m.B, S, H0, a0, sdir, hb);
      for (int k = 0; k < 3; ++k) {
         b.sb[k * st + i] = b.ub[k * st + i] + vb[k] + sdir[k];
         b.Hb0[k * st + i] = hb[k] / mu;
         gv[0] += (double)hb[k] * (double)ex[k];
         gv[2 + k] += (double)hb[k];
      }
      if (b.gp) pair_grads<R, FMT>(a, i, mi, b.S, b.S + st, b.S + 2 * st, hb, sp);
      if (a.uniaxial) gv[1] += ku_grad(m, hb, S);
   }
   pair_flush(sp, b, a.M);
   grad_add(gv, b.g);
}

template <typename R, int FMT>
__global__ void __launch_bounds__(256) adj_k4(const LLGArgs<R> a, AdjBufs<R> b, int64_t t) {
   asm volatile("griddepcontrol.wait;" ::: "memory");  // launched by launch_pdl
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= b.n) return;
   const int st = b.stride;
   const int mi = a.mat ? a.mat[i] : 0;
   const MatParams<R> m = a.mp[mi];
   const R S[3] = {b.S[i], b.S[st + i], b.S[2 * st + i]};
   const R mu = m.mu_s_muB;
   R tg[3] = {0, 0, 0};
   exchange_gather<R, FMT>(a, i, mi, b.Hb0, b.Hb0 + st, b.Hb0 + 2 * st, tg[0], tg[1], tg[2]);
   const R hb0[3] = {b.Hb0[i] * mu, b.Hb0[st + i] * mu, b.Hb0[2 * st + i] * mu};
   R l[3];
   for (int k = 0; k < 3; ++k) l[k] = b.sb[k * st + i] + tg[k] * mu;
   aniso_vjp(a, m, S, hb0, l);
   if (t >= 1) l[2] += (R)(2.0 * b.w * (b.mz[t] - b.target[t - 1]) * (double)m.mu_s_muB / b.musum);
   for (int k = 0; k < 3; ++k) b.lam[k * st + i] = l[k];
}

template <typename R>
__global__ void adj_lambda_init(const LLGArgs<R> a, AdjBufs<R> b, int64_t N) {
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i >= b.n) return;
   const int mi = a.mat ? a.mat[i] : 0;
   const int st = b.stride;
   b.lam[i] = (R)0;
   b.lam[st + i] = (R)0;
   b.lam[2 * st + i] = (R)(2.0 * b.w * (b.mz[N] - b.target[N - 1]) * (double)a.mp[mi].mu_s_muB / b.musum);
}

// m_z after a step: block sums of mu s_z added into out[0]
template <typename R>
__global__ void mz_kernel(int n, const R* __restrict__ sz, const int* __restrict__ mat,
                          const MatParams<R>* __restrict__ mp, double* out) {
   asm volatile("griddepcontrol.wait;" ::: "memory");  // launched by launch_pdl
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   double v = 0.0;
   if (i < n) v = (double)sz[i] * (double)mp[mat ? mat[i] : 0].mu_s_muB;
   for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
   __shared__ double red[8];
   if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
   __syncthreads();
   if (threadIdx.x == 0) {
      double s = 0.0;
      for (int k = 0; k < (int)(blockDim.x >> 5); ++k) s += red[k];
      atomicAdd(out, s);
   }
}

template <typename R, int FMT>
static void adj_step(const LLGArgs<R>& a, const AdjBufs<R>& b, int64_t t, cudaStream_t st) {
   const int g = (b.n + 255) / 256;
   // consecutive small launches: programmatic serialisation hides their gaps
   launch_pdl(adj_k1<R, FMT>, dim3(g), dim3(256), 0, st, a, b);
   launch_pdl(adj_k2<R, FMT>, dim3(g), dim3(256), 0, st, a, b);
   launch_pdl(adj_k3<R, FMT>, dim3(g), dim3(256), 0, st, a, b);
   launch_pdl(adj_k4<R, FMT>, dim3(g), dim3(256), 0, st, a, b, t);
}

template <typename R>
static void adj_step_fmt(int fmt, const LLGArgs<R>& a, const AdjBufs<R>& b, int64_t t, cudaStream_t st) {
   switch (fmt) {
      case FMT_ISO_TAB: adj_step<R, FMT_ISO_TAB>(a, b, t, st); break;
      case FMT_ISO_BOND: adj_step<R, FMT_ISO_BOND>(a, b, t, st); break;
      case FMT_VEC_TAB: adj_step<R, FMT_VEC_TAB>(a, b, t, st); break;
      case FMT_VEC_BOND: adj_step<R, FMT_VEC_BOND>(a, b, t, st); break;
      case FMT_DMI_TAB: adj_step<R, FMT_DMI_TAB>(a, b, t, st); break;
      default: adj_step<R, FMT_TENSOR_BOND>(a, b, t, st); break;
   }
}

template <typename R>
static cudaError_t launch_reciprocal(int fmt, const LLGArgs<R>& a, int* bad, cudaStream_t st) {
   const int g = (a.n + 127) / 128;
   switch (fmt) {
      case FMT_ISO_TAB: adj_reciprocal_kernel<R, FMT_ISO_TAB><<<g, 128, 0, st>>>(a, bad); break;
      case FMT_ISO_BOND: adj_reciprocal_kernel<R, FMT_ISO_BOND><<<g, 128, 0, st>>>(a, bad); break;
      case FMT_VEC_TAB: adj_reciprocal_kernel<R, FMT_VEC_TAB><<<g, 128, 0, st>>>(a, bad); break;
      case FMT_VEC_BOND: adj_reciprocal_kernel<R, FMT_VEC_BOND><<<g, 128, 0, st>>>(a, bad); break;
      case FMT_DMI_TAB: adj_reciprocal_kernel<R, FMT_DMI_TAB><<<g, 128, 0, st>>>(a, bad); break;
      default: adj_reciprocal_kernel<R, FMT_TENSOR_BOND><<<g, 128, 0, st>>>(a, bad); break;
   }
   return cudaGetLastError();
}

}  // namespace vgpu

using namespace vgpu;

namespace {

template <typename T>
struct DevVec {
   T* p = nullptr;
   ~DevVec() { if (p) cudaFree(p); }
   cudaError_t alloc(size_t n) { return cudaMalloc(&p, sizeof(T) * std::max<size_t>(n, 1)); }
};

// one Heun step (the ordinary passes, no thermal term) of the state in `x`
// (3 * stride values, x|y|z), the predictor increment stored
template <typename R>
int forward_step(vgpu_ctx* h, LLGArgs<R> a, R* x, R* pb, R* eb, int stride) {
   a.ax = x; a.ay = x + stride; a.az = x + 2 * stride;
   a.bx = pb; a.by = pb + stride; a.bz = pb + 2 * stride;
   a.ex = eb; a.ey = eb + stride; a.ez = eb + 2 * stride;
   a.thermal = 0;
   cudaError_t e = launch_llg_pass<R>(a, h->sys.fmt, PASS_PREDICTOR, h->sys.nslices, h->stream);
   if (e == cudaSuccess) e = launch_llg_pass<R>(a, h->sys.fmt, PASS_CORRECTOR, h->sys.nslices, h->stream);
   h->kernel_launches += 2;
   return cuda_err(h, e, "adjoint forward");
}

int check_adjoint_ok(vgpu_ctx* h) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   if (h->sys.cell || h->sys.hd_atom || h->sys.sys_off)
      return set_err(h, VGPU_ERR_ARG, "the adjoint does not support dipole fields or batches");
   if (h->params.local_applied_field) return set_err(h, VGPU_ERR_ARG, "the adjoint supports the global applied field only");
   if (h->sys.bq_off) return set_err(h, VGPU_ERR_ARG, "the adjoint does not support biquadratic exchange");
   if (h->sys.aniso_ext) return set_err(h, VGPU_ERR_ARG, "the adjoint supports second-order uniaxial and cubic anisotropy only");
   if (h->sys.n_owned < h->sys.n) return set_err(h, VGPU_ERR_STATE, "the adjoint runs on whole systems (handle holds a shard)");
   return VGPU_OK;
}

double moment_sum(vgpu_ctx* h) {
   double s = 0.0;
   for (int t : h->sys.type_host) s += h->sys.materials[t].mu_s_SI / 9.27400915e-24;
   return s;
}

template <typename R>
int mz_trajectory_typed(vgpu_handle h, uint64_t n_steps, double* mz_out) {
   SysDev& S = h->sys;
   const int st = S.n_alloc;
   DevVec<R> cur, pb, eb;
   DevVec<double> mz;
   cudaError_t e;
   if ((e = cur.alloc(3 * (size_t)st)) || (e = pb.alloc(3 * (size_t)st)) || (e = eb.alloc(3 * (size_t)st)) ||
       (e = mz.alloc(n_steps + 1)))
      return cuda_err(h, e, "trajectory buffers");
   for (int q = 0; q < 3; ++q)
      cudaMemcpyAsync(cur.p + (size_t)q * st, S.s[q], sizeof(R) * st, cudaMemcpyDeviceToDevice, h->stream);
   cudaMemsetAsync(mz.p, 0, sizeof(double) * (n_steps + 1), h->stream);
   LLGArgs<R> a = make_args<R>(h);
   for (uint64_t t = 0; t < n_steps; ++t) {
      if (int rc = forward_step<R>(h, a, cur.p, pb.p, eb.p, st)) return rc;
      launch_pdl(mz_kernel<R>, dim3((S.n + 255) / 256), dim3(256), 0, h->stream, (int)S.n,
                 (const R*)(cur.p + 2 * (size_t)st), (const int*)S.mat, (const MatParams<R>*)S.mp,
                 (double*)(mz.p + t + 1));
   }
   std::vector<double> host(n_steps + 1);
   e = cudaMemcpyAsync(host.data(), mz.p, sizeof(double) * (n_steps + 1), cudaMemcpyDeviceToHost, h->stream);
   if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
   if (e != cudaSuccess) return cuda_err(h, e, "trajectory");
   const double ms = moment_sum(h);
   for (uint64_t t = 0; t < n_steps; ++t) mz_out[t] = host[t + 1] / ms;
   return VGPU_OK;
}

// the couplings must be reciprocal in SI units for the transposed gather
template <typename R>
int check_reciprocal(vgpu_ctx* h) {
   int* bad = nullptr;
   cudaError_t e = cudaMalloc(&bad, sizeof(int));
   if (e != cudaSuccess) return cuda_err(h, e, "adjoint check");
   int hb = 0;
   e = cudaMemsetAsync(bad, 0, sizeof(int), h->stream);
   if (e == cudaSuccess) e = launch_reciprocal<R>(h->sys.fmt, make_args<R>(h), bad, h->stream);
   if (e == cudaSuccess) e = cudaMemcpyAsync(&hb, bad, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
   if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
   cudaFree(bad);
   if (e != cudaSuccess) return cuda_err(h, e, "adjoint check");
   h->kernel_launches++;
   if (hb)
      return set_err(h, VGPU_ERR_ARG,
                     "the adjoint needs reciprocal couplings (mu_s,j J_ji = (mu_s,i J_ij)^T); atom %d breaks it", hb - 1);
   return VGPU_OK;
}

template <typename R>
int adjoint_typed(vgpu_handle h, uint64_t n_steps, const double* target, double w, int32_t every, double* loss_out,
                  double* grad_out, double* pair_out) {
   int rc;
   if ((rc = check_reciprocal<R>(h))) return rc;
   const int M = h->sys.M;
   SysDev& S = h->sys;
   const int n = S.n, st = S.n_alloc;
   const int64_t N = (int64_t)n_steps;
   const int64_t C = every > 0 ? every : (int64_t)std::ceil(std::sqrt((double)N));
   const int64_t ncp = (N + C - 1) / C;
   const size_t v3 = 3 * (size_t)st;
   const int np = 1 + M * M;
   DevVec<R> cp, seg, pb, eb, work;
   DevVec<double> mz, tg, g;
   cudaError_t e;
   if ((e = cp.alloc(v3 * ncp)) || (e = seg.alloc(v3 * (C + 1))) || (e = pb.alloc(v3)) || (e = eb.alloc(v3)) ||
       (e = mz.alloc(N + 1)) || (e = tg.alloc(N)) || (e = g.alloc(5 + np)) || (e = work.alloc(v3 * 10 + st)))
      return cuda_err(h, e, "adjoint buffers");
   cudaMemcpyAsync(tg.p, target, sizeof(double) * N, cudaMemcpyHostToDevice, h->stream);
   cudaMemsetAsync(mz.p, 0, sizeof(double) * (N + 1), h->stream);
   cudaMemsetAsync(g.p, 0, sizeof(double) * (5 + np), h->stream);
   LLGArgs<R> a = make_args<R>(h);
   a.thermal = 0;
   // forward from the current spins (left untouched), checkpoint every C steps
   R* cur = seg.p;  // first slot doubles as the running state
   for (int q = 0; q < 3; ++q)
      cudaMemcpyAsync(cur + (size_t)q * st, S.s[q], sizeof(R) * st, cudaMemcpyDeviceToDevice, h->stream);
   for (int64_t t = 0; t < N; ++t) {
      if (t % C == 0) cudaMemcpyAsync(cp.p + v3 * (t / C), cur, sizeof(R) * v3, cudaMemcpyDeviceToDevice, h->stream);
      if ((rc = forward_step<R>(h, a, cur, pb.p, eb.p, st))) return rc;
      launch_pdl(mz_kernel<R>, dim3((n + 255) / 256), dim3(256), 0, h->stream, (int)n,
                 (const R*)(cur + 2 * (size_t)st), (const int*)S.mat, (const MatParams<R>*)S.mp,
                 (double*)(mz.p + t + 1));
   }
   // loss on the host from m_z(t)
   std::vector<double> mzh(N + 1);
   e = cudaMemcpyAsync(mzh.data(), mz.p, sizeof(double) * (N + 1), cudaMemcpyDeviceToHost, h->stream);
   if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
   if (e != cudaSuccess) return cuda_err(h, e, "adjoint forward");
   const double musum = moment_sum(h);
   // m_z was summed unnormalised: scale the device copy once
   for (int64_t t = 0; t <= N; ++t) mzh[t] /= musum;
   cudaMemcpyAsync(mz.p, mzh.data(), sizeof(double) * (N + 1), cudaMemcpyHostToDevice, h->stream);
   double loss = 0.0;
   for (int64_t t = 1; t <= N; ++t) {
      const double r = mzh[t] - target[t - 1];
      loss += w * r * r;
   }
   AdjBufs<R> b;
   std::memset(&b, 0, sizeof b);
   R* wk = work.p;
   b.sp = wk; b.ex0 = wk + v3; b.ex1 = wk + 2 * v3; b.f0 = wk + 3 * v3; b.ub = wk + 4 * v3;
   b.spb = wk + 5 * v3; b.sb = wk + 6 * v3; b.Hb0 = wk + 7 * v3; b.Hb1 = wk + 8 * v3; b.lam = wk + 9 * v3;
   b.nv = wk + 10 * v3;
   b.g = g.p; b.mz = mz.p; b.target = tg.p; b.w = w; b.musum = musum; b.n = n; b.stride = st;
   b.gp = pair_out ? g.p + 5 : nullptr;
   adj_lambda_init<R><<<(n + 255) / 256, 256, 0, h->stream>>>(a, b, N);
   for (int64_t c = ncp - 1; c >= 0; --c) {
      const int64_t t0 = c * C, t1 = std::min(t0 + C, N);
      cudaMemcpyAsync(seg.p, cp.p + v3 * c, sizeof(R) * v3, cudaMemcpyDeviceToDevice, h->stream);
      for (int64_t t = t0; t < t1 - 1; ++t) {
         R* nxt = seg.p + v3 * (t - t0 + 1);
         cudaMemcpyAsync(nxt, seg.p + v3 * (t - t0), sizeof(R) * v3, cudaMemcpyDeviceToDevice, h->stream);
         if ((rc = forward_step<R>(h, a, nxt, pb.p, eb.p, st))) return rc;
      }
      for (int64_t t = t1 - 1; t >= t0; --t) {
         b.S = seg.p + v3 * (t - t0);
         adj_step_fmt<R>(S.fmt, a, b, t, h->stream);
         h->kernel_launches += 4;
      }
      if ((e = cudaGetLastError()) != cudaSuccess) return cuda_err(h, e, "adjoint backward");
   }
   std::vector<double> gh(5 + np);
   e = cudaMemcpyAsync(gh.data(), g.p, sizeof(double) * gh.size(), cudaMemcpyDeviceToHost, h->stream);
   if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
   if (e != cudaSuccess) return cuda_err(h, e, "adjoint result");
   *loss_out = loss;
   for (int k = 0; k < 5; ++k) grad_out[k] = gh[k];
   if (pair_out)
      for (int k = 0; k < np; ++k) pair_out[k] = gh[5 + k];
   return VGPU_OK;
}

}  // namespace

extern "C" int vgpu_mz_trajectory(vgpu_handle h, uint64_t n_steps, double* mz_out) {
   int rc = check_adjoint_ok(h);
   if (rc) return rc;
   cudaSetDevice(h->device);
   return h->prec == VGPU_PREC_FP64 ? mz_trajectory_typed<double>(h, n_steps, mz_out)
                                    : mz_trajectory_typed<float>(h, n_steps, mz_out);
}

static int adjoint_run(vgpu_handle h, uint64_t n_steps, const double* target, double w, int32_t every,
                       double* loss_out, double* grad_out, double* pair_out) {
   int rc = check_adjoint_ok(h);
   if (rc) return rc;
   if (!target || !loss_out || !grad_out || n_steps == 0) return set_err(h, VGPU_ERR_ARG, "bad adjoint arguments");
   cudaSetDevice(h->device);
   if (pair_out && h->sys.M > kAdjMaxPairMat)
      return set_err(h, VGPU_ERR_ARG, "per-material gradients support at most %d materials", kAdjMaxPairMat);
   return h->prec == VGPU_PREC_FP64
              ? adjoint_typed<double>(h, n_steps, target, w, every, loss_out, grad_out, pair_out)
              : adjoint_typed<float>(h, n_steps, target, w, every, loss_out, grad_out, pair_out);
}

extern "C" int vgpu_adjoint_llg(vgpu_handle h, uint64_t n_steps, const double* target, double w, int32_t every,
                                double* loss_out, double* grad_out) {
   return adjoint_run(h, n_steps, target, w, every, loss_out, grad_out, nullptr);
}

extern "C" int vgpu_adjoint_llg_materials(vgpu_handle h, uint64_t n_steps, const double* target, double w,
                                          int32_t every, double* loss_out, double* grad_out, double* pair_out) {
   if (!pair_out) return set_err(h, VGPU_ERR_ARG, "null pair gradient output");
   return adjoint_run(h, n_steps, target, w, every, loss_out, grad_out, pair_out);
}
