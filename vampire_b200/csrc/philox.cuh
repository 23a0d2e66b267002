// Counter-based Philox4x32-10 generator (Salmon, Moraes, Dror, Shaw,
// "Parallel random numbers: as easy as 1, 2, 3", SC'11) and the Box-Muller
// transform, for in-register thermal noise.  The stream is keyed by a 64-bit
// seed; the counter is (atom, step_lo, step_hi, purpose), so a step's noise
// can be regenerated anywhere (the corrector recomputes what the predictor
// used) and a run resumes bit-exactly from (seed, step).
#pragma once
#include <stdint.h>

#ifdef __CUDACC__
#define VGPU_HD __host__ __device__ __forceinline__
#else
#define VGPU_HD inline
#endif

namespace vgpu {

// purposes (4th counter word)
enum : uint32_t { RNG_THERMAL = 0u, RNG_MC_MOVE = 1u, RNG_MC_ACCEPT = 2u, RNG_THERMAL_HI = 3u, RNG_CMC_MOVE = 4u,
                  RNG_CMC_ACCEPT = 5u };

struct u32x4 { uint32_t x, y, z, w; };

VGPU_HD void mulhilo32(uint32_t a, uint32_t b, uint32_t& hi, uint32_t& lo) {
#ifdef __CUDA_ARCH__
   lo = a * b;
   hi = __umulhi(a, b);
#else
   uint64_t p = (uint64_t)a * (uint64_t)b;
   lo = (uint32_t)p;
   hi = (uint32_t)(p >> 32);
#endif
}

VGPU_HD u32x4 philox4x32_10(u32x4 c, uint32_t k0, uint32_t k1) {
   const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
   const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
   for (int r = 0; r < 10; ++r) {
      uint32_t hi0, lo0, hi1, lo1;
      mulhilo32(M0, c.x, hi0, lo0);
      mulhilo32(M1, c.z, hi1, lo1);
      u32x4 n;
      n.x = hi1 ^ c.y ^ k0;
      n.y = lo1;
      n.z = hi0 ^ c.w ^ k1;
      n.w = lo0;
      c = n;
      k0 += W0;
      k1 += W1;
   }
   return c;
}

// uniform in (0,1): 24-bit float and 32-bit double variants
VGPU_HD float u01f(uint32_t x) { return ((float)(x >> 8) + 0.5f) * (1.0f / 16777216.0f); }
VGPU_HD double u01d(uint32_t x) { return ((double)x + 0.5) * (1.0 / 4294967296.0); }

#ifdef __CUDACC__
// Box-Muller radius sqrt(-2 ln u), u = u01f(x), on the fast hardware
// approximations.  Away from u = 1 the logarithm is the base-2 approximation
// (absolute error <= 2^-22 on [0.5, 2], 2 ulp below); within 1/64 of 1 it is
// the series -ln(1 - v) = v + v^2/2 + v^3/3 + v^4/4 (truncation below 2^-26
// relative) in v = 1 - u, taken exactly from the complemented integer, so the
// radius keeps its accuracy as u -> 1.  Radius error <= 2e-6 absolute.
__device__ __forceinline__ float bm_radius_fast(uint32_t x) {
   const float u = u01f(x);
   const float v = u01f(~x);  // 1 - u, exact where it is used
   const float e_near = v * fmaf(v, fmaf(v, fmaf(v, 0.25f, 1.0f / 3.0f), 0.5f), 1.0f);
   const float e_far = -0.69314718f * __log2f(u);
   float t = 2.0f * (v < 0.015625f ? e_near : e_far), r;
   asm("sqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(t));
   return r;
}

// cos and sin of the Box-Muller angle 2 pi u, u = u01f(x), as the fast
// approximations of the angle 2 pi (u - 1/2) in [-pi, pi) (absolute error
// <= 2^-21.4 there) negated.
__device__ __forceinline__ void bm_angle_fast(uint32_t x, float& c, float& s) {
   __sincosf(6.28318531f * (u01f(x) - 0.5f), &s, &c);
   c = -c;
   s = -s;
}
__device__ __forceinline__ float bm_cos_fast(uint32_t x) { return -__cosf(6.28318531f * (u01f(x) - 0.5f)); }
#endif

}  // namespace vgpu
