// FP32 instantiation of the fused LLG-Heun passes (production precision;
// FMA contraction on), and the bulk-staged variant of the FMT_DMI_TAB passes.
#include "llg_staged.cuh"

namespace vgpu {
template cudaError_t launch_llg_pass<float>(const LLGArgs<float>&, int, int, int, cudaStream_t);
template cudaError_t launch_thermal_noise<float>(const LLGArgs<float>&, cudaStream_t);

int stage_tile_bytes(const std::vector<int>& slice_off, int sl) { return staged_tile_bytes(slice_off, sl); }

template <int MODE, int SL, int NBUF, bool CREC>
static const void* staged_fn() {
   return (const void*)llg_staged_kernel<MODE, SL, NBUF, CREC>;
}

static const void* window_fn(int mode, int sl) {
   const bool p = mode == PASS_PREDICTOR;
#define VGPU_FN(S) \
   if (sl == S) return p ? (const void*)llg_window_kernel<PASS_PREDICTOR, S> : (const void*)llg_window_kernel<PASS_CORRECTOR, S>;
   VGPU_FN(2) VGPU_FN(4) VGPU_FN(8)
#undef VGPU_FN
   return nullptr;
}

static const void* staged_fn(int mode, int sl, int nbuf, bool crec) {
   const bool p = mode == PASS_PREDICTOR;
#define VGPU_FN(S, B)                                                                                          \
   if (sl == S && nbuf == B) {                                                                                 \
      if (crec) return p ? staged_fn<PASS_PREDICTOR, S, B, true>() : staged_fn<PASS_CORRECTOR, S, B, true>();  \
      return p ? staged_fn<PASS_PREDICTOR, S, B, false>() : staged_fn<PASS_CORRECTOR, S, B, false>();          \
   }
   VGPU_FN(2, 1) VGPU_FN(2, 2) VGPU_FN(4, 1) VGPU_FN(4, 2) VGPU_FN(8, 1) VGPU_FN(8, 2)
#undef VGPU_FN
   return nullptr;
}

// The default shape (2-slice tiles, two buffers, compact records) is also
// compiled for every FEAT_FIXED feature set; the launcher takes the one that
// stage_features names (the generic pass when it names none).
using StagedFn = void (*)(LLGArgs<float>, int, int, int);

template <int MODE>
static StagedFn staged_fixed_fn(int feat) {
   switch (feat) {
#define VGPU_F(k) \
   case FEAT_FIXED | ((k) << 1): return llg_staged_kernel<MODE, 2, 2, true, FEAT_FIXED | ((k) << 1)>;
      VGPU_F(0) VGPU_F(1) VGPU_F(2) VGPU_F(3) VGPU_F(4) VGPU_F(5) VGPU_F(6) VGPU_F(7)
      VGPU_F(8) VGPU_F(9) VGPU_F(10) VGPU_F(11) VGPU_F(12) VGPU_F(13) VGPU_F(14) VGPU_F(15)
#undef VGPU_F
      default: return llg_staged_kernel<MODE, 2, 2, true, 0>;
   }
}

static StagedFn staged_fixed_fn(int mode, int feat) {
   return mode == PASS_PREDICTOR ? staged_fixed_fn<PASS_PREDICTOR>(feat) : staged_fixed_fn<PASS_CORRECTOR>(feat);
}

// shared memory of the per-warp pipelined passes
static int warp_smem_bytes(const StageCfg& c) {
   const int mp = c.M <= kStageMaxMat ? ((c.M * (int)sizeof(MatParams<float>) + 15) & ~15) : 0;
   return c.dict_bytes + mp + c.warps * 2 * (c.buf_bytes + kStageOwnArrays * 128);
}

static int warp_mp_bytes(const StageCfg& c) {
   return c.M <= kStageMaxMat ? ((c.M * (int)sizeof(MatParams<float>) + 15) & ~15) : 0;
}

cudaError_t prepare_llg_staged(StageCfg& c, int nslices, int device) {
   c.grid = 0;
   if (c.warps > 0) {
      if (!(c.warps == 2 || c.warps == 4) || !c.crec || c.win) return cudaErrorInvalidValue;
      const int smem = warp_smem_bytes(c);
      int sms = 0, optin = 0;
      cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
      if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
      if (e != cudaSuccess) return e;
      if (smem > optin - 128) return cudaErrorInvalidValue;
      int per_sm = 1 << 30;
      for (int mode = PASS_PREDICTOR; mode <= PASS_CORRECTOR; ++mode) {
         const void* f = mode == PASS_PREDICTOR ? (const void*)llg_warp_kernel<PASS_PREDICTOR>
                                                : (const void*)llg_warp_kernel<PASS_CORRECTOR>;
         if ((e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess) return e;
         int nb = 0;
         if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, f, 32 * c.warps, smem)) != cudaSuccess) return e;
         per_sm = std::min(per_sm, nb);
      }
      if (per_sm < 1) return cudaErrorInvalidValue;
      c.ntiles = nslices;
      c.grid = std::min((nslices + c.warps - 1) / c.warps, per_sm * sms);
      return cudaSuccess;
   }
   if (!(c.sl == 2 || c.sl == 4 || c.sl == 8) || !(c.nbuf == 1 || c.nbuf == 2)) return cudaErrorInvalidValue;
   if (c.win && (c.nbuf != 1 || !c.crec)) return cudaErrorInvalidValue;
   const int smem = c.win ? c.buf_bytes + 12 * c.wmax + c.dict_bytes
                          : staged_smem_bytes(c.sl, c.nbuf, c.buf_bytes, c.dict_bytes, c.M);
   int sms = 0, optin = 0;
   cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
   if (e == cudaSuccess) e = cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, device);
   if (e != cudaSuccess) return e;
   if (smem > optin - 64) return cudaErrorInvalidValue;  // room for the static mbarriers
   int per_sm = 1 << 30;
   const bool fixed = !c.win && c.sl == 2 && c.nbuf == 2 && c.crec;
   for (int mode = PASS_PREDICTOR; mode <= PASS_CORRECTOR; ++mode)
      for (int k = -1; k < (fixed ? 16 : 0); ++k) {
         const void* f = k >= 0 ? (const void*)staged_fixed_fn(mode, FEAT_FIXED | (k << 1))
                         : c.win ? window_fn(mode, c.sl)
                                 : staged_fn(mode, c.sl, c.nbuf, c.crec);
         if ((e = cudaFuncSetAttribute(f, cudaFuncAttributeMaxDynamicSharedMemorySize, smem)) != cudaSuccess)
            return e;
         int nb = 0;
         if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, f, 32 * c.sl, smem)) != cudaSuccess) return e;
         per_sm = std::min(per_sm, nb);
      }
   if (per_sm < 1) return cudaErrorInvalidValue;
   c.ntiles = (nslices + c.sl - 1) / c.sl;
   c.grid = c.nbuf == 1 ? c.ntiles : std::min(c.ntiles, per_sm * sms);
   return cudaSuccess;
}

cudaError_t launch_llg_staged(const LLGArgs<float>& a, int mode, int nslices, const StageCfg& c, cudaStream_t st) {
   if (c.grid == 0) return cudaSuccess;
   if ((a.crec != nullptr) != c.crec) return cudaErrorInvalidValue;  // record layout of the prepared shape
   if (c.warps > 0) {  // per-warp pipelined passes: one slice per warp tile
      const int nsl = (a.n_upd + 31) / 32 - a.slice_first;
      if (nsl <= 0) return cudaSuccess;
      const dim3 g(std::min(c.grid, (nsl + c.warps - 1) / c.warps)), b(32 * c.warps);
      return launch_pdl(mode == PASS_PREDICTOR ? llg_warp_kernel<PASS_PREDICTOR>
                                                      : llg_warp_kernel<PASS_CORRECTOR>,
                               g, b, warp_smem_bytes(c), st, a, nslices, nsl, (int)c.buf_bytes,
                               (int)c.dict_bytes, warp_mp_bytes(c));
   }
   // tiles of the updated range: slices slice_first .. ceil(n_upd / 32) - 1
   const int ntiles = ((a.n_upd + 31) / 32 - a.slice_first + c.sl - 1) / c.sl;
   if (ntiles <= 0) return cudaSuccess;
   if (c.win && a.slice_first != 0) return cudaErrorInvalidValue;  // window plans cover whole shards
   const dim3 g(std::min(c.grid, ntiles)), b(32 * c.sl);
   if (c.win) {
      if (!a.lrec || !a.wseg) return cudaErrorInvalidValue;
      const int smem = c.buf_bytes + 12 * c.wmax + c.dict_bytes;
#define VGPU_WIN(S)                                                                                            \
   if (c.sl == S) {                                                                                            \
      if (mode == PASS_PREDICTOR)                                                                              \
         llg_window_kernel<PASS_PREDICTOR, S><<<g, b, smem, st>>>(a, nslices, c.buf_bytes, c.wmax);            \
      else                                                                                                     \
         llg_window_kernel<PASS_CORRECTOR, S><<<g, b, smem, st>>>(a, nslices, c.buf_bytes, c.wmax);            \
      return cudaGetLastError();                                                                               \
   }
      VGPU_WIN(2) VGPU_WIN(4) VGPU_WIN(8)
#undef VGPU_WIN
      return cudaErrorInvalidValue;
   }
   const int smem = staged_smem_bytes(c.sl, c.nbuf, c.buf_bytes, c.dict_bytes, c.M);
   if (c.sl == 2 && c.nbuf == 2 && c.crec)
      return launch_pdl(staged_fixed_fn(mode, stage_features(a)), g, b, smem, st, a, nslices, ntiles,
                               (int)c.buf_bytes);
#define VGPU_STAGED_C(S, B, C)                                                                                 \
   e = launch_pdl(mode == PASS_PREDICTOR ? llg_staged_kernel<PASS_PREDICTOR, S, B, C>                   \
                                                : llg_staged_kernel<PASS_CORRECTOR, S, B, C>,                  \
                         g, b, smem, st, a, nslices, ntiles, (int)c.buf_bytes);
#define VGPU_STAGED(S, B)                                                                                      \
   if (c.sl == S && c.nbuf == B) {                                                                             \
      cudaError_t e;                                                                                           \
      if (c.crec) { VGPU_STAGED_C(S, B, true) } else { VGPU_STAGED_C(S, B, false) }                            \
      return e;                                                                                                \
   }
   VGPU_STAGED(2, 1) VGPU_STAGED(2, 2) VGPU_STAGED(4, 1) VGPU_STAGED(4, 2) VGPU_STAGED(8, 1) VGPU_STAGED(8, 2)
#undef VGPU_STAGED
#undef VGPU_STAGED_C
   return cudaErrorInvalidValue;
}
}  // namespace vgpu
