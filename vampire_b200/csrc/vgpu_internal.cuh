// Internal declarations shared by the libvgpu CUDA translation units.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "record_plan.h"
#include "vgpu.h"

namespace vgpu {

// ---------------------------------------------------------------------------
// Exchange formats of the sliced-ELL (SELL-32) bond storage.  The uploader
// picks the most compact one that reproduces the reference's per-bond list
// exactly; the per-bond bytes are what the fused kernels stream from HBM.
// ---------------------------------------------------------------------------
enum ExchFmt : int {
   FMT_ISO_TAB = 0,     // J = table[mi][mj]                         0 B/bond
   FMT_ISO_BOND = 1,    // scalar per bond                            4 B/bond
   FMT_VEC_TAB = 2,     // diag(table[mi][mj])                        0 B/bond
   FMT_VEC_BOND = 3,    // 3 per bond                                12 B/bond
   FMT_DMI_TAB = 4,     // diag(table[mi][mj]) + d_ij x s_j          12 B/bond
   FMT_TENSOR_BOND = 5, // full 3x3 per bond                         36 B/bond
   FMT_COUNT = 6
};

// Per-material constants in the device precision.
template <typename R>
struct MatParams {
   R A, B;            // one_oneplusalpha_sq, alpha_oneplusalpha_sq
   R sigma;           // sqrt(T_rescaled) * H_th_sigma
   R ku2, kux, kuy, kuz;
   R kc4;
   R hlx, hly, hlz;   // local applied field (0 if disabled)
   R mu_s_muB;        // moment in Bohr magnetons (stats)
   R dhx, dhy, dhz;   // field change over a linear sweep (batched systems), added as dh * min(step, n)/n
   R alpha, beta_mid; // LLG-Midpoint: damping and -dt A / 2 (LLGMidpoint.cpp:72-73)
   R ku4, ku6, kc6;   // higher-order reduced constants [T] (0 unless enabled)
   R kcb[9];          // rotated cubic basis e1, e2, e3
};

// higher-order anisotropy terms present (LLGArgs::aniso_ext bits)
enum AnisoExt : int { ANI_U4 = 1, ANI_U6 = 2, ANI_C6 = 4, ANI_CROT = 8, ANI_NEEL = 16 };

// Everything one fused LLG pass needs, passed by value.
template <typename R>
struct LLGArgs {
   int n;                    // atoms (array length of the per-atom inputs)
   int n_alloc;              // row stride of SoA per-atom tables (n rounded up to slices, + pad atom)
   int n_upd;                // atoms the passes update: all, or the owned atoms of a shard (0..n_upd-1)
   int slice_first;          // first slice a pass updates (0: from atom 0); the pass covers atoms
                             // 32 slice_first .. n_upd-1 (a shard's core or boundary range)
   uint32_t noise_base;      // added to the atom index in the Philox counter (global index of a shard's atom 0)
   const int* slice_off;     // [nslices+1] SELL-32 entry offsets
   const int* col;           // packed neighbour index (| mat << mat_shift)
   int idx_mask;             // mask of the neighbour index bits
   int mat_shift;            // shift of the neighbour material bits (0: unpacked)
   int tab_scalar;           // diagonal table entries isotropic: use jtab_s (M*M)
   const R* jtab_s;          // scalar material-pair table, or nullptr
   const R* jb[9];           // per-bond exchange arrays in SELL layout
   const int4* rec;          // FP32 FMT_DMI_TAB: packed {index, d_x, d_y, d_z} per bond, or nullptr
   // FP32 FMT_DMI_TAB compact records (taken before rec when set): one word per
   // bond, neighbour | coupling index << crec_shift, and the coupling
   // dictionary: cdict_n entries {J (Jxx), d_x, d_y, d_z}, then (non-scalar
   // diagonal) cdict_n entries {Jyy, Jzz, 0, 0}
   const uint32_t* crec;
   const float4* cdict;
   int crec_shift, cdict_n;
   // window-staged FP32 passes: per bond the word slot | coupling index << 16,
   // slot indexing the tile's window of neighbour spins; per tile the window's
   // segments {first atom, atoms, first slot, 0} (wseg[wtile_seg[t] ..
   // wtile_seg[t+1]]) and its slot count wtile_w[t]
   const uint32_t* lrec;
   const int4* wseg;
   const int* wtile_seg;
   const int* wtile_w;
   const R* jtab;            // material-pair table (M*M or M*M*3)
   int M;                    // number of materials
   const int* mat;           // [n] material id, or nullptr when M == 1
   const MatParams<R>* mp;   // [M]
   int uniaxial, cubic;
   int aniso_ext;            // AnisoExt bits
   int integrator;           // INTEG_HEUN or INTEG_MIDPOINT
   const R* neel;            // [9][n_alloc] per-atom Neel tensors (ANI_NEEL), row-major components
   const int* bq_off;        // biquadratic exchange: SELL-32 slice offsets of its own neighbour list, or nullptr
   const int* bq_col;        // neighbour index per entry (padding: the zero pad atom)
   const R* bq_j;            // isotropic J_bq [T] per entry
   R hx, hy, hz;             // global applied field
   int local_field;          // add MatParams::hl*
   uint64_t ramp_n;          // > 0: add MatParams::dh * min(step, ramp_n) / ramp_n
   const int* sys_off;       // batched systems: first atom of each system, or nullptr
   int m_per_sys;            // materials per system (system = material / m_per_sys)
   int thermal;              // add sigma * xi
   int noise_mode;           // VGPU_NOISE_*
   uint32_t seed_lo, seed_hi;
   uint64_t step;            // Philox counter for this step
   const R* xi;              // replay noise, 3n (x|y|z blocks)
   const int* cell;          // [n] macrocell id, or nullptr
   const R* cell_field;      // [3*ncells] x|y|z blocks, B field
   const R* cell_hd;         // [3*ncells] mu0 Hd field (magnetostatic energy)
   const R* hm_atom;         // [3n] per-atom mu0 Hd field (host-computed), or nullptr
   int ncells;
   const R* hd_atom;         // [3n] per-atom dipole field (host-computed), or nullptr
   R dt, half_dt;
   R* ax; R* ay; R* az;      // state A: s0 (read), s1 (written by corrector)
   R* bx; R* by; R* bz;      // state B: s' (predictor output)
   R* fx; R* fy; R* fz;      // field output (field-only mode)
   R* ex; R* ey; R* ez;      // stored predictor increment f(s0), or nullptr (recovered)
   R* gx; R* gy; R* gz;      // staged passes: the step's external field (thermal, applied,
                             // macrocell dipole), written by the predictor and read back by
                             // the corrector, or nullptr
   int* status;              // device status word (non-finite spin flag)
   int stage_extra_tx;       // staged passes: extra bytes each tile expects (0; > 0 tests the bounded wait)
};

// FP32 DMI record layout a kernel is compiled for (exchange_field)
enum RecLayout : int { REC_ANY = 0, REC_WIDE = 1, REC_COMPACT = 2, REC_WINDOW = 3 };
enum PassMode : int { PASS_PREDICTOR = 0, PASS_CORRECTOR = 1, PASS_FIELD = 2 };
enum Integrator : int { INTEG_HEUN = 0, INTEG_MIDPOINT = 1 };
// compiled pass variants: Heun without / with the higher-order anisotropy
// terms, and the midpoint integrator (with them)
enum PassVariant : int { VAR_HEUN = 0, VAR_HEUN_EXT = 1, VAR_MIDPOINT = 2 };

// launch the fused Heun pass for the given format/mode (llg_kernels.cu)
template <typename R>
cudaError_t launch_llg_pass(const LLGArgs<R>& a, int fmt, int mode, int nslices, cudaStream_t st);

// Bulk-staged FP32 FMT_DMI_TAB passes (llg_kernels_fp32.cu): tiles of sl
// slices, nbuf shared-memory buffers of buf_bytes (the largest tile's records),
// and with compact records (crec) the coupling dictionary (dict_bytes) after them.
constexpr int kStageSmemLimit = 200 * 1024;  // dynamic shared memory the staged passes may take
constexpr int kStageOwnArrays = 11;           // own-atom arrays per staged buffer (32 SL words each)
constexpr int kStageMaxMat = 64;              // material rows the staged passes keep in shared memory
struct StageCfg {
   int sl = 4, nbuf = 1, buf_bytes = 0;
   int M = 1;                 // materials (the staged passes may keep the table in shared memory)
   bool crec = false;
   int dict_bytes = 0;
   int warps = 0;             // per-warp pipelined passes: warps per block (0: tile passes)
   bool win = false;          // window-staged passes (neighbour spins staged too)
   int wmax = 0;              // window slots of the largest tile (multiple of 4)
   int ntiles = 0, grid = 0;  // set by prepare_llg_staged
};

// dynamic shared memory of llg_staged_kernel: nbuf x (records + own-atom
// arrays), the dictionary, the material table when it has <= kStageMaxMat rows
inline int staged_smem_bytes(int sl, int nbuf, int buf_bytes, int dict_bytes, int M) {
   const int mp = M <= kStageMaxMat ? ((M * (int)sizeof(MatParams<float>) + 15) & ~15) : 0;
   return nbuf * (buf_bytes + kStageOwnArrays * 32 * sl * 4) + dict_bytes + mp;
}
int stage_tile_bytes(const std::vector<int>& slice_off, int sl);
cudaError_t prepare_llg_staged(StageCfg& c, int nslices, int device);
cudaError_t launch_llg_staged(const LLGArgs<float>& a, int mode, int nslices, const StageCfg& c, cudaStream_t st);

// write the Philox thermal Gaussians of step a.step into a.fx/fy/fz
template <typename R>
cudaError_t launch_thermal_noise(const LLGArgs<R>& a, cudaStream_t st);

// The passes are instantiated once per precision, in llg_kernels_fp32.cu and
// llg_kernels_fp64.cu (the latter without FMA contraction, for FP64 results
// equal to the reference's); other translation units that see the template
// bodies must not instantiate their own copies.
extern template cudaError_t launch_llg_pass<float>(const LLGArgs<float>&, int, int, int, cudaStream_t);
extern template cudaError_t launch_llg_pass<double>(const LLGArgs<double>&, int, int, int, cudaStream_t);
extern template cudaError_t launch_thermal_noise<float>(const LLGArgs<float>&, cudaStream_t);
extern template cudaError_t launch_thermal_noise<double>(const LLGArgs<double>&, cudaStream_t);

// A kernel launched with programmatic stream serialisation: its blocks may be
// scheduled while the previous kernel of the stream drains.  The kernel must
// execute griddepcontrol.wait before it touches anything that kernel writes
// (the staged LLG passes, the small-mask magnetisation update, the row copy).
template <typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(Args...), dim3 g, dim3 b, int smem, cudaStream_t st, Args... args) {
   cudaLaunchConfig_t cfg = {};
   cfg.gridDim = g;
   cfg.blockDim = b;
   cfg.dynamicSmemBytes = (size_t)smem;
   cfg.stream = st;
   cudaLaunchAttribute attr[1];
   attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
   attr[0].val.programmaticStreamSerializationAllowed = 1;
   cfg.attrs = attr;
   cfg.numAttrs = 1;
   return cudaLaunchKernelEx(&cfg, kernel, args...);
}

}  // namespace vgpu
