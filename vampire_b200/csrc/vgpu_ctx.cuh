// Context object behind a vgpu_handle.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

#include "vgpu.h"
#include "vgpu_internal.cuh"

namespace vgpu {

// Device-side system (pointers owned by vgpu_ctx::allocs).
struct SysDev {
   bool uploaded = false;
   int n = 0, M = 1, nslices = 0, n_alloc = 0, fmt = 0;
   int n_owned = 0;           // atoms 0..n_owned-1 are updated (n unless vgpu_set_owned)
   uint32_t noise_base = 0;   // Philox atom index of local atom 0
   int mat_shift = 0, idx_mask = 0x7fffffff;
   int64_t num_bonds = 0, sell_entries = 0;
   int uniaxial = 0, cubic = 0;
   void* slice_off = nullptr;
   void* col = nullptr;
   void* jb[9] = {nullptr};
   void* rec = nullptr;      // packed 16-byte bond records (FP32 FMT_DMI_TAB)
   void* crec = nullptr;     // compact 4-byte records (FP32 FMT_DMI_TAB, few distinct couplings), or nullptr
   void* cdict = nullptr;    // their coupling dictionary (float4 entries)
   int crec_shift = 0, cdict_n = 0;
   std::vector<uint32_t> crec_host;  // host copy of crec (window planning)
   std::vector<int> off_host;        // host copy of slice_off
   // window plan of the window-staged passes (built on first use for the tile
   // shape and owned-atom count it was made for)
   int win_sl = 0, win_nupd = -1;
   bool win_ok = false;
   int wmax = 0;
   void* lrec = nullptr;
   void* wseg = nullptr;
   void* wtile_seg = nullptr;
   void* wtile_w = nullptr;
   void* jtab_s = nullptr;   // scalar material-pair table (isotropic diagonal)
   int tab_scalar = 0;
   void* jtab = nullptr;
   void* mat = nullptr;
   void* mp = nullptr;
   void* s[3] = {nullptr};   // state A
   void* p[3] = {nullptr};   // state B (predictor)
   void* f[3] = {nullptr};   // field output
   void* e[3] = {nullptr};   // stored predictor increment in use (VGPU_OPT_STORE_INCREMENT)
   void* e_store[3] = {nullptr};  // its buffers, once allocated
   void* g_store[3] = {nullptr};  // staged passes: the step's external field (predictor -> corrector)
   void* xi = nullptr;       // replay noise
   double* stage64 = nullptr;  // [3n] FP64 staging of host transfers (FP32 state)
   int* status = nullptr;
   // macrocell dipole
   int ncells = 0;
   void* cell = nullptr;
   void* cell_field = nullptr;   // [3][ncells] B field (LLG)
   void* cell_hd = nullptr;      // [3][ncells] mu0 Hd field (energies)
   double* mus_SI = nullptr;     // [M] moments in J/T
   void* hd_atom = nullptr;
   void* hm_atom = nullptr;  // per-atom mu0 Hd field for the magnetostatic energy
   void* mc_tab = nullptr;   // Monte Carlo per-material tables
   std::vector<unsigned char> mc_tab_host;  // last contents copied to mc_tab
   const int* sys_off = nullptr;  // batched systems: first atom of each system
   int m_per_sys = 1;
   uint64_t ramp_n = 0;      // batched field sweep length (steps)
   int stage_bytes[4] = {0, 0, 0, 0};  // largest tile's records, tiles of 2 / 4 / 8 / 1 slices
   StageCfg stage;                          // prepared bulk-staged launch (grid 0: not prepared)
   std::vector<int> type_host;
   std::vector<int64_t> row_host;  // CSR kept on the host (colouring, sharding)
   std::vector<int> nl_host;
   std::vector<vgpu_material> materials;
   std::vector<unsigned char> mp_host;  // last material table copied to mp
   // higher-order anisotropy (vgpu_set_anisotropy_ext)
   int aniso_ext = 0;                          // AnisoExt bits
   std::vector<double> ku4_h, ku6_h, kc6_h, kcb_h;  // per material (kcb: 9 each)
   void* neel = nullptr;                       // [9][n_alloc] Neel tensors
   // spin snapshots (vgpu_snapshot_setup): output atom list and FP64 x|y|z buffer
   void* snap_idx = nullptr;
   void* snap_buf = nullptr;
   int64_t snap_n = -1;                        // -1: no list set up
   // biquadratic exchange (vgpu_set_biquadratic): SELL-32 copy of its list
   void* bq_off = nullptr;
   void* bq_col = nullptr;
   void* bq_j = nullptr;
};

int set_err(vgpu_ctx* h, int code, const char* fmt, ...);
int cuda_err(vgpu_ctx* h, cudaError_t e, const char* what);

// kinds of timed device work (vgpu_profile_read)
enum ProfKind : int { PROF_PREDICTOR = 0, PROF_CORRECTOR = 1, PROF_STATS = 2, PROF_DIPOLE = 3, PROF_MC = 4,
                      PROF_OTHER = 5, PROF_KINDS = 6 };

void stats_destroy(vgpu_ctx* h);
void mc_destroy(vgpu_ctx* h);
void dipole_destroy(vgpu_ctx* h);
void batch_destroy(vgpu_ctx* h);
void torque_destroy(vgpu_ctx* h);
void cmc_destroy(vgpu_ctx* h);
int torque_reset(vgpu_ctx* h);
const double* batch_ramp(vgpu_ctx* h);

}  // namespace vgpu

struct vgpu_ctx {
   int device = 0;
   int prec = VGPU_PREC_FP32;
   cudaStream_t stream = nullptr;
   std::string err;
   std::vector<void*> allocs;
   vgpu::SysDev sys;
   vgpu_sim_params params;
   uint64_t step = 0;
   uint64_t seed = 0;
   int noise_mode = VGPU_NOISE_PHILOX;
   bool any_sigma = false;
   int store_increment = -1;  // -1: default (on for FP64, off for FP32)
   bool batch_materials = false;  // batch handle: material rows are per system (no 100 limit)
   int staged = -1;          // VGPU_OPT_STAGED_RECORDS (-1 default)
   int stage_sl = -1, stage_nbuf = -1;  // -1: per record layout (tile_shape in vgpu_api.cu)
   bool stage_wait_test = false;  // VGPU_OPT_STAGE_WAIT_TEST
   int dipole_fft = -1;      // VGPU_OPT_DIPOLE_FFT (-1 default: FFT far field on regular cell grids)
   int compact = -1;         // VGPU_OPT_COMPACT_RECORDS (-1 default: compact records when built)
   int window = -1;          // VGPU_OPT_WINDOW_STAGING (-1 default: off)
   int stage_warps = -1;     // VGPU_OPT_STAGE_WARPS (-1 default; 0 off; 2 or 4 warps per block)

   void* alloc(size_t bytes);
   void release(void* p);    // free one allocation made by alloc (nullptr: nothing)
   void free_system();
   int refresh_materials();
   int check_status();
   void update_sigma_flag();
   // hooks implemented by the other subsystems
   int after_step();          // dipole cadence (dipole.cu)
   int fields_ready();        // VGPU_OK, or an error while a shard's dipole field awaits its moment sum
   void destroy_extras();     // free subsystem state (stats, mc, dipole)
   void* extras[8] = {nullptr};

   // kernel accounting and optional per-launch CUDA-event timing on `stream`
   int64_t kernel_launches = 0;
   bool prof_on = false;
   int prof_every = 1;        // time the launches of one step in prof_every (VGPU_OPT_PROFILE_EVERY)
   struct ProfRec { int kind; cudaEvent_t a, b; };
   std::vector<ProfRec> prof_pending;
   std::vector<cudaEvent_t> event_pool;
   double prof_ms[vgpu::PROF_KINDS] = {0};
   int64_t prof_count[vgpu::PROF_KINDS] = {0};
   cudaEvent_t prof_open = nullptr;
   cudaEvent_t get_event();
   void prof_begin(int kind);
   void prof_end(int kind);
   int prof_collect();
};

namespace vgpu {
template <typename R> LLGArgs<R> make_args(vgpu_ctx* h);
}
