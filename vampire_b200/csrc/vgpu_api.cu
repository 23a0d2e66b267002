// C ABI of libvgpu.so (include/vgpu.h): context, system upload, LLG stepping.
//
// Upload turns the reference's CSR neighbour list and unrolled per-bond
// exchange list (src/exchange/initialize.cpp:70-117,
// unroll_normalised.cpp:37-140) into a sliced-ELL layout with slices of 32
// atoms, and picks the most compact exchange format that reproduces every
// bond's coupling exactly (ExchFmt in vgpu_internal.cuh): couplings that are
// a function of the two materials go to a small table and the neighbour's
// material rides in the top bits of its index, so the only per-bond bytes
// left in HBM are the index and, for DMI, the antisymmetric vector.  When a
// DMI system has few distinct couplings (a crystal: one per bond direction
// and material pair), the FP32 passes take compact records instead: one word
// per bond holding the neighbour and the index of its coupling in a small
// dictionary (build_compact_records).
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "record_plan.h"
#include "vgpu_ctx.cuh"

using namespace vgpu;

namespace vgpu {

std::mutex g_err_mutex;
std::string g_global_err;

int set_err(vgpu_ctx* h, int code, const char* fmt, ...) {
   char buf[1024];
   va_list ap;
   va_start(ap, fmt);
   vsnprintf(buf, sizeof buf, fmt, ap);
   va_end(ap);
   if (h) h->err = buf;
   else {
      std::lock_guard<std::mutex> g(g_err_mutex);
      g_global_err = buf;
   }
   return code;
}

int cuda_err(vgpu_ctx* h, cudaError_t e, const char* what) {
   if (e == cudaSuccess) return VGPU_OK;
   cudaGetLastError();
   return set_err(h, e == cudaErrorMemoryAllocation ? VGPU_ERR_OOM : VGPU_ERR_CUDA, "%s: %s", what,
                  cudaGetErrorString(e));
}

}  // namespace vgpu

void* vgpu_ctx::alloc(size_t bytes) {
   if (bytes == 0) bytes = 16;
   void* p = nullptr;
   cudaError_t e = cudaMalloc(&p, bytes);
   if (e != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
   }
   allocs.push_back(p);
   return p;
}
namespace vgpu {

}  // namespace vgpu

void vgpu_ctx::release(void* p) {
   if (!p) return;
   auto it = std::find(allocs.begin(), allocs.end(), p);
   if (it == allocs.end()) return;
   cudaFree(p);
   allocs.erase(it);
}

void vgpu_ctx::free_system() {
   for (void* p : allocs) cudaFree(p);
   allocs.clear();
   sys = SysDev();
}
namespace vgpu {

template <typename R>
static int upload_vec(vgpu_ctx* h, void** dst, const std::vector<R>& v, const char* what) {
   *dst = h->alloc(v.size() * sizeof(R));
   if (!*dst) return set_err(h, VGPU_ERR_OOM, "cudaMalloc failed for %s (%zu bytes)", what, v.size() * sizeof(R));
   if (v.empty()) return VGPU_OK;
   return cuda_err(h, cudaMemcpyAsync(*dst, v.data(), v.size() * sizeof(R), cudaMemcpyHostToDevice, h->stream), what);
}

// ---------------------------------------------------------------------------
// host-side exchange analysis
// ---------------------------------------------------------------------------
struct BondView {
   int exch_type;
   const double* jl;
   const int32_t* nl_type;
   int64_t num_exchange;
   const double* get(int64_t bond) const {
      const int64_t id = nl_type ? nl_type[bond] : bond;
      const int w = exch_type == VGPU_EXCH_ISOTROPIC ? 1 : exch_type == VGPU_EXCH_VECTORIAL ? 3 : 9;
      return jl + w * id;
   }
};

// Returns the chosen format; fills table (M*M*{1,3}) when a table format is possible.
static int choose_format(const vgpu_system_desc* d, const BondView& bv, std::vector<double>& table, bool can_pack) {
   const int M = d->num_materials;
   const int n = d->num_atoms;
   const int et = d->exchange_type;
   const int tw = et == VGPU_EXCH_ISOTROPIC ? 1 : 3;
   table.assign((size_t)M * M * tw, 0.0);
   std::vector<char> seen((size_t)M * M, 0);
   bool tab_ok = can_pack || M == 1;
   bool antisym_only = true;  // tensor: off-diagonal part antisymmetric
   bool any_d = false;
   for (int i = 0; i < n; ++i) {
      const int mi = d->type[i];
      for (int64_t b = d->nl_start[i]; b <= d->nl_end[i]; ++b) {
         const int mj = d->type[d->nl[b]];
         const double* J = bv.get(b);
         double diag[3];
         if (et == VGPU_EXCH_ISOTROPIC) diag[0] = J[0];
         else if (et == VGPU_EXCH_VECTORIAL) { diag[0] = J[0]; diag[1] = J[1]; diag[2] = J[2]; }
         else {
            diag[0] = J[0]; diag[1] = J[4]; diag[2] = J[8];
            if (J[1] + J[3] != 0.0 || J[2] + J[6] != 0.0 || J[5] + J[7] != 0.0) antisym_only = false;
            if (J[1] != 0.0 || J[2] != 0.0 || J[5] != 0.0) any_d = true;
         }
         if (tab_ok) {
            const size_t key = (size_t)mi * M + mj;
            double* t = &table[key * tw];
            if (!seen[key]) {
               seen[key] = 1;
               for (int k = 0; k < tw; ++k) t[k] = diag[k];
            } else {
               for (int k = 0; k < tw; ++k)
                  if (t[k] != diag[k]) tab_ok = false;
            }
         }
      }
   }
   if (et == VGPU_EXCH_ISOTROPIC) return tab_ok ? FMT_ISO_TAB : FMT_ISO_BOND;
   if (et == VGPU_EXCH_VECTORIAL) return tab_ok ? FMT_VEC_TAB : FMT_VEC_BOND;
   if (antisym_only && tab_ok) return any_d ? FMT_DMI_TAB : FMT_VEC_TAB;
   return FMT_TENSOR_BOND;
}

static int validate(vgpu_ctx* h, const vgpu_system_desc* d) {
   if (!d) return set_err(h, VGPU_ERR_ARG, "null system descriptor");
   if (d->num_atoms <= 0) return set_err(h, VGPU_ERR_ARG, "num_atoms must be positive (got %d)", d->num_atoms);
   if (d->num_atoms > (1 << 30)) return set_err(h, VGPU_ERR_ARG, "num_atoms too large");
   const int max_mat = (h && h->batch_materials) ? 65536 : 100;  // mp::max_materials
   if (d->num_materials <= 0 || d->num_materials > max_mat)
      return set_err(h, VGPU_ERR_ARG, "num_materials must be in 1..%d (got %d)", max_mat, d->num_materials);
   if (d->exchange_type < 0 || d->exchange_type > 2)
      return set_err(h, VGPU_ERR_ARG, "unknown exchange_type %d", d->exchange_type);
   if (!d->nl_start || !d->nl_end || (d->num_bonds > 0 && (!d->nl || !d->jlist)) || !d->type || !d->materials ||
       !d->sx || !d->sy || !d->sz)
      return set_err(h, VGPU_ERR_ARG, "null array in system descriptor");
   if (d->num_bonds < 0 || d->num_bonds >= (int64_t)1 << 31) return set_err(h, VGPU_ERR_ARG, "bad num_bonds");
   const int64_t nex = d->nl_type ? d->num_exchange : d->num_bonds;
   for (int i = 0; i < d->num_atoms; ++i) {
      const int64_t s = d->nl_start[i], e = d->nl_end[i];
      if (s < 0 || e < s - 1 || e >= d->num_bonds)
         return set_err(h, VGPU_ERR_ARG, "corrupt CSR row %d: start %lld end %lld num_bonds %lld", i, (long long)s,
                        (long long)e, (long long)d->num_bonds);
      const int t = d->type[i];
      if (t < 0 || t >= d->num_materials) return set_err(h, VGPU_ERR_ARG, "atom %d has material %d out of range", i, t);
      for (int64_t b = s; b <= e; ++b) {
         const int j = d->nl[b];
         if (j < 0 || j >= d->num_atoms)
            return set_err(h, VGPU_ERR_ARG, "corrupt CSR: bond %lld of atom %d points to %d (num_atoms %d)",
                           (long long)b, i, j, d->num_atoms);
         if (d->nl_type && (d->nl_type[b] < 0 || d->nl_type[b] >= nex))
            return set_err(h, VGPU_ERR_ARG, "bond %lld interaction id out of range", (long long)b);
      }
      if (!std::isfinite(d->sx[i]) || !std::isfinite(d->sy[i]) || !std::isfinite(d->sz[i]))
         return set_err(h, VGPU_ERR_NAN, "initial spin of atom %d is not finite", i);
   }
   return VGPU_OK;
}

template <typename R>
static int upload_typed(vgpu_ctx* h, const vgpu_system_desc* d) {
   const int n = d->num_atoms;
   const int M = d->num_materials;
   const int nslices = (n + 31) / 32;
   const int n_alloc = nslices * 32 + 1;  // + one zero "padding" atom
   const int pad = n_alloc - 1;
   int shift = 1;
   while ((1 << shift) <= pad) ++shift;
   const bool can_pack = M == 1 || ((int64_t)(M - 1) << shift) < ((int64_t)1 << 31);
   BondView bv{d->exchange_type, d->jlist, d->nl_type, d->num_exchange};
   std::vector<double> table;
   const int fmt = d->num_bonds ? choose_format(d, bv, table, can_pack) : FMT_ISO_TAB;
   const bool tabfmt = fmt == FMT_ISO_TAB || fmt == FMT_VEC_TAB || fmt == FMT_DMI_TAB;
   const int use_shift = (tabfmt && M > 1) ? shift : 0;
   if (table.empty()) table.assign((size_t)M * M * 3, 0.0);

   // slice widths and offsets
   std::vector<int> off(nslices + 1, 0);
   for (int s = 0; s < nslices; ++s) {
      int w = 0;
      for (int l = 0; l < 32; ++l) {
         const int i = s * 32 + l;
         if (i < n) w = std::max<int>(w, (int)(d->nl_end[i] - d->nl_start[i] + 1));
      }
      off[s + 1] = off[s] + 32 * w;
   }
   const size_t ne = (size_t)off[nslices];
   std::vector<int> col(ne, pad);
   const int nper = fmt == FMT_ISO_BOND ? 1 : (fmt == FMT_VEC_BOND || fmt == FMT_DMI_TAB) ? 3
                  : fmt == FMT_TENSOR_BOND ? 9 : 0;
   std::vector<std::vector<R>> jb(nper, std::vector<R>(ne, (R)0));
   for (int i = 0; i < n; ++i) {
      const int s = i >> 5, l = i & 31;
      const int mi = d->type[i];
      (void)mi;
      int k = 0;
      for (int64_t b = d->nl_start[i]; b <= d->nl_end[i]; ++b, ++k) {
         const size_t e = (size_t)off[s] + 32 * (size_t)k + l;
         const int j = d->nl[b];
         col[e] = j | (use_shift ? (d->type[j] << use_shift) : 0);
         const double* J = bv.get(b);
         switch (fmt) {
            case FMT_ISO_BOND: jb[0][e] = (R)J[0]; break;
            case FMT_VEC_BOND: jb[0][e] = (R)J[0]; jb[1][e] = (R)J[1]; jb[2][e] = (R)J[2]; break;
            case FMT_DMI_TAB:  // d = (T[2][1], T[0][2], T[1][0])
               jb[0][e] = (R)J[7]; jb[1][e] = (R)J[2]; jb[2][e] = (R)J[3];
               break;
            case FMT_TENSOR_BOND:
               for (int q = 0; q < 9; ++q) jb[q][e] = (R)J[q];
               break;
            default: break;
         }
      }
   }
   std::vector<R> tabR(table.begin(), table.end());
   // scalar table when every diagonal entry is isotropic (Jxx == Jyy == Jzz)
   bool scalar = (fmt == FMT_VEC_TAB || fmt == FMT_DMI_TAB);
   std::vector<R> tabS;
   if (scalar) {
      tabS.resize((size_t)M * M);
      for (size_t q = 0; q < tabS.size(); ++q) {
         if (table[3 * q] != table[3 * q + 1] || table[3 * q] != table[3 * q + 2]) scalar = false;
         tabS[q] = (R)table[3 * q];
      }
   }
   std::vector<int> mat(d->type, d->type + n);
   // state arrays padded to a multiple of 4 entries: window copies move whole
   // 16-byte groups of atoms, the last one reaching up to entry n_alloc4 - 1
   const int n_alloc4 = (n_alloc + 3) & ~3;
   std::vector<R> ax(n_alloc4, (R)0), ay(n_alloc4, (R)0), az(n_alloc4, (R)0);
   for (int i = 0; i < n; ++i) { ax[i] = (R)d->sx[i]; ay[i] = (R)d->sy[i]; az[i] = (R)d->sz[i]; }

   h->free_system();
   SysDev& S = h->sys;
   S.n = n; S.M = M; S.nslices = nslices; S.n_alloc = n_alloc; S.fmt = fmt;
   S.n_owned = n;
   S.mat_shift = use_shift; S.idx_mask = use_shift ? ((1 << use_shift) - 1) : 0x7fffffff;
   S.num_bonds = d->num_bonds; S.sell_entries = (int64_t)ne;
   S.uniaxial = d->uniaxial_enabled; S.cubic = d->cubic_enabled;
   S.type_host = mat;
   S.materials.assign(d->materials, d->materials + M);
   S.row_host.assign(n + 1, 0);
   S.nl_host.clear();
   S.nl_host.reserve((size_t)d->num_bonds);
   for (int i = 0; i < n; ++i) {
      for (int64_t b = d->nl_start[i]; b <= d->nl_end[i]; ++b) S.nl_host.push_back(d->nl[b]);
      S.row_host[i + 1] = (int64_t)S.nl_host.size();
   }
   int rc;
   if ((rc = upload_vec(h, &S.slice_off, off, "slice offsets"))) return rc;
   if ((rc = upload_vec(h, &S.col, col, "neighbour index"))) return rc;
   for (int q = 0; q < nper; ++q)
      if ((rc = upload_vec(h, &S.jb[q], jb[q], "bond couplings"))) return rc;
   if (fmt == FMT_DMI_TAB && sizeof(R) == 4) {
      // one 16-byte record per bond for the fused passes: {index, d_x, d_y, d_z}
      std::vector<int> rec(4 * ne);
      for (size_t e = 0; e < ne; ++e) {
         rec[4 * e] = col[e];
         std::memcpy(&rec[4 * e + 1], &jb[0][e], 4);
         std::memcpy(&rec[4 * e + 2], &jb[1][e], 4);
         std::memcpy(&rec[4 * e + 3], &jb[2][e], 4);
      }
      if ((rc = upload_vec(h, &S.rec, rec, "bond records"))) return rc;
      S.stage_bytes[0] = stage_tile_bytes(off, 2);
      S.stage_bytes[1] = stage_tile_bytes(off, 4);
      S.stage_bytes[2] = stage_tile_bytes(off, 8);
      S.stage_bytes[3] = stage_tile_bytes(off, 1);
      if constexpr (sizeof(R) == 4) {
         std::vector<uint32_t> crec;
         std::vector<float> dict;
         int ndict = 0;
         if (build_compact_records(off, col, n, d->type, M, shift, use_shift, jb, scalar, tabS, tabR, crec, dict,
                                   ndict)) {
            if ((rc = upload_vec(h, &S.crec, crec, "compact bond records"))) return rc;
            if ((rc = upload_vec(h, &S.cdict, dict, "coupling dictionary"))) return rc;
            S.crec_shift = shift;
            S.cdict_n = ndict;
            S.crec_host = std::move(crec);
            S.off_host = off;
         }
      }
   }
   if ((rc = upload_vec(h, &S.jtab, tabR, "coupling table"))) return rc;
   S.tab_scalar = scalar;
   if (scalar) { if ((rc = upload_vec(h, &S.jtab_s, tabS, "scalar coupling table"))) return rc; }
   if (M > 1) {
      std::vector<int> matp(mat);
      matp.resize(n_alloc4, 0);  // padded like the state arrays (whole-slice copies of the staged passes)
      if ((rc = upload_vec(h, &S.mat, matp, "materials"))) return rc;
   }
   if ((rc = upload_vec(h, &S.s[0], ax, "spins"))) return rc;
   if ((rc = upload_vec(h, &S.s[1], ay, "spins"))) return rc;
   if ((rc = upload_vec(h, &S.s[2], az, "spins"))) return rc;
   std::vector<R> zeros(n_alloc4, (R)0);
   for (int q = 0; q < 3; ++q)
      if ((rc = upload_vec(h, &S.p[q], zeros, "predictor state"))) return rc;
   S.mp = h->alloc(sizeof(MatParams<R>) * M);
   if (!S.mp) return set_err(h, VGPU_ERR_OOM, "cudaMalloc failed for material table");
   S.status = (int*)h->alloc(sizeof(int));
   if (!S.status) return set_err(h, VGPU_ERR_OOM, "cudaMalloc failed for status word");
   if ((rc = cuda_err(h, cudaMemsetAsync(S.status, 0, sizeof(int), h->stream), "status"))) return rc;
   S.uploaded = true;
   return h->refresh_materials();
}

template <typename R>
int refresh_materials_typed(vgpu_ctx* h) {
   SysDev& S = h->sys;
   const vgpu_sim_params& p = h->params;
   std::vector<MatParams<R>> mp(S.M);
   for (int m = 0; m < S.M; ++m) {
      const vgpu_material& q = S.materials[m];
      const double T = p.local_temperature ? q.temperature : p.temperature;
      const double a = q.temperature_rescaling_alpha, Tc = q.temperature_rescaling_Tc;
      const double Tr = T < Tc ? Tc * std::pow(T / Tc, a) : T;
      MatParams<R>& o = mp[m];
      o.A = (R)q.one_oneplusalpha_sq;
      o.B = (R)q.alpha_oneplusalpha_sq;
      o.sigma = (R)(std::sqrt(Tr) * q.H_th_sigma);
      o.ku2 = (R)q.ku2;
      o.kux = (R)q.ku_vector[0]; o.kuy = (R)q.ku_vector[1]; o.kuz = (R)q.ku_vector[2];
      o.kc4 = (R)q.kc4;
      o.hlx = (R)q.applied_field[0]; o.hly = (R)q.applied_field[1]; o.hlz = (R)q.applied_field[2];
      o.mu_s_muB = (R)(q.mu_s_SI / 9.27400915e-24);
      o.alpha = (R)q.alpha;
      o.beta_mid = (R)(-1.0 * p.dt * q.one_oneplusalpha_sq * 0.5);
      o.ku4 = S.ku4_h.empty() ? (R)0 : (R)S.ku4_h[m];
      o.ku6 = S.ku6_h.empty() ? (R)0 : (R)S.ku6_h[m];
      o.kc6 = S.kc6_h.empty() ? (R)0 : (R)S.kc6_h[m];
      for (int k = 0; k < 9; ++k)
         o.kcb[k] = S.kcb_h.empty() ? (R)(k % 4 == 0 ? 1 : 0) : (R)S.kcb_h[9 * (size_t)m + k];
      const double* rp = batch_ramp(h);
      o.dhx = rp ? (R)rp[3 * m] : (R)0;
      o.dhy = rp ? (R)rp[3 * m + 1] : (R)0;
      o.dhz = rp ? (R)rp[3 * m + 2] : (R)0;
   }
   // unchanged table (the common case of a per-step parameter sync): no copy,
   // so the call neither waits for the stream nor adds a transfer
   const size_t bytes = sizeof(MatParams<R>) * S.M;
   const unsigned char* raw = (const unsigned char*)mp.data();
   if (S.mp_host.size() == bytes && std::equal(raw, raw + bytes, S.mp_host.begin())) return VGPU_OK;
   S.mp_host.assign(raw, raw + bytes);
   return cuda_err(h, cudaMemcpyAsync(S.mp, mp.data(), bytes, cudaMemcpyHostToDevice, h->stream), "material upload");
}

}  // namespace vgpu

int vgpu_ctx::refresh_materials() {
   if (!sys.uploaded && sys.mp == nullptr) return VGPU_OK;
   return prec == VGPU_PREC_FP64 ? refresh_materials_typed<double>(this) : refresh_materials_typed<float>(this);
}
namespace vgpu {

template <typename R>
LLGArgs<R> make_args(vgpu_ctx* h) {
   SysDev& S = h->sys;
   LLGArgs<R> a;
   memset(&a, 0, sizeof a);
   a.n = S.n;
   a.n_alloc = S.n_alloc;
   a.aniso_ext = S.aniso_ext;
   a.neel = (const R*)S.neel;
   a.bq_off = (const int*)S.bq_off;
   a.bq_col = (const int*)S.bq_col;
   a.bq_j = (const R*)S.bq_j;
   a.n_upd = S.n_owned;
   a.slice_first = 0;
   a.noise_base = S.noise_base;
   a.slice_off = (const int*)S.slice_off;
   a.col = (const int*)S.col;
   a.idx_mask = S.idx_mask;
   a.mat_shift = S.mat_shift;
   for (int q = 0; q < 9; ++q) a.jb[q] = (const R*)S.jb[q];
   a.rec = (const int4*)S.rec;
   if (h->compact != 0 && S.crec) {
      a.crec = (const uint32_t*)S.crec;
      a.cdict = (const float4*)S.cdict;
      a.crec_shift = S.crec_shift;
      a.cdict_n = S.cdict_n;
      if (S.win_ok) {
         a.lrec = (const uint32_t*)S.lrec;
         a.wseg = (const int4*)S.wseg;
         a.wtile_seg = (const int*)S.wtile_seg;
         a.wtile_w = (const int*)S.wtile_w;
      }
   }
   a.tab_scalar = S.tab_scalar;
   a.jtab_s = (const R*)S.jtab_s;
   a.jtab = (const R*)S.jtab;
   a.M = S.M;
   a.mat = (const int*)S.mat;
   a.mp = (const MatParams<R>*)S.mp;
   a.uniaxial = S.uniaxial;
   a.cubic = S.cubic;
   const vgpu_sim_params& p = h->params;
   const double hx = p.applied_enabled ? p.H_applied * p.H_vec[0] : 0.0;
   const double hy = p.applied_enabled ? p.H_applied * p.H_vec[1] : 0.0;
   const double hz = p.applied_enabled ? p.H_applied * p.H_vec[2] : 0.0;
   a.hx = (R)hx; a.hy = (R)hy; a.hz = (R)hz;
   a.local_field = p.applied_enabled && p.local_applied_field;
   a.thermal = p.thermal_enabled && (h->noise_mode == VGPU_NOISE_REPLAY || h->any_sigma);
   a.noise_mode = h->noise_mode;
   a.seed_lo = (uint32_t)h->seed;
   a.seed_hi = (uint32_t)(h->seed >> 32);
   a.step = h->step;
   a.xi = (const R*)S.xi;
   a.cell = (const int*)S.cell;
   a.cell_field = (const R*)S.cell_field;
   a.cell_hd = (const R*)S.cell_hd;
   a.hm_atom = (const R*)S.hm_atom;
   a.ncells = S.ncells;
   a.hd_atom = (const R*)S.hd_atom;
   a.dt = (R)p.dt;
   a.half_dt = (R)(0.5 * p.dt);
   a.ax = (R*)S.s[0]; a.ay = (R*)S.s[1]; a.az = (R*)S.s[2];
   a.bx = (R*)S.p[0]; a.by = (R*)S.p[1]; a.bz = (R*)S.p[2];
   a.fx = (R*)S.f[0]; a.fy = (R*)S.f[1]; a.fz = (R*)S.f[2];
   a.ex = (R*)S.e[0]; a.ey = (R*)S.e[1]; a.ez = (R*)S.e[2];
   a.status = S.status;
   a.stage_extra_tx = h->stage_wait_test ? 16 : 0;
   a.sys_off = S.sys_off;
   a.m_per_sys = S.m_per_sys;
   a.ramp_n = S.ramp_n;
   return a;
}
template LLGArgs<float> make_args<float>(vgpu_ctx*);
template LLGArgs<double> make_args<double>(vgpu_ctx*);

// allocate or drop the stored-increment buffers according to the option
template <typename R>
static int ensure_increment(vgpu_ctx* h) {
   SysDev& S = h->sys;
   const bool want = h->store_increment < 0 ? h->prec == VGPU_PREC_FP64 : h->store_increment != 0;
   if (!want) {
      S.e[0] = S.e[1] = S.e[2] = nullptr;  // buffers (if any) stay owned by allocs until re-upload
      return VGPU_OK;
   }
   if (S.e_store[0]) {
      for (int q = 0; q < 3; ++q) S.e[q] = S.e_store[q];
      return VGPU_OK;
   }
   for (int q = 0; q < 3; ++q) {
      S.e_store[q] = h->alloc(S.n_alloc * sizeof(R));
      if (!S.e_store[q]) return set_err(h, VGPU_ERR_OOM, "cudaMalloc failed for increment buffer");
      S.e[q] = S.e_store[q];
   }
   return VGPU_OK;
}

static int stage_slot(int sl) { return sl == 2 ? 0 : sl == 4 ? 1 : 2; }

// Staged tile shape in use: the options when set, else the measured best per
// record layout (FMT_DMI_TAB FCC 100^3 on B200): 16-byte records one tile of
// 4 slices per block (double buffering halves the resident blocks); compact
// records persistent blocks, two buffers of 2-slice tiles (the next tile's
// copy in flight while this one is computed).
static bool compact_in_use(const vgpu_ctx* h) { return h->compact != 0 && h->sys.crec; }
static int stage_sl_of(const vgpu_ctx* h) { return h->stage_sl > 0 ? h->stage_sl : compact_in_use(h) ? 2 : 4; }
static int stage_nbuf_of(const vgpu_ctx* h) {
   return h->stage_nbuf > 0 ? h->stage_nbuf : compact_in_use(h) ? 2 : 1;
}
// per-warp pipelined passes (compact records, no window): warps per block, or 0
static int stage_warps_of(const vgpu_ctx* h) {
   if (!compact_in_use(h) || h->window == 1) return 0;
   return h->stage_warps > 0 ? h->stage_warps : 0;
}
// window staging is opt-in: measured slower than the L1/L2 gathers of the
// compact passes (one-tile blocks wait for the whole window to land)
static bool window_wanted(const vgpu_ctx* h) {
   return h->window == 1 && h->staged != 0 && compact_in_use(h) && stage_nbuf_of(h) == 1;
}
static int stage_dict_bytes(const SysDev& S) { return S.cdict_n * 16 * (S.tab_scalar ? 1 : 2); }

// bulk-staged passes: FP32 packed records whose tiles fit shared memory.
// Default (-1): on when the two buffers of a tile fit.
template <typename R>
static bool use_staged(vgpu_ctx* h) {
   const SysDev& S = h->sys;
   // the staged passes carry no higher-order anisotropy terms (register budget)
   if (sizeof(R) != 4 || !S.rec || S.n == 0 || h->staged == 0 || S.aniso_ext || S.bq_off) return false;
   const bool crec = h->compact != 0 && S.crec;
   const int bytes = S.stage_bytes[stage_slot(stage_sl_of(h))] / (crec ? 4 : 1);
   return staged_smem_bytes(stage_sl_of(h), stage_nbuf_of(h), bytes, crec ? stage_dict_bytes(S) : 0, S.M) <=
          kStageSmemLimit;
}

template <typename R>
static cudaError_t launch_step_pass(vgpu_ctx* h, const LLGArgs<R>& a, int mode, bool staged) {
   if constexpr (sizeof(R) == 4) {
      if (staged) return launch_llg_staged(a, mode, h->sys.nslices, h->sys.stage, h->stream);
   }
   return launch_llg_pass<R>(a, h->sys.fmt, mode, h->sys.nslices, h->stream);
}

// window plan for the current tile shape and owned atoms (window-staged
// passes: FP32 compact records, staged, one buffer); S.win_ok tells whether
// the passes use it
static int ensure_window_plan(vgpu_ctx* h) {
   SysDev& S = h->sys;
   const bool want = window_wanted(h);
   if (!want) {
      S.win_ok = false;
      return VGPU_OK;
   }
   if (S.win_sl == stage_sl_of(h) && S.win_nupd == S.n_owned) {
      S.win_ok = S.lrec != nullptr;
      return VGPU_OK;
   }
   for (void** p : {&S.lrec, &S.wseg, &S.wtile_seg, &S.wtile_w}) {
      h->release(*p);
      *p = nullptr;
   }
   S.win_sl = stage_sl_of(h);
   S.win_nupd = S.n_owned;
   S.win_ok = false;
   std::vector<uint32_t> lrec;
   std::vector<int4> segs;
   std::vector<int> tseg, tw;
   int wmax = 0;
   if (S.n_owned == 0 ||
       !build_window_plan(S.off_host, S.crec_host, S.crec_shift, S.win_sl, (S.n_owned + 31) / 32, lrec, segs, tseg,
                          tw, wmax))
      return VGPU_OK;
   int rc;
   if ((rc = upload_vec(h, &S.lrec, lrec, "window bond words"))) return rc;
   if ((rc = upload_vec(h, &S.wseg, segs, "window segments"))) return rc;
   if ((rc = upload_vec(h, &S.wtile_seg, tseg, "window tile segments"))) return rc;
   if ((rc = upload_vec(h, &S.wtile_w, tw, "window tile slots"))) return rc;
   S.wmax = (wmax + 3) & ~3;
   S.win_ok = true;
   return VGPU_OK;
}

// increment buffers and the staged launch shape, before any pass
template <typename R>
static int prepare_passes(vgpu_ctx* h, bool* staged_out, int integrator = INTEG_HEUN) {
   int rc0 = ensure_increment<R>(h);
   if (rc0) return rc0;
   const bool staged = integrator == INTEG_HEUN && use_staged<R>(h);
   if (staged && h->sys.stage.grid == 0) {
      if ((rc0 = ensure_window_plan(h))) return rc0;
      StageCfg c;
      c.sl = stage_sl_of(h);
      c.nbuf = stage_nbuf_of(h);
      c.crec = h->compact != 0 && h->sys.crec;
      c.M = h->sys.M;
      c.buf_bytes = h->sys.stage_bytes[stage_slot(c.sl)] / (c.crec ? 4 : 1);
      c.dict_bytes = c.crec ? stage_dict_bytes(h->sys) : 0;
      c.win = c.crec && h->sys.win_ok && c.buf_bytes + 12 * h->sys.wmax + c.dict_bytes <= kStageSmemLimit;
      c.wmax = c.win ? h->sys.wmax : 0;
      c.warps = c.win ? 0 : stage_warps_of(h);
      if (c.warps > 0) c.buf_bytes = h->sys.stage_bytes[3] / 4;  // one slice of compact words
      cudaError_t e = prepare_llg_staged(c, (h->sys.n_owned + 31) / 32, h->device);
      if (e != cudaSuccess) return cuda_err(h, e, "staged pass setup (tile records exceed shared memory?)");
      h->sys.stage = c;
   }
   if (staged && !h->sys.stage.win && !h->sys.g_store[0]) {
      // the step's external field, passed from the predictor to the corrector
      const size_t len = ((size_t)h->sys.n_alloc + 3) & ~(size_t)3;
      for (int q = 0; q < 3; ++q) {
         h->sys.g_store[q] = h->alloc(len * sizeof(R));
         if (!h->sys.g_store[q]) return set_err(h, VGPU_ERR_OOM, "cudaMalloc failed for the external-field buffers");
      }
   }
   *staged_out = staged;
   return VGPU_OK;
}

// one fused pass over the updated atoms 32 first_slice .. end - 1 (end < 0:
// all updated atoms); the corrector whose range ends at the last updated atom
// completes the step (counter, dipole cadence)
template <typename R>
static int run_pass(vgpu_ctx* h, int mode, bool staged, int integrator = INTEG_HEUN, int first_slice = 0,
                    int end = -1) {
   LLGArgs<R> a = make_args<R>(h);
   a.integrator = integrator;
   a.slice_first = first_slice;
   if (end >= 0) a.n_upd = end;
   if (staged && !h->sys.stage.win) {
      a.gx = (R*)h->sys.g_store[0]; a.gy = (R*)h->sys.g_store[1]; a.gz = (R*)h->sys.g_store[2];
   }
   const int kind = mode == PASS_PREDICTOR ? PROF_PREDICTOR : PROF_CORRECTOR;
   h->prof_begin(kind);
   cudaError_t e = launch_step_pass<R>(h, a, mode, staged);
   h->prof_end(kind);
   if (e != cudaSuccess) return cuda_err(h, e, "llg_heun launch");
   h->kernel_launches += 1;
   if (mode == PASS_PREDICTOR || a.n_upd != h->sys.n_owned) return VGPU_OK;
   h->step++;
   return h->after_step();
}

template <typename R>
static int llg_steps_typed(vgpu_ctx* h, uint64_t n_steps, int integrator = INTEG_HEUN) {
   bool staged = false;
   int rc = prepare_passes<R>(h, &staged, integrator);
   for (uint64_t t = 0; t < n_steps && !rc; ++t) {
      rc = h->fields_ready();
      if (!rc) rc = run_pass<R>(h, PASS_PREDICTOR, staged, integrator);
      if (!rc) rc = run_pass<R>(h, PASS_CORRECTOR, staged, integrator);
   }
   return rc;
}

template <typename R>
static int llg_pass_typed(vgpu_ctx* h, int mode) {
   bool staged = false;
   int rc = h->fields_ready();
   if (!rc) rc = prepare_passes<R>(h, &staged);
   return rc ? rc : run_pass<R>(h, mode, staged);
}

// halo transfers of a shard (device buffers of the caller, handle precision)
template <typename R>
__global__ void halo_pack_kernel(const R* __restrict__ x, const R* __restrict__ y, const R* __restrict__ z,
                                 const int* __restrict__ idx, int count, int n, R* __restrict__ out) {
   const int k = blockIdx.x * blockDim.x + threadIdx.x;
   if (k >= count) return;
   const int i = idx[k];
   const bool ok = i >= 0 && i < n;  // out-of-range indices send zeros
   out[k] = ok ? x[i] : (R)0;
   out[count + k] = ok ? y[i] : (R)0;
   out[2 * count + k] = ok ? z[i] : (R)0;
}

template <typename R>
__global__ void halo_unpack_kernel(R* __restrict__ x, R* __restrict__ y, R* __restrict__ z, int first, int count,
                                   const R* __restrict__ in) {
   const int k = blockIdx.x * blockDim.x + threadIdx.x;
   if (k >= count) return;
   x[first + k] = in[k];
   y[first + k] = in[count + k];
   z[first + k] = in[2 * count + k];
}

}  // namespace vgpu

int vgpu_ctx::check_status() {
   if (!sys.uploaded) return VGPU_OK;
   int st = 0;
   int rc = cuda_err(this, cudaMemcpyAsync(&st, sys.status, sizeof(int), cudaMemcpyDeviceToHost, stream), "status read");
   if (rc) return rc;
   rc = cuda_err(this, cudaStreamSynchronize(stream), "synchronize");
   if (rc) return rc;
   if (st == 0) return VGPU_OK;
   // report once: clear the word so that the context stays usable
   rc = cuda_err(this, cudaMemsetAsync(sys.status, 0, sizeof(int), stream), "status reset");
   if (rc) return rc;
   if (st & 1) return set_err(this, VGPU_ERR_NAN, "non-finite or non-normalisable spin produced by the integrator");
   if (st & 2) return set_err(this, VGPU_ERR_TIMEOUT, "a bond-record copy into shared memory did not complete in time");
   return VGPU_OK;
}
namespace vgpu {

}  // namespace vgpu

void vgpu_ctx::update_sigma_flag() {
   any_sigma = false;
   if (!params.thermal_enabled) return;
   for (const vgpu_material& q : sys.materials) {
      const double T = params.local_temperature ? q.temperature : params.temperature;
      if (T > 0.0 && q.H_th_sigma != 0.0) any_sigma = true;
   }
}
namespace vgpu {

}  // namespace vgpu

// ===========================================================================
// exported C ABI
// ===========================================================================
extern "C" const char* vgpu_version(void) { return "vgpu 0.1 sm_100a"; }

extern "C" int vgpu_last_error(vgpu_handle h, char* buf, size_t n) {
   if (!buf || n == 0) return VGPU_ERR_ARG;
   std::string s;
   if (h) s = h->err;
   else {
      std::lock_guard<std::mutex> g(g_err_mutex);
      s = g_global_err;
   }
   snprintf(buf, n, "%s", s.c_str());
   return VGPU_OK;
}

extern "C" int vgpu_create(int device, int precision, vgpu_handle* out) {
   if (!out) return set_err(nullptr, VGPU_ERR_ARG, "null output handle");
   *out = nullptr;
   if (precision != VGPU_PREC_FP32 && precision != VGPU_PREC_FP64)
      return set_err(nullptr, VGPU_ERR_ARG, "unknown precision %d", precision);
   int count = 0;
   cudaError_t e = cudaGetDeviceCount(&count);
   if (e != cudaSuccess || count == 0) {
      cudaGetLastError();
      return set_err(nullptr, VGPU_ERR_CUDA, "no CUDA device available: %s", cudaGetErrorString(e));
   }
   if (device < 0) {
      e = cudaGetDevice(&device);
      if (e != cudaSuccess) return cuda_err(nullptr, e, "cudaGetDevice");
   }
   if (device >= count) return set_err(nullptr, VGPU_ERR_ARG, "device %d out of range (%d devices)", device, count);
   if ((e = cudaSetDevice(device)) != cudaSuccess) return cuda_err(nullptr, e, "cudaSetDevice");
   vgpu_ctx* h = new vgpu_ctx();
   h->device = device;
   h->prec = precision;
   if ((e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking)) != cudaSuccess) {
      delete h;
      return cuda_err(nullptr, e, "cudaStreamCreate");
   }
   memset(&h->params, 0, sizeof h->params);
   h->params.H_vec[2] = 1.0;
   h->params.applied_enabled = 1;
   h->params.thermal_enabled = 1;
   *out = h;
   return VGPU_OK;
}

extern "C" int vgpu_destroy(vgpu_handle h) {
   if (!h) return VGPU_OK;
   cudaSetDevice(h->device);
   cudaStreamSynchronize(h->stream);
   h->destroy_extras();
   h->free_system();
   cudaStreamDestroy(h->stream);
   delete h;
   return VGPU_OK;
}

extern "C" int vgpu_upload_system(vgpu_handle h, const vgpu_system_desc* d) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   cudaSetDevice(h->device);
   int rc = validate(h, d);
   if (rc) return rc;
   h->destroy_extras();
   rc = h->prec == VGPU_PREC_FP64 ? upload_typed<double>(h, d) : upload_typed<float>(h, d);
   if (rc) return rc;
   h->update_sigma_flag();
   return cuda_err(h, cudaStreamSynchronize(h->stream), "upload synchronize");
}

extern "C" int vgpu_validate_system(const vgpu_system_desc* d) { return validate(nullptr, d); }

extern "C" int vgpu_set_params(vgpu_handle h, const vgpu_sim_params* p) {
   if (!h || !p) return set_err(h, VGPU_ERR_ARG, "null argument");
   if (!(p->dt > 0.0) || !std::isfinite(p->dt)) return set_err(h, VGPU_ERR_ARG, "dt must be positive and finite");
   if (!(p->temperature >= 0.0)) return set_err(h, VGPU_ERR_ARG, "temperature must be >= 0");
   cudaSetDevice(h->device);
   h->params = *p;
   h->update_sigma_flag();
   return h->refresh_materials();
}

// host FP64 <-> device state: the caller's doubles are copied as they are
// (a DMA straight from the caller's buffer when it is pinned) and converted on
// the device, so no host-side conversion loop sits on the transfer path.
__global__ void f64_to_state_kernel(const double* __restrict__ in, float* __restrict__ out, int n) {
   for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = (float)in[i];
}
__global__ void state_to_f64_kernel(const float* __restrict__ in, double* __restrict__ out, int n) {
   for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) out[i] = (double)in[i];
}

static int convert_grid(int n) { return std::max(1, std::min((n + 255) / 256, 148 * 8)); }

// device FP64 staging for host transfers of the FP32 state (3n doubles, once)
static double* host_stage(vgpu_ctx* h) {
   if (!h->sys.stage64) h->sys.stage64 = (double*)h->alloc(3 * (size_t)h->sys.n * sizeof(double));
   return h->sys.stage64;
}

template <typename R>
static int set_spins_typed(vgpu_handle h, const double* sx, const double* sy, const double* sz) {
   const int n = h->sys.n;
   const double* src[3] = {sx, sy, sz};
   if (sizeof(R) == 8) {
      for (int q = 0; q < 3; ++q) {
         int rc = cuda_err(h, cudaMemcpyAsync(h->sys.s[q], src[q], n * sizeof(double), cudaMemcpyHostToDevice,
                                              h->stream), "set spins");
         if (rc) return rc;
      }
   } else {
      double* st = host_stage(h);
      if (!st) return set_err(h, VGPU_ERR_OOM, "cudaMalloc failed for transfer staging");
      for (int q = 0; q < 3; ++q) {
         int rc = cuda_err(h, cudaMemcpyAsync(st + (size_t)q * n, src[q], n * sizeof(double), cudaMemcpyHostToDevice,
                                              h->stream), "set spins");
         if (rc) return rc;
         f64_to_state_kernel<<<convert_grid(n), 256, 0, h->stream>>>(st + (size_t)q * n, (float*)h->sys.s[q], n);
         h->kernel_launches++;
      }
      int rc = cuda_err(h, cudaGetLastError(), "set spins convert");
      if (rc) return rc;
   }
   return cuda_err(h, cudaStreamSynchronize(h->stream), "set spins");
}

extern "C" int vgpu_set_spins(vgpu_handle h, const double* sx, const double* sy, const double* sz) {
   if (!h || !sx || !sy || !sz) return set_err(h, VGPU_ERR_ARG, "null argument");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   cudaSetDevice(h->device);
   return h->prec == VGPU_PREC_FP64 ? set_spins_typed<double>(h, sx, sy, sz) : set_spins_typed<float>(h, sx, sy, sz);
}

template <typename R>
static int get_vec_typed(vgpu_handle h, void* const src[3], double* out[3]) {
   const int n = h->sys.n;
   if (sizeof(R) == 8) {
      for (int q = 0; q < 3; ++q) {
         int rc = cuda_err(h, cudaMemcpyAsync(out[q], src[q], n * sizeof(double), cudaMemcpyDeviceToHost, h->stream),
                           "download");
         if (rc) return rc;
      }
   } else {
      double* st = host_stage(h);
      if (!st) return set_err(h, VGPU_ERR_OOM, "cudaMalloc failed for transfer staging");
      for (int q = 0; q < 3; ++q) {
         state_to_f64_kernel<<<convert_grid(n), 256, 0, h->stream>>>((const float*)src[q], st + (size_t)q * n, n);
         h->kernel_launches++;
         int rc = cuda_err(h, cudaMemcpyAsync(out[q], st + (size_t)q * n, n * sizeof(double), cudaMemcpyDeviceToHost,
                                              h->stream), "download");
         if (rc) return rc;
      }
   }
   return cuda_err(h, cudaStreamSynchronize(h->stream), "download");
}

extern "C" int vgpu_get_spins(vgpu_handle h, double* sx, double* sy, double* sz) {
   if (!h || !sx || !sy || !sz) return set_err(h, VGPU_ERR_ARG, "null argument");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   cudaSetDevice(h->device);
   double* out[3] = {sx, sy, sz};
   int rc = h->prec == VGPU_PREC_FP64 ? get_vec_typed<double>(h, h->sys.s, out) : get_vec_typed<float>(h, h->sys.s, out);
   if (rc) return rc;
   return h->check_status();
}

extern "C" int vgpu_set_noise(vgpu_handle h, int mode, uint64_t seed) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   if (mode != VGPU_NOISE_PHILOX && mode != VGPU_NOISE_REPLAY) return set_err(h, VGPU_ERR_ARG, "unknown noise mode %d", mode);
   if (mode == VGPU_NOISE_REPLAY && !h->sys.xi)
      return set_err(h, VGPU_ERR_STATE, "replay mode needs vgpu_set_noise_replay first");
   h->noise_mode = mode;
   h->seed = seed;
   return VGPU_OK;
}

template <typename R>
static int set_replay_typed(vgpu_handle h, const double* xi) {
   const size_t m = 3 * (size_t)h->sys.n;
   if (!h->sys.xi) {
      h->sys.xi = h->alloc(m * sizeof(R));
      if (!h->sys.xi) return set_err(h, VGPU_ERR_OOM, "cudaMalloc failed for replay noise");
   }
   std::vector<R> buf(xi, xi + m);
   int rc = cuda_err(h, cudaMemcpyAsync(h->sys.xi, buf.data(), m * sizeof(R), cudaMemcpyHostToDevice, h->stream), "replay");
   if (rc) return rc;
   return cuda_err(h, cudaStreamSynchronize(h->stream), "replay");
}

extern "C" int vgpu_set_noise_replay(vgpu_handle h, const double* xi) {
   if (!h || !xi) return set_err(h, VGPU_ERR_ARG, "null argument");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   cudaSetDevice(h->device);
   int rc = h->prec == VGPU_PREC_FP64 ? set_replay_typed<double>(h, xi) : set_replay_typed<float>(h, xi);
   if (rc) return rc;
   h->noise_mode = VGPU_NOISE_REPLAY;
   return VGPU_OK;
}

template <typename R>
static int upload_biquadratic(vgpu_handle h, const vgpu_biquadratic_desc* b) {
   SysDev& S = h->sys;
   const int n = S.n, nsl = S.nslices, pad = S.n_alloc - 1;
   std::vector<int> off(nsl + 1, 0);
   for (int sl = 0; sl < nsl; ++sl) {
      int w = 0;
      for (int l = 0; l < 32 && sl * 32 + l < n; ++l) w = std::max(w, b->nl_end[sl * 32 + l] - b->nl_start[sl * 32 + l] + 1);
      off[sl + 1] = off[sl] + 32 * w;
   }
   const size_t ne = (size_t)off[nsl];
   std::vector<int> col(std::max<size_t>(ne, 1), pad);
   std::vector<R> j(std::max<size_t>(ne, 1), (R)0);
   for (int i = 0; i < n; ++i) {
      int k = 0;
      for (int32_t e = b->nl_start[i]; e <= b->nl_end[i]; ++e, ++k) {
         const size_t q = (size_t)off[i >> 5] + 32 * (size_t)k + (i & 31);
         col[q] = b->nl[e];
         j[q] = (R)b->jlist[b->nl_type ? b->nl_type[e] : e];
      }
   }
   int rc;
   if ((rc = upload_vec(h, &S.bq_off, off, "biquadratic slice offsets"))) return rc;
   if ((rc = upload_vec(h, &S.bq_col, col, "biquadratic neighbours"))) return rc;
   if ((rc = upload_vec(h, &S.bq_j, j, "biquadratic couplings"))) return rc;
   return cuda_err(h, cudaStreamSynchronize(h->stream), "biquadratic upload");
}

extern "C" int vgpu_set_biquadratic(vgpu_handle h, const vgpu_biquadratic_desc* b) {
   if (!h || !b) return set_err(h, VGPU_ERR_ARG, "null argument");
   SysDev& S = h->sys;
   if (!S.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   if (S.sys_off) return set_err(h, VGPU_ERR_STATE, "batched systems carry no biquadratic exchange");
   if (S.n_owned < S.n) return set_err(h, VGPU_ERR_STATE, "shards carry no biquadratic exchange list");
   if (S.bq_off) return set_err(h, VGPU_ERR_STATE, "biquadratic exchange already set (upload the system again)");
   if (!b->nl_start || !b->nl_end || (b->num_bonds > 0 && (!b->nl || !b->jlist)))
      return set_err(h, VGPU_ERR_ARG, "incomplete biquadratic descriptor");
   for (int i = 0; i < S.n; ++i) {
      if (b->nl_end[i] < b->nl_start[i] - 1 || b->nl_start[i] < 0 || (int64_t)b->nl_end[i] >= b->num_bonds)
         return set_err(h, VGPU_ERR_ARG, "biquadratic row %d out of range", i);
      for (int32_t e = b->nl_start[i]; e <= b->nl_end[i]; ++e) {
         if (b->nl[e] < 0 || b->nl[e] >= S.n) return set_err(h, VGPU_ERR_ARG, "biquadratic neighbour out of range");
         const int64_t t = b->nl_type ? b->nl_type[e] : e;
         if (t < 0 || t >= b->num_exchange) return set_err(h, VGPU_ERR_ARG, "biquadratic interaction id out of range");
      }
   }
   cudaSetDevice(h->device);
   return h->prec == VGPU_PREC_FP64 ? upload_biquadratic<double>(h, b) : upload_biquadratic<float>(h, b);
}

template <typename R>
static int upload_neel(vgpu_handle h, const double* t) {
   SysDev& S = h->sys;
   const size_t na = (size_t)S.n_alloc;
   std::vector<R> buf(9 * na, (R)0);  // [component][atom], pad rows zero
   for (int i = 0; i < S.n; ++i)
      for (int k = 0; k < 9; ++k) buf[k * na + i] = (R)t[9 * (size_t)i + k];
   if (!S.neel) {
      S.neel = h->alloc(buf.size() * sizeof(R));
      if (!S.neel) return set_err(h, VGPU_ERR_OOM, "cudaMalloc failed for Neel tensors");
   }
   int rc = cuda_err(h, cudaMemcpyAsync(S.neel, buf.data(), buf.size() * sizeof(R), cudaMemcpyHostToDevice, h->stream),
                     "Neel tensors");
   if (rc) return rc;
   return cuda_err(h, cudaStreamSynchronize(h->stream), "Neel tensors");
}

extern "C" int vgpu_set_anisotropy_ext(vgpu_handle h, const vgpu_anisotropy_ext* x) {
   if (!h || !x) return set_err(h, VGPU_ERR_ARG, "null argument");
   SysDev& S = h->sys;
   if (!S.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   if (S.sys_off) return set_err(h, VGPU_ERR_STATE, "batched systems carry second-order uniaxial and cubic anisotropy only");
   const int M = S.M;
   if ((x->uniaxial_fourth && !x->ku4) || (x->uniaxial_sixth && !x->ku6) || (x->cubic_sixth && !x->kc6) ||
       (x->cubic_rotation && !x->kc_basis) || (x->neel && !x->neel_tensor))
      return set_err(h, VGPU_ERR_ARG, "an enabled anisotropy term has no data");
   auto finite = [](const double* v, size_t k) {
      for (size_t q = 0; q < k; ++q)
         if (!std::isfinite(v[q])) return false;
      return true;
   };
   if ((x->uniaxial_fourth && !finite(x->ku4, M)) || (x->uniaxial_sixth && !finite(x->ku6, M)) ||
       (x->cubic_sixth && !finite(x->kc6, M)) || (x->cubic_rotation && !finite(x->kc_basis, 9 * (size_t)M)) ||
       (x->neel && !finite(x->neel_tensor, 9 * (size_t)S.n)))
      return set_err(h, VGPU_ERR_ARG, "non-finite anisotropy constant");
   if (x->cubic_rotation && S.cubic)
      return set_err(h, VGPU_ERR_ARG, "rotated cubic anisotropy replaces the plain cubic term (cubic_enabled = 0)");
   cudaSetDevice(h->device);
   int bits = 0;
   S.ku4_h.assign(x->uniaxial_fourth ? x->ku4 : nullptr, x->uniaxial_fourth ? x->ku4 + M : nullptr);
   S.ku6_h.assign(x->uniaxial_sixth ? x->ku6 : nullptr, x->uniaxial_sixth ? x->ku6 + M : nullptr);
   S.kc6_h.assign(x->cubic_sixth ? x->kc6 : nullptr, x->cubic_sixth ? x->kc6 + M : nullptr);
   S.kcb_h.assign(x->cubic_rotation ? x->kc_basis : nullptr, x->cubic_rotation ? x->kc_basis + 9 * (size_t)M : nullptr);
   if (x->uniaxial_fourth) bits |= ANI_U4;
   if (x->uniaxial_sixth) bits |= ANI_U6;
   if (x->cubic_sixth) bits |= ANI_C6;
   if (x->cubic_rotation) bits |= ANI_CROT;
   if (x->neel) {
      int rc = h->prec == VGPU_PREC_FP64 ? upload_neel<double>(h, x->neel_tensor) : upload_neel<float>(h, x->neel_tensor);
      if (rc) return rc;
      bits |= ANI_NEEL;
   }
   S.aniso_ext = bits;
   return h->refresh_materials();
}

extern "C" int vgpu_set_option(vgpu_handle h, int option, int value) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   switch (option) {
      case VGPU_OPT_STORE_INCREMENT: h->store_increment = value; return VGPU_OK;
      case VGPU_OPT_STAGED_RECORDS:
         if (value < -1 || value > 1) return set_err(h, VGPU_ERR_ARG, "staged records: -1, 0 or 1");
         h->staged = value;
         h->sys.stage.grid = 0;
         return VGPU_OK;
      case VGPU_OPT_STAGE_SLICES:
         if (value != -1 && value != 2 && value != 4 && value != 8)
            return set_err(h, VGPU_ERR_ARG, "stage slices: -1, 2, 4 or 8");
         h->stage_sl = value;
         h->sys.stage.grid = 0;
         return VGPU_OK;
      case VGPU_OPT_STAGE_WAIT_TEST:
         h->stage_wait_test = value != 0;
         return VGPU_OK;
      case VGPU_OPT_DIPOLE_FFT:
         if (value < -1 || value > 1) return set_err(h, VGPU_ERR_ARG, "dipole FFT: -1, 0 or 1");
         h->dipole_fft = value;
         return VGPU_OK;
      case VGPU_OPT_STAGE_BUFFERS:
         if (value != -1 && value != 1 && value != 2) return set_err(h, VGPU_ERR_ARG, "stage buffers: -1, 1 or 2");
         h->stage_nbuf = value;
         h->sys.stage.grid = 0;
         return VGPU_OK;
      case VGPU_OPT_COMPACT_RECORDS:
         if (value < -1 || value > 1) return set_err(h, VGPU_ERR_ARG, "compact records: -1, 0 or 1");
         h->compact = value;
         h->sys.stage.grid = 0;
         return VGPU_OK;
      case VGPU_OPT_WINDOW_STAGING:
         if (value < -1 || value > 1) return set_err(h, VGPU_ERR_ARG, "window staging: -1, 0 or 1");
         h->window = value;
         h->sys.stage.grid = 0;
         return VGPU_OK;
      case VGPU_OPT_STAGE_WARPS:
         if (value != -1 && value != 0 && value != 2 && value != 4)
            return set_err(h, VGPU_ERR_ARG, "stage warps: -1, 0, 2 or 4");
         h->stage_warps = value;
         h->sys.stage.grid = 0;
         return VGPU_OK;
      case VGPU_OPT_PROFILE_EVERY:
         if (value < 1) return set_err(h, VGPU_ERR_ARG, "profile stride must be >= 1");
         h->prof_every = value;
         return VGPU_OK;
      default: return set_err(h, VGPU_ERR_ARG, "unknown option %d", option);
   }
}

extern "C" int vgpu_record_layout(vgpu_handle h, int32_t* layout, int32_t* dict_entries) {
   if (!h || !layout) return set_err(h, VGPU_ERR_ARG, "null argument");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   SysDev& S = h->sys;
   if (dict_entries) *dict_entries = S.cdict_n;
   const bool compact = h->compact != 0 && S.crec;
   *layout = compact ? VGPU_RECORDS_COMPACT : S.rec ? VGPU_RECORDS_WIDE : VGPU_RECORDS_NONE;
   if (compact && h->prec == VGPU_PREC_FP32 && use_staged<float>(h)) {
      const int rc = ensure_window_plan(h);
      if (rc) return rc;
      if (S.win_ok) *layout = VGPU_RECORDS_WINDOW;
   }
   return VGPU_OK;
}

extern "C" int vgpu_exchange_format(vgpu_handle h, int32_t* fmt) {
   if (!h || !fmt) return set_err(h, VGPU_ERR_ARG, "null argument");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   static_assert(FMT_ISO_TAB == VGPU_EXCH_ISO_TAB && FMT_ISO_BOND == VGPU_EXCH_ISO_BOND &&
                     FMT_VEC_TAB == VGPU_EXCH_VEC_TAB && FMT_VEC_BOND == VGPU_EXCH_VEC_BOND &&
                     FMT_DMI_TAB == VGPU_EXCH_DMI_TAB && FMT_TENSOR_BOND == VGPU_EXCH_TENSOR_BOND,
                 "exchange format numbering");
   *fmt = h->sys.fmt;
   return VGPU_OK;
}

extern "C" int vgpu_set_step(vgpu_handle h, uint64_t step) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   h->step = step;
   return VGPU_OK;
}

extern "C" int vgpu_get_step(vgpu_handle h, uint64_t* step) {
   if (!h || !step) return set_err(h, VGPU_ERR_ARG, "null argument");
   *step = h->step;
   return VGPU_OK;
}

extern "C" int vgpu_llg_heun(vgpu_handle h, uint64_t n_steps) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   if (!(h->params.dt > 0.0)) return set_err(h, VGPU_ERR_STATE, "vgpu_set_params not called");
   cudaSetDevice(h->device);
   return h->prec == VGPU_PREC_FP64 ? llg_steps_typed<double>(h, n_steps) : llg_steps_typed<float>(h, n_steps);
}

template <typename R>
static int fields_typed(vgpu_handle h, double* hx, double* hy, double* hz) {
   SysDev& S = h->sys;
   if (!S.f[0]) {
      for (int q = 0; q < 3; ++q) {
         S.f[q] = h->alloc(S.n_alloc * sizeof(R));
         if (!S.f[q]) return set_err(h, VGPU_ERR_OOM, "cudaMalloc failed for field buffer");
      }
   }
   LLGArgs<R> a = make_args<R>(h);
   cudaError_t e = launch_llg_pass<R>(a, S.fmt, PASS_FIELD, S.nslices, h->stream);
   if (e != cudaSuccess) return cuda_err(h, e, "field launch");
   double* out[3] = {hx, hy, hz};
   return get_vec_typed<R>(h, S.f, out);
}

extern "C" int vgpu_get_fields(vgpu_handle h, double* hx, double* hy, double* hz) {
   if (!h || !hx || !hy || !hz) return set_err(h, VGPU_ERR_ARG, "null argument");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   if (int rc = h->fields_ready()) return rc;
   cudaSetDevice(h->device);
   return h->prec == VGPU_PREC_FP64 ? fields_typed<double>(h, hx, hy, hz) : fields_typed<float>(h, hx, hy, hz);
}


template <typename R>
static int noise_typed(vgpu_handle h, uint64_t step, double* xi) {
   SysDev& S = h->sys;
   if (!S.f[0]) {
      for (int q = 0; q < 3; ++q) {
         S.f[q] = h->alloc(S.n_alloc * sizeof(R));
         if (!S.f[q]) return set_err(h, VGPU_ERR_OOM, "cudaMalloc failed for field buffer");
      }
   }
   LLGArgs<R> a = make_args<R>(h);
   a.step = step;
   a.noise_mode = VGPU_NOISE_PHILOX;
   cudaError_t e = launch_thermal_noise<R>(a, h->stream);
   if (e != cudaSuccess) return cuda_err(h, e, "noise launch");
   const int n = S.n;
   double* out[3] = {xi, xi + n, xi + 2 * (size_t)n};
   return get_vec_typed<R>(h, S.f, out);
}

extern "C" int vgpu_llg_midpoint(vgpu_handle h, uint64_t n_steps) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   if (!(h->params.dt > 0.0)) return set_err(h, VGPU_ERR_STATE, "vgpu_set_params not called");
   cudaSetDevice(h->device);
   return h->prec == VGPU_PREC_FP64 ? llg_steps_typed<double>(h, n_steps, INTEG_MIDPOINT)
                                    : llg_steps_typed<float>(h, n_steps, INTEG_MIDPOINT);
}

extern "C" int vgpu_llg_pass(vgpu_handle h, int pass) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   if (!(h->params.dt > 0.0)) return set_err(h, VGPU_ERR_STATE, "vgpu_set_params not called");
   if (pass != VGPU_PASS_PREDICTOR && pass != VGPU_PASS_CORRECTOR) return set_err(h, VGPU_ERR_ARG, "unknown pass %d", pass);
   cudaSetDevice(h->device);
   const int mode = pass == VGPU_PASS_PREDICTOR ? PASS_PREDICTOR : PASS_CORRECTOR;
   return h->prec == VGPU_PREC_FP64 ? llg_pass_typed<double>(h, mode) : llg_pass_typed<float>(h, mode);
}

template <typename R>
static int llg_pass_range_typed(vgpu_ctx* h, int mode, int first, int end) {
   bool staged = false;
   int rc = h->fields_ready();
   if (!rc) rc = prepare_passes<R>(h, &staged);
   if (!rc && staged && h->sys.stage.win && first != 0)
      return set_err(h, VGPU_ERR_STATE, "window-staged passes run whole shards only");
   return rc ? rc : run_pass<R>(h, mode, staged, INTEG_HEUN, first / 32, end);
}

extern "C" int vgpu_llg_pass_range(vgpu_handle h, int pass, int32_t first_atom, int32_t end_atom) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   if (!(h->params.dt > 0.0)) return set_err(h, VGPU_ERR_STATE, "vgpu_set_params not called");
   if (pass != VGPU_PASS_PREDICTOR && pass != VGPU_PASS_CORRECTOR) return set_err(h, VGPU_ERR_ARG, "unknown pass %d", pass);
   if (first_atom < 0 || first_atom % 32 != 0 || end_atom < first_atom || end_atom > h->sys.n_owned)
      return set_err(h, VGPU_ERR_ARG, "range %d..%d: the first atom must be a multiple of 32 and the end at most %d",
                     first_atom, end_atom, h->sys.n_owned);
   if (first_atom == end_atom) return VGPU_OK;
   cudaSetDevice(h->device);
   const int mode = pass == VGPU_PASS_PREDICTOR ? PASS_PREDICTOR : PASS_CORRECTOR;
   return h->prec == VGPU_PREC_FP64 ? llg_pass_range_typed<double>(h, mode, first_atom, end_atom)
                                    : llg_pass_range_typed<float>(h, mode, first_atom, end_atom);
}

extern "C" int vgpu_set_owned(vgpu_handle h, int32_t n_owned, int64_t noise_base) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   SysDev& S = h->sys;
   if (!S.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   if (n_owned < 0 || n_owned > S.n) return set_err(h, VGPU_ERR_ARG, "n_owned %d outside 0..%d", n_owned, S.n);
   if (noise_base < 0 || noise_base + (int64_t)n_owned > ((int64_t)1 << 32))
      return set_err(h, VGPU_ERR_ARG, "noise_base out of the 32-bit atom counter range");
   if (n_owned < S.n && S.bq_off)
      return set_err(h, VGPU_ERR_STATE, "shards carry no biquadratic exchange list");
   if (h->extras[2] && n_owned != S.n_owned)
      return set_err(h, VGPU_ERR_STATE, "the dipole solver is set up: call vgpu_set_owned before vgpu_dipole_setup_shard");
   if (h->extras[1] && n_owned != S.n_owned)
      return set_err(h, VGPU_ERR_STATE, "Monte Carlo colour lists are set up: call vgpu_set_owned before vgpu_mc_setup");
   S.n_owned = n_owned;
   S.noise_base = (uint32_t)noise_base;
   S.stage.grid = 0;
   return VGPU_OK;
}

template <typename R>
static int halo_typed(vgpu_handle h, int which, const int32_t* idx, int32_t first, int32_t count, void* buf,
                      bool pack, cudaStream_t stream = nullptr) {
   SysDev& S = h->sys;
   void* const* st = which == VGPU_STATE_SPIN ? S.s : S.p;
   if (count == 0) return VGPU_OK;
   const int grid = (count + 255) / 256;
   cudaStream_t on = stream ? stream : h->stream;
   if (pack)
      halo_pack_kernel<R><<<grid, 256, 0, on>>>((const R*)st[0], (const R*)st[1], (const R*)st[2], idx, count,
                                                S.n, (R*)buf);
   else
      halo_unpack_kernel<R><<<grid, 256, 0, on>>>((R*)st[0], (R*)st[1], (R*)st[2], first, count,
                                                         (const R*)buf);
   h->kernel_launches++;
   return cuda_err(h, cudaGetLastError(), pack ? "halo pack" : "halo unpack");
}

extern "C" int vgpu_halo_pack(vgpu_handle h, int which, const int32_t* idx, int32_t count, void* out) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   if (which != VGPU_STATE_SPIN && which != VGPU_STATE_PREDICTOR) return set_err(h, VGPU_ERR_ARG, "unknown state");
   if (count < 0 || (count > 0 && (!idx || !out))) return set_err(h, VGPU_ERR_ARG, "bad halo buffer");
   cudaSetDevice(h->device);
   return h->prec == VGPU_PREC_FP64 ? halo_typed<double>(h, which, idx, 0, count, out, true)
                                    : halo_typed<float>(h, which, idx, 0, count, out, true);
}

extern "C" int vgpu_halo_unpack(vgpu_handle h, int which, int32_t first, int32_t count, const void* in) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   if (which != VGPU_STATE_SPIN && which != VGPU_STATE_PREDICTOR) return set_err(h, VGPU_ERR_ARG, "unknown state");
   if (count < 0 || first < 0 || (int64_t)first + count > h->sys.n || (count > 0 && !in))
      return set_err(h, VGPU_ERR_ARG, "halo block %d..%d outside the system", first, first + count);
   cudaSetDevice(h->device);
   return h->prec == VGPU_PREC_FP64 ? halo_typed<double>(h, which, nullptr, first, count, const_cast<void*>(in), false)
                                    : halo_typed<float>(h, which, nullptr, first, count, const_cast<void*>(in), false);
}

extern "C" int vgpu_halo_pack_on(vgpu_handle h, int which, const int32_t* idx, int32_t count, void* out,
                                 void* stream) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   if (which != VGPU_STATE_SPIN && which != VGPU_STATE_PREDICTOR) return set_err(h, VGPU_ERR_ARG, "unknown state");
   if (count < 0 || (count > 0 && (!idx || !out))) return set_err(h, VGPU_ERR_ARG, "bad halo buffer");
   cudaSetDevice(h->device);
   return h->prec == VGPU_PREC_FP64 ? halo_typed<double>(h, which, idx, 0, count, out, true, (cudaStream_t)stream)
                                    : halo_typed<float>(h, which, idx, 0, count, out, true, (cudaStream_t)stream);
}

extern "C" int vgpu_halo_unpack_on(vgpu_handle h, int which, int32_t first, int32_t count, const void* in,
                                   void* stream) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   if (which != VGPU_STATE_SPIN && which != VGPU_STATE_PREDICTOR) return set_err(h, VGPU_ERR_ARG, "unknown state");
   if (count < 0 || first < 0 || (int64_t)first + count > h->sys.n || (count > 0 && !in))
      return set_err(h, VGPU_ERR_ARG, "halo block %d..%d outside the system", first, first + count);
   cudaSetDevice(h->device);
   return h->prec == VGPU_PREC_FP64
              ? halo_typed<double>(h, which, nullptr, first, count, const_cast<void*>(in), false, (cudaStream_t)stream)
              : halo_typed<float>(h, which, nullptr, first, count, const_cast<void*>(in), false, (cudaStream_t)stream);
}

extern "C" int vgpu_thermal_noise(vgpu_handle h, uint64_t step, double* xi) {
   if (!h || !xi) return set_err(h, VGPU_ERR_ARG, "null argument");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   cudaSetDevice(h->device);
   return h->prec == VGPU_PREC_FP64 ? noise_typed<double>(h, step, xi) : noise_typed<float>(h, step, xi);
}
