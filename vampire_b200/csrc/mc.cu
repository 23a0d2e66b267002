// Checkerboard (multi-colour) Metropolis Monte Carlo sweep (K3).
//
// Reference: montecarlo::mc_step (src/montecarlo/mc.cpp:29-127) makes N
// random-site trials per step, each with mc_angle moves
// (src/montecarlo/mc_moves.cpp:71-87: s' = n(s + sigma xi)) and the
// single-spin energy of sim::calculate_spin_energy
// (src/simulate/energy.cpp:147-174), accepting if dE < 0 or
// exp(-dE mu_s/(kB T)) >= U.  That loop is inherently sequential.  Here the
// exchange graph is coloured on the host (greedy; simple-cubic periodic
// lattices with even sides come out bipartite, FCC nearest neighbours need
// four) and one launch updates every site of one colour at once: no two
// sites of a colour interact, so each site's exchange field is fixed while it
// is updated and detailed balance holds per colour.  A sweep visits every
// site exactly once (the reference visits N random sites with replacement);
// the two are compared statistically (m(T), Tc).
//
// Random numbers: one Philox draw, counter (atom, sweep_lo, sweep_hi,
// RNG_MC_MOVE), per FP32 trial: the top 24 bits of its four words give the
// three Gaussians of the move (Box-Muller, as everywhere in FP32), the low
// bytes of three of them the 24-bit acceptance uniform -- disjoint bits of
// independent uniform words, so independent uniforms.  FP64 takes the
// acceptance uniform from a second draw (.., RNG_MC_ACCEPT), all 32 bits of
// each word being used there.  In replay mode, 4 host-supplied numbers per
// site and sweep.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "llg_device.cuh"
#include "vgpu_ctx.cuh"

namespace vgpu {

struct MCState {
   int ncolours = 0;
   std::vector<int> colour_host;      // [n]
   std::vector<int> colour_off;       // [ncolours+1] offsets into the atom list
   int* atoms = nullptr;              // [n] atoms sorted by colour
   int4* entries = nullptr;           // [n] per list position: atom, first SELL entry, row width, material
   unsigned long long* rejects = nullptr;
   void* replay = nullptr;            // [4n] (x|y|z gaussians, uniform) in R
   bool use_replay = false;
   uint64_t sweep = 0;
   double moves = 0.0;
   int n_owned = 0;                   // atoms the sweeps visit (a shard's owned atoms)
   int next_colour = 0;               // vgpu_mc_colour: the colour of the current sweep to run next
};

static MCState* mc_of(vgpu_ctx* h) { return (MCState*)h->extras[1]; }

// What one trial needs of its material, in one aligned record (two 16-byte
// loads in FP32): move width, mu_B / (kB T_rescaled) (kBTBohr), mu_s_SI / mu_B,
// and the uniaxial and cubic constants of the single-spin energy.
template <typename R>
struct alignas(8 * sizeof(R)) MCMat {
   R sigma, beta, mu_ratio, ku2, kux, kuy, kuz, kc4;
};

template <typename R>
struct MCArgs {
   LLGArgs<R> a;
   const int4* entries;  // the colour's trials (list positions)
   int count;
   const MCMat<R>* mat;  // [M]
   const R* replay;      // [4n] or nullptr
   uint64_t sweep;
   unsigned long long* rejects;
};

// dE of atom i (material mi) for the move S -> T in the fixed exchange field
// h; P: any record with ku2, kux, kuy, kuz, kc4 (MatParams or MCMat)
template <typename R, typename P>
__device__ __forceinline__ R site_energy_delta(const LLGArgs<R>& a, int i, int mi, const P& m, const R S[3],
                                               const R T[3], const R h[3]) {
   // dE = E(T) - E(S) for the single-spin energy (exchange field h fixed)
   R d = -((T[0] - S[0]) * (h[0] + a.hx) + (T[1] - S[1]) * (h[1] + a.hy) + (T[2] - S[2]) * (h[2] + a.hz));
   if (a.uniaxial) {
      const R es = S[0] * m.kux + S[1] * m.kuy + S[2] * m.kuz;
      const R et = T[0] * m.kux + T[1] * m.kuy + T[2] * m.kuz;
      d += -m.ku2 * (et * et - es * es);
   }
   if (a.cubic) {
      const R s4 = S[0] * S[0] * S[0] * S[0] + S[1] * S[1] * S[1] * S[1] + S[2] * S[2] * S[2] * S[2];
      const R t4 = T[0] * T[0] * T[0] * T[0] + T[1] * T[1] * T[1] * T[1] + T[2] * T[2] * T[2] * T[2];
      d += (R)(-0.5) * m.kc4 * (t4 - s4);
   }
   if (a.aniso_ext) {
      const MatParams<R>& q = a.mp[mi];
      d += anisotropy_energy<R, R, true>(a, i, q, T) - anisotropy_energy<R, R, true>(a, i, q, S);
   }
   if (a.bq_off) d += biquadratic_energy<R, R>(a, i, T) - biquadratic_energy<R, R>(a, i, S);
   return d;
}

// The trial's list entry holds its atom, row and material, so the row's bond
// words, the own spin and the material record are all requested one load
// after the thread starts (the atom list, the slice offsets and the material
// id were three dependent loads before), and rows of width 6 or 12 (simple
// cubic, FCC) are read with every bond word and neighbour spin in flight at
// once.  Same arithmetic in the same bond order as the generic row loop.
// Blocks of 256, at least VGPU_MC_MIN_BLOCKS per SM: 4 (64 registers, no
// spills) measured fastest on SC 50^3 x 31 temperatures -- 2.905e10
// spin-moves/s against 2.853e10 with 5 (48 registers), 2.70e10 with 6 (40)
// and 2.56e10 with 7 or 8 (spilling); the sweep rate after 500 warm-up sweeps.
#ifndef VGPU_MC_MIN_BLOCKS
#define VGPU_MC_MIN_BLOCKS 4
#endif
template <typename R, int FMT>
__global__ void __launch_bounds__(256, VGPU_MC_MIN_BLOCKS) mc_colour_kernel(const MCArgs<R> p) {
   asm volatile("griddepcontrol.wait;" ::: "memory");  // launched by launch_pdl: the previous colour is done
   const int t = blockIdx.x * blockDim.x + threadIdx.x;
   bool rejected = false;
   if (t < p.count) {
      const LLGArgs<R>& a = p.a;
      const int4 en = __ldg(p.entries + t);
      const int i = en.x, base = en.y, w = en.z, mi = en.w;
      const MCMat<R> mm = p.mat[mi];
      R h[3] = {0, 0, 0};
      if (FMT == FMT_ISO_TAB && w == 6)
         exchange_gather_w<R, FMT, 6, 0, false>(a, base, mi, a.ax, a.ay, a.az, h[0], h[1], h[2], nullptr);
      else if (FMT == FMT_ISO_TAB && w == 12)
         exchange_gather_w<R, FMT, 12, 0, false>(a, base, mi, a.ax, a.ay, a.az, h[0], h[1], h[2], nullptr);
      else
         exchange_gather_row<R, FMT>(a, base, w, mi, a.ax, a.ay, a.az, h[0], h[1], h[2]);
      // magnetostatic energy uses the mu0 Hd field (energy.cpp:123-126)
      if (a.cell) {
         const int c = __ldg(a.cell + i);
         h[0] += __ldg(a.cell_hd + c);
         h[1] += __ldg(a.cell_hd + a.ncells + c);
         h[2] += __ldg(a.cell_hd + 2 * a.ncells + c);
      } else if (a.hm_atom) {
         h[0] += __ldg(a.hm_atom + i); h[1] += __ldg(a.hm_atom + a.n + i); h[2] += __ldg(a.hm_atom + 2 * a.n + i);
      }
      const R S[3] = {a.ax[i], a.ay[i], a.az[i]};
      R g0, g1, g2, u;
      if (p.replay) {
         g0 = p.replay[i]; g1 = p.replay[a.n + i]; g2 = p.replay[2 * a.n + i]; u = p.replay[3 * a.n + i];
      } else {
         // keyed by the global atom index (a shard's atom i is atom noise_base + i)
         const uint32_t gi = (uint32_t)i + a.noise_base;
         const u32x4 c = {gi, (uint32_t)p.sweep, (uint32_t)(p.sweep >> 32), RNG_MC_MOVE};
         const u32x4 r = philox4x32_10(c, a.seed_lo, a.seed_hi);
         if (sizeof(R) == 4) {
            // Box-Muller on the fast approximations (each Gaussian within 1e-5)
            float s1, c1;
            const float r1 = bm_radius_fast(r.x);
            bm_angle_fast(r.y, c1, s1);
            g0 = r1 * c1; g1 = r1 * s1; g2 = bm_radius_fast(r.z) * bm_cos_fast(r.w);
            // u01f keeps the top 24 bits: the low bytes of r.y, r.z, r.w
            u = (R)u01f(((r.y & 0xffu) << 8) | ((r.z & 0xffu) << 16) | (r.w << 24));
         } else {
            const u32x4 c2 = {gi, (uint32_t)p.sweep, (uint32_t)(p.sweep >> 32), RNG_MC_ACCEPT};
            const u32x4 r2 = philox4x32_10(c2, a.seed_lo, a.seed_hi);
            double s1, c1, s2, c2d;
            const double r1 = sqrt(-2.0 * log(u01d(r.x)));
            const double rr = sqrt(-2.0 * log(u01d(r.z)));
            sincospi(2.0 * u01d(r.y), &s1, &c1);
            sincospi(2.0 * u01d(r.w), &s2, &c2d);
            g0 = (R)(r1 * c1); g1 = (R)(r1 * s1); g2 = (R)(rr * c2d);
            u = (R)u01d(r2.x);
         }
      }
      const R sg = mm.sigma;
      R T[3] = {S[0] + g0 * sg, S[1] + g1 * sg, S[2] + g2 * sg};
      const R r = rsqrt_<R>(T[0] * T[0] + T[1] * T[1] + T[2] * T[2]);
      T[0] *= r; T[1] *= r; T[2] *= r;
      const R dE = site_energy_delta<R>(a, i, mi, mm, S, T, h) * mm.mu_ratio;
      bool accept = dE < (R)0;
      if (!accept) {
         const R x = -dE * mm.beta;
         accept = (sizeof(R) == 4 ? (R)expf((float)x) : (R)exp((double)x)) >= u;
      }
      if (accept) {
         a.ax[i] = T[0]; a.ay[i] = T[1]; a.az[i] = T[2];
      } else {
         rejected = true;
      }
   }
   const unsigned ballot = __ballot_sync(0xffffffffu, rejected);
   if ((threadIdx.x & 31) == 0 && ballot) atomicAdd(p.rejects, (unsigned long long)__popc(ballot));
}

// list entries of the colour-sorted atoms (rows from the slice offsets)
__global__ void mc_entries_kernel(const int* __restrict__ atoms, int count, const int* __restrict__ slice_off,
                                  const int* __restrict__ mat, int4* __restrict__ out) {
   const int t = blockIdx.x * blockDim.x + threadIdx.x;
   if (t >= count) return;
   const int i = atoms[t];
   const int off = slice_off[i >> 5];
   out[t] = make_int4(i, off + (i & 31), (slice_off[(i >> 5) + 1] - off) >> 5, mat ? mat[i] : 0);
}

template <typename R, int FMT>
static cudaError_t launch_mc(const MCArgs<R>& p, cudaStream_t st) {
   if (p.count == 0) return cudaSuccess;
   return launch_pdl(mc_colour_kernel<R, FMT>, dim3((p.count + 255) / 256), dim3(256), 0, st, p);
}

template <typename R>
static cudaError_t mc_dispatch(const MCArgs<R>& p, int fmt, cudaStream_t st) {
   switch (fmt) {
      case FMT_ISO_TAB: return launch_mc<R, FMT_ISO_TAB>(p, st);
      case FMT_ISO_BOND: return launch_mc<R, FMT_ISO_BOND>(p, st);
      case FMT_VEC_TAB: return launch_mc<R, FMT_VEC_TAB>(p, st);
      case FMT_VEC_BOND: return launch_mc<R, FMT_VEC_BOND>(p, st);
      case FMT_DMI_TAB: return launch_mc<R, FMT_DMI_TAB>(p, st);
      default: return launch_mc<R, FMT_TENSOR_BOND>(p, st);
   }
}

void cmc_destroy(vgpu_ctx* h);

void mc_destroy(vgpu_ctx* h) {
   MCState* s = mc_of(h);
   if (!s) return;
   cmc_destroy(h);  // its pairing follows this colouring
   cudaFree(s->atoms);
   cudaFree(s->entries);
   cudaFree(s->rejects);
   cudaFree(s->replay);
   delete s;
   h->extras[1] = nullptr;
}

}  // namespace vgpu

using namespace vgpu;

// Host-side greedy colouring of the (symmetrised) exchange graph.
static int greedy_colour(int n, const std::vector<std::vector<int>>& adj, std::vector<int>& colour) {
   colour.assign(n, -1);
   int nc = 0;
   std::vector<int> used;
   for (int i = 0; i < n; ++i) {
      used.assign(nc + 1, 0);
      for (int j : adj[i])
         if (colour[j] >= 0 && colour[j] <= nc) used[colour[j]] = 1;
      int c = 0;
      while (c <= nc && used[c]) ++c;
      colour[i] = c;
      nc = std::max(nc, c + 1);
   }
   return nc;
}

extern "C" int vgpu_mc_setup(vgpu_handle h, const int32_t* colour_in, int32_t* n_colours_out) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   SysDev& S = h->sys;
   if (!S.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   cudaSetDevice(h->device);
   const int n = S.n;
   // neighbour lists back from the host copy kept at upload
   if (S.nl_host.empty() && S.num_bonds > 0) return set_err(h, VGPU_ERR_STATE, "neighbour list not retained");
   std::vector<std::vector<int>> adj(n);
   for (int i = 0; i < n; ++i)
      for (int64_t b = S.row_host[i]; b < S.row_host[i + 1]; ++b) {
         const int j = S.nl_host[b];
         if (j == i) continue;
         adj[i].push_back(j);
         adj[j].push_back(i);
      }
   std::vector<int> colour;
   int nc = 0;
   if (colour_in) {
      colour.assign(colour_in, colour_in + n);
      for (int i = 0; i < n; ++i) {
         if (colour[i] < 0) return set_err(h, VGPU_ERR_ARG, "negative colour at atom %d", i);
         nc = std::max(nc, colour[i] + 1);
      }
      for (int i = 0; i < n; ++i)
         for (int j : adj[i])
            if (colour[j] == colour[i])
               return set_err(h, VGPU_ERR_ARG, "colour conflict: interacting atoms %d and %d share colour %d", i, j,
                              colour[i]);
   } else {
      nc = greedy_colour(n, adj, colour);
   }
   mc_destroy(h);
   MCState* s = new MCState();
   h->extras[1] = s;
   s->ncolours = nc;
   s->colour_host = colour;
   // a shard's sweeps visit its owned atoms only (halo atoms are another
   // rank's, refreshed between the colours by the host)
   const int nu = S.n_owned;
   s->n_owned = nu;
   s->colour_off.assign(nc + 1, 0);
   for (int i = 0; i < nu; ++i) s->colour_off[colour[i] + 1]++;
   for (int c = 0; c < nc; ++c) s->colour_off[c + 1] += s->colour_off[c];
   std::vector<int> order(std::max(nu, 1)), fill(s->colour_off.begin(), s->colour_off.end() - 1);
   for (int i = 0; i < nu; ++i) order[fill[colour[i]]++] = i;
   cudaError_t e;
   if ((e = cudaMalloc(&s->atoms, sizeof(int) * order.size())) != cudaSuccess) return cuda_err(h, e, "mc atoms");
   if ((e = cudaMalloc(&s->entries, sizeof(int4) * order.size())) != cudaSuccess) return cuda_err(h, e, "mc entries");
   if ((e = cudaMalloc(&s->rejects, sizeof(unsigned long long))) != cudaSuccess) return cuda_err(h, e, "mc counter");
   cudaMemcpyAsync(s->atoms, order.data(), sizeof(int) * order.size(), cudaMemcpyHostToDevice, h->stream);
   if (nu > 0) {
      mc_entries_kernel<<<(nu + 255) / 256, 256, 0, h->stream>>>(s->atoms, nu, (const int*)S.slice_off,
                                                                   (const int*)S.mat, s->entries);
      if ((e = cudaGetLastError()) != cudaSuccess) return cuda_err(h, e, "mc entries");
   }
   cudaMemsetAsync(s->rejects, 0, sizeof(unsigned long long), h->stream);
   if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return cuda_err(h, e, "mc setup");
   if (n_colours_out) *n_colours_out = nc;
   return VGPU_OK;
}

extern "C" int vgpu_mc_get_colours(vgpu_handle h, int32_t* colour) {
   if (!h || !colour) return set_err(h, VGPU_ERR_ARG, "null argument");
   MCState* s = mc_of(h);
   if (!s) return set_err(h, VGPU_ERR_STATE, "vgpu_mc_setup not called");
   std::copy(s->colour_host.begin(), s->colour_host.end(), colour);
   return VGPU_OK;
}

template <typename R>
static int mc_replay_typed(vgpu_handle h, const double* r) {
   MCState* s = mc_of(h);
   const size_t m = 4 * (size_t)h->sys.n;
   if (!s->replay) {
      cudaError_t e = cudaMalloc(&s->replay, m * sizeof(R));
      if (e != cudaSuccess) return cuda_err(h, e, "mc replay buffer");
   }
   std::vector<R> buf(r, r + m);
   int rc = cuda_err(h, cudaMemcpyAsync(s->replay, buf.data(), m * sizeof(R), cudaMemcpyHostToDevice, h->stream),
                     "mc replay");
   if (rc) return rc;
   return cuda_err(h, cudaStreamSynchronize(h->stream), "mc replay");
}

extern "C" int vgpu_mc_set_replay(vgpu_handle h, const double* r) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   MCState* s = mc_of(h);
   if (!s) return set_err(h, VGPU_ERR_STATE, "vgpu_mc_setup not called");
   cudaSetDevice(h->device);
   if (!r) {
      s->use_replay = false;
      return VGPU_OK;
   }
   int rc = h->prec == VGPU_PREC_FP64 ? mc_replay_typed<double>(h, r) : mc_replay_typed<float>(h, r);
   if (rc) return rc;
   s->use_replay = true;
   return VGPU_OK;
}

// per-material move width, inverse temperature and moment ratio (mc.cpp:45-53)
// into the handle's device table -- sigma [M], beta [M], mu_ratio [M], then
// (at the next 64-byte boundary) the MCMat records [M]; returns it or nullptr
// (error set).  An unchanged table is not copied again.
static size_t mc_mat_offset(int M) { return (3 * (size_t)M * sizeof(double) + 63) & ~(size_t)63; }

template <typename R>
static const MCMat<R>* mc_mat_records(vgpu_handle h, const R* tab) {
   return reinterpret_cast<const MCMat<R>*>(reinterpret_cast<const char*>(tab) + mc_mat_offset(h->sys.M));
}

template <typename R>
static R* mc_tables(vgpu_handle h) {
   SysDev& S = h->sys;
   const int M = S.M;
   const size_t off = mc_mat_offset(M), bytes = off + (size_t)M * sizeof(MCMat<R>);
   std::vector<unsigned char> host(bytes, 0);
   R* sig = reinterpret_cast<R*>(host.data());
   MCMat<R>* rec = reinterpret_cast<MCMat<R>*>(host.data() + off);
   for (int m = 0; m < M; ++m) {
      const vgpu_material& q = S.materials[m];
      const double T = h->params.local_temperature ? q.temperature : h->params.temperature;
      const double al = q.temperature_rescaling_alpha, Tc = q.temperature_rescaling_Tc;
      const double Tr = T < Tc ? Tc * std::pow(T / Tc, al) : T;
      const double kBTBohr = 9.27400915e-24 / (Tr * 1.3806503e-23);
      sig[m] = (R)(Tr < 1.0 ? 0.02 : std::pow(1.0 / kBTBohr, 0.2) * 0.08);
      sig[M + m] = (R)kBTBohr;
      sig[2 * M + m] = (R)(q.mu_s_SI * 1.07828231e23);
      rec[m] = MCMat<R>{sig[m], sig[M + m], sig[2 * M + m], (R)q.ku2, (R)q.ku_vector[0], (R)q.ku_vector[1],
                        (R)q.ku_vector[2], (R)q.kc4};
   }
   if (!S.mc_tab) {
      S.mc_tab = h->alloc(mc_mat_offset(M) + (size_t)M * sizeof(MCMat<double>));
      if (!S.mc_tab) {
         set_err(h, VGPU_ERR_OOM, "mc tables");
         return nullptr;
      }
      S.mc_tab_host.clear();
   }
   if (S.mc_tab_host != host) {
      if (cuda_err(h, cudaMemcpyAsync(S.mc_tab, host.data(), bytes, cudaMemcpyHostToDevice, h->stream), "mc tables"))
         return nullptr;
      S.mc_tab_host.swap(host);
   }
   return (R*)S.mc_tab;
}

// one colour of the current sweep; the last colour completes the sweep
template <typename R>
static int mc_run_colour(vgpu_handle h, const R* tab, int c) {
   MCState* s = mc_of(h);
   SysDev& S = h->sys;
   MCArgs<R> p;
   memset(&p, 0, sizeof p);
   p.a = make_args<R>(h);
   p.mat = mc_mat_records<R>(h, tab);
   p.replay = s->use_replay ? (const R*)s->replay : nullptr;
   p.sweep = s->sweep;
   p.rejects = s->rejects;
   p.entries = s->entries + s->colour_off[c];
   p.count = s->colour_off[c + 1] - s->colour_off[c];
   h->prof_begin(PROF_MC);
   cudaError_t e = mc_dispatch<R>(p, S.fmt, h->stream);
   h->prof_end(PROF_MC);
   if (e != cudaSuccess) return cuda_err(h, e, "mc launch");
   h->kernel_launches++;
   s->next_colour = c + 1;
   if (s->next_colour == s->ncolours) {
      s->next_colour = 0;
      s->sweep++;
      s->moves += s->n_owned;
   }
   return VGPU_OK;
}

template <typename R>
static int mc_sweeps_typed(vgpu_handle h, uint64_t n_sweeps) {
   MCState* s = mc_of(h);
   const R* tab = mc_tables<R>(h);
   if (!tab) return VGPU_ERR_OOM;
   for (uint64_t sw = 0; sw < n_sweeps; ++sw)
      for (int c = 0; c < s->ncolours; ++c)
         if (const int rc = mc_run_colour<R>(h, tab, c)) return rc;
   return VGPU_OK;
}

template <typename R>
static int mc_colour_typed(vgpu_handle h, int c) {
   const R* tab = mc_tables<R>(h);
   if (!tab) return VGPU_ERR_OOM;
   return mc_run_colour<R>(h, tab, c);
}

extern "C" int vgpu_mc_sweep(vgpu_handle h, uint64_t n_sweeps) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   MCState* s = mc_of(h);
   if (!s) return set_err(h, VGPU_ERR_STATE, "vgpu_mc_setup not called");
   if (!(h->params.temperature >= 0.0)) return set_err(h, VGPU_ERR_STATE, "vgpu_set_params not called");
   if (int rc = h->fields_ready()) return rc;
   if (s->next_colour != 0)
      return set_err(h, VGPU_ERR_STATE, "a sweep run colour by colour (vgpu_mc_colour) is unfinished");
   cudaSetDevice(h->device);
   return h->prec == VGPU_PREC_FP64 ? mc_sweeps_typed<double>(h, n_sweeps) : mc_sweeps_typed<float>(h, n_sweeps);
}

extern "C" int vgpu_mc_colour(vgpu_handle h, int32_t colour) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   MCState* s = mc_of(h);
   if (!s) return set_err(h, VGPU_ERR_STATE, "vgpu_mc_setup not called");
   if (!(h->params.temperature >= 0.0)) return set_err(h, VGPU_ERR_STATE, "vgpu_set_params not called");
   if (int rc = h->fields_ready()) return rc;
   if (colour != s->next_colour)
      return set_err(h, VGPU_ERR_ARG, "colour %d out of order: the current sweep runs colour %d next (of %d)", colour,
                     s->next_colour, s->ncolours);
   cudaSetDevice(h->device);
   return h->prec == VGPU_PREC_FP64 ? mc_colour_typed<double>(h, colour) : mc_colour_typed<float>(h, colour);
}

extern "C" int vgpu_mc_set_sweep(vgpu_handle h, uint64_t sweep) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   MCState* s = mc_of(h);
   if (!s) return set_err(h, VGPU_ERR_STATE, "vgpu_mc_setup not called");
   s->sweep = sweep;
   s->next_colour = 0;
   return VGPU_OK;
}

extern "C" int vgpu_mc_counters(vgpu_handle h, double* moves, double* rejects) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   MCState* s = mc_of(h);
   if (!s) return set_err(h, VGPU_ERR_STATE, "vgpu_mc_setup not called");
   cudaSetDevice(h->device);
   unsigned long long r = 0;
   cudaError_t e = cudaMemcpyAsync(&r, s->rejects, sizeof r, cudaMemcpyDeviceToHost, h->stream);
   if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
   if (e != cudaSuccess) return cuda_err(h, e, "mc counters");
   if (moves) *moves = s->moves;
   if (rejects) *rejects = (double)r;
   return VGPU_OK;
}

// ---------------------------------------------------------------------------
// Constrained Monte Carlo (reference: montecarlo::cmc_step,
// src/montecarlo/cmc.cpp:282-490; CMCinit and polar_rot_matrix, :53-270).
//
// The reference makes N pair moves per step: a random spin takes an angle
// move, a second random spin compensates the moment perpendicular to the
// constraint direction, and the pair is accepted with probability
// exp(-dE/kT) (Mz'/Mz)^2 |s2z/s2z'| (and Mz' > 0), where Mz is the total
// moment along the constraint -- every decision depends on all earlier ones
// through Mz.  Here a step is phases over the colours of the exchange graph,
// twice over (about N pairs, as the reference): in a phase the atoms of one
// colour are paired by a random affine permutation of that colour's list, so
// no atom of any pair interacts with an atom of another pair, and
//
//   propose  (one thread per pair)  the move, the compensating spin, both
//            energy changes, exp(-dE) and the Jacobian factor, and the moment
//            terms mu s of both spins before and after;
//   accept   (one warp)  the pairs in order with the running total moment,
//            exactly the reference's rule: a pair's energy change does not
//            depend on the other pairs of the phase, so the sequence of
//            decisions is that of the sequential chain for this order of
//            pairs; lanes then write the accepted spins.
//
// Every pair move keeps the target distribution (the reference's
// Metropolis-Hastings step with its constraint Jacobian), so the phases
// sample it too; pair selection differs from the reference's (random pairs
// with replacement), so the two are compared statistically.
// ---------------------------------------------------------------------------

namespace vgpu {

struct CMCState {
   double P[9] = {0}, pv[3] = {0, 0, 1};   // frame: P rotates the constraint direction to z
   int maxK = 0;
   int* pairs = nullptr;      // [2 maxK]
   void* prop = nullptr;      // [6 maxK] proposed spins s1', s2' (x|y|z of each, R)
   double* ef = nullptr;      // [maxK] exp(-dE) (negative: sphere rejection)
   double* jac = nullptr;     // [maxK] |s2z / s2z'| in the constraint frame
   double* mom = nullptr;     // [12 maxK] mu1 s1', mu2 s2', mu1 s1, mu2 s2 (x|y|z blocks of maxK each)
   double* u = nullptr;       // [maxK] acceptance uniforms (replay) or nullptr
   double* rnd = nullptr;     // [4 maxK] replayed Gaussians and uniforms
   double* M = nullptr;       // [3] running total moment (mu_B)
   unsigned long long* cnt = nullptr;  // [4] accepted, energy rejections, sphere rejections,
                                       //     rejected single-spin moves (hybrid)
   uint64_t sweep = 0;
   double total = 0.0;
   // hybrid (montecarlo::cmc_mc_step): one constraint per material
   bool hybrid = false;
   int nmat = 0;
   std::vector<int> constrained;       // [nmat]
   std::vector<double> Pm;             // [9M] frames
   double* Mm = nullptr;               // [6M] per material: running moment (3), constraint vector (3)
   int* lists = nullptr;               // atoms by (colour, material), unconstrained last
   int4* list_entries = nullptr;       // MC list entries of lists (single-spin moves)
   std::vector<int> list_off;          // [ncolours * (M + 1) + 1]
   double single_moves = 0.0;
};

static CMCState* cmc_of(vgpu_ctx* h) { return (CMCState*)h->extras[5]; }

void cmc_destroy(vgpu_ctx* h) {
   CMCState* c = cmc_of(h);
   if (!c) return;
   cudaFree(c->pairs); cudaFree(c->prop); cudaFree(c->ef); cudaFree(c->jac); cudaFree(c->mom);
   cudaFree(c->rnd); cudaFree(c->M); cudaFree(c->cnt); cudaFree(c->Mm); cudaFree(c->lists); cudaFree(c->list_entries);
   delete c;
   h->extras[5] = nullptr;
}

template <typename R>
struct CMCArgs {
   LLGArgs<R> a;
   const int* list;     // the colour's atoms (affine pairing) or nullptr
   int count;           // atoms in the list
   uint64_t mul, add;   // pair k = (list[(mul 2k + add) % count], list[(mul (2k+1) + add) % count])
   const int* given;    // explicit pairs [2K] or nullptr
   int K;
   const R* sigma; const R* beta; const R* mu_ratio;
   const double* rnd;   // replayed numbers [4K] or nullptr
   uint64_t sweep; uint32_t phase;
   double P[9];
   int* pairs; R* prop; double* ef; double* jac; double* mom; int maxK;
};

template <typename R, int FMT>
__device__ __forceinline__ R cmc_delta(const LLGArgs<R>& a, int i, int mi, const MatParams<R>& m, const R S[3],
                                       const R T[3], R ratio) {
   R h[3] = {0, 0, 0};
   exchange_gather<R, FMT>(a, i, mi, a.ax, a.ay, a.az, h[0], h[1], h[2]);
   if (a.cell) {
      const int c = __ldg(a.cell + i);
      h[0] += __ldg(a.cell_hd + c); h[1] += __ldg(a.cell_hd + a.ncells + c); h[2] += __ldg(a.cell_hd + 2 * a.ncells + c);
   } else if (a.hm_atom) {
      h[0] += __ldg(a.hm_atom + i); h[1] += __ldg(a.hm_atom + a.n + i); h[2] += __ldg(a.hm_atom + 2 * a.n + i);
   }
   return site_energy_delta<R>(a, i, mi, m, S, T, h) * ratio;
}

template <typename R, int FMT>
__global__ void __launch_bounds__(128) cmc_propose_kernel(const CMCArgs<R> p) {
   const int k = blockIdx.x * blockDim.x + threadIdx.x;
   if (k >= p.K) return;
   const LLGArgs<R>& a = p.a;
   int i1, i2;
   if (p.given) {
      i1 = p.given[2 * k]; i2 = p.given[2 * k + 1];
   } else {
      i1 = __ldg(p.list + (int)((p.mul * (uint64_t)(2 * k) + p.add) % (uint64_t)p.count));
      i2 = __ldg(p.list + (int)((p.mul * (uint64_t)(2 * k + 1) + p.add) % (uint64_t)p.count));
   }
   p.pairs[2 * k] = i1;
   p.pairs[2 * k + 1] = i2;
   const int m1 = a.mat ? __ldg(a.mat + i1) : 0, m2 = a.mat ? __ldg(a.mat + i2) : 0;
   const MatParams<R> mp1 = a.mp[m1], mp2 = a.mp[m2];
   double g0, g1, g2;
   if (p.rnd) {
      g0 = p.rnd[k]; g1 = p.rnd[p.K + k]; g2 = p.rnd[2 * p.K + k];
   } else {
      const u32x4 c = {(uint32_t)k, (uint32_t)p.sweep, (uint32_t)(p.sweep >> 32) ^ (p.phase << 20), RNG_CMC_MOVE};
      const u32x4 r = philox4x32_10(c, a.seed_lo, a.seed_hi);
      double s1, c1, s2, c2;
      const double r1 = sqrt(-2.0 * log(u01d(r.x)));
      const double rr = sqrt(-2.0 * log(u01d(r.z)));
      sincospi(2.0 * u01d(r.y), &s1, &c1);
      sincospi(2.0 * u01d(r.w), &s2, &c2);
      g0 = r1 * c1; g1 = r1 * s1; g2 = rr * c2;
   }
   const R sg = __ldg(p.sigma + m1);
   const R S1[3] = {a.ax[i1], a.ay[i1], a.az[i1]};
   const R S2[3] = {a.ax[i2], a.ay[i2], a.az[i2]};
   R T1[3] = {S1[0] + (R)g0 * sg, S1[1] + (R)g1 * sg, S1[2] + (R)g2 * sg};
   const R r = rsqrt_<R>(T1[0] * T1[0] + T1[1] * T1[1] + T1[2] * T1[2]);
   T1[0] *= r; T1[1] *= r; T1[2] *= r;
   // the constraint frame in FP64 (the compensating spin keeps the
   // perpendicular moment to rounding)
   const double* P = p.P;
   double s1im[3], s1fm[3], s2im[3], s2fm[3];
   for (int q = 0; q < 3; ++q) {
      s1im[q] = P[3 * q] * (double)S1[0] + P[3 * q + 1] * (double)S1[1] + P[3 * q + 2] * (double)S1[2];
      s1fm[q] = P[3 * q] * (double)T1[0] + P[3 * q + 1] * (double)T1[1] + P[3 * q + 2] * (double)T1[2];
      s2im[q] = P[3 * q] * (double)S2[0] + P[3 * q + 1] * (double)S2[1] + P[3 * q + 2] * (double)S2[2];
   }
   const double mu1 = (double)__ldg(p.mu_ratio + m1), mu2 = (double)__ldg(p.mu_ratio + m2);
   const double mr = mu1 / mu2;
   s2fm[0] = mr * (s1im[0] - s1fm[0]) + s2im[0];
   s2fm[1] = mr * (s1im[1] - s1fm[1]) + s2im[1];
   const int st = p.maxK;
   if (!((s2fm[0] * s2fm[0] + s2fm[1] * s2fm[1]) < 1.0) || i1 == i2) {
      p.ef[k] = -1.0;  // off the unit sphere: rejected
      return;
   }
   s2fm[2] = (s2im[2] >= 0.0 ? 1.0 : -1.0) * sqrt(1.0 - s2fm[0] * s2fm[0] - s2fm[1] * s2fm[1]);
   R T2[3];
   for (int q = 0; q < 3; ++q) T2[q] = (R)(P[q] * s2fm[0] + P[3 + q] * s2fm[1] + P[6 + q] * s2fm[2]);
   // the two spins share no bond (one colour), so each energy change sees
   // the other's neighbours as they are
   const R de1 = cmc_delta<R, FMT>(a, i1, m1, mp1, S1, T1, (R)mu1);
   const R de2 = cmc_delta<R, FMT>(a, i2, m2, mp2, S2, T2, (R)mu2);
   const double de21 = (double)de1 * (double)__ldg(p.beta + m1) + (double)de2 * (double)__ldg(p.beta + m2);
   p.ef[k] = exp(-de21);
   p.jac[k] = fabs(s2im[2] / s2fm[2]);
   for (int q = 0; q < 3; ++q) {
      p.prop[q * st + k] = T1[q];
      p.prop[(3 + q) * st + k] = T2[q];
      p.mom[q * st + k] = mu1 * (double)T1[q];
      p.mom[(3 + q) * st + k] = mu2 * (double)T2[q];
      p.mom[(6 + q) * st + k] = mu1 * (double)S1[q];
      p.mom[(9 + q) * st + k] = mu2 * (double)S2[q];
   }
}

// One warp: the pairs in order with the running total moment M (the
// reference's acceptance, cmc.cpp:459-490); each lane holds a chunk's pair,
// every lane follows the same decisions, lane l writes pair l's spins.
template <typename R>
__global__ void __launch_bounds__(32) cmc_accept_kernel(LLGArgs<R> a, int K, int st, const int* __restrict__ pairs,
                                                        const R* __restrict__ prop, const double* __restrict__ ef,
                                                        const double* __restrict__ jac,
                                                        const double* __restrict__ mom, const double* __restrict__ urep,
                                                        uint64_t sweep, uint32_t phase, const double* pvp, double* M,
                                                        unsigned long long* cnt) {
   const int lane = threadIdx.x;
   const unsigned full = 0xffffffffu;
   const double pv[3] = {pvp[0], pvp[1], pvp[2]};
   double Mx = M[0], My = M[1], Mz = M[2];
   unsigned long long nacc = 0, nrej = 0, nsph = 0;
   for (int base = 0; base < K; base += 32) {
      const int k = base + lane;
      const bool on = k < K;
      double e = -1.0, jk = 0.0, u = 0.0, mm[12];
      for (int q = 0; q < 12; ++q) mm[q] = 0.0;
      if (on) {
         e = ef[k];
         if (e >= 0.0) {
            jk = jac[k];
            for (int q = 0; q < 12; ++q) mm[q] = mom[q * st + k];
         }
         if (urep) {
            u = urep[k];
         } else {
            const u32x4 c = {(uint32_t)k, (uint32_t)sweep, (uint32_t)(sweep >> 32) ^ (phase << 20), RNG_CMC_ACCEPT};
            u = u01d(philox4x32_10(c, a.seed_lo, a.seed_hi).x);
         }
      }
      bool mine = false;
      const int nl = min(32, K - base);
      for (int l = 0; l < nl; ++l) {
         const double el = __shfl_sync(full, e, l);
         if (el < 0.0) {
            ++nsph;
            continue;
         }
         double ml[12];
         for (int q = 0; q < 12; ++q) ml[q] = __shfl_sync(full, mm[q], l);
         const double jl = __shfl_sync(full, jk, l), ul = __shfl_sync(full, u, l);
         const double mzo = Mx * pv[0] + My * pv[1] + Mz * pv[2];
         const double nx = Mx + ml[0] + ml[3] - ml[6] - ml[9];
         const double ny = My + ml[1] + ml[4] - ml[7] - ml[10];
         const double nz = Mz + ml[2] + ml[5] - ml[8] - ml[11];
         const double mzn = nx * pv[0] + ny * pv[1] + nz * pv[2];
         const double prob = el * ((mzn / mzo) * (mzn / mzo)) * jl;
         if (prob >= ul && mzn > 0.0) {
            Mx = nx; My = ny; Mz = nz;
            ++nacc;
            if (lane == l) mine = true;
         } else {
            ++nrej;
         }
      }
      if (mine) {
         const int i1 = pairs[2 * k], i2 = pairs[2 * k + 1];
         a.ax[i1] = prop[k]; a.ay[i1] = prop[st + k]; a.az[i1] = prop[2 * st + k];
         a.ax[i2] = prop[3 * st + k]; a.ay[i2] = prop[4 * st + k]; a.az[i2] = prop[5 * st + k];
      }
   }
   if (lane == 0) {
      M[0] = Mx; M[1] = My; M[2] = Mz;
      cnt[0] += nacc; cnt[1] += nrej; cnt[2] += nsph;
   }
}

// total moment sum_i mu_s,i s_i (mu_B) into M (zeroed first), FP64; with
// only_mat >= 0 over the atoms of that material
template <typename R>
__global__ void cmc_moment_kernel(const LLGArgs<R> a, const R* __restrict__ mu_ratio, double* M, int only_mat) {
   double v[3] = {0, 0, 0};
   for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < a.n_upd; i += gridDim.x * blockDim.x) {
      const int mi = a.mat ? __ldg(a.mat + i) : 0;
      if (only_mat >= 0 && mi != only_mat) continue;
      const double mu = (double)__ldg(mu_ratio + mi);
      v[0] += mu * (double)a.ax[i]; v[1] += mu * (double)a.ay[i]; v[2] += mu * (double)a.az[i];
   }
   for (int q = 0; q < 3; ++q) {
      for (int o = 16; o > 0; o >>= 1) v[q] += __shfl_xor_sync(0xffffffffu, v[q], o);
      if ((threadIdx.x & 31) == 0) atomicAdd(M + q, v[q]);
   }
}

template <typename R, int FMT>
static cudaError_t launch_cmc_propose(const CMCArgs<R>& p, cudaStream_t st) {
   if (p.K <= 0) return cudaSuccess;
   cmc_propose_kernel<R, FMT><<<(p.K + 127) / 128, 128, 0, st>>>(p);
   return cudaGetLastError();
}

template <typename R>
static cudaError_t cmc_propose_dispatch(const CMCArgs<R>& p, int fmt, cudaStream_t st) {
   switch (fmt) {
      case FMT_ISO_TAB: return launch_cmc_propose<R, FMT_ISO_TAB>(p, st);
      case FMT_ISO_BOND: return launch_cmc_propose<R, FMT_ISO_BOND>(p, st);
      case FMT_VEC_TAB: return launch_cmc_propose<R, FMT_VEC_TAB>(p, st);
      case FMT_VEC_BOND: return launch_cmc_propose<R, FMT_VEC_BOND>(p, st);
      case FMT_DMI_TAB: return launch_cmc_propose<R, FMT_DMI_TAB>(p, st);
      default: return launch_cmc_propose<R, FMT_TENSOR_BOND>(p, st);
   }
}

}  // namespace vgpu

namespace {

uint64_t splitmix64(uint64_t x) {
   x += 0x9E3779B97F4A7C15ull;
   x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
   x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
   return x ^ (x >> 31);
}

uint64_t gcd64(uint64_t a, uint64_t b) {
   while (b) {
      const uint64_t t = a % b;
      a = b;
      b = t;
   }
   return a;
}

// one phase: K pairs (explicit, or the affine pairing of colour c), proposals
// in parallel, acceptance by one warp
template <typename R>
int cmc_phase(vgpu_handle h, const R* tab, const int* list, int count, const int* given, int K, const double* rnd,
              uint32_t phase, const double* P, double* Mdev) {
   CMCState* c = cmc_of(h);
   CMCArgs<R> p;
   memset(&p, 0, sizeof p);
   p.a = make_args<R>(h);
   p.sigma = tab; p.beta = tab + h->sys.M; p.mu_ratio = tab + 2 * h->sys.M;
   p.sweep = c->sweep; p.phase = phase;
   for (int q = 0; q < 9; ++q) p.P[q] = P[q];
   p.pairs = c->pairs; p.prop = (R*)c->prop; p.ef = c->ef; p.jac = c->jac; p.mom = c->mom; p.maxK = c->maxK;
   p.K = K;
   p.given = given;
   p.rnd = rnd;
   if (!given) {
      p.list = list;
      p.count = count;
      const uint64_t key = splitmix64(h->seed ^ splitmix64(c->sweep * 1024 + phase));
      const uint64_t n = (uint64_t)std::max(p.count, 1);
      uint64_t mul = 1 + splitmix64(key) % n;
      while (gcd64(mul, n) != 1) mul = mul % n + 1;
      p.mul = mul;
      p.add = splitmix64(key + 1) % n;
   }
   h->prof_begin(PROF_MC);
   cudaError_t e = cmc_propose_dispatch<R>(p, h->sys.fmt, h->stream);
   if (e == cudaSuccess && K > 0) {
      cmc_accept_kernel<R><<<1, 32, 0, h->stream>>>(p.a, K, c->maxK, c->pairs, (const R*)c->prop, c->ef, c->jac,
                                                    c->mom, rnd ? rnd + 3 * (size_t)K : nullptr, c->sweep, phase,
                                                    Mdev + 3, Mdev, c->cnt);
      e = cudaGetLastError();
   }
   h->prof_end(PROF_MC);
   if (e != cudaSuccess) return cuda_err(h, e, "cmc launch");
   h->kernel_launches += 2;
   c->total += K;
   return VGPU_OK;
}

template <typename R>
int cmc_recount_moment(vgpu_handle h, const R* tab, double* M, int only_mat) {
   cudaMemsetAsync(M, 0, 3 * sizeof(double), h->stream);
   cmc_moment_kernel<R><<<std::max(1, std::min(1024, (h->sys.n + 255) / 256)), 256, 0, h->stream>>>(
       make_args<R>(h), tab + 2 * h->sys.M, M, only_mat);
   h->kernel_launches++;
   return cuda_err(h, cudaGetLastError(), "cmc moment");
}

// hybrid step (montecarlo::cmc_mc_step, src/montecarlo/cmc_mc.cpp:291-490):
// per colour, the unconstrained materials' atoms take single-spin Metropolis
// moves (once per step) and each constrained material's atoms of the colour
// are paired among themselves (twice over), with that material's frame and
// running moment
template <typename R>
int cmc_hybrid_sweeps(vgpu_handle h, const R* tab, uint64_t n_sweeps) {
   CMCState* c = cmc_of(h);
   MCState* s = mc_of(h);
   const int M = c->nmat, nc = s->ncolours;
   for (uint64_t sw = 0; sw < n_sweeps; ++sw) {
      for (int m = 0; m < M; ++m)
         if (c->constrained[m])
            if (int rc = cmc_recount_moment<R>(h, tab, c->Mm + 6 * m, m)) return rc;
      uint32_t phase = 0;
      for (int round = 0; round < 2; ++round)
         for (int col = 0; col < nc; ++col) {
            if (round == 0) {
               const int u0 = c->list_off[col * (M + 1) + M], u1 = c->list_off[col * (M + 1) + M + 1];
               if (u1 > u0) {
                  MCArgs<R> p;
                  memset(&p, 0, sizeof p);
                  p.a = make_args<R>(h);
                  p.mat = mc_mat_records<R>(h, tab);
                  p.sweep = c->sweep;
                  p.rejects = c->cnt + 3;
                  p.entries = c->list_entries + u0;
                  p.count = u1 - u0;
                  cudaError_t e = mc_dispatch<R>(p, h->sys.fmt, h->stream);
                  if (e != cudaSuccess) return cuda_err(h, e, "cmc single-spin launch");
                  h->kernel_launches++;
                  c->single_moves += p.count;
                  c->total += p.count;
               }
            }
            for (int m = 0; m < M; ++m, ++phase) {
               if (!c->constrained[m]) continue;
               const int a0 = c->list_off[col * (M + 1) + m], a1 = c->list_off[col * (M + 1) + m + 1];
               const int K = (a1 - a0) / 2;
               if (K == 0) continue;
               if (int rc = cmc_phase<R>(h, tab, c->lists + a0, a1 - a0, nullptr, K, nullptr, phase,
                                         c->Pm.data() + 9 * m, c->Mm + 6 * m))
                  return rc;
            }
         }
      c->sweep++;
   }
   return VGPU_OK;
}

template <typename R>
int cmc_sweeps_typed(vgpu_handle h, uint64_t n_sweeps) {
   CMCState* c = cmc_of(h);
   MCState* s = mc_of(h);
   const R* tab = mc_tables<R>(h);
   if (!tab) return VGPU_ERR_OOM;
   if (c->hybrid) return cmc_hybrid_sweeps<R>(h, tab, n_sweeps);
   for (uint64_t sw = 0; sw < n_sweeps; ++sw) {
      // the total moment from the spins at every step, as the reference does
      if (int rc = cmc_recount_moment<R>(h, tab, c->M, -1)) return rc;
      uint32_t phase = 0;
      for (int round = 0; round < 2; ++round)
         for (int col = 0; col < s->ncolours; ++col, ++phase) {
            const int K = (s->colour_off[col + 1] - s->colour_off[col]) / 2;
            if (int rc = cmc_phase<R>(h, tab, s->atoms + s->colour_off[col], s->colour_off[col + 1] - s->colour_off[col],
                                      nullptr, K, nullptr, phase, c->P, c->M))
               return rc;
         }
      c->sweep++;
   }
   return VGPU_OK;
}

}  // namespace

namespace {

// polar_rot_matrix (cmc.cpp:53-135): P = Ry(phi) Rz(theta) with the
// reference's element layout; the constraint vector pv = (0,0,1) P, the third row
void cmc_frame(double phi_deg, double theta_deg, double* P, double* pv) {
   const double d2r = 3.14159265358979323846264338327 / 180.0;
   const double sy = std::sin(phi_deg * d2r), cy = std::cos(phi_deg * d2r);
   const double sz = std::sin(theta_deg * d2r), cz = std::cos(theta_deg * d2r);
   const double Ry[9] = {cy, 0.0, -sy, 0.0, 1.0, 0.0, sy, 0.0, cy};
   const double Rz[9] = {cz, sz, 0.0, -sz, cz, 0.0, 0.0, 0.0, 1.0};
   for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j) {
         double v = 0.0;
         for (int k = 0; k < 3; ++k) v += Ry[3 * i + k] * Rz[3 * k + j];
         P[3 * i + j] = v;
      }
   for (int j = 0; j < 3; ++j) pv[j] = P[6 + j];
}

void constraint_direction(double phi_deg, double theta_deg, double dir[3]) {
   const double d2r = 3.14159265358979323846264338327 / 180.0;
   dir[0] = std::sin(phi_deg * d2r) * std::cos(theta_deg * d2r);
   dir[1] = std::sin(phi_deg * d2r) * std::sin(theta_deg * d2r);
   dir[2] = std::cos(phi_deg * d2r);
}

// a fresh CMC state with the pair buffers; nullptr on error (set)
CMCState* cmc_new(vgpu_handle h) {
   if (!mc_of(h)) {
      int32_t nc = 0;
      if (vgpu_mc_setup(h, nullptr, &nc)) return nullptr;
   }
   cmc_destroy(h);
   CMCState* c = new CMCState();
   h->extras[5] = c;
   MCState* s = mc_of(h);
   int maxK = 1;
   for (int col = 0; col < s->ncolours; ++col) maxK = std::max(maxK, (s->colour_off[col + 1] - s->colour_off[col]) / 2);
   maxK = std::max(maxK, h->sys.n / 2);
   c->maxK = maxK;
   const size_t rs = h->prec == VGPU_PREC_FP64 ? sizeof(double) : sizeof(float);
   cudaError_t e;
   if ((e = cudaMalloc(&c->pairs, sizeof(int) * 2 * maxK)) || (e = cudaMalloc(&c->prop, rs * 6 * maxK)) ||
       (e = cudaMalloc(&c->ef, sizeof(double) * maxK)) || (e = cudaMalloc(&c->jac, sizeof(double) * maxK)) ||
       (e = cudaMalloc(&c->mom, sizeof(double) * 12 * maxK)) || (e = cudaMalloc(&c->rnd, sizeof(double) * 4 * maxK)) ||
       (e = cudaMalloc(&c->M, sizeof(double) * 6)) || (e = cudaMalloc(&c->cnt, sizeof(unsigned long long) * 4))) {
      cmc_destroy(h);
      cuda_err(h, e, "cmc buffers");
      return nullptr;
   }
   cudaMemsetAsync(c->cnt, 0, sizeof(unsigned long long) * 4, h->stream);
   return c;
}

}  // namespace

extern "C" int vgpu_cmc_setup(vgpu_handle h, double phi_deg, double theta_deg, int32_t init_spins) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   if (h->sys.n_owned < h->sys.n) return set_err(h, VGPU_ERR_STATE, "constrained Monte Carlo runs on whole systems");
   cudaSetDevice(h->device);
   CMCState* c = cmc_new(h);
   if (!c) return VGPU_ERR_CUDA;
   cmc_frame(phi_deg, theta_deg, c->P, c->pv);
   cudaMemcpyAsync(c->M + 3, c->pv, sizeof(double) * 3, cudaMemcpyHostToDevice, h->stream);
   if (init_spins) {
      // CMCinit: every spin along the constraint direction
      const int n = h->sys.n;
      std::vector<double> v[3];
      double dir[3];
      constraint_direction(phi_deg, theta_deg, dir);
      for (int q = 0; q < 3; ++q) v[q].assign(n, dir[q]);
      if (int rc = vgpu_set_spins(h, v[0].data(), v[1].data(), v[2].data())) return rc;
   }
   return cuda_err(h, cudaStreamSynchronize(h->stream), "cmc setup");
}

extern "C" int vgpu_cmc_setup_materials(vgpu_handle h, const int32_t* constrained, const double* phi_deg,
                                        const double* theta_deg, int32_t init_spins) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   if (!constrained || !phi_deg || !theta_deg) return set_err(h, VGPU_ERR_ARG, "null argument");
   if (h->sys.n_owned < h->sys.n) return set_err(h, VGPU_ERR_STATE, "constrained Monte Carlo runs on whole systems");
   cudaSetDevice(h->device);
   CMCState* c = cmc_new(h);
   if (!c) return VGPU_ERR_CUDA;
   const int M = h->sys.M, n = h->sys.n;
   c->hybrid = true;
   c->nmat = M;
   c->constrained.assign(constrained, constrained + M);
   c->Pm.assign(9 * (size_t)M, 0.0);
   std::vector<double> mm(6 * (size_t)M, 0.0);
   for (int m = 0; m < M; ++m) {
      double pv[3];
      cmc_frame(phi_deg[m], theta_deg[m], c->Pm.data() + 9 * m, pv);
      for (int q = 0; q < 3; ++q) mm[6 * m + 3 + q] = pv[q];
   }
   // atoms by (colour, material), the unconstrained materials' atoms last
   MCState* s = mc_of(h);
   const int nc = s->ncolours;
   std::vector<std::vector<int>> buckets((size_t)nc * (M + 1));
   for (int i = 0; i < n; ++i) {
      const int m = h->sys.type_host[i];
      buckets[(size_t)s->colour_host[i] * (M + 1) + (constrained[m] ? m : M)].push_back(i);
   }
   std::vector<int> flat;
   c->list_off.assign(buckets.size() + 1, 0);
   for (size_t b = 0; b < buckets.size(); ++b) {
      flat.insert(flat.end(), buckets[b].begin(), buckets[b].end());
      c->list_off[b + 1] = (int)flat.size();
   }
   cudaError_t e;
   if ((e = cudaMalloc(&c->Mm, sizeof(double) * mm.size())) ||
       (e = cudaMalloc(&c->lists, sizeof(int) * std::max<size_t>(flat.size(), 1))) ||
       (e = cudaMalloc(&c->list_entries, sizeof(int4) * std::max<size_t>(flat.size(), 1))))
      return cuda_err(h, e, "cmc lists");
   cudaMemcpyAsync(c->Mm, mm.data(), sizeof(double) * mm.size(), cudaMemcpyHostToDevice, h->stream);
   cudaMemcpyAsync(c->lists, flat.data(), sizeof(int) * flat.size(), cudaMemcpyHostToDevice, h->stream);
   if (!flat.empty()) {
      mc_entries_kernel<<<(int)((flat.size() + 255) / 256), 256, 0, h->stream>>>(
          c->lists, (int)flat.size(), (const int*)h->sys.slice_off, (const int*)h->sys.mat, c->list_entries);
      if ((e = cudaGetLastError()) != cudaSuccess) return cuda_err(h, e, "cmc list entries");
   }
   // the plain frame and moment report the first constrained material
   for (int m = 0; m < M; ++m)
      if (constrained[m]) {
         std::copy(c->Pm.begin() + 9 * m, c->Pm.begin() + 9 * m + 9, c->P);
         for (int q = 0; q < 3; ++q) c->pv[q] = mm[6 * m + 3 + q];
         break;
      }
   if (init_spins) {
      // CMCMCinit: the constrained materials' spins along their directions
      std::vector<double> v[3];
      for (int q = 0; q < 3; ++q) v[q].resize(n);
      if (int rc = vgpu_get_spins(h, v[0].data(), v[1].data(), v[2].data())) return rc;
      for (int i = 0; i < n; ++i) {
         const int m = h->sys.type_host[i];
         if (!constrained[m]) continue;
         double dir[3];
         constraint_direction(phi_deg[m], theta_deg[m], dir);
         for (int q = 0; q < 3; ++q) v[q][i] = dir[q];
      }
      if (int rc = vgpu_set_spins(h, v[0].data(), v[1].data(), v[2].data())) return rc;
   }
   return cuda_err(h, cudaStreamSynchronize(h->stream), "cmc setup");
}

extern "C" int vgpu_cmc_material_moments(vgpu_handle h, double* moments) {
   if (!h || !moments) return set_err(h, VGPU_ERR_ARG, "null argument");
   CMCState* c = cmc_of(h);
   if (!c || !c->hybrid) return set_err(h, VGPU_ERR_STATE, "vgpu_cmc_setup_materials not called");
   cudaSetDevice(h->device);
   std::vector<double> mm(6 * (size_t)c->nmat);
   cudaError_t e = cudaMemcpyAsync(mm.data(), c->Mm, sizeof(double) * mm.size(), cudaMemcpyDeviceToHost, h->stream);
   if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
   if (e != cudaSuccess) return cuda_err(h, e, "cmc moments");
   for (int m = 0; m < c->nmat; ++m)
      for (int q = 0; q < 3; ++q) moments[3 * m + q] = mm[6 * m + q];
   return VGPU_OK;
}

extern "C" int vgpu_cmc_frame(vgpu_handle h, double* P9, double* pv3) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   CMCState* c = cmc_of(h);
   if (!c) return set_err(h, VGPU_ERR_STATE, "vgpu_cmc_setup not called");
   if (P9) std::copy(c->P, c->P + 9, P9);
   if (pv3) std::copy(c->pv, c->pv + 3, pv3);
   return VGPU_OK;
}

static int cmc_ready(vgpu_handle h) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   if (!cmc_of(h) || !mc_of(h)) return set_err(h, VGPU_ERR_STATE, "vgpu_cmc_setup not called");
   if (!(h->params.temperature >= 0.0)) return set_err(h, VGPU_ERR_STATE, "vgpu_set_params not called");
   if (int rc = h->fields_ready()) return rc;
   cudaSetDevice(h->device);
   return VGPU_OK;
}

extern "C" int vgpu_cmc_sweep(vgpu_handle h, uint64_t n_steps) {
   if (int rc = cmc_ready(h)) return rc;
   return h->prec == VGPU_PREC_FP64 ? cmc_sweeps_typed<double>(h, n_steps) : cmc_sweeps_typed<float>(h, n_steps);
}

template <typename R>
static int cmc_pairs_typed(vgpu_handle h, const int32_t* pairs, int32_t K, const double* rnd, const double* M) {
   CMCState* c = cmc_of(h);
   const R* tab = mc_tables<R>(h);
   if (!tab) return VGPU_ERR_OOM;
   int rc = cuda_err(h, cudaMemcpyAsync(c->pairs, pairs, sizeof(int) * 2 * K, cudaMemcpyHostToDevice, h->stream),
                     "cmc pairs");
   if (!rc) rc = cuda_err(h, cudaMemcpyAsync(c->rnd, rnd, sizeof(double) * 4 * K, cudaMemcpyHostToDevice, h->stream),
                          "cmc pairs");
   if (!rc) {
      if (M) rc = cuda_err(h, cudaMemcpyAsync(c->M, M, sizeof(double) * 3, cudaMemcpyHostToDevice, h->stream), "cmc M");
      else rc = cmc_recount_moment<R>(h, tab, c->M, -1);
   }
   if (rc) return rc;
   // the explicit pairs are read back from c->pairs by the proposal kernel
   // (it rewrites the same values)
   rc = cmc_phase<R>(h, tab, nullptr, 0, c->pairs, K, c->rnd, 0, c->P, c->M);
   if (rc) return rc;
   return cuda_err(h, cudaStreamSynchronize(h->stream), "cmc pairs");
}

extern "C" int vgpu_cmc_pairs(vgpu_handle h, const int32_t* pairs, int32_t num_pairs, const double* rnd,
                              const double* moment) {
   if (int rc = cmc_ready(h)) return rc;
   CMCState* c = cmc_of(h);
   if (!pairs || !rnd || num_pairs <= 0 || num_pairs > c->maxK)
      return set_err(h, VGPU_ERR_ARG, "num_pairs must be in 1..%d with pairs and random numbers given", c->maxK);
   MCState* s = mc_of(h);
   for (int k = 0; k < 2 * num_pairs; ++k)
      if (pairs[k] < 0 || pairs[k] >= h->sys.n) return set_err(h, VGPU_ERR_ARG, "pair atom %d out of range", pairs[k]);
   // the pairs of one phase must not interact: all atoms of one colour, each at most once
   std::vector<char> seen(h->sys.n, 0);
   const int col = s->colour_host[pairs[0]];
   for (int k = 0; k < 2 * num_pairs; ++k) {
      if (s->colour_host[pairs[k]] != col) return set_err(h, VGPU_ERR_ARG, "pair atoms of different colours");
      if (seen[pairs[k]]++) return set_err(h, VGPU_ERR_ARG, "atom %d appears twice in one phase", pairs[k]);
   }
   return h->prec == VGPU_PREC_FP64 ? cmc_pairs_typed<double>(h, pairs, num_pairs, rnd, moment)
                                    : cmc_pairs_typed<float>(h, pairs, num_pairs, rnd, moment);
}

extern "C" int vgpu_cmc_get(vgpu_handle h, double* moment, double* counters) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   CMCState* c = cmc_of(h);
   if (!c) return set_err(h, VGPU_ERR_STATE, "vgpu_cmc_setup not called");
   cudaSetDevice(h->device);
   double M[3];
   unsigned long long cnt[4];
   cudaError_t e = cudaMemcpyAsync(M, c->M, sizeof M, cudaMemcpyDeviceToHost, h->stream);
   if (e == cudaSuccess) e = cudaMemcpyAsync(cnt, c->cnt, sizeof cnt, cudaMemcpyDeviceToHost, h->stream);
   if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
   if (e != cudaSuccess) return cuda_err(h, e, "cmc counters");
   if (moment) std::copy(M, M + 3, moment);
   if (counters) {
      // single-spin moves of unconstrained materials (hybrid) count as the
      // reference's: accepted, or energy rejections
      counters[0] = c->total;
      counters[1] = (double)cnt[0] + (c->single_moves - (double)cnt[3]);
      counters[2] = (double)(cnt[1] + cnt[3]);
      counters[3] = (double)cnt[2];
   }
   return VGPU_OK;
}
