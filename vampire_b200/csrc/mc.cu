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
// Random numbers: Philox counter (atom, sweep_lo, sweep_hi, RNG_MC_MOVE) gives
// the three Gaussians of the move, (.., RNG_MC_ACCEPT) the acceptance uniform;
// or, in replay mode, 4 host-supplied numbers per site and sweep.
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
   unsigned long long* rejects = nullptr;
   void* replay = nullptr;            // [4n] (x|y|z gaussians, uniform) in R
   bool use_replay = false;
   uint64_t sweep = 0;
   double moves = 0.0;
   int n_owned = 0;                   // atoms the sweeps visit (a shard's owned atoms)
   int next_colour = 0;               // vgpu_mc_colour: the colour of the current sweep to run next
};

static MCState* mc_of(vgpu_ctx* h) { return (MCState*)h->extras[1]; }

template <typename R>
struct MCArgs {
   LLGArgs<R> a;
   const int* atoms;
   int count;
   const R* sigma;      // [M] move width
   const R* beta;       // [M] mu_B / (kB T_rescaled)  (kBTBohr)
   const R* mu_ratio;   // [M] mu_s_SI / mu_B
   const R* replay;     // [4n] or nullptr
   uint64_t sweep;
   unsigned long long* rejects;
};

template <typename R>
__device__ __forceinline__ R site_energy_delta(const LLGArgs<R>& a, int i, const MatParams<R>& m, const R S[3],
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
   if (a.aniso_ext) d += anisotropy_energy<R, R, true>(a, i, m, T) - anisotropy_energy<R, R, true>(a, i, m, S);
   if (a.bq_off) d += biquadratic_energy<R, R>(a, i, T) - biquadratic_energy<R, R>(a, i, S);
   return d;
}

// Capped at 40 registers (6 blocks of 256 per SM instead of 5): the kernel
// is latency-bound on its gathers, and the extra warps outweigh the spilled
// registers (2.24e10 -> 2.51e10 spin-moves/s on the Curie protocol of SC 50^3
// x 31 temperatures; a cap at 32 spills more and gave 2.39e10).
template <typename R, int FMT>
__global__ void __launch_bounds__(256, 6) mc_colour_kernel(const MCArgs<R> p) {
   const int t = blockIdx.x * blockDim.x + threadIdx.x;
   bool rejected = false;
   if (t < p.count) {
      const LLGArgs<R>& a = p.a;
      const int i = __ldg(p.atoms + t);
      const int mi = a.mat ? __ldg(a.mat + i) : 0;
      const MatParams<R> m = a.mp[mi];
      R h[3] = {0, 0, 0};
      exchange_gather<R, FMT>(a, i, mi, a.ax, a.ay, a.az, h[0], h[1], h[2]);
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
         const u32x4 c2 = {gi, (uint32_t)p.sweep, (uint32_t)(p.sweep >> 32), RNG_MC_ACCEPT};
         const u32x4 r2 = philox4x32_10(c2, a.seed_lo, a.seed_hi);
         if (sizeof(R) == 4) {
            float s1, c1, s2, c2f;
            const float r1 = sqrtf(-2.0f * logf(u01f(r.x)));
            const float rr = sqrtf(-2.0f * logf(u01f(r.z)));
            sincospif(2.0f * u01f(r.y), &s1, &c1);
            sincospif(2.0f * u01f(r.w), &s2, &c2f);
            g0 = r1 * c1; g1 = r1 * s1; g2 = rr * c2f;
            u = (R)u01f(r2.x);
         } else {
            double s1, c1, s2, c2d;
            const double r1 = sqrt(-2.0 * log(u01d(r.x)));
            const double rr = sqrt(-2.0 * log(u01d(r.z)));
            sincospi(2.0 * u01d(r.y), &s1, &c1);
            sincospi(2.0 * u01d(r.w), &s2, &c2d);
            g0 = (R)(r1 * c1); g1 = (R)(r1 * s1); g2 = (R)(rr * c2d);
            u = (R)u01d(r2.x);
         }
      }
      const R sg = __ldg(p.sigma + mi);
      R T[3] = {S[0] + g0 * sg, S[1] + g1 * sg, S[2] + g2 * sg};
      const R r = rsqrt_<R>(T[0] * T[0] + T[1] * T[1] + T[2] * T[2]);
      T[0] *= r; T[1] *= r; T[2] *= r;
      const R dE = site_energy_delta<R>(a, i, m, S, T, h) * __ldg(p.mu_ratio + mi);
      bool accept = dE < (R)0;
      if (!accept) {
         const R x = -dE * __ldg(p.beta + mi);
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

template <typename R, int FMT>
static cudaError_t launch_mc(const MCArgs<R>& p, cudaStream_t st) {
   if (p.count == 0) return cudaSuccess;
   mc_colour_kernel<R, FMT><<<(p.count + 255) / 256, 256, 0, st>>>(p);
   return cudaGetLastError();
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

void mc_destroy(vgpu_ctx* h) {
   MCState* s = mc_of(h);
   if (!s) return;
   cudaFree(s->atoms);
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
   if ((e = cudaMalloc(&s->rejects, sizeof(unsigned long long))) != cudaSuccess) return cuda_err(h, e, "mc counter");
   cudaMemcpyAsync(s->atoms, order.data(), sizeof(int) * order.size(), cudaMemcpyHostToDevice, h->stream);
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
// into the handle's device table; returns it or nullptr (error set)
template <typename R>
static R* mc_tables(vgpu_handle h) {
   SysDev& S = h->sys;
   const int M = S.M;
   std::vector<R> sig(M), beta(M), ratio(M);
   for (int m = 0; m < M; ++m) {
      const vgpu_material& q = S.materials[m];
      const double T = h->params.local_temperature ? q.temperature : h->params.temperature;
      const double al = q.temperature_rescaling_alpha, Tc = q.temperature_rescaling_Tc;
      const double Tr = T < Tc ? Tc * std::pow(T / Tc, al) : T;
      const double kBTBohr = 9.27400915e-24 / (Tr * 1.3806503e-23);
      sig[m] = (R)(Tr < 1.0 ? 0.02 : std::pow(1.0 / kBTBohr, 0.2) * 0.08);
      beta[m] = (R)kBTBohr;
      ratio[m] = (R)(q.mu_s_SI * 1.07828231e23);
   }
   if (!S.mc_tab) {
      S.mc_tab = h->alloc(3 * 100 * sizeof(double));
      if (!S.mc_tab) {
         set_err(h, VGPU_ERR_OOM, "mc tables");
         return nullptr;
      }
   }
   R* tab = (R*)S.mc_tab;
   cudaMemcpyAsync(tab, sig.data(), M * sizeof(R), cudaMemcpyHostToDevice, h->stream);
   cudaMemcpyAsync(tab + 100, beta.data(), M * sizeof(R), cudaMemcpyHostToDevice, h->stream);
   cudaMemcpyAsync(tab + 200, ratio.data(), M * sizeof(R), cudaMemcpyHostToDevice, h->stream);
   return tab;
}

// one colour of the current sweep; the last colour completes the sweep
template <typename R>
static int mc_run_colour(vgpu_handle h, const R* tab, int c) {
   MCState* s = mc_of(h);
   SysDev& S = h->sys;
   MCArgs<R> p;
   memset(&p, 0, sizeof p);
   p.a = make_args<R>(h);
   p.sigma = tab;
   p.beta = tab + 100;
   p.mu_ratio = tab + 200;
   p.replay = s->use_replay ? (const R*)s->replay : nullptr;
   p.sweep = s->sweep;
   p.rejects = s->rejects;
   p.atoms = s->atoms + s->colour_off[c];
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
