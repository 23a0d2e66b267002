// Many independent spin systems of uneven sizes in one persistent launch.
//
// No counterpart in the reference, which runs one system per process.  A batch
// (e.g. 256 nanoparticles of 150-10,000 spins, each with its own temperature
// and field sweep) is held as ONE device system: the systems' atoms are
// concatenated, their materials are replicated per system (so a material row
// carries the system's temperature and its linear field sweep), and the
// Philox stream of system k is that of a single run seeded seed + k with the
// atom's index inside its system -- a batched run draws exactly the numbers
// the same system run alone would.
//
// Persistent kernel: the grid is the number of co-resident thread-block
// clusters times the cluster size C.  Systems are bin-packed (longest first)
// onto the clusters; a cluster owns whole systems, so the only
// synchronisation a Heun step needs -- predictor done before the corrector
// reads s' -- is between the CTAs of one cluster, done with the hardware
// cluster barrier (barrier.cluster arrive/wait, release/acquire).  There is no
// grid-wide barrier and no spin-wait.  Neighbour spins written in the same
// launch are read through L2 (ld.global.cg).  One launch runs S steps; a CUDA
// graph holds {persistent kernel, per-system magnetisation record, step
// advance} and is replayed.  Cluster size and block size come from an
// autotuner that times the candidates on the batch itself.
//
// Shape cluster = 0 runs the batch as the one system it is, with the
// ordinary two step passes per step over all atoms (vgpu_llg_heun) and the
// same per-system records between chunks.  No system is tied to one cluster,
// so the largest particle no longer sets the step time: on 256 particles of
// 150-10,000 spins (380,178 in all) 0.021 ms per step (the passes launched
// with programmatic serialisation) against 0.045 ms for the best persistent
// shape (cluster 8, blocks of 128).  The passes take the step number as a
// kernel argument, so this shape is not captured in a graph.
// Same physics and numbers as the persistent kernel (tests/test_batch_gpu.py).
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "llg_kernels.cuh"
#include "vgpu_ctx.cuh"

namespace cg = cooperative_groups;

namespace vgpu {

struct BatchState {
   int n_sys = 0;
   int m_per_sys = 1;
   std::vector<int> off;             // [n_sys+1] first atom of each system
   int* d_off = nullptr;
   // cluster work lists
   int cluster = 1, block = 256, groups = 0;
   int* d_grp_start = nullptr;       // [groups+1]
   int* d_grp_sys = nullptr;         // [n_sys] systems in group order
   // device step counter and magnetisation history
   unsigned long long* d_step = nullptr;
   unsigned long long* d_rec = nullptr;
   double* d_hist = nullptr;         // [cap][n_sys][4]
   long long hist_cap = 0;
   cudaGraphExec_t graph = nullptr;
   int graph_steps = 0, graph_cluster = 0, graph_block = 0;
   std::vector<double> ramp;         // [M_total*3] field change over the sweep
   uint64_t ramp_n = 0;
};

static BatchState* batch_of(vgpu_ctx* h) { return (BatchState*)h->extras[3]; }

template <typename R, int FMT>
__global__ void batch_persistent_kernel(LLGArgs<R> a, const int* __restrict__ grp_start,
                                        const int* __restrict__ grp_sys, const int* __restrict__ off, int nsteps,
                                        const unsigned long long* __restrict__ step_base) {
   cg::cluster_group cl = cg::this_cluster();
   const int C = (int)cl.num_blocks();
   const int g = blockIdx.x / C;
   const int t = (int)cl.block_rank() * blockDim.x + threadIdx.x;
   const int stride = C * blockDim.x;
   const uint64_t step0 = *step_base;
   const int q0 = grp_start[g], q1 = grp_start[g + 1];
   for (int s = 0; s < nsteps; ++s) {
      a.step = step0 + (uint64_t)s;
      for (int q = q0; q < q1; ++q) {
         const int k = grp_sys[q];
         for (int i = off[k] + t; i < off[k + 1]; i += stride) llg_predict_atom<R, FMT, 1, VAR_HEUN>(a, i);
      }
      cl.sync();  // every s' of the cluster's systems written and visible
      for (int q = q0; q < q1; ++q) {
         const int k = grp_sys[q];
         for (int i = off[k] + t; i < off[k + 1]; i += stride) llg_correct_atom<R, FMT, 1, VAR_HEUN>(a, i);
      }
      cl.sync();  // s1 complete before the next predictor gathers it
   }
}

// per-system magnetisation (m_hat, |m|/m_sat) into the history
template <typename R>
__global__ void batch_record_kernel(int n_sys, const int* __restrict__ off, const R* __restrict__ sx,
                                    const R* __restrict__ sy, const R* __restrict__ sz, const int* __restrict__ mat,
                                    const MatParams<R>* __restrict__ mp, unsigned long long* __restrict__ rec,
                                    long long cap, double* __restrict__ hist) {
   const int k = blockIdx.x;
   if (k >= n_sys) return;
   const unsigned long long r = *rec;
   double m[4] = {0, 0, 0, 0};
   for (int i = off[k] + threadIdx.x; i < off[k + 1]; i += blockDim.x) {
      const double mu = (double)mp[mat ? mat[i] : 0].mu_s_muB;
      m[0] += (double)sx[i] * mu; m[1] += (double)sy[i] * mu; m[2] += (double)sz[i] * mu; m[3] += mu;
   }
   __shared__ double red[4][256];
   for (int q = 0; q < 4; ++q) red[q][threadIdx.x] = m[q];
   __syncthreads();
   for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s)
         for (int q = 0; q < 4; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + s];
      __syncthreads();
   }
   if (threadIdx.x == 0 && (long long)r < cap) {
      const double mx = red[0][0], my = red[1][0], mz = red[2][0], ms = red[3][0];
      const double mm = sqrt(mx * mx + my * my + mz * mz);
      double* o = hist + ((size_t)r * n_sys + k) * 4;
      o[0] = mm > 0 ? mx / mm : 0.0; o[1] = mm > 0 ? my / mm : 0.0; o[2] = mm > 0 ? mz / mm : 0.0;
      o[3] = ms > 0 ? mm / ms : 0.0;
   }
}

__global__ void batch_advance_kernel(unsigned long long* step, unsigned long long* rec, int nsteps, int record) {
   *step += (unsigned long long)nsteps;
   if (record) *rec += 1ull;
}

void batch_destroy(vgpu_ctx* h) {
   BatchState* b = batch_of(h);
   if (!b) return;
   if (b->graph) cudaGraphExecDestroy(b->graph);
   cudaFree(b->d_off); cudaFree(b->d_grp_start); cudaFree(b->d_grp_sys);
   cudaFree(b->d_step); cudaFree(b->d_rec); cudaFree(b->d_hist);
   delete b;
   h->extras[3] = nullptr;
   h->sys.sys_off = nullptr;
}

template <typename R, int FMT>
static cudaError_t launch_persistent(vgpu_ctx* h, const LLGArgs<R>& a, int nsteps) {
   BatchState* b = batch_of(h);
   cudaLaunchConfig_t cfg;
   std::memset(&cfg, 0, sizeof cfg);
   cfg.gridDim = dim3(b->groups * b->cluster);
   cfg.blockDim = dim3(b->block);
   cfg.stream = h->stream;
   cudaLaunchAttribute attr[1];
   attr[0].id = cudaLaunchAttributeClusterDimension;
   attr[0].val.clusterDim.x = b->cluster;
   attr[0].val.clusterDim.y = 1;
   attr[0].val.clusterDim.z = 1;
   cfg.attrs = attr;
   cfg.numAttrs = 1;
   return cudaLaunchKernelEx(&cfg, batch_persistent_kernel<R, FMT>, a, (const int*)b->d_grp_start,
                             (const int*)b->d_grp_sys, (const int*)b->d_off, nsteps,
                             (const unsigned long long*)b->d_step);
}

template <typename R>
static cudaError_t launch_persistent_fmt(vgpu_ctx* h, const LLGArgs<R>& a, int nsteps) {
   switch (h->sys.fmt) {
      case FMT_ISO_TAB: return launch_persistent<R, FMT_ISO_TAB>(h, a, nsteps);
      case FMT_ISO_BOND: return launch_persistent<R, FMT_ISO_BOND>(h, a, nsteps);
      case FMT_VEC_TAB: return launch_persistent<R, FMT_VEC_TAB>(h, a, nsteps);
      case FMT_VEC_BOND: return launch_persistent<R, FMT_VEC_BOND>(h, a, nsteps);
      case FMT_DMI_TAB: return launch_persistent<R, FMT_DMI_TAB>(h, a, nsteps);
      default: return launch_persistent<R, FMT_TENSOR_BOND>(h, a, nsteps);
   }
}

template <typename R>
static const void* persistent_fn(int fmt) {
   switch (fmt) {
      case FMT_ISO_TAB: return (const void*)batch_persistent_kernel<R, FMT_ISO_TAB>;
      case FMT_ISO_BOND: return (const void*)batch_persistent_kernel<R, FMT_ISO_BOND>;
      case FMT_VEC_TAB: return (const void*)batch_persistent_kernel<R, FMT_VEC_TAB>;
      case FMT_VEC_BOND: return (const void*)batch_persistent_kernel<R, FMT_VEC_BOND>;
      case FMT_DMI_TAB: return (const void*)batch_persistent_kernel<R, FMT_DMI_TAB>;
      default: return (const void*)batch_persistent_kernel<R, FMT_TENSOR_BOND>;
   }
}

// Bin-pack systems onto `groups` clusters, longest first (LPT).
static void pack(const std::vector<int>& off, int groups, std::vector<int>& gstart, std::vector<int>& gsys) {
   const int n = (int)off.size() - 1;
   std::vector<int> order(n);
   std::iota(order.begin(), order.end(), 0);
   std::sort(order.begin(), order.end(), [&](int a, int b) { return off[a + 1] - off[a] > off[b + 1] - off[b]; });
   std::vector<long long> load(groups, 0);
   std::vector<std::vector<int>> lists(groups);
   for (int k : order) {
      const int g = (int)(std::min_element(load.begin(), load.end()) - load.begin());
      lists[g].push_back(k);
      load[g] += off[k + 1] - off[k];
   }
   gstart.assign(groups + 1, 0);
   gsys.clear();
   for (int g = 0; g < groups; ++g) {
      gstart[g + 1] = gstart[g] + (int)lists[g].size();
      gsys.insert(gsys.end(), lists[g].begin(), lists[g].end());
   }
}

template <typename R>
static int set_shape_typed(vgpu_ctx* h, int cluster, int block) {
   BatchState* b = batch_of(h);
   if (cluster == 0) {  // the ordinary step passes (block size is theirs)
      b->cluster = 0;
      b->block = 0;
      return VGPU_OK;
   }
   if (cluster < 1 || cluster > 8 || (cluster & (cluster - 1)))
      return set_err(h, VGPU_ERR_ARG, "cluster size must be 0, 1, 2, 4 or 8 (got %d)", cluster);
   if (block < 64 || block > 1024 || block % 32) return set_err(h, VGPU_ERR_ARG, "bad block size %d", block);
   cudaLaunchConfig_t cfg;
   std::memset(&cfg, 0, sizeof cfg);
   cfg.gridDim = dim3(cluster);
   cfg.blockDim = dim3(block);
   cudaLaunchAttribute attr[1];
   attr[0].id = cudaLaunchAttributeClusterDimension;
   attr[0].val.clusterDim.x = cluster;
   attr[0].val.clusterDim.y = 1;
   attr[0].val.clusterDim.z = 1;
   cfg.attrs = attr;
   cfg.numAttrs = 1;
   int nclusters = 0;
   cudaError_t e = cudaOccupancyMaxActiveClusters(&nclusters, persistent_fn<R>(h->sys.fmt), &cfg);
   if (e != cudaSuccess) return cuda_err(h, e, "cudaOccupancyMaxActiveClusters");
   if (nclusters <= 0) return set_err(h, VGPU_ERR_ARG, "shape cluster=%d block=%d cannot be resident", cluster, block);
   const int groups = std::min(nclusters, b->n_sys);
   std::vector<int> gstart, gsys;
   pack(b->off, groups, gstart, gsys);
   cudaFree(b->d_grp_start);
   cudaFree(b->d_grp_sys);
   b->d_grp_start = nullptr;
   b->d_grp_sys = nullptr;
   if ((e = cudaMalloc(&b->d_grp_start, sizeof(int) * gstart.size())) != cudaSuccess) return cuda_err(h, e, "batch");
   if ((e = cudaMalloc(&b->d_grp_sys, sizeof(int) * gsys.size())) != cudaSuccess) return cuda_err(h, e, "batch");
   cudaMemcpyAsync(b->d_grp_start, gstart.data(), sizeof(int) * gstart.size(), cudaMemcpyHostToDevice, h->stream);
   cudaMemcpyAsync(b->d_grp_sys, gsys.data(), sizeof(int) * gsys.size(), cudaMemcpyHostToDevice, h->stream);
   if ((e = cudaStreamSynchronize(h->stream)) != cudaSuccess) return cuda_err(h, e, "batch shape");
   b->cluster = cluster;
   b->block = block;
   b->groups = groups;
   return VGPU_OK;
}

int batch_set_shape(vgpu_ctx* h, int cluster, int block) {
   return h->prec == VGPU_PREC_FP64 ? set_shape_typed<double>(h, cluster, block)
                                    : set_shape_typed<float>(h, cluster, block);
}

template <typename R>
static int run_chunk_typed(vgpu_ctx* h, int nsteps, int record) {
   BatchState* b = batch_of(h);
   if (b->cluster == 0) {
      // the step passes (they advance h->step themselves)
      if (int rc = vgpu_llg_heun(h, (uint64_t)nsteps)) return rc;
   } else {
      LLGArgs<R> a = make_args<R>(h);
      h->prof_begin(PROF_PREDICTOR);
      cudaError_t e = launch_persistent_fmt<R>(h, a, nsteps);
      h->prof_end(PROF_PREDICTOR);
      if (e != cudaSuccess) return cuda_err(h, e, "persistent batch launch");
   }
   if (record) {
      batch_record_kernel<R><<<b->n_sys, 256, 0, h->stream>>>(
          b->n_sys, b->d_off, (const R*)h->sys.s[0], (const R*)h->sys.s[1], (const R*)h->sys.s[2],
          (const int*)h->sys.mat, (const MatParams<R>*)h->sys.mp, b->d_rec, b->hist_cap, b->d_hist);
   }
   batch_advance_kernel<<<1, 1, 0, h->stream>>>(b->d_step, b->d_rec, nsteps, record);
   h->kernel_launches += (b->cluster == 0 ? 1 : 2) + record;  // the step passes count their own
   return cuda_err(h, cudaGetLastError(), "batch launch");
}

template <typename R>
static int run_typed(vgpu_ctx* h, uint64_t n_steps, uint32_t record_every, int use_graph) {
   BatchState* b = batch_of(h);
   const int S = record_every > 0 ? (int)record_every : (int)std::min<uint64_t>(n_steps, 1000);
   const uint64_t chunks = S > 0 ? n_steps / S : 0;
   const int rem = (int)(n_steps - chunks * (uint64_t)S);
   const int record = record_every > 0;
   // history buffer for this run
   if (record) {
      const long long need = (long long)chunks;
      if (need > b->hist_cap) {
         cudaFree(b->d_hist);
         b->d_hist = nullptr;
         cudaError_t e = cudaMalloc(&b->d_hist, sizeof(double) * 4 * (size_t)b->n_sys * std::max(1LL, need));
         if (e != cudaSuccess) return cuda_err(h, e, "batch history");
         b->hist_cap = std::max(1LL, need);
      }
   }
   cudaMemcpyAsync(b->d_step, &h->step, sizeof(uint64_t), cudaMemcpyHostToDevice, h->stream);
   cudaMemsetAsync(b->d_rec, 0, sizeof(unsigned long long), h->stream);
   if (b->cluster == 0) {  // step passes: h->step advances with every step
      for (uint64_t c = 0; c < chunks; ++c)
         if (int rc = run_chunk_typed<R>(h, S, record)) return rc;
      if (rem > 0)
         if (int rc = run_chunk_typed<R>(h, rem, 0)) return rc;
      return VGPU_OK;
   }
   if (use_graph && chunks > 0) {
      if (!b->graph || b->graph_steps != S || b->graph_cluster != b->cluster || b->graph_block != b->block) {
         if (b->graph) { cudaGraphExecDestroy(b->graph); b->graph = nullptr; }
         cudaGraph_t g;
         cudaError_t e = cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal);
         if (e != cudaSuccess) return cuda_err(h, e, "graph capture");
         const bool prof = h->prof_on;
         h->prof_on = false;
         const int64_t kl = h->kernel_launches;
         int rc = run_chunk_typed<R>(h, S, record);
         h->kernel_launches = kl;
         h->prof_on = prof;
         e = cudaStreamEndCapture(h->stream, &g);
         if (rc) return rc;
         if (e != cudaSuccess) return cuda_err(h, e, "graph capture");
         e = cudaGraphInstantiate(&b->graph, g, 0);
         cudaGraphDestroy(g);
         if (e != cudaSuccess) return cuda_err(h, e, "graph instantiate");
         b->graph_steps = S;
         b->graph_cluster = b->cluster;
         b->graph_block = b->block;
      }
      for (uint64_t c = 0; c < chunks; ++c) {
         h->prof_begin(PROF_OTHER);
         cudaError_t e = cudaGraphLaunch(b->graph, h->stream);
         h->prof_end(PROF_OTHER);
         if (e != cudaSuccess) return cuda_err(h, e, "graph launch");
         h->kernel_launches += 2 + record;
      }
   } else {
      for (uint64_t c = 0; c < chunks; ++c) {
         int rc = run_chunk_typed<R>(h, S, record);
         if (rc) return rc;
      }
   }
   if (rem > 0) {
      int rc = run_chunk_typed<R>(h, rem, 0);
      if (rc) return rc;
   }
   h->step += n_steps;
   return VGPU_OK;
}

}  // namespace vgpu

using namespace vgpu;

extern "C" int vgpu_batch_create(int device, int precision, int32_t n_sys, const vgpu_system_desc* descs,
                                 const vgpu_batch_system* systems, const vgpu_sim_params* common,
                                 vgpu_handle* out) {
   if (!out || !descs || !systems || !common || n_sys <= 0)
      return set_err(nullptr, VGPU_ERR_ARG, "bad batch arguments");
   *out = nullptr;
   const int M = descs[0].num_materials;
   for (int k = 0; k < n_sys; ++k) {
      int rc = vgpu_validate_system(&descs[k]);
      if (rc) return rc;
      if (descs[k].num_materials != M || descs[k].exchange_type != descs[0].exchange_type)
         return set_err(nullptr, VGPU_ERR_ARG, "batched systems must share material count and exchange type");
   }
   if ((int64_t)n_sys * M > 65536) return set_err(nullptr, VGPU_ERR_ARG, "too many systems x materials");
   // concatenate
   std::vector<int> off(n_sys + 1, 0);
   int64_t nb = 0;
   for (int k = 0; k < n_sys; ++k) {
      off[k + 1] = off[k] + descs[k].num_atoms;
      nb += descs[k].num_bonds;
   }
   const int n = off[n_sys];
   const int w = descs[0].exchange_type == VGPU_EXCH_ISOTROPIC ? 1 : descs[0].exchange_type == VGPU_EXCH_VECTORIAL ? 3 : 9;
   std::vector<int> st(n), en(n), nl, type(n);
   std::vector<double> jl, sx(n), sy(n), sz(n);
   nl.reserve(nb);
   jl.reserve(nb * w);
   std::vector<vgpu_material> mats((size_t)n_sys * M);
   std::vector<double> ramp((size_t)n_sys * M * 3, 0.0);
   for (int k = 0; k < n_sys; ++k) {
      const vgpu_system_desc& d = descs[k];
      const int o = off[k];
      for (int i = 0; i < d.num_atoms; ++i) {
         st[o + i] = (int)nl.size();
         for (int64_t bnd = d.nl_start[i]; bnd <= d.nl_end[i]; ++bnd) {
            nl.push_back(o + d.nl[bnd]);
            const int64_t id = d.nl_type ? d.nl_type[bnd] : bnd;
            for (int q = 0; q < w; ++q) jl.push_back(d.jlist[w * id + q]);
         }
         en[o + i] = (int)nl.size() - 1;
         type[o + i] = k * M + d.type[i];
         sx[o + i] = d.sx[i]; sy[o + i] = d.sy[i]; sz[o + i] = d.sz[i];
      }
      const vgpu_batch_system& p = systems[k];
      for (int m = 0; m < M; ++m) {
         vgpu_material q = d.materials[m];
         q.temperature = p.temperature;
         for (int c = 0; c < 3; ++c) {
            q.applied_field[c] = p.H_start[c];
            ramp[((size_t)k * M + m) * 3 + c] = p.H_end[c] - p.H_start[c];
         }
         mats[(size_t)k * M + m] = q;
      }
   }
   vgpu_system_desc cd;
   std::memset(&cd, 0, sizeof cd);
   cd.num_atoms = n;
   cd.num_materials = n_sys * M;
   cd.exchange_type = descs[0].exchange_type;
   cd.uniaxial_enabled = descs[0].uniaxial_enabled;
   cd.cubic_enabled = descs[0].cubic_enabled;
   cd.num_bonds = (int64_t)nl.size();
   cd.nl_start = st.data();
   cd.nl_end = en.data();
   cd.nl = nl.data();
   cd.num_exchange = cd.num_bonds;
   cd.jlist = jl.data();
   cd.type = type.data();
   cd.materials = mats.data();
   cd.sx = sx.data(); cd.sy = sy.data(); cd.sz = sz.data();
   vgpu_handle h = nullptr;
   int rc = vgpu_create(device, precision, &h);
   if (rc) return rc;
   h->batch_materials = true;
   rc = vgpu_upload_system(h, &cd);
   if (rc) { char buf[512]; vgpu_last_error(h, buf, sizeof buf); set_err(nullptr, rc, "%s", buf); vgpu_destroy(h); return rc; }
   BatchState* b = new BatchState();
   h->extras[3] = b;
   b->n_sys = n_sys;
   b->m_per_sys = M;
   b->off = off;
   b->ramp = ramp;
   uint64_t nr = 0;
   for (int k = 0; k < n_sys; ++k) nr = std::max<uint64_t>(nr, systems[k].n_ramp);
   b->ramp_n = nr;
   cudaError_t e = cudaMalloc(&b->d_off, sizeof(int) * (n_sys + 1));
   if (e == cudaSuccess) e = cudaMemcpy(b->d_off, off.data(), sizeof(int) * (n_sys + 1), cudaMemcpyHostToDevice);
   if (e == cudaSuccess) e = cudaMalloc(&b->d_step, sizeof(unsigned long long));
   if (e == cudaSuccess) e = cudaMalloc(&b->d_rec, sizeof(unsigned long long));
   if (e != cudaSuccess) { rc = cuda_err(nullptr, e, "batch setup"); vgpu_destroy(h); return rc; }
   h->sys.sys_off = b->d_off;
   h->sys.m_per_sys = M;
   h->sys.ramp_n = nr;
   vgpu_sim_params p = *common;
   p.local_temperature = 1;
   p.local_applied_field = 1;
   rc = vgpu_set_params(h, &p);
   if (!rc) rc = batch_set_shape(h, 1, 256);
   if (rc) { char buf[512]; vgpu_last_error(h, buf, sizeof buf); set_err(nullptr, rc, "%s", buf); vgpu_destroy(h); return rc; }
   *out = h;
   return VGPU_OK;
}

extern "C" int vgpu_batch_set_shape(vgpu_handle h, int32_t cluster, int32_t block) {
   if (!h || !batch_of(h)) return set_err(h, VGPU_ERR_STATE, "not a batch handle");
   cudaSetDevice(h->device);
   return batch_set_shape(h, cluster, block);
}

extern "C" int vgpu_batch_run(vgpu_handle h, uint64_t n_steps, uint32_t record_every, int32_t use_graph) {
   if (!h || !batch_of(h)) return set_err(h, VGPU_ERR_STATE, "not a batch handle");
   cudaSetDevice(h->device);
   return h->prec == VGPU_PREC_FP64 ? run_typed<double>(h, n_steps, record_every, use_graph)
                                    : run_typed<float>(h, n_steps, record_every, use_graph);
}

extern "C" int vgpu_batch_autotune(vgpu_handle h, int32_t trial_steps, int32_t* cluster_out, int32_t* block_out,
                                   double* ms_per_step_out) {
   BatchState* b = h ? batch_of(h) : nullptr;
   if (!b) return set_err(h, VGPU_ERR_STATE, "not a batch handle");
   if (trial_steps <= 0) return set_err(h, VGPU_ERR_ARG, "trial_steps must be positive");
   cudaSetDevice(h->device);
   // the trials advance the state: keep and restore spins and the step counter
   const size_t rs = h->prec == VGPU_PREC_FP64 ? sizeof(double) : sizeof(float);
   const size_t bytes = rs * h->sys.n_alloc;
   std::vector<void*> save(3, nullptr);
   for (int q = 0; q < 3; ++q) {
      cudaError_t e = cudaMalloc(&save[q], bytes);
      if (e != cudaSuccess) {
         for (void* p : save) cudaFree(p);
         return cuda_err(h, e, "autotune backup");
      }
      cudaMemcpyAsync(save[q], h->sys.s[q], bytes, cudaMemcpyDeviceToDevice, h->stream);
   }
   const uint64_t step0 = h->step;
   const int clusters[5] = {0, 1, 2, 4, 8};
   const int blocks[3] = {128, 256, 512};
   double best = 1e300;
   int bc = 1, bb = 256;
   cudaEvent_t e0, e1;
   cudaEventCreate(&e0);
   cudaEventCreate(&e1);
   for (int c : clusters)
      for (int bl : blocks) {
         if (c == 0 && bl != blocks[0]) continue;  // the step passes: one candidate
         if (batch_set_shape(h, c, c == 0 ? 0 : bl) != VGPU_OK) continue;
         if (vgpu_batch_run(h, 2, 0, 0) != VGPU_OK) continue;  // warm-up
         cudaEventRecord(e0, h->stream);
         if (vgpu_batch_run(h, trial_steps, 0, 0) != VGPU_OK) continue;
         cudaEventRecord(e1, h->stream);
         cudaEventSynchronize(e1);
         float ms = 0.f;
         cudaEventElapsedTime(&ms, e0, e1);
         if (ms < best) { best = ms; bc = c; bb = c == 0 ? 0 : bl; }
      }
   cudaEventDestroy(e0);
   cudaEventDestroy(e1);
   for (int q = 0; q < 3; ++q) {
      cudaMemcpyAsync(h->sys.s[q], save[q], bytes, cudaMemcpyDeviceToDevice, h->stream);
   }
   cudaStreamSynchronize(h->stream);
   for (void* p : save) cudaFree(p);
   h->step = step0;
   int rc = batch_set_shape(h, bc, bb);
   if (rc) return rc;
   if (cluster_out) *cluster_out = bc;
   if (block_out) *block_out = bb;
   if (ms_per_step_out) *ms_per_step_out = best / trial_steps;
   return VGPU_OK;
}

extern "C" int vgpu_batch_history(vgpu_handle h, double* out, int64_t max_records, int64_t* n_records) {
   BatchState* b = h ? batch_of(h) : nullptr;
   if (!b) return set_err(h, VGPU_ERR_STATE, "not a batch handle");
   cudaSetDevice(h->device);
   unsigned long long r = 0;
   cudaError_t e = cudaMemcpyAsync(&r, b->d_rec, sizeof r, cudaMemcpyDeviceToHost, h->stream);
   if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
   if (e != cudaSuccess) return cuda_err(h, e, "batch history");
   const long long avail = std::min<long long>((long long)r, b->hist_cap);
   const long long m = std::min<long long>(avail, max_records);
   if (out && m > 0) {
      e = cudaMemcpyAsync(out, b->d_hist, sizeof(double) * 4 * b->n_sys * (size_t)m, cudaMemcpyDeviceToHost,
                          h->stream);
      if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
      if (e != cudaSuccess) return cuda_err(h, e, "batch history");
   }
   if (n_records) *n_records = avail;
   return VGPU_OK;
}

extern "C" int vgpu_batch_system_range(vgpu_handle h, int32_t k, int32_t* first_atom, int32_t* num_atoms) {
   BatchState* b = h ? batch_of(h) : nullptr;
   if (!b) return set_err(h, VGPU_ERR_STATE, "not a batch handle");
   if (k < 0 || k >= b->n_sys) return set_err(h, VGPU_ERR_ARG, "system %d out of range", k);
   if (first_atom) *first_atom = b->off[k];
   if (num_atoms) *num_atoms = b->off[k + 1] - b->off[k];
   return VGPU_OK;
}

// field sweep of every material row (refresh_materials reads it)
const double* vgpu::batch_ramp(vgpu_ctx* h) {
   BatchState* b = batch_of(h);
   return b ? b->ramp.data() : nullptr;
}
