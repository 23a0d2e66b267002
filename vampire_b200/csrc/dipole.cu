// Macrocell dipole field: K5 cell moments and K6 cell-cell field.
//
// Reference: dipole::calculate_field (src/dipole/field.cpp:43-141) ->
// cells::mag (src/cells/mag.cpp:35-77) -> dipole::internal::update_field
// (src/dipole/update.cpp:37-105), with the interaction tensors of the tensor
// solver (src/dipole/tensor.cpp:40, inter.cpp:40-150, intra.cpp:40-140) or the
// macrocell solver (src/dipole/macrocell.cpp:175-225).  The reference stores
// six dense Nc x Nc FP64 matrices (src/dipole/memory.cpp:29-56), 750 GB at
// 125,000 cells; its GPU version is disabled.  Here nothing dense is stored:
//
//   K5  one warp per cell sums mu_s s over the cell's atoms (cell-sorted atom
//       list, FP64), giving the cell moments in J/T and in mu_B for K6;
//   K6  every target cell runs over all source cells in 256-cell shared-memory
//       tiles and adds the bare point-dipole term (3 e e - 1)/r^3 m_j in FP32,
//       folding each tile's sum into FP64;
//   K6n for the pairs within `cutoff` macrocell sizes (tensor solver) the
//       atomistic tensors of inter.cpp/intra.cpp minus the bare term are
//       precomputed once in FP64 (one block per pair) and added in FP64.
//
// B = 0.9274 sum_j T_ij m_j (self term times 0) and mu0 Hd = 0.9274 (sum_j
// T_ij m_j - 0.5 (8 pi / 3 V_i) m_i), as update.cpp:56-99.  Atoms read their
// cell's field through the cell id in the fused LLG passes; atoms of
// non-magnetic materials and of empty cells read a zero row.
//
// On a shard (vgpu_set_owned) K5 sums the shard's owned atoms only and the
// update stops there: the host adds the partial cell moments over ranks in
// the device buffer (the reference's MPI_Allreduce of cells::mag_array,
// src/cells/mag.cpp:69-74) and vgpu_dipole_finish runs K6 on the sums.  Until
// then the passes, statistics and Monte Carlo refuse to run.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <unordered_map>
#include <vector>

#include "dipole_fft.cuh"
#include "vgpu_ctx.cuh"

namespace vgpu {

struct DipoleState {
   int nc = 0;
   int solver = 1;
   int update_rate = 100;
   double size = 0.0, cutoff = 2.0;
   int* cell_start = nullptr;   // [nc+1] offsets into cell_atoms
   int* cell_atoms = nullptr;   // atoms sorted by cell (magnetic atoms only)
   double* mag = nullptr;       // [3][nc] cell moment, J/T
   float4* pos = nullptr;       // [nc] centre (Angstrom), w = 1 if the cell has atoms
   float4* mom = nullptr;       // [nc] moment in mu_B
   double* field = nullptr;     // [6][nc] B (3) and mu0 Hd (3), FP64
   double* self = nullptr;      // [nc] 8 pi / (3 V)
   int* near_start = nullptr;   // [nc+1]
   int* near_j = nullptr;       // [npairs]
   double* near_t = nullptr;    // [6][npairs] T_near - T_bare (xx, xy, xz, yy, yz, zz)
   int npairs = 0;
   // the near pairs in ELL form for the finish kernel: pair k of cell i at
   // [k][i] (near_je) and [q][k][i] (near_te, q = xx, xy, xz, yy, yz, zz), so
   // that a warp of consecutive cells reads consecutive addresses; cells keep
   // their pairs in the CSR order (sorted by source cell)
   int maxp = 0;
   int* near_cnt = nullptr;     // [nc] pairs per cell
   int* near_je = nullptr;      // [maxp][nc]
   double* near_te = nullptr;   // [6][maxp][nc]
   void* table_b = nullptr;     // [3][nc+1] R, cell B field for the LLG passes
   void* table_hd = nullptr;    // [3][nc+1] R, cell mu0 Hd field (energies)
   int* atom_cell = nullptr;    // [n] cell id or nc (zero row)
   FFTField* fft = nullptr;     // far field by FFT convolution (regular cell grids), or direct sum
   std::vector<double> mus_host;
   bool shard = false;          // K5 sums owned atoms; the field waits for the sum over ranks
   bool pending = false;        // partial moments in `mag`, field not yet computed
};

static DipoleState* dip_of(vgpu_ctx* h) { return (DipoleState*)h->extras[2]; }

// K5: cell moments (cells.cpp mag()), FP64.
template <typename R>
__global__ void cell_moment_kernel(int nc, const int* __restrict__ start, const int* __restrict__ atoms,
                                   const R* __restrict__ sx, const R* __restrict__ sy, const R* __restrict__ sz,
                                   const int* __restrict__ mat, const MatParams<R>* __restrict__ mp,
                                   const double* __restrict__ mus_SI, double* __restrict__ mag,
                                   const float4* __restrict__ pos, float4* __restrict__ mom) {
   const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
   const int lane = threadIdx.x & 31;
   if (warp >= nc) return;
   double mx = 0.0, my = 0.0, mz = 0.0;
   for (int k = start[warp] + lane; k < start[warp + 1]; k += 32) {
      const int i = atoms[k];
      const double mu = mus_SI[mat ? mat[i] : 0];
      mx += (double)sx[i] * mu;
      my += (double)sy[i] * mu;
      mz += (double)sz[i] * mu;
   }
#pragma unroll
   for (int o = 16; o > 0; o >>= 1) {
      mx += __shfl_xor_sync(0xffffffffu, mx, o);
      my += __shfl_xor_sync(0xffffffffu, my, o);
      mz += __shfl_xor_sync(0xffffffffu, mz, o);
   }
   if (lane == 0) {
      mag[warp] = mx; mag[nc + warp] = my; mag[2 * nc + warp] = mz;
      const double imuB = 1.0 / 9.27400915e-24;
      mom[warp] = make_float4((float)(mx * imuB), (float)(my * imuB), (float)(mz * imuB), 0.f);
   }
}

// moments in mu_B for K6 from the cell moments summed over ranks
__global__ void cell_mom_kernel(int nc, const double* __restrict__ mag, float4* __restrict__ mom) {
   const int c = blockIdx.x * blockDim.x + threadIdx.x;
   if (c >= nc) return;
   const double imuB = 1.0 / 9.27400915e-24;
   mom[c] = make_float4((float)(mag[c] * imuB), (float)(mag[nc + c] * imuB), (float)(mag[2 * nc + c] * imuB), 0.f);
}

// K6: far field by tiled all-pairs sum (FP32 terms, FP64 across tiles).
// Each thread owns TPT target cells so that every source cell read from
// shared memory serves TPT pair terms.  No branches in the inner loop: empty
// cells carry zero moment and sit far away (their terms vanish), and the
// self pair (r = 0) is removed by taking 1/r = 0 there.
constexpr int kFieldTile = 256;
constexpr int kTargetsPerThread = 4;

__global__ void __launch_bounds__(kFieldTile) cell_field_kernel(int nc, const float4* __restrict__ pos,
                                                                const float4* __restrict__ mom,
                                                                double* __restrict__ field) {
   __shared__ float4 sp[kFieldTile];
   __shared__ float4 sm[kFieldTile];
   constexpr int T = kTargetsPerThread;
   const int i0 = blockIdx.x * (kFieldTile * T) + threadIdx.x;
   float px[T], py[T], pz[T];
   double ax[T], ay[T], az[T];
#pragma unroll
   for (int q = 0; q < T; ++q) {
      const int i = i0 + q * kFieldTile;
      const float4 p = i < nc ? pos[i] : make_float4(0.f, 0.f, 0.f, 0.f);
      px[q] = p.x; py[q] = p.y; pz[q] = p.z;
      ax[q] = ay[q] = az[q] = 0.0;
   }
   // blockIdx.y selects a contiguous share of the source cells; partial sums
   // of the shares meet in FP64 atomics (field is zeroed before the launch)
   const int per = (nc + gridDim.y - 1) / gridDim.y;
   const int src0 = blockIdx.y * per, src1 = min(nc, src0 + per);
   for (int base = src0; base < src1; base += kFieldTile) {
      const int j = base + threadIdx.x;
      sp[threadIdx.x] = j < src1 ? pos[j] : make_float4(1e9f, 1e9f, 1e9f, 0.f);
      sm[threadIdx.x] = j < src1 ? mom[j] : make_float4(0.f, 0.f, 0.f, 0.f);
      __syncthreads();
      float fx[T], fy[T], fz[T];
#pragma unroll
      for (int q = 0; q < T; ++q) fx[q] = fy[q] = fz[q] = 0.f;
#pragma unroll 4
      for (int k = 0; k < kFieldTile; ++k) {
         const float4 pj = sp[k];
         const float4 mj = sm[k];
#pragma unroll
         for (int q = 0; q < T; ++q) {
            const float rx = pj.x - px[q], ry = pj.y - py[q], rz = pj.z - pz[q];
            const float r2 = rx * rx + ry * ry + rz * rz;
            const float ri = r2 > 0.f ? rsqrtf(r2) : 0.f;
            const float ri2 = ri * ri;
            const float ri3 = ri2 * ri;
            const float mr = 3.f * (mj.x * rx + mj.y * ry + mj.z * rz) * ri2;
            fx[q] += (mr * rx - mj.x) * ri3;
            fy[q] += (mr * ry - mj.y) * ri3;
            fz[q] += (mr * rz - mj.z) * ri3;
         }
      }
#pragma unroll
      for (int q = 0; q < T; ++q) { ax[q] += fx[q]; ay[q] += fy[q]; az[q] += fz[q]; }
      __syncthreads();
   }
#pragma unroll
   for (int q = 0; q < T; ++q) {
      const int i = i0 + q * kFieldTile;
      if (i < nc) {
         atomicAdd(field + i, ax[q]);
         atomicAdd(field + nc + i, ay[q]);
         atomicAdd(field + 2 * nc + i, az[q]);
      }
   }
}

// CSR near pairs -> ELL (one thread per pair)
__global__ void near_ell_kernel(int npairs, int nc, int maxp, const int* __restrict__ pair_i,
                                const int* __restrict__ near_start, const int* __restrict__ near_j,
                                const double* __restrict__ near_t, int* __restrict__ je, double* __restrict__ te) {
   const int p = blockIdx.x * blockDim.x + threadIdx.x;
   if (p >= npairs) return;
   const int i = pair_i[p], k = p - near_start[i];
   je[(size_t)k * nc + i] = near_j[p];
   for (int q = 0; q < 6; ++q) te[((size_t)q * maxp + k) * nc + i] = near_t[(size_t)q * npairs + p];
}

// near-field correction and final scaling (update.cpp:56-99)
template <typename R>
__global__ void cell_finish_kernel(int nc, const int* __restrict__ near_cnt, const int* __restrict__ near_je,
                                   const double* __restrict__ near_te, int maxp, const double* __restrict__ mag,
                                   const double* __restrict__ self, const float4* __restrict__ pos,
                                   double* __restrict__ field, R* __restrict__ tb, R* __restrict__ thd) {
   const int i = blockIdx.x * blockDim.x + threadIdx.x;
   if (i > nc) return;
   if (i == nc) {  // zero row read by non-magnetic atoms
      for (int q = 0; q < 3; ++q) { tb[q * (nc + 1) + nc] = (R)0; thd[q * (nc + 1) + nc] = (R)0; }
      return;
   }
   const double imuB = 1.0 / 9.27400915e-24;
   double fx = field[i], fy = field[nc + i], fz = field[2 * nc + i];
   if (near_cnt) {
      const size_t qs = (size_t)maxp * nc;
      const int cnt = near_cnt[i];
      for (int k = 0; k < cnt; ++k) {
         const size_t e = (size_t)k * nc + i;
         const int j = near_je[e];
         const double mx = mag[j] * imuB, my = mag[nc + j] * imuB, mz = mag[2 * nc + j] * imuB;
         const double txx = near_te[e], txy = near_te[qs + e], txz = near_te[2 * qs + e];
         const double tyy = near_te[3 * qs + e], tyz = near_te[4 * qs + e], tzz = near_te[5 * qs + e];
         fx += mx * txx + my * txy + mz * txz;
         fy += mx * txy + my * tyy + mz * tyz;
         fz += mx * txz + my * tyz + mz * tzz;
      }
   }
   const double k = 9.27400915e-01;
   const bool has = pos[i].w != 0.f;
   const double sd = self[i];
   const double mxi = mag[i] * imuB, myi = mag[nc + i] * imuB, mzi = mag[2 * nc + i] * imuB;
   const double bx = has ? fx * k : 0.0, by = has ? fy * k : 0.0, bz = has ? fz * k : 0.0;
   const double hx = has ? (fx - 0.5 * sd * mxi) * k : 0.0;
   const double hy = has ? (fy - 0.5 * sd * myi) * k : 0.0;
   const double hz = has ? (fz - 0.5 * sd * mzi) * k : 0.0;
   field[i] = bx; field[nc + i] = by; field[2 * nc + i] = bz;
   field[3 * nc + i] = hx; field[4 * nc + i] = hy; field[5 * nc + i] = hz;
   tb[i] = (R)bx; tb[(nc + 1) + i] = (R)by; tb[2 * (nc + 1) + i] = (R)bz;
   thd[i] = (R)hx; thd[(nc + 1) + i] = (R)hy; thd[2 * (nc + 1) + i] = (R)hz;
}

// atomistic near tensors (inter.cpp:83-146, intra.cpp:54-138) minus the bare
// term of inter.cpp:66-80; one block per (target, source) pair, FP64
__global__ void near_tensor_kernel(int npairs, const int* __restrict__ pair_i, const int* __restrict__ pair_j,
                                   const int* __restrict__ cstart, const double* __restrict__ ax,
                                   const double* __restrict__ ay, const double* __restrict__ az,
                                   const double* __restrict__ cpos, int bare_fp64, double* __restrict__ out) {
   const int p = blockIdx.x;
   if (p >= npairs) return;
   const int ci = pair_i[p], cj = pair_j[p];
   const int i0 = cstart[ci], ni = cstart[ci + 1] - i0;
   const int j0 = cstart[cj], nj = cstart[cj + 1] - j0;
   double t[6] = {0, 0, 0, 0, 0, 0};
   for (int q = threadIdx.x; q < ni * nj; q += blockDim.x) {
      const int a = i0 + q / nj, b = j0 + q % nj;
      if (ci == cj && a == b) continue;
      const double rx = ax[b] - ax[a], ry = ay[b] - ay[a], rz = az[b] - az[a];
      const double rij = 1.0 / sqrt(rx * rx + ry * ry + rz * rz);
      const double ex = rx * rij, ey = ry * rij, ez = rz * rij;
      const double r3 = rij * rij * rij;
      t[0] += (3.0 * ex * ex - 1.0) * r3;
      t[1] += (3.0 * ex * ey) * r3;
      t[2] += (3.0 * ex * ez) * r3;
      t[3] += (3.0 * ey * ey - 1.0) * r3;
      t[4] += (3.0 * ey * ez) * r3;
      t[5] += (3.0 * ez * ez - 1.0) * r3;
   }
   __shared__ double red[6][256];
   for (int k = 0; k < 6; ++k) red[k][threadIdx.x] = t[k];
   __syncthreads();
   for (int s = blockDim.x / 2; s > 0; s >>= 1) {
      if (threadIdx.x < s)
         for (int k = 0; k < 6; ++k) red[k][threadIdx.x] += red[k][threadIdx.x + s];
      __syncthreads();
   }
   if (threadIdx.x == 0) {
      const double norm = (double)ni * (double)nj;
      double bare[6] = {0, 0, 0, 0, 0, 0};
      if (ci != cj) {
         // the far-field term already added for this pair, taken out again: from
         // FP32 centres for the all-pairs kernel, FP64 for the FFT solver
         double rx, ry, rz;
         if (bare_fp64) {
            rx = cpos[4 * cj] - cpos[4 * ci]; ry = cpos[4 * cj + 1] - cpos[4 * ci + 1];
            rz = cpos[4 * cj + 2] - cpos[4 * ci + 2];
         } else {
            rx = (float)cpos[4 * cj] - (float)cpos[4 * ci];
            ry = (float)cpos[4 * cj + 1] - (float)cpos[4 * ci + 1];
            rz = (float)cpos[4 * cj + 2] - (float)cpos[4 * ci + 2];
         }
         const double r = sqrt(rx * rx + ry * ry + rz * rz);
         const double ri = 1.0 / r, ex = rx * ri, ey = ry * ri, ez = rz * ri, r3 = ri * ri * ri;
         bare[0] = (3.0 * ex * ex - 1.0) * r3; bare[1] = 3.0 * ex * ey * r3; bare[2] = 3.0 * ex * ez * r3;
         bare[3] = (3.0 * ey * ey - 1.0) * r3; bare[4] = 3.0 * ey * ez * r3; bare[5] = (3.0 * ez * ez - 1.0) * r3;
      }
      for (int k = 0; k < 6; ++k) out[k * npairs + p] = red[k][0] / norm - bare[k];
   }
}

void dipole_destroy(vgpu_ctx* h) {
   DipoleState* d = dip_of(h);
   if (!d) return;
   cudaFree(d->cell_start); cudaFree(d->cell_atoms); cudaFree(d->mag); cudaFree(d->pos); cudaFree(d->mom);
   cudaFree(d->field); cudaFree(d->self); cudaFree(d->near_start); cudaFree(d->near_j); cudaFree(d->near_t);
   cudaFree(d->near_cnt); cudaFree(d->near_je); cudaFree(d->near_te);
   cudaFree(d->table_b); cudaFree(d->table_hd); cudaFree(d->atom_cell);
   fft_field_destroy(d->fft);
   h->sys.cell = nullptr;
   h->sys.cell_field = nullptr;
   h->sys.cell_hd = nullptr;
   h->sys.ncells = 0;
   delete d;
   h->extras[2] = nullptr;
}

// K5 over the moment list (all magnetic atoms, or a shard's owned ones)
template <typename R>
static int dipole_moments_typed(vgpu_ctx* h) {
   DipoleState* d = dip_of(h);
   SysDev& S = h->sys;
   const int nc = d->nc;
   h->prof_begin(PROF_DIPOLE);
   cell_moment_kernel<R><<<(nc * 32 + 255) / 256, 256, 0, h->stream>>>(
       nc, d->cell_start, d->cell_atoms, (const R*)S.s[0], (const R*)S.s[1], (const R*)S.s[2], (const int*)S.mat,
       (const MatParams<R>*)S.mp, S.mus_SI, d->mag, d->pos, d->mom);
   h->prof_end(PROF_DIPOLE);
   h->kernel_launches += 1;
   return cuda_err(h, cudaGetLastError(), "dipole cell moments");
}

// K6 and the finish from the cell moments in d->mag; with_mom: first convert
// them to mu_B (moments summed over ranks)
template <typename R>
static int dipole_field_typed(vgpu_ctx* h, bool with_mom) {
   DipoleState* d = dip_of(h);
   const int nc = d->nc;
   h->prof_begin(PROF_DIPOLE);
   int launches = 1;  // the finish, plus the far field below
   if (with_mom && !d->fft) {
      cell_mom_kernel<<<(nc + 255) / 256, 256, 0, h->stream>>>(nc, d->mag, d->mom);
      launches += 1;
   }
   if (d->fft) {
      cudaError_t e = fft_field_apply(d->fft, d->mag, d->field, h->stream, &launches);
      if (e != cudaSuccess) {
         h->prof_end(PROF_DIPOLE);
         return cuda_err(h, e, "dipole FFT far field");
      }
   } else {
      // enough blocks for every SM: split the sources when the targets alone are too few
      const int tblocks = (nc + kFieldTile * kTargetsPerThread - 1) / (kFieldTile * kTargetsPerThread);
      int sms = 148;
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device);
      const int splits = std::max(1, std::min(64, (6 * sms + tblocks - 1) / tblocks));
      cudaMemsetAsync(d->field, 0, sizeof(double) * 3 * nc, h->stream);
      cell_field_kernel<<<dim3(tblocks, splits), kFieldTile, 0, h->stream>>>(nc, d->pos, d->mom, d->field);
      launches += 1;
   }
   cell_finish_kernel<R><<<(nc + 1 + 255) / 256, 256, 0, h->stream>>>(
       nc, d->near_cnt, d->near_je, d->near_te, d->maxp, d->mag, d->self, d->pos, d->field, (R*)d->table_b,
       (R*)d->table_hd);
   h->prof_end(PROF_DIPOLE);
   h->kernel_launches += launches;
   return cuda_err(h, cudaGetLastError(), "dipole field");
}

// whole system: moments and field; shard: partial moments, field pending
template <typename R>
static int dipole_update_typed(vgpu_ctx* h) {
   DipoleState* d = dip_of(h);
   int rc = dipole_moments_typed<R>(h);
   if (rc) return rc;
   if (d->shard) {
      d->pending = true;
      return VGPU_OK;
   }
   return dipole_field_typed<R>(h, false);
}

int dipole_update(vgpu_ctx* h) {
   return h->prec == VGPU_PREC_FP64 ? dipole_update_typed<double>(h) : dipole_update_typed<float>(h);
}

static int dipole_finish(vgpu_ctx* h) {
   int rc = h->prec == VGPU_PREC_FP64 ? dipole_field_typed<double>(h, true) : dipole_field_typed<float>(h, true);
   if (!rc) dip_of(h)->pending = false;
   return rc;
}

}  // namespace vgpu

using namespace vgpu;

int dipole_ready(vgpu_ctx* h) {
   DipoleState* d = dip_of(h);
   if (d && d->pending)
      return set_err(h, VGPU_ERR_STATE,
                     "dipole cell moments of this shard await their sum over ranks and vgpu_dipole_finish");
   return VGPU_OK;
}

int dipole_after_step(vgpu_ctx* h) {
   DipoleState* d = dip_of(h);
   if (!d || d->update_rate <= 0) return VGPU_OK;
   if (h->step % (uint64_t)d->update_rate != 0) return VGPU_OK;
   return dipole_update(h);
}

// Builds the solver from a descriptor of ng atoms (the whole system) with
// material ids gtype; local[i] is the descriptor atom of the handle's atom i
// (nullptr: the handle holds all ng atoms in descriptor order).  Cell moments
// sum the handle's updated atoms; the near tensors use every atom of the
// descriptor, so a shard's near field is the whole system's.
static int dipole_build(vgpu_ctx* h, const vgpu_dipole_desc* dd, int ng, const int* gtype, const int64_t* local) {
   SysDev& S = h->sys;
   const int n = S.n, nc = dd->num_cells;
   if (nc <= 0 || !dd->atom_cell || !dd->cell_pos_mom || !dd->cell_volume || !dd->cell_natoms)
      return set_err(h, VGPU_ERR_ARG, "incomplete dipole descriptor");
   if (dd->solver == VGPU_DIPOLE_TENSOR && (!dd->atom_x || !dd->atom_y || !dd->atom_z))
      return set_err(h, VGPU_ERR_ARG, "tensor solver needs atom coordinates");
   if (!(dd->macro_cell_size > 0.0)) return set_err(h, VGPU_ERR_ARG, "macro_cell_size must be positive");
   for (int g = 0; g < ng; ++g) {
      if (dd->atom_cell[g] < 0 || dd->atom_cell[g] >= nc)
         return set_err(h, VGPU_ERR_ARG, "atom %d has cell %d outside 0..%d", g, dd->atom_cell[g], nc - 1);
      if (gtype[g] < 0 || gtype[g] >= S.M)
         return set_err(h, VGPU_ERR_ARG, "atom %d has material %d outside 0..%d", g, gtype[g], S.M - 1);
   }
   if (local)
      for (int i = 0; i < n; ++i) {
         if (local[i] < 0 || local[i] >= ng)
            return set_err(h, VGPU_ERR_ARG, "local atom %d maps to %lld outside 0..%d", i, (long long)local[i], ng - 1);
         if (gtype[local[i]] != S.type_host[i])
            return set_err(h, VGPU_ERR_ARG, "local atom %d: material %d, whole-system atom %lld: material %d", i,
                           S.type_host[i], (long long)local[i], gtype[local[i]]);
      }
   auto gid = [&](int i) { return local ? (int)local[i] : i; };
   cudaSetDevice(h->device);
   dipole_destroy(h);
   DipoleState* d = new DipoleState();
   h->extras[2] = d;
   d->shard = local != nullptr;
   d->nc = nc;
   d->solver = dd->solver;
   d->update_rate = dd->update_rate;
   d->size = dd->macro_cell_size;
   d->cutoff = dd->cutoff;
   const int M = S.M;
   std::vector<double> mus(M);
   std::vector<char> magnetic(M);
   for (int m = 0; m < M; ++m) {
      mus[m] = S.materials[m].mu_s_SI;
      magnetic[m] = S.materials[m].non_magnetic == 0;
   }
   // cell-sorted lists of magnetic atoms (cells::mag skips non-magnetic
   // ones): the handle's updated atoms for the moments, every descriptor atom
   // for the near tensors (the same list on a whole system)
   auto cell_sort = [&](int count, auto cell_of, auto type_of, std::vector<int>& start, std::vector<int>& atoms) {
      start.assign(nc + 1, 0);
      for (int i = 0; i < count; ++i)
         if (magnetic[type_of(i)]) start[cell_of(i) + 1]++;
      for (int c = 0; c < nc; ++c) start[c + 1] += start[c];
      atoms.resize(start[nc]);
      std::vector<int> fill(start.begin(), start.end() - 1);
      for (int i = 0; i < count; ++i)
         if (magnetic[type_of(i)]) atoms[fill[cell_of(i)]++] = i;
   };
   std::vector<int> start, atoms, gstart, gatoms;
   cell_sort(local ? S.n_owned : n, [&](int i) { return dd->atom_cell[gid(i)]; },
             [&](int i) { return S.type_host[i]; }, start, atoms);
   if (local) cell_sort(ng, [&](int g) { return dd->atom_cell[g]; }, [&](int g) { return gtype[g]; }, gstart, gatoms);
   const std::vector<int>& nstart_atoms = local ? gstart : start;
   const std::vector<int>& natoms_list = local ? gatoms : atoms;
   // atoms read the zero row when their cell is empty or they are non-magnetic
   std::vector<int> acell(n);
   for (int i = 0; i < n; ++i) {
      const int c = dd->atom_cell[gid(i)];
      acell[i] = (dd->cell_natoms[c] > 0 && magnetic[S.type_host[i]]) ? c : nc;
   }
   std::vector<float4> pos(nc);
   std::vector<double> self(nc);
   for (int c = 0; c < nc; ++c) {
      // empty cells (zero moment) are parked far away so K6 needs no test for them
      pos[c] = dd->cell_natoms[c] > 0
                   ? make_float4((float)dd->cell_pos_mom[4 * c], (float)dd->cell_pos_mom[4 * c + 1],
                                 (float)dd->cell_pos_mom[4 * c + 2], 1.f)
                   : make_float4(1e9f, 1e9f, 1e9f, 0.f);
      self[c] = dd->cell_natoms[c] > 0 ? 8.0 * M_PI / (3.0 * dd->cell_volume[c]) : 0.0;
   }
   // far field by FFT when the occupied cells form a regular grid
   if (h->dipole_fft != 0) {
      cudaError_t fe = cudaSuccess;
      std::string why;
      d->fft = fft_field_create(nc, dd->cell_pos_mom, dd->cell_natoms, dd->macro_cell_size, h->prec == VGPU_PREC_FP32,
                                h->stream, &fe, &why);
      if (fe != cudaSuccess) {
         int rc = cuda_err(h, fe, "dipole FFT setup");
         dipole_destroy(h);
         return rc;
      }
   }
   // near pairs (tensor solver), classified in FP64 exactly as inter.cpp:66,83
   std::vector<int> pi, pj, nstart(nc + 1, 0);
   if (dd->solver == VGPU_DIPOLE_TENSOR) {
      const double bin = std::max(dd->cutoff * dd->macro_cell_size, 1e-6) * 1.0001;
      std::unordered_map<long long, std::vector<int>> grid;
      auto key = [&](long long x, long long y, long long z) { return (x * 1000003LL + y) * 1000033LL + z; };
      for (int c = 0; c < nc; ++c) {
         if (dd->cell_natoms[c] <= 0) continue;
         const long long gx = (long long)std::floor(dd->cell_pos_mom[4 * c] / bin);
         const long long gy = (long long)std::floor(dd->cell_pos_mom[4 * c + 1] / bin);
         const long long gz = (long long)std::floor(dd->cell_pos_mom[4 * c + 2] / bin);
         grid[key(gx, gy, gz)].push_back(c);
      }
      std::vector<std::vector<int>> near(nc);
      for (int i = 0; i < nc; ++i) {
         if (dd->cell_natoms[i] <= 0) continue;
         const double* P = dd->cell_pos_mom + 4 * i;
         const long long gx = (long long)std::floor(P[0] / bin), gy = (long long)std::floor(P[1] / bin),
                         gz = (long long)std::floor(P[2] / bin);
         for (long long x = gx - 1; x <= gx + 1; ++x)
            for (long long y = gy - 1; y <= gy + 1; ++y)
               for (long long z = gz - 1; z <= gz + 1; ++z) {
                  auto it = grid.find(key(x, y, z));
                  if (it == grid.end()) continue;
                  for (int j : it->second) {
                     if (j == i) { near[i].push_back(j); continue; }
                     const double rx = dd->cell_pos_mom[4 * j] - P[0];
                     const double ry = dd->cell_pos_mom[4 * j + 1] - P[1];
                     const double rz = dd->cell_pos_mom[4 * j + 2] - P[2];
                     const double rij = 1.0 / sqrt(rx * rx + ry * ry + rz * rz);
                     if ((1.0 / rij) / dd->macro_cell_size <= dd->cutoff) near[i].push_back(j);
                  }
               }
         std::sort(near[i].begin(), near[i].end());
      }
      for (int i = 0; i < nc; ++i) {
         nstart[i + 1] = nstart[i] + (int)near[i].size();
         for (int j : near[i]) { pi.push_back(i); pj.push_back(j); }
      }
   }
   d->npairs = (int)pj.size();
   cudaError_t e = cudaSuccess;
   auto up = [&](void** dst, const void* src, size_t bytes) {
      if (e != cudaSuccess) return;
      e = cudaMalloc(dst, std::max<size_t>(bytes, 16));
      if (e == cudaSuccess && bytes) e = cudaMemcpyAsync(*dst, src, bytes, cudaMemcpyHostToDevice, h->stream);
   };
   up((void**)&d->cell_start, start.data(), sizeof(int) * (nc + 1));
   up((void**)&d->cell_atoms, atoms.data(), sizeof(int) * atoms.size());
   acell.resize(((size_t)S.n_alloc + 3) & ~(size_t)3, nc);  // padded like the state arrays
   up((void**)&d->atom_cell, acell.data(), sizeof(int) * acell.size());
   up((void**)&d->pos, pos.data(), sizeof(float4) * nc);
   up((void**)&d->self, self.data(), sizeof(double) * nc);
   if (e == cudaSuccess) e = cudaMalloc(&d->mag, sizeof(double) * 3 * nc);
   if (e == cudaSuccess) e = cudaMalloc(&d->mom, sizeof(float4) * nc);
   if (e == cudaSuccess) e = cudaMalloc(&d->field, sizeof(double) * 6 * nc);
   const size_t rs = h->prec == VGPU_PREC_FP64 ? sizeof(double) : sizeof(float);
   if (e == cudaSuccess) e = cudaMalloc(&d->table_b, rs * 3 * (nc + 1));
   if (e == cudaSuccess) e = cudaMalloc(&d->table_hd, rs * 3 * (nc + 1));
   if (e == cudaSuccess && !S.mus_SI) {
      S.mus_SI = (double*)h->alloc(sizeof(double) * 100);
      if (!S.mus_SI) e = cudaErrorMemoryAllocation;
   }
   if (e == cudaSuccess) e = cudaMemcpyAsync(S.mus_SI, mus.data(), sizeof(double) * M, cudaMemcpyHostToDevice, h->stream);
   if (e == cudaSuccess && d->npairs > 0) {
      up((void**)&d->near_start, nstart.data(), sizeof(int) * (nc + 1));
      up((void**)&d->near_j, pj.data(), sizeof(int) * pj.size());
      int *dpi = nullptr, *dpj = nullptr, *gs = nullptr;
      double *ax = nullptr, *ay = nullptr, *az = nullptr, *cp = nullptr;
      // coordinates in cell-sorted order for the near-tensor kernel
      const size_t na = natoms_list.size();
      std::vector<double> cx(na), cy(na), cz(na);
      for (size_t k = 0; k < na; ++k) {
         const int g = local ? natoms_list[k] : gid(natoms_list[k]);
         cx[k] = dd->atom_x[g]; cy[k] = dd->atom_y[g]; cz[k] = dd->atom_z[g];
      }
      if (local) up((void**)&gs, nstart_atoms.data(), sizeof(int) * (nc + 1));
      up((void**)&dpi, pi.data(), sizeof(int) * pi.size());
      up((void**)&dpj, pj.data(), sizeof(int) * pj.size());
      up((void**)&ax, cx.data(), sizeof(double) * cx.size());
      up((void**)&ay, cy.data(), sizeof(double) * cy.size());
      up((void**)&az, cz.data(), sizeof(double) * cz.size());
      up((void**)&cp, dd->cell_pos_mom, sizeof(double) * 4 * nc);
      if (e == cudaSuccess) e = cudaMalloc(&d->near_t, sizeof(double) * 6 * d->npairs);
      if (e == cudaSuccess) {
         near_tensor_kernel<<<d->npairs, 256, 0, h->stream>>>(d->npairs, dpi, dpj, local ? gs : d->cell_start, ax,
                                                               ay, az, cp, d->fft != nullptr, d->near_t);
         e = cudaGetLastError();
      }
      // ELL copy for the finish kernel; the CSR arrays are set-up only
      std::vector<int> cnt(nc);
      for (int c = 0; c < nc; ++c) {
         cnt[c] = nstart[c + 1] - nstart[c];
         d->maxp = std::max(d->maxp, cnt[c]);
      }
      up((void**)&d->near_cnt, cnt.data(), sizeof(int) * nc);
      if (e == cudaSuccess) e = cudaMalloc(&d->near_je, sizeof(int) * (size_t)d->maxp * nc);
      if (e == cudaSuccess) e = cudaMemsetAsync(d->near_je, 0, sizeof(int) * (size_t)d->maxp * nc, h->stream);
      if (e == cudaSuccess) e = cudaMalloc(&d->near_te, sizeof(double) * 6 * (size_t)d->maxp * nc);
      if (e == cudaSuccess) e = cudaMemsetAsync(d->near_te, 0, sizeof(double) * 6 * (size_t)d->maxp * nc, h->stream);
      if (e == cudaSuccess) {
         near_ell_kernel<<<(d->npairs + 255) / 256, 256, 0, h->stream>>>(d->npairs, nc, d->maxp, dpi, d->near_start,
                                                                          d->near_j, d->near_t, d->near_je,
                                                                          d->near_te);
         e = cudaGetLastError();
      }
      if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
      cudaFree(dpi); cudaFree(dpj); cudaFree(gs); cudaFree(ax); cudaFree(ay); cudaFree(az); cudaFree(cp);
      cudaFree(d->near_start); cudaFree(d->near_j); cudaFree(d->near_t);
      d->near_start = d->near_j = nullptr;
      d->near_t = nullptr;
   }
   if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
   if (e != cudaSuccess) {
      int rc = cuda_err(h, e, "dipole setup");
      dipole_destroy(h);
      return rc;
   }
   S.ncells = nc + 1;  // tables have a zero row at index nc
   S.cell = d->atom_cell;
   S.cell_field = d->table_b;
   S.cell_hd = d->table_hd;
   // field at the current spins (dipole::initialize calls calculate_field(0));
   // on a shard the partial moments, the field once they are summed
   return dipole_update(h);
}

extern "C" int vgpu_dipole_setup(vgpu_handle h, const vgpu_dipole_desc* dd) {
   if (!h || !dd) return set_err(h, VGPU_ERR_ARG, "null argument");
   SysDev& S = h->sys;
   if (!S.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   if (S.n_owned < S.n)
      return set_err(h, VGPU_ERR_STATE, "the handle holds a shard: set the dipole solver up with vgpu_dipole_setup_shard");
   return dipole_build(h, dd, S.n, S.type_host.data(), nullptr);
}

extern "C" int vgpu_dipole_setup_shard(vgpu_handle h, const vgpu_dipole_desc* whole, int64_t n_global,
                                       const int32_t* global_type, const int64_t* local) {
   if (!h || !whole || !global_type || !local) return set_err(h, VGPU_ERR_ARG, "null argument");
   SysDev& S = h->sys;
   if (!S.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   if (n_global < S.n || n_global > INT32_MAX) return set_err(h, VGPU_ERR_ARG, "n_global %lld below the shard's %d atoms or too large", (long long)n_global, S.n);
   return dipole_build(h, whole, (int)n_global, global_type, local);
}

extern "C" int vgpu_dipole_moment_buffer(vgpu_handle h, double** dev, int64_t* count) {
   if (!h || !dev || !count) return set_err(h, VGPU_ERR_ARG, "null argument");
   DipoleState* d = dip_of(h);
   if (!d) return set_err(h, VGPU_ERR_STATE, "vgpu_dipole_setup not called");
   *dev = d->mag;
   *count = 3 * (int64_t)d->nc;
   return VGPU_OK;
}

extern "C" int vgpu_dipole_pending(vgpu_handle h, int32_t* pending) {
   if (!h || !pending) return set_err(h, VGPU_ERR_ARG, "null argument");
   DipoleState* d = dip_of(h);
   *pending = d && d->pending ? 1 : 0;
   return VGPU_OK;
}

extern "C" int vgpu_dipole_finish(vgpu_handle h) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   DipoleState* d = dip_of(h);
   if (!d) return set_err(h, VGPU_ERR_STATE, "vgpu_dipole_setup not called");
   cudaSetDevice(h->device);
   return dipole_finish(h);
}

extern "C" int vgpu_dipole_update(vgpu_handle h) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   if (!dip_of(h)) return set_err(h, VGPU_ERR_STATE, "vgpu_dipole_setup not called");
   cudaSetDevice(h->device);
   return dipole_update(h);
}

extern "C" int vgpu_dipole_method(vgpu_handle h, int32_t* method) {
   if (!h || !method) return set_err(h, VGPU_ERR_ARG, "null argument");
   DipoleState* d = dip_of(h);
   if (!d) return set_err(h, VGPU_ERR_STATE, "vgpu_dipole_setup not called");
   *method = d->fft ? VGPU_DIPOLE_FAR_FFT : VGPU_DIPOLE_FAR_DIRECT;
   return VGPU_OK;
}

extern "C" int vgpu_dipole_get_cells(vgpu_handle h, double* mag, double* b_field, double* hd_field) {
   if (!h) return set_err(nullptr, VGPU_ERR_ARG, "null handle");
   DipoleState* d = dip_of(h);
   if (!d) return set_err(h, VGPU_ERR_STATE, "vgpu_dipole_setup not called");
   cudaSetDevice(h->device);
   const int nc = d->nc;
   cudaError_t e = cudaSuccess;
   if (mag) e = cudaMemcpyAsync(mag, d->mag, sizeof(double) * 3 * nc, cudaMemcpyDeviceToHost, h->stream);
   if (e == cudaSuccess && b_field)
      e = cudaMemcpyAsync(b_field, d->field, sizeof(double) * 3 * nc, cudaMemcpyDeviceToHost, h->stream);
   if (e == cudaSuccess && hd_field)
      e = cudaMemcpyAsync(hd_field, d->field + 3 * nc, sizeof(double) * 3 * nc, cudaMemcpyDeviceToHost, h->stream);
   if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
   return cuda_err(h, e, "dipole download");
}

template <typename R>
static int set_atom_field_typed(vgpu_handle h, const double* b[3], const double* m[3]) {
   SysDev& S = h->sys;
   const int n = S.n;
   if (!S.hd_atom) {
      S.hd_atom = h->alloc(3 * (size_t)n * sizeof(R));
      S.hm_atom = h->alloc(3 * (size_t)n * sizeof(R));
      if (!S.hd_atom || !S.hm_atom) return set_err(h, VGPU_ERR_OOM, "cudaMalloc failed for atom dipole field");
   }
   std::vector<R> buf(3 * (size_t)n);
   for (int q = 0; q < 3; ++q)
      for (int i = 0; i < n; ++i) buf[(size_t)q * n + i] = (R)b[q][i];
   int rc = cuda_err(h, cudaMemcpyAsync(S.hd_atom, buf.data(), buf.size() * sizeof(R), cudaMemcpyHostToDevice,
                                        h->stream), "atom dipole field");
   if (rc) return rc;
   rc = cuda_err(h, cudaStreamSynchronize(h->stream), "atom dipole field");
   if (rc) return rc;
   for (int q = 0; q < 3; ++q)
      for (int i = 0; i < n; ++i) buf[(size_t)q * n + i] = m[q] ? (R)m[q][i] : (R)0;
   rc = cuda_err(h, cudaMemcpyAsync(S.hm_atom, buf.data(), buf.size() * sizeof(R), cudaMemcpyHostToDevice,
                                    h->stream), "atom demag field");
   if (rc) return rc;
   return cuda_err(h, cudaStreamSynchronize(h->stream), "atom demag field");
}

extern "C" int vgpu_set_dipole_field(vgpu_handle h, const double* bx, const double* by, const double* bz,
                                     const double* hx, const double* hy, const double* hz) {
   if (!h || !bx || !by || !bz) return set_err(h, VGPU_ERR_ARG, "null argument");
   if (!h->sys.uploaded) return set_err(h, VGPU_ERR_STATE, "no system uploaded");
   if (dip_of(h)) return set_err(h, VGPU_ERR_STATE, "device dipole solver active; host fields not used");
   cudaSetDevice(h->device);
   const double* b[3] = {bx, by, bz};
   const double* m[3] = {hx, hy, hz};
   return h->prec == VGPU_PREC_FP64 ? set_atom_field_typed<double>(h, b, m) : set_atom_field_typed<float>(h, b, m);
}
