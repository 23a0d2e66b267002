// Far-field macrocell dipole sum by FFT convolution (FP64).
//
// The far field of every cell is H_i = sum_{j != i} T(r_j - r_i) m_j with the
// bare point-dipole tensor T(r) = (3 e e - 1)/|r|^3 (src/dipole/inter.cpp:66-80
// for cells beyond the cutoff; src/dipole/macrocell.cpp for all pairs).  When
// the occupied cells sit on one regular grid (every full cell of a lattice
// does: its magnetic centre is the cell origin plus a fixed offset), T depends
// only on the grid offset, so the sum is a linear convolution of the moment
// grid with T.  It is evaluated as a circular convolution on a grid padded to
// P >= 2G - 1 points per axis (G = occupied extent), with P a power of two:
//
//   scatter  m_j (mu_B) into the G-box of three complex grids (zero at empty
//            cells of the box)
//   FFT      each grid along x and y (radix-2, one shared-memory tile of lines
//            per block; strided axes load W adjacent x columns per block so
//            every global access is a W*16-byte segment)
//   z        per z column: forward transform, H(k) = T(k) M(k) (T symmetric
//            3x3, six spectra computed once), inverse transform, in one kernel
//   iFFT     along y, x, and gather H at the occupied cells (1/P^3 scaling).
//
// The transforms skip the lines that carry only zeros or whose results are not
// needed: the moments occupy the G-box, so the forward x pass runs only the
// gy*gz lines of the box (points past gx read as zero), the y pass only the
// planes z < gz (points past gy read as zero) and the z transform reads zero
// past gz and keeps only z < gz; the inverse y pass runs and keeps only those
// planes' y < gy, the inverse x pass only the box lines' x < gx.  At a 50^3
// grid (P = 128) this is about half of the line transforms of full passes,
// the spectra never leave shared memory, and the grid needs no clearing.
//
// Precision follows the handle: in the FP64 build every step is FP64, so the
// result equals the direct FP64 sum to rounding (~1e-15 of the field); the
// FP32 production handles transform FP32 grids (the tensor spectra computed
// in FP64 once and rounded, twiddles rounded from FP64, moments and fields
// FP64 at the ends), about 1e-6 of the field.  Cost O(P^3 log P) instead of
// O(Nc^2): at 125,000 cells (a 50^3 grid, P = 128) a few hundred microseconds
// instead of tens of milliseconds.  Twiddle factors are tabulated on the host
// in double precision.
#include "dipole_fft.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

namespace vgpu {

struct FFTField {
   int nc = 0;
   int p[3] = {0, 0, 0};       // padded points per axis (powers of two)
   int logp[3] = {0, 0, 0};
   int g[3] = {0, 0, 0};       // occupied extent in cells
   size_t np = 0;              // p[0] * p[1] * p[2]
   double2* tspec = nullptr;   // [6][np] spectra of Txx, Txy, Txz, Tyy, Tyz, Tzz
   double2* grid = nullptr;    // [3][np] moment grids, transformed in place
   double2* tw[3] = {nullptr, nullptr, nullptr};  // [p/2] exp(-2 pi i k / p) per axis
   bool fp32 = false;          // FP32 transforms (the buffers below) instead of the FP64 ones
   float2* tspec32 = nullptr;  // [6][np] the spectra rounded to FP32
   float2* grid32 = nullptr;   // [3][np]
   float2* tw32[3] = {nullptr, nullptr, nullptr};
   int* cell_lin = nullptr;    // [nc] linear grid index, or -1 (empty cell)
   int* box_cell = nullptr;    // [gx*gy*gz] cell at each box point (x fastest), or -1
};

namespace {

constexpr int kFFTThreads = 256;
constexpr int kFFTTile = 2048;  // complex points per block tile (32 KB of shared memory)

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
   return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
   return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// complex value of the transform's precision
template <typename C> __device__ __forceinline__ C cval(double x, double y);
template <> __device__ __forceinline__ double2 cval<double2>(double x, double y) { return make_double2(x, y); }
template <> __device__ __forceinline__ float2 cval<float2>(double x, double y) {
   return make_float2((float)x, (float)y);
}

// radix-2 decimation-in-time butterflies over `nlines` lines of n points held
// in shared memory in bit-reversed order (line-major); results in natural order
template <typename C>
__device__ void fft_smem(C* s, int n, int nlines, const C* __restrict__ tw, bool inverse) {
   const int half = n >> 1;
   for (int h = 1; h < n; h <<= 1) {
      const int step = half / h;  // twiddle stride: exp(-2 pi i j / (2h)) = tw[j * n / (2h)]
      for (int b = threadIdx.x; b < nlines * half; b += blockDim.x) {
         const int line = b / half, k = b - line * half;
         const int j = k % h, grp = k / h;
         const int i0 = line * n + grp * 2 * h + j, i1 = i0 + h;
         C w = tw[j * step];
         if (inverse) w.y = -w.y;
         const C u = s[i0];
         const C v = cmul(w, s[i1]);
         s[i0] = {u.x + v.x, u.y + v.y};
         s[i1] = {u.x - v.x, u.y - v.y};
      }
      __syncthreads();
   }
}

// lines along x (contiguous): block = `lines` lines of one grid, line r of
// the nrows transformed being the x line (y, z) = (r % rpp, r / rpp) at
// (z * py + y) * n; points p >= ld read as zero, points p < st are stored
template <typename C>
__global__ void __launch_bounds__(kFFTThreads) fft_x_kernel(C* __restrict__ data, size_t np, int n, int logn,
                                                            int lines, const C* __restrict__ tw, int inverse,
                                                            int nrows, int rpp, int py, int ld, int st) {
   __shared__ C s[kFFTTile];
   C* grid = data + (size_t)blockIdx.y * np;
   const int r0 = blockIdx.x * lines;
   const int tot = lines * n;
   auto row = [&](int r) { return ((size_t)(r / rpp) * py + (size_t)(r % rpp)) * n; };
   for (int e = threadIdx.x; e < tot; e += blockDim.x) {
      const int line = e / n, p = e - line * n;
      const int r = r0 + line;
      s[line * n + (int)(__brev((unsigned)p) >> (32 - logn))] =
          r < nrows && p < ld ? grid[row(r) + p] : cval<C>(0.0, 0.0);
   }
   __syncthreads();
   fft_smem(s, n, lines, tw, inverse != 0);
   for (int e = threadIdx.x; e < tot; e += blockDim.x) {
      const int line = e / n, p = e - line * n;
      const int r = r0 + line;
      if (r < nrows && p < st) grid[row(r) + p] = s[e];
   }
}

// lines along y or z: block = W adjacent x columns of one (other) index;
// point p of column w sits at base + p * stride + w; points p >= ld read as
// zero, points p < st are stored
template <typename C>
__global__ void __launch_bounds__(kFFTThreads) fft_strided_kernel(C* __restrict__ data, size_t np, int n, int logn,
                                                                  int W, size_t stride, size_t other_stride,
                                                                  const C* __restrict__ tw, int inverse, int ld,
                                                                  int st) {
   __shared__ C s[kFFTTile];
   C* base = data + (size_t)blockIdx.z * np + (size_t)blockIdx.y * other_stride + (size_t)blockIdx.x * W;
   const int tot = W * n;
   for (int e = threadIdx.x; e < tot; e += blockDim.x) {
      const int p = e / W, w = e - p * W;
      s[w * n + (int)(__brev((unsigned)p) >> (32 - logn))] =
          p < ld ? base[(size_t)p * stride + w] : cval<C>(0.0, 0.0);
   }
   __syncthreads();
   fft_smem(s, n, W, tw, inverse != 0);
   for (int e = threadIdx.x; e < tot; e += blockDim.x) {
      const int p = e / W, w = e - p * W;
      if (p < st) base[(size_t)p * stride + w] = s[w * n + p];
   }
}

// The middle of the convolution in one pass over z columns: for W adjacent x
// columns at one y, the three moment components' forward z transforms (points
// z >= gz read as zero), the product H(k) = T(k) M(k) at every k, and the
// inverse z transforms, of which z < gz is stored.  The same butterflies and
// products as separate z passes around multiply_kernel, without writing the
// spectra to memory and reading them back.
constexpr int kFuseTile = 3072;  // complex points per block: 3 components x W x pz (48 KB)

template <typename C>
__device__ __forceinline__ void tensor_times(const C* __restrict__ t, size_t np, size_t q, C mx, C my, C mz, C h[3]) {
   const C xx = t[q], xy = t[np + q], xz = t[2 * np + q];
   const C yy = t[3 * np + q], yz = t[4 * np + q], zz = t[5 * np + q];
   C hx = cmul(xx, mx), hy = cmul(xy, mx), hz = cmul(xz, mx);
   C a = cmul(xy, my), b = cmul(xz, mz);
   hx.x += a.x + b.x; hx.y += a.y + b.y;
   a = cmul(yy, my); b = cmul(yz, mz);
   hy.x += a.x + b.x; hy.y += a.y + b.y;
   a = cmul(yz, my); b = cmul(zz, mz);
   hz.x += a.x + b.x; hz.y += a.y + b.y;
   h[0] = hx; h[1] = hy; h[2] = hz;
}

template <typename C>
__global__ void __launch_bounds__(kFFTThreads) fft_z_multiply_kernel(C* __restrict__ data, const C* __restrict__ t,
                                                                     size_t np, int px, int py, int n, int logn, int W,
                                                                     int gz, const C* __restrict__ tw) {
   __shared__ C s[kFuseTile];
   const size_t stride = (size_t)px * py;
   const size_t col0 = (size_t)blockIdx.y * px + (size_t)blockIdx.x * W;  // (x0, y) in the z = 0 plane
   const int tot = W * n;
   for (int e = threadIdx.x; e < 3 * tot; e += blockDim.x) {
      const int c = e / tot, r = e - c * tot;
      const int p = r / W, w = r - p * W;
      s[(c * W + w) * n + (int)(__brev((unsigned)p) >> (32 - logn))] =
          p < gz ? data[(size_t)c * np + col0 + (size_t)p * stride + w] : cval<C>(0.0, 0.0);
   }
   __syncthreads();
   fft_smem(s, n, 3 * W, tw, false);
   // H = T M at every (w, k), all read before any is written back at its
   // bit-reversed position for the inverse
   constexpr int kMaxPer = kFuseTile / 3 / kFFTThreads;  // points per thread
   C h[kMaxPer][3];
#pragma unroll
   for (int u = 0; u < kMaxPer; ++u) {
      const int r = threadIdx.x + u * kFFTThreads;
      if (r < tot) {
         const int k = r / W, w = r - k * W;
         tensor_times(t, np, col0 + (size_t)k * stride + w, s[w * n + k], s[(W + w) * n + k], s[(2 * W + w) * n + k],
                      h[u]);
      }
   }
   __syncthreads();
#pragma unroll
   for (int u = 0; u < kMaxPer; ++u) {
      const int r = threadIdx.x + u * kFFTThreads;
      if (r < tot) {
         const int k = r / W, w = r - k * W;
         const int kr = (int)(__brev((unsigned)k) >> (32 - logn));
#pragma unroll
         for (int c = 0; c < 3; ++c) s[(c * W + w) * n + kr] = h[u][c];
      }
   }
   __syncthreads();
   fft_smem(s, n, 3 * W, tw, true);
   for (int e = threadIdx.x; e < 3 * tot; e += blockDim.x) {
      const int c = e / tot, r = e - c * tot;
      const int p = r / W, w = r - p * W;
      if (p < gz) data[(size_t)c * np + col0 + (size_t)p * stride + w] = s[(c * W + w) * n + p];
   }
}

// bare tensor on the padded grid: offset (dx, dy, dz) cells, zero at the
// origin and beyond the occupied extent
__global__ void tensor_grid_kernel(double2* __restrict__ t, size_t np, int px, int py, int pz, int gx, int gy, int gz,
                                   double size) {
   for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < np; q += (size_t)gridDim.x * blockDim.x) {
      const int x = (int)(q % px), y = (int)((q / px) % py), z = (int)(q / ((size_t)px * py));
      const int dx = x < px / 2 ? x : x - px, dy = y < py / 2 ? y : y - py, dz = z < pz / 2 ? z : z - pz;
      double v[6] = {0, 0, 0, 0, 0, 0};
      const bool in = abs(dx) < gx && abs(dy) < gy && abs(dz) < gz && (dx | dy | dz) != 0;
      if (in) {
         const double rx = dx * size, ry = dy * size, rz = dz * size;
         const double rij = 1.0 / sqrt(rx * rx + ry * ry + rz * rz);
         const double ex = rx * rij, ey = ry * rij, ez = rz * rij;
         const double r3 = rij * rij * rij;
         v[0] = (3.0 * ex * ex - 1.0) * r3;
         v[1] = (3.0 * ex * ey) * r3;
         v[2] = (3.0 * ex * ez) * r3;
         v[3] = (3.0 * ey * ey - 1.0) * r3;
         v[4] = (3.0 * ey * ez) * r3;
         v[5] = (3.0 * ez * ez - 1.0) * r3;
      }
#pragma unroll
      for (int k = 0; k < 6; ++k) t[k * np + q] = make_double2(v[k], 0.0);
   }
}

// the moments (mu_B) at every point of the G-box, zero at its empty cells
template <typename C>
__global__ void scatter_moments_kernel(int nc, const int* __restrict__ box_cell, int gx, int gy, int nbox,
                                       const double* __restrict__ mag, C* __restrict__ grid, int px, int py,
                                       size_t np) {
   const int b = blockIdx.x * blockDim.x + threadIdx.x;
   if (b >= nbox) return;
   const int c = box_cell[b];
   const int x = b % gx, y = (b / gx) % gy, z = b / (gx * gy);
   const size_t q = ((size_t)z * py + y) * px + x;
   const double imuB = 1.0 / 9.27400915e-24;
   grid[q] = cval<C>(c >= 0 ? mag[c] * imuB : 0.0, 0.0);
   grid[np + q] = cval<C>(c >= 0 ? mag[nc + c] * imuB : 0.0, 0.0);
   grid[2 * np + q] = cval<C>(c >= 0 ? mag[2 * nc + c] * imuB : 0.0, 0.0);
}

template <typename C>
__global__ void gather_field_kernel(int nc, const int* __restrict__ lin, const C* __restrict__ grid, size_t np,
                                    double scale, double* __restrict__ field) {
   const int c = blockIdx.x * blockDim.x + threadIdx.x;
   if (c >= nc) return;
   const int q = lin[c];
   field[c] = q < 0 ? 0.0 : (double)grid[q].x * scale;
   field[nc + c] = q < 0 ? 0.0 : (double)grid[np + q].x * scale;
   field[2 * nc + c] = q < 0 ? 0.0 : (double)grid[2 * np + q].x * scale;
}

// the FP64 spectra or twiddles rounded to FP32
__global__ void round_complex_kernel(const double2* __restrict__ in, float2* __restrict__ out, size_t n) {
   for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
      out[q] = make_float2((float)in[q].x, (float)in[q].y);
}

int ilog2(int v) {
   int l = 0;
   while ((1 << l) < v) ++l;
   return l;
}

int grid_blocks(size_t np) { return (int)std::min<size_t>((np + 255) / 256, 148 * 16); }

// forward 3-D FFT of `ncomp` consecutive grids, all lines (the tensor spectra)
cudaError_t fft3d(FFTField* f, double2* data, int ncomp, cudaStream_t st) {
   const int px = f->p[0], py = f->p[1], pz = f->p[2];
   {  // x: lines of px points, kFFTTile / px lines per block
      const int nrows = py * pz;
      const int lines = std::max(1, std::min(kFFTTile / px, nrows));
      dim3 grid((unsigned)((nrows + lines - 1) / lines), (unsigned)ncomp);
      fft_x_kernel<double2><<<grid, kFFTThreads, 0, st>>>(data, f->np, px, f->logp[0], lines, f->tw[0], 0, nrows,
                                                          py, py, px, px);
   }
   {  // y: stride px, W adjacent x columns, one block per (x chunk, z)
      const int W = std::max(1, std::min(kFFTTile / py, px));
      dim3 grid((unsigned)(px / W), (unsigned)pz, (unsigned)ncomp);
      fft_strided_kernel<double2><<<grid, kFFTThreads, 0, st>>>(data, f->np, py, f->logp[1], W, (size_t)px,
                                                                (size_t)px * py, f->tw[1], 0, py, py);
   }
   {  // z: stride px*py, one block per (x chunk, y)
      const int W = std::max(1, std::min(kFFTTile / pz, px));
      dim3 grid((unsigned)(px / W), (unsigned)py, (unsigned)ncomp);
      fft_strided_kernel<double2><<<grid, kFFTThreads, 0, st>>>(data, f->np, pz, f->logp[2], W, (size_t)px * py,
                                                                (size_t)px, f->tw[2], 0, pz, pz);
   }
   return cudaGetLastError();
}

// the x and y passes of the moment transform (forward: x then y; inverse: y
// then x), pruned to the G-box; the z passes run in fft_z_multiply_kernel
template <typename C>
cudaError_t fft_box(FFTField* f, C* grid_data, C* const* tw, bool inverse, cudaStream_t st, int* launches) {
   const int px = f->p[0], py = f->p[1];
   const int gx = f->g[0], gy = f->g[1], gz = f->g[2];
   auto xpass = [&]() {
      const int nrows = gy * gz;
      const int lines = std::max(1, std::min(kFFTTile / px, nrows));
      dim3 grid((unsigned)((nrows + lines - 1) / lines), 3u);
      fft_x_kernel<C><<<grid, kFFTThreads, 0, st>>>(grid_data, f->np, px, f->logp[0], lines, tw[0], inverse, nrows,
                                                    gy, py, inverse ? px : gx, inverse ? gx : px);
   };
   auto ypass = [&]() {
      const int W = std::max(1, std::min(kFFTTile / py, px));
      dim3 grid((unsigned)(px / W), (unsigned)gz, 3u);
      fft_strided_kernel<C><<<grid, kFFTThreads, 0, st>>>(grid_data, f->np, py, f->logp[1], W, (size_t)px,
                                                          (size_t)px * py, tw[1], inverse, inverse ? py : gy,
                                                          inverse ? gy : py);
   };
   if (inverse) { ypass(); xpass(); }
   else { xpass(); ypass(); }
   if (launches) *launches += 2;
   return cudaGetLastError();
}

template <typename C>
cudaError_t field_apply(FFTField* f, C* grid, const C* tspec, C* const* tw, const double* mag, double* field,
                        cudaStream_t st, int* launches) {
   cudaError_t e = cudaSuccess;
   const int nc = f->nc;
   const int nbox = f->g[0] * f->g[1] * f->g[2];
   scatter_moments_kernel<C><<<(nbox + 255) / 256, 256, 0, st>>>(nc, f->box_cell, f->g[0], f->g[1], nbox, mag, grid,
                                                                 f->p[0], f->p[1], f->np);
   if ((e = fft_box<C>(f, grid, tw, false, st, launches)) != cudaSuccess) return e;
   {
      const int pz = f->p[2];
      const int W = std::max(1, std::min(kFuseTile / (3 * pz), f->p[0]));
      dim3 g((unsigned)(f->p[0] / W), (unsigned)f->p[1]);
      fft_z_multiply_kernel<C><<<g, kFFTThreads, 0, st>>>(grid, tspec, f->np, f->p[0], f->p[1], pz, f->logp[2], W,
                                                          f->g[2], tw[2]);
   }
   if ((e = fft_box<C>(f, grid, tw, true, st, launches)) != cudaSuccess) return e;
   gather_field_kernel<C><<<(nc + 255) / 256, 256, 0, st>>>(nc, f->cell_lin, grid, f->np, 1.0 / (double)f->np, field);
   if (launches) *launches += 3;
   return cudaGetLastError();
}

}  // namespace

FFTField* fft_field_create(int nc, const double* cpos, const int* natoms, double size, bool fp32, cudaStream_t st,
                           cudaError_t* err, std::string* why) {
   *err = cudaSuccess;
   int first = -1;
   for (int c = 0; c < nc && first < 0; ++c)
      if (natoms[c] > 0) first = c;
   if (first < 0 || !(size > 0.0)) {
      *why = "no occupied cells";
      return nullptr;
   }
   // grid coordinates of every occupied cell relative to the first one
   std::vector<long long> gi(3 * (size_t)nc, 0);
   long long lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
   for (int c = 0; c < nc; ++c) {
      if (natoms[c] <= 0) continue;
      for (int a = 0; a < 3; ++a) {
         const double u = (cpos[4 * c + a] - cpos[4 * first + a]) / size;
         const double r = std::nearbyint(u);
         if (std::fabs(u - r) > 1e-9) {
            *why = "cell centres are not on one regular grid";
            return nullptr;
         }
         gi[3 * (size_t)c + a] = (long long)r;
         lo[a] = std::min(lo[a], (long long)r);
         hi[a] = std::max(hi[a], (long long)r);
      }
   }
   FFTField* f = new FFTField();
   f->nc = nc;
   size_t np = 1;
   for (int a = 0; a < 3; ++a) {
      const long long G = hi[a] - lo[a] + 1;
      int P = 2;
      while (P < 2 * G - 1 && P <= 1024) P <<= 1;
      if (P > 1024) {
         *why = "cell grid too large for the FFT solver";
         delete f;
         return nullptr;
      }
      f->g[a] = (int)G;
      f->p[a] = P;
      f->logp[a] = ilog2(P);
      np *= (size_t)P;
   }
   if (np > ((size_t)1 << 25)) {
      *why = "padded cell grid above 2^25 points";
      delete f;
      return nullptr;
   }
   f->np = np;
   // linear index of each occupied cell; two cells on one grid point are not a grid
   std::vector<int> lin(nc, -1);
   {
      std::vector<char> used(np, 0);
      for (int c = 0; c < nc; ++c) {
         if (natoms[c] <= 0) continue;
         const size_t x = (size_t)(gi[3 * (size_t)c] - lo[0]), y = (size_t)(gi[3 * (size_t)c + 1] - lo[1]),
                      z = (size_t)(gi[3 * (size_t)c + 2] - lo[2]);
         const size_t q = (z * f->p[1] + y) * f->p[0] + x;
         if (used[q]) {
            *why = "two cells share a grid point";
            delete f;
            return nullptr;
         }
         used[q] = 1;
         lin[c] = (int)q;
      }
   }
   cudaError_t e = cudaMalloc(&f->tspec, sizeof(double2) * 6 * np);
   if (e == cudaSuccess) e = cudaMalloc(&f->grid, sizeof(double2) * 3 * np);
   if (e == cudaSuccess) e = cudaMalloc(&f->cell_lin, sizeof(int) * std::max(nc, 1));
   if (e == cudaSuccess) e = cudaMemcpyAsync(f->cell_lin, lin.data(), sizeof(int) * nc, cudaMemcpyHostToDevice, st);
   // cell at each point of the G-box
   const size_t nbox = (size_t)f->g[0] * f->g[1] * f->g[2];
   std::vector<int> boxc(nbox, -1);
   for (int c = 0; c < nc; ++c) {
      if (lin[c] < 0) continue;
      const size_t q = (size_t)lin[c];
      const size_t x = q % f->p[0], y = (q / f->p[0]) % f->p[1], z = q / ((size_t)f->p[0] * f->p[1]);
      boxc[(z * f->g[1] + y) * f->g[0] + x] = c;
   }
   if (e == cudaSuccess) e = cudaMalloc(&f->box_cell, sizeof(int) * nbox);
   if (e == cudaSuccess) e = cudaMemcpyAsync(f->box_cell, boxc.data(), sizeof(int) * nbox, cudaMemcpyHostToDevice, st);
   std::vector<std::vector<double2>> tw(3);
   for (int a = 0; a < 3 && e == cudaSuccess; ++a) {
      const int P = f->p[a];
      tw[a].resize(P / 2);
      for (int k = 0; k < P / 2; ++k) {
         const double ang = -2.0 * M_PI * (double)k / (double)P;
         tw[a][k] = make_double2(std::cos(ang), std::sin(ang));
      }
      e = cudaMalloc(&f->tw[a], sizeof(double2) * (P / 2));
      if (e == cudaSuccess)
         e = cudaMemcpyAsync(f->tw[a], tw[a].data(), sizeof(double2) * (P / 2), cudaMemcpyHostToDevice, st);
   }
   if (e == cudaSuccess) {
      tensor_grid_kernel<<<grid_blocks(np), 256, 0, st>>>(f->tspec, np, f->p[0], f->p[1], f->p[2], f->g[0], f->g[1],
                                                          f->g[2], size);
      e = cudaGetLastError();
   }
   if (e == cudaSuccess) e = fft3d(f, f->tspec, 6, st);
   if (e == cudaSuccess && fp32) {
      // FP32 transforms: the spectra and twiddles rounded once; the FP64
      // moment grid is not needed
      f->fp32 = true;
      e = cudaMalloc(&f->tspec32, sizeof(float2) * 6 * np);
      if (e == cudaSuccess) e = cudaMalloc(&f->grid32, sizeof(float2) * 3 * np);
      if (e == cudaSuccess) {
         round_complex_kernel<<<grid_blocks(6 * np), 256, 0, st>>>(f->tspec, f->tspec32, 6 * np);
         e = cudaGetLastError();
      }
      for (int a = 0; a < 3 && e == cudaSuccess; ++a) {
         e = cudaMalloc(&f->tw32[a], sizeof(float2) * (f->p[a] / 2));
         if (e == cudaSuccess) {
            round_complex_kernel<<<1, 256, 0, st>>>(f->tw[a], f->tw32[a], (size_t)(f->p[a] / 2));
            e = cudaGetLastError();
         }
      }
   }
   if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // host tables above leave scope
   if (e == cudaSuccess && f->fp32) {
      cudaFree(f->tspec);
      cudaFree(f->grid);
      f->tspec = nullptr;
      f->grid = nullptr;
   }
   if (e != cudaSuccess) {
      *err = e;
      fft_field_destroy(f);
      return nullptr;
   }
   return f;
}

cudaError_t fft_field_apply(FFTField* f, const double* mag, double* field, cudaStream_t st, int* launches) {
   if (f->fp32) return field_apply<float2>(f, f->grid32, f->tspec32, f->tw32, mag, field, st, launches);
   return field_apply<double2>(f, f->grid, f->tspec, f->tw, mag, field, st, launches);
}

void fft_field_destroy(FFTField* f) {
   if (!f) return;
   cudaFree(f->tspec);
   cudaFree(f->grid);
   cudaFree(f->cell_lin);
   cudaFree(f->box_cell);
   cudaFree(f->tspec32);
   cudaFree(f->grid32);
   for (int a = 0; a < 3; ++a) {
      cudaFree(f->tw[a]);
      cudaFree(f->tw32[a]);
   }
   delete f;
}

void fft_field_shape(const FFTField* f, int p[3]) {
   for (int a = 0; a < 3; ++a) p[a] = f ? f->p[a] : 0;
}

}  // namespace vgpu
