// Far-field macrocell dipole sum by FFT convolution on the cell grid.
#pragma once
#include <cuda_runtime.h>

#include <string>

namespace vgpu {

struct FFTField;

// Builds the FFT far-field solver when every occupied cell centre lies on one
// regular grid of pitch `size` (to 1e-9 of the pitch) and the padded grid is
// small enough; otherwise returns nullptr with the reason in *why (and
// *err == cudaSuccess).  cpos holds x, y, z, w per cell (Angstrom); cells with
// natoms <= 0 are empty.  fp32: the transforms of every update in FP32 (the
// spectra computed in FP64 and rounded), else FP64.  Work is queued on `st`.
FFTField* fft_field_create(int nc, const double* cpos, const int* natoms, double size, bool fp32, cudaStream_t st,
                           cudaError_t* err, std::string* why);

// field[q * nc + c] = sum over occupied j != c of the bare point-dipole
// tensor (3 e e - 1)/r^3 (r in Angstrom) times m_j in mu_B, for q = x, y, z;
// mag is [3][nc] in J/T.  Empty cells get 0.
cudaError_t fft_field_apply(FFTField* f, const double* mag, double* field, cudaStream_t st, int* launches);

void fft_field_destroy(FFTField* f);

// padded grid size (points per axis) of a solver, for reporting
void fft_field_shape(const FFTField* f, int p[3]);

}  // namespace vgpu
