// Macrocell dipole field (K5 cell moments, K6 cell-cell field).
#include "vgpu_ctx.cuh"

namespace vgpu {
void dipole_destroy(vgpu_ctx* h) { (void)h; }
}  // namespace vgpu

int dipole_after_step(vgpu_ctx* h) { (void)h; return VGPU_OK; }
