// FP32 instantiation of the fused LLG-Heun passes (production precision;
// FMA contraction on).
#include "llg_kernels.cuh"

namespace vgpu {
template cudaError_t launch_llg_pass<float>(const LLGArgs<float>&, int, int, int, cudaStream_t);
template cudaError_t launch_thermal_noise<float>(const LLGArgs<float>&, cudaStream_t);
}  // namespace vgpu
