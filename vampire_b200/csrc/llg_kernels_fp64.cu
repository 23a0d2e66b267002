// FP64 instantiation of the fused LLG-Heun passes.  Built with -fmad=false
// (see vampire_b200/build.py) so that every product and sum rounds as the
// reference's g++ -O3 x86-64 build does (no fused multiply-add), and run with
// the stored predictor increment: the FP64 trajectory then follows the
// reference CPU integrator to the last bit.
#include "llg_kernels.cuh"

namespace vgpu {
template cudaError_t launch_llg_pass<double>(const LLGArgs<double>&, int, int, int, cudaStream_t);
template cudaError_t launch_thermal_noise<double>(const LLGArgs<double>&, cudaStream_t);
}  // namespace vgpu
