"""B200-native spin-update hot path of VAMPIRE (LLG-Heun, Metropolis MC,
macrocell dipole field, magnetisation/energy reductions).

The compute path is libvgpu.so (hand-written sm_100a CUDA behind the C ABI of
include/vgpu.h, built by ``build``).  This package holds its Python binding
(``vgpu``), the system model and synthetic builders (``system``), the
batched runner with its autotuner (``batch``), the adjoint autograd wrapper
(``adjoint``), the multi-GPU shards (``shard``) and the spin-snapshot writer
(``config``).  The host-side mirror of the reference's ``gpu::`` /
``vcuda::`` interface is C++: ``host/vcuda_b200.cpp``.
"""
__version__ = "0.1.0"
