"""B200-native spin-update hot path of VAMPIRE (LLG-Heun, Metropolis MC,
macrocell dipole field, magnetisation/energy reductions).

The compute path is libvgpu.so (hand-written sm_100a CUDA behind the C ABI of
include/vgpu.h); this package holds its Python binding (``vgpu``), the
system model and synthetic builders (``system``) and the host-side mirror of
the reference's ``gpu::`` interface (``gpu``).
"""
__version__ = "0.1.0"
