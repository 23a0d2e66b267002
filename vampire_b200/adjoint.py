"""Gradients of a trajectory loss through the LLG-Heun integrator.

No counterpart in the reference (which has no derivatives).  The loss is
L = sum_{t=1..N} dt_SI (m_z(t) - target_t)^2, m_z the moment-weighted mean of
s_z after step t, and its gradient with respect to the exchange constant J
(every coupling scaled together), the uniaxial constant Ku and the applied
field (Hx, Hy, Hz) comes from the hand-written adjoint kernels of
libvgpu.so (vgpu_adjoint_llg, sqrt(N)-step checkpointing with recomputation),
wrapped as a torch.autograd.Function for fitting.  The adjoint runs in FP32
(FP64 sums for m_z, the loss and the gradients) unless the FP64 debug build
is asked for; both agree with central differences of the FP64 forward loss
to about 1e-5 on the benchmark problem.  For systems of several
materials, and tensor or DMI couplings, loss_and_grad_materials adds the
gradients with respect to each material pair's exchange constant and the
DMI strength (vgpu_adjoint_llg_materials).

The benchmark problem: simple-cubic 32^3 periodic, T = 0, alpha = 0.1,
dt = 1e-16 s, 2,000 steps, seeded initial state tilted 30 degrees from z;
target m_z(t) from J = 10e-21 J, Ku = 5e-24 J, H = (0, 0, 0.5) T; gradient at
J = 11.2e-21 J, Ku = 6.69e-24 J, H = (0, 0, 0.4) T.
"""
from __future__ import annotations

import ctypes as C
from typing import Sequence

import numpy as np

from . import system as S
from . import vgpu as V

TARGET_PARAMS = (10e-21, 5e-24, (0.0, 0.0, 0.5))
START_PARAMS = (11.2e-21, 6.69e-24, (0.0, 0.0, 0.4))


def tilted_spins(n: int, seed: int, theta_deg: float = 30.0) -> np.ndarray:
    """Unit spins at `theta_deg` from +z with seeded random azimuths."""
    rng = np.random.default_rng(seed)
    phi = rng.uniform(0.0, 2.0 * np.pi, n)
    th = np.deg2rad(theta_deg)
    return np.stack([np.sin(th) * np.cos(phi), np.sin(th) * np.sin(phi), np.full(n, np.cos(th))])


def system(J: float, Ku: float, H: Sequence[float], L: int = 32, seed: int = 2025) -> S.SpinSystem:
    """The adjoint benchmark system at parameters (J [J], Ku [J/atom], H [T])."""
    h = np.asarray(H, dtype=np.float64)
    m = S.Material(alpha=0.1, mu_s_muB=1.72, Ku=Ku)
    p = S.SimParams(dt_SI=1e-16, temperature=0.0, H_applied=1.0, H_vec=tuple(h), thermal=False)
    s = S.build("sc", L, L, L, 3.0, [m], [[J]], p, spins=tilted_spins(L ** 3, seed))
    s.uniaxial = True  # keep the anisotropy term on even when Ku = 0
    return s


class AdjointRunner:
    """Device simulation that returns (loss, dL/d[J, Ku, Hx, Hy, Hz]); the
    adjoint runs in `precision` ("fp32": production, "fp64": debug build)
    with FP64 sums for m_z, the loss and the gradients."""

    def __init__(self, L: int = 32, seed: int = 2025, device: int = 0, precision: str = "fp32"):
        self.L, self.seed, self.device, self.precision = L, seed, device, precision

    def loss_and_grad(self, J: float, Ku: float, H: Sequence[float], target: np.ndarray, every: int = 0):
        s = system(J, Ku, H, self.L, self.seed)
        with V.Simulation(s, device=self.device, precision=self.precision) as sim:
            tg = np.ascontiguousarray(target, dtype=np.float64)
            g = np.zeros(5)
            loss = C.c_double()
            sim._check(V.lib().vgpu_adjoint_llg(sim.handle, C.c_uint64(tg.size), tg.ctypes.data_as(V._D),
                                                C.c_double(s.params.dt_SI), C.c_int32(every), C.byref(loss),
                                                g.ctypes.data_as(V._D)))
        grad = np.array([g[0] / J, g[1], g[2], g[3], g[4]])
        return loss.value, grad

    def trajectory(self, J: float, Ku: float, H: Sequence[float], n_steps: int) -> np.ndarray:
        """m_z(t), t = 1..n_steps, of the device forward run."""
        s = system(J, Ku, H, self.L, self.seed)
        out = np.zeros(n_steps)
        with V.Simulation(s, device=self.device, precision=self.precision) as sim:
            sim._check(V.lib().vgpu_mz_trajectory(sim.handle, C.c_uint64(n_steps), out.ctypes.data_as(V._D)))
        return out


def loss_and_grad_materials(s: S.SpinSystem, target: np.ndarray, device: int = 0, every: int = 0,
                            precision: str = "fp32"):
    """Adjoint of the trajectory loss of any system (device build of
    `precision`, at most 8 materials, reciprocal couplings;
    vgpu_adjoint_llg_materials).
    Returns (loss, grad[5] as vgpu_adjoint_llg, dL/d(DMI scale),
    pair[M, M] = dL/d(scale of the couplings from material a to b)).  For
    an exchange matrix J_SI, dL/dJ_ab = pair[a, b] / J_SI[a, b]."""
    M = s.materials.size
    tg = np.ascontiguousarray(target, dtype=np.float64)
    g = np.zeros(5)
    pair = np.zeros(1 + M * M)
    loss = C.c_double()
    with V.Simulation(s, device=device, precision=precision) as sim:
        sim._check(V.lib().vgpu_adjoint_llg_materials(
            sim.handle, C.c_uint64(tg.size), tg.ctypes.data_as(V._D), C.c_double(s.params.dt_SI), C.c_int32(every),
            C.byref(loss), g.ctypes.data_as(V._D), pair.ctypes.data_as(V._D)))
    return loss.value, g, float(pair[0]), pair[1:].reshape(M, M)


def mz_trajectory(s: S.SpinSystem, n_steps: int, device: int = 0) -> np.ndarray:
    """m_z(t), t = 1..n_steps, of the device FP64 forward run of system s."""
    out = np.zeros(n_steps)
    with V.Simulation(s, device=device, precision="fp64") as sim:
        sim._check(V.lib().vgpu_mz_trajectory(sim.handle, C.c_uint64(n_steps), out.ctypes.data_as(V._D)))
    return out


def torch_loss_fn(runner: AdjointRunner, target: np.ndarray):
    """torch.autograd.Function mapping (J, Ku, H[3]) tensors to the scalar loss;
    backward supplies the adjoint gradient."""
    import torch

    class _TrajectoryLoss(torch.autograd.Function):
        @staticmethod
        def forward(ctx, J, Ku, H):
            loss, grad = runner.loss_and_grad(float(J), float(Ku), H.detach().cpu().numpy(), target)
            ctx.save_for_backward(torch.tensor(grad, dtype=torch.float64))
            return torch.tensor(loss, dtype=torch.float64)

        @staticmethod
        def backward(ctx, gout):
            (grad,) = ctx.saved_tensors
            return gout * grad[0], gout * grad[1], gout * grad[2:5]

    return _TrajectoryLoss.apply
