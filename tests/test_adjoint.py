"""Adjoint gradients of the trajectory loss (CPU oracle and device kernels)
against central finite differences (FP64, h = 1e-6 relative), to 1e-4
relative."""
import numpy as np
import pytest

from oracle import oracle as O
from vampire_b200 import adjoint as A


def _oracle_loss(J, Ku, H, target, L, seed):
    s = A.system(J, Ku, H, L, seed)
    return O.OracleSystem(s).trajectory_loss(s.spins, target, s.params.dt_SI)


def _fd_grad(J, Ku, H, target, L, seed, rel=1e-6):
    p = np.array([J, Ku, *H], dtype=np.float64)
    scale = np.array([J, Ku, 0.4, 0.4, 0.4])  # field components step relative to |H|
    g = np.zeros(5)
    for k in range(5):
        h = rel * scale[k]
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        g[k] = (_oracle_loss(pp[0], pp[1], pp[2:], target, L, seed) -
                _oracle_loss(pm[0], pm[1], pm[2:], target, L, seed)) / (2 * h)
    return g


@pytest.mark.parametrize("every", [0, 7, 1000])
def test_cpu_adjoint_matches_finite_differences(every):
    L, seed, n = 5, 11, 150
    st = A.system(*A.TARGET_PARAMS, L=L, seed=seed)
    target = O.OracleSystem(st).mz_trajectory(st.spins, n)
    J, Ku, H = A.START_PARAMS
    s = A.system(J, Ku, H, L, seed)
    loss, g = O.OracleSystem(s).adjoint(s.spins, target, s.params.dt_SI, every=every)
    assert abs(loss - _oracle_loss(J, Ku, H, target, L, seed)) <= 1e-12 * abs(loss)
    grad = np.array([g[0] / J, g[1], g[2], g[3], g[4]])
    fd = _fd_grad(J, Ku, H, target, L, seed)
    scale = np.abs(fd).max(axis=0)
    for k in range(5):
        # components are compared relative to their own size; Hx, Hy (zero by
        # symmetry of the mean) relative to the largest field component
        ref = max(abs(fd[k]), 1e-3 * max(abs(fd[2:]).max(), 1e-300) if k >= 2 else abs(fd[k]))
        assert abs(grad[k] - fd[k]) <= 1e-4 * ref, (k, grad[k], fd[k])


@pytest.mark.gpu
def test_device_adjoint_config4(vgpu_lib):
    """Config 4: SC 32^3, 2,000 steps, sqrt(N) checkpointing on the device.
    The device gradient agrees with the FP64 CPU adjoint and with central
    finite differences of the device FP64 forward loss to 1e-4 relative."""
    runner = A.AdjointRunner(L=32, seed=2025)
    n = 2000
    target = runner.trajectory(*A.TARGET_PARAMS, n)
    J, Ku, H = A.START_PARAMS
    loss, grad = runner.loss_and_grad(J, Ku, H, target)
    # FP64 CPU adjoint on the same problem
    s = A.system(J, Ku, H, 32, 2025)
    cl, cg = O.OracleSystem(s).adjoint(s.spins, target, s.params.dt_SI)
    cgrad = np.array([cg[0] / J, cg[1], cg[2], cg[3], cg[4]])
    assert abs(loss - cl) <= 1e-9 * abs(cl)
    big = np.abs(cgrad).max()
    for k in range(5):
        ref = abs(cgrad[k]) if k < 2 or k == 4 else abs(cgrad[2:]).max()
        assert abs(grad[k] - cgrad[k]) <= 1e-4 * max(ref, 1e-12 * big), (k, grad[k], cgrad[k])
    # central differences of the device forward loss for J, Ku, Hz
    p = np.array([J, Ku, *H])
    for k, sc in ((0, J), (1, Ku), (4, 0.4)):
        h = 1e-6 * sc
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        lp = runner.loss_and_grad(pp[0], pp[1], pp[2:], target)[0]
        lm = runner.loss_and_grad(pm[0], pm[1], pm[2:], target)[0]
        fd = (lp - lm) / (2 * h)
        assert abs(grad[k] - fd) <= 1e-4 * abs(fd), (k, grad[k], fd)


@pytest.mark.gpu
def test_autograd_function(vgpu_lib):
    import torch
    runner = A.AdjointRunner(L=8, seed=3)
    target = runner.trajectory(*A.TARGET_PARAMS, 200)
    f = A.torch_loss_fn(runner, target)
    J = torch.tensor(11.2e-21, dtype=torch.float64, requires_grad=True)
    Ku = torch.tensor(6.69e-24, dtype=torch.float64, requires_grad=True)
    H = torch.tensor([0.0, 0.0, 0.4], dtype=torch.float64, requires_grad=True)
    loss = f(J, Ku, H)
    loss.backward()
    _, g = runner.loss_and_grad(11.2e-21, 6.69e-24, (0.0, 0.0, 0.4), target)
    assert float(J.grad) == pytest.approx(g[0], rel=1e-12)
    assert float(Ku.grad) == pytest.approx(g[1], rel=1e-12)
    assert np.allclose(H.grad.numpy(), g[2:], rtol=1e-12)
