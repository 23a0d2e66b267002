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
@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_device_adjoint_config4(vgpu_lib, prec):
    """Config 4: SC 32^3, 2,000 steps, sqrt(N) checkpointing on the device,
    in the FP32 production build and the FP64 debug build.  The device
    gradient agrees with the FP64 CPU adjoint (1e-4 relative; the FP32
    trajectory's own rounding is the difference there) and with central
    finite differences of the device FP64 forward loss to 1e-4 relative."""
    runner = A.AdjointRunner(L=32, seed=2025, precision=prec)
    r64 = A.AdjointRunner(L=32, seed=2025, precision="fp64")
    n = 2000
    target = r64.trajectory(*A.TARGET_PARAMS, n)
    J, Ku, H = A.START_PARAMS
    loss, grad = runner.loss_and_grad(J, Ku, H, target)
    # FP64 CPU adjoint on the same problem
    s = A.system(J, Ku, H, 32, 2025)
    cl, cg = O.OracleSystem(s).adjoint(s.spins, target, s.params.dt_SI)
    cgrad = np.array([cg[0] / J, cg[1], cg[2], cg[3], cg[4]])
    assert abs(loss - cl) <= (1e-4 if prec == "fp32" else 1e-9) * abs(cl)
    big = np.abs(cgrad).max()
    for k in range(5):
        ref = abs(cgrad[k]) if k < 2 or k == 4 else abs(cgrad[2:]).max()
        assert abs(grad[k] - cgrad[k]) <= 1e-4 * max(ref, 1e-12 * big), (k, grad[k], cgrad[k])
    # central differences of the device FP64 forward loss for J, Ku, Hz
    p = np.array([J, Ku, *H])
    for k, sc in ((0, J), (1, Ku), (4, 0.4)):
        h = 1e-6 * sc
        pp, pm = p.copy(), p.copy()
        pp[k] += h
        pm[k] -= h
        lp = r64.loss_and_grad(pp[0], pp[1], pp[2:], target)[0]
        lm = r64.loss_and_grad(pm[0], pm[1], pm[2:], target)[0]
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


def _alloy(J, D, H, L=3, seed=5):
    """FCC L^3 periodic A/B alloy (moments 1.72 and 2.3 mu_B, so the
    normalised couplings are not symmetric), nn exchange matrix J [J], the
    three-site DMI with constants D [J], cubic anisotropy, T = 0, applied
    field H [T], spins tilted 30 degrees from z."""
    from vampire_b200 import system as S
    mats = [S.Material(alpha=0.05, mu_s_muB=1.72, Kc=1e-24), S.Material(alpha=0.1, mu_s_muB=2.3, Kc=0.5e-24)]
    p = S.SimParams(dt_SI=1e-16, temperature=0.0, H_applied=1.0, H_vec=tuple(H), thermal=False)
    n = 4 * L ** 3
    types = (np.random.default_rng(seed).random(n) < 0.5).astype(np.int32)
    return S.build("fcc", L, L, L, 3.54, mats, np.asarray(J), p, types=types, dmi_SI=np.asarray(D),
                   spins=A.tilted_spins(n, seed + 1))


ALLOY_J = np.array([[11.2e-21, 5e-21], [5e-21, 9e-21]])
ALLOY_H = (0.0, 0.0, 0.4)


def _alloy_loss(J, D, H, target):
    s = _alloy(J, D, H)
    return O.OracleSystem(s).trajectory_loss(s.spins, target, s.params.dt_SI)


def _alloy_target(n):
    st = _alloy(0.9 * ALLOY_J, 0.12 * ALLOY_J, (0.0, 0.0, 0.5))
    return O.OracleSystem(st).mz_trajectory(st.spins, n)


def test_cpu_adjoint_two_material_dmi_matches_finite_differences():
    """Two materials of different moments with tensor exchange + three-site
    DMI: the CPU adjoint's transposed gather (mu_s-weighted) against central
    differences (h = 1e-6 relative) of the oracle's forward loss, for the
    common coupling scale and the field; 1e-4 relative."""
    n = 150
    target = _alloy_target(n)
    D = 0.1 * ALLOY_J
    s = _alloy(ALLOY_J, D, ALLOY_H)
    loss, g = O.OracleSystem(s).adjoint(s.spins, target, s.params.dt_SI)
    assert abs(loss - _alloy_loss(ALLOY_J, D, ALLOY_H, target)) <= 1e-12 * abs(loss)
    h = 1e-6
    fd_scale = (_alloy_loss(ALLOY_J * (1 + h), D * (1 + h), ALLOY_H, target) -
                _alloy_loss(ALLOY_J * (1 - h), D * (1 - h), ALLOY_H, target)) / (2 * h)
    assert abs(g[0] - fd_scale) <= 1e-4 * abs(fd_scale), (g[0], fd_scale)
    hz = 1e-6 * 0.4
    fd_hz = (_alloy_loss(ALLOY_J, D, (0, 0, 0.4 + hz), target) - _alloy_loss(ALLOY_J, D, (0, 0, 0.4 - hz), target)) / (2 * hz)
    assert abs(g[4] - fd_hz) <= 1e-4 * abs(fd_hz), (g[4], fd_hz)


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_device_adjoint_per_material_exchange_and_dmi(vgpu_lib, prec):
    """The device adjoint on the two-material DMI alloy: the five gradients
    equal the FP64 CPU adjoint's (1e-9 relative in the FP64 build, 1e-4 in
    FP32), and the per-material-pair exchange gradients dL/dJ_ab and the
    DMI-scale gradient agree with central differences (h = 1e-6 relative) of
    the oracle's forward loss to 1e-4 relative; their sum is the
    common-scale gradient."""
    n = 150
    target = _alloy_target(n)
    D = 0.1 * ALLOY_J
    s = _alloy(ALLOY_J, D, ALLOY_H)
    loss, g, gdmi, pair = A.loss_and_grad_materials(s, target, precision=prec)
    cl, cg = O.OracleSystem(s).adjoint(s.spins, target, s.params.dt_SI)
    tol = 1e-4 if prec == "fp32" else 1e-9
    assert abs(loss - cl) <= max(tol, 1e-10) * abs(cl)
    for k in (0, 1, 4):
        assert abs(g[k] - cg[k]) <= tol * max(abs(cg[k]), 1e-30), (k, g[k], cg[k])
    # the same sum by bonds and by fields: FP32 products rounded apart in FP32
    assert abs(pair.sum() + gdmi - g[0]) <= (1e-6 if prec == "fp32" else 1e-9) * abs(g[0])
    h = 1e-6
    for a in range(2):
        for b in range(2):
            Jp, Jm = ALLOY_J.copy(), ALLOY_J.copy()
            Jp[a, b] *= 1 + h
            Jm[a, b] *= 1 - h
            fd = (_alloy_loss(Jp, D, ALLOY_H, target) - _alloy_loss(Jm, D, ALLOY_H, target)) / (2 * h * ALLOY_J[a, b])
            got = pair[a, b] / ALLOY_J[a, b]
            assert abs(got - fd) <= 1e-4 * abs(fd), (a, b, got, fd)
    fd = (_alloy_loss(ALLOY_J, D * (1 + h), ALLOY_H, target) - _alloy_loss(ALLOY_J, D * (1 - h), ALLOY_H, target)) / (2 * h)
    assert abs(gdmi - fd) <= 1e-4 * abs(fd), (gdmi, fd)


@pytest.mark.gpu
def test_device_adjoint_refuses_non_reciprocal_couplings(vgpu_lib):
    """An exchange matrix with J_01 != J_10 gives couplings that are not
    reciprocal; the adjoint says so instead of returning a wrong gradient."""
    from vampire_b200 import vgpu
    J = ALLOY_J.copy()
    J[0, 1] *= 1.5
    s = _alloy(J, 0.1 * ALLOY_J, ALLOY_H)
    with pytest.raises(vgpu.VGPUError) as e:
        A.loss_and_grad_materials(s, np.zeros(10))
    assert "reciprocal" in str(e.value)
