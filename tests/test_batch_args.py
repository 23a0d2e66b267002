"""Fault injection on the host for the batched runner: vgpu_batch_create
checks its arguments and every system before it touches a device, so an
empty, mixed, corrupt or oversize batch is refused with VGPU_ERR_ARG (or the
validator's code) and a message, and no handle is made.  No GPU."""
import numpy as np
import pytest

from vampire_b200 import batch as B
from vampire_b200 import system as S
from vampire_b200 import vgpu as V


def _on_cpu():
    from conftest import gpu_available
    return not gpu_available()


def _params(n):
    return [{"temperature": 0.0, "H_start": (0.0, 0.0, 0.0), "H_end": (0.0, 0.0, 0.0), "n_ramp": 0}] * n


def _sc(n_mat, L=2):
    mats = [S.Material(alpha=0.1, mu_s_muB=1.72) for _ in range(n_mat)]
    J = np.full((n_mat, n_mat), 11.2e-21)
    types = np.arange(L ** 3) % n_mat
    return S.build("sc", L, L, L, 3.0, mats, J, S.SimParams(dt_SI=1e-16), types=types)


def _refused(systems, words=""):
    with pytest.raises(V.VGPUError) as e:
        B.Batch(systems, _params(len(systems)))
    assert words in str(e.value), str(e.value)
    return e.value.code


def test_empty_batch_is_refused(vgpu_lib):
    assert _refused([], "bad batch arguments") == V.ERR_ARG


def test_mixed_material_counts_are_refused(vgpu_lib):
    assert _refused([_sc(1), _sc(2)], "share material count") == V.ERR_ARG


def test_corrupt_system_in_a_batch_is_refused(vgpu_lib):
    bad = _sc(1)
    bad.spins = bad.spins.copy()
    bad.spins[0, 3] = np.nan
    assert _refused([_sc(1), bad, _sc(1)]) in (V.ERR_ARG, V.ERR_NAN)


def test_oversize_batch_is_refused(vgpu_lib):
    # the per-system material tables are limited to 65,536 rows (systems x materials)
    s = _sc(8)
    assert _refused([s] * 8193, "too many systems") == V.ERR_ARG
    if _on_cpu():  # one system fewer passes the argument checks and stops at the missing device
        assert _refused([s] * 8192) == V.ERR_CUDA
