"""vgpu_magnetization_noalloc: the magnetisation reduction for callers that
cannot call cudaMalloc (graph capture that forbids allocation, plugins whose
host framework owns the device memory).  It allocates nothing itself; its
block partials go to a fixed scratch array compiled into libvgpu.so.

Checked through the C ABI against the existing entry point
(vgpu_stats_update + vgpu_stats_get_magnetization) on the same spins, on two
calls in a row (the scratch keeps the previous call's contents), and against
the size limit.  This file sorts last so a run that stops at its first
failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import load_golden, ref_spins

pytestmark = pytest.mark.gpu


def _call(lib, t, mask, size, out, stream):
    return lib.vgpu_magnetization_noalloc(
        C.c_void_p(t["sx"].data_ptr()), C.c_void_p(t["sy"].data_ptr()), C.c_void_p(t["sz"].data_ptr()),
        C.c_void_p(t["mu"].data_ptr()), C.c_void_p(mask.data_ptr()), C.c_int32(mask.numel()), C.c_int32(size),
        C.c_void_p(out.data_ptr()), C.c_void_p(stream))


@pytest.mark.parametrize("name,step,mask_name", [("fcc4_dmi_t300", 2, "material"), ("sc20_t0", 10000, "system")])
def test_noalloc_matches_stats_entry_point(vgpu_lib, name, step, mask_name):
    import torch
    from vampire_b200 import vgpu
    s, d = load_golden(name)
    mask_np, size = s.masks[mask_name]
    sp = ref_spins(d, step)
    with vgpu.Simulation(s) as sim:
        sim.set_spins(sp)
        mid = sim.add_mask(mask_np, size)
        sim.stats_update(magnetization=True)
        want, _, _ = sim.magnetization(mid)
        dev_spins = sim.spins().astype(np.float32)  # the FP32 state the device reduced
    mu = (s.materials["mu_s_SI"] / 9.27400915e-24).astype(np.float32)[s.type]
    t = {k: torch.tensor(v, device="cuda") for k, v in
         (("sx", dev_spins[0]), ("sy", dev_spins[1]), ("sz", dev_spins[2]), ("mu", mu))}
    mask = torch.tensor(mask_np.astype(np.int32), device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        out = torch.full((4 * size,), float("nan"), dtype=torch.float64, device="cuda")
        rc = _call(vgpu_lib, t, mask, size, out, stream)
        assert rc == 0, vgpu._last_error(None)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        assert np.abs(got - want).max() < 1e-9, (call, got, want)


def test_noalloc_rejects_oversize_mask(vgpu_lib):
    import torch
    from vampire_b200 import vgpu
    n = 1000
    t = {k: torch.ones(n, dtype=torch.float32, device="cuda") for k in ("sx", "sy", "sz", "mu")}
    mask = torch.zeros(n, dtype=torch.int32, device="cuda")
    out = torch.zeros(4 * 65, dtype=torch.float64, device="cuda")
    rc = _call(vgpu_lib, t, mask, 65, out, 0)
    assert rc == vgpu.ERR_ARG
    assert "64" in vgpu._last_error(None)
