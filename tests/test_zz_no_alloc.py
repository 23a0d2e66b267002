"""vgpu_magnetization_noalloc: the magnetisation reduction for callers that
cannot call cudaMalloc (a plugin whose host framework's allocator owns the
device memory, or a time-critical loop that must not stall on cudaMalloc's
device synchronisation).  It allocates nothing itself; its block partials go
to a fixed scratch array compiled into libvgpu.so.

Checked through the C ABI against the existing entry point
(vgpu_stats_update + vgpu_stats_get_magnetization) on the same spins, on two
calls in a row (the scratch keeps the previous call's contents), on a system
large enough that every one of the 256 partial blocks walks several hundred
atoms (against an FP64 NumPy sum), and against the size limit.  This file
sorts last so a run that stops at its first failure has already run every
other test.
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


@pytest.mark.parametrize("size", [1, 3, 64])
def test_noalloc_large_system(vgpu_lib, size):
    """300,000 atoms (more than 256 blocks x 256 threads): random unit spins
    and moments, a random mask over `size` bins with a few out-of-range
    entries (skipped), against an FP64 NumPy masked sum, two calls in a row."""
    import torch
    from vampire_b200 import vgpu
    n = 300_000
    rng = np.random.default_rng(size)
    sp = rng.standard_normal((3, n))
    sp /= np.linalg.norm(sp, axis=0)
    sp = sp.astype(np.float32)
    mu = rng.uniform(0.5, 3.0, n).astype(np.float32)
    mask_np = rng.integers(0, size, n).astype(np.int32)
    if size > 1:
        mask_np[:: size * 100] = size if size % 2 else -1  # out of range: counted in no bin
    want = np.zeros(4 * size)
    for b in range(size):
        sel = mask_np == b
        v = (sp[:, sel].astype(np.float64) * mu[sel].astype(np.float64)).sum(1)
        tot = mu[sel].astype(np.float64).sum()
        if tot > 0:
            want[4 * b:4 * b + 4] = np.r_[v / np.linalg.norm(v), np.linalg.norm(v) / tot]
    t = {k: torch.tensor(v, device="cuda") for k, v in (("sx", sp[0]), ("sy", sp[1]), ("sz", sp[2]), ("mu", mu))}
    mask = torch.tensor(mask_np, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    for call in range(2):
        out = torch.full((4 * size,), float("nan"), dtype=torch.float64, device="cuda")
        rc = _call(vgpu_lib, t, mask, size, out, stream)
        assert rc == 0, vgpu._last_error(None)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        # |m| of random spins is small (~1e-3), so compare on the absolute sums' scale
        assert np.abs(got - want).max() < 1e-9, (call, np.abs(got - want).max())


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
