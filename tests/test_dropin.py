"""The drop-in: the unmodified reference program built with -DCUDA, whose
vcuda:: backend is vampire_b200/host/vcuda_b200.cpp over libvgpu.so
(oracle/_ref/vampire-b200, built by oracle/build_ref.py), against the same
reference built serial (oracle/_ref/vampire-serial) on the same input.
"""
import os
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

from conftest import REPO, gpu_available
from oracle.refinputs import SC_MAT, fcc_input, fcc_mat, sc_input

B200 = REPO / "oracle" / "_ref" / "vampire-b200"
SERIAL = REPO / "oracle" / "_ref" / "vampire-serial"

pytestmark = pytest.mark.skipif(not (B200.exists() and SERIAL.exists()),
                                reason="reference programs not built (python oracle/build_ref.py)")


def _run(exe, extra_input="", env=None, steps=200, T=0.0, system="sc10"):
    d = Path(tempfile.mkdtemp(prefix="dropin_"))
    out = (f"sim:total-time-steps={steps}\nsim:time-steps-increment=10\n"
           "output:precision=16\noutput:time-steps\noutput:magnetisation\n" + extra_input)
    if system == "sc10":
        inp, mat = sc_input(10, T=T, extra=out), SC_MAT
    else:  # FCC 10^3 A/B alloy, tensor exchange + DMI + cubic anisotropy
        inp, mat = fcc_input(10, T=T, extra=out), fcc_mat()
    (d / "input").write_text(inp)
    (d / "m.mat").write_text(mat)
    e = dict(os.environ)
    e.update(env or {})
    r = subprocess.run([str(exe)], cwd=d, capture_output=True, text=True, timeout=600, env=e)
    return r, d


def _table(d):
    rows = [l.split() for l in (d / "output").read_text().splitlines() if l.strip() and not l.startswith("#")]
    return np.array([[float(x) for x in r] for r in rows])


def test_dropin_fails_loudly_without_device():
    if gpu_available():
        pytest.skip("a GPU is present")
    r, _ = _run(B200, steps=10)
    assert r.returncode != 0
    assert "B200 backend" in r.stdout + r.stderr


@pytest.mark.gpu
def test_dropin_fp64_matches_serial_reference():
    """gpu::initialize/llg_heun/stats through the B200 backend (FP64 build)
    reproduce the reference program's magnetisation output."""
    rs, ds = _run(SERIAL)
    rg, dg = _run(B200, env={"VGPU_PRECISION": "fp64"})
    assert rs.returncode == 0, rs.stdout[-2000:]
    assert rg.returncode == 0, rg.stdout[-2000:] + rg.stderr[-2000:]
    a, b = _table(ds), _table(dg)
    assert a.shape == b.shape and a.shape[0] >= 20
    assert np.abs(a - b).max() < 1e-10


@pytest.mark.gpu
def test_dropin_fp32_device_statistics():
    """FP32 build with statistics on the device (gpu:calculate-statistics-on-cpu=false)."""
    rs, ds = _run(SERIAL, steps=100)
    rg, dg = _run(B200, extra_input="gpu:calculate-statistics-on-cpu=false\n", steps=100)
    assert rg.returncode == 0, rg.stdout[-2000:] + rg.stderr[-2000:]
    a, b = _table(ds), _table(dg)
    assert a.shape == b.shape
    assert np.abs(a - b).max() < 1e-5


@pytest.mark.gpu
@pytest.mark.parametrize("solver", ["macrocell", "tensor"])
def test_dropin_fcc_dmi_dipole_on_device(solver):
    """FCC 10^3 A/B alloy with tensor exchange, three-site DMI, cubic
    anisotropy and the macrocell dipole field (2x2x2-cell macrocells, update
    every 100 steps): the reference program with the B200 backend (FP64
    build) holds the dipole solver on the device -- no spins cross to the
    host for dipole::calculate_field -- and reproduces the serial reference's
    magnetisation output over 300 steps, across the updates at steps 100, 200
    and 300."""
    dip = f"cells:macro-cell-size=7.08 !A\ndipole:solver={solver}\ndipole:field-update-rate=100\n"
    rs, ds = _run(SERIAL, extra_input=dip, steps=300, system="fcc10")
    rg, dg = _run(B200, extra_input=dip, env={"VGPU_PRECISION": "fp64"}, steps=300, system="fcc10")
    assert rs.returncode == 0, rs.stdout[-2000:]
    assert rg.returncode == 0, rg.stdout[-2000:] + rg.stderr[-2000:]
    log = "".join(p.read_text() for p in dg.glob("log*"))
    assert "dipole field on the device" in log
    a, b = _table(ds), _table(dg)
    assert a.shape == b.shape and a.shape[0] >= 30
    assert np.abs(a - b).max() < 1e-10, np.abs(a - b).max()


HARNESS = REPO / "oracle" / "_ref" / "vampire-harness"
HARNESS_B200 = REPO / "oracle" / "_ref" / "vampire-harness-b200"


def _mc_run(exe, extra_args, T=600.0, eq=1000, av=3000, every=10, integrator="monte-carlo", extra=""):
    from oracle import oracle as O
    mat = SC_MAT.replace("initial-spin-direction=random", "initial-spin-direction=0,0,1")
    inp = sc_input(10, T=T, H=0.0, integrator=integrator, extra="montecarlo:algorithm=angle\n" + extra)
    d = Path(tempfile.mkdtemp(prefix="dropin_mc_"))
    (d / "input").write_text(inp)
    (d / "m.mat").write_text(mat)
    out = d / "out"
    out.mkdir()
    r = subprocess.run([str(exe), "--out", str(out), "--steps", str(eq + av), "--mag-every", str(every),
                        "--mag-start", str(eq)] + extra_args, cwd=d, capture_output=True, text=True, timeout=900)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    return O.load_dump(out), d


@pytest.mark.gpu
@pytest.mark.skipif(not HARNESS_B200.exists(), reason="B200 harness not built")
def test_dropin_mc_hook_matches_serial_statistically():
    """The gpu::mc_step hook (the host-side change INTEGRATION.md shows,
    vcuda::mc_step -> vgpu_mc_sweep) run inside the reference's own start-up
    and step loop: SC 10^3 at 600 K, 1000 + 3000 sweeps, against the
    reference's sequential montecarlo::mc_step on the same input.  Every
    sweep makes N trials on both; <|m|> agrees within 4 standard errors
    (10 blocks of 300 sweeps each)."""
    ds, _ = _mc_run(HARNESS, [])
    dg, wd = _mc_run(HARNESS_B200, ["--gpu-mc"])
    log = "".join(p.read_text() for p in wd.glob("log*"))
    assert "B200 backend" in log
    res = []
    for d in (ds, dg):
        tr = d["mag_trace"].reshape(-1, 4)[:, 3]
        b = tr[: len(tr) // 10 * 10].reshape(10, -1).mean(1)
        res.append((tr.mean(), b.std(ddof=1) / np.sqrt(10)))
        moves, _ = d["mc_counters"]
        assert moves == 1000 * 4000
    (ms, es), (mg, eg) = res
    print(f"<|m|> serial {ms:.5f} +- {es:.5f}, gpu hook {mg:.5f} +- {eg:.5f}")
    assert abs(ms - mg) <= 4.0 * np.hypot(es, eg) + 1e-4


@pytest.mark.gpu
@pytest.mark.skipif(not HARNESS_B200.exists(), reason="B200 harness not built")
def test_dropin_cmc_hook_matches_serial_statistically():
    """Constrained Monte Carlo through the gpu::cmc_step hook (vcuda::cmc_step
    -> vgpu_cmc_setup with sim::constraint_phi/theta, vgpu_cmc_sweep) inside
    the reference's start-up: SC 10^3 at 600 K, constraint (30, 45) degrees,
    1000 + 3000 steps, against the reference's montecarlo::cmc_step on the
    same input.  The moment stays along the constraint and its size agrees
    within 4 standard errors; the counters come back into montecarlo::cmc."""
    extra = "sim:constraint-angle-phi=30\nsim:constraint-angle-theta=45\n"
    ds, _ = _mc_run(HARNESS, [], integrator="constrained-monte-carlo", extra=extra)
    dg, _ = _mc_run(HARNESS_B200, ["--gpu-mc"], integrator="constrained-monte-carlo", extra=extra)
    pv = ds["cmc_frame"][9:12]  # the device's frame equals it (tests/test_cmc.py)
    res = []
    for d in (ds, dg):
        tr = d["mag_trace"].reshape(-1, 4)[:, :3]
        par = tr @ pv
        assert np.abs(tr - np.outer(par, pv)).max() < 1e-5
        b = par[: len(par) // 10 * 10].reshape(10, -1).mean(1)
        res.append((par.mean(), b.std(ddof=1) / np.sqrt(10)))
        total, success, erej, srej = d["cmc_counters"]
        assert total >= 0.9 * 1000 * 4000 and success + erej + srej == total
    (ms, es), (mg, eg) = res
    print(f"<m.e> serial {ms:.5f} +- {es:.5f}, gpu hook {mg:.5f} +- {eg:.5f}")
    assert abs(ms - mg) <= 4.0 * np.hypot(es, eg) + 1e-4
