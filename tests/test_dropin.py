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
from oracle.refinputs import SC_MAT, sc_input

B200 = REPO / "oracle" / "_ref" / "vampire-b200"
SERIAL = REPO / "oracle" / "_ref" / "vampire-serial"

pytestmark = pytest.mark.skipif(not (B200.exists() and SERIAL.exists()),
                                reason="reference programs not built (python oracle/build_ref.py)")


def _run(exe, extra_input="", env=None, steps=200, T=0.0):
    d = Path(tempfile.mkdtemp(prefix="dropin_"))
    inp = sc_input(10, T=T, extra=f"sim:total-time-steps={steps}\nsim:time-steps-increment=10\n"
                                  "output:precision=16\noutput:time-steps\noutput:magnetisation\n" + extra_input)
    (d / "input").write_text(inp)
    (d / "m.mat").write_text(SC_MAT)
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
