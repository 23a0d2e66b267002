"""The C-ABI library loads, exports every symbol include/vgpu.h declares, and
its host-side validation works without a GPU."""
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

from conftest import REPO, load_golden


def declared_symbols():
    out = set()
    for h in (REPO / "include").glob("*.h"):
        out |= set(re.findall(r"^\s*(?:int|const char\*|void)\s+(vgpu_\w+)\s*\(", h.read_text(), re.M))
    return out


def test_exports_every_declared_symbol(vgpu_lib):
    syms = declared_symbols()
    assert len(syms) >= 10
    nm = subprocess.run(["nm", "-D", "--defined-only", str(REPO / "vampire_b200" / "libvgpu.so")],
                        capture_output=True, text=True, check=True).stdout
    exported = set(re.findall(r" T (vgpu_\w+)", nm))
    missing = syms - exported
    assert not missing, missing
    for s in syms:
        getattr(vgpu_lib, s)  # resolvable through ctypes


def test_version(vgpu_lib):
    from vampire_b200 import vgpu
    assert "sm_100a" in vgpu.version()


def test_validate_accepts_reference_system(vgpu_lib):
    from vampire_b200 import vgpu
    s, _ = load_golden("fcc4_dmi_t300")
    vgpu.validate_system(s)


@pytest.mark.parametrize("corruption", ["neighbour_out_of_range", "row_past_end", "bad_material", "nan_spin",
                                        "negative_neighbour"])
def test_validate_rejects_corrupt_input(vgpu_lib, corruption):
    """Fault injection on the host: a corrupt CSR, a bad material id or a NaN
    spin is refused with a message before anything reaches a device."""
    from vampire_b200 import vgpu
    s, _ = load_golden("sc6_open_t300")
    s = s.copy()
    if corruption == "neighbour_out_of_range":
        s.nl = s.nl.copy(); s.nl[5] = s.n + 3
    elif corruption == "negative_neighbour":
        s.nl = s.nl.copy(); s.nl[9] = -1
    elif corruption == "row_past_end":
        s.nl_end = s.nl_end.copy(); s.nl_end[-1] = s.num_bonds + 4
    elif corruption == "bad_material":
        s.type = s.type.copy(); s.type[3] = 7
    elif corruption == "nan_spin":
        s.spins = s.spins.copy(); s.spins[1, 2] = np.nan
    with pytest.raises(vgpu.VGPUError) as e:
        vgpu.validate_system(s)
    assert e.value.code in (vgpu.ERR_ARG, vgpu.ERR_NAN)
    assert len(str(e.value)) > 20


def test_no_cpu_fallback_without_device(vgpu_lib):
    """Without a CUDA device the library refuses (no silent CPU path)."""
    from conftest import gpu_available
    from vampire_b200 import vgpu
    if gpu_available():
        pytest.skip("a GPU is present")
    s, _ = load_golden("sc8_t0")
    with pytest.raises(vgpu.VGPUError) as e:
        vgpu.Simulation(s)
    assert e.value.code == vgpu.ERR_CUDA
