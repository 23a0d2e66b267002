"""Spin snapshots in the reference's configuration-output format.

Fixtures (tests/golden/sc8_config): the reference program's own binary spin
files and meta files for the sc8_t0 input at steps 10 and 60
(tests/golden/make_golden.py sc8_config).  On the CPU the writers reproduce
those files byte for byte from their contents; on the GPU the FP64 build,
stepping the same system from the same start, gathers snapshots on the device
that write out byte for byte as the reference's files (the FP64 trajectory is
the reference's own), and the FP32 build to 1e-5."""
import numpy as np
import pytest

from conftest import REPO, load_golden

CFG = REPO / "tests" / "golden" / "sc8_config"


def _ref_data(k):
    b = (CFG / f"spins-{k:08d}.data").read_bytes()
    n = int(np.frombuffer(b[:8], dtype=np.uint64)[0])
    return b, np.frombuffer(b[8:], dtype=np.float64), n


def _ref_meta(k):
    lines = (CFG / f"spins-{k:08d}.meta").read_text().splitlines()
    val = {ln.split(":")[0]: ln.split(":", 1)[1].strip() for ln in lines if not ln.startswith("#") and ":" in ln}
    date = next(ln for ln in lines if ln.startswith("# Date: "))[len("# Date: "):]
    return lines, val, date


def test_writers_reproduce_reference_files(tmp_path):
    from vampire_b200 import config as cfg
    for k in (0, 1):
        raw, data, n = _ref_data(k)
        assert n == 512 and data.size == 3 * n
        cfg.write_spins_binary(tmp_path / "s.data", data)
        assert (tmp_path / "s.data").read_bytes() == raw
        lines, val, date = _ref_meta(k)
        m = [float(x) for x in val["Magnetisation"].split("\t")]
        cfg.write_spins_meta(tmp_path / "s.meta", f"spins-{k:08d}.data", float(val["Time"]),
                             float(val["Temperature"]), (0.0, 0.0, 1.0), 0.1, m, date=date)
        assert (tmp_path / "s.meta").read_text().splitlines() == lines


def test_text_writer_and_output_bounds(tmp_path):
    from vampire_b200 import config as cfg
    data = np.array([0.5, -0.25, 1e-15, 1.0, 0.0, -0.0])
    cfg.write_spins_text(tmp_path / "s.txt", data)
    assert (tmp_path / "s.txt").read_text() == "2\n0.5\t-0.25\t1e-15\n1\t0\t-0\n"
    coords = np.array([[0.0, 5.0, 10.0, 2.0], [0.0, 5.0, 10.0, 9.0], [0.0, 5.0, 10.0, 4.0]])
    assert cfg.output_atom_list(coords, (10.0, 10.0, 10.0)).tolist() == [0, 1, 2, 3]
    assert cfg.output_atom_list(coords, (10.0, 10.0, 10.0), (0.1, 0.0, 0.0), (0.6, 1.0, 1.0)).tolist() == [1, 3]


@pytest.mark.gpu
@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_device_snapshots_match_reference_files(vgpu_lib, tmp_path, prec):
    from vampire_b200 import config as cfg
    from vampire_b200 import vgpu as V
    s, _ = load_golden("sc8_t0")
    with V.Simulation(s, precision=prec) as sim:
        mid = sim.add_mask(*s.masks["system"])
        snaps = cfg.SpinSnapshots(sim, np.arange(s.n), directory=tmp_path)
        done = 0
        for k, step in ((0, 10), (1, 60)):
            sim.llg_heun(step - done)
            done = step
            sim.stats_update(magnetization=True)
            m, _, _ = sim.magnetization(mid)
            path = snaps.write(step * 1e-16, 0.0, (0.0, 0.0, 1.0), 0.1, m[:3])
            raw, ref, _ = _ref_data(k)
            if prec == "fp64":
                assert path.read_bytes() == raw
                got_meta = [ln for ln in (tmp_path / f"spins-{k:08d}.meta").read_text().splitlines()
                            if not ln.startswith("# Date")]
                ref_meta = [ln for ln in _ref_meta(k)[0] if not ln.startswith("# Date")]
                assert got_meta == ref_meta
            else:
                got = np.frombuffer(path.read_bytes()[8:], dtype=np.float64)
                assert np.abs(got - ref).max() < 1e-5


@pytest.mark.gpu
def test_snapshot_subset_order_and_errors(vgpu_lib):
    from vampire_b200 import vgpu as V
    s, _ = load_golden("sc8_t0")
    with V.Simulation(s, precision="fp64") as sim:
        with pytest.raises(V.VGPUError) as e:
            V.check(V.lib().vgpu_snapshot(sim.handle, None), sim.handle)
        assert e.value.code == V.ERR_STATE
        with pytest.raises(V.VGPUError) as e:
            sim.snapshot_setup([0, s.n])
        assert e.value.code == V.ERR_ARG
        ids = np.array([7, 3, 500, 3])
        sim.snapshot_setup(ids)
        got = sim.snapshot().reshape(-1, 3)
        np.testing.assert_array_equal(got, sim.spins()[:, ids].T)
