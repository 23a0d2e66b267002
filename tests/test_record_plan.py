"""Host-side record planning checked on the CPU (no GPU): the compact bond
words with their coupling dictionary, and the window plans of the
window-staged passes (vampire_b200/csrc/record_plan.h), built for the systems
the GPU tests and the benchmark use.  tests/plan_check.cpp is compiled with
g++ against the header and checks every invariant the device passes rely on
(alignment and bounds of every bulk copy, slot-to-neighbour mapping)."""
import shutil
import subprocess

import numpy as np
import pytest

from conftest import REPO

CUDA_INC = "/usr/local/cuda/include"


@pytest.fixture(scope="module")
def checker(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    exe = tmp_path_factory.mktemp("plan") / "plan_check"
    subprocess.run([gxx, "-O2", "-std=c++17", "-pthread", f"-I{REPO / 'vampire_b200' / 'csrc'}", f"-I{CUDA_INC}",
                    str(REPO / "tests" / "plan_check.cpp"), "-o", str(exe)], check=True)
    return exe


def _run(checker, s, tmp_path):
    assert s.exch_type == 2 and s.nl_type is None
    f = tmp_path / "sys.bin"
    with open(f, "wb") as fh:
        fh.write(np.array([s.n, len(s.materials)], dtype=np.int32).tobytes())
        fh.write(np.array([s.nl.size], dtype=np.int64).tobytes())
        for a in (s.nl_start, s.nl_end, s.nl, s.type):
            fh.write(np.ascontiguousarray(a, dtype=np.int32).tobytes())
        fh.write(np.ascontiguousarray(s.jlist, dtype=np.float64).tobytes())
    out = subprocess.run([str(checker), str(f)], capture_output=True, text=True)
    assert out.returncode == 0, out.stderr
    return out.stdout.split("\n")


def _fcc(L, kind="scalar", seed=7):
    from vampire_b200 import system
    if kind == "open":
        return system.config_fcc_tensor(L=L, seed=seed, periodic=(True, True, False))
    s = system.config_fcc_tensor(L=L, seed=seed)
    if kind != "scalar":
        J = s.jlist.reshape(-1, 3, 3).copy()
        if kind == "diag":
            J[:, 1, 1] *= 0.9
            J[:, 2, 2] *= 1.1
        else:
            d = np.random.default_rng(3).normal(scale=0.05, size=(J.shape[0], 3))
            J[:, 2, 1], J[:, 1, 2] = d[:, 0], -d[:, 0]
            J[:, 0, 2], J[:, 2, 0] = d[:, 1], -d[:, 1]
            J[:, 1, 0], J[:, 0, 1] = d[:, 2], -d[:, 2]
        s.jlist = np.ascontiguousarray(J.ravel())
    return s


@pytest.mark.parametrize("L,kind", [(2, "scalar"), (5, "scalar"), (12, "scalar"), (5, "diag"), (6, "open"),
                                    (25, "scalar")])
def test_compact_and_window_plans(checker, tmp_path, L, kind):
    lines = _run(checker, _fcc(L, kind), tmp_path)
    ncomp = int(lines[0].split()[1])
    assert 0 < ncomp <= 512
    win = [ln for ln in lines if ln.startswith("window")]
    assert len(win) == 3 and all("none" not in ln for ln in win), win


def test_many_couplings_have_no_compact_records(checker, tmp_path):
    lines = _run(checker, _fcc(5, "random_d"), tmp_path)
    assert lines[0] == "compact none"


def test_shuffled_numbering_has_no_window(checker, tmp_path):
    """A random atom numbering scatters every tile's neighbours over the whole
    system: the window plan refuses it (the passes keep compact records)."""
    from vampire_b200 import system
    s = _fcc(12)
    perm = np.random.default_rng(5).permutation(s.n)
    inv = np.empty_like(perm)
    inv[perm] = np.arange(s.n)
    deg = s.nl_end - s.nl_start + 1
    rows = [s.nl[s.nl_start[p]: s.nl_end[p] + 1] for p in perm]
    jl = s.jlist.reshape(-1, 9)
    jrows = [jl[s.nl_start[p]: s.nl_end[p] + 1] for p in perm]
    nl = inv[np.concatenate(rows)].astype(np.int32)
    start = np.concatenate([[0], np.cumsum(deg[perm])[:-1]]).astype(np.int32)
    t = system.SpinSystem(n=s.n, nl_start=start, nl_end=(start + deg[perm] - 1).astype(np.int32), nl=nl,
                          jlist=np.ascontiguousarray(np.concatenate(jrows).ravel()), exch_type=2,
                          type=s.type[perm].astype(np.int32), materials=s.materials, spins=s.spins[:, perm],
                          params=s.params)
    lines = _run(checker, t, tmp_path)
    assert lines[0].startswith("compact ")
    assert any("none" in ln for ln in lines if ln.startswith("window")), lines
