"""Batched uneven systems (persistent cluster kernel, CUDA graph, autotuner).

Every batched system must reproduce the same system run alone (plain
two-launch path, noise seed + k), whatever the cluster shape (or with the
batch stepped by the ordinary passes, shape 0); in FP64 at T=0 it must follow
the FP64 oracle.  The persistent launch must beat one plain
launch sequence per system by at least 5x.
"""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _small_ensemble(n=12, temperature=None, n_ramp=400):
    from vampire_b200 import batch as B
    return B.nanoparticle_ensemble(n=n, seed=3, n_ramp=n_ramp, temperature=temperature)


@pytest.mark.parametrize("shape", [(1, 128), (2, 256), (4, 256), (8, 128), (0, 0)])
def test_persistent_matches_single_runs(vgpu_lib, shape):
    """T>0 with field sweep: each system of the persistent batch (or of the
    batch stepped by the ordinary passes, shape (0, 0)) equals the system
    stepped alone with its own temperature, swept field and seed + k, and the
    records are the systems' magnetisation."""
    from vampire_b200 import batch as B
    from vampire_b200 import vgpu
    systems, params = _small_ensemble()
    steps = 60
    with B.Batch(systems, params, noise_seed=11) as b:
        b.set_shape(*shape)
        b.run(steps, record_every=20)
        got = b.spins()
        hist = b.history()
    assert hist.shape == (3, len(systems), 4)
    for k in (0, 5, len(systems) - 1):
        s = systems[k].copy()
        s.params.temperature = params[k]["temperature"]
        with vgpu.Simulation(s, noise_seed=11 + k) as sim:
            for t in range(steps):
                f = min(t, params[k]["n_ramp"]) / params[k]["n_ramp"]
                s.params.H_applied = 2.0 - 4.0 * f
                sim.set_params(s.params)
                sim.llg_heun(1)
            want = sim.spins()
        assert np.abs(got[k] - want).max() < 2e-5, (k, np.abs(got[k] - want).max())
        # the record after 60 steps is this system's magnetisation
        v = (got[k] * 1.72).sum(1)
        np.testing.assert_allclose(hist[-1, k, :3], v / np.linalg.norm(v), atol=1e-6)


def test_plain_batched_path_matches_persistent(vgpu_lib):
    from vampire_b200 import batch as B
    systems, params = _small_ensemble()
    with B.Batch(systems, params, noise_seed=2) as a, B.Batch(systems, params, noise_seed=2) as b:
        a.llg_heun(50)
        b.set_shape(4, 256)
        b.run(50)
        for x, y in zip(a.spins(), b.spins()):
            assert np.abs(x - y).max() < 2e-6


def test_fp64_batch_follows_oracle_at_t0(vgpu_lib):
    from oracle import oracle as O
    from vampire_b200 import batch as B
    systems, params = _small_ensemble(n=6, temperature=0.0, n_ramp=0)
    for p in params:
        p["H_end"] = p["H_start"]
    rng = np.random.default_rng(1)
    for s in systems:  # tilted start so that the dynamics is non-trivial
        sp = s.spins + 0.4 * rng.standard_normal(s.spins.shape)
        s.spins = sp / np.linalg.norm(sp, axis=0)
    with B.Batch(systems, params, precision="fp64") as b:
        b.set_shape(2, 128)
        b.run(40)
        got = b.spins()
    for k, s in enumerate(systems):
        s2 = s.copy()
        s2.params.temperature = 0.0
        s2.params.H_applied = 0.0
        s2.params.local_applied_field = True
        s2.materials["applied_field"] = np.array([0.0, 0.0, 2.0])
        want = O.OracleSystem(s2).llg_heun(s.spins, 40)
        assert np.abs(got[k] - want).max() < 1e-11  # batch kernels are built with FMA contraction


def test_autotune_picks_a_valid_shape(vgpu_lib, tmp_path):
    from vampire_b200 import batch as B
    systems, params = _small_ensemble(n=40)
    with B.Batch(systems, params) as b:
        before = b.spins()
        got = b.autotune(trial_steps=20, cache=tmp_path / "tune.json")
        after = b.spins()
        assert (got["cluster"] in (1, 2, 4, 8) and got["block"] in (128, 256, 512)) or \
            (got["cluster"], got["block"]) == (0, 0)
        assert got["ms_per_step"] > 0
        assert b.step == 0
        for x, y in zip(before, after):
            assert np.array_equal(x, y)  # the trials restore the state
        again = b.autotune(cache=tmp_path / "tune.json")
        assert again["cluster"] == got["cluster"]


def test_batched_beats_per_system_launches(vgpu_lib):
    """256 nanoparticles: one persistent launch per 100 steps (graph replay)
    against 256 separate plain launch sequences, same steps."""
    from vampire_b200 import batch as B
    from vampire_b200 import vgpu
    systems, params = B.nanoparticle_ensemble(256)
    steps = 200
    with B.Batch(systems, params) as b:
        b.autotune(trial_steps=20)
        b.run(100, record_every=100)  # warm-up, graph build
        t0 = time.perf_counter()
        b.run(steps, record_every=100)
        b.history()
        t_batch = time.perf_counter() - t0
    sims = []
    for k, s in enumerate(systems):
        s.params.temperature = params[k]["temperature"]
        sims.append(vgpu.Simulation(s, noise_seed=k))
    for sim in sims:
        sim.llg_heun(2)
    for sim in sims:
        sim.synchronize()
    t0 = time.perf_counter()
    for sim in sims:
        sim.llg_heun(steps)
    for sim in sims:
        sim.synchronize()
    t_plain = time.perf_counter() - t0
    for sim in sims:
        sim.close()
    print(f"batched {t_batch * 1e3:.1f} ms, per-system {t_plain * 1e3:.1f} ms, ratio {t_plain / t_batch:.1f}")
    assert t_plain / t_batch >= 5.0
