"""Parity of the fused CUDA LLG-Heun path with the reference.

Every test calls the CUDA kernels through the C ABI (vampire_b200.vgpu) and
compares with the reference's own trajectories (tests/golden, produced by the
reference objects) or with the FP64 oracle that those fixtures pin.

Tolerances (max per-spin component deviation):
  FP32 build: 1e-5;  FP64 build: 1e-12 (1e-11 for 200 FCC DMI steps).
"""
import numpy as np
import pytest

from conftest import load_golden, ref_spins

pytestmark = pytest.mark.gpu

TOL32 = 1e-5
TOL64 = 1e-12


@pytest.fixture(scope="module")
def V(vgpu_lib):
    from vampire_b200 import vgpu
    return vgpu


@pytest.mark.parametrize("name", ["sc8_t0", "sc6_open_t300", "fcc4_dmi_t0", "sc20_t0"])
@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_fields_match_oracle(V, name, prec):
    """Total field (exchange incl. DMI tensor + anisotropy + applied) at the
    reference's initial spins."""
    from oracle import oracle as O
    s, d = load_golden(name)
    with V.Simulation(s, precision=prec) as sim:
        got = sim.fields()
    o = O.OracleSystem(s)
    want = o.spin_fields(s.spins) + o.external_fields(None)
    scale = np.abs(want).max()
    tol = 2e-6 if prec == "fp32" else 1e-12
    assert np.abs(got - want).max() <= tol * scale


# FP32 trajectories from a random initial state diverge from the FP64
# reference: the relaxation amplifies differences about 1e5x over 10^4 steps,
# so the FP32 rounding of the initial state alone ends 9e-4 away at step
# 10,000 (tests/test_lyapunov.py, on the FP64 oracle).  The FP32 bound is held
# over the first 100 steps; later the per-spin deviation is bounded and the
# system magnetisation and energy must still agree.  The FP64 build follows
# the reference bit for bit.
FP32_HORIZON = 100


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_sc8_t0_trajectory(V, prec):
    s, d = load_golden("sc8_t0")
    errs = {}
    with V.Simulation(s, precision=prec) as sim:
        done = 0
        for t in (1, 2, 10, 100, 1000, 2000):
            sim.llg_heun(t - done)
            done = t
            errs[t] = float(np.abs(sim.spins() - ref_spins(d, t)).max())
    print(f"sc8 {prec} error vs reference: {errs}")
    for t, e in errs.items():
        if prec == "fp64":
            assert e <= TOL64, (t, e)
        elif t <= FP32_HORIZON:
            assert e <= TOL32, (t, e)
        else:
            assert e < 0.1, (t, e)   # bounded divergence, no blow-up


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
def test_config0_t0_10000_steps(V, prec):
    """Config 0 (SC 20^3 periodic, J=11.2e-21 J, Ku=6.69e-24 J, H=0.1 T,
    alpha=0.1, dt=1e-16 s) from the reference's random initial state, 10,000
    deterministic steps against the reference's own trajectory.  FP64: 1e-12
    per spin throughout.  FP32: 1e-5 per spin to step 100; at step 10,000 the
    per-spin deviation is set by the dynamics' amplification of rounding (no
    FP32 state can hold 1e-5 there, tests/test_lyapunov.py), so the system
    magnetisation and total energy are checked against the reference's
    statistics (5e-3 absolute, 1e-4 relative) and the spins to 0.1."""
    s, d = load_golden("sc20_t0")
    with V.Simulation(s, precision=prec) as sim:
        done = 0
        errs = {}
        for t in (1, 100, 10000):
            sim.llg_heun(t - done)
            done = t
            errs[t] = float(np.abs(sim.spins() - ref_spins(d, t)).max())
        mid = sim.add_mask(*s.masks["system"])
        sim.stats_update(magnetization=True, energy=True)
        m, _, _ = sim.magnetization(mid)
        e, _, _ = sim.energy(mid)
    dm = float(np.abs(m[:4] - d["mag_system_10000"][:4]).max())
    de = float(abs(e[0] - d["energy_system_10000"][0]) / abs(d["energy_system_10000"][0]))
    print(f"config0 {prec} max per-spin error vs reference: {errs}; step 10,000: |dm| {dm:.2e}, dE/E {de:.2e}")
    if prec == "fp64":
        assert max(errs.values()) <= TOL64, errs
        assert dm < 1e-12 and de < 1e-11
    else:
        assert errs[1] <= TOL32 and errs[100] <= TOL32, errs
        assert errs[10000] < 0.1, errs
        assert dm < 5e-3 and de < 1e-4, (dm, de)


def test_fp32_stored_increment_option(V):
    """Storing the predictor increment (instead of recovering it from s0 and
    s') gives the same FP32 step to rounding."""
    s, d = load_golden("sc20_t0")
    with V.Simulation(s) as a, V.Simulation(s) as b:
        V.check(V.lib().vgpu_set_option(b.handle, 1, 1), b.handle)
        a.llg_heun(10)
        b.llg_heun(10)
        assert np.abs(a.spins() - b.spins()).max() < 1e-6


@pytest.mark.parametrize("L", [5, 12])
@pytest.mark.parametrize("sl,nbuf", [(2, 1), (4, 1), (4, 2), (8, 1), (8, 2)])
def test_staged_records_match_plain(V, L, sl, nbuf):
    """The bulk-staged passes (records copied per tile into shared memory)
    give the per-thread-load passes' FP32 results bit for bit: FCC L^3 tensor
    exchange + DMI, two materials, cubic anisotropy, T=300 K Philox noise.
    L=5 (500 spins) leaves a ragged last tile; L=12 (6912 spins) gives many
    tiles per persistent block."""
    from vampire_b200 import system
    s = system.config_fcc_tensor(L=L, seed=7)
    with V.Simulation(s, noise_seed=11) as plain, V.Simulation(s, noise_seed=11) as st:
        plain.set_option(V.OPT_STAGED_RECORDS, 0)
        st.set_option(V.OPT_STAGED_RECORDS, 1)
        st.set_option(V.OPT_STAGE_SLICES, sl)
        st.set_option(V.OPT_STAGE_BUFFERS, nbuf)
        plain.llg_heun(25)
        st.llg_heun(25)
        np.testing.assert_array_equal(st.spins(), plain.spins())


@pytest.mark.parametrize("L", [5, 12])
@pytest.mark.parametrize("warps", [2, 4])
def test_warp_pipelined_passes_match_plain(V, L, warps):
    """The per-warp pipelined passes (VGPU_OPT_STAGE_WARPS: every warp walks
    its own one-slice tiles with two buffers, no block-wide barrier) give the
    plain passes' FP32 results bit for bit, with the dipole field on."""
    from vampire_b200 import system
    s = system.config_fcc_tensor(L=L, seed=7, dipole=True)
    with V.Simulation(s, noise_seed=11) as plain, V.Simulation(s, noise_seed=11) as st:
        plain.set_option(V.OPT_STAGED_RECORDS, 0)
        st.set_option(V.OPT_STAGE_WARPS, warps)
        assert st.record_layout()[0] == V.RECORDS_COMPACT
        for sim in (plain, st):
            sim.dipole_setup(s.cells)
        plain.llg_heun(25)
        st.llg_heun(25)
        np.testing.assert_array_equal(st.spins(), plain.spins())


def test_warp_pipelined_ranges_match_plain(V):
    from vampire_b200 import system
    s = system.config_fcc_tensor(L=8, seed=7)
    with V.Simulation(s, noise_seed=11) as plain, V.Simulation(s, noise_seed=11) as st:
        plain.set_option(V.OPT_STAGED_RECORDS, 0)
        st.set_option(V.OPT_STAGE_WARPS, 4)
        cut = (s.n // 2) // 32 * 32
        for _ in range(5):
            plain.llg_heun(1)
            for which in (V.PASS_PREDICTOR, V.PASS_CORRECTOR):
                st.llg_pass_range(which, 0, cut)
                st.llg_pass_range(which, cut, s.n)
        assert st.step == plain.step == 5
        np.testing.assert_array_equal(st.spins(), plain.spins())


def test_staged_wait_timeout_reports_and_recovers(V):
    """Failure path of the bounded waits: with the test option every tile's
    barrier expects 16 bytes more than its bulk copy delivers, so the wait
    gives up after its limit (1 s), the step reports VGPU_ERR_TIMEOUT, and
    the handle keeps working once the option is off again."""
    from vampire_b200 import system
    s = system.config_fcc_tensor(L=2, seed=7)  # 32 spins: one slice, one tile
    with V.Simulation(s) as sim, V.Simulation(s) as ref:
        sim.set_option(V.OPT_STAGED_RECORDS, 1)
        start = sim.spins()
        sim.set_option(V.OPT_STAGE_WAIT_TEST, 1)
        with pytest.raises(V.VGPUError) as e:
            sim.llg_heun(1)
            sim.synchronize()
        assert e.value.code == V.ERR_TIMEOUT
        sim.set_option(V.OPT_STAGE_WAIT_TEST, 0)
        sim.set_spins(start)
        sim.step = 0
        sim.llg_heun(3)
        ref.set_option(V.OPT_STAGED_RECORDS, 0)
        ref.llg_heun(3)
        np.testing.assert_array_equal(sim.spins(), ref.spins())


def test_stage_option_checks(V):
    from vampire_b200 import system
    s = system.config_fcc_tensor(L=3, seed=7)
    with V.Simulation(s) as sim:
        for opt, bad in ((V.OPT_STAGED_RECORDS, 2), (V.OPT_STAGE_SLICES, 6), (V.OPT_STAGE_BUFFERS, 3),
                         (V.OPT_WINDOW_STAGING, 2)):
            with pytest.raises(V.VGPUError) as e:
                sim.set_option(opt, bad)
            assert e.value.code == V.ERR_ARG
        sim.set_option(V.OPT_STAGED_RECORDS, 1)
        sim.llg_heun(2)
        assert np.isfinite(sim.spins()).all()


def _fcc_variant(kind, L):
    """FCC L^3 tensor exchange + DMI systems for the record-layout tests:
    "scalar" (isotropic diagonal, the benchmark's physics), "diag" (Jyy, Jzz
    scaled per bond: a non-scalar material-pair diagonal), "random_d" (a
    random antisymmetric part per bond: more distinct couplings than the
    dictionary holds), "open" (open z surfaces: ragged rows)."""
    from vampire_b200 import system
    if kind == "open":  # open z surfaces: slices of width 12 and narrower
        return system.config_fcc_tensor(L=L, seed=7, periodic=(True, True, False))
    s = system.config_fcc_tensor(L=L, seed=7)
    if kind == "scalar":
        return s
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


@pytest.mark.parametrize("kind", ["scalar", "diag", "open"])
@pytest.mark.parametrize("L", [5, 12])
@pytest.mark.parametrize("staged,sl", [(0, 4), (1, 2), (1, 4), (1, 8)])
def test_compact_records_match_wide(V, kind, L, staged, sl):
    """Compact records (one word per bond + coupling dictionary) and, in the
    staged passes, window staging (neighbour spins bulk-copied per tile too)
    give the 16-byte records' FP32 results bit for bit, for scalar and
    non-scalar material-pair diagonals and every tile shape."""
    s = _fcc_variant(kind, L)
    with V.Simulation(s, noise_seed=11) as wide, V.Simulation(s, noise_seed=11) as comp, \
            V.Simulation(s, noise_seed=11) as win:
        for sim in (wide, comp, win):
            sim.set_option(V.OPT_STAGED_RECORDS, staged)
            sim.set_option(V.OPT_STAGE_SLICES, sl)
        wide.set_option(V.OPT_COMPACT_RECORDS, 0)
        comp.set_option(V.OPT_WINDOW_STAGING, 0)
        win.set_option(V.OPT_WINDOW_STAGING, 1)
        win.set_option(V.OPT_STAGE_BUFFERS, 1)
        lay, nd = comp.record_layout()
        assert lay == V.RECORDS_COMPACT and 0 < nd <= 512
        assert wide.record_layout()[0] == V.RECORDS_WIDE
        assert win.record_layout()[0] == (V.RECORDS_WINDOW if staged else V.RECORDS_COMPACT)
        for sim in (wide, comp, win):
            sim.llg_heun(25)
        np.testing.assert_array_equal(comp.spins(), wide.spins())
        np.testing.assert_array_equal(win.spins(), wide.spins())


def test_window_staging_shards_and_wait_timeout(V):
    """Window-staged passes on a shard (owned atoms only: the plan is redone
    for the owned count) match the plain passes, and their bounded wait
    reports VGPU_ERR_TIMEOUT and recovers like the record-staged passes."""
    s = _fcc_variant("scalar", 6)
    with V.Simulation(s, noise_seed=4) as win, V.Simulation(s, noise_seed=4) as plain:
        plain.set_option(V.OPT_STAGED_RECORDS, 0)
        win.set_option(V.OPT_WINDOW_STAGING, 1)
        win.set_option(V.OPT_STAGE_BUFFERS, 1)
        for sim in (win, plain):
            sim.set_owned(s.n - 100, 0)
        assert win.record_layout()[0] == V.RECORDS_WINDOW
        win.llg_heun(5)
        plain.llg_heun(5)
        np.testing.assert_array_equal(win.spins(), plain.spins())
        start = win.spins()
        win.set_option(V.OPT_STAGE_WAIT_TEST, 1)
        with pytest.raises(V.VGPUError) as e:
            win.llg_heun(1)
            win.synchronize()
        assert e.value.code == V.ERR_TIMEOUT
        win.set_option(V.OPT_STAGE_WAIT_TEST, 0)
        win.set_spins(start)
        plain.set_spins(start)
        win.step = plain.step = 0
        win.llg_heun(3)
        plain.llg_heun(3)
        np.testing.assert_array_equal(win.spins(), plain.spins())


def test_compact_records_fallback_and_option(V):
    """More distinct couplings than the dictionary holds: the upload keeps the
    16-byte records only, and the passes give the plain passes' results.
    Option values outside -1..1 are refused."""
    s = _fcc_variant("random_d", 5)
    with V.Simulation(s, noise_seed=2) as st, V.Simulation(s, noise_seed=2) as plain:
        assert st.record_layout() == (V.RECORDS_WIDE, 0)
        with pytest.raises(V.VGPUError) as e:
            st.set_option(V.OPT_COMPACT_RECORDS, 2)
        assert e.value.code == V.ERR_ARG
        st.set_option(V.OPT_STAGED_RECORDS, 1)
        plain.set_option(V.OPT_STAGED_RECORDS, 0)
        st.llg_heun(10)
        plain.llg_heun(10)
        np.testing.assert_array_equal(st.spins(), plain.spins())
    from vampire_b200 import system
    with V.Simulation(system.config_fcc_tensor(L=3, seed=1), precision="fp64") as sim:
        assert sim.record_layout()[0] == V.RECORDS_NONE


@pytest.mark.parametrize("name,steps", [("sc10_t300", 2), ("sc6_open_t300", 3), ("fcc4_dmi_t300", 2)])
@pytest.mark.parametrize("prec,tol", [("fp64", TOL64), ("fp32", TOL32)])
def test_replayed_noise(V, name, steps, prec, tol):
    """T>0 with the reference's own Gaussian stream (noise-replay mode): each
    stochastic Heun step matches the reference."""
    s, d = load_golden(name)
    with V.Simulation(s, precision=prec) as sim:
        for t in range(1, steps + 1):
            sim.set_noise_replay(d[f"xi_{t}"])
            sim.llg_heun(1)
            if f"sx_{t}" in d:
                err = np.abs(sim.spins() - ref_spins(d, t)).max()
                assert err <= tol, (t, err)


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-11), ("fp32", TOL32)])
def test_fcc_dmi_200_steps(V, prec, tol):
    s, d = load_golden("fcc4_dmi_t0")
    with V.Simulation(s, precision=prec) as sim:
        sim.llg_heun(200)
        err = np.abs(sim.spins() - ref_spins(d, 200)).max()
    assert err <= tol, err


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-6), ("fp32", 2e-5)])
def test_single_spin_known_answer(V, prec, tol):
    """The reference's applied-field known-answer test on the GPU: analytic
    precession/relaxation of one spin in 10 T (tests/physical/AppliedField)."""
    s, d = load_golden("single_spin_applied")
    lam, H, g, dt = 1.0, 10.0, 1.76e11, 1e-16
    with V.Simulation(s, precision=prec) as sim:
        done = 0
        for t in (50, 1000, 5000, 10000):
            sim.llg_heun(t - done)
            done = t
            got = sim.spins()[:, 0]
            arg = g * H * t * dt / (1 + lam * lam)
            exact = np.array([np.cos(arg) / np.cosh(lam * arg), np.sin(arg) / np.cosh(lam * arg),
                              np.tanh(lam * arg)])
            assert np.abs(got - exact).max() < tol


@pytest.mark.parametrize("prec", ["fp32", "fp64"])
def test_philox_noise_matches_restatement(V, prec):
    """The in-register Philox Gaussians equal an independent NumPy restatement."""
    from oracle import philox as P
    s, _ = load_golden("sc10_t300")
    with V.Simulation(s, precision=prec, noise_seed=0x1234_5678_9ABC) as sim:
        for step in (0, 1, 2**33 + 5):
            got = sim.thermal_noise(step)
            want = P.thermal_gaussians(s.n, step, seed=0x1234_5678_9ABC, fp64=(prec == "fp64"))
            assert np.abs(got - want).max() < (2e-5 if prec == "fp32" else 1e-12)


def test_fp32_gaussians_error_bound(V):
    """The FP32 Box-Muller on the fast hardware approximations (base-2 log,
    series near u = 1, approximate square root and sine/cosine) stays within
    1e-5 of the exact transform of the same Philox uniforms over 900,000
    Gaussians, radii near zero (u within 1/64 of 1) included, with the moments
    of a unit Gaussian."""
    from oracle import philox as P
    s, _ = load_golden("sc10_t300")
    err, got_all = 0.0, []
    with V.Simulation(s, precision="fp32", noise_seed=0xC0FFEE) as sim:
        for step in range(300):
            got = sim.thermal_noise(step)
            want = P.thermal_gaussians(s.n, step, seed=0xC0FFEE)
            err = max(err, float(np.abs(got - want).max()))
            got_all.append(got)
    g = np.concatenate(got_all)
    assert err < 1e-5, err
    assert abs(g.mean()) < 5e-3 and abs(g.var() - 1.0) < 1e-2
    assert abs(np.mean(g ** 4) - 3.0) < 5e-2
    assert np.isfinite(g).all() and np.abs(g).min() < 1e-3


@pytest.mark.parametrize("name", ["sc10_t300", "fcc4_dmi_t300"])
def test_philox_step_matches_oracle(V, name):
    """One T>0 step with the built-in Philox noise equals the oracle's step
    driven by the same Gaussians (predictor and corrector regenerate them)."""
    from oracle import oracle as O
    s, _ = load_golden(name)
    with V.Simulation(s, precision="fp64", noise_seed=99) as sim:
        sim.step = 17
        xi = sim.thermal_noise(17)
        sim.llg_heun(1)
        got = sim.spins()
        assert sim.step == 18
    want = O.OracleSystem(s).llg_heun(s.spins, 1, xi=xi)
    assert np.abs(got - want).max() < 1e-12


def test_counter_based_resume(V):
    """Resuming from (spins, step) reproduces the uninterrupted run bit for bit."""
    s, _ = load_golden("sc10_t300")
    with V.Simulation(s, noise_seed=5) as a:
        a.llg_heun(20)
        ref = a.spins()
    with V.Simulation(s, noise_seed=5) as b:
        b.llg_heun(8)
        mid, st = b.spins(), b.step
    with V.Simulation(s, noise_seed=5) as c:
        c.set_spins(mid)
        c.step = st
        c.llg_heun(12)
        # spins pass through FP64 on the host; FP32 round trip is exact
        assert np.array_equal(c.spins(), ref)


def test_thermal_equilibrium_single_spin_boltzmann(V):
    """Philox thermal noise gives the Boltzmann distribution: many independent
    uniaxial macrospins (no exchange) at T sample
    P(theta) ~ sin(theta) exp(Ku sin^2(theta)/kT)... checked through <s_z^2>
    against the numerically integrated expectation (the concept of the
    reference's tests/physical/Thermal, with kB = 1.3806503e-23)."""
    from vampire_b200 import system as S
    n = 20000
    m = S.Material(alpha=1.0, mu_s_muB=1.72, Ku=1e-23)
    T = 50.0
    # dt = 1e-14 s: gamma H_K dt ~ 0.02 rad, relaxation in ~1e3 steps
    p = S.SimParams(dt_SI=1e-14, temperature=T, H_applied=0.0)
    sys_ = S.build("sc", n, 1, 1, 10.0, [m], [[0.0]], p, periodic=(False, False, False),
                   spins=np.tile(np.array([[0.0], [0.0], [1.0]]), (1, n)))
    with V.Simulation(sys_, noise_seed=11) as sim:
        sim.llg_heun(10000)
        sz2 = []
        for _ in range(20):
            sim.llg_heun(1000)
            sz2.append(np.mean(sim.spins()[2] ** 2))
    # expectation of cos^2 over P(theta) ~ sin exp(K cos^2 / kT) (up to a constant)
    K = 1e-23 / (S.KB * T)
    c = np.linspace(-1, 1, 200001)
    w = np.exp(K * c * c)
    want = np.trapezoid(c * c * w, c) / np.trapezoid(w, c)
    got = float(np.mean(sz2))
    assert abs(got - want) < 0.01, (got, want)


def test_status_flags_nonfinite(V):
    """A spin state that cannot be normalised is reported, not hidden."""
    s, _ = load_golden("sc8_t0")
    with V.Simulation(s) as sim:
        bad = s.spins.copy()
        bad[:, 3] = 0.0  # zero-length spin -> 0/0 in the corrector
        sim.set_spins(bad)
        sim.llg_heun(1)
        with pytest.raises(V.VGPUError) as e:
            sim.spins()
        assert e.value.code == V.ERR_NAN


def test_profile_sampling(V):
    """VGPU_OPT_PROFILE_EVERY = k times the launches of the steps whose
    counter is a multiple of k; the kernel-launch count still covers every
    launch, and a stride below 1 is refused."""
    from vampire_b200 import system as S
    s = S.config_fcc_tensor(L=4, seed=5)
    with V.Simulation(s) as sim:
        with pytest.raises(V.VGPUError) as e:
            sim.set_option(V.OPT_PROFILE_EVERY, 0)
        assert e.value.code == V.ERR_ARG
        sim.set_option(V.OPT_PROFILE_EVERY, 5)
        sim.profile(True)
        sim.llg_heun(20)
        prof = sim.profile_read()
        sim.profile(False)
    assert prof["predictor"]["count"] == 4 and prof["corrector"]["count"] == 4
    assert prof["predictor"]["ms"] > 0.0
    assert prof["kernel_launches"] >= 40


@pytest.mark.parametrize("prec,tol", [("fp64", 1e-12), ("fp32", TOL32)])
def test_llg_midpoint_matches_reference(V, prec, tol):
    """sim::LLG_Midpoint (src/simulate/LLGMidpoint.cpp) on the device: 100
    deterministic steps of the reference's own SC 8^3 run, and two
    stochastic steps with its Gaussian stream."""
    s, d = load_golden("sc8_midpoint_t0")
    with V.Simulation(s, precision=prec) as sim:
        sim.llg_midpoint(1)
        e1 = np.abs(sim.spins() - ref_spins(d, 1)).max()
        sim.llg_midpoint(99)
        e100 = np.abs(sim.spins() - ref_spins(d, 100)).max()
    print(f"midpoint {prec}: step 1 {e1:.2e}, step 100 {e100:.2e}")
    assert e1 <= tol and e100 <= tol
    s, d = load_golden("sc8_midpoint_t300")
    with V.Simulation(s, precision=prec) as sim:
        for t in (1, 2):
            sim.set_noise_replay(d[f"xi_{t}"])
            sim.llg_midpoint(1)
            assert np.abs(sim.spins() - ref_spins(d, t)).max() <= tol, t
