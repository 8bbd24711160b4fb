"""Pin the CPU oracle against the reference's own known-answer tests, re-expressed in NumPy.

Each test cites the reference test it restates. These run on the CPU only; they make the oracle
trustworthy before any GPU result is compared with it.
"""
import math

import numpy as np
import pytest

from oracle import gbght_oracle as O
from gbght import seed as S

TWO_PI = 2 * math.pi


def _grid(N, L=TWO_PI):
    x = np.arange(N) * (L / N)
    z3, y3, x3 = np.meshgrid(x, x, x, indexing="ij")
    return x3, y3, z3


def diffnorm(a, b):
    return math.sqrt(float(np.sum(np.abs(a - b) ** 2)))


# --- test/observables_analytic.jl:43-88 -----------------------------------------------------------

def test_observables_closed_forms():
    N, A, B, C, D, nu, kap = 16, 0.7, -0.4, 1.1, 0.9, 0.03, 0.05
    dom = O.Domain(N)
    x, y, z = _grid(N)
    u = np.stack([A * np.sin(y), B * np.sin(z), C * np.sin(x)])
    phi = D * np.sin(x)
    uh, ph = dom.to_spectral(u), dom.to_spectral(phi)
    sq = A * A + B * B + C * C
    assert O.kinetic_energy(dom, uh) == pytest.approx(sq / 4, rel=1e-13)
    assert O.dissipation(dom, uh, nu) == pytest.approx(nu * sq / 2, rel=1e-13)
    assert O.scalar_variance(dom, ph) == pytest.approx(D * D / 2, rel=1e-13)
    assert O.scalar_dissipation(dom, ph, kap) == pytest.approx(kap * D * D, rel=1e-13)
    E = O.energy_spectrum(dom, uh)
    assert E[1] == pytest.approx(sq / 4, rel=1e-13)
    assert E.sum() == pytest.approx(E[1], rel=1e-13)
    _, _, _, speed = O.deposit(dom, O.State(uh, ph))
    assert speed == pytest.approx(math.sqrt(sq), rel=1e-13)


def test_mask_is_zero_one_and_cutoff():
    # test/dealiasing.jl:14-20; test/observables_analytic.jl:96-103
    for N in (12, 16, 48):
        dom = O.Domain(N)
        assert set(np.unique(dom.mask)) <= {0.0, 1.0}
        assert dom.cutoff == pytest.approx((2 / 3) * (N / 2), rel=1e-14)
    # N = 48: the cutoff rounds to exactly 16 and |κ|² = 256 lies on the closed ball's edge
    dom = O.Domain(48)
    assert dom.cutoff == 16.0
    assert dom.mask[0, 0, 16] == 1.0 and dom.mask[0, 0, 17] == 0.0


def test_parseval_spectrum_sums_to_energy():
    # test/validation.jl:13-36
    dom = O.Domain(32)
    uh = S.seed_velocity(32, 0.7, seed=3)
    E = O.energy_spectrum(dom, uh)
    assert E.sum() * dom.k0 == pytest.approx(O.kinetic_energy(dom, uh), rel=1e-13)
    ph = S.seed_scalar(32, 0.4, seed=4)
    assert O.scalar_spectrum(dom, ph).sum() == pytest.approx(O.scalar_variance(dom, ph), rel=1e-13)


# --- test/scalar.jl ----------------------------------------------------------------------------

@pytest.mark.parametrize("scheme", ["rk3", "rk4"])
def test_exact_diffusion_zero_velocity(scheme):
    # test/scalar.jl:42-60: with u = 0 the scalar decays by the integrating factor alone
    N, nu, Sc = 16, 0.1, 0.7
    dom = O.Domain(N)
    cond = O.Conditions(viscosity=nu, schmidt=Sc)
    ph0 = S.seed_scalar(N, 1.0, seed=3)
    st = O.State(np.zeros((3,) + dom.shape_spectral, complex), ph0.copy())
    dt, n = 0.02, 25
    for _ in range(n):
        st = O.step(dom, cond, st, dt, scheme)
    expected = ph0 * np.exp(-(nu / Sc) * dom.k2 * dt * n)
    assert diffnorm(st.phih, expected) / math.sqrt(float(np.sum(np.abs(expected) ** 2))) < 1e-10


def test_scalar_rhs_mean_exactly_zero():
    # test/scalar.jl:95-118
    N = 16
    dom = O.Domain(N)
    uh = S.seed_velocity(N, 0.5, seed=7)
    ph = S.seed_scalar(N, 1.0, seed=8)
    ph[0, 0, 0] = 3.0
    u, phi = dom.to_physical(uh), dom.to_physical(ph)
    nh = O.scalar_rhs(dom, O.Conditions(viscosity=0.05), uh, u, phi)
    assert nh[0, 0, 0] == 0


def test_scalar_mean_conserved():
    # test/scalar.jl:80-93 (forcing aside: the scalar mean mode is untouched by the advection)
    N = 16
    dom = O.Domain(N)
    cond = O.Conditions(viscosity=0.1)
    ph = S.seed_scalar(N, 1.0, seed=6)
    ph[0, 0, 0] = 3.0
    st = O.State(S.seed_velocity(N, 0.5, seed=5), ph)
    for _ in range(30):
        st = O.step(dom, cond, st, 0.02, "rk4")
    assert st.phih[0, 0, 0] == pytest.approx(3.0, rel=1e-13)


# --- test/integrators.jl -----------------------------------------------------------------------

def _integrate(dom, cond, uh0, ph0, dt, n, scheme):
    st = O.State(uh0.copy(), None if ph0 is None else ph0.copy())
    for _ in range(n):
        st = O.step(dom, cond, st, dt, scheme)
    return st


def test_rk3_self_convergence_ratio():
    # test/integrators.jl:49-78 and test/scalar.jl:63-78
    N = 16
    dom = O.Domain(N)
    cond = O.Conditions(viscosity=0.1)
    uh0, ph0 = S.seed_velocity(N, 0.5, seed=1), S.seed_scalar(N, 1.0, seed=2)
    T, n = 0.4, 8
    p1 = _integrate(dom, cond, uh0, ph0, T / n, n, "rk3")
    p2 = _integrate(dom, cond, uh0, ph0, T / (2 * n), 2 * n, "rk3")
    p4 = _integrate(dom, cond, uh0, ph0, T / (4 * n), 4 * n, "rk3")
    assert 5.0 < diffnorm(p1.uh, p2.uh) / diffnorm(p2.uh, p4.uh) < 12.0
    assert 5.0 < diffnorm(p1.phih, p2.phih) / diffnorm(p2.phih, p4.phih) < 12.0


def test_rk4_self_convergence_ratio():
    # test/integrators.jl:165-188
    N = 32
    dom = O.Domain(N)
    cond = O.Conditions(viscosity=0.02)
    uh0 = S.seed_velocity(N, 0.5, seed=7)
    T, n = 0.5, 8
    u1 = _integrate(dom, cond, uh0, None, T / n, n, "rk4")
    u2 = _integrate(dom, cond, uh0, None, T / (2 * n), 2 * n, "rk4")
    u4 = _integrate(dom, cond, uh0, None, T / (4 * n), 4 * n, "rk4")
    assert 10.0 < diffnorm(u1.uh, u2.uh) / diffnorm(u2.uh, u4.uh) < 26.0


def test_temporal_convergence_orders_of_the_four_schemes():
    # test/integrators.jl:47-80: RK3 and SSPRK3 third order, Heun second, RK3 faster than Heun;
    # the two RK3 tableaux agree as Δt → 0 but differ at one Δt
    N = 16
    dom = O.Domain(N)
    cond = O.Conditions(viscosity=0.1, scalar=False)
    uh0 = S.seed_velocity(N, 0.5, seed=7)
    T, n = 0.5, 8
    runs = {sch: [_integrate(dom, cond, uh0, None, T / (k * n), k * n, sch).uh for k in (1, 2, 4)]
            for sch in ("rk3", "ssprk3", "heun")}
    ratio = {sch: diffnorm(r[0], r[1]) / diffnorm(r[1], r[2]) for sch, r in runs.items()}
    assert 5.0 < ratio["rk3"] < 12.0
    assert 5.0 < ratio["ssprk3"] < 12.0
    assert 3.0 < ratio["heun"] < 6.0
    assert ratio["rk3"] > ratio["heun"]
    assert diffnorm(runs["rk3"][2], runs["ssprk3"][2]) < diffnorm(runs["rk3"][0], runs["ssprk3"][0])
    assert diffnorm(runs["rk3"][0], runs["ssprk3"][0]) > 0


@pytest.mark.parametrize("scheme", ["heun", "ssprk3"])
def test_exact_diffusion_and_linear_growth_heun_ssprk3(scheme):
    # test/scalar.jl:42-60 for the other two schemes: with u = 0 the scalar moves by the
    # integrating factor alone (the SSPRK3 stages transport back and forth and recombine to E(Δt));
    # and a shear mode under Linear grows at exactly A − ν|κ|²
    N, nu, Sc = 16, 0.1, 0.7
    dom = O.Domain(N)
    ph0 = S.seed_scalar(N, 1.0, seed=3)
    st = O.State(np.zeros((3,) + dom.shape_spectral, complex), ph0.copy())
    dt, n = 0.02, 25
    for _ in range(n):
        st = O.step(dom, O.Conditions(viscosity=nu, schmidt=Sc), st, dt, scheme)
    expected = ph0 * np.exp(-(nu / Sc) * dom.k2 * dt * n)
    assert diffnorm(st.phih, expected) / math.sqrt(float(np.sum(np.abs(expected) ** 2))) < 1e-12
    x3, y3, z3 = _grid(N)
    uh0 = dom.to_spectral(np.stack([np.sin(y3), np.zeros_like(y3), np.zeros_like(y3)]))
    cond = O.Conditions(viscosity=0.05, scalar=False, velocity_forcing=O.Linear(0.7))
    st = _integrate(dom, cond, uh0, None, dt, n, scheme)
    expected = uh0 * math.exp((0.7 - 0.05) * dt * n)
    assert diffnorm(st.uh, expected) / math.sqrt(float(np.sum(np.abs(expected) ** 2))) < 1e-12


def test_recommended_cfl():
    # test/integrators.jl:114-118
    assert O.recommended_cfl("rk3") > O.recommended_cfl("heun")
    assert 0 < O.recommended_cfl("heun") < 1 and 0 < O.recommended_cfl("rk3") < 1
    assert O.recommended_cfl("ssprk3") == O.recommended_cfl("rk3")


@pytest.mark.parametrize("forcing", [O.ConstantPower(0.2), O.Linear(0.5), O.VarianceController(1.5, turnover_time=1.0)],
                         ids=["constant_power", "linear", "variance_controller"])
@pytest.mark.parametrize("scheme,floor", [("rk3", 2.5), ("rk4", 3.5), ("ssprk3", 2.5), ("heun", 1.7)])
def test_order_kept_under_forcing(scheme, floor, forcing):
    # test/integrators.jl:132-162: a state-dependent forcing through the per-stage source and a
    # steady rate through the integrating factor keep the scheme's order (measured ≥ 2.5 for RK3;
    # RK4 held to ≥ 3.5 here)
    N = 16
    dom = O.Domain(N)
    cond = O.Conditions(viscosity=0.05, velocity_forcing=forcing)
    uh0 = S.seed_velocity(N, 0.5, seed=7)
    T = 0.2
    ref = _integrate(dom, cond, uh0, None, T / 1024, 1024, scheme).uh
    e32 = np.max(np.abs(_integrate(dom, cond, uh0, None, T / 32, 32, scheme).uh - ref))
    e64 = np.max(np.abs(_integrate(dom, cond, uh0, None, T / 64, 64, scheme).uh - ref))
    assert math.log2(e32 / e64) >= floor


# --- test/forcing.jl ---------------------------------------------------------------------------

def test_constant_power_injects_its_rate():
    # test/forcing.jl:92-104: ⟨û, f⟩ = ε at rtol 1e-8
    N = 24
    dom = O.Domain(N)
    uh = S.seed_velocity(N, 0.5, seed=11)
    f = O.ConstantPower(0.3)
    A, band = O.constant_power_amplitude(dom, f, uh, np.finfo(float).eps)
    assert dom.inner(uh, A * band * uh) == pytest.approx(0.3, rel=1e-8)


def test_constant_power_bounded_and_solenoidal():
    # test/forcing.jl:115-122
    N = 24
    dom = O.Domain(N)
    cond = O.Conditions(viscosity=0.05, velocity_forcing=O.ConstantPower(0.5))
    st = _integrate(dom, cond, S.seed_velocity(N, 0.5, seed=11), None, 0.01, 100, "rk3")
    k = O.kinetic_energy(dom, st.uh)
    assert math.isfinite(k) and k > 0
    div = (dom.kx * st.uh[0] + dom.ky * st.uh[1]) + dom.kz * st.uh[2]
    assert math.sqrt(float(np.sum(np.abs(div) ** 2))) / math.sqrt(float(np.sum(np.abs(st.uh) ** 2))) < 1e-8


def test_empty_band_clamps_amplitude():
    # src/Forcing.jl:110-111,1091-1101: a band holding nothing gets A = 0, never an unbounded kick
    N = 16
    dom = O.Domain(N)
    uh = S.seed_velocity(N, 0.5, seed=2)
    band = O.band_indicator(dom, O.ConstantPower(0.1))
    uh = uh * (1 - band)
    A, _ = O.constant_power_amplitude(dom, O.ConstantPower(0.1), uh, np.finfo(float).eps)
    assert A == 0.0


def test_linear_rate_amplitude():
    # test/forcing.jl:80-90: A on the band, zero outside, on exactly the band's modes
    dom = O.Domain(24)
    f = O.Linear(0.7)
    rate = O.steady_rate(dom, f)
    assert rate.max() == 0.7 and rate.min() == 0.0
    assert np.array_equal(rate != 0, O.band_indicator(dom, f) != 0)
    assert not np.any(O.steady_rate(dom, O.ConstantPower(0.1)))   # only Linear is steady


@pytest.mark.parametrize("N", [16, 24])
def test_linear_unbounded_band_is_every_mode_but_the_mean(N):
    # test/forcing.jl:457-461: highest_shell = Inf forces every stored mode except κ = 0
    rate = O.steady_rate(O.Domain(N), O.Linear(0.1, highest_shell=math.inf))
    assert np.count_nonzero(rate == 0) == 1 and rate[0, 0, 0] == 0
    assert np.all((rate == 0) | (rate == 0.1))


def test_linear_injects_energy_stays_solenoidal():
    # test/forcing.jl:106-113
    N = 24
    dom = O.Domain(N)
    uh0 = S.seed_velocity(N, 0.5, seed=11)
    unforced = _integrate(dom, O.Conditions(viscosity=0.05), uh0, None, 0.01, 60, "rk3")
    forced = _integrate(dom, O.Conditions(viscosity=0.05, velocity_forcing=O.Linear(1.0)), uh0, None, 0.01, 60, "rk3")
    assert O.kinetic_energy(dom, forced.uh) > O.kinetic_energy(dom, unforced.uh)
    div = (dom.kx * forced.uh[0] + dom.ky * forced.uh[1]) + dom.kz * forced.uh[2]
    assert math.sqrt(float(np.sum(np.abs(div) ** 2))) / math.sqrt(float(np.sum(np.abs(forced.uh) ** 2))) < 1e-8


@pytest.mark.parametrize("scheme", ["rk3", "rk4"])
def test_linear_shear_mode_grows_exactly(scheme):
    # A single shear mode u = (sin y, 0, 0) has u×ω = (0, ½ sin 2y, 0), a gradient that the Leray
    # projection removes: the mode evolves by the integrating factor alone, at net rate A − ν|κ|².
    N, nu, A = 16, 0.05, 0.7
    dom = O.Domain(N)
    x3, y3, z3 = _grid(N)
    u = np.stack([np.sin(y3), np.zeros_like(y3), np.zeros_like(y3)])
    uh0 = dom.to_spectral(u)
    cond = O.Conditions(viscosity=nu, scalar=False, velocity_forcing=O.Linear(A))
    dt, n = 0.02, 25
    st = _integrate(dom, cond, uh0, None, dt, n, scheme)
    expected = uh0 * math.exp((A - nu) * dt * n)
    assert diffnorm(st.uh, expected) / math.sqrt(float(np.sum(np.abs(expected) ** 2))) < 1e-12


@pytest.mark.parametrize("scheme", ["rk3", "rk4"])
def test_scalar_linear_grows_exactly_with_zero_velocity(scheme):
    # test/forcing.jl:124-139 (variance builds), held here to the closed form: with u = 0 the
    # scalar moves by the integrating factor alone, φ̂(T) = exp((A·band − ϰ|κ|²)T) φ̂(0). The seed
    # keeps shells 1–2 and a weaker copy of the rest, standing in for the test's peak at shell 2.
    N, nu, Sc, A = 24, 0.05, 1.0, 1.0
    dom = O.Domain(N)
    f = O.Linear(A)
    band = O.band_indicator(dom, f)
    ph0 = S.seed_scalar(N, 0.1, seed=9) * (band + 0.1 * (1 - band))
    cond = O.Conditions(viscosity=nu, schmidt=Sc, scalar_forcing=f)
    st = O.State(np.zeros((3,) + dom.shape_spectral, complex), ph0.copy())
    dt, n = 0.01, 40
    for _ in range(n):
        st = O.step(dom, cond, st, dt, scheme)
    assert O.scalar_variance(dom, st.phih) > O.scalar_variance(dom, ph0)
    expected = ph0 * np.exp((A * band - (nu / Sc) * dom.k2) * dt * n)
    assert diffnorm(st.phih, expected) / math.sqrt(float(np.sum(np.abs(expected) ** 2))) < 1e-12


def test_scalar_constant_power_injects_its_rate():
    # the scalar's ConstantPower (target factor 1): d⟨φ²⟩/dt = 2⟨φ, f⟩ = ε_φ
    N = 24
    dom = O.Domain(N)
    ph = S.seed_scalar(N, 0.4, seed=12)
    src = O.stage_source(dom, O.ConstantPower(0.3), ph, np.finfo(float).eps, 0.05)
    assert 2 * dom.inner(ph, src) == pytest.approx(0.3, rel=1e-12)


def test_variance_controller_holds_the_whole_field_normalising_by_the_band():
    # test/forcing.jl:322-349: A = (ε − G(k − k∞)/tℓ)/(2 k_band), read back off the applied source
    N, nu = 24, 0.05
    dom = O.Domain(N)
    uh = S.seed_velocity(N, 0.5, seed=11)
    f = O.VarianceController(0.5, turnover_time=0.8, gain=1.0)
    src = O.stage_source(dom, f, uh, np.finfo(float).eps, nu)
    band = O.band_indicator(dom, f)
    k_whole = 0.5 * dom.inner(uh, uh)
    k_band = 0.5 * dom.inner(uh, uh, band)
    eps = nu * dom.inner(uh, uh, dom.k2)
    expected = (eps - f.gain * (k_whole - f.target) / f.turnover_time) / (2 * k_band)
    probe = band * uh
    applied = dom.inner(src, probe) / dom.inner(probe, probe)
    assert applied == pytest.approx(expected, rel=1e-10)
    wrong = (eps - f.gain * (k_band - f.target) / f.turnover_time) / (2 * k_band)
    assert not applied == pytest.approx(wrong, rel=1e-3)


def test_variance_controller_scalar_dissipation_matches():
    # test/forcing.jl:486-518: at gain 0 the scalar controller's A is ConstantPower's at ε = ε_φ,
    # and halving ϰ halves it
    N = 16
    dom = O.Domain(N)
    ph = S.seed_scalar(N, 0.4, seed=31)
    kappa = 0.05 / 0.7
    eps_phi = O.scalar_dissipation(dom, ph, kappa)
    eT = np.finfo(float).eps
    A_ctrl, _ = O.constant_power_amplitude(dom, O.VarianceController(1.0, turnover_time=1.0, gain=0.0), ph, eT, kappa)
    A_cp, _ = O.constant_power_amplitude(dom, O.ConstantPower(eps_phi), ph, eT, kappa)
    assert A_ctrl == pytest.approx(A_cp, rel=1e-12)
    A_half, _ = O.constant_power_amplitude(dom, O.VarianceController(1.0, turnover_time=1.0, gain=0.0), ph, eT,
                                           kappa / 2)
    assert A_half == pytest.approx(A_cp / 2, rel=1e-12)


def test_variance_controller_gain_zero_is_the_marginal_law():
    # test/forcing.jl:388-405: k conserved at its initial value, never restored to the target
    N = 24
    dom = O.Domain(N)
    cond = O.Conditions(viscosity=0.05, scalar=False, velocity_forcing=O.VarianceController(1.5, 1.0, gain=0.0))
    run = O.Run(dom, cond, O.State(S.seed_velocity(N, 0.5, seed=3), None), scheme="rk4", cfl=0.5)
    k0 = O.kinetic_energy(dom, run.state.uh)
    for _ in range(150):
        run.advance(None)
    k = O.kinetic_energy(dom, run.state.uh)
    assert k == pytest.approx(k0, rel=0.05)
    assert abs(k - 1.5) > 0.8


def test_variance_controller_relaxes_to_its_target():
    # dk/dt = −G(k − k∞)/tℓ, exactly for the continuous law: after t = tℓ/G the gap has shrunk by e
    N = 16
    dom = O.Domain(N)
    f = O.VarianceController(0.8, turnover_time=0.5, gain=1.0)
    cond = O.Conditions(viscosity=0.05, scalar=False, velocity_forcing=f)
    uh0 = S.seed_velocity(N, 0.5, seed=4)
    dt, n = 0.005, 100
    st = _integrate(dom, cond, uh0, None, dt, n, "rk4")
    k = O.kinetic_energy(dom, st.uh)
    expected = 0.8 + (0.5 - 0.8) * math.exp(-f.gain * dt * n / f.turnover_time)
    assert k == pytest.approx(expected, rel=1e-6)


@pytest.mark.parametrize("N", [16, 24])
@pytest.mark.parametrize("over", ["band", "total"])
def test_variance_rescaling_unbounded_band_rescales_the_whole_field(N, over):
    # test/forcing.jl:440-452: with highest_shell = Inf both modes hold k = target exactly, by one
    # uniform factor
    dom = O.Domain(N)
    uh = S.seed_velocity(N, 0.7, seed=N)
    expected = uh * math.sqrt(1.3 / O.kinetic_energy(dom, uh))
    v = O.project_forcing(dom, O.VarianceRescaling(1.3, over, highest_shell=math.inf), uh, np.finfo(float).eps)
    assert O.kinetic_energy(dom, v) == pytest.approx(1.3, rel=1e-12)
    assert np.max(np.abs(v - expected)) <= 1e-12 * np.max(np.abs(expected))


def test_variance_rescaling_band_and_total():
    # src/Forcing.jl:575-596: :band holds the band's value, :total the whole field's; a :total
    # target below what lies outside the band zeroes the band; an empty band is left alone
    N = 16
    dom = O.Domain(N)
    eT = np.finfo(float).eps
    uh = S.seed_velocity(N, 0.5, seed=5)
    f = O.VarianceRescaling(0.2, "band")
    band = O.band_indicator(dom, f)
    v = O.project_forcing(dom, f, uh, eT)
    assert O.kinetic_energy(dom, band * v) == pytest.approx(0.2, rel=1e-12)
    assert np.array_equal((1 - band) * v, (1 - band) * uh)
    v = O.project_forcing(dom, O.VarianceRescaling(0.7, "total"), uh, eT)
    assert O.kinetic_energy(dom, v) == pytest.approx(0.7, rel=1e-12)
    outside = O.kinetic_energy(dom, (1 - band) * uh)
    v = O.project_forcing(dom, O.VarianceRescaling(0.5 * outside, "total"), uh, eT)
    assert np.max(np.abs(band * v)) == 0.0
    empty = (1 - band) * uh
    assert np.array_equal(O.project_forcing(dom, O.VarianceRescaling(0.7, "total"), empty, eT), empty)
    ph = S.seed_scalar(N, 0.4, seed=6)   # the scalar's variance, target factor 1
    w = O.project_forcing(dom, O.VarianceRescaling(0.9, "total"), ph, eT)
    assert O.scalar_variance(dom, w) == pytest.approx(0.9, rel=1e-12)


def test_variance_rescaling_costs_the_order():
    # test/integrators.jl:159-161: the post-step projection is first order, by construction
    N = 16
    dom = O.Domain(N)
    cond = O.Conditions(viscosity=0.05, velocity_forcing=O.VarianceRescaling(1.5, "total"))
    uh0 = S.seed_velocity(N, 0.5, seed=7)
    T = 0.2
    ref = _integrate(dom, cond, uh0, None, T / 1024, 1024, "rk3").uh
    e32 = np.max(np.abs(_integrate(dom, cond, uh0, None, T / 32, 32, "rk3").uh - ref))
    e64 = np.max(np.abs(_integrate(dom, cond, uh0, None, T / 64, 64, "rk3").uh - ref))
    assert math.log2(e32 / e64) < 1.5


def test_scalar_forcing_needs_the_scalar():
    # src/Generator.jl:312-316
    with pytest.raises(ValueError, match="no scalar"):
        O.Conditions(viscosity=0.1, scalar=False, scalar_forcing=O.Linear(1.0))


# --- test/regressions/r6-inclusive-ball-exact.jl -------------------------------------------------

def test_closed_ball_exact_against_zero_padded_product():
    Np = 12
    d1, d2 = O.Domain(Np), O.Domain(2 * Np)
    uh = S.seed_velocity(Np, 0.5, seed=3)
    rng = np.random.default_rng(11)
    populated = 0
    for i3 in range(Np):
        for i2 in range(Np):
            for i1 in range(Np // 2 + 1):
                k = np.array([i1, O._axis_integers(Np)[i2], O._axis_integers(Np)[i3]], float)
                if int(k @ k) != 16:
                    continue
                c = rng.standard_normal(3) + 1j * rng.standard_normal(3)
                c = c - k * (k @ c) / 16
                uh[:, i3, i2, i1] = 0.4 * c
                populated += 1
    assert populated == 5

    def mapidx(i):
        return i if i <= Np // 2 else i + Np

    def term(dom, vh):
        u = dom.to_physical(vh)
        w = dom.to_physical(O.curl(dom, vh))
        ln = np.stack([u[1] * w[2] - u[2] * w[1], u[2] * w[0] - u[0] * w[2], u[0] * w[1] - u[1] * w[0]])
        return O.leray(dom, dom.to_spectral(ln))

    big = np.zeros((3,) + d2.shape_spectral, complex)
    for i3 in range(Np):
        for i2 in range(Np):
            big[:, mapidx(i3), mapidx(i2), : Np // 2 + 1] = 8 * uh[:, i3, i2, :]
    raw = term(d1, uh)
    full = term(d2, big)
    oracle = np.zeros_like(raw)
    for i3 in range(Np):
        for i2 in range(Np):
            oracle[:, i3, i2, :] = full[:, mapidx(i3), mapidx(i2), : Np // 2 + 1] / 8
    kmag = np.sqrt(d1.k2)
    ref = np.max(np.abs(oracle))
    inside = kmag < 4 - 1e-9
    on = np.abs(kmag - 4) < 1e-9
    assert np.max(np.abs(raw - oracle) * inside) / ref < 1e-12
    assert np.max(np.abs(raw - oracle) * on) / ref < 1e-12


# --- test/regressions/r7-reality-projection-forced-run.jl -----------------------------------------

def test_planted_anti_hermitian_pair_removed_by_one_step():
    N = 16
    dom = O.Domain(N)
    uh = S.seed_velocity(N, 0.5, seed=1)
    ph = S.seed_scalar(N, 0.5, seed=2)
    d = 2e-6 * np.max(np.abs(uh[:, :, :, 0]))
    uh[:, 0, 1, 0] += 1j * d
    uh[:, 0, N - 1, 0] += 1j * d
    ph[0, 1, 0] += 1j * d
    ph[0, N - 1, 0] += 1j * d
    st = O.step(dom, O.Conditions(viscosity=0.05, velocity_forcing=O.ConstantPower(0.1)), O.State(uh, ph), 0.01)
    for f in (st.uh, st.phih):
        plane = f[..., 0]
        neg = (-np.arange(N)) % N
        partner = np.conj(plane[..., neg, :][..., :, neg])
        assert np.max(np.abs(plane - partner)) == 0.0


# --- test/particles.jl -------------------------------------------------------------------------

def test_adams_weights_classical():
    # test/particles.jl:194-214
    def nodes(k):
        return tuple(-(i - 0.0) for i in range(k))
    assert np.allclose(O.adams_weights(nodes(1), 1.0), [1.0])
    assert np.allclose(O.adams_weights(nodes(2), 1.0), np.array([3, -1]) / 2)
    assert np.allclose(O.adams_weights(nodes(4), 1.0), np.array([55, -59, 37, -9]) / 24)
    assert np.allclose(O.adams_weights((1.0,) + nodes(1), 1.0), np.array([1, 1]) / 2)
    assert np.allclose(O.adams_weights((1.0,) + nodes(2), 1.0), np.array([5, 8, -1]) / 12)
    assert np.allclose(O.adams_weights(nodes(3), 1.0), np.array([23, -16, 5]) / 12)
    assert np.allclose(O.adams_weights((1.0,) + nodes(3), 1.0), np.array([9, 19, -5, 1]) / 24)
    assert np.allclose(O.adams_weights((1.0,) + nodes(4), 1.0), np.array([251, 646, -264, 106, -19]) / 720)
    uneven = (0.0, -0.3, -1.2, -1.4)
    assert sum(O.adams_weights(uneven, 0.7)) == pytest.approx(0.7, rel=1e-14)
    assert sum(w * x ** 3 for w, x in zip(O.adams_weights(uneven, 0.7), uneven)) == pytest.approx(0.7 ** 4 / 4,
                                                                                                 rel=1e-12)
    eight = tuple(-0.37 * i - 0.05 * (i + 1) ** 2 for i in range(8))
    assert sum(w * x ** 7 for w, x in zip(O.adams_weights(eight, 0.9), eight)) == pytest.approx(0.9 ** 8 / 8,
                                                                                                rel=1e-8)


# The straining flow of test/particles.jl:24-40: u_x = cos(ωt)·s·(x − x_c), reproduced exactly by
# Catmull–Rom, with the trajectory known in closed form.
STRAIN, FREQUENCY, CENTRE, START = 1.0, 3.0, math.pi, math.pi + 0.4


def _strain_exact(t):
    return CENTRE + (START - CENTRE) * math.exp(STRAIN * math.sin(FREQUENCY * t) / FREQUENCY)


def _strain_field(dom, t):
    u = np.zeros((3, dom.N, dom.N, dom.N))
    u[0] = (math.cos(FREQUENCY * t) * STRAIN * (np.arange(dom.N) * dom.dx - CENTRE))[None, None, :]
    return u


def strain_error(scheme, steps, exact_start):
    """test/particles.jl:46-67: the largest error along a pass; `exact_start` seeds the trail with
    the exact earlier samples at −h, −2h, … (h the first step)."""
    kind, k = scheme
    dom = O.Domain(16)
    X = np.array([[START], [1.0], [1.0]])
    trail = []
    if exact_start:
        h = steps[0]
        for j in range(k - 1, 0, -1):
            t = -j * h
            trail.insert(0, (t, np.array([[math.cos(FREQUENCY * t) * STRAIN * (_strain_exact(t) - CENTRE)], [0.0], [0.0]])))
    trail.insert(0, (0.0, O.interpolate(dom, _strain_field(dom, 0.0), X)))
    t, largest = 0.0, 0.0
    for h in steps:
        u = _strain_field(dom, t + h)
        J, corrected = (k, kind == "abm") if len(trail) >= k else (len(trail), True)
        X, _ = O.advect_adams(dom, X, [v for _, v in trail[:J]], [tt for tt, _ in trail[:J]], u, h, corrected)
        t += h
        trail = [(t, O.interpolate(dom, u, X))] + trail[:k - 1]
        largest = max(largest, abs(X[0, 0] - _strain_exact(t)))
    return largest


def _uniform(n, T=2.0):
    return [T / n] * n


def _uneven(n, T=2.0):
    h = np.array([1 + 0.3 * math.sin(7 * (i + 1)) for i in range(n)])
    return list(h * (T / h.sum()))


def _shortened(scheme, n, T=2.0, tau=1 / FREQUENCY):
    p = O.tracer_order(*scheme)
    dt = T / n
    steps, t = [], 0.0
    while t < T - 1e-12:
        h = min(dt, tau * (dt / tau) ** (p / 3)) if not steps else min(dt, O.startup_growth(p) * steps[-1])
        h = min(h, T - t)
        steps.append(h)
        t += h
    return steps


def _order(errors):
    return math.log2(errors[-2] / errors[-1])


@pytest.mark.parametrize("steps_of", [_uniform, _uneven], ids=["uniform", "uneven"])
def test_each_particle_scheme_converges_at_its_order(steps_of):
    # test/particles.jl:216-231: AB(k) at order k, ABM(k) at order k + 1, from exact earlier samples
    for scheme in [("ab", k) for k in range(1, 9)] + [("abm", k) for k in range(1, 8)]:
        p = O.tracer_order(*scheme)
        counts = (32, 64, 128) if p >= 6 else (64, 128, 256)
        errors = [strain_error(scheme, steps_of(n), True) for n in counts]
        assert abs(_order(errors) - p) < 0.5, (scheme, _order(errors))
    for k in range(1, 8):
        assert strain_error(("abm", k), _uniform(64), True) < strain_error(("ab", k + 1), _uniform(64), True)


def test_particle_startup_orders():
    # test/particles.jl:233-251: the ordinary start-up leaves a third-order error
    counts = (64, 128, 256)
    ref = [strain_error(("abm", 4), _uniform(n), False) for n in counts]
    assert 2.7 < _order(ref) < 3.3
    for scheme in (("ab", 6), ("ab", 8), ("abm", 7)):
        errors = [strain_error(scheme, _uniform(n), False) for n in counts]
        assert 2.7 < _order(errors) < 3.3
        assert errors[-1] == pytest.approx(ref[-1], rel=0.05)
    errors = [strain_error(("ab", 4), _uniform(n), False) for n in counts]
    assert 2.7 < _order(errors) < 3.5 and ref[-1] / 2 < errors[-1] < 2 * ref[-1]
    errors = [strain_error(("ab", 2), _uniform(n), False) for n in counts]
    assert 1.7 < _order(errors) < 2.3


def test_shortened_first_steps_restore_the_order():
    # test/particles.jl:253-271
    for scheme in [("ab", k) for k in range(3, 9)] + [("abm", k) for k in range(2, 8)]:
        errors = [strain_error(scheme, _shortened(scheme, n), False) for n in (32, 64, 128)]
        assert _order(errors) > O.tracer_order(*scheme) - 0.6, scheme
        assert errors[1] < 4 * strain_error(scheme, _uniform(64), True)
    p, tau, dt = 8, 1 / FREQUENCY, 2.0 / 64
    steps, t = [], 0.0
    while t < 2.0 - 1e-12:
        h = min(dt, tau * (dt / tau) ** (p / 3)) if not steps else min(dt, 2.0 * steps[-1])
        h = min(h, 2.0 - t)
        steps.append(h)
        t += h
    assert strain_error(("ab", 8), steps, False) > 20 * strain_error(("ab", 8), _shortened(("ab", 8), 64), False)


def test_tracers_uniform_flow_exact_and_wrap():
    # test/particles.jl:94-121
    N = 16
    dom = O.Domain(N)
    X0 = np.array([[0.1, 1.0, 2.0], [0.2, 2.0, 3.0], [0.3, 3.0, 4.0]]).T.copy()  # (3, M)
    u = np.zeros((3, N, N, N))
    u[0] = 0.5
    X, f0 = X0.copy(), O.interpolate(dom, u, X0)
    for _ in range(20):
        X, _ = O.advect_heun(dom, X, f0, u, 0.005)
        f0 = O.interpolate(dom, u, X)
    assert np.allclose(X[0], np.mod(X0[0] + 0.5 * 20 * 0.005, TWO_PI))
    assert np.allclose(X[1:], X0[1:])
    X = np.full((3, 1), 6.2)
    u[0] = 1.0
    f0 = O.interpolate(dom, u, X)
    for _ in range(30):
        X, _ = O.advect_heun(dom, X, f0, u, 0.02)
        f0 = O.interpolate(dom, u, X)
    assert np.all((X >= 0) & (X < TWO_PI))


def test_constant_field_interpolates_exactly():
    # test/particles.jl:134-140
    N = 16
    dom = O.Domain(N)
    X = S.seed_tracers(200, seed=5)
    f = np.full((N, N, N), 1.7)
    assert np.allclose(O.interpolate(dom, f, X), 1.7, rtol=1e-14)


def test_heun_second_order_on_straining_flow():
    # test/particles.jl:24-60,216-231: u_x = cos(ωt)·s·(x − x_c), a field Catmull–Rom reproduces
    N, s, w, xc, x0 = 16, 1.0, 3.0, math.pi, math.pi + 0.4
    dom = O.Domain(N)

    def exact(t):
        return xc + (x0 - xc) * math.exp(s * math.sin(w * t) / w)

    def field(t):
        u = np.zeros((3, N, N, N))
        xs = np.arange(N) * dom.dx
        u[0] = (math.cos(w * t) * s * (xs - xc))[None, None, :]
        return u

    def err(n):
        h = 2.0 / n
        X = np.array([[x0], [1.0], [1.0]])
        f0 = O.interpolate(dom, field(0.0), X)
        t, largest = 0.0, 0.0
        for _ in range(n):
            un = field(t + h)
            X, _ = O.advect_heun(dom, X, f0, un, h)
            t += h
            f0 = O.interpolate(dom, un, X)
            largest = max(largest, abs(X[0, 0] - exact(t)))
        return largest

    e = [err(n) for n in (64, 128, 256)]
    assert abs(math.log2(e[1] / e[2]) - 2.0) < 0.5


# --- test/below_scale.jl -------------------------------------------------------------------------

def _embed(uh, N, M):
    """The band-limited field's coefficients on an M-point grid (zero padding, rescaled for the
    unnormalised transform)."""
    out = np.zeros((3, M, M, M // 2 + 1), complex)
    m = np.fft.fftfreq(N, 1.0 / N).round().astype(int)
    for iz, mz in enumerate(m):
        for iy, my in enumerate(m):
            out[:, mz % M, my % M, : N // 2 + 1] = uh[:, iz, iy, :]
    return out * (M / N) ** 3


def _box_mean(a, q, axis):
    n = a.shape[axis]
    ext = np.concatenate([a, np.take(a, range(q), axis=axis)], axis=axis)
    c = np.cumsum(ext, axis=axis)
    lead = np.take(c, range(q - 1, q - 1 + n), axis=axis)
    lag = np.concatenate([np.zeros_like(np.take(a, [0], axis=axis)), np.take(c, range(n - 1), axis=axis)], axis=axis)
    return (lead - lag) / q


@pytest.mark.parametrize("N", [16, 12])
def test_energy_below_scale(N):
    # test/below_scale.jl:66-100: the largest side returns the whole-field pair, both rise with l,
    # and the definition in physical space (remove each box's mean on an 8× finer grid, average over
    # positions) agrees elementwise to 2/q² for a box of q fine points
    dom = O.Domain(N)
    uh = S.seed_velocity(N, 1.5, seed=N)
    nu = 0.02
    scales, k, eps = O.energy_below_scale(dom, uh, nu)
    assert np.allclose(scales, [n * 2 * math.pi / N for n in range(1, N + 1)], rtol=1e-15)
    assert k[-1] == pytest.approx(O.kinetic_energy(dom, uh), rel=1e-12)
    assert eps[-1] == pytest.approx(O.dissipation(dom, uh, nu), rel=1e-12)
    assert np.all(np.diff(k) >= 0) and np.all(np.diff(eps) >= 0) and np.all(k > 0)
    refine = 8
    M = refine * N
    u = sfft_irfft(_embed(uh, N, M), M)
    total = float((u ** 2).sum()) / M ** 3 / 2
    q = refine * np.arange(1, N + 1)
    for i, qq in enumerate(q):
        b = u
        for axis in (1, 2, 3):
            b = _box_mean(b, qq, axis)
        phys = total - float((b ** 2).sum()) / M ** 3 / 2
        assert abs(k[i] - phys) / phys < 2 / qq ** 2


def sfft_irfft(fh, M):
    return np.fft.irfftn(fh, s=(M, M, M), axes=(-3, -2, -1))


# --- test/observables_analytic.jl:78-110 ---------------------------------------------------------

def test_derivative_skewness():
    # zero for a field of three single modes, odd in the velocity, non-zero for a random field
    N = 16
    dom = O.Domain(N)
    x, y, z = _grid(N)
    uh = dom.to_spectral(np.stack([0.7 * np.sin(y), -0.4 * np.sin(z), 1.1 * np.sin(x)]))
    assert abs(O.derivative_skewness(dom, uh)) < 1e-12
    seeded = S.seed_velocity(N, 1.0, seed=5)
    sk = O.derivative_skewness(dom, seeded)
    assert sk != 0
    assert O.derivative_skewness(dom, -seeded) == pytest.approx(-sk, rel=1e-12)


def test_skewness_denominator_dirichlet_route():
    # ⟨S:S⟩ from the physical strain equals ½Σ|κ|²|û|² for a solenoidal field
    N = 32
    dom = O.Domain(N)
    uh = S.seed_velocity(N, 1.5, seed=8)
    s = O.strain_physical(dom, uh)
    direct = float((s[:3] ** 2).sum() + 2 * (s[3:] ** 2).sum()) / N ** 3
    assert direct == pytest.approx(dom.inner(uh, uh, dom.k2) / 2, rel=1e-12)


# --- the tangent-linear model and the discrete adjoint of the step (the adjoint form's checker) ---

def _random_state(dom, seed):
    v = S.seed_velocity(dom.N, 0.3, seed=seed)
    return O.reality_projection(dom, O.leray(dom, v, dom.mask))


@pytest.mark.parametrize("scheme,forcing", [("rk4", None), ("rk3", None), ("rk4", O.Linear(0.4)),
                                            ("rk4", O.ConstantPower(0.1)),
                                            ("rk4", O.VarianceController(0.4, turnover_time=0.5, gain=2.0)),
                                            ("rk4", O.VarianceRescaling(0.45, "total")),
                                            ("rk3", O.VarianceRescaling(0.3, "band")),
                                            ("heun", O.ConstantPower(0.1)), ("ssprk3", O.ConstantPower(0.1)),
                                            ("ssprk3", O.VarianceRescaling(0.45, "total"))])
def test_tangent_matches_central_differences(scheme, forcing):
    # J·δû against (F(û + εδû) − F(û − εδû))/(2ε), relative 1e-6
    dom = O.Domain(16)
    cond = O.Conditions(viscosity=0.02, scalar=False, velocity_forcing=forcing)
    uh, v = S.seed_velocity(16, 0.5, seed=3), _random_state(dom, 4)
    dt, eps = 0.02, 1e-5
    F0, Jv = O.step_tangent(dom, cond, uh, v, dt, scheme)
    Fp = O.step(dom, cond, O.State(uh + eps * v), dt, scheme).uh
    Fm = O.step(dom, cond, O.State(uh - eps * v), dt, scheme).uh
    ref = O.step(dom, cond, O.State(uh), dt, scheme).uh
    assert np.allclose(F0, ref, rtol=0, atol=1e-13 * np.abs(ref).max())
    fd = (Fp - Fm) / (2 * eps)
    assert np.linalg.norm(Jv - fd) / np.linalg.norm(fd) < 1e-6


@pytest.mark.parametrize("scheme,forcing", [("rk4", None), ("rk3", None), ("rk4", O.Linear(0.4)),
                                            ("rk4", O.ConstantPower(0.1)),
                                            ("rk4", O.VarianceController(0.4, turnover_time=0.5, gain=2.0)),
                                            ("rk4", O.VarianceRescaling(0.45, "total")),
                                            ("rk3", O.VarianceRescaling(0.3, "band")),
                                            ("heun", O.ConstantPower(0.1)), ("ssprk3", O.ConstantPower(0.1)),
                                            ("ssprk3", O.VarianceRescaling(0.45, "total"))])
def test_adjoint_dot_product_identity(scheme, forcing):
    # ⟨J v, w⟩ = ⟨v, Jᵀ w⟩ to round-off, for states in the retained, Hermitian space
    dom = O.Domain(16)
    cond = O.Conditions(viscosity=0.02, scalar=False, velocity_forcing=forcing)
    uh = S.seed_velocity(16, 0.5, seed=5)
    v, w = _random_state(dom, 6), _random_state(dom, 7)
    _, Jv = O.step_tangent(dom, cond, uh, v, 0.02, scheme)
    JTw = O.step_adjoint(dom, cond, uh, w, 0.02, scheme)
    lhs, rhs = O.spectral_dot(dom, Jv, w), O.spectral_dot(dom, v, JTw)
    assert lhs == pytest.approx(rhs, rel=1e-12)


def test_adjoint_gradient_of_the_kinetic_energy():
    # ∇ of k(F(û)) by the adjoint against central differences along three directions, 1e-6
    dom = O.Domain(16)
    cond = O.Conditions(viscosity=0.02, scalar=False)
    uh = S.seed_velocity(16, 0.5, seed=8)
    dt, eps = 0.02, 1e-5
    F0 = O.step(dom, cond, O.State(uh), dt).uh
    # k = ½Σw|û|²/N⁶, so its gradient in the spectral inner product is F/N⁶
    grad = O.step_adjoint(dom, cond, uh, F0 / float(dom.N) ** 6, dt)
    for seed in (9, 10, 11):
        v = _random_state(dom, seed)
        kp = O.kinetic_energy(dom, O.step(dom, cond, O.State(uh + eps * v), dt).uh)
        km = O.kinetic_energy(dom, O.step(dom, cond, O.State(uh - eps * v), dt).uh)
        assert O.spectral_dot(dom, grad, v) == pytest.approx((kp - km) / (2 * eps), rel=1e-6)


def _random_scalar(dom, seed):
    return O.reality_projection(dom, S.seed_scalar(dom.N, 0.3, seed=seed) * dom.mask)


@pytest.mark.parametrize("G,vf,sf", [((0.0, 0.0, 0.0), None, O.Linear(0.2)),
                                     ((1.0, 0.0, 0.0), O.ConstantPower(0.1), O.Linear(0.2)),
                                     ((0.0, 0.0, 1.0), O.Linear(0.3), O.ConstantPower(0.05)),
                                     ((0.0, 1.0, 0.0), O.VarianceController(0.4, turnover_time=0.5),
                                      O.VarianceRescaling(0.3, "total"))],
                         ids=["linear_phi", "benchmark_forcing", "cp_phi", "controller_u_rescale_phi"])
@pytest.mark.parametrize("scheme", ["rk4", "heun", "ssprk3"])
def test_coupled_tangent_and_adjoint(G, vf, sf, scheme):
    # the coupled velocity + scalar step (the benchmark's pair: ConstantPower on the velocity, the
    # mean gradient): the tangent against central differences, and the dot-product identity over
    # both fields
    dom = O.Domain(16)
    cond = O.Conditions(viscosity=0.02, schmidt=0.7, mean_gradient=G, velocity_forcing=vf, scalar_forcing=sf)
    uh, ph = S.seed_velocity(16, 0.5, seed=12), S.seed_scalar(16, 0.5, seed=13)
    v, vp = _random_state(dom, 14), _random_scalar(dom, 15)
    w, wp = _random_state(dom, 16), _random_scalar(dom, 17)
    dt, eps = 0.02, 1e-5
    Fu, Fp, Ju, Jp = O.step_tangent(dom, cond, uh, v, dt, scheme, ph=ph, dph=vp)
    st0 = O.step(dom, cond, O.State(uh, ph), dt, scheme)
    assert np.allclose(Fu, st0.uh, rtol=0, atol=1e-13 * np.abs(st0.uh).max())
    assert np.allclose(Fp, st0.phih, rtol=0, atol=1e-13 * np.abs(st0.phih).max())
    sp = O.step(dom, cond, O.State(uh + eps * v, ph + eps * vp), dt, scheme)
    sm = O.step(dom, cond, O.State(uh - eps * v, ph - eps * vp), dt, scheme)
    for J, fp, fm in ((Ju, sp.uh, sm.uh), (Jp, sp.phih, sm.phih)):
        fd = (fp - fm) / (2 * eps)
        assert np.linalg.norm(J - fd) / np.linalg.norm(fd) < 1e-6
    lu, lp = O.step_adjoint(dom, cond, uh, w, dt, scheme, ph=ph, lam_p=wp)
    lhs = O.spectral_dot(dom, Ju, w) + O.spectral_dot(dom, Jp, wp)
    rhs = O.spectral_dot(dom, v, lu) + O.spectral_dot(dom, vp, lp)
    assert lhs == pytest.approx(rhs, rel=1e-12)


def test_adjoint_chained_over_steps():
    # the gradient of k after three coupled steps: the one-step adjoint applied backwards over
    # the stored step states (what a checkpointed gradient recomputes), against central differences
    dom = O.Domain(16)
    cond = O.Conditions(viscosity=0.02, mean_gradient=(0.0, 1.0, 0.0), velocity_forcing=O.ConstantPower(0.1))
    uh, ph = S.seed_velocity(16, 0.5, seed=18), S.seed_scalar(16, 0.5, seed=19)
    dt, eps, n = 0.02, 1e-5, 3
    states = [O.State(uh, ph)]
    for _ in range(n):
        states.append(O.step(dom, cond, states[-1], dt))
    lu, lp = states[-1].uh / float(dom.N) ** 6, np.zeros_like(ph)   # ∇k in the spectral product
    for st in reversed(states[:-1]):
        lu, lp = O.step_adjoint(dom, cond, st.uh, lu, dt, ph=st.phih, lam_p=lp)

    def k_after(du, dp):
        st = O.State(uh + du, ph + dp)
        for _ in range(n):
            st = O.step(dom, cond, st, dt)
        return O.kinetic_energy(dom, st.uh)

    v, vp = _random_state(dom, 20), _random_scalar(dom, 21)
    fd = (k_after(eps * v, eps * vp) - k_after(-eps * v, -eps * vp)) / (2 * eps)
    assert O.spectral_dot(dom, v, lu) + O.spectral_dot(dom, vp, lp) == pytest.approx(fd, rel=1e-6)


def test_tracer_push_tangent_and_adjoint():
    # the Heun push and closing deposit through the Catmull–Rom gather, as a map of (û, X, f0):
    # the tangent against central differences, and the dot-product identity
    dom = O.Domain(16)
    rng = np.random.default_rng(3)
    uh = S.seed_velocity(16, 0.5, seed=22)
    X = S.seed_tracers(40, seed=23)
    f0 = O.interpolate(dom, dom.to_physical(uh), X) + 0.01 * rng.standard_normal((3, 40))
    h, eps = 0.03, 1e-6
    v, vX, vf = _random_state(dom, 24), rng.standard_normal((3, 40)), rng.standard_normal((3, 40))
    Xn, fn, dXn, dfn = O.heun_push_tangent(dom, uh, X, f0, h, v, vX, vf)
    Xr, _ = O.advect_heun(dom, X, f0, dom.to_physical(uh), h)
    assert np.max(np.abs(Xn - Xr)) < 1e-14

    def push(e):
        u = dom.to_physical(uh + e * v)
        Xa, _ = O.advect_heun(dom, X + e * vX, f0 + e * vf, u, h)
        return Xa, O.interpolate(dom, u, Xa)
    (Xp, fp), (Xm, fm) = push(eps), push(-eps)
    assert np.linalg.norm(dXn - (Xp - Xm) / (2 * eps)) / np.linalg.norm(dXn) < 1e-6
    assert np.linalg.norm(dfn - (fp - fm) / (2 * eps)) / np.linalg.norm(dfn) < 1e-6
    wX, wf = rng.standard_normal((3, 40)), rng.standard_normal((3, 40))
    lu, lX, lf0 = O.heun_push_adjoint(dom, uh, X, f0, h, wX, wf)
    lhs = float(np.sum(dXn * wX) + np.sum(dfn * wf))
    rhs = O.spectral_dot(dom, v, lu) + float(np.sum(vX * lX) + np.sum(vf * lf0))
    assert lhs == pytest.approx(rhs, rel=1e-12)


@pytest.mark.parametrize("n,snaps", [(8, 2), (10, 3), (6, 1), (5, 0), (20, 3)])
def test_binomial_checkpointing_gives_the_stored_gradient(n, snaps):
    # the checkpointed gradient over n coupled steps equals, bitwise, the one with every state
    # stored, while holding at most `snaps` states besides the start
    dom = O.Domain(12)
    cond = O.Conditions(viscosity=0.03, mean_gradient=(1.0, 0.0, 0.0), velocity_forcing=O.ConstantPower(0.1))
    st0 = O.State(S.seed_velocity(12, 0.5, seed=25), S.seed_scalar(12, 0.5, seed=26))
    dt = 0.02

    def loss_grad(st):   # k + ⟨φ²⟩ in the spectral product
        n6 = float(dom.N) ** 6
        return st.uh / n6, 2.0 * st.phih / n6

    states = [st0]
    for _ in range(n):
        states.append(O.step(dom, cond, states[-1], dt))
    lu, lp = loss_grad(states[-1])
    for x in reversed(states[:-1]):
        lu, lp = O.step_adjoint(dom, cond, x.uh, lu, dt, ph=x.phih, lam_p=lp)
    (gu, gp), stats = O.gradient_checkpointed(dom, cond, st0, dt, n, loss_grad, snaps)
    assert np.array_equal(gu, lu) and np.array_equal(gp, lp)
    assert stats["peak"] <= snaps
    assert stats["forward_steps"] <= O.binomial_repetitions(n, snaps) * n


def test_adjoint_of_a_whole_iteration_with_tracers():
    # one `advance` iteration: the coupled step, then the Heun push and closing deposit in the new
    # field. The loss reads the fields and the tracers, L = k + ½Σ|X_new − X₀|² + ½Σf_new²; its
    # gradient with respect to (û, φ̂, X, f₀) by the chained adjoints, against central differences
    dom = O.Domain(16)
    cond = O.Conditions(viscosity=0.02, mean_gradient=(1.0, 0.0, 0.0), velocity_forcing=O.ConstantPower(0.1))
    rng = np.random.default_rng(11)
    uh, ph = S.seed_velocity(16, 0.5, seed=27), S.seed_scalar(16, 0.5, seed=28)
    X = S.seed_tracers(30, seed=29)
    f0 = O.interpolate(dom, dom.to_physical(uh), X)
    dt = 0.02
    n6 = float(dom.N) ** 6

    def forward(uh_, ph_, X_, f0_):
        st = O.step(dom, cond, O.State(uh_, ph_), dt)
        Xn, _ = O.advect_heun(dom, X_, f0_, dom.to_physical(st.uh), dt)
        fn = O.interpolate(dom, dom.to_physical(st.uh), Xn)
        return st, Xn, fn

    def loss(uh_, ph_, X_, f0_):
        st, Xn, fn = forward(uh_, ph_, X_, f0_)
        return O.kinetic_energy(dom, st.uh) + 0.5 * float(np.sum((Xn - X) ** 2)) + 0.5 * float(np.sum(fn ** 2))

    st, Xn, fn = forward(uh, ph, X, f0)
    lu_push, lX, lf0 = O.heun_push_adjoint(dom, st.uh, X, f0, dt, Xn - X, fn)
    lu, lp = O.step_adjoint(dom, cond, uh, st.uh / n6 + lu_push, dt, ph=ph, lam_p=np.zeros_like(ph))
    v, vp = _random_state(dom, 30), _random_scalar(dom, 31)
    vX, vf = rng.standard_normal((3, 30)), rng.standard_normal((3, 30))
    eps = 1e-6
    fd = (loss(uh + eps * v, ph + eps * vp, X + eps * vX, f0 + eps * vf)
          - loss(uh - eps * v, ph - eps * vp, X - eps * vX, f0 - eps * vf)) / (2 * eps)
    ad = O.spectral_dot(dom, v, lu) + O.spectral_dot(dom, vp, lp) + float(np.sum(vX * lX) + np.sum(vf * lf0))
    assert ad == pytest.approx(fd, rel=1e-6)
