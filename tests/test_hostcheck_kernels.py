"""CPU check of the kernel bodies and the C ABI against the oracle.

The host-check build compiles the same CTA bodies and the same C ABI as the CUDA library, with
one thread per block and every launch run block by block on the CPU. Agreement here at round-off
level shows that the kernels' layouts, pruning, index arithmetic and launch sequence restate the
reference's step. The GPU suite (test_gpu_parity.py) repeats these comparisons on the device.
"""
import math

import numpy as np
import pytest

import gbght
from gbght import seed as S
from oracle import gbght_oracle as O
from pairs import advance_both, compare, make_case, rel_l2


@pytest.mark.parametrize("N,steps,forcing,G", [
    (16, 6, None, (0.0, 0.0, 0.0)),
    (16, 6, 0.1, (1.0, 0.0, 0.0)),
    (12, 4, 0.1, (0.0, 0.0, 0.0)),      # 3 | N: the closed ball's boundary shell
    (24, 3, None, (0.0, 1.0, 0.0)),     # radix 3·8
    (48, 2, 0.1, (1.0, 0.0, 0.0)),      # radix 3·4·4, |κ|² = 256 on the cutoff
])
def test_step_matches_oracle(hostcheck_library, N, steps, forcing, G):
    run, orun = make_case(N, forcing=forcing, G=G, tracers=32, library=hostcheck_library)
    advance_both(run, orun, steps, dt=0.005)
    res = compare(run, orun, tol=2e-14)
    assert res["X_err"] < 1e-13


@pytest.mark.parametrize("scheme", ["IFLowStorageRK4", "IFLowStorageRK3"])
def test_linear_forcing_both_fields_matches_oracle(hostcheck_library, scheme):
    # Linear on the velocity (shells 1–2) and on the scalar (shells 2–Inf), with the mean gradient
    run, orun = make_case(16, forcing=gbght.Linear(0.7), scalar_forcing=gbght.Linear(0.4, 2, math.inf),
                          G=(0.0, 0.0, 1.0), tracers=16, scheme=scheme, library=hostcheck_library)
    advance_both(run, orun, 4, dt=0.01)
    res = compare(run, orun, tol=2e-14)
    assert res["X_err"] < 1e-13


@pytest.mark.parametrize("vf,sf", [
    (gbght.VarianceController(0.4, turnover_time=0.5, gain=2.0), gbght.ConstantPower(0.2)),
    (gbght.ConstantPower(0.1), gbght.VarianceController(0.3, turnover_time=0.5, gain=1.0, highest_shell=3)),
    (gbght.VarianceRescaling(0.45, "total"), gbght.VarianceRescaling(0.2, "band", 1, math.inf)),
    (gbght.VarianceRescaling(0.3, "band", 2, 3), gbght.VarianceRescaling(0.6, "total")),
], ids=["controller_u+cp_phi", "cp_u+controller_phi", "rescale_total_u+band_phi", "rescale_band_u+total_phi"])
def test_band_forcings_both_fields_match_oracle(hostcheck_library, vf, sf):
    # the per-stage amplitudes (ConstantPower, VarianceController) and the post-step rescale
    # (VarianceRescaling) on each field, with the mean gradient and the tracers
    run, orun = make_case(16, forcing=vf, scalar_forcing=sf, G=(1.0, 0.0, 0.0), tracers=16, library=hostcheck_library)
    advance_both(run, orun, 4, dt=0.01)
    res = compare(run, orun, tol=2e-14)
    assert res["X_err"] < 1e-13


def test_rescaling_holds_the_target_exactly(hostcheck_library):
    run, _ = make_case(16, forcing=gbght.VarianceRescaling(0.45, "total"),
                       scalar_forcing=gbght.VarianceRescaling(0.6, "total", 1, math.inf), library=hostcheck_library)
    for _ in range(3):
        run.advance(0.01)
        ob = run.observables()
        assert ob["kinetic_energy"] == pytest.approx(0.45, rel=1e-13)
        assert ob["scalar_variance"] == pytest.approx(0.6, rel=1e-13)


@pytest.mark.parametrize("scheme", ["IFHeun", "IFSSPRK3"])
@pytest.mark.parametrize("vf,sf", [(0.1, None), (gbght.Linear(0.5), gbght.VarianceRescaling(0.3, "total")),
                                   (gbght.VarianceController(0.4, turnover_time=0.5), gbght.ConstantPower(0.2))],
                         ids=["cp", "linear+rescale", "controller+cp"])
def test_heun_and_ssprk3_match_oracle(hostcheck_library, scheme, vf, sf):
    # the two schemes outside the low-storage loop, with the forcings, G, CFL steps and tracers
    run, orun = make_case(16, forcing=vf, scalar_forcing=sf, G=(0.0, 0.0, 1.0), tracers=16, scheme=scheme,
                          cfl=0.25, library=hostcheck_library)
    taken = advance_both(run, orun, 4, dt=None)
    for d_lib, d_ora in taken:
        assert d_lib == pytest.approx(d_ora, rel=1e-13)
    res = compare(run, orun, tol=2e-14)
    assert res["X_err"] < 1e-13


def test_recommended_cfl(hostcheck_library):
    # test/integrators.jl:114-118, and the ceilings themselves (src/Propagator.jl:906-913)
    got = {s: gbght.recommended_cfl(s, library=hostcheck_library)
           for s in ("IFLowStorageRK4", "IFLowStorageRK3", "IFHeun", "IFSSPRK3")}
    assert got == {"IFLowStorageRK4": 0.96, "IFLowStorageRK3": 0.5, "IFHeun": 0.25, "IFSSPRK3": 0.5}
    with pytest.raises(ValueError):
        gbght.recommended_cfl("IFEuler", library=hostcheck_library)


def test_ensemble_steps_equal_separate_runs(hostcheck_library):
    # members of uneven sizes and configurations stepped together equal the same runs stepped alone
    def members():
        return [make_case(12, forcing=0.1, library=hostcheck_library)[0],
                make_case(16, scalar=False, scheme="IFLowStorageRK3", library=hostcheck_library)[0],
                make_case(24, forcing=gbght.Linear(0.3), scheme="IFHeun", library=hostcheck_library)[0]]
    ens_runs, alone = members(), members()
    ens = gbght.Ensemble(ens_runs)
    for _ in range(3):
        ens.step(0.01)
        for r in alone:
            r.step(0.01)
            r.deposit()
    for a, b in zip(ens_runs, alone):
        ua, pa = a.export_state()
        ub, pb = b.export_state()
        assert np.array_equal(ua, ub) and (pa is None or np.array_equal(pa, pb))
        assert a.max_speed() == b.max_speed()
    ens.close()
    with pytest.raises(ValueError, match="twice"):
        gbght.Ensemble([ens_runs[0], ens_runs[0]])


def test_rk3_and_cfl_steps_match(hostcheck_library):
    run, orun = make_case(16, forcing=0.2, scheme="IFLowStorageRK3", tracers=16, library=hostcheck_library)
    taken = advance_both(run, orun, 5, dt=None)
    for d_lib, d_ora in taken:
        assert d_lib == pytest.approx(d_ora, rel=1e-13)
    compare(run, orun, tol=2e-14)


def test_velocity_only_run(hostcheck_library):
    run, orun = make_case(16, scalar=False, forcing=0.1, library=hostcheck_library)
    advance_both(run, orun, 4, dt=0.01)
    compare(run, orun, tol=2e-14)


def test_observables_and_spectra(hostcheck_library):
    run, orun = make_case(24, forcing=0.1, library=hostcheck_library)
    advance_both(run, orun, 2, dt=0.01)
    ob = run.observables()
    d, st = orun.dom, orun.state
    assert ob["kinetic_energy"] == pytest.approx(O.kinetic_energy(d, st.uh), rel=1e-13)
    assert ob["dissipation"] == pytest.approx(O.dissipation(d, st.uh, 0.01), rel=1e-13)
    assert ob["scalar_variance"] == pytest.approx(O.scalar_variance(d, st.phih), rel=1e-13)
    assert ob["scalar_dissipation"] == pytest.approx(O.scalar_dissipation(d, st.phih, 0.01), rel=1e-13)
    assert np.allclose(run.energy_spectrum(), O.energy_spectrum(d, st.uh), rtol=1e-12, atol=1e-16)
    assert np.allclose(run.scalar_spectrum(), O.scalar_spectrum(d, st.phih), rtol=1e-12, atol=1e-16)
    assert run.max_speed() == pytest.approx(orun.speed, rel=1e-13)


@pytest.mark.parametrize("N", [16, 12])
def test_energy_below_scale_matches_oracle(hostcheck_library, N):
    run, orun = make_case(N, viscosity=0.02, energy=1.5, forcing=0.1, library=hostcheck_library)
    advance_both(run, orun, 2, dt=0.01)
    scales, k, eps = run.energy_below_scale()
    s_o, k_o, e_o = O.energy_below_scale(orun.dom, orun.state.uh, 0.02)
    assert np.array_equal(scales, s_o)
    assert np.allclose(k, k_o, rtol=1e-12, atol=0) and np.allclose(eps, e_o, rtol=1e-12, atol=0)


def test_derivative_skewness_matches_oracle(hostcheck_library):
    run, orun = make_case(16, forcing=0.1, tracers=8, library=hostcheck_library)
    advance_both(run, orun, 2, dt=0.01)
    sk = run.derivative_skewness()
    assert sk == pytest.approx(O.derivative_skewness(orun.dom, orun.state.uh), rel=1e-12)
    # the diagnostic leaves the run as it was: the next step is the oracle's
    advance_both(run, orun, 2, dt=0.01)
    compare(run, orun, tol=2e-14)


def test_deposited_velocity_and_interpolation(hostcheck_library):
    run, orun = make_case(16, tracers=8, library=hostcheck_library)
    u = run.velocity_physical()
    assert np.max(np.abs(u - orun.u)) < 1e-14
    X = S.seed_tracers(50, seed=9)
    assert np.max(np.abs(run.interpolate_velocity(X) - O.interpolate(orun.dom, orun.u, X))) < 1e-14


def test_separate_calls_equal_advance(hostcheck_library):
    # step! → deposit! → advect! → deposit!(tracers) is the same iteration as advance!
    a, _ = make_case(16, forcing=0.1, tracers=20, library=hostcheck_library)
    b, _ = make_case(16, forcing=0.1, tracers=20, library=hostcheck_library)
    a.advance(0.01)
    b.step(0.01)
    b.deposit()
    b.advect(0.01)
    b.deposit_tracers(0.01)
    ua, pa = a.export_state()
    ub, pb = b.export_state()
    assert np.array_equal(ua, ub) and np.array_equal(pa, pb)
    assert np.array_equal(a.tracers(), b.tracers())
    assert np.array_equal(a.tracer_sample()[0], b.tracer_sample()[0])


def test_reality_projection_removes_planted_violation(hostcheck_library):
    # test/regressions/r7-reality-projection-forced-run.jl:20-40
    N = 16
    uh = S.seed_velocity(N, 0.5, seed=1)
    ph = S.seed_scalar(N, 0.5, seed=2)
    d = 2e-6 * np.max(np.abs(uh[:, :, :, 0]))
    uh[:, 0, 1, 0] += 1j * d
    uh[:, 0, N - 1, 0] += 1j * d
    ph[0, 1, 0] += 1j * d
    ph[0, N - 1, 0] += 1j * d
    run, _ = make_case(N, forcing=0.1, uh=uh, ph=ph, library=hostcheck_library)
    run.advance(0.01)
    ue, pe = run.export_state()
    neg = (-np.arange(N)) % N
    for f in (ue, pe):
        plane = f[..., 0]
        partner = np.conj(plane[..., neg, :][..., :, neg])
        assert np.max(np.abs(plane - partner)) == 0.0


@pytest.mark.parametrize("scheme", [("AB", 4), ("ABM", 3), ("AB", 8), ("ABM", 7), ("Heun", 1)])
def test_adams_schemes_in_a_prescribed_straining_flow(hostcheck_library, scheme):
    # test/particles.jl:46-67 through the library: the straining flow written into the deposit slot,
    # the trail seeded with the exact earlier samples by the checkpoint restore, then per step the
    # field at the new time, the particle step and the deposit. Positions equal the oracle's.
    from test_oracle_known_answers import CENTRE, FREQUENCY, START, STRAIN, _strain_exact, _strain_field
    N, k = 16, scheme[1]
    dom = O.Domain(N)
    run = gbght.Run(gbght.Setup(grid_points_per_axis=N, tracers=1, tracer_scheme=scheme[0], tracer_steps=k),
                    library=hostcheck_library)
    X = np.array([[START], [1.0], [1.0]])
    steps = [2.0 / 48 * (1 + 0.3 * math.sin(7 * (i + 1))) for i in range(24)]
    run.deposit_prescribed_velocity(_strain_field(dom, 0.0))
    run.import_tracers(X)
    trail = []
    for j in range(k - 1, 0, -1):
        t = -j * steps[0]
        v = np.array([[math.cos(FREQUENCY * t) * STRAIN * (_strain_exact(t) - CENTRE)], [0.0], [0.0]])
        run.restore_tracer_sample(v, t)
        trail.insert(0, (t, v))
    run.deposit_tracers(0.0)
    trail.insert(0, (0.0, O.interpolate(dom, _strain_field(dom, 0.0), X)))
    kind = "ab" if scheme[0] == "AB" else "abm"
    t = 0.0
    for h in steps:
        u = _strain_field(dom, t + h)
        run.deposit_prescribed_velocity(u)
        run.advect(h)
        t += h
        run.deposit_tracers(t)
        J, corrected = (k, kind == "abm") if len(trail) >= k else (len(trail), True)
        X, _ = O.advect_adams(dom, X, [v for _, v in trail[:J]], [tt for tt, _ in trail[:J]], u, h, corrected)
        trail = [(t, O.interpolate(dom, u, X))] + trail[:k - 1]
        assert np.max(np.abs(run.tracers() - X)) < 1e-14
        F, tf = run.tracer_sample()
        assert tf == t and np.max(np.abs(F - trail[0][1])) < 1e-14
    assert abs(X[0, 0] - _strain_exact(t)) < 1e-4


@pytest.mark.parametrize("scheme,shortened", [(("AB", 4), False), (("ABM", 3), True), (("AB", 6), True)])
def test_adams_run_matches_oracle(hostcheck_library, scheme, shortened):
    # advance! with a multistep particle scheme on a forced flow: the trail fills through the lower
    # ABM members, and under shortened_first_steps the first steps follow the start-up bound
    run, orun = make_case(16, forcing=0.1, tracers=24, tracer_scheme=scheme, shortened_first_steps=shortened,
                          library=hostcheck_library)
    taken = advance_both(run, orun, 8, dt=None)
    for d_lib, d_ora in taken:
        assert d_lib == pytest.approx(d_ora, rel=1e-13)
    if shortened:
        assert taken[0][0] < 0.7 * taken[-1][0]   # the start is shortened, then grows back
    res = compare(run, orun, tol=2e-14)
    assert res["X_err"] < 1e-13
    if shortened:
        with pytest.raises(ValueError, match="shortened_first_steps"):
            run.advance(0.01)


def test_particle_scheme_refusals(hostcheck_library):
    # test/particles.jl:184-192
    def run(scheme, k):
        return gbght.Run(gbght.Setup(grid_points_per_axis=16, tracers=4, tracer_scheme=scheme, tracer_steps=k),
                         library=hostcheck_library)
    for scheme, k in (("AB", 0), ("AB", 9), ("ABM", 0), ("ABM", 8), ("Heun", 2)):
        with pytest.raises(ValueError):
            run(scheme, k)
    run("AB", 8).close()
    run("ABM", 7).close()


def test_prescribed_uniform_flow_advects_exactly(hostcheck_library):
    # test/particles.jl:94-108 through the prescribed-flow fake (test/prescribed_flow.jl)
    N = 16
    X0 = np.array([[0.1, 1.0, 2.0], [0.2, 2.0, 3.0], [0.3, 3.0, 4.0]]).T.copy()
    setup = gbght.Setup(grid_points_per_axis=N, tracers=3)
    run = gbght.Run(setup, library=hostcheck_library)
    u = np.zeros((3, N, N, N))
    u[0] = 0.5
    run.deposit_prescribed_velocity(u)
    run.import_tracers(X0)
    run.deposit_tracers(0.0)
    t = 0.0
    for _ in range(20):
        run.deposit_prescribed_velocity(u)
        run.advect(0.005)
        t += 0.005
        run.deposit_tracers(t)
    X = run.tracers()
    assert np.allclose(X[0], np.mod(X0[0] + 0.5 * 20 * 0.005, 2 * np.pi))
    assert np.allclose(X[1:], X0[1:])
