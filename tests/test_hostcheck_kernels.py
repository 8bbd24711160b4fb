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
