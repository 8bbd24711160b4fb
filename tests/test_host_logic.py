"""The C ABI's argument and schedule refusals, which mirror the reference's ArgumentError and
ErrorException cases. These run through the host-check build; the refusals are host code shared
with the CUDA library."""
import math

import numpy as np
import pytest

import gbght
from gbght import seed as S
from pairs import make_case


def test_bad_configurations_are_argument_errors(hostcheck_library):
    with pytest.raises(ValueError, match="viscosity"):
        gbght.Run(gbght.Setup(grid_points_per_axis=16, viscosity=0.0), library=hostcheck_library)
    with pytest.raises(ValueError, match="schmidt"):
        gbght.Run(gbght.Setup(grid_points_per_axis=16, schmidt=-1.0), library=hostcheck_library)
    with pytest.raises(ValueError, match="grid_points_per_axis"):
        gbght.Run(gbght.Setup(grid_points_per_axis=20), library=hostcheck_library)
    with pytest.raises(ValueError, match="mean scalar gradient"):
        gbght.Run(gbght.Setup(grid_points_per_axis=16, scalar=False, mean_gradient=(1.0, 0, 0)),
                  library=hostcheck_library)


def test_bad_forcing_bands_are_argument_errors(hostcheck_library):
    # src/Forcing.jl:387-403 (`_check_shells`) for both fields' bands; src/Generator.jl:312-316
    def run(**kw):
        return gbght.Run(gbght.Setup(grid_points_per_axis=16, **kw), library=hostcheck_library)
    for make in (lambda f: run(velocity_forcing=f), lambda f: run(scalar_forcing=f)):
        with pytest.raises(ValueError, match="lowest_shell"):
            make(gbght.Linear(0.5, lowest_shell=0))
        with pytest.raises(ValueError, match="integer shell"):
            make(gbght.Linear(0.5, highest_shell=2.5))
        with pytest.raises(ValueError, match="at least `lowest_shell`"):
            make(gbght.Linear(0.5, lowest_shell=3, highest_shell=2))
        with pytest.raises(ValueError, match="finite"):
            make(gbght.Linear(math.nan))
        make(gbght.Linear(0.5, highest_shell=math.inf)).close()
    with pytest.raises(ValueError, match="lowest_shell"):
        run(velocity_forcing=gbght.ConstantPower(0.1, lowest_shell=0))
    with pytest.raises(ValueError, match="carries no scalar"):
        run(scalar=False, scalar_forcing=gbght.Linear(1.0))


def test_bad_controller_and_rescaling_are_argument_errors(hostcheck_library):
    # src/Forcing.jl:558-572 (VarianceRescaling) and :828-875 (VarianceController)
    def run(**kw):
        return gbght.Run(gbght.Setup(grid_points_per_axis=16, **kw), library=hostcheck_library)
    for field in ("velocity_forcing", "scalar_forcing"):
        with pytest.raises(ValueError, match="`target` must be finite and positive"):
            run(**{field: gbght.VarianceController(0.0, turnover_time=1.0)})
        with pytest.raises(ValueError, match="`gain` must be finite and non-negative"):
            run(**{field: gbght.VarianceController(1.5, turnover_time=1.0, gain=-1.0)})
        with pytest.raises(ValueError, match="`gain` must be finite and non-negative"):
            run(**{field: gbght.VarianceController(1.5, turnover_time=1.0, gain=math.inf)})
        with pytest.raises(ValueError, match="`turnover_time` must be finite and positive"):
            run(**{field: gbght.VarianceController(1.5, turnover_time=0.0)})
        run(**{field: gbght.VarianceController(1.5, turnover_time=1.0, gain=0.0)}).close()   # the marginal law
        with pytest.raises(ValueError, match="`target` must be finite and non-negative"):
            run(**{field: gbght.VarianceRescaling(-1.0, "band")})
        with pytest.raises(ValueError, match="`over` must be :band or :total"):
            run(**{field: gbght.VarianceRescaling(1.0, "shell")})
        with pytest.raises(ValueError, match="lowest_shell"):
            run(**{field: gbght.VarianceRescaling(1.0, "total", lowest_shell=0)})
        run(**{field: gbght.VarianceRescaling(0.0, "total", highest_shell=math.inf)}).close()


def test_state_outside_the_retained_ball_is_refused(hostcheck_library):
    N = 16
    run = gbght.Run(gbght.Setup(grid_points_per_axis=N), library=hostcheck_library)
    uh = S.seed_velocity(N, 0.5, seed=0)
    ph = S.seed_scalar(N, 0.5, seed=1)
    uh[0, 0, 0, N // 2] = 1.0            # the Nyquist plane: outside the 2/3 ball
    with pytest.raises(ValueError, match="outside the retained"):
        run.import_state(uh, ph)


def test_step_needs_a_current_deposit(hostcheck_library):
    run, _ = make_case(16, library=hostcheck_library)
    run.step(0.01)
    with pytest.raises(gbght.ScheduleError, match="stale"):
        run.step(0.01)
    run.deposit()
    run.step(0.01)


def test_nonpositive_or_nonfinite_steps_are_refused(hostcheck_library):
    run, _ = make_case(16, tracers=4, library=hostcheck_library)
    for bad in (0.0, -0.01, math.inf, math.nan):
        with pytest.raises(ValueError):
            run.step(bad)
    with pytest.raises(ValueError):
        run.advance(math.inf)


def test_particle_schedule_refusals(hostcheck_library):
    run, _ = make_case(16, tracers=4, library=hostcheck_library)
    # the fields have not moved past the tracers' sample: the push is refused
    with pytest.raises(gbght.ScheduleError, match="one step ahead"):
        run.advect(0.01)
    run.step(0.01)
    run.deposit()
    with pytest.raises(ValueError, match="positive"):
        run.advect(-1.0)
    # a second sample at the same positions is refused
    with pytest.raises(gbght.ScheduleError):
        run.deposit_tracers(0.01)
    run.advect(0.01)
    with pytest.raises(ValueError, match="later"):
        run.deposit_tracers(0.0)
    run.deposit_tracers(0.01)
    # an iteration whose fields were stepped alone is refused whole
    run.step(0.01)
    run.deposit()
    run.advect(0.01)
    with pytest.raises(gbght.ScheduleError):
        run.advance(0.01)


def test_blowup_guard_names_the_step(hostcheck_library):
    N = 16
    uh = S.seed_velocity(N, 0.5, seed=0)
    ph = S.seed_scalar(N, 0.5, seed=1)
    uh[0, 0, 1, 1] = complex(np.nan, 0.0)   # a retained mode made non-finite on the host
    run, _ = make_case(N, uh=uh, ph=ph, library=hostcheck_library)
    assert not math.isfinite(run.max_speed())
    with pytest.raises(gbght.ScheduleError, match="blown up"):
        run.advance(None)
    with pytest.raises(gbght.ScheduleError, match="blown up"):
        run.advance(0.01)
    assert run.status_word() & 0x1


def test_empty_band_clamps_and_flags(hostcheck_library):
    N = 16
    uh = S.seed_velocity(N, 0.5, seed=0)
    k2 = S.wavenumbers(N)[3]
    uh = uh * ~((k2 >= 0.25) & (k2 <= 6.25))[None]
    run, _ = make_case(N, uh=uh, forcing=0.1, library=hostcheck_library)
    run.advance(0.01)
    assert run.status_word() & 0x2


@pytest.mark.parametrize("sf", [gbght.ConstantPower(0.2), gbght.VarianceController(0.5, turnover_time=1.0),
                                gbght.VarianceRescaling(0.5, "total"), gbght.VarianceRescaling(0.5, "band")],
                         ids=["constant_power", "controller", "rescale_total", "rescale_band"])
def test_empty_scalar_band_is_left_alone_and_flagged(hostcheck_library, sf):
    # src/Forcing.jl:110-111 with 575-596 and 1091-1101: an empty band gets no amplitude and no
    # rescale. With u = 0 the scalar band stays empty through the step, so the scalar moves by
    # diffusion alone, as the oracle's does, and the status word carries the empty-band bit.
    from pairs import advance_both
    N = 16
    k2 = S.wavenumbers(N)[3]
    ph = S.seed_scalar(N, 0.5, seed=1) * ~((k2 >= 0.25) & (k2 <= 6.25))
    run, orun = make_case(N, uh=np.zeros((3, N, N, N // 2 + 1), complex), ph=ph, scalar_forcing=sf,
                          library=hostcheck_library)
    advance_both(run, orun, 3, dt=0.01)
    ue, pe = run.export_state()
    assert not np.any(ue)
    assert np.linalg.norm(pe - orun.state.phih) <= 2e-14 * np.linalg.norm(orun.state.phih)
    expected = ph * np.exp(-0.01 * k2 * 0.03)
    assert np.max(np.abs(pe - expected)) <= 1e-14 * np.max(np.abs(ph))
    assert run.status_word() & 0x2


def test_empty_velocity_band_skips_the_rescale(hostcheck_library):
    # a single shear mode on shell 3 has a gradient Lamb vector: the band 1–2 stays empty, the
    # rescale is skipped, and the mode decays by viscosity alone
    from pairs import advance_both, compare
    N = 16
    uh = np.zeros((3, N, N, N // 2 + 1), complex)   # u_x = sin 3y, exactly
    uh[0, 0, 3, 0] = -0.5j * N ** 3
    uh[0, 0, N - 3, 0] = 0.5j * N ** 3
    run, orun = make_case(N, uh=uh, scalar=False, forcing=gbght.VarianceRescaling(0.45, "total"),
                          library=hostcheck_library)
    advance_both(run, orun, 2, dt=0.01)
    compare(run, orun, tol=2e-14)
    ue, _ = run.export_state()
    assert np.max(np.abs(ue - uh * np.exp(-0.01 * 9 * 0.02))) <= 1e-13 * np.max(np.abs(uh))
    assert run.status_word() & 0x2


def test_expired_device_wait_is_a_device_error(hostcheck_library):
    # the host-check build stands the expiry in for the device's barrier; the path from the raised
    # bit to GBGHT_ERR_DEVICE and the status word is the library's own
    run, _ = make_case(16, forcing=0.1, tracers=64, library=hostcheck_library)
    with pytest.raises(gbght.DeviceError, match="bounded wait"):
        run.selftest_wait_timeout(1000)
    assert run.status_word() & 0x4
    assert run.status_word() == 0
    run.advance(0.01)
    with pytest.raises(ValueError):
        run.selftest_wait_timeout(0)


def test_trail_export_holds_every_sample(hostcheck_library):
    run, _ = make_case(16, forcing=0.1, tracers=64, tracer_scheme=("AB", 3), library=hostcheck_library)
    assert [t for t, _ in run.tracer_trail()] == [0.0]
    for _ in range(4):
        run.advance(0.01)
    trail = run.tracer_trail()
    assert len(trail) == 3
    assert [t for t, _ in trail] == pytest.approx([0.02, 0.03, 0.04], abs=1e-15)
    F, t = run.tracer_sample()
    assert t == trail[-1][0] and np.array_equal(F, trail[-1][1])


@pytest.mark.parametrize("tracer_scheme", [("Heun", 1), ("AB", 3)])
def test_checkpoint_continues_bitwise(hostcheck_library, tracer_scheme):
    from checkpoint import continuation_is_bitwise
    N, M = 16, 100
    setup = gbght.Setup(grid_points_per_axis=N, viscosity=0.01, velocity_forcing=gbght.ConstantPower(0.1),
                        mean_gradient=(1.0, 0.0, 0.0), tracers=M, tracer_scheme=tracer_scheme[0],
                        tracer_steps=tracer_scheme[1])
    continuation_is_bitwise(setup, S.seed_velocity(N, 0.5, seed=0), S.seed_scalar(N, 0.5, seed=1),
                            S.seed_tracers(M, seed=2), before=4, after=3, library=hostcheck_library)
