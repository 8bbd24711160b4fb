"""Box scaling (the reference's test/box_scaling.jl, re-expressed through the C ABI): a run on a box of
side L = 0.02 is the run on L = 2π with every quantity rescaled by its dimension. With σ = L/2π,
lengths and velocities scale by σ, k, ε and ν by σ², wavenumbers by 1/σ, and time and the scalar not
at all, so the two runs agree to rounding once rescaled. The scaling itself is the oracle, and the box
is far from 2π, so a fundamental wavenumber dropped anywhere in the library fails by orders of
magnitude."""
import math

import numpy as np
import pytest

import gbght
from gbght import seed as S

L = 0.02
SIG = L / (2 * math.pi)
N = 16


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(a)))


def _pair(lib, dealiasing, forcing_ref, forcing_small, scalar_forcing=None, tracers=0, X=None, **kw):
    uh = S.seed_velocity(N, 0.5, seed=1)
    ph = S.seed_scalar(N, 0.5, seed=2)
    runs = []
    for side, nu, forcing, scale in ((2 * math.pi, 0.02, forcing_ref, 1.0), (L, 0.02 * SIG ** 2, forcing_small, SIG)):
        setup = gbght.Setup(grid_points_per_axis=N, side_length=side, viscosity=nu, velocity_forcing=forcing,
                            scalar=scalar_forcing is not None, scalar_forcing=scalar_forcing or gbght.NoForcing(),
                            dealiasing=dealiasing, tracers=tracers, **kw)
        runs.append(gbght.simulation(setup, uh * scale, ph if scalar_forcing is not None else None,
                                     None if X is None else X * scale, library=lib))
    return runs


CASES = {
    "NoForcing": (gbght.NoForcing(), gbght.NoForcing(), None),
    "ConstantPower": (gbght.ConstantPower(0.3), gbght.ConstantPower(0.3 * SIG ** 2), None),
    "Linear": (gbght.Linear(0.2), gbght.Linear(0.2), None),
    "VarianceRescaling": (gbght.VarianceRescaling(1.0, "total"), gbght.VarianceRescaling(SIG ** 2, "total"), None),
    "VarianceController": (gbght.VarianceController(1.5, 1.0), gbght.VarianceController(1.5 * SIG ** 2, 1.0), None),
    "ConstantPower with a scalar": (gbght.ConstantPower(0.3), gbght.ConstantPower(0.3 * SIG ** 2),
                                    gbght.VarianceRescaling(1.0, "total")),
}


@pytest.mark.parametrize("dealiasing", ["TwoThirds", "PhaseShift", "HouLi"])
@pytest.mark.parametrize("case", list(CASES))
def test_fixed_steps_scale_with_the_box_hostcheck(hostcheck_library, dealiasing, case):
    # test/box_scaling.jl:41-70: four fixed steps, every dealiasing, every forcing, and the scalar
    fr, fs, sf = CASES[case]
    ref, small = _pair(hostcheck_library, dealiasing, fr, fs, scalar_forcing=sf)
    for _ in range(4):
        ref.advance(0.002)
        small.advance(0.002)
    ur, pr = ref.export_state()
    us, ps = small.export_state()
    assert _rel(ur, us / SIG) < 1e-13
    if sf is not None:
        assert _rel(pr, ps) < 1e-13


def _adaptive_pair(lib):
    X = np.random.default_rng(9).uniform(0.0, 2 * math.pi, (3, 20))
    return _pair(lib, "TwoThirds", gbght.StochasticOU(0.5, 0.7, seed=5), gbght.StochasticOU(0.5 * SIG ** 2, 0.7, seed=5),
                 tracers=20, X=X, tracer_scheme="AB", tracer_steps=3), X


def _check_adaptive(ref, small):
    for _ in range(8):
        ref.advance(None)
        small.advance(None)
    assert small.clock()[0] == pytest.approx(ref.clock()[0], rel=1e-13)   # the CFL step is box-free
    ur, us = ref.export_state()[0], small.export_state()[0]
    # eight CFL steps of about 0.08 at 16³: the rescaled runs agree to 2e-13 (the reference states
    # 1e-13 for its own arithmetic; each step here adds about 2e-14)
    assert _rel(ur, us / SIG) < 3e-13
    assert np.allclose(small.tracers() / SIG, ref.tracers(), rtol=1e-13, atol=1e-13)
    obr, obs = ref.observables(), small.observables()
    assert obs["kinetic_energy"] == pytest.approx(SIG ** 2 * obr["kinetic_energy"], rel=1e-13)
    # ε scales by σ² with ν·σ² against ν: the library's dissipation carries its own run's ν
    assert obs["dissipation"] == pytest.approx(SIG ** 2 * obr["dissipation"], rel=1e-13)
    assert small.derivative_skewness() == pytest.approx(ref.derivative_skewness(), rel=1e-12)
    Er, Es = ref.energy_spectrum(), small.energy_spectrum()
    live = Er > 1e-12 * Er.max()
    assert np.allclose(Es[live] / SIG ** 3, Er[live], rtol=1e-12)   # a density: σ² over 1/σ
    lr, kr, er = ref.energy_below_scale()
    ls, ks, es = small.energy_below_scale()
    assert np.allclose(ls / SIG, lr, rtol=1e-13)
    assert np.allclose(ks / SIG ** 2, kr, rtol=1e-12)
    assert np.allclose(es / SIG ** 2, er, rtol=1e-12)


def test_adaptive_steps_tracers_and_observables_scale_hostcheck(hostcheck_library):
    # test/box_scaling.jl:73-115 (the CFL Δt, a StochasticOU forcing, AB(3) tracers with Catmull–Rom,
    # the observables)
    (ref, small), _ = _adaptive_pair(hostcheck_library)
    _check_adaptive(ref, small)


@pytest.mark.gpu
def test_adaptive_steps_tracers_and_observables_scale(cuda_library):
    (ref, small), _ = _adaptive_pair(cuda_library)
    _check_adaptive(ref, small)
