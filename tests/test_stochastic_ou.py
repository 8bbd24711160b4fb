"""StochasticOU (src/Forcing.jl:1224-1415): the host's Ornstein–Uhlenbeck process and the library's
additive force, against the oracle given the same process, through the C ABI."""
import math

import numpy as np
import pytest

import gbght
from gbght import stochastic as SO
from pairs import compare, make_case


def _ou_case(library, N, precision="fp64", scalar_ou=True, tracers=0):
    vf = gbght.StochasticOU(0.05, 0.5, 1, 2, seed=7)
    sf = gbght.StochasticOU(0.02, 0.3, 1, 3, seed=8) if scalar_ou else None
    return make_case(N, viscosity=0.01, forcing=vf, scalar_forcing=sf, G=(1.0, 0.0, 0.0), tracers=tracers,
                     precision=precision, library=library)


def _advance_pair(run, orun, steps, dt):
    for _ in range(steps):
        run.advance(dt)
        # the oracle is given the force the library was given for this step
        orun.cond.velocity_forcing.process = run.processes[0].amplitudes.copy()
        if 1 in run.processes:
            orun.cond.scalar_forcing.process = run.processes[1].amplitudes.copy()
        orun.advance(dt)


def test_ou_process_is_stationary_with_the_correlation_time():
    # the force's mean square stays at σ² in expectation, and its lag-one correlation is exp(−Δt/T_L)
    p = SO.OUProcess(0.05, 0.5, 1, 2, seed=3, vector=True)
    dt, ms, prods = 0.1, [], []
    prev = p.amplitudes.copy()
    for _ in range(4000):
        a = p.advance(dt)
        ms.append(p.mean_square())
        prods.append(float(np.sum((np.conj(prev) * a).real)) / max(1e-300, float(np.sum(np.abs(prev) ** 2))))
        prev = a.copy()
    assert np.mean(ms) == pytest.approx(0.05, rel=0.05)
    assert np.mean(prods) == pytest.approx(math.exp(-dt / 0.5), abs=0.02)
    # transverse and band-limited
    kx, ky, kz = SO._wavenumbers(p.n, p.L)
    div = kx * p.amplitudes[0] + ky * p.amplitudes[1] + kz * p.amplitudes[2]
    assert np.max(np.abs(div)) < 1e-14 * np.max(np.abs(p.amplitudes))
    assert not np.any(p.amplitudes * (1 - p.band))


def test_stochastic_ou_matches_the_oracle_hostcheck(hostcheck_library):
    run, orun = _ou_case(hostcheck_library, 16, tracers=50)
    _advance_pair(run, orun, 5, 0.01)
    compare(run, orun, tol=1e-12)


def test_stochastic_ou_schedule_and_refusals_hostcheck(hostcheck_library):
    run, _ = _ou_case(hostcheck_library, 16, scalar_ou=False)
    assert run.lib.gbght_step(run.h, 0.01) == gbght.ERR_SCHEDULE   # no force set for this step
    run.step(0.01)                                                 # the binding sets it first
    run.deposit()
    assert run.lib.gbght_step(run.h, 0.01) == gbght.ERR_SCHEDULE   # a force serves one step
    with pytest.raises(ValueError, match="companion grid"):
        run.set_forcing_source(0, np.zeros((3, 8, 8, 5), np.complex128))
    with pytest.raises(ValueError, match="past the dealias cutoff"):
        gbght.Run(gbght.Setup(grid_points_per_axis=8, velocity_forcing=gbght.StochasticOU(0.1, 1.0, 1, 3)),
                  library=hostcheck_library)
    with pytest.raises(ValueError, match="finite `highest_shell`"):
        gbght.Run(gbght.Setup(grid_points_per_axis=16, velocity_forcing=gbght.StochasticOU(0.1, 1.0, 1, math.inf)),
                  library=hostcheck_library)


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32_mixed", 1e-5)])
def test_stochastic_ou_matches_the_oracle(cuda_library, precision, tol):
    run, orun = _ou_case(cuda_library, 64, precision=precision, tracers=500)
    _advance_pair(run, orun, 10, 0.005)
    compare(run, orun, tol=tol, check_tracers=precision == "fp64")
