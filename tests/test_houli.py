"""HouLi dealiasing (src/SimulationDomain.jl:131,365-376): no cutoff, the nonlinear terms filtered by
exp(−strength·(|κ|/κ_Ny)^order); the library stores every mode but the Nyquist planes, where the
filter is at round-off. Against the oracle with the same filter, through the C ABI."""
import math

import numpy as np
import pytest

import gbght
from gbght import seed as S
from oracle import gbght_oracle as O
from pairs import advance_both, compare, make_case


def test_houli_filter_known_answers():
    dom = O.Domain(32, dealiasing="HouLi")
    assert dom.mask.max() == 1.0 and dom.mask[0, 0, 0] == 1.0
    kny = 16.0
    # the damping at the Nyquist wavenumber is eps (strength −log eps), and 4/5 of the way it is mild
    assert math.exp(-(-math.log(np.finfo(float).eps)) * 1.0) == pytest.approx(np.finfo(float).eps)
    k2 = dom.k2
    at = np.isclose(np.sqrt(k2), 0.8 * kny)
    if at.any():
        assert dom.mask[at].min() > 0.99


@pytest.mark.parametrize("N", [12, 16])
def test_houli_matches_the_oracle_hostcheck(hostcheck_library, N):
    run, orun = make_case(N, forcing=0.1, G=(1.0, 0.0, 0.0), tracers=100, dealiasing="HouLi",
                          library=hostcheck_library)
    assert run.K == N // 2 - 1
    advance_both(run, orun, 5, dt=0.01)
    # the oracle keeps the Nyquist planes, at round-off under the filter
    compare(run, orun, tol=1e-12)


def test_houli_state_fills_the_box_hostcheck(hostcheck_library):
    # unlike the 2/3 rule, HouLi leaves the modes past 2/3 of Nyquist energetic
    N = 16
    run, _ = make_case(N, forcing=0.1, dealiasing="HouLi", library=hostcheck_library)
    for _ in range(5):
        run.advance(0.02)
    u, _ = run.export_state()
    dom = O.Domain(N)
    outside = (dom.k2 > dom.cutoff ** 2)[None]
    assert np.abs(u * outside).max() > 1e-8 * np.abs(u).max()
    with pytest.raises(ValueError, match="TwoThirds"):
        run.adjoint_create(1)


@pytest.mark.gpu
@pytest.mark.parametrize("N,precision,tol", [(64, "fp64", 1e-12), (64, "fp32_mixed", 1e-5), (128, "fp64", 1e-12)])
def test_houli_matches_the_oracle(cuda_library, N, precision, tol):
    run, orun = make_case(N, viscosity=0.005, forcing=0.1, G=(1.0, 0.0, 0.0), tracers=1000, dealiasing="HouLi",
                          precision=precision, library=cuda_library)
    advance_both(run, orun, 5 if N == 64 else 2, dt=0.005)
    compare(run, orun, tol=tol, check_tracers=precision == "fp64")


@pytest.mark.gpu
def test_wide_and_two_thirds_runs_share_a_process(cuda_library):
    # runs of one precision and N under different bands share kernels whose shared memory grows with
    # K: a TwoThirds run built after a HouLi one must not shrink what the HouLi run's launches need
    wide, _ = make_case(32, forcing=0.1, dealiasing="HouLi", library=cuda_library)
    narrow, _ = make_case(32, forcing=0.1, library=cuda_library)
    for r in (wide, narrow, wide):
        r.advance(0.004)
    wide.close()
    narrow.close()
