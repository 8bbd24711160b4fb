"""The wider interpolation stencils, LalescuSpline(n; smoothness) and LagrangeSpline(n)
(src/Particles.jl:61-70), in the oracle (known answers) and in the library (against the oracle)."""
import numpy as np
import pytest

import gbght
from oracle import gbght_oracle as O
from pairs import advance_both, compare, make_case

SCHEMES = [("LalescuSpline", 6, 1), ("LalescuSpline", 8, 2), ("LalescuSpline", 8, 3), ("LagrangeSpline", 6, 0),
           ("LagrangeSpline", 8, 0)]


def _weights(scheme, t):
    P = O.stencil_polynomials(scheme)
    return np.array([np.polynomial.polynomial.polyval(t, P[j]) for j in range(P.shape[0])])


@pytest.mark.parametrize("scheme", SCHEMES, ids=[f"{k}{n}_{m}" for k, n, m in SCHEMES])
def test_stencil_known_answers(scheme):
    kind, n, m = scheme
    t = np.linspace(0.0, 1.0, 11)
    w = _weights(scheme, t)
    taps = np.arange(n) - (n // 2 - 1)
    assert np.allclose(w.sum(axis=0), 1.0, atol=1e-14)        # constants exactly
    assert np.allclose((w * taps[:, None]).sum(axis=0), t, atol=1e-13)   # linear exactly
    if kind == "LagrangeSpline":
        for d in range(n):   # polynomials through degree n − 1 exactly
            assert np.allclose((w * taps[:, None] ** d).sum(axis=0), t ** d, atol=1e-12)
        assert np.allclose(w[:, 0], np.eye(n)[n // 2 - 1], atol=1e-14)   # interpolating at the nodes
    else:
        # interpolating at both ends, and C^m: a value's weight in cell i + 1 is its tap's weight
        # shifted by one, so the derivatives 1..m at t = 1 of w_j equal those at t = 0 of w_(j−1)
        P = O.stencil_polynomials(scheme)
        assert np.allclose(w[:, 0], np.eye(n)[n // 2 - 1], atol=1e-13)
        assert np.allclose(w[:, -1], np.eye(n)[n // 2], atol=1e-13)
        for k in range(1, m + 1):
            dP = np.array([np.polynomial.polynomial.polyder(P[j], k) for j in range(n)])
            at1 = np.array([np.polynomial.polynomial.polyval(1.0, dP[j]) for j in range(n)])
            at0 = np.array([np.polynomial.polynomial.polyval(0.0, dP[j]) for j in range(n)])
            assert np.allclose(at1[1:], at0[:-1], atol=1e-12) and abs(at1[0]) < 1e-12 and abs(at0[-1]) < 1e-12


def test_lalescu_four_is_catmull_rom():
    t = np.linspace(0.0, 1.0, 7)
    assert np.allclose(_weights(("LalescuSpline", 4, 1), t), np.array(O.catmull_rom_weights(t)), atol=1e-15)


@pytest.mark.parametrize("scheme", SCHEMES[:2] + SCHEMES[3:4], ids=["lalescu6_1", "lalescu8_2", "lagrange6"])
def test_wider_stencils_match_the_oracle_hostcheck(hostcheck_library, scheme):
    run, orun = make_case(16, forcing=0.1, tracers=200, interpolation=scheme, library=hostcheck_library)
    advance_both(run, orun, 4, dt=0.01)
    res = compare(run, orun, tol=1e-12)
    assert res["X_err"] < 1e-10


def test_stencil_refusals_hostcheck(hostcheck_library):
    with pytest.raises(ValueError, match="4, 6 or 8"):
        gbght.Run(gbght.Setup(grid_points_per_axis=16, tracers=4, interpolation=("LagrangeSpline", 5, 0)),
                  library=hostcheck_library)
    with pytest.raises(ValueError, match="smoothness"):
        gbght.Run(gbght.Setup(grid_points_per_axis=16, tracers=4, interpolation=("LalescuSpline", 4, 3)),
                  library=hostcheck_library)


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", SCHEMES, ids=[f"{k}{n}_{m}" for k, n, m in SCHEMES])
def test_wider_stencils_match_the_oracle(cuda_library, scheme):
    run, orun = make_case(64, forcing=0.1, tracers=2000, interpolation=scheme, library=cuda_library)
    advance_both(run, orun, 5, dt=0.01)
    res = compare(run, orun, tol=1e-12)
    assert res["X_err"] < 1e-10
