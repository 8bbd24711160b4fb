"""PhaseShift dealiasing (src/SimulationDomain.jl:177-184, src/Generator.jl:502-519,668-704): each
stage's nonlinear terms are the average of the grid's and those of the grid displaced by half a cell
along every axis, shifted back, on the closed ball of radius (2√2/3)·κ_Ny.

The oracle's restatement is pinned the way the reference's own test pins it (test/dealiasing.jl:
69-114): a field band-limited to the ball has a product that aliases into the ball on the N-point
grid, and the averaged term must equal the exact one a 2N zero-padded grid gives, while the raw
N-grid term must not. The library is then compared with the oracle through the C ABI."""
import math

import numpy as np
import pytest

import gbght
from oracle import gbght_oracle as O
from pairs import advance_both, compare, make_case


def _ball_field(dom, seed, ncomp=3, peak=4.0, mean_square=None):
    """A real random field filling PhaseShift's ball, its spectrum peaked at shell `peak`
    (solenoidal for three components), scaled to the box mean square `mean_square` when given."""
    rng = np.random.default_rng(seed)
    shape = (ncomp,) + dom.shape_spectral
    c = rng.standard_normal(shape) + 1j * rng.standard_normal(shape)
    k = np.sqrt(dom.k2)
    c = c * ((k / peak) ** 2 * np.exp(-((k / peak) ** 2))) * dom.mask
    if ncomp == 3:
        c = O.leray(dom, c)
    c = dom.to_spectral(dom.to_physical(c)) * dom.mask   # the Hermitian part
    if mean_square is not None:
        c = c * math.sqrt(mean_square / (2.0 * dom.inner(c, c)))
    return c if ncomp == 3 else c[0]


def _mapidx(i, N):
    return i if i <= N // 2 else i + N


def _embed(a, N):
    """Coefficients of an N-grid field on the 2N grid (zero padding, ×8 for the unnormalised
    transform)."""
    out = np.zeros(a.shape[:-3] + (2 * N, 2 * N, N + 1), complex)
    for i3 in range(N):
        for i2 in range(N):
            out[..., _mapidx(i3, N), _mapidx(i2, N), : N // 2 + 1] = 8 * a[..., i3, i2, :]
    return out


def _restrict(b, N):
    out = np.zeros(b.shape[:-3] + (N, N, N // 2 + 1), complex)
    for i3 in range(N):
        for i2 in range(N):
            out[..., i3, i2, :] = b[..., _mapidx(i3, N), _mapidx(i2, N), : N // 2 + 1] / 8
    return out


def test_phase_shift_ball_and_cfl():
    N = 12
    dps, d23 = O.Domain(N, dealiasing="PhaseShift"), O.Domain(N)
    assert set(np.unique(dps.mask)) <= {0.0, 1.0}
    assert dps.cutoff == pytest.approx((2 * math.sqrt(2) / 3) * (N / 2))
    assert dps.mask.sum() > d23.mask.sum()   # keeps more than the 2/3 ball
    # the boundary shell |m|² = 2N²/9 = 32 is kept (a closed ball)
    on = np.isclose(dps.k2, 32.0)
    assert on.any() and dps.mask[on].min() == 1.0
    # recommended_cfl: ×(2/3)/(2√2/3) = 1/√2 of the 2/3 rule's (test/dealiasing.jl:64-65)
    for scheme in ("IFLowStorageRK3", "IFLowStorageRK4", "IFHeun"):
        base = gbght.recommended_cfl(scheme)
        assert gbght.recommended_cfl(scheme, "PhaseShift") == pytest.approx(base / math.sqrt(2), rel=1e-15)
        assert gbght.recommended_cfl(scheme, "HouLi") == pytest.approx(base * 2 / 3, rel=1e-15)


def test_phase_shift_dealiases_exactly_against_zero_padded_product():
    # test/dealiasing.jl:69-114, the velocity's term
    N = 12
    dps, d2 = O.Domain(N, dealiasing="PhaseShift"), O.Domain(2 * N)
    uh = _ball_field(dps, 3)
    cond = O.Conditions(viscosity=1.0)
    u, w = dps.to_physical(uh), dps.to_physical(O.curl(dps, uh))
    ps = O.velocity_rhs(dps, cond, uh, u, w, np.finfo(float).eps)
    raw = O.leray(dps, dps.to_spectral(O._cross(u, w)))
    big = _embed(uh, N)
    exact = _restrict(O.leray(d2, d2.to_spectral(O._cross(d2.to_physical(big), d2.to_physical(O.curl(d2, big))))), N)
    exact[:, 0, 0, 0] = 0.0
    mask = dps.mask[None]
    ref = np.max(np.abs(exact) * mask)
    assert np.max(np.abs(ps - exact) * mask) / ref < 1e-10
    assert np.max(np.abs(raw - exact) * mask) / ref > 1e-2   # the raw product is aliased


def test_phase_shift_scalar_flux_dealiases_exactly():
    # the scalar's −𝔻∇·(uφ) against the zero-padded flux, and the raw flux's aliasing
    N = 12
    dps, d2 = O.Domain(N, dealiasing="PhaseShift"), O.Domain(2 * N)
    uh, ph = _ball_field(dps, 5), _ball_field(dps, 6, ncomp=1)
    cond = O.Conditions(viscosity=1.0)
    u, phi = dps.to_physical(uh), dps.to_physical(ph)
    ps = O.scalar_rhs(dps, cond, uh, u, phi, ph)

    def div(dom, fh):
        return -(1j * ((dom.dkx * fh[0] + dom.dky * fh[1]) + dom.dkz * fh[2]))

    raw = div(dps, dps.to_spectral(u * phi[None]))
    bu, bp = _embed(uh, N), _embed(ph, N)
    exact = _restrict(div(d2, d2.to_spectral(d2.to_physical(bu) * d2.to_physical(bp)[None])), N)
    mask = dps.mask
    ref = np.max(np.abs(exact) * mask)
    assert np.max(np.abs(ps - exact) * mask) / ref < 1e-10
    assert np.max(np.abs(raw - exact) * mask) / ref > 1e-2


def test_phase_shift_refuses_the_tangent():
    dom = O.Domain(8, dealiasing="PhaseShift")
    uh = np.zeros((3,) + dom.shape_spectral, complex)
    with pytest.raises(ValueError, match="PhaseShift"):
        O.step_tangent(dom, O.Conditions(viscosity=0.1, scalar=False), uh, uh, 0.01)


def _case(N, library, precision="fp64", tracers=100, **kw):
    # box mean squares ⟨|u|²⟩ = ⟨φ²⟩ = ½, physical sizes like the seeders' (an unscaled field is
    # physically tiny, and the ConstantPower rate ε/(2E) would then amplify it by orders of
    # magnitude in one step)
    dom = O.Domain(N, dealiasing="PhaseShift")
    uh = _ball_field(dom, 1, mean_square=1.0)
    ph = _ball_field(dom, 2, ncomp=1, mean_square=1.0)
    return make_case(N, viscosity=0.01, forcing=0.1, G=(1.0, 0.0, 0.0), tracers=tracers, dealiasing="PhaseShift",
                     precision=precision, library=library, uh=uh, ph=ph, **kw)


@pytest.mark.parametrize("N", [12, 16])
def test_phase_shift_matches_the_oracle_hostcheck(hostcheck_library, N):
    run, orun = _case(N, hostcheck_library)
    assert run.K == int(math.floor(math.sqrt(2) * N / 3))
    advance_both(run, orun, 4, dt=0.01)
    compare(run, orun, tol=1e-12)


@pytest.mark.parametrize("scheme", ["IFLowStorageRK3", "IFHeun", "IFSSPRK3"])
def test_phase_shift_schemes_hostcheck(hostcheck_library, scheme):
    run, orun = _case(12, hostcheck_library, tracers=0, scheme=scheme)
    advance_both(run, orun, 3, dt=0.01)
    compare(run, orun, tol=1e-12)


def test_phase_shift_keeps_the_wider_band_and_refuses_the_adjoint_hostcheck(hostcheck_library):
    N = 16
    run, _ = _case(N, hostcheck_library, tracers=0)
    for _ in range(3):
        run.advance(0.02)
    u, _ = run.export_state()
    d23 = O.Domain(N)
    outside = (d23.k2 > d23.cutoff ** 2)[None]
    assert np.abs(u * outside).max() > 1e-6 * np.abs(u).max()   # energy past the 2/3 ball
    dps = O.Domain(N, dealiasing="PhaseShift")
    assert np.abs(u * (1.0 - dps.mask)[None]).max() == 0.0    # and none past the PhaseShift ball
    with pytest.raises(ValueError, match="TwoThirds"):
        run.adjoint_create(1)


@pytest.mark.gpu
@pytest.mark.parametrize("N,precision,tol", [(64, "fp64", 1e-12), (64, "fp32_mixed", 1e-5), (128, "fp64", 1e-12)])
def test_phase_shift_matches_the_oracle(cuda_library, N, precision, tol):
    run, orun = _case(N, cuda_library, precision=precision, tracers=1000)
    advance_both(run, orun, 4 if N == 64 else 2, dt=0.005)
    compare(run, orun, tol=tol, check_tracers=precision == "fp64")


@pytest.mark.parametrize("forcing", ["Linear", "VarianceController", "VarianceRescaling", "StochasticOU"])
def test_phase_shift_with_the_other_forcings_hostcheck(hostcheck_library, forcing):
    # the displaced-grid average ahead of the forcings' sources and projections
    vf = {"Linear": gbght.Linear(0.2), "VarianceController": gbght.VarianceController(0.3, 1.0),
          "VarianceRescaling": gbght.VarianceRescaling(0.3, "total"),
          "StochasticOU": gbght.StochasticOU(0.05, 0.5, 1, 2, seed=7)}[forcing]
    dom = O.Domain(12, dealiasing="PhaseShift")
    run, orun = make_case(12, viscosity=0.01, forcing=vf, dealiasing="PhaseShift", library=hostcheck_library,
                          uh=_ball_field(dom, 1, mean_square=1.0), ph=_ball_field(dom, 2, ncomp=1, mean_square=1.0))
    for _ in range(3):
        run.advance(0.01)
        if forcing == "StochasticOU":   # the oracle is given the force the library was given
            orun.cond.velocity_forcing.process = run.processes[0].amplitudes.copy()
        orun.advance(0.01)
    compare(run, orun, tol=1e-12)
