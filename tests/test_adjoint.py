"""The discrete adjoint of the field step against the oracle's (oracle.step_adjoint, pinned there by
central finite differences and the dot-product identity), through the C ABI.

CPU tests run the host-check build (the same CTA bodies on one CPU thread); GPU tests run the CUDA
library. The adjoint lives on the retained 2/3 ball, so the oracle's Jᵀλ is compared on the ball.
"""
import math

import numpy as np
import pytest

import gbght
from gbght import adjoint as AD
from gbght import seed as S
from oracle import gbght_oracle as O
from pairs import oracle_forcing, rel_l2


def _rand_ball(dom, rng, shape):
    return (rng.standard_normal(shape) + 1j * rng.standard_normal(shape)) * dom.mask


def adjoint_pair(library, N, *, forcing=None, scalar_forcing=None, G=(0.0, 0.0, 0.0), scalar=True,
                 scheme="IFLowStorageRK4", precision="fp64", dt=0.01, viscosity=0.01, seed=5):
    """(library Jᵀλ, oracle Jᵀλ on the ball, run, setup) for one step at a seeded state."""
    uh = S.seed_velocity(N, 0.5, seed=0)
    ph = S.seed_scalar(N, 0.5, seed=1) if scalar else None
    dom = O.Domain(N)
    rng = np.random.default_rng(seed)
    lam = _rand_ball(dom, rng, (3,) + dom.shape_spectral)
    lamp = _rand_ball(dom, rng, dom.shape_spectral) if scalar else None
    setup = gbght.Setup(grid_points_per_axis=N, viscosity=viscosity, scalar=scalar,
                        velocity_forcing=forcing or gbght.NoForcing(),
                        scalar_forcing=scalar_forcing or gbght.NoForcing(), mean_gradient=G, scheme=scheme,
                        precision=precision)
    run = gbght.simulation(setup, uh, ph, library=library)
    run.adjoint_create(2)
    run.adjoint_import(lam, lamp)
    run.adjoint_step(dt)
    lib = run.adjoint_export()
    cond = O.Conditions(viscosity=viscosity, scalar=scalar, velocity_forcing=oracle_forcing(forcing),
                        scalar_forcing=oracle_forcing(scalar_forcing), mean_gradient=G)
    osch = {"IFLowStorageRK4": "rk4", "IFLowStorageRK3": "rk3"}[scheme]
    if scalar:
        ou, op = O.step_adjoint(dom, cond, uh, lam, dt, osch, ph, lamp)
        ora = (ou * dom.mask, op * dom.mask)
    else:
        ora = (O.step_adjoint(dom, cond, uh, lam, dt, osch) * dom.mask, None)
    return lib, ora, run, (uh, ph, lam, lamp, dom, cond, osch)


CASES = {
    "unforced_G": dict(G=(1.0, 0.5, 0.0)),
    "constant_power": dict(forcing=gbght.ConstantPower(0.1), G=(1.0, 0.0, 0.0)),
    "both_fields": dict(forcing=gbght.Linear(0.3), scalar_forcing=gbght.ConstantPower(0.05, 1, 3), G=(0.0, 1.0, 0.0)),
    "rk3_velocity_only": dict(forcing=gbght.ConstantPower(0.2), scalar=False, scheme="IFLowStorageRK3"),
}


@pytest.mark.parametrize("case", list(CASES), ids=list(CASES))
def test_adjoint_step_matches_the_oracle_hostcheck(hostcheck_library, case):
    (lu, lp), (ou, op), run, _ = adjoint_pair(hostcheck_library, 12, **CASES[case])
    assert rel_l2(lu, ou) <= 1e-13
    if op is not None:
        assert rel_l2(lp, op) <= 1e-13
    uh = S.seed_velocity(12, 0.5, seed=0)
    ue, _ = run.export_state()
    assert np.array_equal(ue, uh)   # the state is left as it was


def _spectral_dot(dom, a, b):
    return O.spectral_dot(dom, a, b)


def test_forcing_gradient_matches_finite_differences_hostcheck(hostcheck_library):
    # d⟨λ, F(q; ε)⟩/dε for both fields' ConstantPower rates, against central differences of the oracle
    N, dt = 12, 0.01
    vf, sf = gbght.ConstantPower(0.1), gbght.ConstantPower(0.05)
    _, _, run, (uh, ph, lam, lamp, dom, cond, osch) = adjoint_pair(hostcheck_library, N, forcing=vf, scalar_forcing=sf,
                                                                   G=(1.0, 0.0, 0.0), dt=dt)
    gu, gp = run.forcing_gradient()
    h = 1e-6

    def pairing(eu, ep):
        c = O.Conditions(viscosity=0.01, velocity_forcing=O.ConstantPower(eu), scalar_forcing=O.ConstantPower(ep),
                         mean_gradient=(1.0, 0.0, 0.0))
        st = O.step(dom, c, O.State(uh.copy(), ph.copy()), dt, osch)
        return _spectral_dot(dom, lam, st.uh) + _spectral_dot(dom, lamp, st.phih)
    fu = (pairing(0.1 + h, 0.05) - pairing(0.1 - h, 0.05)) / (2 * h)
    fp = (pairing(0.1, 0.05 + h) - pairing(0.1, 0.05 - h)) / (2 * h)
    assert gu == pytest.approx(fu, rel=1e-6)
    assert gp == pytest.approx(fp, rel=1e-6)


def test_adjoint_refusals_hostcheck(hostcheck_library):
    run = gbght.Run(gbght.Setup(grid_points_per_axis=12, scheme="IFHeun"), library=hostcheck_library)
    with pytest.raises(ValueError, match="low-storage"):
        run.adjoint_create(2)
    run = gbght.Run(gbght.Setup(grid_points_per_axis=12, velocity_forcing=gbght.VarianceRescaling(0.5, "band")),
                    library=hostcheck_library)
    with pytest.raises(ValueError, match="ConstantPower"):
        run.adjoint_create(2)
    run = gbght.Run(gbght.Setup(grid_points_per_axis=12), library=hostcheck_library)
    with pytest.raises(gbght.DeviceError, match="not set up"):
        run.adjoint_step(0.01)
    run.adjoint_create(1)
    dom = O.Domain(12)
    bad = np.ones((3,) + dom.shape_spectral, np.complex128)
    with pytest.raises(ValueError, match="outside the retained"):
        run.adjoint_import(bad, np.zeros(dom.shape_spectral, np.complex128))
    lu, _ = run.adjoint_export()
    assert not lu.any()
    with pytest.raises(ValueError, match="snapshot"):
        run.snapshot_save(3)


def test_snapshots_restore_the_state_hostcheck(hostcheck_library):
    N = 12
    setup = gbght.Setup(grid_points_per_axis=N, velocity_forcing=gbght.ConstantPower(0.1))
    run = gbght.simulation(setup, S.seed_velocity(N, 0.5, seed=0), S.seed_scalar(N, 0.5, seed=1),
                           library=hostcheck_library)
    run.adjoint_create(2)
    u0, p0 = run.export_state()
    run.snapshot_save(1)
    run.advance(0.01)
    run.snapshot_load(1)
    with pytest.raises(gbght.ScheduleError):
        run.step(0.01)   # the deposit is stale after a load
    run.deposit()
    u1, p1 = run.export_state()
    assert np.array_equal(u0, u1) and np.array_equal(p0, p1)


def oracle_window_gradient(dom, cond, uh, ph, dts, n0, n1):
    """∂L/∂q_0 of L = mean over n0..n1 of ⟨φ²⟩ by the oracle: every state stored, the adjoints
    chained backwards."""
    states = [O.State(uh.copy(), ph.copy())]
    for d in dts:
        states.append(O.step(dom, cond, states[-1], d, "rk4"))
    N6 = float(dom.N) ** 6
    w = 1.0 / (n1 - n0 + 1)
    lu = np.zeros_like(uh)
    lp = np.zeros_like(ph)
    for k in range(len(dts), -1, -1):
        if k < len(dts):
            lu, lp = O.step_adjoint(dom, cond, states[k].uh, lu, dts[k], "rk4", states[k].phih, lp)
        if n0 <= k <= n1:
            lp = lp + w * 2.0 * states[k].phih / N6
    return lu * dom.mask, lp * dom.mask


def test_checkpointed_sweep_matches_the_oracle_hostcheck(hostcheck_library):
    # 7 uneven steps, a window loss over steps 3..7, two snapshot slots: recomputation from slots
    N = 12
    uh, ph = S.seed_velocity(N, 0.5, seed=0), S.seed_scalar(N, 0.5, seed=1)
    dts = [0.01, 0.012, 0.009, 0.011, 0.01, 0.008, 0.013]
    setup = gbght.Setup(grid_points_per_axis=N, velocity_forcing=gbght.ConstantPower(0.1), mean_gradient=(1.0, 0.0, 0.0))
    run = gbght.simulation(setup, uh, ph, library=hostcheck_library)
    run.adjoint_create(2)
    (lu, lp), _, sweep = AD.gradient(run, dts, AD.scalar_variance_window(3, 7), snapshots=2)
    dom = O.Domain(N)
    cond = O.Conditions(viscosity=0.01, velocity_forcing=O.ConstantPower(0.1), mean_gradient=(1.0, 0.0, 0.0))
    ou, op = oracle_window_gradient(dom, cond, uh, ph, dts, 3, 7)
    assert rel_l2(lu, ou) <= 1e-12 and rel_l2(lp, op) <= 1e-12
    assert sweep.adjoint_steps == 7 and sweep.peak <= 2
    ue, pe = run.export_state()
    assert np.array_equal(ue, uh) and np.array_equal(pe, ph)


# ------------------------------------------------------------------------------------------------
# GPU
# ------------------------------------------------------------------------------------------------
@pytest.mark.gpu
@pytest.mark.parametrize("case", list(CASES), ids=list(CASES))
@pytest.mark.parametrize("N,precision,tol", [(64, "fp64", 1e-12), (64, "fp32_mixed", 1e-5), (128, "fp64", 1e-12)])
def test_adjoint_step_matches_the_oracle(cuda_library, case, N, precision, tol):
    (lu, lp), (ou, op), _, _ = adjoint_pair(cuda_library, N, precision=precision, **CASES[case])
    assert rel_l2(lu, ou) <= tol
    if op is not None:
        assert rel_l2(lp, op) <= tol


@pytest.mark.gpu
def test_dot_product_identity_against_the_oracle_tangent(cuda_library):
    # ⟨J v, w⟩ = ⟨v, Jᵀ w⟩ with J v the oracle's tangent-linear step and Jᵀ w the GPU adjoint
    N, dt = 64, 0.01
    vf = gbght.ConstantPower(0.1)
    (lu, lp), _, _, (uh, ph, lam, lamp, dom, cond, osch) = adjoint_pair(cuda_library, N, forcing=vf,
                                                                        G=(1.0, 0.0, 0.0), dt=dt)
    rng = np.random.default_rng(11)
    vu, vp = _rand_ball(dom, rng, (3,) + dom.shape_spectral), _rand_ball(dom, rng, dom.shape_spectral)
    vu = O.leray(dom, vu)
    _, _, ju, jp = O.step_tangent(dom, cond, uh, vu, dt, osch, ph, vp)
    left = O.spectral_dot(dom, ju, lam) + O.spectral_dot(dom, jp, lamp)
    right = O.spectral_dot(dom, vu, lu) + O.spectral_dot(dom, vp, lp)
    assert right == pytest.approx(left, rel=1e-12)


def _c4_forward_loss(library, setup, uh, ph, X, dts, n0, n1):
    """L = mean over steps n0..n1 of ⟨φ²⟩ + (1/M) Σ_p |u(X_p)|² at step n1, the tracers advected by
    Heun from X along the fixed Δt sequence."""
    run = gbght.simulation(setup, uh, ph, X, library=library)
    total = 0.0
    for k in range(len(dts) + 1):
        if k > 0:
            run.advance(dts[k - 1])
        if n0 <= k <= n1:
            total += run.observables()["scalar_variance"]
    f, _ = run.tracer_sample()
    run.close()
    return total / (n1 - n0 + 1) + float(np.sum(f * f)) / f.shape[1]


@pytest.mark.gpu
def test_c4_gradient_against_central_differences(cuda_library):
    # 128³ forced velocity + scalar, ν = ϰ = 6e-3, ConstantPower ε = 0.1 on shells 1–2, G = 1 along x,
    # IF-RK4, 16384 Heun tracers. Loss: the scalar variance averaged over steps 100..200 plus the
    # mean squared velocity sampled at the tracers at step 200 (Δt held at the CFL sequence of the
    # unperturbed run). Gradients with respect to ε and the initial velocity, by the checkpointed
    # reverse sweep with 16 stored states, against central differences (h = 1e-6) of the FP64
    # forward along 8 seeded directions.
    N, M, nsteps, n0 = 128, 16384, 200, 100
    uh, ph, X = S.seed_velocity(N, 0.5, seed=0), S.seed_scalar(N, 0.5, seed=1), S.seed_tracers(M, seed=2)
    eps = 0.1

    def setup(e):
        return gbght.Setup(grid_points_per_axis=N, viscosity=6e-3, velocity_forcing=gbght.ConstantPower(e),
                           mean_gradient=(1.0, 0.0, 0.0), cfl=0.5, tracers=M)
    ref = gbght.simulation(setup(eps), uh, ph, X, library=cuda_library)
    dts = [ref.advance(None) for _ in range(nsteps)]
    ref.close()
    run = gbght.simulation(setup(eps), uh, ph, X, library=cuda_library)
    run.adjoint_create(16)
    loss_grad = AD.combined(AD.scalar_variance_window(n0, nsteps), AD.tracer_kinetic_energy(nsteps))
    (lu, lp), (geps, _), sweep = AD.gradient(run, dts, loss_grad, snapshots=16)
    assert sweep.peak <= 16 and sweep.adjoint_steps == nsteps
    h = 1e-6
    fd = (_c4_forward_loss(cuda_library, setup(eps + h), uh, ph, X, dts, n0, nsteps)
          - _c4_forward_loss(cuda_library, setup(eps - h), uh, ph, X, dts, n0, nsteps)) / (2 * h)
    errs = [abs(geps - fd) / abs(fd)]
    dom = O.Domain(N)
    rng = np.random.default_rng(2024)
    for _ in range(8):
        v = O.leray(dom, _rand_ball(dom, rng, (3,) + dom.shape_spectral))
        v *= np.linalg.norm(uh) / np.linalg.norm(v)
        # a Hermitian kx = 0 plane keeps the perturbed state a real field
        v = O.reality_projection(dom, v)
        dL = (_c4_forward_loss(cuda_library, setup(eps), uh + h * v, ph, X, dts, n0, nsteps)
              - _c4_forward_loss(cuda_library, setup(eps), uh - h * v, ph, X, dts, n0, nsteps)) / (2 * h)
        ad = O.spectral_dot(dom, lu, v)
        errs.append(abs(ad - dL) / abs(dL))
    # and the initial positions, along one seeded direction
    vX = rng.standard_normal((3, M)) * 1e-2
    dL = (_c4_forward_loss(cuda_library, setup(eps), uh, ph, X + h * vX, dts, n0, nsteps)
          - _c4_forward_loss(cuda_library, setup(eps), uh, ph, X - h * vX, dts, n0, nsteps)) / (2 * h)
    errs.append(abs(float(np.sum(sweep.tracer_gradient * vX)) - dL) / abs(dL))
    print(f"C4 128^3: dL/deps adjoint {geps:.10e} fd {fd:.10e}; relative errors {['%.1e' % e for e in errs]}; "
          f"{sweep.forward_steps} recomputed steps, {sweep.peak} slots")
    assert max(errs) <= 1e-6


def iteration_adjoint_pair(library, N, M, *, precision="fp64", dt=0.01, seed=9):
    """The reverse of one advance! iteration with Heun tracers through the library and the oracle
    (heun_push_adjoint, then step_adjoint on the state cotangent with the push's part added)."""
    uh, ph, X = S.seed_velocity(N, 0.5, seed=0), S.seed_scalar(N, 0.5, seed=1), S.seed_tracers(M, seed=2)
    dom = O.Domain(N)
    rng = np.random.default_rng(seed)
    lam, lamp = _rand_ball(dom, rng, (3,) + dom.shape_spectral), _rand_ball(dom, rng, dom.shape_spectral)
    lX, lf = rng.standard_normal((3, M)), rng.standard_normal((3, M))
    setup = gbght.Setup(grid_points_per_axis=N, viscosity=0.01, velocity_forcing=gbght.ConstantPower(0.1),
                        mean_gradient=(1.0, 0.0, 0.0), tracers=M, precision=precision)
    run = gbght.simulation(setup, uh, ph, X, library=library)
    f0, _ = run.tracer_sample()
    run.adjoint_create(1)
    run.adjoint_import(lam, lamp)
    run.adjoint_tracers_import(lX, lf)
    run.adjoint_advance(dt)
    lib = run.adjoint_export() + run.adjoint_tracers_export()
    cond = O.Conditions(viscosity=0.01, velocity_forcing=O.ConstantPower(0.1), mean_gradient=(1.0, 0.0, 0.0))
    st = O.step(dom, cond, O.State(uh.copy(), ph.copy()), dt)
    lu_push, oX, of = O.heun_push_adjoint(dom, st.uh, X, f0, dt, lX, lf)
    ou, op = O.step_adjoint(dom, cond, uh, lam + lu_push, dt, "rk4", ph, lamp)
    return lib, (ou * dom.mask, op * dom.mask, oX, of), run, (uh, ph, X, f0)


def test_iteration_adjoint_with_tracers_matches_the_oracle_hostcheck(hostcheck_library):
    (lu, lp, lX, lf), (ou, op, oX, of), run, (uh, ph, X, f0) = iteration_adjoint_pair(hostcheck_library, 12, 40)
    assert rel_l2(lu, ou) <= 1e-12 and rel_l2(lp, op) <= 1e-12
    assert rel_l2(lX, oX) <= 1e-12 and rel_l2(lf, of) <= 1e-12
    ue, _ = run.export_state()
    assert np.array_equal(ue, uh) and np.array_equal(run.tracers(), X)
    F, _ = run.tracer_sample()
    assert np.array_equal(F, f0)   # the run is left at (q, X, f)
    run.advance(0.01)              # and its schedule is intact


def test_particle_deposit_adjoint_matches_the_oracle_hostcheck(hostcheck_library):
    N, M = 12, 40
    uh, ph, X = S.seed_velocity(N, 0.5, seed=0), S.seed_scalar(N, 0.5, seed=1), S.seed_tracers(M, seed=2)
    setup = gbght.Setup(grid_points_per_axis=N, tracers=M)
    run = gbght.simulation(setup, uh, ph, X, library=hostcheck_library)
    run.adjoint_create(0)
    lf = np.random.default_rng(3).standard_normal((3, M))
    run.adjoint_tracers_import(np.zeros((3, M)), lf)
    run.adjoint_deposit_tracers()
    lu, _ = run.adjoint_export()
    lX, lf_after = run.adjoint_tracers_export()
    dom = O.Domain(N)
    ou_phys, oX = O.interpolate_adjoint(dom, dom.to_physical(uh), X, lf)
    ou = dom.to_spectral(ou_phys) / float(N) ** 3 * dom.mask
    assert rel_l2(lu, ou) <= 1e-12 and rel_l2(lX, oX) <= 1e-12 and not lf_after.any()


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("fp32_mixed", 1e-5)])
def test_iteration_adjoint_with_tracers_matches_the_oracle(cuda_library, precision, tol):
    (lu, lp, lX, lf), (ou, op, oX, of), _, _ = iteration_adjoint_pair(cuda_library, 64, 2000, precision=precision)
    assert rel_l2(lu, ou) <= tol and rel_l2(lp, op) <= tol
    assert rel_l2(lX, oX) <= tol and rel_l2(lf, of) <= tol
