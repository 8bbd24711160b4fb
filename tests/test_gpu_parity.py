"""Parity of the CUDA library (sm_100a) with the CPU oracle, through the C ABI.

The bar (FP64): relative L2 error of the spectral fields ≤ 1e-12 after 100 steps of the 64³
decaying case, and equal tracer cell indices. The FP32-mixed form is held to a short-time field
error and to per-shell spectrum errors of at most 1e-5, each against the FP64 oracle.
"""
import math

import numpy as np
import pytest

import gbght
from gbght import seed as S
from oracle import gbght_oracle as O
from pairs import advance_both, compare, make_case, rel_l2

pytestmark = pytest.mark.gpu


def test_decaying_64_cubed_100_steps(cuda_library):
    # the CPU-runnable case: 64³, ν = κ = 0.01, Sc = 1, unforced, IF-RK4, Δt = 0.005, 100 steps,
    # k⁴ seed spectrum, k = 0.5, ⟨φ²⟩ = 0.5, 4096 tracers
    run, orun = make_case(64, viscosity=0.01, tracers=4096, library=cuda_library)
    advance_both(run, orun, 100, dt=0.005)
    res = compare(run, orun, tol=1e-12)
    assert res["X_err"] < 1e-10
    F, t = run.tracer_sample()
    assert t == pytest.approx(orun.time, rel=0, abs=0)
    assert np.max(np.abs(F - orun.f0)) < 1e-10


@pytest.mark.parametrize("N,steps", [(32, 20), (48, 5), (12, 10), (16, 10), (8, 10), (24, 10)])
def test_forced_with_mean_gradient_cfl(cuda_library, N, steps):
    run, orun = make_case(N, viscosity=0.01, forcing=0.1, G=(1.0, 0.0, 0.0), tracers=256, library=cuda_library)
    taken = advance_both(run, orun, steps, dt=None)
    for d_lib, d_ora in taken:
        assert d_lib == pytest.approx(d_ora, rel=1e-12)
    compare(run, orun, tol=1e-12)


def test_rk3_velocity_only(cuda_library):
    run, orun = make_case(32, scalar=False, forcing=0.2, scheme="IFLowStorageRK3", library=cuda_library)
    advance_both(run, orun, 10, dt=0.01)
    compare(run, orun, tol=1e-12)


def test_larger_grids_short(cuda_library):
    for N in (96, 128):
        run, orun = make_case(N, viscosity=0.005, forcing=0.1, G=(1.0, 0.0, 0.0), tracers=1000, library=cuda_library)
        advance_both(run, orun, 2, dt=0.002)
        compare(run, orun, tol=1e-12)


@pytest.mark.parametrize("N,precision", [(192, "fp64"), (256, "fp64"), (256, "fp32_mixed"), (384, "fp64")])
def test_production_paths_one_step(cuda_library, N, precision):
    # The paths the 512³ benchmark runs, on radix-3 plans (192 = 8·3·8, 384 = 8·2·3·8) and on
    # 256 = 8·4·8:
    # - TMEM-resident z rows;
    # - the FP64 turnaround with the φ lines transformed aside;
    # - the FP32 occupancy of the y and z passes;
    # - the traversal sort.
    run, orun = make_case(N, viscosity=0.005, forcing=0.1, G=(1.0, 0.0, 0.0), tracers=2000, precision=precision,
                          library=cuda_library)
    advance_both(run, orun, 1, dt=0.002)
    if precision == "fp64":
        res = compare(run, orun, tol=1e-12)
        assert res["X_err"] < 1e-10
    else:
        compare(run, orun, tol=1e-5, check_tracers=False)


@pytest.mark.parametrize("N,precision,steps", [(64, "fp64", 20), (256, "fp64", 1), (64, "fp32_mixed", 10)])
def test_linear_forcing_both_fields(cuda_library, N, precision, steps):
    # Linear on the velocity (shells 1–2) and on the scalar (shells 2–Inf): the steady rate in the
    # integrating factor of both fields' epilogues, beside the mean gradient and the tracers
    run, orun = make_case(N, viscosity=0.005, forcing=gbght.Linear(0.7), scalar_forcing=gbght.Linear(0.4, 2, math.inf),
                          G=(0.0, 1.0, 0.0), tracers=1000, precision=precision, library=cuda_library)
    advance_both(run, orun, steps, dt=0.004)
    if precision == "fp64":
        res = compare(run, orun, tol=1e-12)
        assert res["X_err"] < 1e-10
    else:
        compare(run, orun, tol=1e-5, check_tracers=False)


BAND_FORCINGS = {
    "controller_u+cp_phi": (gbght.VarianceController(0.4, turnover_time=0.5, gain=2.0), gbght.ConstantPower(0.2)),
    "cp_u+controller_phi": (gbght.ConstantPower(0.1),
                            gbght.VarianceController(0.3, turnover_time=0.5, gain=1.0, highest_shell=3)),
    "rescale_total_u+band_phi": (gbght.VarianceRescaling(0.45, "total"), gbght.VarianceRescaling(0.2, "band", 1, math.inf)),
}


@pytest.mark.parametrize("name", list(BAND_FORCINGS))
@pytest.mark.parametrize("N,precision,steps", [(64, "fp64", 10), (256, "fp64", 1), (64, "fp32_mixed", 5)])
def test_band_forcings_both_fields(cuda_library, name, N, precision, steps):
    # per-stage amplitudes (ConstantPower, VarianceController) and the post-step rescale
    # (VarianceRescaling) on each field, with the mean gradient and the tracers
    vf, sf = BAND_FORCINGS[name]
    run, orun = make_case(N, viscosity=0.005, forcing=vf, scalar_forcing=sf, G=(1.0, 0.0, 0.0), tracers=1000,
                          precision=precision, library=cuda_library)
    advance_both(run, orun, steps, dt=0.004)
    if precision == "fp64":
        res = compare(run, orun, tol=1e-12)
        assert res["X_err"] < 1e-10
    else:
        compare(run, orun, tol=1e-5, check_tracers=False)


@pytest.mark.parametrize("scheme", ["IFHeun", "IFSSPRK3"])
@pytest.mark.parametrize("N,precision,steps", [(64, "fp64", 10), (256, "fp64", 1), (64, "fp32_mixed", 5)])
def test_heun_and_ssprk3(cuda_library, scheme, N, precision, steps):
    # the two schemes outside the low-storage loop: ConstantPower on the velocity, Linear on the
    # scalar, G, CFL steps at the schemes' own ceilings, tracers
    run, orun = make_case(N, viscosity=0.005, forcing=0.1, scalar_forcing=gbght.Linear(0.3), G=(1.0, 0.0, 0.0),
                          tracers=1000, scheme=scheme, cfl=0.25, precision=precision, library=cuda_library)
    taken = advance_both(run, orun, steps, dt=None)
    if precision == "fp64":
        for d_lib, d_ora in taken:
            assert d_lib == pytest.approx(d_ora, rel=1e-12)
        res = compare(run, orun, tol=1e-12)
        assert res["X_err"] < 1e-10
    else:
        compare(run, orun, tol=1e-5, check_tracers=False)


@pytest.mark.parametrize("scheme,shortened", [(("AB", 4), False), (("ABM", 3), True), (("AB", 8), True)])
def test_adams_particle_schemes(cuda_library, scheme, shortened):
    # AB(k)/ABM(k) tracers on a forced 64³ run: the trail fills through the lower ABM members and,
    # when shortened, the first steps follow the start-up bound; positions and samples match
    run, orun = make_case(64, forcing=0.1, tracers=3000, tracer_scheme=scheme, shortened_first_steps=shortened,
                          library=cuda_library)
    taken = advance_both(run, orun, 10, dt=None)
    for d_lib, d_ora in taken:
        assert d_lib == pytest.approx(d_ora, rel=1e-12)
    res = compare(run, orun, tol=1e-12)
    assert res["X_err"] < 1e-10
    F, t = run.tracer_sample()
    assert t == pytest.approx(orun.time, rel=1e-12)   # the sum of CFL steps equal to 1e-12
    assert np.max(np.abs(F - orun.f0)) < 1e-10


@pytest.mark.parametrize("N,precision", [(64, "fp64"), (128, "fp64"), (64, "fp32_mixed")])
def test_energy_below_scale(cuda_library, N, precision):
    # kinetic_energy_and_dissipation_below_scale against the oracle's sums
    run, orun = make_case(N, viscosity=0.01, energy=1.5, forcing=0.1, precision=precision, library=cuda_library)
    advance_both(run, orun, 2, dt=0.004)
    scales, k, eps = run.energy_below_scale()
    s_o, k_o, e_o = O.energy_below_scale(orun.dom, orun.state.uh, 0.01)
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert np.array_equal(scales, s_o)
    assert np.allclose(k, k_o, rtol=tol, atol=0) and np.allclose(eps, e_o, rtol=tol, atol=0)
    assert np.all(np.diff(k) >= 0) and k[-1] == pytest.approx(run.observables()["kinetic_energy"], rel=1e-12)


@pytest.mark.parametrize("N,precision", [(64, "fp64"), (192, "fp64"), (64, "fp32_mixed")])
def test_derivative_skewness(cuda_library, N, precision):
    run, orun = make_case(N, viscosity=0.005, forcing=0.1, tracers=500, precision=precision, library=cuda_library)
    advance_both(run, orun, 2, dt=0.004)
    sk = run.derivative_skewness()
    assert sk == pytest.approx(O.derivative_skewness(orun.dom, orun.state.uh), rel=1e-12 if precision == "fp64" else 1e-4)
    if precision == "fp64":   # the diagnostic leaves the run as it was
        advance_both(run, orun, 1, dt=0.004)
        compare(run, orun, tol=1e-12)


def test_rescaling_holds_the_target_exactly(cuda_library):
    run, _ = make_case(64, forcing=gbght.VarianceRescaling(0.45, "total"),
                       scalar_forcing=gbght.VarianceRescaling(0.6, "total", 1, math.inf), library=cuda_library)
    for _ in range(3):
        run.advance(0.005)
        ob = run.observables()
        assert ob["kinetic_energy"] == pytest.approx(0.45, rel=1e-13)
        assert ob["scalar_variance"] == pytest.approx(0.6, rel=1e-13)


def test_scalar_linear_exact_growth_with_zero_velocity(cuda_library):
    # test/forcing.jl:124-139 held to the closed form φ̂(T) = exp((A·band − ϰ|κ|²)T) φ̂(0)
    N, nu, Sc, A = 32, 0.05, 1.0, 1.0
    band = O.band_indicator(O.Domain(N), O.Linear(A))
    ph0 = S.seed_scalar(N, 0.1, seed=9) * (band + 0.1 * (1 - band))
    run = gbght.simulation(gbght.Setup(grid_points_per_axis=N, viscosity=nu, schmidt=Sc, scalar_forcing=gbght.Linear(A)),
                           np.zeros((3, N, N, N // 2 + 1), complex), ph0, library=cuda_library)
    for _ in range(40):
        run.advance(0.01)
    _, pe = run.export_state()
    expected = ph0 * np.exp((A * band - (nu / Sc) * S.wavenumbers(N)[3]) * 0.4)
    assert rel_l2(pe, expected) < 1e-12
    assert run.observables()["scalar_variance"] > O.scalar_variance(O.Domain(N), ph0)


def test_observables_spectra_speed(cuda_library):
    run, orun = make_case(64, forcing=0.1, library=cuda_library)
    advance_both(run, orun, 3, dt=0.005)
    ob = run.observables()
    d, st = orun.dom, orun.state
    assert ob["kinetic_energy"] == pytest.approx(O.kinetic_energy(d, st.uh), rel=1e-12)
    assert ob["dissipation"] == pytest.approx(O.dissipation(d, st.uh, 0.01), rel=1e-12)
    assert ob["scalar_variance"] == pytest.approx(O.scalar_variance(d, st.phih), rel=1e-12)
    assert ob["scalar_dissipation"] == pytest.approx(O.scalar_dissipation(d, st.phih, 0.01), rel=1e-12)
    assert np.allclose(run.energy_spectrum(), O.energy_spectrum(d, st.uh), rtol=1e-11, atol=1e-18)
    assert np.allclose(run.scalar_spectrum(), O.scalar_spectrum(d, st.phih), rtol=1e-11, atol=1e-18)
    assert run.max_speed() == pytest.approx(orun.speed, rel=1e-12)
    assert np.max(np.abs(run.velocity_physical() - orun.u)) < 1e-12


def test_exact_diffusion_with_zero_velocity(cuda_library):
    # test/scalar.jl:42-60: φ̂(T) = exp(−ϰ|κ|²T) φ̂(0) to round-off
    N, nu, Sc = 32, 0.1, 0.7
    ph0 = S.seed_scalar(N, 1.0, seed=3)
    run = gbght.simulation(gbght.Setup(grid_points_per_axis=N, viscosity=nu, schmidt=Sc),
                           np.zeros((3, N, N, N // 2 + 1), complex), ph0, library=cuda_library)
    for _ in range(25):
        run.advance(0.02)
    _, pe = run.export_state()
    expected = ph0 * np.exp(-(nu / Sc) * S.wavenumbers(N)[3] * 0.5)
    assert rel_l2(pe, expected) < 1e-10


def test_planted_reality_violation_removed(cuda_library):
    N = 32
    uh = S.seed_velocity(N, 0.5, seed=1)
    ph = S.seed_scalar(N, 0.5, seed=2)
    d = 2e-6 * np.max(np.abs(uh[:, :, :, 0]))
    uh[:, 0, 1, 0] += 1j * d
    uh[:, 0, N - 1, 0] += 1j * d
    ph[0, 1, 0] += 1j * d
    ph[0, N - 1, 0] += 1j * d
    run, _ = make_case(N, forcing=0.1, uh=uh, ph=ph, library=cuda_library)
    run.advance(0.01)
    ue, pe = run.export_state()
    neg = (-np.arange(N)) % N
    for f in (ue, pe):
        plane = f[..., 0]
        assert np.max(np.abs(plane - np.conj(plane[..., neg, :][..., :, neg]))) == 0.0


def test_separate_calls_equal_advance(cuda_library):
    a, _ = make_case(32, forcing=0.1, tracers=500, library=cuda_library)
    b, _ = make_case(32, forcing=0.1, tracers=500, library=cuda_library)
    a.advance(0.01)
    b.step(0.01)
    b.deposit()
    b.advect(0.01)
    b.deposit_tracers(0.01)
    ua, pa = a.export_state()
    ub, pb = b.export_state()
    assert np.array_equal(ua, ub) and np.array_equal(pa, pb)
    assert np.array_equal(a.tracers(), b.tracers())


def test_traversal_order_does_not_change_results(cuda_library):
    # The tracer pass visits tracers tile by tile (the traversal sort). Handing the same tracers in
    # another order must give the same positions and samples, permuted alike: bitwise.
    N, M = 64, 3000
    uh = S.seed_velocity(N, 0.5, seed=3)
    ph = S.seed_scalar(N, 0.5, seed=4)
    X = S.seed_tracers(M, seed=5)
    perm = np.random.default_rng(6).permutation(M)
    setup = gbght.Setup(grid_points_per_axis=N, viscosity=0.01, tracers=M)
    a = gbght.simulation(setup, uh, ph, X, library=cuda_library)
    b = gbght.simulation(setup, uh, ph, np.ascontiguousarray(X[:, perm]), library=cuda_library)
    for _ in range(3):
        assert a.advance(0.005) == b.advance(0.005)
    assert np.array_equal(a.tracers()[:, perm], b.tracers())
    Fa, ta = a.tracer_sample()
    Fb, tb = b.tracer_sample()
    assert ta == tb and np.array_equal(Fa[:, perm], Fb)


def test_nonfinite_state_trips_the_guard(cuda_library):
    N = 32
    uh = S.seed_velocity(N, 0.5, seed=0)
    uh[0, 0, 1, 1] = complex(np.nan, 0.0)
    run, _ = make_case(N, uh=uh, tracers=10, library=cuda_library)
    with pytest.raises(gbght.ScheduleError, match="blown up"):
        run.advance(0.01)


def test_nonfinite_scalar_is_a_blow_up(cuda_library):
    # A non-finite scalar is a blow-up. The x pass packs n_z and uφ into one complex line, so
    # within the step it also reaches the velocity, and the velocity guard (checked first) names it.
    N = 32
    ph = S.seed_scalar(N, 0.5, seed=1)
    ph[1, 1, 1] = complex(np.inf, 0.0)
    run, _ = make_case(N, ph=ph, library=cuda_library)
    with pytest.raises(gbght.ScheduleError, match="blown up"):
        run.advance(0.01)


def test_fp32_mixed_short_time_error(cuda_library):
    # FP32 transforms, products and updates; FP64 integrating factor, forcing normalisation,
    # spectra and tracer positions. Short-time field error and spectra against the FP64 oracle.
    run, orun = make_case(64, forcing=0.1, G=(1.0, 0.0, 0.0), precision="fp32_mixed", tracers=1000,
                          library=cuda_library)
    advance_both(run, orun, 10, dt=0.005)
    ue, pe = run.export_state()
    assert rel_l2(ue, orun.state.uh) < 1e-5
    assert rel_l2(pe, orun.state.phih) < 1e-5
    for got, want in ((run.energy_spectrum(), O.energy_spectrum(orun.dom, orun.state.uh)),
                      (run.scalar_spectrum(), O.scalar_spectrum(orun.dom, orun.state.phih))):
        live = want > 1e-6 * want.max()
        assert np.max(np.abs(got[live] - want[live]) / want[live]) < 1e-5


def test_full_size_512_cubed_properties(cuda_library):
    # The benchmark's 512³ workload (ConstantPower on shells 1–2, G along x, tracers), two CFL steps
    # in each precision form, held to properties that do not depend on the size:
    # - the state stays solenoidal and its kx = 0 plane exactly Hermitian;
    # - the observables and the spectrum agree with sums over the exported state (Parseval);
    # - the deposited max speed is the max over the exported physical velocity;
    # - the FP32-mixed spectra stay within 1e-5 of the FP64 ones on every live shell.
    N, M = 512, 100_000
    uh0 = S.seed_velocity(N, 0.5, seed=0)
    ph0 = S.seed_scalar(N, 0.5, seed=1)
    X0 = S.seed_tracers(M, seed=2)
    spectra = {}
    for precision in ("fp64", "fp32_mixed"):
        setup = gbght.Setup(grid_points_per_axis=N, viscosity=8.5e-4, velocity_forcing=gbght.ConstantPower(0.1),
                            mean_gradient=(1.0, 0.0, 0.0), tracers=M, precision=precision)
        run = gbght.simulation(setup, uh0, ph0, X0, library=cuda_library)
        for _ in range(2):
            run.advance(None)
        spectra[precision] = (run.energy_spectrum(), run.scalar_spectrum())
        if precision == "fp64":
            ue, pe = run.export_state()
            kx, ky, kz, k2 = S.wavenumbers(N)
            num, den = 0.0, 0.0
            for z in range(0, N, 64):   # |κ·û| against |κ||û|, in slabs
                sl = slice(z, z + 64)
                div = (kx * ue[0, sl] + ky * ue[1, sl]) + kz[sl] * ue[2, sl]
                num += float(np.sum(np.abs(div) ** 2))
                den += float(np.sum(k2[sl] * (np.abs(ue[0, sl]) ** 2 + np.abs(ue[1, sl]) ** 2 + np.abs(ue[2, sl]) ** 2)))
            assert math.sqrt(num / den) < 1e-13
            neg = (-np.arange(N)) % N
            for f in (ue, pe):
                plane = f[..., 0]
                assert np.max(np.abs(plane - np.conj(plane[..., neg, :][..., :, neg]))) == 0.0
            w = np.full(N // 2 + 1, 2.0)
            w[0] = 1.0
            w[N // 2] = 1.0
            n6 = float(N) ** 6
            k_host = sum(float(np.sum((np.abs(ue[c]) ** 2) * w)) for c in range(3)) / n6 / 2
            var_host = float(np.sum((np.abs(pe) ** 2) * w)) / n6
            ob = run.observables()
            assert ob["kinetic_energy"] == pytest.approx(k_host, rel=1e-12)
            assert ob["scalar_variance"] == pytest.approx(var_host, rel=1e-12)
            E, P = spectra[precision]
            assert float(E.sum()) == pytest.approx(ob["kinetic_energy"], rel=1e-12)   # Δκ = 1 at L = 2π
            assert float(P.sum()) == pytest.approx(ob["scalar_variance"], rel=1e-12)
            del ue, pe
            u = run.velocity_physical()
            speed = math.sqrt(float(np.max(u[0] * u[0] + u[1] * u[1] + u[2] * u[2])))
            assert run.max_speed() == pytest.approx(speed, rel=1e-14)
            del u
        run.close()
    for i in (0, 1):
        ref, got = spectra["fp64"][i], spectra["fp32_mixed"][i]
        live = ref > 1e-6 * ref.max()
        assert np.max(np.abs(got[live] - ref[live]) / ref[live]) < 1e-5


def test_ensemble_graph_equals_separate_runs(cuda_library):
    # one captured CUDA graph over members of uneven sizes, schemes and forcings (each on its own
    # stream), replayed: bitwise the runs stepped alone
    def members():
        return [make_case(32, forcing=0.1, library=cuda_library)[0],
                make_case(48, scalar=False, scheme="IFLowStorageRK3", library=cuda_library)[0],
                make_case(64, forcing=gbght.Linear(0.3), scheme="IFSSPRK3", library=cuda_library)[0],
                make_case(64, forcing=0.1, precision="fp32_mixed", library=cuda_library)[0]]
    ens_runs, alone = members(), members()
    ens = gbght.Ensemble(ens_runs)
    for k in range(4):
        dt = 0.004 if k < 3 else 0.003   # a new dt captures a new graph
        ens.step(dt)
        for r in alone:
            r.step(dt)
            r.deposit()
    for a, b in zip(ens_runs, alone):
        ua, pa = a.export_state()
        ub, pb = b.export_state()
        assert np.array_equal(ua, ub) and (pa is None or np.array_equal(pa, pb))
        assert a.max_speed() == b.max_speed()
    ens.close()


def test_ensemble_of_uneven_grids_throughput(cuda_library):
    # 96 FP32-mixed members, 32 each of 32³, 48³ and 64³, ν drawn per member from a seed: the
    # graph-replayed ensemble step against stepping the members one by one
    import time
    rng = np.random.default_rng(7)
    runs = []
    for i, N in enumerate([32] * 32 + [48] * 32 + [64] * 32):
        nu = float(rng.uniform(0.005, 0.02))
        runs.append(make_case(N, viscosity=nu, forcing=0.1, precision="fp32_mixed", seeds=(i, i + 1000, i + 2000),
                              library=cuda_library)[0])
    ens = gbght.Ensemble(runs)
    ens.step(0.002)          # capture
    K = 20
    runs[0].synchronize()
    t0 = time.perf_counter()
    for _ in range(K):
        ens.step(0.002)
    t_graph = time.perf_counter() - t0
    t0 = time.perf_counter()
    for _ in range(K):
        for r in runs:
            r.step(0.002)
            r.deposit()
    t_seq = time.perf_counter() - t0
    pts = sum(r.N ** 3 for r in runs)
    print(f"\nensemble 96 members (32x 32^3, 48^3, 64^3), FP32-mixed, IF-RK4: graph {K * 96 / t_graph:.0f} "
          f"member-steps/s ({5 * pts * K / t_graph:.3e} grid-point-stages/s), one by one "
          f"{K * 96 / t_seq:.0f} member-steps/s, ratio {t_seq / t_graph:.2f}")
    assert t_graph < t_seq
    ens.close()
