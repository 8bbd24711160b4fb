"""The benchmark's configurations against the oracle, the boundary's device-memory route, the
checkpoint's bitwise continuation and the bounded waits' failure path, on the GPU through the C ABI.

- The headline 512³ FP64 form: one whole iteration (`advance!`) of the 512³ forced workload with
  10⁶ tracers against the oracle, relative L2 ≤ 1e-12 and equal tracer cells.
- The 256³ forced configuration (ν = ϰ = 2.1e-3, ConstantPower ε = 0.1 on shells 1–2, G = 1 along x,
  CFL 0.5, 10⁵ tracers): FP64 against the oracle for 10 steps at ≤ 1e-12; the FP32-mixed form's
  short-time field error against the same oracle trajectory at ≤ 1e-5; and its long-time spectra
  against the FP64 form's over 500 steps, compared window by window within the windows' sampling
  error (the trajectories decorrelate, so only the statistics can agree).
"""
import math

import numpy as np
import pytest

import gbght
from gbght import seed as S
from oracle import gbght_oracle as O
from pairs import compare, make_case, rel_l2

pytestmark = pytest.mark.gpu

C1 = dict(viscosity=2.1e-3, forcing=0.1, G=(1.0, 0.0, 0.0), cfl=0.5)


def test_expired_device_wait_is_a_device_error(cuda_library):
    # a barrier armed for a copy that is never issued, waited on for at most 20000 cycles: the wait
    # expires, raises the status bit and returns; the run then keeps stepping
    run, orun = make_case(32, forcing=0.1, tracers=64, library=cuda_library)
    with pytest.raises(gbght.DeviceError, match="bounded wait"):
        run.selftest_wait_timeout(20000)
    assert run.status_word() & 0x4
    assert run.status_word() == 0
    for _ in range(3):
        run.advance(0.01)
        orun.advance(0.01)
    compare(run, orun, tol=1e-12)


@pytest.mark.parametrize("precision,tracer_scheme", [("fp64", ("Heun", 1)), ("fp64", ("AB", 3)),
                                                     ("fp32_mixed", ("ABM", 2))])
def test_checkpoint_continues_bitwise(cuda_library, precision, tracer_scheme):
    # test/hdf5_checkpoint.jl:112-116: a run restored from a checkpoint (state, positions, the
    # trail, the clock) continues the checkpointed one bit for bit
    from checkpoint import continuation_is_bitwise
    N, M = 64, 2000
    setup = gbght.Setup(grid_points_per_axis=N, viscosity=0.005, velocity_forcing=gbght.ConstantPower(0.1),
                        mean_gradient=(1.0, 0.0, 0.0), tracers=M, precision=precision,
                        tracer_scheme=tracer_scheme[0], tracer_steps=tracer_scheme[1])
    continuation_is_bitwise(setup, S.seed_velocity(N, 0.5, seed=0), S.seed_scalar(N, 0.5, seed=1),
                            S.seed_tracers(M, seed=2), before=5, after=5, library=cuda_library)


@pytest.mark.parametrize("precision", ["fp64", "fp32_mixed"])
def test_device_memory_state_and_tracers(cuda_library, precision):
    # the state and the positions handed over as CUDA tensors (a CuArray's role) are read and
    # written in place by the library, bit for bit as the host route
    import torch
    N, M = 64, 1000
    uh, ph, X = S.seed_velocity(N, 0.5, seed=7), S.seed_scalar(N, 0.5, seed=8), S.seed_tracers(M, seed=9)
    setup = gbght.Setup(grid_points_per_axis=N, viscosity=0.01, velocity_forcing=gbght.ConstantPower(0.1),
                        mean_gradient=(0.0, 1.0, 0.0), tracers=M, precision=precision)
    host = gbght.simulation(setup, uh, ph, X, library=cuda_library)
    dev = gbght.Run(setup, library=cuda_library)
    dev.import_state(torch.from_numpy(uh).cuda(), torch.from_numpy(ph).cuda())
    dev.deposit()
    dev.import_tracers(torch.from_numpy(X).cuda())
    dev.deposit_tracers(0.0)
    for _ in range(3):
        host.advance(None)
        dev.advance(None)
    u_h, p_h = host.export_state()
    du = torch.full((3, N, N, N // 2 + 1), complex(math.nan, math.nan), dtype=torch.complex128, device="cuda")
    dp = torch.full((N, N, N // 2 + 1), complex(math.nan, math.nan), dtype=torch.complex128, device="cuda")
    dev.export_state(out=(du, dp))
    torch.cuda.synchronize()
    assert np.array_equal(du.cpu().numpy(), u_h) and np.array_equal(dp.cpu().numpy(), p_h)
    dX = torch.zeros((3, M), dtype=torch.float64, device="cuda")
    dev.tracers(out=dX)
    torch.cuda.synchronize()
    assert np.array_equal(dX.cpu().numpy(), host.tracers())
    # a state outside the retained ball is refused from device memory too, leaving the run as it was
    bad = torch.from_numpy(uh).cuda()
    bad[0, N // 2 - 1, 1, N // 2] = 1.0
    with pytest.raises(ValueError, match="outside the retained"):
        dev.import_state(bad, torch.from_numpy(ph).cuda())
    u_d, _ = dev.export_state()
    assert np.array_equal(u_d, u_h)


def test_headline_512_cubed_one_iteration_against_the_oracle(cuda_library):
    # the benchmark's workload: 512³, ν = ϰ = 8.5e-4, ConstantPower ε = 0.1 on shells 1–2, G = 1
    # along x, 10⁶ tracers, IF-RK4 at CFL 0.5; one advance! on each side
    run, orun = make_case(512, viscosity=8.5e-4, forcing=0.1, G=(1.0, 0.0, 0.0), tracers=1_000_000, cfl=0.5,
                          library=cuda_library)
    d_lib = run.advance(None)
    d_ora = orun.advance(None)
    assert d_lib == pytest.approx(d_ora, rel=1e-12)
    res = compare(run, orun, tol=1e-12)
    assert res["X_err"] < 1e-10
    print(f"512^3 FP64 one iteration vs oracle: u {res['u']:.2e} phi {res['phi']:.2e} X {res['X_err']:.2e}")


def _spectra_err(run, E, P):
    e, p = run.energy_spectrum(), run.scalar_spectrum()
    live, livep = E > 1e-6 * E.max(), P > 1e-6 * P.max()
    return (float(np.max(np.abs(e[live] - E[live]) / E[live])), float(np.max(np.abs(p[livep] - P[livep]) / P[livep])))


def test_c1_256_cubed_fp64_and_fp32_short_time_against_the_oracle(cuda_library):
    N, M, steps = 256, 100_000, 10
    run, orun = make_case(N, tracers=M, library=cuda_library, **C1)
    setup32 = gbght.Setup(grid_points_per_axis=N, viscosity=C1["viscosity"], velocity_forcing=gbght.ConstantPower(0.1),
                          mean_gradient=C1["G"], tracers=M, cfl=C1["cfl"], precision="fp32_mixed")
    uh, ph, X = S.seed_velocity(N, 0.5, seed=0), S.seed_scalar(N, 0.5, seed=1), S.seed_tracers(M, seed=2)
    run32 = gbght.simulation(setup32, uh, ph, X, library=cuda_library)
    for _ in range(steps):
        d_ora = orun.advance(None)
        assert run.advance(None) == pytest.approx(d_ora, rel=1e-12)
        run32.advance(d_ora)   # the oracle's Δt sequence, so the comparison is of the fields alone
    res = compare(run, orun, tol=1e-12)
    assert res["X_err"] < 1e-10
    u32, p32 = run32.export_state()
    eu, ep = rel_l2(u32, orun.state.uh), rel_l2(p32, orun.state.phih)
    E, P = O.energy_spectrum(orun.dom, orun.state.uh), O.scalar_spectrum(orun.dom, orun.state.phih)
    se, sp = _spectra_err(run32, E, P)
    ex = float(np.max(np.abs(run32.tracers() - orun.X)))
    print(f"C1 256^3 after {steps} steps: FP64 u {res['u']:.2e} phi {res['phi']:.2e}; FP32-mixed u {eu:.2e} "
          f"phi {ep:.2e} E(k) {se:.2e} E_phi(k) {sp:.2e} X {ex:.2e}")
    assert eu <= 1e-5 and ep <= 1e-5
    assert se <= 1e-5 and sp <= 1e-5


def windowed_spectra(run, steps, burn, window, batch):
    """Per window of `window` steps after `burn`: the mean E(κ), E_φ(κ) over its steps and the
    standard error of that mean from `window // batch` batch means."""
    Es, Ps = [], []
    for k in range(steps):
        run.advance(None)
        if k >= burn:
            Es.append(run.energy_spectrum())
            Ps.append(run.scalar_spectrum())
    out = []
    for w0 in range(0, len(Es) - window + 1, window):
        res = []
        for series in (np.array(Es[w0:w0 + window]), np.array(Ps[w0:w0 + window])):
            b = series.reshape(window // batch, batch, -1).mean(axis=1)
            res.append((series.mean(axis=0), b.std(axis=0, ddof=1) / math.sqrt(b.shape[0])))
        out.append(res)
    return out


def test_c1_fp32_long_time_spectra_within_sampling_error(cuda_library):
    # 500 steps of the 256³ configuration in both forms, each at its own CFL Δt; after 100 steps,
    # four windows of 100 steps. Per window and live shell, the FP32-mixed mean spectrum must lie
    # within three standard errors (the two forms' batch-mean errors combined) of the FP64 mean,
    # or within 1e-5 of it.
    N, M = 256, 100_000
    uh, ph, X = S.seed_velocity(N, 0.5, seed=0), S.seed_scalar(N, 0.5, seed=1), S.seed_tracers(M, seed=2)
    wins = {}
    for form in ("fp64", "fp32_mixed"):
        setup = gbght.Setup(grid_points_per_axis=N, viscosity=C1["viscosity"], velocity_forcing=gbght.ConstantPower(0.1),
                            mean_gradient=C1["G"], tracers=M, cfl=C1["cfl"], precision=form)
        run = gbght.simulation(setup, uh, ph, X, library=cuda_library)
        wins[form] = windowed_spectra(run, 500, 100, 100, 20)
        run.close()
    worst = []
    for w64, w32 in zip(wins["fp64"], wins["fp32_mixed"]):
        for (m64, s64), (m32, s32) in zip(w64, w32):
            live = m64 > 1e-6 * m64.max()
            z = np.abs(m32 - m64)[live] / np.maximum(3 * np.hypot(s64, s32)[live], 1e-5 * m64[live])
            worst.append((float(z.max()), float(np.max(np.abs(m32 - m64)[live] / m64[live]))))
    print("C1 windows (max |diff|/(3 se), max rel diff), E then E_phi per window:", worst)
    assert all(z <= 1.0 for z, _ in worst)
