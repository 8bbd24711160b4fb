"""Benchmark: 512³ forced velocity + scalar IF-RK4 steps/s on one B200 (replicas on N GPUs).

Workload (the headline configuration): a 512³ periodic box, ν = ϰ = 8.5e-4 (Sc = 1),
ConstantPower forcing ε = 0.1 on shells 1–2 (|k| ≤ 2.5), uniform mean scalar gradient G = 1
along x, 10⁶ uniform-random tracers advected by Heun with Catmull–Rom interpolation, IF-RK4 at
CFL 0.5. Synthetic seeded start: k⁴exp(−2(k/4)²) spectrum, k = 0.5, ⟨φ²⟩ = 0.5. A step is one
full iteration of the run layer (`advance!`): the 5-stage field step, the closing deposit, the
tracer push and particle deposit, and the blow-up guards.

`value` is steps/s of the plain FP64 form with the state resident in HBM, timed with CUDA events
on the library's own stream. The FP32-mixed form is measured on the same workload and reported
beside it. `e2e` is timed through the public API from pinned host buffers: the state upload, the
K steps and the state download. Under torchrun every rank runs its own replica (the path does
not shard), and the timed region is the max over ranks.

--impl reference times the CPU restatement of the reference's step (NumPy + scipy.fft on all host
cores) on the same workload: whole iterations of its run layer (step, deposit, tracer push and
particle deposit, guards), as many as fit a time budget and at least one, and beside them one
iteration each at 64³ and 256³.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "gbghomogeneousturbulence.jl_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "512³ IF-RK4 steps/s, FP32-mixed vs FP64 on one B200 at ≤1e-5 spectrum err"
WORKLOAD = dict(N=512, viscosity=8.5e-4, schmidt=1.0, injection_rate=0.1, shells=(1, 2), G=(1.0, 0.0, 0.0),
                tracers=1_000_000, cfl=0.5, scheme="IFLowStorageRK4")
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
# DRAM traffic per launch over algorithmic bytes (dram__bytes_read + dram__bytes_write of one ncu
# capture of the kernel at 256³, one launch, over the launch's algorithmic bytes), applied to the
# 512³ launch: the kernel's traffic scales with the tiles it processes.
TRAFFIC_RATIO = {("x_products", "fp64"): 1.141 / 1.171, ("x_products", "fp32_mixed"): 0.596 / 0.586}
FALLBACK_HBM = 6650.0


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def max_over_ranks(x, device="cpu"):
    """The largest of x over the ranks of the process group (x itself without one). Every rank
    calls it, in the same order, so the collective steps match across ranks."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return float(x)
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_rate(world_size, steps, slowest_s):
    """Whole-job steps/s of independent replicas: every rank runs `steps` steps of its own field,
    and the job takes as long as its slowest rank."""
    return world_size * steps / slowest_s


def _peaks():
    try:
        with open(PEAKS_FILE) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


SCHEME_NAME = {"IFLowStorageRK4": "IF-RK4", "IFLowStorageRK3": "IF-RK3", "IFHeun": "IFHeun", "IFSSPRK3": "IFSSPRK3"}
# the schemes' advective-CFL ceilings under the 2/3 rule (src/Propagator.jl:906-919)
SCHEME_CFL = {"IFLowStorageRK4": 0.96, "IFLowStorageRK3": 0.5, "IFHeun": 0.25, "IFSSPRK3": 0.5}


def _cfl(args):
    """The workload's CFL number, lowered to the scheme's own ceiling where that is smaller."""
    return min(WORKLOAD["cfl"], SCHEME_CFL[args.scheme])


def _config(args, N):
    return {"workload": f"{N}^3 forced velocity+scalar {SCHEME_NAME[args.scheme]}, nu=kappa={WORKLOAD['viscosity']}, "
                        f"ConstantPower eps={WORKLOAD['injection_rate']} |k|<=2.5, G=1 along x, "
                        f"{args.tracers} Heun/Catmull-Rom tracers, CFL {_cfl(args)}",
            "grid": N, "tracers": args.tracers, "scheme": args.scheme, "dealiasing": "2/3 closed ball",
            "start": "seeded k^4 spectrum (synthetic), not a stationary state",
            "l2": "inputs larger than L2 (state alone >= 1.3 GB)",
            "parallelism": f"replicas x{args.gpus}"}


# ------------------------------------------------------------------------------------------------
# clocks sampled during the timed region
# ------------------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device, self.proc = device, None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.text = ""
        if self.proc is None:
            return
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out = ""
        self.text = out or ""

    def summary(self):
        rows = []
        for line in self.text.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        reasons = sorted({names[i] for _, _, r in rows for i, v in enumerate(r) if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": reasons, "samples": len(rows)}


# ------------------------------------------------------------------------------------------------
# our arm
# ------------------------------------------------------------------------------------------------
def algorithmic_bytes_per_step(N, K, w_complex, has_scalar=True):
    """Bytes each kernel kind must move per step (the pruned transform design: inputs plus
    outputs over the retained box, kx ∈ [0, K], ky', kz' ∈ [−K, K])."""
    KX1, NY2 = K + 1, 2 * K + 1
    S = 5
    ninv, nfwd = (7, 6) if has_scalar else (6, 3)
    b = {}
    # S stages of ninv slots, except the first stage's velocity slots, which reuse the closing
    # deposit's y-inverse of the previous step; plus that deposit (3 slots)
    b["y_inverse"] = ((S - 1) * ninv + (ninv - 3) + 3) * N * KX1 * (NY2 + N) * w_complex
    b["x_products"] = S * N * N * KX1 * (ninv + nfwd) * w_complex
    b["y_forward"] = S * nfwd * N * KX1 * (N + NY2) * w_complex
    nst = 4 if has_scalar else 3
    state_rw = (S * nst + (S - 1) * nst + S * nst + (S - 1) * nst) * NY2 * NY2 * KX1 * w_complex
    b["z_epilogue"] = S * (nfwd + ninv) * N * NY2 * KX1 * w_complex + state_rw
    b["x_velocity"] = 3 * N * N * KX1 * w_complex + 3 * N ** 3 * (w_complex // 2)
    return b


def launches_per_step(has_scalar=True, forced=True):
    return {"y_inverse": 6, "x_products": 5, "y_forward": 5, "z_epilogue": 5, "x_velocity": 1,
            "force_amp": 5 if forced else 0, "reality": 1, "tracers": 1, "observables": 1 if has_scalar else 0,
            "traversal": 3}


def make_inputs(N, M, seed_base=0):
    from gbght import seed as S
    uh = S.seed_velocity(N, 0.5, seed=seed_base + 0)
    ph = S.seed_scalar(N, 0.5, seed=seed_base + 1)
    X = S.seed_tracers(M, seed=seed_base + 2)
    return uh, ph, X


def pinned_like(a):
    """A NumPy view of pinned (page-locked) host memory holding a copy of `a`."""
    import torch
    t = torch.empty(a.nbytes, dtype=torch.uint8, pin_memory=True)
    v = t.numpy().view(a.dtype).reshape(a.shape)
    v[...] = a
    return v, t


def run_form(args, precision, device, inputs, timed=True):
    import gbght
    N, M = args.grid, args.tracers
    uh, ph, X = inputs
    setup = gbght.Setup(grid_points_per_axis=N, viscosity=WORKLOAD["viscosity"], schmidt=WORKLOAD["schmidt"],
                        velocity_forcing=gbght.ConstantPower(WORKLOAD["injection_rate"], *WORKLOAD["shells"]),
                        mean_gradient=WORKLOAD["G"], tracers=M, cfl=_cfl(args), scheme=args.scheme, precision=precision,
                        device=device)
    run = gbght.simulation(setup, uh, ph, X)
    for _ in range(args.warmup):
        run.advance(None)
    return run


def timed_steps(run, K, sampler=None):
    run.synchronize()
    run.profile(True)
    run.timer_start()
    for _ in range(K):
        run.advance(None)
    ms = run.timer_stop()
    prof = run.profile_read()
    run.profile(False)
    return ms, prof


def time_diagnostics(run):
    """The occasional diagnostics on the end state, outside the timed region: the time between CUDA
    events on the run's stream around one call each (the call's own host work included), and the
    values."""
    out = {}
    run.synchronize()
    run.timer_start()
    sk = run.derivative_skewness()
    out["derivative_skewness_ms"] = round(run.timer_stop(), 3)
    out["derivative_skewness"] = sk
    run.timer_start()
    _, k, _ = run.energy_below_scale()
    out["energy_below_scale_ms"] = round(run.timer_stop(), 3)
    out["energy_below_scale_k_at_dx"] = float(k[0])
    return out


def e2e_run(args, precision, device, inputs, K):
    """Through the public API from pinned host buffers: upload the state and tracers, K steps with
    their per-step host readbacks, download the final state."""
    import gbght
    N, M = args.grid, args.tracers
    uh, ph, X = inputs
    puh, t1 = pinned_like(uh)
    pph, t2 = pinned_like(ph)
    pX, t3 = pinned_like(X)
    out_u = np.empty_like(uh)
    out_p = np.empty_like(ph)
    pu, t4 = pinned_like(out_u)
    pp, t5 = pinned_like(out_p)
    setup = gbght.Setup(grid_points_per_axis=N, viscosity=WORKLOAD["viscosity"], schmidt=WORKLOAD["schmidt"],
                        velocity_forcing=gbght.ConstantPower(WORKLOAD["injection_rate"], *WORKLOAD["shells"]),
                        mean_gradient=WORKLOAD["G"], tracers=M, cfl=_cfl(args), scheme=args.scheme, precision=precision,
                        device=device)
    run = gbght.Run(setup)
    run.synchronize()
    t0 = time.perf_counter()
    run.import_state(puh, pph)
    run.deposit()
    run.import_tracers(pX)
    run.deposit_tracers(0.0)
    for _ in range(K):
        run.advance(None)
    u, p = run.export_state(out=(pu, pp))
    run.synchronize()
    el = time.perf_counter() - t0
    h2d = puh.nbytes + pph.nbytes + pX.nbytes + K * 8
    # per step: max|u| (8 B) and the scalar-variance guard (4 doubles per ky' row, read back)
    d2h = u.nbytes + p.nbytes + K * (8 + 4 * 8 * (2 * run.K + 1))
    run.close()
    return K / el, h2d / K, d2h / K


def adjoint_cost(args, device, inputs, reps=3):
    """The discrete adjoint's cost on the workload (FP64, no tracers): CUDA-event time of one
    gbght_adjoint_step (the step's stages run again, then reversed) against one field step
    (gbght_step + gbght_deposit), each the mean of `reps` after one untimed call."""
    import gbght
    N = args.grid
    uh, ph, _ = inputs
    setup = gbght.Setup(grid_points_per_axis=N, viscosity=WORKLOAD["viscosity"], schmidt=WORKLOAD["schmidt"],
                        velocity_forcing=gbght.ConstantPower(WORKLOAD["injection_rate"], *WORKLOAD["shells"]),
                        mean_gradient=WORKLOAD["G"], cfl=_cfl(args), scheme=args.scheme, device=device)
    if args.scheme not in ("IFLowStorageRK4", "IFLowStorageRK3"):
        return None
    run = gbght.simulation(setup, uh, ph)
    dt = run.cfl_timestep()
    run.adjoint_create(0)
    run.adjoint_import(uh, ph)

    def timed(fn):
        fn()
        run.synchronize()
        run.timer_start()
        for _ in range(reps):
            fn()
        return run.timer_stop() / reps

    def field_step():
        run.step(dt)
        run.deposit()
    fwd = timed(field_step)
    run.profile(True)
    adj = timed(lambda: run.adjoint_step(dt))
    prof = run.profile_read()
    run.profile(False)
    run.close()
    return {"forward_field_step_ms": round(fwd, 3), "adjoint_step_ms": round(adj, 3),
            "ratio": round(adj / fwd, 3), "form": "fp64", "grid": N,
            "kernels_per_adjoint_step_ms": {k: round(v[1] / (reps + 1), 3) for k, v in prof.items() if v[0]}}


def dealiasing_cost(args, device, inputs, reps=3):
    """The field step's cost under each dealiasing strategy on the workload (FP64 and FP32-mixed, no
    tracers): CUDA-event time of gbght_step + gbght_deposit, the mean of `reps` after one untimed
    step, with the per-kernel times of PhaseShift's step."""
    import gbght
    N = args.grid
    uh, ph, _ = inputs
    out = {}
    for precision in ("fp64", "fp32_mixed"):
        row = {}
        for dea in ("TwoThirds", "HouLi", "PhaseShift"):
            setup = gbght.Setup(grid_points_per_axis=N, viscosity=WORKLOAD["viscosity"], schmidt=WORKLOAD["schmidt"],
                                velocity_forcing=gbght.ConstantPower(WORKLOAD["injection_rate"], *WORKLOAD["shells"]),
                                mean_gradient=WORKLOAD["G"], cfl=_cfl(args), scheme=args.scheme, device=device,
                                precision=precision, dealiasing=dea)
            run = gbght.simulation(setup, uh, ph)
            dt = run.cfl_timestep()
            run.step(dt)
            run.deposit()
            run.synchronize()
            run.profile(True)
            run.timer_start()
            for _ in range(reps):
                run.step(dt)
                run.deposit()
            ms = run.timer_stop() / reps
            prof = run.profile_read()
            run.profile(False)
            run.close()
            row[dea] = {"field_step_ms": round(ms, 3)}
            if dea == "PhaseShift":
                row[dea]["kernels_ms_per_step"] = {k: round(v[1] / reps, 3) for k, v in prof.items() if v[0]}
        for dea in ("HouLi", "PhaseShift"):
            row[dea]["ratio_vs_two_thirds"] = round(row[dea]["field_step_ms"] / row["TwoThirds"]["field_step_ms"], 3)
        out[precision] = row
    return {"grid": N, "forms": out}


def c1_statistics(device, steps=500, burn=100, window=100, batch=20, short=20):
    """The 256³ forced configuration (ν = ϰ = 2.1e-3, ConstantPower ε = 0.1 on shells 1–2, G = 1,
    CFL 0.5, 10⁵ tracers) in both forms on the GPU: the FP32-mixed form's relative L2 field error
    against the FP64 form after `short` steps of the FP64 Δt sequence, and the long-time spectra
    over `steps` steps, each form at its own CFL Δt, compared window by window (mean E(κ), E_φ(κ)
    after `burn` steps, in windows of `window` steps, standard errors from batch means)."""
    import gbght
    N, M = 256, 100_000
    uh, ph, X = make_inputs(N, M, seed_base=0)

    def make(form):
        setup = gbght.Setup(grid_points_per_axis=N, viscosity=2.1e-3, velocity_forcing=gbght.ConstantPower(0.1),
                            mean_gradient=(1.0, 0.0, 0.0), tracers=M, cfl=0.5, precision=form, device=device)
        return gbght.simulation(setup, uh, ph, X)
    a, b = make("fp64"), make("fp32_mixed")
    for _ in range(short):
        b.advance(a.advance(None))
    ua, pa = a.export_state()
    ub, pb = b.export_state()
    out = {"short_steps": short,
           "field_rel_l2_u": float(np.linalg.norm(ub - ua) / np.linalg.norm(ua)),
           "field_rel_l2_phi": float(np.linalg.norm(pb - pa) / np.linalg.norm(pa))}
    a.close()
    b.close()
    wins = {}
    for form in ("fp64", "fp32_mixed"):
        run = make(form)
        Es, Ps = [], []
        for k in range(steps):
            run.advance(None)
            if k >= burn:
                Es.append(run.energy_spectrum())
                Ps.append(run.scalar_spectrum())
        run.close()
        res = []
        for w0 in range(0, len(Es) - window + 1, window):
            pair = []
            for series in (np.array(Es[w0:w0 + window]), np.array(Ps[w0:w0 + window])):
                bm = series.reshape(window // batch, batch, -1).mean(axis=1)
                pair.append((series.mean(axis=0), bm.std(axis=0, ddof=1) / math.sqrt(bm.shape[0])))
            res.append(pair)
        wins[form] = res
    rel, z = [], []
    for w64, w32 in zip(wins["fp64"], wins["fp32_mixed"]):
        for (m64, s64), (m32, s32) in zip(w64, w32):
            live = m64 > 1e-6 * m64.max()
            d = np.abs(m32 - m64)[live]
            rel.append(float(np.max(d / m64[live])))
            z.append(float(np.max(d / np.hypot(s64, s32)[live].clip(min=1e-300))))
    out.update({"long_steps": steps, "windows": len(wins["fp64"]), "window_steps": window,
                "spectrum_window_max_rel_diff": max(rel[0::2]), "scalar_spectrum_window_max_rel_diff": max(rel[1::2]),
                "max_diff_in_standard_errors": max(z)})
    return out


def ensemble_rate(device, steps=300, alone_steps=30, sweep_steps=40):
    """The batched ensemble: 96 FP32-mixed members, 32 each of 32³, 48³ and 64³, ν drawn from
    [0.005, 0.02] per member, ConstantPower ε = 0.1, G = 1, IF-RK4, stepped together under one CUDA
    graph (gbght_ensemble_step). The ensemble's autotuner picks the member batching (the group size,
    1 = one launch per member and pass), then `steps` steps are timed; each group size is also timed
    over `sweep_steps` steps, and the members are timed stepped one by one."""
    import gbght
    from gbght import seed as S
    rng = np.random.default_rng(7)
    runs = []
    for i, n in enumerate([32] * 32 + [48] * 32 + [64] * 32):
        setup = gbght.Setup(grid_points_per_axis=n, viscosity=float(rng.uniform(0.005, 0.02)),
                            velocity_forcing=gbght.ConstantPower(0.1), mean_gradient=(1.0, 0.0, 0.0),
                            precision="fp32_mixed", device=device)
        runs.append(gbght.simulation(setup, S.seed_velocity(n, 0.5, seed=100 + i), S.seed_scalar(n, 0.5, seed=300 + i)))
    dt = 0.002
    ens = gbght.Ensemble(runs)

    def timed(nsteps):
        ens.step(dt)   # a capture when the batching changed
        runs[0].synchronize()
        t0 = time.perf_counter()
        for _ in range(nsteps):
            ens.step(dt)
        return len(runs) * nsteps / (time.perf_counter() - t0)
    sweep = {}
    for g in (1, 2, 4, 8, 16, 32):
        ens.set_batching(g)
        sweep[g] = {"member_steps_per_s": round(timed(sweep_steps), 1), "launching_units": ens.units()}
    ens.autotune()
    while not ens.tuning()[1]:
        ens.step(dt)
    chosen, _, tune_ms = ens.tuning()
    rate = timed(steps)
    units = ens.units()
    ens.close()
    for r in runs:
        r.advance(dt)
    t0 = time.perf_counter()
    for _ in range(alone_steps):
        for r in runs:
            r.step(dt)
            r.deposit()
    alone = len(runs) * alone_steps / (time.perf_counter() - t0)
    for r in runs:
        r.close()
    return {"members": len(runs), "grids": "32x32^3 + 32x48^3 + 32x64^3", "form": "fp32_mixed", "steps": steps,
            "member_steps_per_s": round(rate, 1), "group_size": chosen, "launching_units": units,
            "autotune_replay_ms": [round(v, 3) for v in tune_ms], "by_group_size": sweep,
            "member_steps_per_s_one_by_one": round(alone, 1), "speedup_vs_one_by_one": round(rate / alone, 3),
            "speedup_vs_one_launch_per_member": round(rate / sweep[1]["member_steps_per_s"], 3),
            "timing": "host wall clock around synchronising calls"}


def cpu_steps(N, M, budget_s, min_steps=1, max_steps=None):
    """Whole iterations of the oracle's run layer (`advance!`: the IF-RK4 step, the deposit, the
    Heun push and particle deposit, the guards) on the workload at N³ with M tracers, NumPy +
    scipy.fft on every host core: as many as fit `budget_s` seconds, at least `min_steps` and at most
    `max_steps`. The run's
    construction (seeding, the first deposit and particle sample) is not timed. Returns the steps
    run and the seconds they took."""
    from oracle import gbght_oracle as O
    uh, ph, X = make_inputs(N, M, seed_base=0)
    dom = O.Domain(N)
    cond = O.Conditions(viscosity=WORKLOAD["viscosity"], schmidt=WORKLOAD["schmidt"],
                        velocity_forcing=O.ConstantPower(WORKLOAD["injection_rate"], *WORKLOAD["shells"]),
                        mean_gradient=WORKLOAD["G"])
    run = O.Run(dom, cond, O.State(uh, ph), X=X, scheme="rk4", cfl=WORKLOAD["cfl"])
    del uh, ph, X
    n, total = 0, 0.0
    while (n < min_steps or total < budget_s) and (max_steps is None or n < max_steps):
        t0 = time.perf_counter()
        run.advance(None)
        total += time.perf_counter() - t0
        n += 1
        if n >= min_steps and total + total / n > budget_s:
            break
    return n, total


def cpu_baseline_line(args, budget_s, max_steps=None):
    """The `cpu_baseline` object: full oracle iterations of the benchmark's workload."""
    n, total = cpu_steps(args.grid, args.tracers, budget_s, max_steps=max_steps)
    return {"value": n / total, "unit": "steps/s", "cores": os.cpu_count(), "kind": "port",
            "sample": f"{n} full step(s) of the {args.grid}^3 workload with {args.tracers} tracers (advance!: "
                      f"IF-RK4 step, deposit, Heun push, particle deposit, guards) on the NumPy/scipy.fft "
                      f"oracle, {total:.1f} s"}


def ours(args):
    import torch
    ws, rank, local = _dist()
    device = local
    torch.cuda.set_device(device)
    if ws > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600))
    N = args.grid
    inputs = make_inputs(N, args.tracers, seed_base=0)
    hbm, peak_kind = _peaks()
    results = {}
    forms = ["fp64", "fp32_mixed"] if args.form == "both" else [args.form]
    for form in forms:
        run = run_form(args, form, device, inputs)
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()
        with ClockSampler(device) as cs:
            ms, prof = timed_steps(run, args.steps)
        el = max_over_ranks(ms / 1e3, f"cuda:{device}")
        spectra = (run.energy_spectrum(), run.scalar_spectrum())
        results[form] = dict(el=el, prof=prof, clocks=cs.summary(), K=run.K, spectra=spectra,
                             diagnostics=time_diagnostics(run))
        run.close()
        del run
    # end-to-end through the public API (host buffers), the headline form
    e2e_val, h2d, d2h = (float("nan"), 0, 0) if args.no_e2e else e2e_run(args, forms[0], device, inputs, args.steps)
    if ws > 1:
        e2e_val = 1.0 / max_over_ranks(1.0 / e2e_val, f"cuda:{device}")
    if rank == 0:
        head = results[forms[0]]
        value = replica_rate(ws, args.steps, head["el"])
        w_complex = 16 if forms[0] == "fp64" else 8
        ab = algorithmic_bytes_per_step(N, head["K"], w_complex)
        prof = head["prof"]
        kind = max(ab, key=lambda k: prof[k][1])
        n_launch, tot_ms = prof[kind]
        achieved = ab[kind] * args.steps / (tot_ms / 1e3) / 1e9 if tot_ms > 0 else 0.0
        line = {
            "metric": METRIC, "value": round(value, 4), "unit": "steps/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(head["el"] * 1e3 / args.steps, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64" if forms[0] == "fp64" else "f32",
            "data": "synthetic (seeded k^4 spectrum, uniform tracers)", "config": _config(args, N),
            "grid_point_stages_per_s": value * 5 * N ** 3,
            "roofline": {"bound": "hbm", "kernel": kind, "achieved": round(achieved, 1), "peak": hbm,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
                         "unit": "GB/s", "frac": round(achieved / hbm, 4),
                         "algorithmic_bytes_per_launch": ab[kind] / max(1, n_launch / args.steps),
                         "avg_launch_ms": tot_ms / max(1, n_launch),
                         "traffic": (round(ab[kind] / max(1, n_launch / args.steps) * TRAFFIC_RATIO[(kind, forms[0])])
                                     if (kind, forms[0]) in TRAFFIC_RATIO else None),
                         "traffic_source": "ncu dram__bytes_read+write of one launch at 256^3, scaled to this "
                                           "launch by the tiles processed"},
            "kernels": {k: {"launches": v[0], "ms": round(v[1], 3)} for k, v in prof.items() if v[0]},
            "gpu_launches": int(sum(v[0] for v in prof.values())),
            "clocks": head["clocks"],
            "diagnostics": head["diagnostics"],
            "e2e": {"value": round(e2e_val, 4), "unit": "steps/s", "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h)},
        }
        if "fp32_mixed" in results and "fp64" in results:
            m = results["fp32_mixed"]
            mv = replica_rate(ws, args.steps, m["el"])
            E64, P64 = results["fp64"]["spectra"]
            E32, P32 = m["spectra"]
            live = E64 > 1e-6 * E64.max()
            livep = P64 > 1e-6 * P64.max()
            line["forms"] = {"fp32_mixed": {"value": round(mv, 4), "unit": "steps/s",
                                            "ratio_vs_fp64": round(mv / value, 3),
                                            "kernels": {k: {"launches": v[0], "ms": round(v[1], 3)}
                                                        for k, v in m["prof"].items() if v[0]},
                                            "clocks": m["clocks"],
                                            "spectrum_rel_err_after_K_steps": float(np.max(np.abs(E32[live] - E64[live]) / E64[live])),
                                            "scalar_spectrum_rel_err_after_K_steps": float(np.max(np.abs(P32[livep] - P64[livep]) / P64[livep]))}}
        if ws == 1 and args.extras == "dealiasing":
            line["dealiasing"] = dealiasing_cost(args, device, inputs)
        if ws == 1 and args.extras == "ensemble":
            line.setdefault("forms", {})["ensemble"] = ensemble_rate(device)
        if ws == 1 and args.extras in ("all", "adjoint"):
            line["adjoint"] = adjoint_cost(args, device, inputs)
            if args.extras == "all":
                line["dealiasing"] = dealiasing_cost(args, device, inputs)
                line.setdefault("forms", {}).setdefault("fp32_mixed", {})["c1_256cubed"] = c1_statistics(device)
                line["forms"]["ensemble"] = ensemble_rate(device)
        if ws == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline_line(args, budget_s=60.0)
        print(json.dumps(line), flush=True)
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()


def reference(args):
    ws, rank, _ = _dist()
    if rank != 0:
        return
    N = args.grid
    cb = cpu_baseline_line(args, budget_s=120.0, max_steps=max(1, args.steps))
    n = int(cb["sample"].split()[0])
    small = {}
    for n_small, m_small in ((64, 4096), (256, 100_000)):
        if n_small < N:
            k, t = cpu_steps(n_small, m_small, budget_s=0.0)
            small[f"{n_small}^3"] = {"ms_per_step": round(t / k * 1e3, 1), "tracers": m_small}
    v = cb["value"]
    line = {"metric": METRIC, "value": v, "unit": "steps/s", "n_gpus": ws, "steps": n, "warmup": 0,
            "ms_per_step": 1e3 / v, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded k^4 spectrum, uniform tracers)", "config": _config(args, N),
            "impl": "reference", "cpu_baseline": cb, "cpu_smaller_grids": small,
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--grid", type=int, default=WORKLOAD["N"])
    ap.add_argument("--tracers", type=int, default=WORKLOAD["tracers"])
    ap.add_argument("--form", default="both", choices=["both", "fp64", "fp32_mixed"])
    ap.add_argument("--scheme", default=WORKLOAD["scheme"], choices=list(SCHEME_NAME),
                    help="the field integration scheme (the metric is quoted on IFLowStorageRK4)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (quick kernel timing)")
    ap.add_argument("--extras", default="all", choices=["all", "adjoint", "dealiasing", "ensemble", "none"],
                    help="the further legs rank 0 runs at N=1: the adjoint's cost, the 256^3 precision statistics "
                         "and the ensemble (all), the adjoint alone, or none")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        reference(args)
    else:
        ours(args)


if __name__ == "__main__":
    main()
