"""Run the same seeded case through the library and through the oracle, and compare.

Every comparison here is library-under-test against the CPU oracle (oracle/gbght_oracle.py).
"""
from __future__ import annotations

import math

import numpy as np

import gbght
from gbght import seed as S
from oracle import gbght_oracle as O


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


ORACLE_SCHEME = {"IFLowStorageRK4": "rk4", "IFLowStorageRK3": "rk3", "IFHeun": "heun", "IFSSPRK3": "ssprk3"}


def oracle_forcing(f):
    """The oracle's counterpart of a library forcing object (None for NoForcing)."""
    if f is None or isinstance(f, gbght.NoForcing):
        return None
    if isinstance(f, gbght.ConstantPower):
        return O.ConstantPower(f.injection_rate, f.lowest_shell, f.highest_shell)
    if isinstance(f, gbght.Linear):
        return O.Linear(f.rate, f.lowest_shell, f.highest_shell)
    if isinstance(f, gbght.VarianceController):
        return O.VarianceController(f.target, f.turnover_time, f.gain, f.lowest_shell, f.highest_shell)
    if isinstance(f, gbght.StochasticOU):
        return O.StochasticOU(f.forcing_variance, f.correlation_time, f.lowest_shell, f.highest_shell)
    if isinstance(f, gbght.VarianceRescaling):
        return O.VarianceRescaling(f.target, f.over, f.lowest_shell, f.highest_shell)
    raise ValueError(f"no oracle forcing for {f!r}")


def make_case(N, *, viscosity=0.01, schmidt=1.0, scalar=True, forcing=None, G=(0.0, 0.0, 0.0), tracers=0,
              scheme="IFLowStorageRK4", precision="fp64", cfl=0.5, seeds=(0, 1, 2), energy=0.5, variance=0.5,
              library=None, uh=None, ph=None, X=None, scalar_forcing=None, tracer_scheme=("Heun", 1),
              shortened_first_steps=False, interpolation=("CatmullRom", 4, 1), dealiasing="TwoThirds",
              tracer_gather="auto"):
    """Build a library run and an oracle run on identical seeded inputs, both freshly deposited.

    `forcing` is a ConstantPower ε (a number) or a library forcing object; `scalar_forcing` is a
    library forcing object for the scalar."""
    if uh is None:
        uh = S.seed_velocity(N, energy, seed=seeds[0])
    if ph is None and scalar:
        ph = S.seed_scalar(N, variance, seed=seeds[1])
    if X is None and tracers:
        X = S.seed_tracers(tracers, seed=seeds[2])
    if isinstance(forcing, (int, float)):
        lib_forcing = gbght.ConstantPower(forcing) if forcing else gbght.NoForcing()
    else:
        lib_forcing = forcing or gbght.NoForcing()
    lib_sforcing = scalar_forcing or gbght.NoForcing()
    setup = gbght.Setup(grid_points_per_axis=N, viscosity=viscosity, schmidt=schmidt, scalar=scalar,
                        velocity_forcing=lib_forcing, scalar_forcing=lib_sforcing, mean_gradient=G,
                        tracers=tracers, scheme=scheme, precision=precision, cfl=cfl,
                        tracer_scheme=tracer_scheme[0], tracer_steps=tracer_scheme[1],
                        shortened_first_steps=shortened_first_steps, interpolation=interpolation,
                        dealiasing=dealiasing, tracer_gather=tracer_gather)
    run = gbght.simulation(setup, uh, ph if scalar else None, X, library=library)
    dom = O.Domain(N, dealiasing=dealiasing)
    cond = O.Conditions(viscosity=viscosity, schmidt=schmidt, scalar=scalar,
                        velocity_forcing=oracle_forcing(lib_forcing), mean_gradient=G,
                        scalar_forcing=oracle_forcing(lib_sforcing))
    orun = O.Run(dom, cond, O.State(uh.copy(), ph.copy() if scalar else None),
                 X=None if not tracers else X.copy(), scheme=ORACLE_SCHEME[scheme],
                 cfl=cfl, tracer_scheme=("ab" if tracer_scheme[0] == "AB" else "abm", tracer_scheme[1]),
                 shortened_first_steps=shortened_first_steps, interpolation=tuple(interpolation))
    return run, orun


def advance_both(run, orun, nsteps, dt=None):
    taken = []
    for _ in range(nsteps):
        d_lib = run.advance(dt)
        d_ora = orun.advance(dt)
        taken.append((d_lib, d_ora))
    return taken


def compare(run, orun, *, tol, check_tracers=True):
    """Relative L2 of the spectral fields, the tracer cells and positions, the observables."""
    ue, pe = run.export_state()
    out = {"u": rel_l2(ue, orun.state.uh)}
    if orun.state.phih is not None:
        out["phi"] = rel_l2(pe, orun.state.phih)
    assert out["u"] <= tol, out
    if "phi" in out:
        assert out["phi"] <= tol, out
    if check_tracers and orun.X is not None:
        X = run.tracers()
        dx = orun.dom.dx
        cells_lib = np.floor(X / dx).astype(np.int64) % orun.dom.N
        cells_ora = np.floor(orun.X / dx).astype(np.int64) % orun.dom.N
        out["cells_equal"] = bool(np.array_equal(cells_lib, cells_ora))
        out["X_err"] = float(np.max(np.abs(X - orun.X)))
        assert out["cells_equal"], out
    return out
