"""Gradients through many steps: the step's discrete adjoint (`gbght_adjoint_step`) applied backwards
over states recomputed from device snapshots, with a binomial checkpointing schedule.

The reference has no AD; this is the host side of the differentiation form. It plays the role of
a ChainRulesCore `rrule` around `run!` in Julia (the pullback of n calls of `step!`), or of a
torch.autograd.Function's backward. The loss is a sum of terms ℓ_k(q_k) over the states q_k,
k = 0..n, of n steps of sizes dts[k] (held fixed: the CFL rule's choice of Δt is not
differentiated). `loss_grad(run, k)` adds ∂ℓ_k/∂q_k to the run's adjoint register while the run
holds q_k (for instance through `Run.adjoint_add_observable`).

Schedule (Griewank & Walther 2000, "revolve"): with s snapshot slots, the span [k0, k0 + k) is split
where C(s + r − 1, s) of its steps are left to the recursion, r the fewest repetitions with
C(s + r, s) ≥ k; so at most r·n steps are recomputed. With no slot left, every state is recomputed
from the span's start. The same schedule as the CPU oracle's `gradient_checkpointed`.
"""
from __future__ import annotations

import math

import numpy as np


def binomial_repetitions(n: int, snaps: int) -> int:
    """The fewest r with C(snaps + r, snaps) ≥ n (r = n without snapshots)."""
    if snaps == 0:
        return n
    r = 1
    while math.comb(snaps + r, snaps) < n:
        r += 1
    return r


def binomial_split(n: int, snaps: int) -> int:
    """Where the schedule stores its next state in a span of n steps with `snaps` slots free."""
    r = binomial_repetitions(n, snaps)
    m = math.comb(snaps + r - 1, snaps)
    return min(max(1, n - m), n - 1)


class Reverse:
    """The reverse sweep of n steps from the run's current state q_0, keeping at most `snapshots`
    states on the device (slot 0 holds q_0). The run must have been given that many slots
    (`Run.adjoint_create(snapshots)`). After `run()`, the run's adjoint register holds ∂L/∂q_0, its
    forcing gradient holds ∂L/∂ε, and the run is back at q_0 with a current deposit."""

    def __init__(self, run, dts, loss_grad, snapshots: int):
        if snapshots < 1:
            raise ValueError("the reverse sweep needs at least the start's snapshot slot")
        self.run, self.dts, self.loss_grad, self.snapshots = run, [float(d) for d in dts], loss_grad, snapshots
        # with tracers, a step is a whole advance! iteration (the push and the particle deposit too)
        self.tracers = run.setup.tracers > 0
        self.cur = None          # the step index of the state the run holds
        self.forward_steps = 0   # steps recomputed by the reverse sweep
        self.adjoint_steps = 0
        self.peak = 0            # most snapshot slots held at once

    def _load(self, slot: int, k0: int):
        if self.cur != k0:
            self.run.snapshot_load(slot)
            self.cur = k0

    def _advance(self, k: int, count=True):
        for _ in range(k):
            self.run.deposit()
            if self.tracers:
                self.run.advance(self.dts[self.cur])
            else:
                self.run.step(self.dts[self.cur])
            self.cur += 1
            if count:
                self.forward_steps += 1

    def _reverse_one(self, k0: int):
        # the run holds q_k0; λ holds ∂L/∂q_(k0+1) (with every later term)
        if self.tracers:
            self.run.adjoint_advance(self.dts[k0])
        else:
            self.run.adjoint_step(self.dts[k0])
        self.adjoint_steps += 1
        self.loss_grad(self.run, k0)

    def _back(self, slot: int, k0: int, k: int, free: list):
        if k == 1:
            self._load(slot, k0)
            self._reverse_one(k0)
            return
        if not free:
            for i in range(k - 1, -1, -1):
                self._load(slot, k0)
                self._advance(i)
                self._reverse_one(k0 + i)
            return
        m = binomial_split(k, len(free))
        self._load(slot, k0)
        self._advance(m)
        s = free.pop()
        self.run.snapshot_save(s)
        self.peak = max(self.peak, self.snapshots - len(free))
        self._back(s, k0 + m, k - m, free)
        free.append(s)
        self._back(slot, k0, m, free)

    def run_sweep(self):
        run, n = self.run, len(self.dts)
        run.snapshot_save(0)
        self.cur = 0
        self.peak = 1
        self._advance(n, count=False)   # the forward sweep to the end
        self.loss_grad(run, n)
        self._back(0, 0, n, list(range(self.snapshots - 1, 0, -1)))
        run.snapshot_load(0)
        run.deposit()
        self.cur = 0
        if self.tracers:   # the construction's particle deposit f₀ = u₀(X₀)
            run.adjoint_deposit_tracers()
        return self


def gradient(run, dts, loss_grad, snapshots: int = 16):
    """∂L/∂q_0 (λ_u, λ_φ in the state's layout) and ∂L/∂ε (velocity, scalar) of the loss
    Σ_k ℓ_k(q_k) over `len(dts)` steps from the run's current state, by the checkpointed reverse
    sweep. The adjoint register and the forcing gradient are cleared first (and the tracer
    cotangents, for a run with tracers: then a step is an advance! iteration, `loss_grad` may add
    to the tracer cotangents through `Run.adjoint_tracers_import`, and `sweep.tracer_gradient`
    holds ∂L/∂X_0 at the end)."""
    run.adjoint_clear()
    if run.setup.tracers:
        z = np.zeros((3, run.setup.tracers))
        run.adjoint_tracers_import(z, z)
    sweep = Reverse(run, dts, loss_grad, snapshots).run_sweep()
    lam = run.adjoint_export()
    if run.setup.tracers:
        sweep.tracer_gradient = run.adjoint_tracers_export()[0]
    return lam, run.forcing_gradient(), sweep


def tracer_kinetic_energy(step: int, weight: float = 1.0):
    """loss_grad of L = weight · (1/M) Σ_p |u(X_p)|² over the tracers' newest samples at `step`
    (λ_f += 2·weight·f/M there)."""
    def loss_grad(run, k):
        if k == step:
            f, _ = run.tracer_sample()
            lX, lf = run.adjoint_tracers_export()
            run.adjoint_tracers_import(lX, lf + 2.0 * weight * f / f.shape[1])
    return loss_grad


def combined(*terms):
    """The loss_grad of a sum of losses."""
    def loss_grad(run, k):
        for t in terms:
            t(run, k)
    return loss_grad


def scalar_variance_window(n0: int, n1: int):
    """loss_grad of L = mean over steps n0..n1 of ⟨φ²⟩."""
    w = 1.0 / (n1 - n0 + 1)

    def loss_grad(run, k):
        if n0 <= k <= n1:
            run.adjoint_add_observable("scalar_variance", w)
    return loss_grad
