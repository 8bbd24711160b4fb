"""A checkpoint's save and restore through the C ABI, as the reference's HDF5 extension does it
(ext/GBGHomogeneousTurbulenceHDF5Ext.jl:426-561): the spectral state, the tracer positions, every
sample of the tracers' trail with its time, and the clock. The restored run must continue the
checkpointed one bitwise (test/hdf5_checkpoint.jl:112-116)."""
from __future__ import annotations

import numpy as np

import gbght


def save(run: gbght.Run) -> dict:
    uh, ph = run.export_state()
    ck = {"uh": uh, "ph": ph, "clock": run.clock()}
    if run.setup.tracers:
        ck["X"] = run.tracers()
        ck["trail"] = run.tracer_trail()
    return ck


def restore(setup: gbght.Setup, ck: dict, library=None) -> gbght.Run:
    """A new run from a checkpoint: the state and its deposit, the positions, the older trail
    samples restored oldest first, the newest taken again by the particle deposit at its time,
    and the clock."""
    run = gbght.Run(setup, library=library)
    run.import_state(ck["uh"], ck["ph"])
    run.deposit()
    if setup.tracers:
        run.import_tracers(ck["X"])
        run.reset_tracer_trail()
        trail = ck["trail"]
        for t, values in trail[:-1]:
            run.restore_tracer_sample(values, t)
        t_new, newest = trail[-1]
        run.deposit_tracers(t_new)
        F, t = run.tracer_sample()
        assert t == t_new and np.array_equal(F, newest)
    run.set_clock(*ck["clock"])
    return run


def continuation_is_bitwise(setup: gbght.Setup, uh, ph, X, before: int, after: int, library=None):
    """Run `before + after` steps in one run, and `before` steps, a checkpoint, a restore into a new
    run and `after` steps; the two must agree bit for bit."""
    a = gbght.simulation(setup, uh, ph, X, library=library)
    b = gbght.simulation(setup, uh, ph, X, library=library)
    for _ in range(before):
        a.advance(None)
        b.advance(None)
    c = restore(setup, save(b), library=library)
    b.close()
    for _ in range(after):
        da = a.advance(None)
        dc = c.advance(None)
        assert da == dc
    ua, pa = a.export_state()
    uc, pc = c.export_state()
    assert np.array_equal(ua, uc) and (pa is None or np.array_equal(pa, pc))
    if setup.tracers:
        assert np.array_equal(a.tracers(), c.tracers())
        for (ta, fa), (tc, fc) in zip(a.tracer_trail(), c.tracer_trail()):
            assert ta == tc and np.array_equal(fa, fc)
    assert a.clock() == c.clock()
