"""Both Catmull–Rom tracer gathers, one thread per tracer and warp-cooperative (16 lanes per tracer,
one (z, y) row of the stencil per lane), against the oracle's gather on the same physical field: the
sums run in the same order with the same roundings, so the values agree bit for bit (`interpolate!`,
src/Particles.jl:290-293), and runs with either gather advance their tracers identically."""
import numpy as np
import pytest

from oracle import gbght_oracle as O
from pairs import make_case


@pytest.mark.gpu
@pytest.mark.parametrize("gather", ["per_tracer", "warp"])
@pytest.mark.parametrize("precision", ["fp64", "fp32_mixed"])
def test_gathers_are_the_oracle_gather_bit_for_bit(cuda_library, precision, gather):
    N = 64
    run, _ = make_case(N, forcing=0.1, tracers=1000, precision=precision, tracer_gather=gather, library=cuda_library)
    run.advance(0.004)
    U = run.velocity_physical()    # the deposited field the gathers read
    X = np.random.default_rng(5).uniform(-1.0, 7.5, (3, 4099))   # across the wrap, a ragged count
    got = run.interpolate_velocity(X)
    want = O.interpolate(O.Domain(N), U.astype(np.float64), X)
    assert np.array_equal(got, want), float(np.max(np.abs(got - want)))
    # the push's own samples: the trail's newest sample is the gather at the new positions
    F, _ = run.tracer_sample()
    assert np.array_equal(F, O.interpolate(O.Domain(N), U.astype(np.float64), run.tracers()))


@pytest.mark.gpu
def test_both_gathers_advance_tracers_identically(cuda_library):
    runs = [make_case(64, forcing=0.1, tracers=3001, tracer_scheme=("ABM", 3), tracer_gather=g,
                      library=cuda_library)[0] for g in ("per_tracer", "warp")]
    for _ in range(4):
        for r in runs:
            r.advance(0.004)
    assert np.array_equal(runs[0].tracers(), runs[1].tracers())
    assert np.array_equal(runs[0].tracer_sample()[0], runs[1].tracer_sample()[0])
