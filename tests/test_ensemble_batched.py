"""Member-batched ensembles: members whose step launches the same kernels form a group, and the
captured graph holds one launch per pass for the group. Each member must still be stepped as it is
alone, whatever its viscosity, side length, forcing rate or mean gradient: to round-off, since the
group's kernels are a separate compilation of the same CTA code (bit for bit with batching off)."""
import math

import numpy as np
import pytest

import gbght
from pairs import make_case


def _rel(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _members(lib):
    rng = np.random.default_rng(3)
    runs = []
    # a group of four 32³ FP32-mixed RK4 ConstantPower runs with different ν, ε, G and seeds
    for i in range(4):
        runs.append(make_case(32, viscosity=float(rng.uniform(0.005, 0.02)), forcing=float(rng.uniform(0.05, 0.2)),
                              G=(float(i), 0.0, 0.0), precision="fp32_mixed", seeds=(i, 10 + i, 20 + i),
                              library=lib)[0])
    # a group of three 48³ FP64 IFHeun velocity-only runs with a Linear forcing
    for i in range(3):
        runs.append(make_case(48, scalar=False, forcing=gbght.Linear(0.1 * (i + 1)), scheme="IFHeun",
                              seeds=(30 + i, 40 + i, 50 + i), library=lib)[0])
    # a group of two 32³ FP64 HouLi SSPRK3 runs
    for i in range(2):
        runs.append(make_case(32, forcing=0.1, scheme="IFSSPRK3", dealiasing="HouLi", seeds=(60 + i, 70 + i, 80 + i),
                              library=lib)[0])
    # lone members: PhaseShift, VarianceController, and a one-member configuration
    runs.append(make_case(32, forcing=0.1, dealiasing="PhaseShift", library=lib)[0])
    runs.append(make_case(32, forcing=gbght.VarianceController(0.5, 1.0, 1.0), library=lib)[0])
    runs.append(make_case(64, forcing=0.1, scheme="IFLowStorageRK3", library=lib)[0])
    return runs


@pytest.mark.gpu
@pytest.mark.parametrize("batching", [True, False])
def test_batched_ensemble_equals_separate_runs(cuda_library, batching):
    ens_runs, alone = _members(cuda_library), _members(cuda_library)
    ens = gbght.Ensemble(ens_runs)
    ens.set_batching(batching)
    assert ens.units() == 0
    for k in range(4):
        dt = 0.004 if k < 3 else 0.003   # a new dt captures a new graph and new launch records
        ens.step(dt)
        for r in alone:
            r.step(dt)
            r.deposit()
    # three groups and three lone members, or one unit per member
    assert ens.units() == (6 if batching else len(ens_runs))
    for a, b in zip(ens_runs, alone):
        ua, pa = a.export_state()
        ub, pb = b.export_state()
        if batching:
            tol = 1e-6 if a.setup.precision == "fp32_mixed" else 1e-14
            assert _rel(ua, ub) <= tol and (pa is None or _rel(pa, pb) <= tol)
            assert a.max_speed() == pytest.approx(b.max_speed(), rel=tol)
        else:
            assert np.array_equal(ua, ub) and (pa is None or np.array_equal(pa, pb))
            assert a.max_speed() == b.max_speed()
    # the members stay usable runs: one more step alone continues bit for bit
    ens.close()
    for a, b in zip(ens_runs[:3], alone[:3]):
        a.advance(0.002)
        b.advance(0.002)
        assert _rel(a.export_state()[0], b.export_state()[0]) <= 1e-6


@pytest.mark.gpu
def test_batched_ensemble_side_lengths(cuda_library):
    # side lengths differ within a group (the geometry is per member)
    from gbght import seed as S
    runs, alone = [], []
    for L in (2 * math.pi, 4.0, 8.0):
        for dst in (runs, alone):
            setup = gbght.Setup(grid_points_per_axis=32, side_length=L, viscosity=0.01,
                                velocity_forcing=gbght.ConstantPower(0.1), precision="fp32_mixed")
            dst.append(gbght.simulation(setup, S.seed_velocity(32, 0.5, seed=1), S.seed_scalar(32, 0.5, seed=2),
                                        library=cuda_library))
    ens = gbght.Ensemble(runs)
    ens.set_batching(True)
    for _ in range(3):
        ens.step(0.003)
        for r in alone:
            r.step(0.003)
            r.deposit()
    assert ens.units() == 1
    for a, b in zip(runs, alone):
        assert _rel(a.export_state()[0], b.export_state()[0]) <= 1e-6
    ens.close()


@pytest.mark.gpu
def test_identical_members_stay_bitwise_equal(cuda_library):
    # members with equal inputs in one group are stepped by the same code: bitwise equal
    runs = [make_case(32, forcing=0.1, library=cuda_library)[0] for _ in range(3)]
    ens = gbght.Ensemble(runs)
    ens.set_batching(True)
    for _ in range(3):
        ens.step(0.003)
    assert ens.units() == 1
    u0 = runs[0].export_state()[0]
    for r in runs[1:]:
        assert np.array_equal(r.export_state()[0], u0)
    ens.close()


@pytest.mark.gpu
def test_autotune_picks_a_group_size(cuda_library):
    # four batchable 32³ members: the tuner tries group sizes 1, 2 and 4, two steps each, keeps the
    # fastest, and the members keep agreeing with their lone steps to round-off throughout
    runs = [make_case(32, forcing=0.1, seeds=(i, 7 + i, 9 + i), library=cuda_library)[0] for i in range(4)]
    alone = [make_case(32, forcing=0.1, seeds=(i, 7 + i, 9 + i), library=cuda_library)[0] for i in range(4)]
    ens = gbght.Ensemble(runs)
    ens.autotune()
    steps = 0
    while not ens.tuning()[1]:
        ens.step(0.003)
        steps += 1
        assert steps <= 12
    chosen, done, ms = ens.tuning()
    assert done and chosen in (1, 2, 4) and len(ms) == 3 and steps == 6
    ens.step(0.003)
    assert ens.units() == 4 // chosen
    for r in alone:
        for _ in range(steps + 1):
            r.step(0.003)
            r.deposit()
    for a, b in zip(runs, alone):
        assert _rel(a.export_state()[0], b.export_state()[0]) <= 1e-14
    ens.close()
