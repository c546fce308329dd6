"""The autotuner's host logic (pysurf_b200.tuning), on CPU with a fake timer: candidates, size classes,
the choice of the fastest, one middle-sized case timed per class, lookups that never time, and the
saved choices."""
import json
from types import SimpleNamespace

import pytest

from pysurf_b200 import tuning
from pysurf_b200.tuning import Autotuner, Tuning


def fakeCase(particles, dimensions=2, kernel='wendlandC2'):
    return SimpleNamespace(dimensions=dimensions, kernelType=kernel, state=SimpleNamespace(nParticles=particles))


def test_candidates_are_valid_settings():
    for dim in (2, 3):
        choices = tuning.candidates(dim)
        assert len(set(choices)) == len(choices) > 1
        assert all(c.cellsPerSupport in (1, 2, 3, 4) and c.threadsPerParticle in (1, 2, 4, 8) for c in choices)
        assert Tuning() in choices      # the default is always among them


def test_size_classes_are_half_octaves_per_dimension_and_kernel():
    assert tuning.sizeClass(2, 'wendlandC2', 100_000) == tuning.sizeClass(2, 'wendlandC2', 110_000)
    assert tuning.sizeClass(2, 'wendlandC2', 100_000) != tuning.sizeClass(2, 'wendlandC2', 150_000)
    assert tuning.sizeClass(2, 'wendlandC2', 100_000) != tuning.sizeClass(3, 'wendlandC2', 100_000)
    assert tuning.sizeClass(2, 'wendlandC2', 100_000) != tuning.sizeClass(2, 'cubicSpline', 100_000)
    assert tuning.sizeClass(2, 'wendlandC2', 0) == tuning.sizeClass(2, 'wendlandC2', 1)


def test_the_fastest_candidate_wins_and_ties_go_to_the_earlier():
    table = {Tuning(2, 4): 1.0, Tuning(3, 8): 0.5, Tuning(4, 2): 0.5}
    timer = lambda case, choice, **kw: table[choice]        # noqa: E731
    result = tuning.tuneCase(fakeCase(1000), timer=timer, choices=list(table))
    assert result.best == Tuning(3, 8)
    assert [row['ms_per_step'] for row in result.table()] == [0.5, 0.5, 1.0]
    with pytest.raises(RuntimeError):
        tuning.tuneCase(fakeCase(1000), timer=lambda case, choice, **kw: float('nan'), choices=[Tuning()])
    with pytest.raises(ValueError):
        tuning.tuneCase(fakeCase(1000), timer=timer, choices=[])


def test_prepare_times_one_middle_sized_case_per_class_and_choose_never_times():
    timed = []

    def timer(case, choice, **kw):
        timed.append((case.state.nParticles, choice))
        # the small class prefers eight threads a particle, the large one two
        return {8: 1.0, 4: 2.0, 2: 3.0}[choice.threadsPerParticle] * (1 if case.state.nParticles < 50_000 else
                                                                      {8: 3.0, 4: 2.0, 2: 0.5}[choice.threadsPerParticle])

    small = [fakeCase(n) for n in (20_000, 21_000, 22_000)]
    large = [fakeCase(n) for n in (100_000, 101_000, 102_000, 103_000)]
    tuner = Autotuner(timer=timer)
    tuned = tuner.prepare(small + large)
    assert len(tuned) == 2
    sizes = sorted({n for n, _ in timed})
    assert sizes == [21_000, 102_000]          # the middle member of each class (upper middle of four)
    assert tuner.choose(small[0]).threadsPerParticle == 8
    assert tuner.choose(large[-1]).threadsPerParticle == 2
    count = len(timed)
    assert tuner.choose(fakeCase(5_000_000)) == Tuning()      # an unprepared class: the default, untimed
    assert tuner.prepare(small + large) == {} and len(timed) == count     # known classes are not timed again


def test_prepare_takes_specs_through_a_builder():
    tuner = Autotuner(timer=lambda case, choice, **kw: float(choice.cellsPerSupport))
    tuner.prepare([1100, 1200, 40_000], builder=fakeCase)
    assert tuner.choose(fakeCase(1150)).cellsPerSupport == 2
    assert len(tuner.choices) == 2


def test_choices_are_saved_and_loaded(tmp_path):
    tuner = Autotuner(timer=lambda case, choice, **kw: float(choice.threadsPerParticle))
    tuner.prepare([fakeCase(30_000), fakeCase(300_000, dimensions=3)])
    path = tmp_path / 'tuning.json'
    tuner.save(str(path))
    again = Autotuner(timer=None)
    again.load(str(path))
    assert again.choices == tuner.choices and again.tables == tuner.tables
    data = json.loads(path.read_text())
    key = next(iter(data['choices']))
    data['choices'][key]['threadsPerParticle'] = 3
    path.write_text(json.dumps(data))
    with pytest.raises(ValueError):
        Autotuner().load(str(path))
