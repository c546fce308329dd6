"""The autotuner on the GPU: every candidate times, a tuned case is the same alone and in the mix, and
it breaks where the default settings break, within 1% in time and crest position."""
import pytest

from pysurf_b200 import batch, tuning

pytestmark = pytest.mark.gpu


def test_tuned_cases_are_the_same_alone_and_in_the_mix_and_break_where_the_defaults_do():
    specs = [batch.CaseSpec(0, 1 / 15, 0.45, 16), batch.CaseSpec(1, 1 / 10, 0.3, 12),
             batch.CaseSpec(2, 1 / 25, 0.5, 14)]
    tuner = tuning.Autotuner(steps=5, warmup=2)
    tuned = tuner.prepare(specs, batch.buildCase)
    assert tuned and set(tuned) == set(tuner.choices)
    for table in tuned.values():
        assert len(table) == len(tuning.candidates(2))
        assert all(row['ms_per_step'] > 0.0 for row in table)
    mixed = batch.BatchRunner(slots=3, tuner=tuner).run(specs)
    broke = 0
    for spec, m in zip(specs, mixed):
        case = batch.buildCase(spec)
        alone = batch.solveCase(spec, case=case, tuning=tuner.choose(case))
        plain = batch.solveCase(spec)
        assert m.error is None and alone.error is None and plain.error is None
        assert alone.key() == m.key()
        if plain.breakingTime == plain.breakingTime:
            broke += 1
            assert abs(m.breakingTime - plain.breakingTime) <= 0.01 * plain.breakingTime
            assert abs(m.breakingCrestX - plain.breakingCrestX) <= 0.01 * plain.breakingCrestX
    assert broke > 0


def test_timing_a_choice_gives_milliseconds_a_step():
    case = batch.buildCase(batch.CaseSpec(0, 1 / 15, 0.45, 12))
    for choice in (tuning.Tuning(2, 8), tuning.Tuning(4, 2)):
        ms = tuning.timeTuning(case, choice, steps=4, warmup=2)
        assert 0.0 < ms < 1000.0
