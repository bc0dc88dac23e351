"""The cost models of the equal-budget rule against the reference's own records (CPU): the single-lane engines'
cycle identities against their RTL latencies (data/results/a59/A59.json) and model F against the x16 MDI point's
recorded cost per anneal (data/results/a513/analysis.json, P1), through arpeggio_b200.budget."""
import json
import os

import pytest

from conftest import GOLDEN


def _fixture():
    return json.load(open(os.path.join(GOLDEN, 'golden_cycles.json')))


@pytest.mark.parametrize('point', ['p1', 'p2'])
def test_engine_cycles_equal_recorded_rtl_latencies(point):
    from arpeggio_b200 import budget
    for K, v in _fixture()['a59'][point].items():
        fa = budget.cycles_first_accept(v['arpeggio_tests'], v['arpeggio_F'])
        ch = budget.cycles_chord(v['chord_L'], v['chord_F'], v['chord_n1'])
        assert fa == pytest.approx(v['arpeggio_lat'], rel=1e-12), (point, K)
        assert ch == pytest.approx(v['chord_lat'], rel=1e-12), (point, K)


def test_model_f_reproduces_recorded_cost_per_anneal():
    from arpeggio_b200 import budget
    f = _fixture()['a513_P1']
    got = budget.cost_per_anneal(f['counters_fx'])
    assert set(got) == set(f['cost_per_anneal_fx'])
    for K, v in f['cost_per_anneal_fx'].items():
        assert got[K] == pytest.approx(v, rel=1e-12)


def test_cycle_cost_per_anneal_from_counters():
    from arpeggio_b200 import budget
    cnt = {'1': [35, 162, 1], '2': [120, 375, 2]}
    assert budget.cost_per_anneal(cnt, 'cycles', 'arpeggio') == {'1': 3 * 162 + 2 * 35, '2': (3 * 375 + 2 * 120) / 2}
    with pytest.raises(ValueError):
        budget.cost_per_anneal(cnt, 'cycles', 'chord')  # the Chord cycles need the n1 counter
    chord = {'1': [31, 256, 1, 11]}
    assert budget.cost_per_anneal(chord, 'cycles', 'chord') == {'1': 3 * 256 + 31 + 11}
    assert budget.x_of(cnt, {'1': 2 * (3 * 162 + 2 * 35)}, 'cycles') == pytest.approx(0.5)
