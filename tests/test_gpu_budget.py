"""Equal modelled budgets for the two policies (the reference's model F): Chord's default MDI schedule sets the
budget on a tuning batch, and Arpeggio's S* is the largest sweep count within it."""
import pytest

pytestmark = pytest.mark.gpu


def test_arpeggio_sweeps_matched_to_chord_budget():
    from arpeggio_b200 import budget, channel
    b = channel.draw(1000, 20.0, 0, 300, 16, 16)
    chord = dict(T0=0.3, T1=0.3, q=0.4, start='rand', Ns=32)          # MDICHORD (mdi_solvers.py:18)
    S, xs, ref = budget.match_sweeps(b['H'], b['y'], b['N0'], 16, 1, chord, grid=(16, 32, 64, 96, 128, 192))
    assert set(ref) <= {'1', '2', '3'} and all(v > 256 * int(k) for k, v in ref.items())  # L_K plus flips
    assert S is not None and xs[S] <= 1.0
    bigger = [s for s in xs if s > S]
    assert all(xs[s] > 1.0 for s in bigger)
    assert all(xs[a] <= xs[c] for a, c in zip(sorted(xs), sorted(xs)[1:]))  # cost grows with the sweeps
    assert budget.cycles_first_accept(162, 35) == 3 * 162 + 2 * 35
