"""Equal modelled budgets for the two policies: Chord's default MDI schedule sets the budget on a tuning batch, and
Arpeggio's S* is the largest sweep count within it, in the reference's model F (tests or steps + flips) and in the
single-lane engines' cycles (first accept 3 tests + 2 F, Chord 3 L + F + n1)."""
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('cost', ['F', 'cycles'])
def test_arpeggio_sweeps_matched_to_chord_budget(cost):
    from arpeggio_b200 import budget, channel
    b = channel.draw(1000, 20.0, 0, 300, 16, 16)
    chord = dict(T0=0.3, T1=0.3, q=0.4, start='rand', Ns=32)          # MDICHORD (mdi_solvers.py:18)
    S, xs, ref = budget.match_sweeps(b['H'], b['y'], b['N0'], 16, 1, chord, grid=(16, 32, 64, 96, 128, 192),
                                     cost=cost)
    per_step = 1 if cost == 'F' else 3
    assert set(ref) <= {'1', '2', '3'} and all(v > per_step * 256 * int(k) for k, v in ref.items())
    assert S is not None and xs[S] <= 1.0
    bigger = [s for s in xs if s > S]
    assert all(xs[s] > 1.0 for s in bigger)
    assert all(xs[a] <= xs[c] for a, c in zip(sorted(xs), sorted(xs)[1:]))  # cost grows with the sweeps
    assert budget.cycles_first_accept(162, 35) == 3 * 162 + 2 * 35


def test_chord_round_counts_flipping_rounds_like_the_oracle():
    """arp_anneal_chord_dd_n1: spins, energies and counters as arp_anneal_chord_dd, and per anneal the rounds with at
    least one flip, equal to the oracle's count (n1 of arpeggio_ref59.anneal)."""
    from arpeggio_b200 import arpeggiofx, channel
    from arpeggio_b200.detector import chord_schedule
    nth = max(1, min(16, os.cpu_count() or 1))
    for nt, K, steps in ((16, 1, 256), (32, 2, 128), (64, 1, 64)):
        B, R, P = 40, 6, 2 * K
        bb = channel.draw(70 + nt, 14.0, 0, B, nt, 16)
        _, _, xq = O.mmse(bb['H'].numpy(), bb['y'].numpy(), bb['N0'], 16)
        Gf, hf, _ = O.ising_delta_compressed(bb['H'].numpy(), bb['y'].numpy(), xq)
        G, h = O.quantize_compressed(Gf, hf)
        T, q, c = chord_schedule(steps, 0.3, 0.3, 0.4, kappa=0.3)
        dev = torch.device('cuda')
        Gd, hd = torch.from_numpy(G).to(dev), torch.from_numpy(h).to(dev)
        Td = torch.tensor(T, dtype=torch.int32, device=dev)
        cd = torch.tensor(c, dtype=torch.int32, device=dev)
        inst = torch.arange(B, dtype=torch.int32, device=dev) * 3 + 5
        n1 = torch.zeros(B, R, dtype=torch.int64, device=dev)
        key = 0x5EED0000 + nt
        s, de, st, status = arpeggiofx.anneal(Gd, hd, P, R, Td, q, inst, key, 'rand', 'chord', cd, n1=n1)
        s2, de2, st2, _ = arpeggiofx.anneal(Gd, hd, P, R, Td, q, inst, key, 'rand', 'chord', cd)
        torch.cuda.synchronize()
        arpeggiofx.check_status(status)
        os_, ode, ost, on1 = O.anneal_chord_n1(G, h, P, R, T, c, q, inst.cpu().numpy(), key, 'rand', nthreads=nth)
        assert torch.equal(s, s2) and torch.equal(de, de2) and torch.equal(st, st2)
        assert np.array_equal(s.cpu().numpy(), os_) and np.array_equal(de.cpu().numpy(), ode)
        assert np.array_equal(st.cpu().numpy(), ost)
        assert np.array_equal(n1.cpu().numpy(), on1)
        assert (on1 <= len(T)).all() and (on1 <= ost[..., 0]).all()
