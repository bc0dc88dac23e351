"""The reference's C++ Chord engine model (arpeggio/sim/x3model/engine_model.cpp, built from its source into
oracle/_ref/libape.so by `make -C oracle ref`) as a second pin of the oracle's Chord round on compressed problems:
with Philox numbers (philox = 1) the engine's best spins, best energy changes and flip counts equal the oracle's
bit for bit.  CPU only; skipped where the engine was not built (no reference tree at build time)."""
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), '..'))
from oracle import oracle as O  # noqa: E402
from oracle import ref_engine  # noqa: E402

NTH = min(8, os.cpu_count() or 1)


def _engine():
    if not ref_engine.available():
        pytest.skip('reference engine not built (make -C oracle ref needs the reference tree)')


def _random_dd(B, D, snr, seed):
    from arpeggio_b200 import channel
    b = channel.draw(seed, snr, 0, B, D // 2, 16)
    _, _, xq = O.mmse(b['H'].numpy(), b['y'].numpy(), b['N0'], 16)
    Gf, hf, _ = O.ising_delta_compressed(b['H'].numpy(), b['y'].numpy(), xq)
    return O.quantize_compressed(Gf, hf)


@pytest.mark.parametrize('D,K,R,steps,kappa,snr', [
    (64, 1, 8, 256, 0.0, 14.0),    # 32 users: Chord's default schedule (128 steps per copy pair, T 0.3, q 0.4)
    (32, 1, 8, 256, 0.3, 20.0),    # 16 users, Onsager term on
    (64, 2, 4, 128, 0.3, 10.0),    # four copies
    (96, 3, 2, 96, 0.0, 18.0),     # six copies, 48 users
    (128, 1, 2, 64, 0.3, 22.0),    # 64 users, shortened
])
def test_oracle_chord_equals_reference_engine(D, K, R, steps, kappa, snr):
    _engine()
    from arpeggio_b200.detector import chord_schedule
    B, P = 12, 2 * K
    G, h = _random_dd(B, D, snr, 700 + D + K)
    T, q, c = chord_schedule(steps, 0.3, 0.3, 0.4, kappa=kappa)
    key = 0x5EED00C0FFEE + D
    inst = (np.arange(B, dtype=np.int64) * 13 + 5) & 0xFFFFFFFF
    es, ede, cyc, est = ref_engine.solve_batch(G, h, P, R, T, c, q, inst, key, nthreads=NTH)
    os_, ode, ost = O.anneal_dd(G, h, P, R, T, q, inst, key, 'rand', policy='chord', c=c, nthreads=NTH)
    assert np.array_equal(es, os_)
    assert np.array_equal(ede, ode)
    assert np.array_equal(est[:, 1], ost[..., 0].sum(axis=1))  # flips per problem
    assert (est[:, 0] == R * len(T)).all()                      # one decision op per step
    assert (cyc > 0).all()


def test_engine_refuses_wide_words():
    """The engine holds G, h, T and c in int16 words; wider inputs are refused before the call."""
    _engine()
    G = np.zeros((1, 32, 32), np.int32)
    G[0, 0, 0] = 40000
    with pytest.raises(ValueError):
        ref_engine.solve_batch(G, np.zeros((1, 32), np.int32), 2, 1, [100], [0], 0, [0], 1)


@pytest.mark.parametrize('D,K,R,steps,kappa,snr', [
    (64, 1, 8, 256, 0.0, 14.0),    # 32 users, Chord's default schedule
    (32, 1, 8, 256, 0.3, 20.0),    # 16 users, Onsager term on
    (64, 2, 4, 128, 0.3, 10.0),    # four copies
    (96, 3, 2, 96, 0.3, 18.0),     # six copies, 48 users
    (128, 1, 2, 64, 0.0, 22.0),    # 64 users, shortened
])
def test_oracle_chord_with_engine_numbers_equals_reference_engine(D, K, R, steps, kappa, snr):
    """The engine's own numbers (philox = 0: hash-seeded xorshift32 per lane, 16-bit draws), the mode its
    production scripts run: the oracle's restatement gives the engine's best spins, energies and flips."""
    _engine()
    from arpeggio_b200.detector import chord_schedule
    B, P = 12, 2 * K
    G, h = _random_dd(B, D, snr, 900 + D + K)
    T, q, c = chord_schedule(steps, 0.3, 0.3, 0.4, kappa=kappa)
    key = 0x0DDBA11C0FFEE + D
    inst = (np.arange(B, dtype=np.int64) * 29 + 3) & 0xFFFFFFFF
    es, ede, _, est = ref_engine.solve_batch(G, h, P, R, T, c, q, inst, key, nthreads=NTH, philox=0)
    os_, ode, ost = O.anneal_chord_hw(G, h, P, R, T, c, q, inst, key, nthreads=NTH)
    assert np.array_equal(es, os_)
    assert np.array_equal(ede, ode)
    assert np.array_equal(est[:, 1], ost[..., 0].sum(axis=1))
    assert (ost[..., 1] == len(T)).all()
    # a different stream from the Philox mode on the same problems
    ps, _, _, _ = ref_engine.solve_batch(G, h, P, R, T, c, q, inst, key, nthreads=NTH, philox=1)
    assert not np.array_equal(ps, es)
