"""The CPU oracle against the reference's own outputs (fixtures made by tests/golden/make_golden.py)
and against the recorded B200 runs (tests/golden/pin_a513.json, made by tests/golden/pin_a513.py)."""
import json
import os

import numpy as np
import pytest

from oracle import oracle as O

from conftest import GOLDEN


def test_philox_kat(golden):
    z = golden('golden_philox.npz')
    assert np.array_equal(O.philox(z['kat_in']), z['kat_out'])
    assert np.array_equal(O.philox(z['rnd_in']), z['rnd_out'])


def _arp_cases():
    z = np.load(os.path.join(GOLDEN, 'golden_arpeggio.npz'))
    return [str(n) for n in z['names']]


@pytest.mark.parametrize('name', _arp_cases())
@pytest.mark.parametrize('mode', ['arpeggio', 'par'])
def test_anneal_dd_vs_arpeggio_ref59(golden, name, mode):
    z = golden('golden_arpeggio.npz')
    P, R, q, k0, k1, st = [int(v) for v in z[name + '/meta']]
    s, de, stt = O.anneal_dd(z[name + '/G'], z[name + '/h'], P, R, z[name + '/T'], q, z[name + '/inst'],
                             k0 | (k1 << 32), 'rand' if st == 0 else 'bal', policy=mode, nthreads=2)
    assert np.array_equal(s, z['%s/%s/spins' % (name, mode)])
    assert np.array_equal(de, z['%s/%s/de' % (name, mode)])
    assert np.array_equal(stt, z['%s/%s/st' % (name, mode)])


def _chord_cases():
    z = np.load(os.path.join(GOLDEN, 'golden_chord.npz'))
    return [str(n) for n in z['names']]


@pytest.mark.parametrize('name', _chord_cases())
@pytest.mark.parametrize('mode', ['chains', 'best'])
def test_chord_vs_chord_fx(golden, name, mode):
    z = golden('golden_chord.npz')
    q, S, P, R, s0, s1, inst0 = [int(v) for v in z[name + '/meta']]
    s, e = O.chord_fx(z[name + '/J'], z[name + '/h'], z[name + '/h0'], z[name + '/T'], z[name + '/c'], q, S, P, R,
                      s0 | (s1 << 32), inst0, mode, nthreads=2)
    assert np.array_equal(s, z['%s/%s_s' % (name, mode)])
    assert np.array_equal(e, z['%s/%s_e' % (name, mode)])


def test_counter_identity(golden):
    """tests = passes + flips not on a pass's last lane (arpx55.py:31-33, test_a55.py:72)."""
    z = golden('golden_arpeggio.npz')
    name = 'x16_K1_pick_rand'
    G, h = z[name + '/G'], z[name + '/h']
    P, R, q, k0, k1, st = [int(v) for v in z[name + '/meta']]
    T = z[name + '/T']
    s, de, stt = O.anneal_dd(G, h, P, R, T, q, z[name + '/inst'], k0 | (k1 << 32), 'rand')
    assert (stt[..., 1] >= len(T)).all() and (stt[..., 1] <= len(T) + stt[..., 0]).all()


def test_pin_a513_recorded_b200_runs():
    """The oracle inside the reference's own detection chain reproduced the B200 records exactly."""
    res = json.load(open(os.path.join(GOLDEN, 'pin_a513.json')))
    for tag in ('x16', 'x32', 'x64'):
        assert res[tag]['counters_equal'] and res[tag]['biterr_equal'], tag


def test_quantize_compressed_matches_reference(golden):
    """The numpy restatement of to_fixed + compress, fed the reference's own float chain, gives its integers
    on nearly every entry (float32 vs float64 rounding may move an entry sitting on a rounding boundary)."""
    z = golden('golden_mapping.npz')
    for tag in ('x16', 'x32', 'x64'):
        H, y, xq = z[tag + '/H'], z[tag + '/y'], z[tag + '/xq']
        for K in (1, 2):
            Gf, hf, scale = O.ising_delta_compressed(H, y, xq)
            np.testing.assert_allclose(scale, z['%s/K%d/scale' % (tag, K)], rtol=1e-5)
            G, h = O.quantize_compressed(Gf, hf)
            assert np.abs(G - z['%s/K%d/G' % (tag, K)]).max() <= 1
            assert np.abs(h - z['%s/K%d/h' % (tag, K)]).max() <= 1
            assert (G == z['%s/K%d/G' % (tag, K)]).mean() > 0.999


def test_readout_matches_reference(golden):
    z = golden('golden_mapping.npz')
    for tag in ('x16', 'x32', 'x64'):
        H, y, xq = z[tag + '/H'], z[tag + '/y'], z[tag + '/xq']
        for K in (1, 2):
            S = z['%s/K%d/S' % (tag, K)]
            Lc = O.spins_to_levels_delta(S, xq, K, 16)
            assert np.array_equal(Lc, z['%s/K%d/Lc' % (tag, K)])
            np.testing.assert_allclose(O.dist(H, y, Lc), z['%s/K%d/dist' % (tag, K)], rtol=1e-4, atol=1e-4)
            sel, _ = O.select(H, y, Lc, xq)
            assert np.array_equal(sel, z['%s/K%d/sel' % (tag, K)])
            assert np.array_equal(O.levels_to_bits(sel, 16), z['%s/K%d/bits' % (tag, K)])


def test_list_llr_restatement_matches_reference(golden):
    """The numpy list_llr (float64) against mimo.list_llr (float32 torch) on the golden candidate lists."""
    z = golden('golden_mapping.npz')
    for tag in ('x16', 'x32', 'x64'):
        H, y, xq, N0 = z[tag + '/H'], z[tag + '/y'], z[tag + '/xq'], float(z[tag + '/N0'][0])
        for K in (1, 2):
            Lc = O.spins_to_levels_delta(z['%s/K%d/S' % (tag, K)], xq, K, 16)
            allc = np.concatenate([Lc, xq[:, None, :]], 1)
            d = O.dist(H, y, allc)
            best = allc[np.arange(allc.shape[0]), d.argmin(1)]
            llr = O.list_llr(H, y, N0, allc, d, best, 16, clip=1e4)
            np.testing.assert_allclose(llr, z['%s/K%d/llr' % (tag, K)], rtol=1e-3, atol=2e-2)
