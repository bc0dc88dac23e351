"""BER statistics and per-batch records against the reference's own analysis functions (golden_stats.npz)."""
import numpy as np

from arpeggio_b200 import records, stats


def test_boot_ber_matches_reference(golden):
    z = golden('golden_stats.npz')
    lo, hi, _ = stats.boot_ber(z['a'], 64, B=500)
    assert (lo, hi) == tuple(z['boot_ber'])


def test_boot_ratio_and_mcnemar_match_reference(golden):
    z = golden('golden_stats.npz')
    assert stats.boot_ratio(z['a'], z['b'], B=800) == tuple(z['boot_ratio'])
    p, x, y = stats.mcnemar(z['a'], z['b'])
    assert (p, x, y) == tuple(z['mcnemar'])


def test_ber_gate_and_cp():
    e = np.zeros(1000, dtype=np.int64)
    e[:5] = 1
    ok, ber = stats.ber_inside(e, 64, 0.0, 1e-4)
    assert ok and ber == 5 / 64000
    lo, hi = stats.cp_interval(5, 64000)
    assert lo < ber < hi


def test_records_roundtrip_and_resume(tmp_path):
    path = records.batch_path(str(tmp_path), 'x16', 'arpeggiofx_64_0.1_0.1_0_rand_32', 20.0, 3)
    assert path.endswith('x16/arpeggiofx_64_0.1_0.1_0_rand_32/snr_20.00/b00003.npz')
    assert not records.done(path)
    rng = np.random.default_rng(1)
    be = (rng.random(50) < 0.1).astype(np.int64) * 2
    lv = rng.choice([-3, -1, 1, 3], size=(50, 32))
    records.write_batch(path, be, lv, np.full(50, 228.0), dict(m=50, seed=102))
    assert records.done(path)
    r = records.read_batch(path)
    assert np.array_equal(r['biterr'], be.astype(np.uint8))
    assert np.array_equal(r['err_idx'], np.nonzero(be)[0])
    assert np.array_equal(r['xhat'], lv[be > 0].astype(np.int8))
    assert r['info'] == dict(m=50, seed=102)
    assert np.array_equal(records.point_biterr(str(tmp_path), 'x16', 'arpeggiofx_64_0.1_0.1_0_rand_32', 20.0),
                          be.astype(np.uint8))
