"""BER inside the reference's bootstrap CI at every recorded point: the multi-stage detector on the device, with
int32 fixed-point fields and with FP32 fields, on the same draws as the recorded B200 runs of the reference
(data/results/a513_fixed: x16 at 20 dB, x32 and x64 at 22 dB; fixture golden_a513_points.npz, made from those
records), against the 95 % cluster-bootstrap interval of the recorded per-use bit errors on the same uses
(stats.boot_ber restates stats_chord.boot_ber).  The fixed-point path also matches the record use by use."""
import numpy as np
import pytest

from arpeggio_b200 import stats

pytestmark = pytest.mark.gpu

# batches of each recorded point used here (of 200 / 300 / 600), keeping the run to seconds
BATCHES = {'x16': 100, 'x32': 100, 'x64': 30}


@pytest.fixture(scope='module')
def detected(golden):
    import torch
    from arpeggio_b200 import channel, mdi
    z = golden('golden_a513_points.npz')
    out = {}
    for tag, nb in BATCHES.items():
        nt, snr, seed, m = [v for v in z[tag + '/meta']]
        nt, seed, m = int(nt), int(seed), int(m)
        pick = str(z[tag + '/pick'])
        rec = z[tag + '/biterr'][:nb].astype(np.int64).reshape(-1)
        got = {}
        for prec in ('int', 'f32'):
            errs = []
            for bi in range(nb):
                b = channel.draw(seed, snr, bi, m, nt, 16)
                levels, _, _, _ = mdi.detect(b['H'], b['y'], b['N0'], 16, channel.draw_seed(seed, snr, bi), pick,
                                             precision=prec)
                bt = channel.levels_to_bits(b['l'], 16)
                bh = channel.levels_to_bits(levels.cpu().to(torch.float32), 16)
                errs.append((bt != bh).sum(-1).numpy())
            got[prec] = np.concatenate(errs).astype(np.int64)
        out[tag] = (rec, got, 4 * nt)
    return out


@pytest.mark.parametrize('tag', list(BATCHES))
@pytest.mark.parametrize('prec', ['int', 'f32'])
def test_ber_inside_reference_bootstrap_ci(detected, tag, prec):
    rec, got, bits = detected[tag]
    lo, hi, _ = stats.boot_ber(rec, bits, B=2000)
    ok, ber = stats.ber_inside(got[prec], bits, lo, hi)
    assert ok, (tag, prec, ber, lo, hi, rec.sum() / (len(rec) * bits))


@pytest.mark.parametrize('tag', list(BATCHES))
def test_fixed_point_matches_the_record_use_by_use(detected, tag):
    rec, got, _ = detected[tag]
    assert (got['int'] == rec).mean() >= 0.99
