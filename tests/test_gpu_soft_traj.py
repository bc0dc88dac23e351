"""Trajectory soft output on the device: the sampler (arp_soft_trajectory) against the oracle's restatement with the
same Philox draws -- per-bit minima, best distance and best levels bit for bit -- and the chain's LLRs consistent with
its decision (QPSK and 16-QAM on the RI map, random and MMSE starts, a hot start)."""
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu
NTH = max(1, min(16, os.cpu_count() or 1))


@pytest.mark.parametrize('nt,M,R,S,warm,hot', [(16, 4, 8, 64, False, False), (16, 16, 12, 96, False, True),
                                               (32, 16, 9, 48, True, False), (24, 16, 4, 40, False, False)])
def test_soft_trajectory_equals_oracle(nt, M, R, S, warm, hot):
    from arpeggio_b200 import channel, soft
    B = 24
    b = channel.draw(500 + nt + M, 12.0, 0, B, nt, M)
    out = soft.detect_llr(b['H'], b['y'], b['N0'], M, R=R, S=S, tpost_mult=1.5, q=0.0,
                          t_hot=0.5 if hot else None, hot_frac=0.3 if hot else 0.0, warm=warm, seed=0xC0FFEE + nt,
                          inst0=7)
    torch.cuda.synchronize()
    c = lambda t: t.cpu().numpy()
    D = 2 * nt
    m0, m1, bd, bl = O.soft_trajectory(c(out['J']), c(out['h0']), c(out['h0']), c(out['scale']), c(out['c0']),
                                       c(out['T']), c(out['sP']) if warm else None, 0.0, S, R, D, M,
                                       c(out['inst']).view(np.uint32), 0xC0FFEE + nt, nthreads=NTH)
    assert np.array_equal(c(out['m0']), m0)
    assert np.array_equal(c(out['m1']), m1)
    assert np.array_equal(c(out['best_d']), bd)
    assert np.array_equal(c(out['best_l']), bl)
    # the LLR signs follow the decision's bits (the trajectory minima use the sampler's running float distance, the
    # list its exact one, as in the reference, so near-ties may differ)
    llr = out['llr']
    bits = soft.levels_to_bits(out['l_hat'], M).bool()
    assert torch.isfinite(llr).all()
    sure = llr.abs() > 0.1
    assert ((llr > 0) == bits)[sure].float().mean() >= 0.99
    # the best visited state is at least as close as the sampler reported
    d_best = soft.dist(b['H'].cuda(), b['y'].cuda(), out['best_l'].float()[:, None, :])[:, 0]
    assert torch.allclose(d_best, out['best_d'], rtol=1e-3, atol=1e-3)


def test_soft_trajectory_checks_shapes():
    from arpeggio_b200 import _lib
    L = _lib.lib()
    args = [None] * 7 + [0.0, 8, 4, 65, 16, 1, None, 0, 0, None, None, None, None, None]
    assert L.arp_soft_trajectory(*args) == 1  # N = 130 > 128
    args[11] = 64
    assert L.arp_soft_trajectory(*args) == 1  # 64-QAM is not on the reference's RI map
    args[11], args[10] = 16, 32
    assert L.arp_soft_trajectory(*args) == 3  # null pointers
