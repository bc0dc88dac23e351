"""Trajectory LLRs (CPU): arpeggio_b200.soft.trajectory_llr against the reference's own mimo.trajectory_llr
(arpeggio/mimo/mimo.py:397-413) on golden inputs made by tests/golden/make_golden.py (16-QAM and QPSK)."""
import os

import numpy as np
import pytest
import torch

from conftest import GOLDEN


@pytest.mark.parametrize('M', [16, 4])
def test_trajectory_llr_matches_reference(M):
    from arpeggio_b200 import soft
    z = np.load(os.path.join(GOLDEN, 'golden_trajectory.npz'))
    g = lambda k: torch.from_numpy(z['M%d/%s' % (M, k)])
    l_hat, llr = soft.trajectory_llr(g('H'), g('y'), float(z['M%d/N0' % M][0]), M, g('best_l'), g('best_d'), g('m0'),
                                     g('m1'), g('mmse'), clip=1e4)
    assert torch.equal(l_hat, g('l_hat'))
    ref = g('llr')
    assert torch.isfinite(llr).all()
    np.testing.assert_allclose(llr.numpy(), ref.numpy(), rtol=1e-5, atol=1e-4 * float(ref.abs().max()))


def test_neighbours_flip_one_gray_bit():
    from arpeggio_b200 import soft
    l = torch.tensor([[-3., -1., 1., 3.]])
    nb = soft.neighbours(l, 16)
    b0 = soft.levels_to_bits(l, 16)
    bn = soft.levels_to_bits(nb, 16)
    diff = (bn != b0[:, None, :]).sum(-1)
    assert (diff == 1).all()  # every neighbour differs in exactly one bit
    assert (bn != b0[:, None, :]).float().argmax(-1).tolist() == [list(range(8))]  # bit k of neighbour k
