"""The RI map with first-accept annealing on the full J in FP32 fields (16 users x 16 antennas, 16-QAM, 64 spins
as 2 s1 + s2, 16 anneals per use started at the MMSE spins): the map against the float64 restatement of
mimo.ising, the anneal against the CPU FP32 restatement (>= 99.9% of anneals with identical decisions) with best
energies within 1e-5 relative of the FP64 recomputation, and the decisions against the CPU chain."""
import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _problem(B, snr, seed):
    from arpeggio_b200 import channel
    b = channel.draw(seed, snr, 0, B, 16, 16)
    return b, b['H'].numpy(), b['y'].numpy()


def test_ri_map_matches_float64_ising():
    from arpeggio_b200 import detector
    b, H, y = _problem(64, 12.0, 31)
    out = detector.detect_ri(b['H'], b['y'], 16, N0=b['N0'], anneals=2, sweeps=2)
    torch.cuda.synchronize()
    z, mu, xq = O.mmse(H, y, b['N0'], 16)
    hreg, h0, J, sP, scale = O.ising_ri(H, y, z, 16)
    assert np.array_equal(out['xq'].cpu().numpy(), xq.astype(np.int8))
    assert (out['sP'].cpu().numpy() == sP).mean() >= 0.999
    np.testing.assert_allclose(out['scale'].cpu().numpy(), scale, rtol=1e-5)
    np.testing.assert_allclose(out['J'].cpu().numpy(), J, rtol=2e-5, atol=2e-6)
    np.testing.assert_allclose(out['h0'].cpu().numpy(), h0, rtol=2e-5, atol=2e-6)
    ok = (out['sP'].cpu().numpy() == sP).all(-1)
    np.testing.assert_allclose(out['h'].cpu().numpy()[ok], hreg[ok], rtol=2e-5, atol=2e-6)


@pytest.mark.parametrize('policy,start', [('arpeggio', 'mmse'), ('arpeggio', 'rand'), ('chord', 'rand')])
def test_full_f32_anneal_vs_oracle_and_fp64_energy(policy, start):
    from arpeggio_b200 import detector
    b, H, y = _problem(128, 10.0, 32)
    R = 16
    out = detector.detect_ri(b['H'], b['y'], 16, N0=b['N0'], anneals=R, sweeps=32, T0=0.3, T1=0.05, q=0.0, seed=11,
                             start=start, policy=policy, kappa=0.3)
    torch.cuda.synchronize()
    J, h, sP = out['J'].cpu().numpy(), out['h'].cpu().numpy(), out['sP'].cpu().numpy()
    ws, wde, wst = O.anneal_full_f32(J, h, out['P'], R, out['T'], out['q'], np.arange(128), 11,
                                     sP if start == 'mmse' else None, policy, None, nthreads=8) if policy == 'arpeggio' \
        else O.anneal_full_f32(J, h, out['P'], R, out['T'], out['q'], np.arange(128), 11, None, policy,
                               detector.chord_schedule(64, 0.3, 0.05, 0.0, 0.3, precision='f32')[2], nthreads=8)
    s, de, st = out['spins'].cpu().numpy(), out['de'].cpu().numpy(), out['st'].cpu().numpy()
    same = (s == ws).all(-1) & (st == wst).all(-1) & (de == wde)
    assert same.mean() >= 0.999, same.mean()
    # best energies: start energy (FP64) + tracked change vs the FP64 energy of the best state
    if start == 'mmse':
        s0 = np.repeat(sP[:, None, :], R, 1)
    else:
        s0 = np.zeros((128, R, J.shape[1]), dtype=np.int8)
        for bb in range(128):
            for r in range(R):
                w = np.array([[0xFFFFFFFF, i, r, bb, 11, 0] for i in range(J.shape[1])])
                s0[bb, r] = np.where(O.philox(w)[:, 0] >= 2 ** 31, 1, -1)
    e_best = O.energy_full(h, J, s)
    e_start = O.energy_full(h, J, s0)
    rel = np.abs(e_start + de.astype(np.float64) - e_best) / np.maximum(np.abs(e_best), 1e-30)
    assert rel.max() <= 1e-5, rel.max()


def test_ri_detection_vs_cpu_chain():
    from arpeggio_b200 import detector
    b, H, y = _problem(256, 14.0, 33)
    out = detector.detect_ri(b['H'], b['y'], 16, N0=b['N0'], anneals=16, sweeps=64, seed=5)
    torch.cuda.synchronize()
    J, h, sP, xq = (out[k].cpu().numpy() for k in ('J', 'h', 'sP', 'xq'))
    ws, _, _ = O.anneal_full_f32(J, h, 2, 16, out['T'], out['q'], np.arange(256), 5, sP, nthreads=8)
    cand = 2 * ws[..., :16 * 2].astype(np.int64)[..., :32] + ws[..., 32:].astype(np.int64)
    sel, _ = O.select(H, y, cand, xq.astype(np.int64))
    assert (sel == out['levels'].cpu().numpy()).all(-1).mean() >= 0.99
    # the selection keeps the MMSE decision in the list, so the decision is never farther from y than it
    d_sel = out['dist'].cpu().numpy().astype(np.float64)
    d_mmse = O.dist(H, y, xq.astype(np.int64)[:, None, :])[:, 0]
    assert (d_sel <= d_mmse * (1 + 1e-5) + 1e-6).all()
