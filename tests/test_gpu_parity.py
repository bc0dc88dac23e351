"""GPU parity: every kernel through the C ABI against the reference's outputs (fixtures) and the CPU oracle.

Integer paths are bit-exact; FP32-field anneals must take the same flip decisions on >= 99.9% of anneals and
track energies within 1e-5 relative of an FP64 recomputation; the float mapping stage must give the
reference's hard guess and (nearly) its integer coefficients."""
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O

from conftest import GOLDEN

pytestmark = pytest.mark.gpu
NTH = max(1, min(16, os.cpu_count() or 1))


def _names(f):
    return [str(n) for n in np.load(os.path.join(GOLDEN, f))['names']]


def _u32(x):
    return torch.as_tensor(np.asarray(x, dtype=np.int64) & 0xFFFFFFFF).to(torch.int32).cuda()


def test_device_philox_kat(golden):
    from arpeggio_b200 import chordfx
    z = golden('golden_philox.npz')
    k = chordfx.Kernel()
    for a, b in (('kat_in', 'kat_out'), ('rnd_in', 'rnd_out')):
        out = k.philox_kat(torch.from_numpy(z[a].astype(np.int64))).cpu().numpy()
        assert np.array_equal(out.astype(np.uint32), z[b])


@pytest.mark.parametrize('name', _names('golden_arpeggio.npz'))
def test_first_accept_bit_exact_vs_reference(golden, name):
    """arpeggiofx.solve (reference contract) == arpeggio_ref59.anneal outputs."""
    from arpeggio_b200 import arpeggiofx
    z = golden('golden_arpeggio.npz')
    P, R, q, k0, k1, st = [int(v) for v in z[name + '/meta']]
    s, de, stt = arpeggiofx.solve(z[name + '/G'], z[name + '/h'], P, R, [int(v) for v in z[name + '/T']], q,
                                  z[name + '/inst'], k0 | (k1 << 32), 'rand' if st == 0 else 'bal')
    assert np.array_equal(s, z[name + '/arpeggio/spins'])
    assert np.array_equal(de, z[name + '/arpeggio/de'])
    assert np.array_equal(stt, z[name + '/arpeggio/st'])


def _device_problem(z, name):
    G = torch.from_numpy(z[name + '/G']).cuda()
    return (G.transpose(1, 2).contiguous(), torch.from_numpy(z[name + '/h']).cuda(),
            torch.from_numpy(z[name + '/T']).cuda(), _u32(z[name + '/inst']))


@pytest.mark.parametrize('name', _names('golden_arpeggio.npz'))
def test_chord_round_bit_exact_vs_reference(golden, name):
    """policy='chord' on the compressed problem == arpeggio_ref59.anneal mode 'par'."""
    from arpeggio_b200 import arpeggiofx
    z = golden('golden_arpeggio.npz')
    P, R, q, k0, k1, st = [int(v) for v in z[name + '/meta']]
    Gt, h, T, inst = _device_problem(z, name)
    s, de, stt, status = arpeggiofx.anneal(Gt, h, P, R, T, q, inst, k0 | (k1 << 32), 'rand' if st == 0 else 'bal',
                                           policy='chord')
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    assert np.array_equal(s.cpu().numpy(), z[name + '/par/spins'])
    assert np.array_equal(de.cpu().numpy(), z[name + '/par/de'])
    assert np.array_equal(stt.cpu().numpy(), z[name + '/par/st'])


@pytest.mark.parametrize('name', _names('golden_chord.npz'))
@pytest.mark.parametrize('mode', ['chains', 'best'])
def test_chord_full_bit_exact_vs_chord_fx(golden, name, mode):
    """Kernel.chord (reference contract, full int16 J) == chordfx.chord_fx outputs."""
    from arpeggio_b200 import chordfx
    z = golden('golden_chord.npz')
    q, S, P, R, s0, s1, inst0 = [int(v) for v in z[name + '/meta']]
    F = dict(J=torch.from_numpy(z[name + '/J']), h=torch.from_numpy(z[name + '/h']),
             h0=torch.from_numpy(z[name + '/h0']), T=torch.from_numpy(z[name + '/T']),
             c=torch.from_numpy(z[name + '/c']), q=q, S=S)
    k = chordfx.Kernel()
    stats = torch.zeros(4, dtype=torch.int64, device='cuda')
    s, e = k.chord(F, R, s0 | (s1 << 32), P=P, inst0=inst0, mode=mode, stats=stats)
    torch.cuda.synchronize()
    assert int(k.last_status.item()) == 0
    assert np.array_equal(s.cpu().numpy(), z['%s/%s_s' % (name, mode)])
    assert np.array_equal(e.cpu().numpy(), z['%s/%s_e' % (name, mode)])
    assert int(stats[3].item()) == S * R * F["h"].shape[0]


@pytest.mark.parametrize('N,P,R,S,kappa,offset,warps', [
    (256, 2, 64, 64, 0.3, 0, 0),    # 16 warps per block (one block per SM)
    (256, 1, 24, 40, 0.3, 0, 0),    # one phase: the Onsager sign of the previous step's flips
    (256, 8, 16, 48, 0.0, 1, 0),    # eight phases; J one element off a 16-byte boundary (plain-load staging)
    (192, 3, 20, 30, 0.3, 0, 5),    # a given width that is not a power of two
    (64, 2, 40, 100, 0.3, 0, 0),    # a partial last quad of sweeps
])
def test_chord_full_vs_oracle_wide(N, P, R, S, kappa, offset, warps):
    """arp_anneal_chord on dDI problems expanded to a full int16 J (chord_ref.expand) against the oracle's chord_fx
    restatement: spins, energies and counters bit for bit in both modes, at block widths and phase counts the golden
    cases do not reach."""
    from arpeggio_b200 import chordfx
    B, D = 12, N // 2
    G, h, _, _ = _random_dd(B, D, 1, 12.0, 300 + N + P)
    J, hN = O.expand(G, h, 1)  # the phases P need not be the dDI copy count: the kernel takes any J
    h0 = (hN // 3).astype(np.int32)
    T, c, q = O.chord_schedule(S, 0.3, 0.05, 0.4, kappa=kappa)
    seed, inst0 = 0x1234ABCD5678 + N, 0xFFFFFFF0
    Jd = torch.zeros(B * N * N + offset, dtype=torch.int16, device='cuda')
    Jd[offset:] = torch.from_numpy(J.reshape(-1))
    F = dict(J=Jd[offset:].view(B, N, N), h=torch.from_numpy(hN).cuda(), h0=torch.from_numpy(h0).cuda(),
             T=torch.from_numpy(T).cuda(), c=torch.from_numpy(c).cuda(), q=q, S=S)
    if offset:
        assert F['J'].data_ptr() % 16 != 0
    k = chordfx.Kernel()
    for mode in ('chains', 'best'):
        stats = torch.zeros(4, dtype=torch.int64, device='cuda')
        s, e = k.chord(F, R, seed, P=P, inst0=inst0, mode=mode, warps=warps, stats=stats)
        torch.cuda.synchronize()
        assert int(k.last_status.item()) == 0
        os_, oe = O.chord_fx(J, hN, h0, T, c, q, S, P, R, seed, inst0=inst0, mode=mode, nthreads=NTH)
        assert np.array_equal(s.cpu().numpy(), os_), mode
        assert np.array_equal(e.cpu().numpy(), oe), mode
        assert int(stats[3].item()) == S * R * B


def _random_dd(B, D, K, snr, seed):
    """Realistic compressed integer dDI problems from this package's draws and the oracle's float64 mapping."""
    from arpeggio_b200 import channel
    b = channel.draw(seed, snr, 0, B, D // 2, 16)
    _, _, xq = O.mmse(b['H'].numpy(), b['y'].numpy(), b['N0'], 16)
    Gf, hf, _ = O.ising_delta_compressed(b['H'].numpy(), b['y'].numpy(), xq)
    G, h = O.quantize_compressed(Gf, hf)
    return G, h, Gf.astype(np.float32), hf.astype(np.float32)


@pytest.mark.parametrize('D,K,R,S,start,policy', [
    (64, 1, 32, 32, 'rand', 'arpeggio'),    # x32 pick (abl_far_32_0.1_0.1_0_rand_8)
    (32, 1, 16, 64, 'rand', 'arpeggio'),    # x16 pick
    (128, 1, 8, 16, 'bal', 'arpeggio'),     # x64 pick, shortened
    (64, 2, 8, 8, 'bal', 'arpeggio'),
    (96, 3, 4, 4, 'rand', 'arpeggio'),
    (64, 1, 32, 128, 'rand', 'chord'),      # Chord MDI schedule (128 steps per copy pair)
    (128, 2, 4, 32, 'bal', 'chord'),
])
def test_anneal_vs_oracle_at_scale(D, K, R, S, start, policy):
    """Bit-exact against the oracle on hundreds of real sub-problems per shape."""
    from arpeggio_b200 import arpeggiofx
    from arpeggio_b200.detector import arpeggio_schedule, chord_schedule
    B = 96 if D >= 96 else 256
    G, h, _, _ = _random_dd(B, D, K, 14.0, 1000 + D + K)
    P = 2 * K
    if policy == 'arpeggio':
        T, q, c = arpeggio_schedule(S, 0.1, 0.1, 0.0, K)
    else:
        T, q, c = chord_schedule(S * P, 0.3, 0.3, 0.4, kappa=0.3)
    key = 0xC0FFEE1234567 + D
    inst = np.arange(B, dtype=np.int64) + 17
    ws, wde, wst = O.anneal_dd(G, h, P, R, T, q, inst, key, start, policy=policy, c=c, nthreads=NTH)
    Gt = torch.from_numpy(G).cuda().transpose(1, 2).contiguous()
    s, de, st, status = arpeggiofx.anneal(Gt, torch.from_numpy(h).cuda(), P, R,
                                          torch.tensor(T, dtype=torch.int32, device='cuda'), q, _u32(inst), key,
                                          start, policy, None if c is None else
                                          torch.tensor(c, dtype=torch.int32, device='cuda'))
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    assert np.array_equal(s.cpu().numpy(), ws)
    assert np.array_equal(de.cpu().numpy(), wde)
    assert np.array_equal(st.cpu().numpy(), wst)


@pytest.mark.parametrize('D,K,B,start,policy', [
    (2, 1, 5, 'rand', 'arpeggio'),
    (14, 3, 70, 'bal', 'arpeggio'),
    (40, 1, 64, 'rand', 'arpeggio'),     # at most 64 problems: the launch without the register bound
    (40, 1, 65, 'rand', 'arpeggio'),     # one more: the bounded kernel
    (70, 2, 65, 'rand', 'chord'),
    (100, 1, 33, 'bal', 'arpeggio'),
    (126, 3, 9, 'rand', 'chord'),
])
def test_ragged_sizes_vs_oracle(D, K, B, start, policy):
    """Coordinate counts that leave padding lanes (not a multiple of 32), odd batch sizes on both sides of the
    small-batch launch, every copy count: bit-exact against the oracle."""
    from arpeggio_b200 import arpeggiofx
    from arpeggio_b200.detector import arpeggio_schedule, chord_schedule
    R, S = 8, 8
    G, h, _, _ = _random_dd(B, D, K, 12.0, 3000 + D * 7 + B)
    P = 2 * K
    if policy == 'arpeggio':
        T, q, c = arpeggio_schedule(S, 0.1, 0.1, 0.0, K)
    else:
        T, q, c = chord_schedule(S * P, 0.3, 0.3, 0.4, kappa=0.3)
    key = 0x5EEDF00D + D + B
    inst = np.arange(B, dtype=np.int64) + 3
    ws, wde, wst = O.anneal_dd(G, h, P, R, T, q, inst, key, start, policy=policy, c=c, nthreads=NTH)
    Gt = torch.from_numpy(G).cuda().transpose(1, 2).contiguous()
    s, de, st, status = arpeggiofx.anneal(Gt, torch.from_numpy(h).cuda(), P, R,
                                          torch.tensor(T, dtype=torch.int32, device='cuda'), q, _u32(inst), key,
                                          start, policy, None if c is None else
                                          torch.tensor(c, dtype=torch.int32, device='cuda'))
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    assert np.array_equal(s.cpu().numpy(), ws)
    assert np.array_equal(de.cpu().numpy(), wde)
    assert np.array_equal(st.cpu().numpy(), wst)


def _start_spins(B, R, P, D, key, start, inst):
    """Start states by the reference's counters (arpeggio_fx.cu:48-57), for the FP64 energy check."""
    k0, k1 = key & 0xFFFFFFFF, key >> 32
    s = np.zeros((B, R, P, D), dtype=np.int8)
    for b in range(B):
        for r in range(R):
            if start == 'rand':
                w = np.array([[0xFFFFFFFF, p * D + j, r, inst[b], k0, k1] for p in range(P) for j in range(D)])
                s[b, r] = np.where(O.philox(w)[:, 0] >= 2 ** 31, 1, -1).reshape(P, D)
            else:
                s[b, r] = 0  # balanced: every coordinate has P/2 copies up, m = 0
    return s.reshape(B, R, P * D)


@pytest.mark.parametrize('policy', ['arpeggio', 'chord'])
@pytest.mark.parametrize('D,K,start', [(64, 1, 'rand'), (128, 1, 'bal'), (32, 3, 'rand')])
def test_f32_fields_vs_oracle(policy, D, K, start):
    """FP32 fields: >= 99.9% of anneals take identical decisions (same flips, tests, best state) as the CPU
    FP32 restatement; best energies within 1e-5 relative of the FP64 recomputation."""
    from arpeggio_b200 import arpeggiofx
    from arpeggio_b200.detector import arpeggio_schedule, chord_schedule
    B, R, P = 64, 16, 2 * K
    _, _, Gf, hf = _random_dd(B, D, K, 16.0, 2000 + D)
    if policy == 'arpeggio':
        T, q, c = arpeggio_schedule(16, 0.3, 0.05, 0.0, K, precision='f32')
    else:
        T, q, c = chord_schedule(32 * P, 0.3, 0.3, 0.4, kappa=0.3, precision='f32')
    key, inst = 0xFEEDF00D + D, np.arange(B, dtype=np.int64)
    ws, wde, wst = O.anneal_dd_f32(Gf, hf, P, R, T, q, inst, key, start, policy=policy, c=c, nthreads=NTH)
    Gt = torch.from_numpy(Gf).cuda().transpose(1, 2).contiguous()
    s, de, st, status = arpeggiofx.anneal(Gt, torch.from_numpy(hf).cuda(), P, R,
                                          torch.tensor(T, dtype=torch.float32, device='cuda'), q, _u32(inst), key,
                                          start, policy,
                                          None if c is None else torch.tensor(c, dtype=torch.float32, device='cuda'),
                                          precision='f32')
    torch.cuda.synchronize()
    assert int(status.item()) == 0
    s, de, st = s.cpu().numpy(), de.cpu().numpy(), st.cpu().numpy()
    same = (s == ws).all(-1) & (st == wst).all(-1) & (de == wde)
    assert same.mean() >= 0.999, 'identical anneals %.4f' % same.mean()
    s0 = _start_spins(B, R, P, D, key, start, inst)
    e_best = 2 * O.energy_dd(Gf, hf, s, K)
    e_start = 2 * O.energy_dd(Gf, hf, s0, K)
    final = e_start + de.astype(np.float64)
    rel = np.abs(final - e_best) / np.maximum(np.abs(e_best), 1e-30)
    assert rel.max() <= 1e-5, rel.max()


def test_map_vs_reference(golden):
    """arp_map_dd on the reference's draws: the same hard MMSE guess, scale within 1e-5, integer G/h equal on
    >= 99.9% of entries and never off by more than one unit."""
    from arpeggio_b200 import _lib
    z = golden('golden_mapping.npz')
    L = _lib.lib()
    for tag in ('x16', 'x32', 'x64'):
        H = torch.from_numpy(z[tag + '/H']).cuda().contiguous()
        y = torch.from_numpy(z[tag + '/y']).cuda().contiguous()
        B, NR2, D = H.shape
        N0 = float(z[tag + '/N0'][0])
        s2 = torch.full((B,), (N0 / 2) / 5.0, dtype=torch.float32, device='cuda')
        G = torch.empty(B, D, D, dtype=torch.int32, device='cuda')
        h = torch.empty(B, D, dtype=torch.int32, device='cuda')
        xq = torch.empty(B, D, dtype=torch.int8, device='cuda')
        sc = torch.empty(B, dtype=torch.float32, device='cuda')
        _lib.check(L.arp_map_dd(_lib.ptr(H), _lib.ptr(y), _lib.ptr(s2), B, NR2, D, 16, 1, _lib.ptr(G), _lib.ptr(h),
                                _lib.ptr(xq), _lib.ptr(sc), None, _lib.stream_ptr()), 'map')
        torch.cuda.synchronize()
        assert np.array_equal(xq.cpu().numpy(), z[tag + '/xq'].astype(np.int8)), tag
        np.testing.assert_allclose(sc.cpu().numpy(), z[tag + '/K1/scale'], rtol=1e-5)
        Gr, hr = z[tag + '/K1/G'], z[tag + '/K1/h']
        Gg, hg = G.cpu().numpy(), h.cpu().numpy()
        assert np.abs(Gg - Gr).max() <= 1 and np.abs(hg - hr).max() <= 1, tag
        assert (Gg == Gr).mean() >= 0.999 and (hg == hr).mean() >= 0.99, tag


@pytest.mark.parametrize('nt,nr,M', [(8, 8, 16), (16, 16, 16), (32, 32, 16), (24, 36, 64), (48, 72, 4), (64, 64, 16),
                                     (64, 128, 16)])
def test_map_gram_is_exact(nt, nr, M):
    """The Gram formed on the tensor cores (8-bit digit products, exact integer accumulation): the float problem's
    G = Q / scale equals the oracle's restatement of the digit scheme (oracle.gram_digits) bit for bit, is exactly
    symmetric, and stays within two float32 roundings plus 2^-24 of the problem's largest |G| of the float64 Gram,
    at every map width and row count."""
    from arpeggio_b200 import _lib, channel
    B = 64
    b = channel.draw(900 + nt, 14.0, 0, B, nt, M, nr=nr)
    H = b['H'].cuda().contiguous()
    y = b['y'].cuda().contiguous()
    _, NR2, D = H.shape
    s2 = torch.full((B,), 0.05, dtype=torch.float32, device='cuda')
    G = torch.empty(B, D, D, dtype=torch.float32, device='cuda')
    h = torch.empty(B, D, dtype=torch.float32, device='cuda')
    xq = torch.empty(B, D, dtype=torch.int8, device='cuda')
    sc = torch.empty(B, dtype=torch.float32, device='cuda')
    L = _lib.lib()
    _lib.check(L.arp_map_dd(_lib.ptr(H), _lib.ptr(y), _lib.ptr(s2), B, NR2, D, M, 0, _lib.ptr(G), _lib.ptr(h),
                            _lib.ptr(xq), _lib.ptr(sc), None, _lib.stream_ptr()), 'map')
    torch.cuda.synchronize()
    Gg, scg = G.cpu().numpy(), sc.cpu().numpy()
    assert np.array_equal(Gg, np.swapaxes(Gg, 1, 2))
    Qo = O.gram_digits(b['H'].numpy())
    assert np.array_equal(Gg, (Qo / scg[:, None, None]).astype(np.float32))
    Hd = b['H'].numpy().astype(np.float64)
    ref = np.einsum('bki,bkj->bij', Hd, Hd) / scg[:, None, None]
    ulp = np.spacing(np.abs(ref).astype(np.float32)).astype(np.float64)
    tol = ulp + 2.0 ** -24 * np.abs(ref).reshape(B, -1).max(-1)[:, None, None]  # two roundings + dropped digits
    assert (np.abs(Gg.astype(np.float64) - ref) <= tol).all()


def test_readout_vs_reference(golden):
    """arp_readout_dd on fixed spin sets == mimo.spins_to_levels_delta + select + levels_to_bits."""
    from arpeggio_b200 import _lib
    z = golden('golden_mapping.npz')
    L = _lib.lib()
    for tag in ('x16', 'x32', 'x64'):
        for K in (1, 2):
            H = torch.from_numpy(z[tag + '/H']).cuda().contiguous()
            y = torch.from_numpy(z[tag + '/y']).cuda().contiguous()
            B, NR2, D = H.shape
            S = torch.from_numpy(z['%s/K%d/S' % (tag, K)]).cuda().contiguous()
            R = S.shape[1]
            xq = torch.from_numpy(z[tag + '/xq'].astype(np.int8)).cuda()
            lv = torch.empty(B, D, dtype=torch.int8, device='cuda')
            bits = torch.empty(B, 2 * D, dtype=torch.int8, device='cuda')
            dist = torch.empty(B, dtype=torch.float32, device='cuda')
            pick = torch.empty(B, dtype=torch.int32, device='cuda')
            _lib.check(L.arp_readout_dd(_lib.ptr(H), _lib.ptr(y), _lib.ptr(xq), _lib.ptr(S), B, NR2, D, 2 * K, R, 16,
                                        _lib.ptr(lv), _lib.ptr(bits), _lib.ptr(dist), _lib.ptr(pick),
                                        _lib.stream_ptr()), 'readout')
            torch.cuda.synchronize()
            assert np.array_equal(lv.cpu().numpy(), z['%s/K%d/sel' % (tag, K)]), (tag, K)
            assert np.array_equal(bits.cpu().numpy(), z['%s/K%d/bits' % (tag, K)]), (tag, K)
            dref = np.concatenate([z['%s/K%d/dist' % (tag, K)],
                                   O.dist(z[tag + '/H'], z[tag + '/y'], z[tag + '/xq'][:, None, :])], 1).min(1)
            np.testing.assert_allclose(dist.cpu().numpy(), dref, rtol=1e-4, atol=1e-5)


def test_detector_matches_oracle_chain():
    """The three-launch detector on reference draws vs the CPU chain (float64 mapping, oracle anneal,
    select): the same decisions on >= 99% of uses and the same bit-error count within a few bits."""
    from arpeggio_b200 import channel, detector
    B, nt, snr, R = 512, 16, 16.0, 16
    b = channel.draw(4242, snr, 0, B, nt, 16)
    out = detector.detect(b['H'], b['y'], 16, snr_db=snr, policy='arpeggio', anneals=R, seed=99)
    H, y = b['H'].numpy(), b['y'].numpy()
    _, _, xq = O.mmse(H, y, b['N0'], 16)
    Gf, hf, _ = O.ising_delta_compressed(H, y, xq)
    G, h = O.quantize_compressed(Gf, hf)
    T, q, _ = detector.arpeggio_schedule(64, 0.1, 0.1, 0.0, 1)
    s, _, _ = O.anneal_dd(G, h, 2, R, T, q, np.arange(B), 99, 'rand', nthreads=NTH)
    cand = O.spins_to_levels_delta(s, xq, 1, 16)
    sel, _ = O.select(H, y, cand, xq)
    agree = (sel == out['levels']).all(-1).mean()
    assert agree >= 0.99, agree
    bt = O.levels_to_bits(b['l'].numpy(), 16)
    e_gpu = int((O.levels_to_bits(out['levels'], 16) != bt).sum())
    e_cpu = int((O.levels_to_bits(sel, 16) != bt).sum())
    assert abs(e_gpu - e_cpu) <= max(4, 0.05 * e_cpu), (e_gpu, e_cpu)
    assert np.array_equal(out['bits'], O.levels_to_bits(out['levels'], 16))


def test_range_error_is_reported_not_faulted():
    """Coefficients beyond the exact 32-bit field range: the kernel writes ARP_ERR_RANGE and skips the problem."""
    from arpeggio_b200 import arpeggiofx, _lib
    B, D, P, R = 2, 32, 2, 2
    Gt = torch.zeros(B, D, D, dtype=torch.int32, device='cuda')
    Gt[1, 3, 5] = 1 << 20
    h = torch.zeros(B, D, dtype=torch.int32, device='cuda')
    T = torch.full((4,), 400, dtype=torch.int32, device='cuda')
    s, de, st, status = arpeggiofx.anneal(Gt, h, P, R, T, 0, _u32(np.arange(B)), 1, 'rand')
    torch.cuda.synchronize()
    assert int(status.item()) == 2
    with pytest.raises(_lib.ArpError):
        arpeggiofx.check_status(status)


def test_side_stream_and_repeatability():
    """Stream-ordered on a side stream; two runs give identical results (counter-based RNG)."""
    from arpeggio_b200 import channel, detector
    b = channel.draw_device(5, 18.0, 300, 32, 16)
    det = detector.Detector(300, 32, anneals=8)
    det.set_noise(18.0)
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        o1 = [x.clone() for x in det.run(b['H'], b['y'], seed=3, stream=st)]
        o2 = [x.clone() for x in det.run(b['H'], b['y'], seed=3, stream=st)]
    st.synchronize()
    det.check()
    for a_, b_ in zip(o1, o2):
        assert torch.equal(a_, b_)


def test_pipelined_host_path_equals_one_run():
    """Detector.run_host (pinned host buffers, pieces overlapped with copies) gives exactly the one-run outputs."""
    from arpeggio_b200 import channel, detector
    B = 1000
    d = channel.draw_device(11, 12.0, B, 32, 16)
    det = detector.Detector(B, 32, anneals=8)
    det.set_noise(12.0)
    bits, levels, dist = [x.clone() for x in det.run(d['H'], d['y'], seed=5)]
    Hh, yh = d['H'].cpu().pin_memory(), d['y'].cpu().pin_memory()
    bo = torch.empty(bits.shape, dtype=torch.int8).pin_memory()
    do = torch.empty(B, dtype=torch.float32).pin_memory()
    det.run_host(Hh, yh, 5, bo, do, torch.empty_like(d['H']), torch.empty_like(d['y']), chunks=7)
    torch.cuda.synchronize()
    det.check()
    assert torch.equal(bo, bits.cpu())
    assert torch.equal(do, dist.cpu())
    # back-to-back calls on the detector's own two staging buffers (the next batch's copy overlaps this batch's
    # detection): every call's outputs equal its one-run outputs, also with other inputs in between
    d2 = channel.draw_device(12, 14.0, B, 32, 16)
    H2h, y2h = d2['H'].cpu().pin_memory(), d2['y'].cpu().pin_memory()
    outs = [(torch.empty(bits.shape, dtype=torch.int8).pin_memory(), torch.empty(B, dtype=torch.float32).pin_memory())
            for _ in range(4)]
    for i, (o_b, o_d) in enumerate(outs):
        hh, yy = (Hh, yh) if i % 2 == 0 else (H2h, y2h)
        det.run_host(hh, yy, 5 + i, o_b, o_d, chunks=1 + i)
    torch.cuda.synchronize()
    det.check()
    for i, (o_b, o_d) in enumerate(outs):
        dd = d if i % 2 == 0 else d2
        rb, _, rd = det.run(dd['H'], dd['y'], seed=5 + i)
        torch.cuda.synchronize()
        assert torch.equal(o_b, rb.cpu()) and torch.equal(o_d, rd.cpu()), i


def test_fused_c_entry_equals_staged_calls():
    """arp_detect_dd (one C call, caller workspace) == the three stage entries with per-stage events."""
    from arpeggio_b200 import channel, detector
    for policy, precision in (('arpeggio', 'int'), ('chord', 'int'), ('arpeggio', 'f32')):
        B = 700
        d = channel.draw_device(21, 10.0, B, 16, 16)
        det = detector.Detector(B, 16, anneals=6, policy=policy, precision=precision)
        det.set_noise(10.0)
        fused = [x.clone() for x in det.run(d['H'], d['y'], seed=9)] + [det.spins.clone()]
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        staged = [x.clone() for x in det.run(d['H'], d['y'], seed=9, events=ev)] + [det.spins.clone()]
        torch.cuda.synchronize()
        det.check()
        for a_, b_ in zip(fused, staged):
            assert torch.equal(a_, b_), (policy, precision)


def test_small_batch_split_and_graph_replay():
    """A batch smaller than the GPU splits each problem's anneals over blocks; results equal the oracle's, and a
    captured single-frame graph gives the same outputs as a direct run."""
    from arpeggio_b200 import channel, detector
    B, R = 3, 32
    b = channel.draw(55, 12.0, 0, B, 32, 16)
    det = detector.Detector(B, 32, anneals=R)
    det.set_noise(12.0)
    bits, levels, dist = [x.clone() for x in det.run(b['H'].cuda(), b['y'].cuda(), seed=77)]
    torch.cuda.synchronize()
    det.check()
    T, q = det.schedule['T'], det.schedule['q']
    ws, wde, wst = O.anneal_dd(det.G.cpu().numpy(), det.h.cpu().numpy(), 2, R, T, q, np.arange(B), 77, 'rand',
                               nthreads=NTH)
    assert np.array_equal(det.spins.cpu().numpy(), ws)
    assert np.array_equal(det.de.cpu().numpy(), wde)
    assert np.array_equal(det.st.cpu().numpy(), wst)
    Hh, yh = b['H'].pin_memory(), b['y'].pin_memory()
    bo = torch.empty(bits.shape, dtype=torch.int8).pin_memory()
    do = torch.empty(B, dtype=torch.float32).pin_memory()
    g = det.capture(Hh, yh, 77, bo, do, torch.empty_like(b['H'].cuda()), torch.empty_like(b['y'].cuda()))
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(bo, bits.cpu()) and torch.equal(do, dist.cpu())


def test_soft_output_llr_vs_reference(golden):
    """arp_readout_llr_dd == mimo.list_llr (the reference's dDI soft detector, softlib.detect_llr 'aned') on the
    golden candidate lists: the same decision and LLRs within the float32 tolerance of differences of distances."""
    from arpeggio_b200 import _lib
    z = golden('golden_mapping.npz')
    L = _lib.lib()
    for tag in ('x16', 'x32', 'x64'):
        for K in (1, 2):
            H = torch.from_numpy(z[tag + '/H']).cuda().contiguous()
            y = torch.from_numpy(z[tag + '/y']).cuda().contiguous()
            B, NR2, D = H.shape
            S = torch.from_numpy(z['%s/K%d/S' % (tag, K)]).cuda().contiguous()
            R = S.shape[1]
            xq = torch.from_numpy(z[tag + '/xq'].astype(np.int8)).cuda()
            N0 = torch.full((B,), float(z[tag + '/N0'][0]), dtype=torch.float32, device='cuda')
            lv = torch.empty(B, D, dtype=torch.int8, device='cuda')
            bits = torch.empty(B, 2 * D, dtype=torch.int8, device='cuda')
            dist = torch.empty(B, dtype=torch.float32, device='cuda')
            llr = torch.empty(B, 2 * D, dtype=torch.float32, device='cuda')
            _lib.check(L.arp_readout_llr_dd(_lib.ptr(H), _lib.ptr(y), _lib.ptr(xq), _lib.ptr(S), B, NR2, D, 2 * K, R,
                                            16, _lib.ptr(N0), 1e4, _lib.ptr(lv), _lib.ptr(bits), _lib.ptr(dist), None,
                                            _lib.ptr(llr), _lib.stream_ptr()), 'readout_llr')
            torch.cuda.synchronize()
            assert np.array_equal(lv.cpu().numpy(), z['%s/K%d/sel' % (tag, K)]), (tag, K)
            np.testing.assert_allclose(llr.cpu().numpy(), z['%s/K%d/llr' % (tag, K)], rtol=1e-3, atol=5e-2)


def test_detector_soft_output_vs_oracle():
    """Detector.run_soft: LLRs of the GPU's own candidate list equal the numpy list_llr over the same list."""
    from arpeggio_b200 import channel, detector
    B, nt, snr = 200, 16, 10.0
    b = channel.draw(808, snr, 0, B, nt, 16)
    det = detector.Detector(B, nt, anneals=8)
    det.set_noise(snr)
    bits, levels, dist, llr = det.run_soft(b['H'].cuda(), b['y'].cuda(), 4, b['N0'])
    torch.cuda.synchronize()
    det.check()
    H, y = b['H'].numpy(), b['y'].numpy()
    xq = det.xq.cpu().numpy().astype(np.int64)
    cand = O.spins_to_levels_delta(det.spins.cpu().numpy(), xq, 1, 16)
    allc = np.concatenate([cand, xq[:, None, :]], 1)
    d = O.dist(H, y, allc)
    best = allc[np.arange(B), d.argmin(1)]
    assert (best == levels.cpu().numpy()).all(-1).mean() >= 0.99
    ref = O.list_llr(H, y, b['N0'], allc, d, levels.cpu().numpy().astype(np.int64), 16, clip=1e4)
    np.testing.assert_allclose(llr.cpu().numpy(), ref, rtol=1e-3, atol=5e-2)
    # a bit whose LLR disagrees with the decision can only come from a bit-flip neighbour closer to y than every
    # list entry (the decision is the list's minimum)
    lv, bh = llr.cpu().numpy(), bits.cpu().numpy().astype(bool)
    nb = O.gray_neighbours(levels.cpu().numpy().astype(np.int64), 16)
    dn = O.dist(H, y, nb)
    closer = dn < dist.cpu().numpy().astype(np.float64)[:, None] * (1 - 1e-4)
    assert not ((lv > 0) != bh)[~closer.any(1)].any()


def test_64qam_detection_vs_oracle_chain():
    """64-QAM (3 Gray bits per dimension; no reference counterpart, so the check is the oracle's own chain):
    the same decisions on >= 99% of uses, levels odd in [-7, 7], bits the Gray code of the levels."""
    from arpeggio_b200 import channel, detector
    B, nt, snr, R = 256, 16, 24.0, 16
    b = channel.draw(6464, snr, 0, B, nt, 64)
    out = detector.detect(b['H'], b['y'], 64, snr_db=snr, policy='arpeggio', anneals=R, seed=3, sweeps=32)
    H, y = b['H'].numpy(), b['y'].numpy()
    _, _, xq = O.mmse(H, y, b['N0'], 64)
    assert (xq == out['xq']).mean() >= 0.999
    Gf, hf, _ = O.ising_delta_compressed(H, y, out['xq'].astype(np.int64))
    G, h = O.quantize_compressed(Gf, hf)
    T, q, _ = detector.arpeggio_schedule(32, 0.1, 0.1, 0.0, 1)
    s, _, _ = O.anneal_dd(G, h, 2, R, T, q, np.arange(B), 3, 'rand', nthreads=NTH)
    lo = out['levels']
    assert set(np.unique(lo)) <= {-7, -5, -3, -1, 1, 3, 5, 7}
    cand = np.clip(out['xq'][:, None, :].astype(np.int64) + s.reshape(B, R, 2, -1).sum(2), -7, 7)
    sel, _ = O.select(H, y, cand, out['xq'].astype(np.int64))
    assert (sel == lo).all(-1).mean() >= 0.99
    assert np.array_equal(out['bits'], O.levels_to_bits(lo, 64))
    ber = (O.levels_to_bits(lo, 64) != O.levels_to_bits(b['l'].numpy(), 64)).mean()
    ber_q = (O.levels_to_bits(out['xq'], 64) != O.levels_to_bits(b['l'].numpy(), 64)).mean()
    assert ber <= ber_q

