"""Host-side checks that need no GPU: the C-ABI library loads and exports every declared symbol, the
reference-compatible draws and schedules, and the oracle's restated readout."""
import os
import re

import numpy as np
import pytest
import torch

from conftest import ROOT


def declared_symbols():
    names = []
    inc = os.path.join(ROOT, 'include')
    for f in sorted(os.listdir(inc)):
        if f.endswith('.h'):
            src = open(os.path.join(inc, f)).read()
            names += re.findall(r'^\s*(?:const\s+)?\w+\*?\s+\*?(arp_\w+)\s*\(', src, flags=re.M)
    return names


def test_library_exports_every_declared_symbol():
    from arpeggio_b200 import _lib
    L = _lib.lib()
    names = declared_symbols()
    assert len(names) >= 9
    for n in names:
        assert hasattr(L, n), n
        assert n in _lib.SIGNATURES, 'no ctypes signature for %s' % n
    assert L.arp_version().startswith(b'arpeggio_b200')
    assert L.arp_status_string(2) == b'coefficients or schedule beyond the exact 32-bit field range'


def test_host_rejects_bad_shapes_without_gpu():
    """Shape and argument errors are found on the host before any launch."""
    from arpeggio_b200 import _lib
    L = _lib.lib()
    # D = 129 > 128, P = 3 (not a dDI copy count), R = 0: rejected before touching any pointer
    assert L.arp_anneal_first_accept(None, None, None, 1, 0, 2, 1, 129, 1, None, 0, 0, 0, None, None, None, None,
                                     None) == 1
    assert L.arp_anneal_first_accept(None, None, None, 1, 0, 3, 1, 32, 1, None, 0, 0, 0, None, None, None, None,
                                     None) == 1
    assert L.arp_anneal_chord_dd(None, None, None, None, 1, 0, 2, 0, 32, 1, None, 0, 0, 0, None, None, None, None,
                                 None) == 1
    assert L.arp_anneal_chord(None, None, None, None, None, 0, 8, 2, 4, 96, 1, 0, 0, 0, 0, 8, None, None, None, None,
                              None) == 1  # (N/P) % 32 != 0
    assert L.arp_anneal_dd_f32(2, None, None, None, None, 1, 0.0, 2, 1, 32, 1, None, 0, 0, 0, None, None, None, None,
                               None) == 3  # bad policy
    # null pointers with a non-empty batch
    assert L.arp_anneal_first_accept(None, None, None, 1, 0, 2, 1, 32, 1, None, 0, 0, 0, None, None, None, None,
                                     None) == 3
    assert L.arp_map_dd(None, None, None, 1, 64, 64, 16, 1, None, None, None, None, None, None) == 3
    # empty batch is a no-op
    assert L.arp_anneal_first_accept(None, None, None, 1, 0, 2, 1, 32, 0, None, 0, 0, 0, None, None, None, None,
                                     None) == 0
    # the native serving loop checks its tables before any CUDA call: bad counts, a stream with null buffers,
    # requests that no lane can take; nothing to serve is a no-op
    assert L.arp_serve_run(None, -1, None, 0, 1.0, None) == 3
    bad = (_lib.ServeStream * 1)()
    bad[0].n, bad[0].h_elems, bad[0].y_elems, bad[0].bits_per = 2, 4, 2, 2
    assert L.arp_serve_run(bad, 1, None, 0, 1.0, None) == 3
    H, y, f, rid = (np.zeros(8, np.float32), np.zeros(4, np.float32), np.zeros(2, np.float32),
                    np.zeros(2, np.int32))
    t, bits, done = np.zeros(2), np.zeros(4, np.int8), np.zeros(2)
    ok = (_lib.ServeStream * 1)(_lib.ServeStream(H.ctypes.data, y.ctypes.data, f.ctypes.data, f.ctypes.data,
                                                 rid.ctypes.data, t.ctypes.data, 2, 4, 2, 2, bits.ctypes.data,
                                                 f.ctypes.data, done.ctypes.data))
    assert L.arp_serve_run(ok, 1, None, 0, 1.0, None) == 3
    assert L.arp_serve_run(None, 0, None, 0, 1.0, None) == 0
    # the autotuner hook: policy 2 (the warm-started first accept) exists for P = 2, int32 only
    assert L.arp_anneal_tune(64, 4, 2, 0, 4) == 1 and L.arp_anneal_tune(64, 2, 2, 1, 4) == 1
    assert L.arp_anneal_tune(64, 2, 3, 0, 4) == 1 and L.arp_anneal_tune(64, 2, 2, 0, 3) == 3
    assert L.arp_anneal_tune(64, 2, 2, 0, 4) == 0 and L.arp_anneal_tune(64, 2, 2, 0, 0) == 0


def test_draw_matches_reference(golden):
    """channel.draw restates arpx.draw bit for bit (same torch generator order)."""
    from arpeggio_b200 import channel
    z = golden('golden_mapping.npz')
    for nt, snr, B, seed in ((16, 12.0, 16, 9700), (32, 16.0, 8, 9701), (64, 20.0, 4, 9702)):
        b = channel.draw(seed, snr, 0, B, nt, 16)
        tag = 'x%d' % nt
        assert np.array_equal(b['H'].numpy(), z[tag + '/H'])
        assert np.array_equal(b['y'].numpy(), z[tag + '/y'])
        assert np.array_equal(b['l'].numpy(), z[tag + '/l'])
        assert b['N0'] == pytest.approx(float(z[tag + '/N0'][0]))


def test_schedules_match_reference(golden):
    """Integer Arpeggio schedule equals run_a513.arpeggio_schedule's (fixtures carry it)."""
    from arpeggio_b200 import detector
    from oracle import oracle as O
    z = golden('golden_arpeggio.npz')
    T, q, c = detector.arpeggio_schedule(64, 0.1, 0.1, 0.0, 1)
    assert T == [int(v) for v in z['x16_K1_pick_rand/T']] and q == 0 and c is None
    T, q, c = detector.arpeggio_schedule(8, 1.2, 0.1, 0.2, 1)
    assert T == [int(v) for v in z['x16_K1_hot_bal/T']] and q == int(z['x16_K1_hot_bal/meta'][2])
    T2, q2 = O.arpeggio_schedule(1.2, 0.1, 8, 0.2, 1)
    assert T == T2 and q == q2
    zc = golden('golden_chord.npz')
    for name, (S, t0, t1, q, kappa) in (('32x32_16QAM_dDI_K1_kappa', (128, 0.3, 0.2, 0.4, 0.3)),
                                        ('16x16_QPSK_RI_kappa', (128, 2.0, 0.05, 0.5, 0.3))):
        T, qi, c = detector.chord_schedule(S, t0, t1, q, kappa)
        assert T == [int(v) for v in zc[name + '/T']]
        assert c == [int(v) for v in zc[name + '/c']]
        assert qi == int(zc[name + '/meta'][0])


def test_to_fixed_mirror_matches_reference(golden):
    """chordfx.to_fixed (this package) on the reference's float dict gives the reference's integers."""
    from arpeggio_b200 import chordfx, channel
    z = golden('golden_chord.npz')
    name = '16x16_16QAM_dDI_K1'
    # rebuild the float problem as make_golden did (CPU generator, mimo.make_batch model)
    # and compare only what to_fixed derives from the schedule; J/h come from the fixture itself
    F = dict(J=torch.from_numpy(z[name + '/J'].astype(np.float32) / 4096), h=torch.from_numpy(z[name + '/h'] / 4096.0),
             h0=torch.from_numpy(z[name + '/h0'] / 4096.0))
    G = chordfx.to_fixed(F, 256, 0.3, 0.3, 0.4, 0.0)
    assert torch.equal(G['J'], torch.from_numpy(z[name + '/J']))
    assert torch.equal(G['h'].to(torch.int32), torch.from_numpy(z[name + '/h']))
    assert torch.equal(G['T'], torch.from_numpy(z[name + '/T']))
    _ = channel


def test_oracle_f32_rule_is_deterministic():
    """The FP32 oracle is a pure function of its inputs (threads do not change results)."""
    from oracle import oracle as O
    rng = np.random.default_rng(3)
    B, D, P, R = 3, 40, 2, 4
    A = rng.normal(size=(B, 2 * D, D))
    Q = np.einsum('bki,bkj->bij', A, A)
    h = rng.normal(size=(B, D))
    sc = np.maximum(np.abs(Q).reshape(B, -1).max(1), np.abs(h).max(1))
    G, hh = (Q / sc[:, None, None]).astype(np.float32), (h / sc[:, None]).astype(np.float32)
    T = [0.3] * 16
    a = O.anneal_dd_f32(G, hh, P, R, T, 0.1, np.arange(B), 77, 'rand', nthreads=1)
    b = O.anneal_dd_f32(G, hh, P, R, T, 0.1, np.arange(B), 77, 'rand', nthreads=4)
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_detect_entry_checks_workspace_before_launch():
    """A workspace smaller than arp_detect_dd_workspace() is refused on the host (ARP_ERR_WORKSPACE)."""
    import ctypes
    from arpeggio_b200 import _lib
    L = _lib.lib()
    offs = (ctypes.c_size_t * 7)()
    need = L.arp_detect_dd_workspace(100, 64, 2, 32, 0, offs)
    assert need >= 100 * 64 * 64 * 4 + 100 * 32 * 128 and all(o % 256 == 0 for o in offs)
    assert list(offs) == sorted(offs)
    fake = ctypes.c_void_p(256)  # never dereferenced: the size check comes first
    rc = L.arp_detect_dd(fake, fake, fake, 100, 64, 64, 16, 0, 0, 2, 32, fake, None, 64, 0.0, 0, 1, 2, 0, fake,
                         need - 1, fake, fake, fake, None, None, None)
    assert rc == 6
    rc = L.arp_detect_dd(fake, fake, fake, 100, 64, 64, 16, 2, 0, 2, 32, fake, None, 64, 0.0, 0, 1, 2, 0, fake,
                         need, fake, fake, fake, None, None, None)
    assert rc == 3  # bad policy
