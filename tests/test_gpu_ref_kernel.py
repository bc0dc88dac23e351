"""The reference's own CUDA kernels, compiled from their sources into oracle/_ref/ by `make -C oracle ref-gpu`,
beside this project's on the same inputs, keys and instance numbers: the first-accept kernel
(arpeggio/sim/arpeggio_fx.cu, one thread per anneal) against arp_anneal_first_accept -- spins, best energies and
flip/test counters bit for bit -- and the Chord kernel (arpeggio/mimo/chord_kernel.cu) against arp_anneal_chord
on the golden Chord problems -- spins, energies and counters bit for bit; both pairs timed on the same GPU.
Skipped where the reference kernels were not built (no reference tree at build time)."""
import ctypes
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
REF_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), '..', 'oracle', '_ref')
REF_SO = os.path.join(REF_DIR, 'libref_arpeggio.so')
REF_CHORD_SO = os.path.join(REF_DIR, 'libref_chord.so')
M32 = 0xFFFFFFFF


def _ref():
    if not os.path.exists(REF_SO):
        pytest.skip('reference kernel not built (make -C oracle ref-gpu needs the reference tree)')
    L = ctypes.CDLL(REF_SO)
    P_, I, U = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32
    L.ref_arpeggio_fx.argtypes = [P_, P_, P_, I, I, I, I, I, I, P_, U, U, I, P_, P_, P_, P_]
    return L


def _problems(B, nt, snr, seed, R, sweeps):
    from arpeggio_b200 import channel, warm
    d = channel.draw_device(seed, snr, B, nt, 16)
    det = warm.WarmDetector(B, nt, anneals=R, sweeps=sweeps)
    det.set_noise(N0=d['N0'])
    det.run(d['H'], d['y'], seed=seed, warm=False)  # forms the integer problem G, h
    torch.cuda.synchronize()
    return det


def _run_both(det, R, P, start, key, reps=1):
    from arpeggio_b200 import _lib
    L = _ref()
    B, D = det.B, det.D
    T = torch.tensor(det.schedule['T'], dtype=torch.int32, device='cuda')
    q = int(det.schedule['q'])
    inst = torch.arange(B, dtype=torch.int32, device='cuda') * 7 + 3
    outs = []
    times = []
    for which in ('ref', 'ours'):
        s = torch.empty(B, R, P * D, dtype=torch.int8, device='cuda')
        de = torch.empty(B, R, dtype=torch.int64, device='cuda')
        st = torch.empty(B, R, 2, dtype=torch.int64, device='cuda')
        stat = torch.zeros(1, dtype=torch.int32, device='cuda')

        def launch():
            if which == 'ref':  # G is symmetric, so it is also its own transpose Gt
                assert L.ref_arpeggio_fx(_lib.ptr(det.G), _lib.ptr(det.h), _lib.ptr(T), len(T), q, P, R, D, B,
                                         _lib.ptr(inst), key & M32, key >> 32, start, _lib.ptr(s), _lib.ptr(de),
                                         _lib.ptr(st), _lib.stream_ptr()) == 0
            else:
                _lib.check(_lib.lib().arp_anneal_first_accept(_lib.ptr(det.G), _lib.ptr(det.h), _lib.ptr(T), len(T),
                                                              q, P, R, D, B, _lib.ptr(inst), key & M32, key >> 32,
                                                              start, _lib.ptr(s), _lib.ptr(de), _lib.ptr(st),
                                                              _lib.ptr(stat), _lib.stream_ptr()), 'anneal')
        launch()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            launch()
        e1.record()
        torch.cuda.synchronize()
        assert int(stat.item()) == 0
        times.append(e0.elapsed_time(e1) / reps)
        outs.append((s, de, st))
    return outs, times


@pytest.mark.parametrize('nt,R,sweeps,start', [(32, 32, 32, 0), (32, 8, 16, 1), (64, 8, 16, 1), (16, 16, 64, 0)])
def test_reference_kernel_bit_exact(nt, R, sweeps, start):
    det = _problems(256, nt, 14.0, 60 + nt, R, sweeps)
    (ref, ours), _ = _run_both(det, R, 2, start, 0x1234567890ABCDEF)
    for a, b in zip(ref, ours):
        assert torch.equal(a, b)


def test_reference_kernel_timing_x32():
    """The benchmark's configuration (32 users, 16-QAM, 32 anneals x 32 sweeps, 'rand' start) on 4096 channel
    uses: the same outputs, and both kernels' device time (printed; run with -s to see it)."""
    det = _problems(4096, 32, 14.0, 77, 32, 32)
    (ref, ours), (t_ref, t_ours) = _run_both(det, 32, 2, 0, 0xC0FFEE, reps=3)
    for a, b in zip(ref, ours):
        assert torch.equal(a, b)
    print('\nreference arpeggio_fx: %.3f ms, this project: %.3f ms for 4096 uses x 32 anneals (%.1fx)'
          % (t_ref, t_ours, t_ref / t_ours))
    assert t_ours < t_ref


def _ref_chord():
    if not os.path.exists(REF_CHORD_SO):
        pytest.skip('reference Chord kernel not built (make -C oracle ref-gpu needs the reference tree)')
    L = ctypes.CDLL(REF_CHORD_SO)
    P_, I, U = ctypes.c_void_p, ctypes.c_int, ctypes.c_uint32
    L.ref_chord.argtypes = [P_, P_, P_, P_, P_, I, I, I, I, I, I, U, U, I, I, I, P_, P_, P_, P_]
    return L


def _chord_both(F, R, P, seed, inst0, mode, reps=1):
    from arpeggio_b200 import _lib, chordfx
    L = _ref_chord()
    B, N = F['h'].shape
    dev = torch.device('cuda')
    F = dict(F, J=F['J'].to(dev, torch.int16).contiguous(), h=F['h'].to(dev, torch.int32).contiguous(),
             h0=F['h0'].to(dev, torch.int32).contiguous(), T=F['T'].to(dev, torch.int32).contiguous(),
             c=F['c'].to(dev, torch.int32).contiguous())  # both kernels read device-resident inputs
    J = F['J']
    h, h0 = F['h'].to(dev, torch.int32).contiguous(), F['h0'].to(dev, torch.int32).contiguous()
    T, c = F['T'].to(dev, torch.int32).contiguous(), F['c'].to(dev, torch.int32).contiguous()
    shape_e, shape_s = ((B,), (B, N)) if mode == 'best' else ((B, R), (B, R, N))
    re_e = torch.empty(shape_e, dtype=torch.int32, device=dev)
    re_s = torch.empty(shape_s, dtype=torch.int8, device=dev)
    re_st = torch.zeros(4, dtype=torch.int64, device=dev)
    k = chordfx.Kernel()
    our_st = torch.zeros(4, dtype=torch.int64, device=dev)

    def ref_launch(st):
        assert L.ref_chord(_lib.ptr(J), _lib.ptr(h), _lib.ptr(h0), _lib.ptr(T), _lib.ptr(c), int(F['q']), int(F['S']),
                           P, R, N, B, seed & M32, seed >> 32, inst0, 1 if mode == 'best' else 0, 8, _lib.ptr(re_e),
                           _lib.ptr(re_s), _lib.ptr(st), _lib.stream_ptr()) == 0

    ref_launch(re_st)
    s, e = k.chord(F, R, seed, P=P, inst0=inst0, mode=mode, stats=our_st)
    torch.cuda.synchronize()
    times = []
    for fn in (lambda: ref_launch(None), lambda: k.chord(F, R, seed, P=P, inst0=inst0, mode=mode)):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1) / reps)
    return (re_s, re_e.to(torch.int64), re_st), (s, e, our_st), times


def _golden_chord(golden, name):
    z = golden('golden_chord.npz')
    q, S, P, R, s0, s1, inst0 = [int(v) for v in z[name + '/meta']]
    F = dict(J=torch.from_numpy(z[name + '/J']), h=torch.from_numpy(z[name + '/h']),
             h0=torch.from_numpy(z[name + '/h0']), T=torch.from_numpy(z[name + '/T']),
             c=torch.from_numpy(z[name + '/c']), q=q, S=S)
    return F, P, R, s0 | (s1 << 32), inst0


def _chord_names():
    from conftest import GOLDEN
    return [str(n) for n in np.load(os.path.join(GOLDEN, 'golden_chord.npz'))['names']]


@pytest.mark.parametrize('name', _chord_names())
@pytest.mark.parametrize('mode', ['chains', 'best'])
def test_reference_chord_kernel_bit_exact(golden, name, mode):
    F, P, R, seed, inst0 = _golden_chord(golden, name)
    ref, ours, _ = _chord_both(F, R, P, seed, inst0, mode)
    for a, b in zip(ref, ours):
        assert torch.equal(a, b)


def test_reference_chord_kernel_timing(golden):
    """The largest golden Chord problem tiled to 2048 problems (distinct instance numbers): the same outputs,
    and both kernels' device time (printed; run with -s)."""
    names = _chord_names()
    F, P, R, seed, inst0 = max((_golden_chord(golden, n) for n in names), key=lambda t: t[0]['h'].shape[1])
    B0 = F['h'].shape[0]
    rep = -(-2048 // B0)
    F = {k: (v.repeat((rep,) + (1,) * (v.dim() - 1))[:2048] if k in ('J', 'h', 'h0') else v) for k, v in F.items()}
    ref, ours, (t_ref, t_ours) = _chord_both(F, R, P, seed, inst0, 'chains', reps=3)
    for a, b in zip(ref, ours):
        assert torch.equal(a, b)
    print('\nreference chord_m%d: %.3f ms, this project: %.3f ms for 2048 problems x %d anneals, N = %d (%.2fx)'
          % (F['h'].shape[1] // 32, t_ref, t_ours, R, F['h'].shape[1], t_ref / t_ours))
    assert t_ours < t_ref


@pytest.mark.parametrize('nt,K,steps,kappa', [(32, 1, 256, 0.0), (16, 1, 256, 0.3), (64, 2, 64, 0.3)])
def test_chord_round_equals_reference_engine(nt, K, steps, kappa):
    """This project's Chord round on compressed problems (arp_anneal_chord_dd, 'rand' start) against the reference's
    C++ engine model (arpeggio/sim/x3model/engine_model.cpp, Philox numbers, built into oracle/_ref/libape.so):
    best spins and best energy changes bit for bit, flips per problem equal."""
    from arpeggio_b200 import arpeggiofx
    from arpeggio_b200.detector import chord_schedule
    from oracle import ref_engine
    if not ref_engine.available():
        pytest.skip('reference engine not built (make -C oracle ref needs the reference tree)')
    B, R, P = 48, 8, 2 * K
    det = _problems(B, nt, 14.0, 90 + nt, R, 8)
    T, q, c = chord_schedule(steps, 0.3, 0.3, 0.4, kappa=kappa)
    key = 0xABCDEF0123 + nt
    inst = torch.arange(B, dtype=torch.int32, device='cuda') * 11 + 1
    s, de, st, status = arpeggiofx.anneal(det.G, det.h, P, R, torch.tensor(T, dtype=torch.int32, device='cuda'), q,
                                          inst, key, 'rand', 'chord', torch.tensor(c, dtype=torch.int32, device='cuda'))
    torch.cuda.synchronize()
    arpeggiofx.check_status(status)
    es, ede, _, est = ref_engine.solve_batch(det.G.cpu().numpy(), det.h.cpu().numpy(), P, R, T, c, q,
                                             inst.cpu().numpy().view(np.uint32), key, nthreads=os.cpu_count() or 1)
    assert np.array_equal(s.cpu().numpy(), es)
    assert np.array_equal(de.cpu().numpy(), ede)
    assert np.array_equal(st[..., 0].sum(dim=1).cpu().numpy(), est[:, 1])


@pytest.mark.parametrize('nt,K,steps,kappa', [(32, 1, 256, 0.0), (16, 1, 256, 0.3), (64, 1, 64, 0.0),
                                              (32, 2, 128, 0.3), (48, 3, 48, 0.0)])
def test_chord_engine_numbers_equal_reference_engine(nt, K, steps, kappa):
    """arp_anneal_chord_engine (Chord with the engine's own numbers, the mode of the reference's production scripts)
    against the reference's C++ engine model run with philox = 0 and against the oracle's restatement: best spins and
    best energy changes bit for bit, flips per problem equal."""
    from arpeggio_b200 import arpeggiofx
    from arpeggio_b200.detector import chord_schedule
    from oracle import oracle as O
    from oracle import ref_engine
    B, R, P = 48, 8, 2 * K
    det = _problems(B, nt, 14.0, 120 + nt, R, 8)
    T, q, c = chord_schedule(steps, 0.3, 0.3, 0.4, kappa=kappa)
    key = 0xFEEDFACE12345 + nt
    inst = torch.arange(B, dtype=torch.int32, device='cuda') * 5 + 2
    s, de, st, status = arpeggiofx.anneal_engine(det.G, det.h, P, R, torch.tensor(T, dtype=torch.int32, device='cuda'),
                                                 q, inst, key, torch.tensor(c, dtype=torch.int32, device='cuda'))
    torch.cuda.synchronize()
    arpeggiofx.check_status(status)
    G, h, it = det.G.cpu().numpy(), det.h.cpu().numpy(), inst.cpu().numpy().view(np.uint32)
    os_, ode, ost = O.anneal_chord_hw(G, h, P, R, T, c, q, it, key, nthreads=os.cpu_count() or 1)
    assert np.array_equal(s.cpu().numpy(), os_)
    assert np.array_equal(de.cpu().numpy(), ode)
    assert np.array_equal(st.cpu().numpy(), ost)
    if ref_engine.available():
        es, ede, _, est = ref_engine.solve_batch(G, h, P, R, T, c, q, it, key, nthreads=os.cpu_count() or 1,
                                                 philox=0)
        assert np.array_equal(s.cpu().numpy(), es)
        assert np.array_equal(de.cpu().numpy(), ede)
        assert np.array_equal(st[..., 0].sum(dim=1).cpu().numpy(), est[:, 1])
