"""The reference's own first-accept CUDA kernel (arpeggio/sim/arpeggio_fx.cu, compiled from its source into
oracle/_ref/ by `make -C oracle ref-gpu`, one thread per anneal) and this project's kernel on the same integer
problems, keys and instance numbers: spins, best energies and flip/test counters bit for bit, and both timed on
the same GPU.  Skipped where the reference kernel was not built (no reference tree at build time)."""
import ctypes
import os

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
REF_SO = os.path.join(os.path.dirname(os.path.abspath(__file__)), '..', 'oracle', '_ref', 'libref_arpeggio.so')
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
