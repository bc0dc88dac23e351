"""The allocation-free detector entry point, arp_detect_dd_static.

It is for callers that cannot allocate device memory -- a receive chain with a hard per-frame latency
budget (cudaMalloc synchronises the device and takes unbounded time) or a plugin inside a host program
that owns all device memory -- so its intermediates live in a fixed array inside the library instead of a
caller workspace.  This file runs after every other test file: the checks below compare its output with the
workspace entry point's on two calls in a row (different shapes, so the shared array's leftover contents
from the first call must not leak into the second), and check that an oversize batch is refused."""
import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _static_call(det, H, y, seed, outs, status):
    from arpeggio_b200 import _lib
    bits, levels, dist, pick = outs
    rc = _lib.lib().arp_detect_dd_static(
        _lib.ptr(H), _lib.ptr(y), _lib.ptr(det.sigma2), det.B, det.NR2, det.D, det.M,
        0 if det.policy == 'arpeggio' else 1, 1 if det.precision == 'f32' else 0, det.P, det.R,
        _lib.ptr(det.T), _lib.ptr(det.c), int(det.T.shape[0]), float(det.q), 0, seed & 0xFFFFFFFF, seed >> 32,
        0 if det.start == 'rand' else 1, _lib.ptr(bits), _lib.ptr(levels), _lib.ptr(dist), _lib.ptr(pick),
        _lib.ptr(status), _lib.stream_ptr())
    return rc


def test_static_entry_matches_workspace_entry_twice():
    from arpeggio_b200 import channel, detector
    cases = [(32, 'arpeggio', 'int', 600, 14.0, 11), (16, 'chord', 'f32', 900, 10.0, 0x1234567890ABCDEF)]
    for nt, policy, precision, B, snr, seed in cases:
        d = channel.draw_device(seed & 0xFFFF, snr, B, nt, 16)
        det = detector.Detector(B, nt, anneals=12, policy=policy, precision=precision)
        det.set_noise(snr)
        want = [x.clone() for x in det.run(d['H'], d['y'], seed)] + [det.pick.clone()]  # arp_detect_dd
        outs = (torch.full_like(det.bits, -7), torch.full_like(det.levels, -7), torch.full_like(det.dist, -7.0),
                torch.full_like(det.pick, -7))
        status = torch.zeros(1, dtype=torch.int32, device='cuda')
        assert _static_call(det, d['H'], d['y'], seed, outs, status) == 0
        torch.cuda.synchronize()
        det.check()
        assert int(status.item()) == 0
        got = [outs[0], outs[1], outs[2], outs[3]]
        for g, w in zip(got, want):
            assert torch.equal(g, w), (nt, policy, precision)


def test_static_entry_refuses_batches_beyond_its_array():
    """arp_detect_dd_workspace() above the 32 MiB array -> ARP_ERR_WORKSPACE, before any launch."""
    from arpeggio_b200 import _lib, detector
    det = detector.Detector(4, 32, anneals=32)
    L = _lib.lib()
    need = L.arp_detect_dd_workspace(4000, 64, 2, 32, 0, None)
    assert need > (32 << 20)
    fake = torch.zeros(16, dtype=torch.float32, device='cuda')
    p = _lib.ptr(fake)
    rc = L.arp_detect_dd_static(p, p, p, 4000, 64, 64, 16, 0, 0, 2, 32, _lib.ptr(det.T), None,
                                int(det.T.shape[0]), 0.0, 0, 1, 2, 0, p, p, p, None, None, _lib.stream_ptr())
    assert rc == 6
    _ = (ctypes, np)
