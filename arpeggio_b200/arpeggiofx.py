"""Anneals on compressed dDI problems behind the interface of the reference's arpeggio/sim/arpeggiofx.py.

`solve` keeps the reference signature and return values (arpeggiofx.py:22-44): integer G (B, D, D) and h
(B, D) from chord_ref.compress, P copies, R anneals, one temperature per pass T, q, instance numbers, a
64-bit Philox key, start 'rand' or 'bal' -> numpy (best spins (B, R, P*D) int8 copy-major, best energy
change (B, R) int64, (B, R, 2) int64 [flips, tests]).  It copies to the device, runs
arp_anneal_first_accept, synchronises and copies back, as the reference does.

`anneal` is the device-resident form: torch CUDA tensors in and out, launched on the current stream, no
synchronisation; it also exposes Chord's round (policy='chord', with the Onsager term c) and FP32 fields
(precision='f32')."""
import numpy as np
import torch

from . import _lib

M32 = 0xFFFFFFFF
POLICIES = ('arpeggio', 'chord')


def _u32(x, dev):
    return torch.as_tensor(np.asarray(x, dtype=np.int64) & M32).to(torch.int32).to(dev).contiguous()


@torch.no_grad()
def anneal(Gt, h, P, R, T, q, inst, key, start='rand', policy='arpeggio', c=None, precision='int', out=None,
           status=None, stream=None, n1=None):
    """Device anneal.  Gt (B, D, D) transposed coupling (Gt[b, j, i] = G[b, i, j]) on the GPU, int32 for
    precision 'int' or float32 for 'f32'; h (B, D) likewise; T (L,) and c (L,) or None device tensors;
    inst (B,) int32 bit patterns of uint32 instance numbers.  Returns (spins (B, R, P D) int8,
    de (B, R) int64 or float32, st (B, R, 2) int64, status (1,) int32) without synchronising.  n1: for the integer
    Chord round, an int64 (B, R) device tensor that receives the rounds with at least one flip per anneal (the term
    of the Chord engine's latency 3 L + F + n1)."""
    if policy not in POLICIES:
        raise ValueError('policy must be one of %s' % (POLICIES,))
    B, D, _ = Gt.shape
    dev = Gt.device
    f32 = precision == 'f32'
    if precision not in ('int', 'f32'):
        raise ValueError("precision must be 'int' or 'f32'")
    if out is None:
        out = (torch.empty(B, R, P * D, dtype=torch.int8, device=dev),
               torch.empty(B, R, dtype=torch.float32 if f32 else torch.int64, device=dev),
               torch.empty(B, R, 2, dtype=torch.int64, device=dev))
    if status is None:
        status = torch.zeros(1, dtype=torch.int32, device=dev)
    s_, de, st = out
    L = lib = _lib.lib()
    L = int(T.shape[0])
    k0, k1, sv = key & M32, (key >> 32) & M32, 0 if start == 'rand' else 1
    args = (_lib.ptr(s_), _lib.ptr(de), _lib.ptr(st), _lib.ptr(status), _lib.stream_ptr(stream))
    if f32:
        rc = lib.arp_anneal_dd_f32(0 if policy == 'arpeggio' else 1, _lib.ptr(Gt), _lib.ptr(h), _lib.ptr(T),
                                   _lib.ptr(c), L, float(q), P, R, D, B, _lib.ptr(inst), k0, k1, sv, *args)
    elif policy == 'arpeggio':
        rc = lib.arp_anneal_first_accept(_lib.ptr(Gt), _lib.ptr(h), _lib.ptr(T), L, int(q), P, R, D, B,
                                         _lib.ptr(inst), k0, k1, sv, *args)
    elif n1 is not None:
        rc = lib.arp_anneal_chord_dd_n1(_lib.ptr(Gt), _lib.ptr(h), _lib.ptr(T), _lib.ptr(c), L, int(q), P, R, D, B,
                                        _lib.ptr(inst), k0, k1, sv, _lib.ptr(s_), _lib.ptr(de), _lib.ptr(st),
                                        _lib.ptr(n1), _lib.ptr(status), _lib.stream_ptr(stream))
    else:
        rc = lib.arp_anneal_chord_dd(_lib.ptr(Gt), _lib.ptr(h), _lib.ptr(T), _lib.ptr(c), L, int(q), P, R, D, B,
                                     _lib.ptr(inst), k0, k1, sv, *args)
    _lib.check(rc, 'anneal(%s, %s)' % (policy, precision))
    return s_, de, st, status


@torch.no_grad()
def anneal_engine(Gt, h, P, R, T, q, inst, key, c=None, out=None, status=None, stream=None):
    """Chord's round with the random numbers of the reference's C++ engine model run without Philox
    (engine_model.cpp engine_solve_batch with philox = 0): per-coordinate xorshift32 generators seeded from
    (key, inst, r), which also give the start spins.  Device tensors as in `anneal` (T and c one entry per step);
    returns (spins, de, st, status) without synchronising."""
    B, D, _ = Gt.shape
    dev = Gt.device
    if out is None:
        out = (torch.empty(B, R, P * D, dtype=torch.int8, device=dev),
               torch.empty(B, R, dtype=torch.int64, device=dev),
               torch.empty(B, R, 2, dtype=torch.int64, device=dev))
    if status is None:
        status = torch.zeros(1, dtype=torch.int32, device=dev)
    s_, de, st = out
    rc = _lib.lib().arp_anneal_chord_engine(_lib.ptr(Gt), _lib.ptr(h), _lib.ptr(T), _lib.ptr(c), int(T.shape[0]),
                                            int(q), P, R, D, B, _lib.ptr(inst), key & M32, (key >> 32) & M32,
                                            _lib.ptr(s_), _lib.ptr(de), _lib.ptr(st), _lib.ptr(status),
                                            _lib.stream_ptr(stream))
    _lib.check(rc, 'anneal_engine')
    return s_, de, st, status


def check_status(status):
    """Raises if a device-side check failed (synchronises on the status word)."""
    v = int(status.item())
    _lib.check(v, 'device check')


@torch.no_grad()
def solve(G, h, P, R, T, q, inst, key, start):
    """Reference contract of arpeggiofx.solve (arpeggio/sim/arpeggiofx.py:22-44)."""
    G = torch.as_tensor(G)
    h = torch.as_tensor(h)
    B, D, _ = G.shape
    assert D <= 128 and P in (2, 4, 6) and len(T) >= 1
    Gt = G.transpose(1, 2).contiguous().to(torch.int32).cuda()
    hh = h.to(torch.int32).contiguous().cuda()
    Tt = torch.tensor([int(x) for x in T], dtype=torch.int32, device='cuda')
    it = _u32(inst, 'cuda')
    s_, de, st, status = anneal(Gt, hh, P, R, Tt, q, it, key, start)
    torch.cuda.synchronize()
    check_status(status)
    return s_.cpu().numpy(), de.cpu().numpy(), st.cpu().numpy()
