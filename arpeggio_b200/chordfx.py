"""Fixed-point Chord behind the interface of the reference's arpeggio/mimo/chordfx.py.

`to_fixed` (chordfx.py:60-76) turns the float Ising dict of mimo.ising / ising_delta_at into the integer
problem; `Kernel` keeps the launcher's methods (`chord`, chordfx.py:189-208; `philox_kat`, :180-187) but
runs this project's sm_100a kernels through the C ABI instead of loading a cubin."""
import torch

from . import _lib

QSCALE = 4096
MASK = 0xFFFFFFFF
# Random123 known-answer vectors (kat_vectors, philox4x32 10): counter, key -> output.
KAT = [((0, 0, 0, 0), (0, 0), (0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8)),
       ((MASK, MASK, MASK, MASK), (MASK, MASK), (0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd)),
       ((0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344), (0xa4093822, 0x299f31d0),
        (0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1))]


def geom(t0, t1, S, device='cpu'):
    """Geometric temperature ladder, computed in float64 and rounded once to float32 (mimo.py:199-201)."""
    k = torch.arange(S, device=device, dtype=torch.float64)
    return (t0 * (t1 / t0) ** (k / max(1, S - 1))).to(torch.float32)


def to_fixed(I, S, t0, t1, q, kappa=0.0, ramp=True, Q=QSCALE):
    """Integer inputs of the Chord kernel (chordfx.py:60-76): J symmetrised then round(J Q) int16, h and h0
    round(x Q) int32, T_k = round(T Q), Onsager c_k = round(kappa T_{k-1} rho_k Q), q = round(q Q)."""
    J = (I['J'] + I['J'].transpose(1, 2)) / 2
    Ji = torch.round(J * Q).to(torch.int16)
    hi = torch.round(I['h'] * Q).to(torch.int32)
    h0i = torch.round(I['h0'] * Q).to(torch.int32)
    T = geom(t0, t1, S).double()
    rho = torch.ones(S, dtype=torch.float64)
    if ramp:
        t = torch.arange(S, dtype=torch.float64)
        rho = torch.where(t >= 0.7 * S, (S - 1 - t) / max(1.0, S - 1 - 0.7 * S), torch.ones_like(t))
    c = torch.zeros(S, dtype=torch.float64)
    c[1:] = kappa * T[:-1] * rho[1:]
    dev = I['h'].device
    return dict(J=Ji.contiguous(), h=hi.contiguous(), h0=h0i.contiguous(),
                T=torch.round(T * Q).to(torch.int32).to(dev), c=torch.round(c * Q).to(torch.int32).to(dev),
                q=int(round(q * Q)), S=S, Q=Q)


class Kernel:
    """Launcher with the methods of chordfx.Kernel (chordfx.py:130-208).  `cubin` is accepted for signature
    compatibility and ignored: the kernels live in libarpeggio_b200.so."""
    MPLS = (1, 2, 3, 4, 6, 8)

    def __init__(self, cubin=None):
        self.lib = _lib.lib()

    def philox_kat(self, words):
        """words: (n, 6) uint32 (counter, key) -> (n, 4) outputs from the device Philox."""
        n = words.shape[0]
        inp = words.to(torch.int64).to(torch.int32).cuda().contiguous()
        out = torch.zeros(n, 4, dtype=torch.int32, device='cuda')
        _lib.check(self.lib.arp_philox_kat(_lib.ptr(inp), _lib.ptr(out), n, _lib.stream_ptr()), 'philox_kat')
        torch.cuda.synchronize()
        return out.to(torch.int64) & MASK

    def chord(self, F, R, seed, P=1, inst0=0, mode='chains', warps=0, stats=None):
        """Kernel run with the same contract as chord_fx; returns (spins int8, 2 E0 int64) on the device.
        warps: anneals per block in flight (0 = the width with the most resident warps per SM); the reference's
        default is 8, and the outputs do not depend on it."""
        B, N = F['h'].shape
        assert N % 32 == 0 and (N // P) % 32 == 0, 'spins per copy must be a multiple of 32'
        assert N // 32 in self.MPLS, 'unsupported spin count %d' % N
        dev = F['h'].device if F['h'].is_cuda else torch.device('cuda')
        J = F['J'].to(dev, torch.int16).contiguous()
        h = F['h'].to(dev, torch.int32).contiguous()
        h0 = F['h0'].to(dev, torch.int32).contiguous()
        T = F['T'].to(dev, torch.int32).contiguous()
        c = F['c'].to(dev, torch.int32).contiguous()
        if mode == 'best':
            out_e = torch.empty(B, dtype=torch.int64, device=dev)
            out_s = torch.empty(B, N, dtype=torch.int8, device=dev)
        else:
            out_e = torch.empty(B, R, dtype=torch.int64, device=dev)
            out_s = torch.empty(B, R, N, dtype=torch.int8, device=dev)
        status = torch.zeros(1, dtype=torch.int32, device=dev)
        rc = self.lib.arp_anneal_chord(_lib.ptr(J), _lib.ptr(h), _lib.ptr(h0), _lib.ptr(T), _lib.ptr(c), int(F['q']),
                                       int(F['S']), P, R, N, B, seed & MASK, (seed >> 32) & MASK, inst0 & MASK,
                                       1 if mode == 'best' else 0, warps, _lib.ptr(out_e), _lib.ptr(out_s),
                                       _lib.ptr(stats), _lib.ptr(status), _lib.stream_ptr())
        _lib.check(rc, 'chord')
        self.last_status = status
        return out_s, out_e


def spins_float(s8):
    return s8.to(torch.float32)

