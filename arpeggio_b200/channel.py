"""Synthetic channel uses (y = H x + n), the reference's model and random-number order.

`draw` restates arpx.draw (arpeggio/sim/arpx.py:35-52) on a CPU torch.Generator seeded by
draw_seed(seed, snr, bi): uniform Gray PAM levels, i.i.d. CN(0, 1) channel entries scaled by the
constellation factor a and lifted to [[Re, -Im], [Im, Re]] (mimo.py:55-58), N0 = Nt / 10^(SNR/10), y formed
in float64 and rounded once to float32 -- so that draws are identical to the reference's on any host.
`draw_device` is the same model on a CUDA generator (different random numbers) for large timing batches."""
import math

import torch

PAM = {4: dict(levels=[-1, 1], a=1 / math.sqrt(2)), 16: dict(levels=[-3, -1, 1, 3], a=1 / math.sqrt(10)),
       64: dict(levels=[-7, -5, -3, -1, 1, 3, 5, 7], a=1 / math.sqrt(42))}


def draw_seed(seed, snr, bi):
    return seed * 1_000_003 + int(round(snr * 100)) * 10_007 + bi


def complex_to_real(Hc):
    Hr, Hi = Hc.real, Hc.imag
    return torch.cat([torch.cat([Hr, -Hi], -1), torch.cat([Hi, Hr], -1)], -2)


def draw(seed, snr, bi, B, nt, M, nr=None, dev='cpu'):
    """Returns dict(H (B, 2nr, 2nt), y (B, 2nr), l (B, 2nt) levels, N0, M, Nt, Nr)."""
    nr = nt if nr is None else nr
    g = torch.Generator(device='cpu')
    g.manual_seed(draw_seed(seed, snr, bi))
    a = PAM[M]['a']
    lv = torch.tensor(PAM[M]['levels'], dtype=torch.float32)
    l = lv[torch.randint(0, len(lv), (B, 2 * nt), generator=g)]
    Hc = torch.complex(torch.randn(B, nr, nt, generator=g), torch.randn(B, nr, nt, generator=g)) / math.sqrt(2)
    H = complex_to_real(Hc) * a
    N0 = nt * 1.0 / (10 ** (snr / 10))
    n = torch.randn(B, 2 * nr, generator=g) * math.sqrt(N0 / 2)
    y = ((H.double() * l.double()[:, None, :]).sum(-1) + n.double()).float()
    return dict(H=H.to(dev), y=y.to(dev), l=l.to(dev), N0=N0, M=M, Nt=nt, Nr=nr)


@torch.no_grad()
def draw_device(seed, snr, B, nt, M, nr=None, dev='cuda'):
    """The same model drawn on the device (for large timing batches); snr may be a scalar or (B,) tensor."""
    nr = nt if nr is None else nr
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    a = PAM[M]['a']
    lv = torch.tensor(PAM[M]['levels'], dtype=torch.float32, device=dev)
    l = lv[torch.randint(0, len(lv), (B, 2 * nt), generator=g, device=dev)]
    Hc = torch.complex(torch.randn(B, nr, nt, generator=g, device=dev),
                       torch.randn(B, nr, nt, generator=g, device=dev)) / math.sqrt(2)
    H = complex_to_real(Hc) * a
    snr = torch.as_tensor(snr, dtype=torch.float32, device=dev).reshape(-1)
    N0 = nt / (10 ** (snr / 10))
    n = torch.randn(B, 2 * nr, generator=g, device=dev) * torch.sqrt(N0 / 2)[:, None].expand(B, 1)
    y = torch.einsum('bij,bj->bi', H, l) + n
    return dict(H=H.contiguous(), y=y.contiguous(), l=l, N0=N0.expand(B).contiguous(), M=M, Nt=nt, Nr=nr)


def levels_to_bits(l, M):
    """Gray bits per real dimension, MSB first (mimo.py:45-51; 64-QAM: the binary-reflected Gray code of the level
    index, which is also what the QPSK and 16-QAM tables are)."""
    if M == 4:
        return (l > 0).to(torch.int8)
    if M == 16:
        b1 = (l > 0).to(torch.int8)
        b2 = (l.abs() == 1).to(torch.int8)
        return torch.stack([b1, b2], dim=-1).flatten(-2)
    i = ((l.to(torch.int64) + 7) // 2)
    g = i ^ (i >> 1)
    return torch.stack([(g >> (2 - k)) & 1 for k in range(3)], dim=-1).flatten(-2).to(torch.int8)
