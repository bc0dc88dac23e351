"""Trajectory soft output on the RI map: Chord's synchronous rule run as a sampler of the detection posterior on the
device (arp_soft_trajectory; the reference's mimo.chord_soft, arpeggio/mimo/mimo.py:332-394), keeping for every bit
the smallest ||y - H x||^2 seen with it 0 and with it 1 over all visited states of all chains, and the max-log LLRs
formed from those minima, the best state, the MMSE decision and the single-bit-flip neighbours of the decision
(mimo.trajectory_llr, mimo.py:397-413, with mimo.list_llr, mimo.py:434-462).  The chain is softlib.detect_llr's
'saneNA' method (arpeggio/mimo/softlib.py:48-53): RI map from the MMSE estimate, sampler, LLRs.

The sampler's random numbers are this project's Philox counters (the reference draws from torch.rand), so a chain's
trajectory is its own; the rule, the temperatures, the visited-state minima and the LLR formation follow the
reference, and the LLR step is pinned to the reference's trajectory_llr on golden inputs."""
import numpy as np
import torch

from . import _lib
from .detector import M32, el2

QAM_BITS = {4: 1, 16: 2}


def levels_to_bits(l, M):
    """(..., D) levels -> (..., D nb) Gray bits, MSB first per dimension (mimo.levels_to_bits, mimo.py:45-51)."""
    if M == 4:
        return (l > 0).to(torch.int8)
    return torch.stack([(l > 0), (l.abs() == 1)], -1).flatten(-2).to(torch.int8)


def neighbours(best, M):
    """Single-bit-flip neighbours of the levels best (B, D): (B, D nb, D), dimension-major, MSB first (the
    construction of mimo.list_llr, mimo.py:441-455: flipping b1 negates the level, flipping b2 of 16-QAM maps
    +-1 <-> +-3)."""
    B, D = best.shape
    nb = QAM_BITS[M]
    out = best[:, None, :].repeat(1, D * nb, 1)
    idx = torch.arange(D, device=best.device)
    out[:, idx * nb, idx] = -best
    if nb == 2:
        out[:, idx * nb + 1, idx] = torch.sign(best) * (4 - best.abs())
    return out


def dist(H, y, L):
    """||y - H l||^2 for candidate levels L (B, K, D) (mimo.dist, mimo.py:416-418)."""
    return ((y[:, None, :] - torch.einsum('bij,bkj->bki', H, L.to(H.dtype))) ** 2).sum(-1)


def _n0(N0, ref):
    n0 = torch.as_tensor(N0, dtype=ref.dtype, device=ref.device)
    return n0.reshape(-1, 1) if n0.dim() > 0 and n0.numel() > 1 else n0


def list_llr(H, y, N0, M, allc, d, best, clip=50.0):
    """mimo.list_llr: max-log LLRs (positive = bit 1) over the list (allc, d) and the bit-flip neighbours of best."""
    nbr = neighbours(best, M)
    allc2 = torch.cat([allc, nbr.to(allc.dtype)], 1)
    d2 = torch.cat([d, dist(H, y, nbr)], 1)
    bits = levels_to_bits(allc2, M).bool()
    inf = torch.tensor(float('inf'), device=H.device)
    m1 = torch.where(bits, d2[..., None], inf).amin(1)
    m0 = torch.where(~bits, d2[..., None], inf).amin(1)
    return ((m0 - m1) / _n0(N0, m0)).clamp(-clip, clip)


def trajectory_llr(H, y, N0, M, best_l, best_d, m0, m1, mmse_levels, clip=50.0):
    """mimo.trajectory_llr: LLRs from the trajectory minima (m0, m1) folded with the list {best state, MMSE
    decision}, the decision the closer of the two; bits without a counter-hypothesis in the trajectory take the
    list LLR over the list and the decision's bit-flip neighbours.  Returns (l_hat (B, D), llr (B, D nb))."""
    allc = torch.stack([best_l.to(torch.float32), mmse_levels.to(torch.float32)], 1)
    d = dist(H, y, allc)
    l_hat = allc[torch.arange(allc.shape[0], device=allc.device), d.argmin(1)]
    llr_list = list_llr(H, y, N0, M, allc, d, l_hat, clip=float('inf'))
    bits = levels_to_bits(allc, M).bool()
    inf = float('inf')
    m1 = torch.minimum(m1, torch.where(bits, d[..., None], inf).amin(1))
    m0 = torch.minimum(m0, torch.where(~bits, d[..., None], inf).amin(1))
    llr = (m0 - m1) / _n0(N0, m0)
    llr = torch.where(torch.isfinite(llr), llr, llr_list)
    return l_hat, llr.clamp(-clip, clip)


def temperatures(scale, N0, S, tpost_mult=1.0, t_hot=None, hot_frac=0.0, t_abs=None):
    """(B, S) float32 per-step temperatures of chord_soft: T_post = N0 / (2 scale) x tpost_mult (or t_abs), with an
    optional hot start at t_hot for the first hot_frac of the steps, geometric down to T_post (mimo.py:346-368)."""
    B = scale.shape[0]
    if t_abs is not None:
        Tp = torch.full((B, 1), float(t_abs), dtype=torch.float64, device=scale.device)
    else:
        n0 = torch.as_tensor(N0, dtype=torch.float64, device=scale.device).reshape(-1, 1)
        Tp = (n0 / (2 * scale.double()[:, None]) * tpost_mult).expand(B, 1)
    nh = max(1, int(hot_frac * S)) if (t_hot is not None and hot_frac > 0) else 0
    k = torch.arange(S, dtype=torch.float64, device=scale.device)[None, :]
    T = Tp.expand(B, S).clone()
    if nh > 0:
        hot = (t_hot * (Tp / t_hot) ** (k / max(1, nh - 1))) if nh > 1 else Tp.expand(B, S)
        T = torch.where(k < nh, hot, T)
    return T.float().contiguous()


@torch.no_grad()
def detect_llr(H, y, N0, M=16, R=16, S=256, tpost_mult=1.0, q=0.0, t_hot=None, hot_frac=0.0, t_abs=None, reg=False,
               warm=False, seed=0, inst0=0, r=0.15, clip=1e4, stream=None):
    """softlib.detect_llr's 'saneNA' chain on the device: the RI map (MMSE estimate, hard decision), R chains of S
    synchronous steps of Chord's rule on the unregularised field h0 (or the RI field with reg=True), from random
    spins (or the MMSE spins with warm=True), then trajectory_llr.  H (B, 2Nr, 2Nt), y (B, 2Nr) float32 on the
    device, N0 a scalar or (B,).  Returns dict(llr (B, D nb), l_hat (B, D), best_l, best_d, m0, m1, mmse_levels)."""
    if M not in QAM_BITS:
        raise ValueError('trajectory soft output serves QPSK and 16-QAM (the reference RI map)')
    L = _lib.lib()
    H = torch.as_tensor(H, dtype=torch.float32).cuda().contiguous()
    y = torch.as_tensor(y, dtype=torch.float32).cuda().contiguous()
    B, NR2, D = H.shape
    dev = H.device
    n0 = torch.as_tensor(N0, dtype=torch.float64).reshape(-1)
    s2 = ((n0 / 2) / el2(M)).float().to(dev)
    sigma2 = s2.expand(B).contiguous() if s2.numel() == 1 else s2.contiguous()
    N = 2 * D if M == 16 else D
    f = torch.float32
    J = torch.empty(B, N, N, dtype=f, device=dev)
    h0, h = torch.empty(B, N, dtype=f, device=dev), torch.empty(B, N, dtype=f, device=dev)
    sP = torch.empty(B, N, dtype=torch.int8, device=dev)
    xq = torch.empty(B, D, dtype=torch.int8, device=dev)
    scale = torch.empty(B, dtype=f, device=dev)
    sp = _lib.stream_ptr(stream)
    _lib.check(L.arp_map_ri(_lib.ptr(H), _lib.ptr(y), _lib.ptr(sigma2), B, NR2, D, M, float(r), _lib.ptr(J),
                            _lib.ptr(h0), _lib.ptr(h), _lib.ptr(sP), _lib.ptr(xq), _lib.ptr(scale), sp), 'map_ri')
    # ||y - H x||^2 = scale E0(s) + c0, the constant from the MMSE spins (mimo.py:370-372)
    sPf = sP.float()
    lP = sPf if M == 4 else 2 * sPf[:, :D] + sPf[:, D:]
    e0 = -(sPf * h0).sum(-1) - (sPf * torch.einsum('bij,bj->bi', J, sPf)).sum(-1)
    c0 = (dist(H, y, lP[:, None, :])[:, 0] - scale * e0).contiguous()
    T = temperatures(scale, N0, S, tpost_mult, t_hot, hot_frac, t_abs)
    m0 = torch.empty(B, D * QAM_BITS[M], dtype=f, device=dev)
    m1 = torch.empty_like(m0)
    best_d = torch.empty(B, dtype=f, device=dev)
    best_l = torch.empty(B, D, dtype=torch.int8, device=dev)
    iv = (np.arange(inst0, inst0 + B, dtype=np.int64) & M32).astype(np.uint32).view(np.int32)
    inst = torch.from_numpy(iv).to(dev)
    _lib.check(L.arp_soft_trajectory(_lib.ptr(J), _lib.ptr(h if reg else h0), _lib.ptr(h0), _lib.ptr(scale),
                                     _lib.ptr(c0), _lib.ptr(T), _lib.ptr(sP) if warm else None, float(q), S, R, D, M, B,
                                     _lib.ptr(inst), seed & M32, (seed >> 32) & M32, _lib.ptr(m0), _lib.ptr(m1),
                                     _lib.ptr(best_d), _lib.ptr(best_l), sp), 'soft_trajectory')
    mmse = xq.float()
    l_hat, llr = trajectory_llr(H, y, N0 if n0.numel() == 1 else n0.to(dev), M, best_l.float(), best_d, m0, m1, mmse,
                                clip=clip)
    return dict(llr=llr, l_hat=l_hat, best_l=best_l, best_d=best_d, m0=m0, m1=m1, mmse_levels=mmse, J=J, h0=h0, h=h,
                sP=sP, scale=scale, c0=c0, T=T, inst=inst)
