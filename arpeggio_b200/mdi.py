"""Multi-stage delta-Ising detection (MDI-MIMO) on the device, with the reference's control flow.

`detect` restates run_a513.detect / mdi_logged (arpeggio/sim/local_code_a513/run_a513.py:42-130, the same walk as
mimo.mdi, arpeggio/mimo/mimo.py:553-602): guesses MMSE and ordered MMSE-SIC; per stage the radius R_g of
each guess (mimo.mdi_radius), and for each guess, K = 1..Rmax and each distinct total radius t (ascending)
of the uses that need K, one solver call over those uses with ceil(Ns / t) anneals on the dDI problem of
2K copies around the guess; a guess is replaced by its closest candidate when strictly closer; after the
stages the closer of the two guesses is the decision.  The anneal keys and instance numbers are the
reference's (key = seed_base + call * 0xD1B54A32D192ED03 + 0xA513, seed_base = seed * 0x9E3779B97F4A7C15,
inst = the use's index in the batch), so with the reference's draws the first-accept anneals see exactly the
sub-problems, keys and counters of the recorded B200 runs wherever the float mapping rounds the same way.

The host only walks the groups (it reads each stage's radii back to form them); every per-use computation
is a kernel: arp_mdi_guesses, arp_mdi_radius, arp_mdi_map, the anneal, arp_mdi_update, arp_mdi_select."""
import math

import numpy as np
import torch

from . import _lib
from .arpeggiofx import anneal, check_status
from .detector import PAM, arpeggio_schedule, chord_schedule, el2

M64 = 0xFFFFFFFFFFFFFFFF
M32 = 0xFFFFFFFF
KEY_STEP = 0xD1B54A32D192ED03
KEY_TAG = 0xA513
# Table I settings of the MDI wrapper (arpeggio/mimo/mdi_solvers.py:19-22)
MDI_CFG = {(16, 16): dict(Rmax=3, S=8), (32, 16): dict(Rmax=3, S=8), (64, 16): dict(Rmax=3, S=8),
           (32, 4): dict(Rmax=1, S=1)}


def parse_pick(pick):
    """abl_far_<S>_<T0>_<T1>_<q>_<start>_<Ns> (run_a513.parse_pick, run_a513.py:35-39) -> dict."""
    a = pick.split('_')
    assert a[0] == 'abl' and a[1] == 'far' and len(a) == 8, pick
    return dict(S=int(a[2]), T0=float(a[3]), T1=float(a[4]), q=float(a[5]), start=a[6], Ns=int(a[7]))


@torch.no_grad()
def detect(H, y, N0, M, seed, pick, Rmax=None, stages=None, policy='arpeggio', precision='int', counters=None):
    """H (B, 2Nr, 2Nt), y (B, 2Nr) float32 (device or host), N0 scalar, M in {4, 16}; seed = the batch's draw
    seed (run_a513 passes arpx.draw_seed(seed, snr, bi)); pick: dict or abl_far_* string.
    Returns (levels (B, D) int8 on the device, anneals per use (B,) float64 numpy, per-K counters
    {K: [flips, tests, anneals]}, for the integer Chord round {K: [flips, steps, anneals, n1]} with n1 the rounds
    that flipped)."""
    pk = parse_pick(pick) if isinstance(pick, str) else dict(pick)
    dev = torch.device('cuda')
    H = torch.as_tensor(H, dtype=torch.float32).to(dev).contiguous()
    y = torch.as_tensor(y, dtype=torch.float32).to(dev).contiguous()
    B, NR2, D = H.shape
    cfg = MDI_CFG.get((D // 2, M), dict(Rmax=3, S=8))
    Rmax = cfg['Rmax'] if Rmax is None else Rmax
    S = cfg['S'] if stages is None else stages
    L = _lib.lib()
    sp = _lib.stream_ptr()
    sigma2 = torch.full((B,), (N0 / 2) / el2(M), dtype=torch.float32, device=dev)
    G = 2
    cur = torch.empty(B, G, D, dtype=torch.int8, device=dev)
    xm, xs = torch.empty(B, D, dtype=torch.int8, device=dev), torch.empty(B, D, dtype=torch.int8, device=dev)
    _lib.check(L.arp_mdi_guesses(_lib.ptr(H), _lib.ptr(y), _lib.ptr(sigma2), B, NR2, D, M, _lib.ptr(xm),
                                 _lib.ptr(xs), sp), 'mdi_guesses')
    cur[:, 0].copy_(xm)
    cur[:, 1].copy_(xs)
    Rd = torch.empty(B, G, dtype=torch.int32, device=dev)
    dist = torch.empty(B, G, dtype=torch.float32, device=dev)
    ann = np.zeros(B)
    cnt = counters if counters is not None else {}
    seed_base = (seed * 0x9E3779B97F4A7C15) & M64
    calls = 0
    qscale = 1 if precision == 'int' else 0
    tdt = torch.int32 if precision == 'int' else torch.float32
    sched = {}
    for K in range(1, Rmax + 1):
        if policy == 'arpeggio':
            T, q, c = arpeggio_schedule(pk['S'], pk['T0'], pk['T1'], pk['q'], K, precision)
        else:  # Chord's MDI schedule: 128 steps per copy pair (mdi_solvers.py:18, MDICHORD)
            T, q, c = chord_schedule(pk.get('steps_per_copy_pair', 128) * 2 * K, pk['T0'], pk['T1'], pk['q'],
                                     pk.get('kappa', 0.0), precision=precision)
        sched[K] = (torch.tensor(T, dtype=tdt, device=dev), q,
                    None if c is None else torch.tensor(c, dtype=tdt, device=dev))
    status = torch.zeros(1, dtype=torch.int32, device=dev)
    for st in range(S):
        _lib.check(L.arp_mdi_radius(_lib.ptr(H), _lib.ptr(y), _lib.ptr(cur), B, NR2, D, G, M, Rmax, _lib.ptr(Rd),
                                    _lib.ptr(dist), sp), 'mdi_radius')
        R = Rd.cpu().numpy()
        tot = R.sum(1)
        if int(tot.max()) == 0:
            break
        nxt = cur.clone()
        bd = dist.clone()
        for gi in range(G):
            for K in range(1, Rmax + 1):
                need = R[:, gi] >= K
                if not need.any():
                    continue
                P = 2 * K
                for t in np.unique(tot[need]).tolist():
                    idx_np = np.nonzero(need & (tot == t))[0]
                    n = len(idx_np)
                    na = math.ceil(pk['Ns'] / t)
                    idx = torch.from_numpy(idx_np.astype(np.int32)).to(dev)
                    Gm = torch.empty(n, D, D, dtype=tdt, device=dev)
                    hm = torch.empty(n, D, dtype=tdt, device=dev)
                    xq = torch.empty(n, D, dtype=torch.int8, device=dev)
                    sc = torch.empty(n, dtype=torch.float32, device=dev)
                    _lib.check(L.arp_mdi_map(_lib.ptr(H), _lib.ptr(y), _lib.ptr(idx), n, NR2, D, M, _lib.ptr(cur),
                                             G, gi, qscale, _lib.ptr(Gm), _lib.ptr(hm), _lib.ptr(xq), _lib.ptr(sc),
                                             _lib.ptr(status), sp), 'mdi_map')
                    key = (seed_base + calls * KEY_STEP + KEY_TAG) & M64
                    calls += 1
                    T, q, c = sched[K]
                    n1 = (torch.empty(n, na, dtype=torch.int64, device=dev)
                          if policy == 'chord' and precision == 'int' else None)
                    spins, de, stt, _ = anneal(Gm, hm, P, na, T, q, idx, key, pk['start'], policy, c, precision,
                                               status=status, n1=n1)
                    _lib.check(L.arp_mdi_update(_lib.ptr(H), _lib.ptr(y), _lib.ptr(idx), n, NR2, D, P, na, M,
                                                _lib.ptr(cur), G, gi, _lib.ptr(spins), _lib.ptr(nxt), _lib.ptr(bd),
                                                sp), 'mdi_update')
                    v = cnt.setdefault(str(K), [0, 0, 0] if n1 is None else [0, 0, 0, 0])
                    s_ = stt.sum((0, 1)).tolist()
                    v[0] += int(s_[0])
                    v[1] += int(s_[1])
                    v[2] += int(na * n)
                    if n1 is not None:
                        v[3] += int(n1.sum())
                    ann[idx_np] += na
        cur = nxt
    _lib.check(L.arp_mdi_radius(_lib.ptr(H), _lib.ptr(y), _lib.ptr(cur), B, NR2, D, G, M, Rmax, _lib.ptr(Rd),
                                _lib.ptr(dist), sp), 'mdi_radius')
    levels = torch.empty(B, D, dtype=torch.int8, device=dev)
    bits = torch.empty(B, D * PAM[M]['bits'], dtype=torch.int8, device=dev)
    _lib.check(L.arp_mdi_select(_lib.ptr(cur), _lib.ptr(dist), B, D, G, M, _lib.ptr(levels), _lib.ptr(bits), sp),
               'mdi_select')
    torch.cuda.synchronize()
    check_status(status)
    return levels, ann, cnt, bits
