"""CPU oracle for the delta-encoded Ising MIMO detector path -- TEST INFRASTRUCTURE ONLY.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import this module, and only
as the checker (or as the timed CPU restatement of the reference's algorithm).  The product path
(arpeggio_b200) never imports it and fails loudly when its CUDA library is missing.

Two halves:
  * ctypes bindings of arp_oracle.c (Philox4x32-10, integer and FP32 anneals, chord_fx);
  * numpy restatements of the host-side mapping and readout of arpeggio/mimo/mimo.py and
    arpeggio/mimo/chordfx.py, each citing the reference function it follows.

Parity pins: tests/golden/*.npz were produced by importing the reference itself
(tests/golden/make_golden.py); tests/test_oracle_golden.py checks this module against them.
"""
import ctypes
import math
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, 'liboracle.so')
MASK = 0xFFFFFFFF
QSCALE = 4096
_lib = None

_P = ctypes.c_void_p


def build():
    subprocess.check_call(['make', '-s', '-C', HERE], stdout=subprocess.DEVNULL)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(os.path.join(HERE, 'arp_oracle.c')):
            build()
        L = ctypes.CDLL(LIB)
        L.orc_philox_batch.argtypes = [_P, _P, ctypes.c_int]
        L.orc_anneal_dd.argtypes = [_P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _P,
                                    ctypes.c_int, ctypes.c_int32, _P, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int,
                                    ctypes.c_int, _P, _P, _P, ctypes.c_int]
        L.orc_anneal_chord.argtypes = [_P, _P, _P, _P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32,
                                       ctypes.c_int, _P, _P, ctypes.c_int]
        L.orc_anneal_dd_f32.argtypes = [_P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _P,
                                        ctypes.c_int, ctypes.c_float, _P, ctypes.c_uint32, ctypes.c_uint32,
                                        ctypes.c_int, ctypes.c_int, _P, _P, _P, ctypes.c_int]
        L.orc_anneal_full_f32.argtypes = [_P, _P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P,
                                          _P, ctypes.c_int, ctypes.c_float, _P, ctypes.c_uint32, ctypes.c_uint32,
                                          ctypes.c_int, _P, _P, _P, ctypes.c_int]
        L.orc_anneal_chord_hw.argtypes = [_P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _P,
                                          ctypes.c_int, ctypes.c_int32, _P, ctypes.c_uint64, _P, _P, _P, ctypes.c_int]
        L.orc_soft_trajectory.argtypes = [_P, _P, _P, _P, _P, _P, _P, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, ctypes.c_uint32,
                                          ctypes.c_uint32, _P, _P, _P, _P, ctypes.c_int]
        L.orc_anneal_chord_dd_n1.argtypes = [_P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, _P,
                                             ctypes.c_int, ctypes.c_int32, _P, ctypes.c_uint32, ctypes.c_uint32,
                                             ctypes.c_int, _P, _P, _P, _P, ctypes.c_int]
        _lib = L
    return _lib


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


# ---------------------------------------------------------------- RNG
def philox(words):
    """words (n, 6) uint32: counter c0..c3, key k0, k1 -> (n, 4) uint32 (chordfx.py:39-49)."""
    w = np.ascontiguousarray(np.asarray(words, dtype=np.uint64) & MASK, dtype=np.uint32)
    out = np.zeros((w.shape[0], 4), dtype=np.uint32)
    lib().orc_philox_batch(_ptr(w), _ptr(out), w.shape[0])
    return out


# ---------------------------------------------------------------- anneals
def anneal_dd(G, h, P, R, T, q, inst, key, start, policy='arpeggio', c=None, nthreads=1):
    """Integer anneal on the compressed dDI problem; contract of arpeggiofx.solve
    (arpeggio/sim/arpeggiofx.py:22-44) and arpeggio_ref59.anneal (rtl_a59/src/arpeggio_ref59.py:41-85).
    Returns spins (B, R, P*D) int8 copy-major, best energy change (B, R) int64, (B, R, 2) [flips, tests]."""
    G = np.ascontiguousarray(G, dtype=np.int32)
    h = np.ascontiguousarray(h, dtype=np.int32)
    B, D, _ = G.shape
    T = np.ascontiguousarray([int(x) for x in T], dtype=np.int32)
    cc = None if c is None else np.ascontiguousarray([int(x) for x in c], dtype=np.int32)
    it = np.ascontiguousarray(np.asarray(inst, dtype=np.int64) & MASK, dtype=np.uint32)
    out_s = np.zeros((B, R, P * D), dtype=np.int8)
    out_de = np.zeros((B, R), dtype=np.int64)
    out_st = np.zeros((B, R, 2), dtype=np.int64)
    rc = lib().orc_anneal_dd(_ptr(G), _ptr(h), B, D, P, R, _ptr(T), _ptr(cc), len(T), int(q), _ptr(it),
                             key & MASK, (key >> 32) & MASK, 0 if start == 'rand' else 1,
                             0 if policy == 'arpeggio' else 1, _ptr(out_s), _ptr(out_de), _ptr(out_st), nthreads)
    if rc:
        raise ValueError('orc_anneal_dd: unsupported shape')
    return out_s, out_de, out_st


def anneal_chord_n1(G, h, P, R, T, c, q, inst, key, start, nthreads=1):
    """anneal_dd's Chord round plus the rounds with at least one flip per anneal (n1 of arpeggio_ref59.anneal,
    rtl_a59/src/arpeggio_ref59.py:74), the term of the Chord engine's latency 3 L + F + n1.  Returns spins, best
    energy change, (flips, tests) and n1 (B, R) int64."""
    G = np.ascontiguousarray(G, dtype=np.int32)
    h = np.ascontiguousarray(h, dtype=np.int32)
    B, D, _ = G.shape
    T = np.ascontiguousarray([int(x) for x in T], dtype=np.int32)
    cc = None if c is None else np.ascontiguousarray([int(x) for x in c], dtype=np.int32)
    it = np.ascontiguousarray(np.asarray(inst, dtype=np.int64) & MASK, dtype=np.uint32)
    out_s = np.zeros((B, R, P * D), dtype=np.int8)
    out_de = np.zeros((B, R), dtype=np.int64)
    out_st = np.zeros((B, R, 2), dtype=np.int64)
    out_n1 = np.zeros((B, R), dtype=np.int64)
    rc = lib().orc_anneal_chord_dd_n1(_ptr(G), _ptr(h), B, D, P, R, _ptr(T), _ptr(cc), len(T), int(q), _ptr(it),
                                      key & MASK, (key >> 32) & MASK, 0 if start == 'rand' else 1, _ptr(out_s),
                                      _ptr(out_de), _ptr(out_st), _ptr(out_n1), nthreads)
    if rc:
        raise ValueError('orc_anneal_chord_dd_n1: unsupported shape')
    return out_s, out_de, out_st, out_n1


def soft_trajectory(J, hf, h0, scale, c0, T, s0, q, S, R, D, M, inst, key, nthreads=1):
    """The trajectory sampler of mimo.chord_soft (arpeggio/mimo/mimo.py:332-394) with this project's Philox draws,
    restated operation for operation as the device computes it.  Returns m0, m1 (B, D nb), best_d (B), best_l
    (B, D)."""
    J = np.ascontiguousarray(J, dtype=np.float32)
    B = J.shape[0]
    nb = 2 if M == 16 else 1
    arr = lambda a: np.ascontiguousarray(a, dtype=np.float32)
    hf, h0, scale, c0, T = arr(hf), arr(h0), arr(scale), arr(c0), arr(T)
    s0 = None if s0 is None else np.ascontiguousarray(s0, dtype=np.int8)
    it = np.ascontiguousarray(np.asarray(inst, dtype=np.int64) & MASK, dtype=np.uint32)
    m0 = np.zeros((B, D * nb), dtype=np.float32)
    m1 = np.zeros((B, D * nb), dtype=np.float32)
    bd = np.zeros(B, dtype=np.float32)
    bl = np.zeros((B, D), dtype=np.int8)
    rc = lib().orc_soft_trajectory(_ptr(J), _ptr(hf), _ptr(h0), _ptr(scale), _ptr(c0), _ptr(T), _ptr(s0), float(q),
                                   S, R, D, M, B, _ptr(it), key & MASK, (key >> 32) & MASK, _ptr(m0), _ptr(m1),
                                   _ptr(bd), _ptr(bl), nthreads)
    if rc:
        raise ValueError('orc_soft_trajectory: unsupported shape')
    return m0, m1, bd, bl


def anneal_chord_hw(G, h, P, R, T, c, q, inst, key, nthreads=1):
    """Chord's round on the compressed problem with the random numbers of the reference's C++ engine model run
    without Philox (arpeggio/sim/x3model/engine_model.cpp, philox = 0; restated in arp_oracle.c).  T and c (L,)
    one entry per step (c may be None).  Returns spins (B, R, P*D) int8, best energy change (B, R) int64 and
    (B, R, 2) [flips, steps]."""
    G = np.ascontiguousarray(G, dtype=np.int32)
    h = np.ascontiguousarray(h, dtype=np.int32)
    B, D, _ = G.shape
    T = np.ascontiguousarray([int(x) for x in T], dtype=np.int32)
    cc = None if c is None else np.ascontiguousarray([int(x) for x in c], dtype=np.int32)
    it = np.ascontiguousarray(np.asarray(inst, dtype=np.int64) & MASK, dtype=np.uint32)
    out_s = np.zeros((B, R, P * D), dtype=np.int8)
    out_de = np.zeros((B, R), dtype=np.int64)
    out_st = np.zeros((B, R, 2), dtype=np.int64)
    rc = lib().orc_anneal_chord_hw(_ptr(G), _ptr(h), B, D, P, R, _ptr(T), _ptr(cc), len(T), int(q), _ptr(it),
                                   key & 0xFFFFFFFFFFFFFFFF, _ptr(out_s), _ptr(out_de), _ptr(out_st), nthreads)
    if rc:
        raise ValueError('orc_anneal_chord_hw: unsupported shape')
    return out_s, out_de, out_st


def anneal_dd_f32(G, h, P, R, T, q, inst, key, start, policy='arpeggio', c=None, nthreads=1):
    """FP32-field anneal on the compressed dDI problem (float rule written out in arp_oracle.c)."""
    G = np.ascontiguousarray(G, dtype=np.float32)
    h = np.ascontiguousarray(h, dtype=np.float32)
    B, D, _ = G.shape
    T = np.ascontiguousarray(T, dtype=np.float32)
    cc = None if c is None else np.ascontiguousarray(c, dtype=np.float32)
    it = np.ascontiguousarray(np.asarray(inst, dtype=np.int64) & MASK, dtype=np.uint32)
    out_s = np.zeros((B, R, P * D), dtype=np.int8)
    out_de = np.zeros((B, R), dtype=np.float32)
    out_st = np.zeros((B, R, 2), dtype=np.int64)
    rc = lib().orc_anneal_dd_f32(_ptr(G), _ptr(h), B, D, P, R, _ptr(T), _ptr(cc), len(T), float(q), _ptr(it),
                                 key & MASK, (key >> 32) & MASK, 0 if start == 'rand' else 1,
                                 0 if policy == 'arpeggio' else 1, _ptr(out_s), _ptr(out_de), _ptr(out_st), nthreads)
    if rc:
        raise ValueError('orc_anneal_dd_f32: unsupported shape')
    return out_s, out_de, out_st


def anneal_full_f32(J, h, P, R, T, q, inst, key, s0=None, policy='arpeggio', c=None, nthreads=1):
    """FP32-field anneal on a full symmetric J (B, N, N) with N/P lanes per bank (rule in arp_oracle.c, after
    arpeggio/sim/arpx55.py:28-99); s0 (B, N) start spins or None for 'rand'.  Returns spins (B, R, N) int8,
    best energy change (B, R) float32 (E0 units: flipping s_g changes E0 by 2 s_g u_g), (B, R, 2) [flips, tests]."""
    J = np.ascontiguousarray(J, dtype=np.float32)
    h = np.ascontiguousarray(h, dtype=np.float32)
    B, N = h.shape
    T = np.ascontiguousarray(T, dtype=np.float32)
    cc = None if c is None else np.ascontiguousarray(c, dtype=np.float32)
    ss = None if s0 is None else np.ascontiguousarray(s0, dtype=np.int8)
    it = np.ascontiguousarray(np.asarray(inst, dtype=np.int64) & MASK, dtype=np.uint32)
    out_s = np.zeros((B, R, N), dtype=np.int8)
    out_de = np.zeros((B, R), dtype=np.float32)
    out_st = np.zeros((B, R, 2), dtype=np.int64)
    rc = lib().orc_anneal_full_f32(_ptr(J), _ptr(h), _ptr(ss), B, N, P, R, _ptr(T), _ptr(cc), len(T), float(q),
                                   _ptr(it), key & MASK, (key >> 32) & MASK, 0 if policy == 'arpeggio' else 1,
                                   _ptr(out_s), _ptr(out_de), _ptr(out_st), nthreads)
    if rc:
        raise ValueError('orc_anneal_full_f32: unsupported shape')
    return out_s, out_de, out_st


def ising_ri(H, y, z_mmse, M, r=0.15):
    """mimo.ising (mimo.py:132-149), float64: T = [2I, I] (16-QAM) or I (QPSK), h = 2 (HT)^T y, J = -offdiag(T^T Q T),
    scale = max(|h|, |J|); returns h_reg = h0 + 2 r sP, h0, J (scaled), sP (spins of the hard MMSE z), scale."""
    H = np.asarray(H, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    D = H.shape[-1]
    T = np.eye(D) if M == 4 else np.concatenate([2 * np.eye(D), np.eye(D)], 1)
    HT = H @ T
    h = 2 * np.einsum('bij,bi->bj', HT, y)
    Q = np.einsum('bki,bkj->bij', HT, HT)
    J = -(Q - np.einsum('bii->bi', Q)[:, :, None] * np.eye(Q.shape[-1]))
    scale = np.maximum(np.abs(h).max(-1), np.abs(J).reshape(J.shape[0], -1).max(-1))
    scale = np.maximum(scale, 1e-12)
    h0 = h / scale[:, None]
    J = J / scale[:, None, None]
    l = quantize_levels(np.asarray(z_mmse, dtype=np.float64), M)
    sP = l.copy() if M == 4 else np.concatenate([np.where(l > 0, 1.0, -1.0), np.where((l == 3) | (l == -1), 1.0, -1.0)], -1)
    return h0 + 2 * r * sP, h0, J, sP, scale


def energy_full(h, J, s):
    """E0 = -h.s - s^T J s for s (B, R, N) (mimo.energy0, mimo.py:193-195), float64."""
    h = np.asarray(h, dtype=np.float64)
    J = np.asarray(J, dtype=np.float64)
    s = np.asarray(s, dtype=np.float64)
    return -(s * h[:, None, :]).sum(-1) - np.einsum('bri,bij,brj->br', s, J, s)


def chord_fx(J, h, h0, T, c, q, S, P, R, seed, inst0=0, mode='chains', nthreads=1):
    """chordfx.chord_fx (arpeggio/mimo/chordfx.py:80-118) on int16 J (B, N, N), int32 h/h0 (B, N).
    Returns (spins int8 (B, R, N) or (B, N), 2 E0 int64 (B, R) or (B,))."""
    J = np.ascontiguousarray(J, dtype=np.int16)
    h = np.ascontiguousarray(h, dtype=np.int32)
    h0 = np.ascontiguousarray(h0, dtype=np.int32)
    B, N = h.shape
    T = np.ascontiguousarray([int(x) for x in T], dtype=np.int32)
    c = np.ascontiguousarray([int(x) for x in c], dtype=np.int32)
    if mode == 'best':
        out_e = np.zeros(B, dtype=np.int64)
        out_s = np.zeros((B, N), dtype=np.int8)
    else:
        out_e = np.zeros((B, R), dtype=np.int64)
        out_s = np.zeros((B, R, N), dtype=np.int8)
    rc = lib().orc_anneal_chord(_ptr(J), _ptr(h), _ptr(h0), _ptr(T), _ptr(c), int(q), int(S), P, R, N, B,
                                seed & MASK, (seed >> 32) & MASK, inst0 & MASK, 1 if mode == 'best' else 0,
                                _ptr(out_e), _ptr(out_s), nthreads)
    if rc:
        raise ValueError('orc_anneal_chord: unsupported shape')
    return out_s, out_e


# ---------------------------------------------------------------- constellation (mimo.py:19-51)
PAM = {4: dict(levels=[-1, 1], a=1 / math.sqrt(2), bits=1),
       16: dict(levels=[-3, -1, 1, 3], a=1 / math.sqrt(10), bits=2),
       64: dict(levels=[-7, -5, -3, -1, 1, 3, 5, 7], a=1 / math.sqrt(42), bits=3)}


def levels_to_bits(l, M):
    """mimo.levels_to_bits (mimo.py:45-51): per dimension MSB first (64-QAM, which the reference does not have:
    the binary-reflected Gray code of the level index)."""
    l = np.asarray(l)
    if M == 4:
        return (l > 0).astype(np.int8)
    if M == 64:
        i = (l.astype(np.int64) + 7) // 2
        g = i ^ (i >> 1)
        return np.stack([(g >> (2 - k)) & 1 for k in range(3)], -1).reshape(*l.shape[:-1], -1).astype(np.int8)
    b1 = (l > 0).astype(np.int8)
    b2 = (np.abs(l) == 1).astype(np.int8)
    return np.stack([b1, b2], -1).reshape(*l.shape[:-1], -1)


def quantize_levels(z, M):
    """mimo.quantize_levels (mimo.py:86-88): nearest level, first on ties."""
    lv = np.asarray(PAM[M]['levels'], dtype=z.dtype)
    return lv[np.abs(z[..., None] - lv).argmin(-1)]


# ---------------------------------------------------------------- MMSE and dDI mapping (float64)
def mmse(H, y, N0, M):
    """mimo.mmse (mimo.py:98-109) and mimo._mu (:176-182) in float64: z, mu, hard guess x_q."""
    H = np.asarray(H, dtype=np.float64)
    y = np.asarray(y, dtype=np.float64)
    lv = np.asarray(PAM[M]['levels'], dtype=np.float64)
    el2 = float((lv ** 2).mean())
    G = np.einsum('bki,bkj->bij', H, H)
    D = G.shape[-1]
    A = G + (N0 / 2) / el2 * np.eye(D)
    z = np.linalg.solve(A, np.einsum('bki,bk->bi', H, y)[..., None])[..., 0]
    mu = np.diagonal(np.linalg.solve(A, G), axis1=-2, axis2=-1)
    return z, mu, quantize_levels(z / mu, M)


def ising_delta_compressed(H, y, xg):
    """mimo.ising_delta_at (mimo.py:506-523) for any K, in compressed form: the N x N coupling is
    J = -offdiag(Q (x) 1 1^T) with Q = H^T H, so G = Q/scale and h = 2 H^T (y - H xg)/scale;
    scale = max(|h|_inf, |Q|_inf) (every entry of Q, the diagonal included, is an off-diagonal
    entry of J once K >= 1).  Returns float64 (G, h, scale)."""
    H = np.asarray(H, dtype=np.float64)
    yb = np.asarray(y, dtype=np.float64) - np.einsum('bij,bj->bi', H, np.asarray(xg, dtype=np.float64))
    h = 2 * np.einsum('bij,bi->bj', H, yb)
    Q = np.einsum('bki,bkj->bij', H, H)
    scale = np.maximum(np.abs(h).max(-1), np.abs(Q).reshape(Q.shape[0], -1).max(-1))
    scale = np.maximum(scale, 1e-12)
    return Q / scale[:, None, None], h / scale[:, None], scale


def gram_digits(H):
    """Q = H^T H as this project's map forms it on the tensor cores (no reference counterpart: the reference forms
    it in FP32 with torch matmul, mimo.py:100-104): per use H scaled by 2^s (largest |H| just below 2^30), rounded
    to integers x, split into signed base-256 digits x = sum_a 2^(8a) d_a; the products d_a^T d_b of weight
    a + b >= 3 summed exactly (integers, then a float64 sum that is exact below 2^53 steps of 2^24), scaled by
    2^-2s and rounded once to float32.  Returns float32 Q (B, D, D)."""
    H = np.asarray(H, dtype=np.float32)
    B, NR2, D = H.shape
    out = np.zeros((B, D, D), dtype=np.float32)
    pairs = [(a, b) for a in range(4) for b in range(4) if a + b >= 3]
    for u in range(B):
        m = float(np.abs(H[u]).max())
        s = 30 - np.frexp(m)[1] if m > 0 else 0
        x = np.rint(np.ldexp(H[u].astype(np.float64), s)).astype(np.int64)
        d = []
        for _ in range(3):
            lo = ((x & 0xFF) ^ 0x80) - 0x80
            d.append(lo)
            x = (x - lo) >> 8
        d.append(x)
        cls = {w: np.zeros((D, D), dtype=np.int64) for w in (3, 4, 5, 6)}
        for a, b in pairs:
            cls[a + b] += d[a].T @ d[b]
        q = sum(np.ldexp(cls[w].astype(np.float64), 8 * w) for w in (6, 5, 4, 3))
        out[u] = np.ldexp(q, -2 * s).astype(np.float32)
    return out


def geom(t0, t1, S):
    """mimo.geom (mimo.py:199-201): float64 schedule rounded once to float32."""
    k = np.arange(S, dtype=np.float64)
    return (t0 * (t1 / t0) ** (k / max(1, S - 1))).astype(np.float32)


def arpeggio_schedule(T0, T1, S, q, K, Q=QSCALE):
    """run_a513.arpeggio_schedule (sim/local_code_a513/run_a513.py:83-87): S sweeps x P passes."""
    Tsw = [int(round(float(v) * Q)) for v in geom(T0, T1, S).astype(np.float64)]
    return [t for t in Tsw for _ in range(2 * K)], int(round(q * Q))


def chord_schedule(S, t0, t1, q, kappa=0.0, ramp=True, Q=QSCALE):
    """The schedule half of chordfx.to_fixed (chordfx.py:66-76): T, c (S,) int32 and q."""
    T = geom(t0, t1, S).astype(np.float64)
    rho = np.ones(S)
    if ramp:
        t = np.arange(S, dtype=np.float64)
        rho = np.where(t >= 0.7 * S, (S - 1 - t) / max(1.0, S - 1 - 0.7 * S), 1.0)
    c = np.zeros(S)
    c[1:] = kappa * T[:-1] * rho[1:]
    return (np.round(T * Q).astype(np.int32), np.round(c * Q).astype(np.int32), int(round(q * Q)))


def quantize_compressed(Gf, hf, Q=QSCALE):
    """chordfx.to_fixed + chord_ref.compress (chordfx.py:60-65, chord_ref.py:47-59) on the compressed
    form: the symmetrised G rounded half-to-even (torch.round) to int16, h to int32."""
    Gs = (Gf + np.swapaxes(Gf, 1, 2)) / 2
    return np.round(Gs * Q).astype(np.int32), np.round(hf * Q).astype(np.int32)


def expand(G, h, K):
    """chord_ref.expand (chord_ref.py:62-69): compressed (G, h) -> int16 J (B, N, N), int32 h (B, N)."""
    B, D, _ = G.shape
    N = 2 * K * D
    J = -np.tile(G, (1, 2 * K, 2 * K))
    J[:, np.arange(N), np.arange(N)] = 0
    return J.astype(np.int16), np.tile(h, (1, 2 * K)).astype(np.int32)


# ---------------------------------------------------------------- readout (mimo.py:185-190, 416-431)
def spins_to_levels_delta(S, xq, K, M):
    S = np.asarray(S)
    D = xq.shape[-1]
    d = S.reshape(*S.shape[:-1], 2 * K, D).astype(np.int64).sum(-2)
    lv = PAM[M]['levels']
    return np.clip(xq[:, None, :] + d, lv[0], lv[-1])


def dist(H, y, L):
    """||y - H l||^2 for candidates L (B, C, D) (mimo.dist)."""
    r = np.asarray(y, dtype=np.float64)[:, None, :] - np.einsum('bij,bkj->bki', np.asarray(H, dtype=np.float64), L)
    return (r ** 2).sum(-1)


def select(H, y, cand, guess):
    """mimo.select (mimo.py:421-425): the lowest distance among the candidates and the guess."""
    allc = np.concatenate([cand, guess[:, None, :]], 1)
    d = dist(H, y, allc)
    im = d.argmin(1)
    return allc[np.arange(allc.shape[0]), im], d[np.arange(allc.shape[0]), im]


def energy_dd(G, h, S, K):
    """Ising energy E0 = -h0.s - s^T J s of dDI spins S (B, R, 2K D) in the compressed form:
    E0 = -h.m + m^T G m - P tr(G), m = sum over copies (mimo.energy0, mimo.py:193-195). float64."""
    G = np.asarray(G, dtype=np.float64)
    h = np.asarray(h, dtype=np.float64)
    B, D, _ = G.shape
    P = 2 * K
    m = np.asarray(S, dtype=np.float64).reshape(S.shape[0], S.shape[1], P, D).sum(2)
    tr = np.trace(G, axis1=1, axis2=2)
    return -(m * h[:, None]).sum(-1) + np.einsum('brj,bjk,brk->br', m, G, m) - P * tr[:, None]


def gray_neighbours(l, M):
    """Single-bit-flip neighbours of levels l (B, D): (B, D*nb, D), bit order dim-major, MSB first
    (the construction of mimo.list_llr, mimo.py:441-455)."""
    l = np.asarray(l)
    B, D = l.shape
    nb = PAM[M]['bits']
    out = np.repeat(l[:, None, :], D * nb, axis=1).copy()
    for j in range(D):
        for k in range(nb):
            v = l[:, j]
            out[:, j * nb + k, j] = -v if k == 0 else np.sign(v) * (4 - np.abs(v))
    return out


def list_llr(H, y, N0, allc, d, best, M, clip=50.0):
    """mimo.list_llr (mimo.py:434-462): max-log LLRs (positive = bit 1) over the list (allc, d) and the
    single-bit-flip neighbours of `best`, clipped to +-clip.  float64."""
    nbr = gray_neighbours(best, M)
    allc2 = np.concatenate([allc, nbr], 1)
    d2 = np.concatenate([d, dist(H, y, nbr)], 1)
    bits = levels_to_bits(allc2, M).astype(bool)
    m1 = np.where(bits, d2[..., None], np.inf).min(1)
    m0 = np.where(~bits, d2[..., None], np.inf).min(1)
    return np.clip((m0 - m1) / N0, -clip, clip)


# ---------------------------------------------------------------- learned warm start (no reference counterpart)
# The reference has no learned component, so these restate this package's own warm-start definitions (feature
# map, bf16 MLP, warm start, warm anneal) for the GPU parity tests; parity here is self-consistency, not a pin
# to the reference.
NF, NH, NO = 16, 256, 16


def bf16(x):
    """Round float32 to bfloat16 (nearest, ties to even), returned as float32."""
    x = np.ascontiguousarray(x, dtype=np.float32)
    u = x.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return (r & 0xFFFFFFFF).astype(np.uint32).view(np.float32).reshape(x.shape)


def warm_features(G, h, xq, zs, snr_db, M, P, levels=None):
    """Per-coordinate features (B*D, 16) float32 before bf16 rounding, and labels (levels - xq)/2 + P/2."""
    G = np.asarray(G, dtype=np.float64)
    h = np.asarray(h, dtype=np.float64)
    B, D, _ = G.shape
    dg = np.diagonal(G, axis1=1, axis2=2)
    off = G.copy()
    off[:, np.arange(D), np.arange(D)] = 0
    ss = (off ** 2).sum(1)
    mdg = dg.mean(1, keepdims=True)
    Lmax = {4: 1, 16: 3, 64: 7}[M]
    x = np.asarray(xq, dtype=np.float64)
    f = np.zeros((B, D, NF))
    with np.errstate(divide='ignore', invalid='ignore'):
        f[..., 0] = np.clip(np.where(dg > 0, h / (4 * dg), 0), -8, 8)
        f[..., 1] = np.where(mdg > 0, dg / mdg, 0)
        f[..., 2] = np.minimum(np.where(dg > 0, np.sqrt(ss) / dg, 0), 64)
    f[..., 3] = 0 if snr_db is None else np.asarray(snr_db, dtype=np.float64)[:, None] * 0.05
    f[..., 4] = x / Lmax
    f[..., 5] = x == Lmax
    f[..., 6] = x == -Lmax
    f[..., 7] = 0 if zs is None else np.clip(0.5 * (np.asarray(zs, dtype=np.float64) - x), -4, 4)
    f[..., 8] = 1
    # two Jacobi refinements of the single-coordinate move (others at their previous greedy move)
    xi = np.asarray(xq, dtype=np.int64)

    def quant(u):
        m = 2 * np.clip(np.rint(u), -1, 1).astype(np.int64)
        m = np.where(xi + m > Lmax, Lmax - xi, m)
        return np.where(xi + m < -Lmax, -Lmax - xi, m)
    with np.errstate(divide='ignore', invalid='ignore'):
        m = np.where(dg > 0, quant(np.where(dg > 0, h / (4 * dg), 0)), 0)
        for k in (9, 10):
            acc = np.einsum('bij,bi->bj', off, m.astype(np.float64))
            u = np.clip(np.where(dg > 0, (h - 2 * acc) / (4 * dg), 0), -8, 8)
            f[..., k] = u
            m = np.where(dg > 0, quant(u), 0)
    lab = None
    if levels is not None:
        lab = np.clip((np.asarray(levels, dtype=np.int64) - np.asarray(xq, dtype=np.int64)) // 2 + P // 2, 0, P)
        lab = lab.reshape(-1).astype(np.int8)
    return f.reshape(B * D, NF).astype(np.float32), lab


def mlp_forward(X, W1, b1, W2, b2, W3t, b3):
    """The warm-start MLP with the device's roundings: bf16 operands, fp32 accumulate, bf16 hidden activations."""
    Xb = bf16(X)
    H1 = bf16(np.maximum(Xb @ bf16(W1).T + b1, 0))
    H2 = bf16(np.maximum(H1 @ bf16(W2).T + b2, 0))
    Z = H2 @ bf16(W3t) + b3
    return H1, H2, Z.astype(np.float32)


def mlp_backward(X, labels, C, W1, W2, W3t, H1, H2, Z):
    """Gradients of the summed softmax cross-entropy (over the first C logits) with the device's roundings
    (bf16 logit gradients and masked hidden gradients).  Returns dict of sums over rows (unscaled)."""
    lab = np.asarray(labels, dtype=np.int64)
    z = Z[:, :C].astype(np.float64)
    zm = z.max(1, keepdims=True)
    e = np.exp(z - zm)
    p = e / e.sum(1, keepdims=True)
    valid = lab >= 0
    g = np.zeros((Z.shape[0], NO))
    g[:, :C] = p
    g[np.arange(len(lab))[valid], lab[valid]] -= 1
    g[~valid] = 0
    loss = float((np.log(e.sum(1)) + zm[:, 0] - z[np.arange(len(lab)), np.maximum(lab, 0)])[valid].sum())
    dZ3 = bf16(g.astype(np.float32))
    gW3t = H2.T.astype(np.float64) @ dZ3
    gb3 = dZ3.sum(0)
    dZ2 = bf16(np.where(H2 > 0, dZ3 @ bf16(W3t).T, 0).astype(np.float32))
    gW2 = dZ2.T.astype(np.float64) @ H1
    gb2 = dZ2.sum(0)
    dZ1 = bf16(np.where(H1 > 0, dZ2 @ bf16(W2), 0).astype(np.float32))
    gW1 = dZ1.T.astype(np.float64) @ bf16(X)
    gb1 = dZ1.sum(0)
    return dict(W1=gW1, b1=gb1, W2=gW2, b2=gb2, W3t=gW3t, b3=gb3, loss=loss, dZ3=dZ3, dZ2=dZ2, dZ1=dZ1)


def warm_start(logits, G, h, xq, P, M):
    """Start spin sums m0 (B, D), flip-test order perm (B, D), start energy e0 (B) and kept (B): argmax class
    c -> m = 2c - P clamped to the constellation; order by descending 1 - p(m = 0) (ties by index); the start
    is kept iff e0 = 2 (m^T G m - h^T m) <= 0 (the anneal's energy units), else m = 0 in index order."""
    G = np.asarray(G)
    B, D, _ = G.shape
    C = P + 1
    Lmax = {4: 1, 16: 3, 64: 7}[M]
    z = np.asarray(logits, dtype=np.float32).reshape(B, D, -1)[..., :C].astype(np.float64)
    am = z.argmax(-1)
    e = np.exp(z - z.max(-1, keepdims=True))
    pz = e[..., P // 2] / e.sum(-1)
    sc = (1 - pz).astype(np.float32)
    x = np.asarray(xq, dtype=np.int64)
    m = 2 * am - P
    m = np.where(x + m > Lmax, Lmax - x, m)
    m = np.where(x + m < -Lmax, -Lmax - x, m)
    integer = np.issubdtype(G.dtype, np.integer)
    Gd = G.astype(np.int64) if integer else G.astype(np.float64)
    hd = np.asarray(h).astype(np.int64) if integer else np.asarray(h, dtype=np.float64)
    e0 = 2 * (np.einsum('bi,bij,bj->b', m, Gd, m) - (hd * m).sum(1))
    keep = e0 <= 0
    perm = np.zeros((B, D), dtype=np.uint8)
    m0 = np.where(keep[:, None], m, 0).astype(np.int8)
    for b in range(B):
        if keep[b]:
            order = sorted(range(D), key=lambda j: (-float(sc[b, j]), j))
            perm[b] = order
        else:
            perm[b] = np.arange(D)
    return m0, perm, np.where(keep, e0, 0), keep.astype(np.int32)


def warm_cdf(logits, xq, P, M, tau, kept):
    """Sampling thresholds (B, D, 2) uint32 of the sampled warm start (P = 2): softmax(tau z) over the classes
    m in {-2, 0, 2} whose level x + m stays inside the constellation; t0 = floor(2^32 p(m=-2)) (0 if -2 is out),
    t1 = floor(2^32 (p(m=-2) + p(m=0))) (0xFFFFFFFF if +2 is out); problems with kept = 0 get (0, 0xFFFFFFFF).
    Computed in float64: the device's single-precision exponentials agree to a few thousand units of 2^-32."""
    assert P == 2
    xq = np.asarray(xq, dtype=np.int64)
    B, D = xq.shape
    Lmax = {4: 1, 16: 3, 64: 7}[M]
    z = np.asarray(logits, dtype=np.float32).reshape(B, D, -1)[..., :3].astype(np.float64)
    q = np.exp(tau * (z - z.max(-1, keepdims=True)))
    ok0 = xq - 2 >= -Lmax
    ok2 = xq + 2 <= Lmax
    q0 = np.where(ok0, q[..., 0], 0.0)
    q2 = np.where(ok2, q[..., 2], 0.0)
    qs = q0 + q[..., 1] + q2
    t0 = np.where(ok0, np.floor(q0 / qs * 2.0 ** 32), 0)
    t1 = np.where(ok2, np.floor((q0 + q[..., 1]) / qs * 2.0 ** 32), 0xFFFFFFFF)
    out = np.stack([np.minimum(t0, 0xFFFFFFFF), np.minimum(t1, 0xFFFFFFFF)], -1).astype(np.uint32)
    keep = np.asarray(kept).astype(bool)
    out[~keep] = np.array([0, 0xFFFFFFFF], dtype=np.uint32)
    return out


def warm_counts(logits, P, kept, conf_min, r_easy, R):
    """Per-problem anneal counts (B) and confidences (B): confidence = sum_j log max_c softmax(z_j)_c over the
    P + 1 classes (float64; the device sums single-precision logarithms, so counts can differ only where the
    confidence is within a few 1e-4 of conf_min); r_easy where kept and confidence > conf_min, else R."""
    kept = np.asarray(kept).astype(bool)
    B = kept.shape[0]
    z = np.asarray(logits, dtype=np.float32).reshape(B, -1, np.asarray(logits).shape[-1])[..., :P + 1]
    z = z.astype(np.float64)
    conf = -np.log(np.exp(z - z.max(-1, keepdims=True)).sum(-1)).sum(-1)
    return np.where(kept & (conf > conf_min), r_easy, R).astype(np.int32), conf


def anneal_dd_warm(G, h, P, R, T, q, inst, key, m0, perm, nthreads=1, warm_r=None, cdf=None, ra=None):
    """First accept from the given start in the given flip-test order: the problem relabelled into scan order
    (position j' = coordinate perm[j']), annealed from spin sums m0 with the 'bal' pattern where m0 = 0, and the
    spins relabelled back.  With cdf (B, D, 2) uint32 (warm_cdf) anneals 0 < r < warm_r draw their start spin
    sums from the thresholds with word 1 of their start Philox block.  With ra (B) int32 problem b runs anneals
    r < ra[b] only; the others report zero spin sums, INT64_MAX and zero statistics."""
    G = np.asarray(G, dtype=np.int32)
    h = np.asarray(h, dtype=np.int32)
    B, D, _ = G.shape
    pm = np.asarray(perm, dtype=np.int64)
    bi = np.arange(B)[:, None]
    Gp = np.ascontiguousarray(G[bi[:, :, None], pm[:, :, None], pm[:, None, :]], dtype=np.int32)
    hp = np.ascontiguousarray(h[bi, pm], dtype=np.int32)
    mp = np.ascontiguousarray(np.asarray(m0, dtype=np.int8)[bi, pm], dtype=np.int8)
    cp = None if cdf is None else np.ascontiguousarray(np.asarray(cdf, dtype=np.uint32)[bi, pm], dtype=np.uint32)
    rp = None if ra is None else np.ascontiguousarray(ra, dtype=np.int32)
    T = np.ascontiguousarray([int(x) for x in T], dtype=np.int32)
    it = np.ascontiguousarray(np.asarray(inst, dtype=np.int64) & MASK, dtype=np.uint32)
    out_s = np.zeros((B, R, P * D), dtype=np.int8)
    out_de = np.zeros((B, R), dtype=np.int64)
    out_st = np.zeros((B, R, 2), dtype=np.int64)
    L = lib()
    L.orc_anneal_dd_warm.argtypes = [_P, _P, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, _P, ctypes.c_int,
                                     ctypes.c_int32, _P, ctypes.c_uint32, ctypes.c_uint32, _P, ctypes.c_int, _P, _P, _P,
                                     _P, _P, ctypes.c_int]
    rc = L.orc_anneal_dd_warm(_ptr(Gp), _ptr(hp), B, D, P, R, _ptr(T), len(T), int(q), _ptr(it), key & MASK,
                              (key >> 32) & MASK, _ptr(mp), R if warm_r is None else int(warm_r),
                              None if cp is None else _ptr(cp), None if rp is None else _ptr(rp), _ptr(out_s),
                              _ptr(out_de), _ptr(out_st), nthreads)
    if rc:
        raise ValueError('orc_anneal_dd_warm: unsupported shape')
    s = out_s.reshape(B, R, P, D)
    back = np.empty_like(s)
    back[np.arange(B)[:, None, None, None], np.arange(R)[None, :, None, None], np.arange(P)[None, None, :, None],
         pm[:, None, None, :]] = s
    return back.reshape(B, R, P * D), out_de, out_st
