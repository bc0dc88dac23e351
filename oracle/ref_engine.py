"""The reference's C++ Chord engine model (arpeggio/sim/x3model/engine_model.cpp), compiled from its own source by
`make -C oracle ref` into oracle/_ref/libape.so, reached through its batch entry point `engine_solve_batch`
(engine_model.cpp:336-379).  Test infrastructure and a CPU baseline only: the tests pin the oracle's and the
library's Chord round (compressed G, Philox counters of the first-accept kernel) against it, and bench.py times it.

What the engine computes with philox = 1 (seeder stage C :142-163, R-port :197-227, decision D2/D1/D0 :229-270, final
best check :128): start spins 'rand' from word 0
of Philox block (2^32 - 1, p D + j, r, inst); fields w = h - 2 G m; step k tests copy p = k % P, every coordinate
against the start-of-step snapshot, flip iff u 4 T_k > (s w_j + 2 G_jj + q - c_k + 2 T_k) 2^32 with u word n & 3 of
block (n >> 2, p D + j, r, inst), n = k // P; the flips commit in coordinate order (energy 4 s w_j + 8 G_jj, fields
w += 4 s G_j); the best state is the first minimum over the step ends.  G, h, T and c are int16 in the engine."""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, '_ref', 'libape.so')
_lib = None


def available():
    return os.path.exists(SO)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError('%s not built (make -C oracle ref needs the reference tree)' % SO)
        L = ctypes.CDLL(SO)
        P_, I = ctypes.c_void_p, ctypes.c_int
        L.engine_solve_batch.argtypes = [I, I, I, I, I, P_, P_, I, I, I, P_, P_, I, P_, ctypes.c_uint64, P_, P_, P_,
                                         P_, I]
        L.engine_solve_batch.restype = I
        _lib = L
    return _lib


def _i16(x, what):
    a = np.asarray(x, dtype=np.int64)
    if a.size and (a.min() < -32768 or a.max() > 32767):
        raise ValueError('%s does not fit the engine\'s int16 words' % what)
    return np.ascontiguousarray(a, dtype=np.int16)


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def solve_batch(G, h, P, R, T, c, q, inst, key, contexts=4, nthreads=1, philox=1):
    """B sub-problems, one engine each.  G (B, D, D) and h (B, D) integers, T and c (S,) one entry per step
    (S <= 1024), q an integer, inst (B,) uint32, key the 64-bit Philox key.  Returns spins (B, R, P D) int8
    copy-major, best energy change (B, R) int64, cycles (B,) from the first coupling row to idle and
    stats (B, 4) = [decision ops (steps), flips, field-init ops, R-port busy cycles] summed over the R anneals.
    philox = 0 runs the engine with its own numbers (hash-seeded xorshift32 per lane, 16-bit draws), the mode of
    the reference's production scripts."""
    G = _i16(G, 'G')
    h = _i16(h, 'h')
    B, D, _ = G.shape
    S = len(T)
    if not (1 <= S <= 1024) or len(c) != S or P > 6 or P < 1:
        raise ValueError('engine: 1 <= S <= 1024 steps, len(c) == S and P <= 6')
    seedl = max(1, D // 32)
    if D % seedl:
        raise ValueError('engine: D must be a multiple of its seeder width max(1, D // 32)')
    T16, c16 = _i16(T, 'T'), _i16(c, 'c')
    it = np.ascontiguousarray(np.asarray(inst, dtype=np.int64) & 0xFFFFFFFF, dtype=np.uint32)
    spins = np.zeros((B, R, P * D), np.int8)
    de = np.zeros((B, R), np.int64)
    cyc = np.zeros(B, np.int64)
    st = np.zeros((B, 4), np.int64)
    lib().engine_solve_batch(D, contexts, seedl, 1 if philox else 0, B, _ptr(G), _ptr(h), P, R, S, _ptr(T16), _ptr(c16), int(q),
                             _ptr(it), ctypes.c_uint64(key & 0xFFFFFFFFFFFFFFFF), _ptr(spins), _ptr(de), _ptr(cyc),
                             _ptr(st), int(nthreads))
    return spins, de, cyc, st
