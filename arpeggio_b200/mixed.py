"""Mixed-size detection in one captured CUDA graph, with an autotuner for the anneal kernel's launch width.

A mixed batch holds channel uses of many size classes (users x antennas x constellation).  Each class has a
preallocated detector (plain or warm-started) and device buffers; `capture` records one CUDA graph in which every
class's pipeline (map -> [network -> warm start] -> anneal -> readout) runs on its own stream forked from the
capture stream, so one replay detects the whole batch with the classes overlapping on the GPU.

`Autotuner` times the anneal kernel of each class at every launch width (warps per block: anneals per CTA in
flight) on a sample of that class's uses and installs the fastest through arp_anneal_tune; the choice never
changes results (each anneal depends only on its problem and index)."""
import json

import numpy as np
import torch

from . import _lib, channel
from .detector import Detector
from .warm import WarmDetector

USERS = (8, 16, 24, 32, 48, 64)
ANTENNA_RATIOS = (1.0, 1.5, 2.0)
CONSTELLATIONS = (4, 16, 64)


def mixed_classes():
    """The mixed-size workload: users x antenna ratio x constellation (54 classes)."""
    return [(nt, int(round(nt * r)), M) for nt in USERS for r in ANTENNA_RATIOS for M in CONSTELLATIONS]


class Autotuner:
    """Per size class (coordinates D, copies P): the anneal launch width (warps per block = anneals per CTA in flight)
    with the shortest device time on a sample of the class's uses, installed through arp_anneal_tune, and, when asked,
    the field precision (int32 fixed point or FP32) whose anneal is faster.  The width never changes results; the
    precision does (the FP32 rule is a different, equally valid detector), so it is chosen only when the caller
    offers both."""

    WIDTHS = (1, 2, 4, 8)

    def __init__(self):
        self.table = {}

    def _time(self, det, H, y, seed, reps):
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(4)]
        det.run(H, y, seed, events=ev)
        ms = 0.0
        for _ in range(reps):
            det.run(H, y, seed, events=ev)
            torch.cuda.synchronize()
            ms += ev[1].elapsed_time(ev[2])
        return ms / reps

    def tune(self, det, H, y, seed=1, reps=3, precisions=('int',)):
        D, P = det.D, det.P
        key = (D, P, 0, 0)
        if key in self.table:
            return self.table[key]
        L = _lib.lib()
        entry = {'precision_ms': {}}
        for prec in precisions:
            pc = 0 if prec == 'int' else 1
            d = det if prec == det.precision else Detector(det.B, det.nt, det.nr, det.M, 'arpeggio', det.R, det.K,
                                                             start=det.start, precision=prec, device=det.device)
            if d is not det:
                d.sigma2.copy_(det.sigma2)
            best, best_ms, times = 0, float('inf'), {}
            for w in self.WIDTHS:
                _lib.check(L.arp_anneal_tune(D, P, 0, pc, w), 'anneal_tune')
                times[w] = self._time(d, H, y, seed, reps)
                if times[w] < best_ms:
                    best, best_ms = w, times[w]
            _lib.check(L.arp_anneal_tune(D, P, 0, pc, best), 'anneal_tune')
            self.table.setdefault((D, P, 0, pc), {})
            entry['precision_ms'][prec] = best_ms
            if prec == det.precision:
                entry.update(warps=best, anneal_ms=times)
            else:
                self.table[(D, P, 0, pc)] = {'warps': best, 'anneal_ms': times}
        entry['precision'] = min(entry['precision_ms'], key=entry['precision_ms'].get)
        self.table[key] = entry
        return entry

    def reset(self):
        L = _lib.lib()
        for (D, P, pol, prec) in self.table:
            L.arp_anneal_tune(D, P, pol, prec, 0)
        self.table = {}

    def dumps(self):
        return json.dumps({'%d,%d,%d,%d' % k: v for k, v in self.table.items()})


class MixedBatch:
    """Preallocated detectors for `counts` {(nt, nr, M): uses}; plain MMSE-started Arpeggio (warm-started with an
    MLP) at the Arpeggio picks' budgets, `anneals` anneals per use.  persistent=True (plain detectors only): the
    maps and readouts stay per class on forked streams, and every class's anneals run in the persistent grids of
    arp_anneal_first_accept_mixed (one launch per slot count, blocks pulling problems from a device work counter);
    the outputs equal the per-class path's."""

    def __init__(self, counts, anneals=32, mlp=None, streams=8, device='cuda', persistent=False):
        if persistent and mlp is not None:
            raise ValueError('the persistent anneal serves the plain MMSE-started detectors')
        self.persistent = persistent
        self.counters = torch.zeros(16, dtype=torch.int32, device=device)  # 4 per slot-count group
        self.device = torch.device(device)
        self.classes = [tuple(c) for c in counts]
        self.counts = {tuple(c): int(n) for c, n in counts.items()}
        self.dets, self.H, self.y, self.l = {}, {}, {}, {}
        for cls in self.classes:
            nt, nr, M = cls
            n = self.counts[cls]
            if mlp is not None:
                self.dets[cls] = WarmDetector(n, nt, nr, M, anneals=anneals, mlp=mlp, device=self.device)
            else:
                self.dets[cls] = Detector(n, nt, nr, M, 'arpeggio', anneals, 1, start='bal', device=self.device)
            self.H[cls] = torch.empty(n, 2 * nr, 2 * nt, dtype=torch.float32, device=self.device)
            self.y[cls] = torch.empty(n, 2 * nr, dtype=torch.float32, device=self.device)
        self.streams = [torch.cuda.Stream(device=self.device) for _ in range(streams)]
        self.graph = None

    def draw(self, seed, snr_lo=5.0, snr_hi=25.0):
        """Seeded Rayleigh uses for every class, SNR uniform in [snr_lo, snr_hi] dB; keeps the true levels."""
        g = torch.Generator().manual_seed(seed)
        for i, cls in enumerate(self.classes):
            nt, nr, M = cls
            n = self.counts[cls]
            snr = snr_lo + (snr_hi - snr_lo) * torch.rand(n, generator=g)
            d = channel.draw_device(seed * 1000 + i, snr, n, nt, M, nr=nr, dev=self.device)
            self.H[cls].copy_(d['H'])
            self.y[cls].copy_(d['y'])
            self.l[cls] = d['l']
            self.dets[cls].set_noise(N0=d['N0'])
        torch.cuda.synchronize()

    def run(self, seed):
        """Every class on a stream forked from the current stream, joined back at the end (graph-capturable)."""
        if self.persistent:
            return self._run_persistent(seed)
        cur = torch.cuda.current_stream()
        for i, cls in enumerate(self.classes):
            s = self.streams[i % len(self.streams)]
            s.wait_stream(cur)
            with torch.cuda.stream(s):
                self.dets[cls].run(self.H[cls], self.y[cls], seed, stream=s)
        for s in self.streams:
            cur.wait_stream(s)

    def _run_persistent(self, seed):
        """Classes grouped by slot count (ceil(D / 32)); each group on its own stream: its maps, one persistent anneal
        launch for all of its classes, its readouts, so one group's anneal overlaps another's maps, readouts and
        drain."""
        cur = torch.cuda.current_stream()
        groups = {}
        for cls in self.classes:
            groups.setdefault((2 * cls[0] + 31) // 32, []).append(cls)
        L = _lib.lib()
        used = []
        for gi, ns in enumerate(sorted(groups, reverse=True)):
            s = self.streams[gi % len(self.streams)]
            s.wait_stream(cur)
            used.append(s)
            members = groups[ns]
            with torch.cuda.stream(s):
                for cls in members:
                    self.dets[cls].stage_map(self.H[cls], self.y[cls], stream=s)
                table = (_lib.MixedClass * len(members))(*[self.dets[c].mixed_class() for c in members])
                st = self.dets[members[0]].status
                _lib.check(L.arp_anneal_first_accept_mixed(table, len(members), 2, seed & 0xFFFFFFFF,
                                                           (seed >> 32) & 0xFFFFFFFF, 0,
                                                           _lib.ptr(self.counters[4 * gi:4 * gi + 4]), _lib.ptr(st),
                                                           _lib.stream_ptr(s)), 'anneal_mixed')
                for cls in members:
                    self.dets[cls].stage_readout(self.H[cls], self.y[cls], stream=s)
        for s in used:  # only the streams this call forked (joining an unforked one breaks a capture)
            cur.wait_stream(s)

    def capture(self, seed):
        """One CUDA graph of run(seed); launch widths and kernel attributes are settled by a warm-up run first."""
        s = torch.cuda.Stream(device=self.device)
        s.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(s):
            self.run(seed)
        torch.cuda.current_stream().wait_stream(s)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.run(seed)
        self.graph = g
        return g

    def tune(self, tuner, precisions=('int',)):
        """Tunes the anneal width (and, with precisions=('int', 'f32'), the field precision) once per problem size
        (coordinates D), on the largest class of that size with its drawn uses (call draw() first)."""
        by_d = {}
        for cls in self.classes:
            D = 2 * cls[0]
            if D not in by_d or self.counts[cls] > self.counts[by_d[D]]:
                by_d[D] = cls
        for D, cls in sorted(by_d.items()):
            tuner.tune(self.dets[cls], self.H[cls], self.y[cls], precisions=precisions)
        return tuner.table

    def apply_precision(self, tuner):
        """Rebuilds, for the per-class graph path, the detectors of every size whose tuned precision differs from
        theirs (the persistent anneal serves integer fields only).  Returns the classes rebuilt."""
        if self.persistent:
            return []
        done = []
        for cls in self.classes:
            det = self.dets[cls]
            e = tuner.table.get((det.D, det.P, 0, 0))
            if e is None or e.get('precision', det.precision) == det.precision:
                continue
            nd = Detector(det.B, det.nt, det.nr, det.M, 'arpeggio', det.R, det.K, start=det.start,
                          precision=e['precision'], device=det.device)
            nd.sigma2.copy_(det.sigma2)
            self.dets[cls] = nd
            done.append(cls)
        return done

    def check(self):
        for det in self.dets.values():
            det.check()

    def ber(self):
        """Bit error rate per constellation over the last run."""
        err, tot = {}, {}
        for cls, det in self.dets.items():
            M = cls[2]
            bt = channel.levels_to_bits(self.l[cls], M)
            err[M] = err.get(M, 0) + int((det.bits != bt).sum())
            tot[M] = tot.get(M, 0) + bt.numel()
        return {'%d-QAM' % M: err[M] / tot[M] for M in err}


def mixed_counts(total, seed=0):
    """Uses per class of a `total`-use mixed batch drawn uniformly over mixed_classes()."""
    cls = mixed_classes()
    n = np.random.default_rng(seed).multinomial(total, [1.0 / len(cls)] * len(cls))
    return {c: int(k) for c, k in zip(cls, n) if k > 0}


def timed_replay(graph, reps=3):
    graph.replay()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        graph.replay()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


