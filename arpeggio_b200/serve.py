"""Serving: continuous batching of per-frame detection requests of mixed sizes.

A frame is one channel use of some size class (users, antennas, constellation).  Each class has an arrival
stream in pinned host memory: H (n, 2 nr, 2 nt), y (n, 2 nr), N0 (n), arrival times (n, seconds, ascending)
and request ids.  The server keeps, per class, `inflight` lanes -- a preallocated detector of `slots` uses
(channel state stays on the device), its own CUDA stream and staging buffers -- and runs this loop:

  * admission: a free lane takes every request of its class that has arrived and is not yet taken, up to its
    slot count (slots are fixed by the HBM budget at construction; a class is accepted only if its kernels'
    shared memory fits), copies their H, y and noise in, detects, copies bits and distances out and records
    an event -- all on the lane's stream, so batches of one class and of different classes overlap on the GPU;
    a batch of at most GRAPH_MAX uses is staged into the lane's pinned buffers and replays a graph captured at
    construction for the next power-of-two size (one launch; the padding uses are detected and discarded);
  * completion: a lane whose event has completed hands its results to the requests' rows of the class's
    output arrays and becomes free; each request's latency is completion time minus arrival time.

Server.serve(native=True) runs this loop in the library (arp_serve_run): the same admission and completion rules,
with each lane holding a second set of graphs -- the chain alone on the lane's device buffers, one per power-of-two
batch up to its slots -- so the loop copies a batch's inputs straight from the class arrays to the device and its
bits and distances straight back into the class's output rows, with no interpreter and no host-side data copies
between a request's arrival and its completion.  The Python loop (serve() or step()) stays the default: under
overload its slower admission batches more and sustains more frames/s.

A request's result does not depend on what it is batched with: every problem anneals with the server's Philox
key and the request id as its instance number (the kernels' per-problem counters), and every stage works per
problem.  Requests that arrive while others are on the GPU are taken by the next free lane."""
import time

import numpy as np
import torch

from . import _lib
from .detector import PAM, el2
from .warm import NF, NO, WarmDetector


GRAPH_MAX = 64  # batches of up to this many uses replay a captured graph (one launch instead of ~15)


class _Lane:
    def __init__(self, cls, slots, anneals, sweeps, mlp, device, key):
        nt, nr, M = cls
        self.det = WarmDetector(slots, nt, nr, M, anneals=anneals, sweeps=sweeps, mlp=mlp, device=device)
        self.stream = torch.cuda.Stream(device=device)
        self.Hd = torch.empty(slots, 2 * nr, 2 * nt, dtype=torch.float32, device=device)
        self.yd = torch.empty(slots, 2 * nr, dtype=torch.float32, device=device)
        self.instd = torch.empty(slots, dtype=torch.int32, device=device)
        self.done = torch.cuda.Event()
        self.busy = None  # (first, last, graph bucket or 0) rows of the class stream in flight
        self.key = key
        # small batches: fixed pinned staging and one captured graph per power-of-two size
        g = min(GRAPH_MAX, slots)
        self.Hh = torch.empty(g, 2 * nr, 2 * nt, dtype=torch.float32).pin_memory()
        self.yh = torch.empty(g, 2 * nr, dtype=torch.float32).pin_memory()
        self.insth = torch.empty(g, dtype=torch.int32).pin_memory()
        self.s2h = torch.zeros(g, dtype=torch.float32).pin_memory()
        self.snrh = torch.zeros(g, dtype=torch.float32).pin_memory()
        self.bitsh = torch.empty(g, self.det.bits.shape[1], dtype=torch.int8).pin_memory()
        self.disth = torch.empty(g, dtype=torch.float32).pin_memory()
        # numpy views of the pinned staging: the loop stages requests with plain host copies (no tensor dispatch)
        self.np = {k: getattr(self, k).numpy() for k in ('Hh', 'yh', 'insth', 's2h', 'snrh', 'bitsh', 'disth')}
        self.graphs = {}
        kb = 1
        while kb <= g:
            self.graphs[kb] = self._capture(kb)
            kb *= 2
        # the native loop's graphs: the chain alone on the lane's device buffers, for the batch sizes of
        # native_sizes (inputs copied in and results out by the loop itself); padding slots hold zeros (noise
        # variance 1) or an earlier batch's inputs
        self.Hd.zero_()
        self.yd.zero_()
        self.instd.zero_()
        self.det.sigma2.fill_(1.0)
        self.det.snr_db.zero_()
        self.dgraphs = [(kb, self._capture_device(kb)) for kb in native_sizes(slots)]

    def _body(self, kb):
        det = self.det
        self.Hd[:kb].copy_(self.Hh[:kb], non_blocking=True)
        self.yd[:kb].copy_(self.yh[:kb], non_blocking=True)
        self.instd[:kb].copy_(self.insth[:kb], non_blocking=True)
        det.sigma2[:kb].copy_(self.s2h[:kb], non_blocking=True)
        det.snr_db[:kb].copy_(self.snrh[:kb], non_blocking=True)
        bits, _, dist = det.run(self.Hd[:kb], self.yd[:kb], self.key, n=kb, inst=self.instd[:kb])
        self.bitsh[:kb].copy_(bits, non_blocking=True)
        self.disth[:kb].copy_(dist, non_blocking=True)

    def _capture_device(self, kb):
        det = self.det
        run = lambda: det.run(self.Hd[:kb], self.yd[:kb], self.key, n=kb, inst=self.instd[:kb])
        with torch.cuda.stream(self.stream):
            run()  # settles launch widths and kernel attributes outside the capture
        self.stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=self.stream):
            run()
        return g

    def _capture(self, kb):
        self.Hh[:kb].zero_()
        self.yh[:kb].zero_()
        self.insth[:kb].zero_()
        self.s2h[:kb].fill_(1.0)
        with torch.cuda.stream(self.stream):
            self._body(kb)  # settles launch widths and kernel attributes outside the capture
        self.stream.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=self.stream):
            self._body(kb)
        return g


def native_sizes(slots):
    """Batch sizes of a lane's native-loop graphs: powers of two to 64, then steps of about a quarter (multiples
    of 32) up to the lane's slots, so a batch pads at most ~25 % beyond 64 requests (at most 32 sizes)."""
    sizes = [kb for kb in (1, 2, 4, 8, 16, 32, 64) if kb <= slots]
    kb = 64
    while kb < slots and len(sizes) < 32:  # beyond 32 sizes the lane takes at most the last one per batch
        kb = min(slots, max(kb + 32, (int(kb * 1.25) + 31) // 32 * 32))
        sizes.append(kb)
    return sizes


def shared_bytes(cls, anneals):
    """The largest per-block shared memory of the class's kernels: the anneal's G (D rows padded to 32-lane
    slots, int32) and the readout's transposed H, residual and candidates."""
    nt, nr, M = cls
    D, NR2 = 2 * nt, 2 * nr
    anneal = D * 32 * (-(-D // 32)) * 4
    readout = 4 * (D * (NR2 + 1) + NR2 + 8) + 32 + (anneals + 1) * D + 16
    return max(anneal, readout)


def lane_bytes(cls, slots, anneals, warm):
    """Device bytes of one lane: detector workspace and buffers, MLP activations, staging."""
    nt, nr, M = cls
    D, NR2, P = 2 * nt, 2 * nr, 2
    offs = (__import__('ctypes').c_size_t * 7)()
    ws = _lib.lib().arp_detect_dd_workspace(slots, D, P, anneals, 0, offs)
    nb = D * PAM[M]['bits']
    per = D * (4 + NF * 2 + 2) + 8 + 4 + 4 + D + nb + 4 + 4 + 4 * (NR2 * D + NR2) + 12
    if warm:
        per += D * NO * 4  # logits; the fused network keeps its hidden activations on chip
    return ws + slots * per


class Server:
    """Continuous-batching detection server over size classes (nt, nr, M)."""

    def __init__(self, classes, mlp=None, anneals=32, sweeps=None, slots=4096, inflight=2, hbm_budget=8 << 30,
                 seed=0x5EED, device='cuda'):
        self.device = torch.device(device)
        self.key = seed & 0xFFFFFFFFFFFFFFFF
        self.classes = [tuple(c) for c in classes]
        self.lanes, self.slots = {}, {}
        share = hbm_budget // max(1, len(self.classes))
        for cls in self.classes:
            nt, nr, M = cls
            if 2 * nt > 128 or M not in PAM:
                raise ValueError('size class %s: the anneal keeps at most 128 coordinates in shared memory' % (cls,))
            if shared_bytes(cls, anneals) > 227 * 1024:
                raise ValueError('size class %s: shared memory beyond 227 KB per block' % (cls,))
            cap = slots
            while cap > 1 and inflight * lane_bytes(cls, cap, anneals, mlp is not None) > share:
                cap //= 2
            self.slots[cls] = cap
            self.lanes[cls] = [_Lane(cls, cap, anneals, sweeps, mlp, self.device, self.key) for _ in range(inflight)]
        self.streams = {}

    def open(self, cls, H, y, N0, t_arrival, rid):
        """Registers the arrival stream of a class (pinned host tensors; t_arrival ascending, seconds) and output
        buffers for it (bits (n, D log2(M)/2) int8, dist (n), done (n) completion times)."""
        cls = tuple(cls)
        nt, nr, M = cls
        n = H.shape[0]
        N0 = torch.as_tensor(N0, dtype=torch.float64).reshape(-1).expand(n)
        st = {'H': H, 'y': y, 't': np.asarray(t_arrival, dtype=np.float64), 'rid': rid,
              's2': ((N0 / 2) / el2(M)).float().contiguous().pin_memory(),
              'snr': (10 * torch.log10(nt / N0)).float().contiguous().pin_memory(),
              'rid_t': torch.as_tensor(np.asarray(rid, dtype=np.int64) & 0xFFFFFFFF).to(torch.int32).pin_memory(),
              'bits': torch.empty(n, 2 * nt * PAM[M]['bits'], dtype=torch.int8).pin_memory(),
              'dist': torch.empty(n, dtype=torch.float32).pin_memory(),
              'done': np.full(n, np.nan), 'next': 0, 'batches': 0}
        st['np'] = {k: st[k].numpy() for k in ('H', 'y', 's2', 'snr', 'rid_t', 'bits', 'dist')}
        self.streams[cls] = st
        return st

    def _launch(self, cls, lane, a, b):
        st, det, k = self.streams[cls], lane.det, b - a
        if k <= len(lane.Hh):
            # small batch: stage into the lane's pinned buffers, replay the graph of the next power of two
            kb = 1 << (k - 1).bit_length()
            src, dst = st['np'], lane.np
            dst['Hh'][:k] = src['H'][a:b]
            dst['yh'][:k] = src['y'][a:b]
            dst['insth'][:k] = src['rid_t'][a:b]
            dst['s2h'][:k] = src['s2'][a:b]
            dst['snrh'][:k] = src['snr'][a:b]
            with torch.cuda.stream(lane.stream):
                lane.graphs[kb].replay()
            lane.done.record(lane.stream)
            lane.busy = (a, b, kb)
            st['batches'] += 1
            return
        with torch.cuda.stream(lane.stream):
            lane.Hd[:k].copy_(st['H'][a:b], non_blocking=True)
            lane.yd[:k].copy_(st['y'][a:b], non_blocking=True)
            lane.instd[:k].copy_(st['rid_t'][a:b], non_blocking=True)
            det.sigma2[:k].copy_(st['s2'][a:b], non_blocking=True)
            det.snr_db[:k].copy_(st['snr'][a:b], non_blocking=True)
        bits, _, dist = det.run(lane.Hd[:k], lane.yd[:k], self.key, n=k, stream=lane.stream, inst=lane.instd[:k])
        with torch.cuda.stream(lane.stream):
            st['bits'][a:b].copy_(bits, non_blocking=True)
            st['dist'][a:b].copy_(dist, non_blocking=True)
        lane.done.record(lane.stream)
        lane.busy = (a, b, 0)
        st['batches'] += 1

    def _serve_native(self, timeout):
        cls_list, streams, lanes = _native_streams(self)
        batches = np.zeros(max(1, len(cls_list)), dtype=np.int64)
        rc = _lib.lib().arp_serve_run(streams, len(cls_list), lanes, len(lanes), float(timeout), batches.ctypes.data)
        if rc == 5:  # ARP_ERR_TIMEOUT
            raise TimeoutError('serving loop did not drain within %.0f s' % timeout)
        _lib.check(rc, 'serve')
        for i, cls in enumerate(cls_list):
            st = self.streams[cls]
            st['batches'] += int(batches[i])
            st['next'] = len(st['t'])

    def step(self, now):
        """One pass of the loop at time `now` (seconds on the arrival clock): completions, then admissions.
        Returns the number of requests still pending or in flight."""
        left = 0
        for cls, lanes in self.lanes.items():
            st = self.streams.get(cls)
            if st is None:
                continue
            for lane in lanes:
                if lane.busy is not None and lane.done.query():
                    a, b, kb = lane.busy
                    if kb:  # results of a graph batch arrive in the lane's pinned staging
                        st['np']['bits'][a:b] = lane.np['bitsh'][:b - a]
                        st['np']['dist'][a:b] = lane.np['disth'][:b - a]
                    st['done'][a:b] = now
                    lane.busy = None
            arrived = int(np.searchsorted(st['t'], now, side='right'))
            for lane in lanes:
                if lane.busy is None and st['next'] < arrived:
                    a = st['next']
                    b = min(arrived, a + self.slots[cls])
                    self._launch(cls, lane, a, b)
                    st['next'] = b
            left += (len(st['t']) - st['next']) + sum(1 for ln in lanes if ln.busy is not None)
        return left

    def serve(self, clock=None, timeout=120.0, native=False):
        """Runs the loop until every registered request is done.  clock(): seconds on the arrival clock
        (default: wall time since the call).  native: the same rules in the library (arp_serve_run: admission,
        copies, graph replay and completion polling without the interpreter, a graph per batch size of
        native_sizes); else this module's step() loop.  The native loop halves the median latency at moderate
        load (1e5 frames/s); under overload (1e6 frames/s) the Python loop, which admits later and so batches
        more, sustains more frames/s.  Returns per-class latency statistics."""
        if native:
            if clock is not None:
                raise ValueError('the native loop keeps its own clock (seconds since the call)')
            self._serve_native(timeout)
        else:
            t0 = time.perf_counter()
            clock = clock or (lambda: time.perf_counter() - t0)
            while True:
                now = clock()
                if self.step(now) == 0:
                    break
                if time.perf_counter() - t0 > timeout:
                    raise TimeoutError('serving loop did not drain within %.0f s' % timeout)
        for lanes in self.lanes.values():
            for lane in lanes:
                lane.stream.synchronize()
                lane.det.check()
        out = {}
        for cls, st in self.streams.items():
            lat = (st['done'] - st['t']) * 1e6
            out['%dx%d %d-QAM' % (cls[0], cls[1], cls[2])] = {
                'requests': int(len(lat)), 'batches': st['batches'], 'slots': self.slots[cls],
                'p50_us': float(np.percentile(lat, 50)), 'p99_us': float(np.percentile(lat, 99)),
                'max_us': float(lat.max())}
        return out


def _native_streams(server):
    """The arp_serve_stream and arp_serve_lane tables of a server's opened classes (stream index = class order)."""
    import ctypes
    cls_list = [c for c in server.lanes if c in server.streams]
    streams = (_lib.ServeStream * len(cls_list))()
    lanes = []
    for i, cls in enumerate(cls_list):
        st = server.streams[cls]
        n = len(st['t'])
        st['t_c'] = np.ascontiguousarray(st['t'], dtype=np.float64)
        for k in ('H', 'y', 's2', 'snr', 'rid_t', 'bits', 'dist'):
            if not st[k].is_contiguous():
                raise ValueError('request stream %s of class %s must be contiguous' % (k, cls))
        streams[i] = _lib.ServeStream(st['H'].data_ptr(), st['y'].data_ptr(), st['s2'].data_ptr(),
                                      st['snr'].data_ptr(), st['rid_t'].data_ptr(), st['t_c'].ctypes.data, n,
                                      int(st['H'][0].numel()) if n else 1, int(st['y'][0].numel()) if n else 1,
                                      int(st['bits'].shape[1]), st['bits'].data_ptr(), st['dist'].data_ptr(),
                                      st['done'].ctypes.data)
        for lane in server.lanes[cls]:
            det = lane.det
            n_g = len(lane.dgraphs)
            sizes = (ctypes.c_int * 32)(*([kb for kb, _ in lane.dgraphs] + [0] * (32 - n_g)))
            g = (ctypes.c_void_p * 32)(*([gr.raw_cuda_graph_exec() for _, gr in lane.dgraphs] + [None] * (32 - n_g)))
            lanes.append(_lib.ServeLane(i, lane.stream.cuda_stream, n_g, sizes, g, lane.Hd.data_ptr(),
                                        lane.yd.data_ptr(), det.sigma2.data_ptr(), det.snr_db.data_ptr(),
                                        lane.instd.data_ptr(), det.bits.data_ptr(), det.dist.data_ptr()))
    return cls_list, streams, (_lib.ServeLane * len(lanes))(*lanes)


def poisson_arrivals(n, rate, rng):
    """n arrival times (s) of a Poisson process of `rate` frames/s."""
    return np.cumsum(rng.exponential(1.0 / rate, size=n))
