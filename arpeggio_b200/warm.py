"""Learned warm start for Arpeggio's first-accept anneal (no counterpart in the reference).

A per-coordinate MLP reads, for each coordinate j of a mapped dDI problem, the matched-filter output of the
residual around the guess (h_j, as the best single-coordinate move h_j / 4G_jj in level steps), the diagonal
G_jj (relative to the problem's mean) and the coupling of j to the other coordinates, the SNR, the guess level
and the MMSE soft residual, and emits logits over the coordinate's spin sum m_j in {-P, ..., P} (step 2).  The
argmax becomes the anneal's start state, 1 - p(m_j = 0) orders the first-accept scan (likely moves are tested
first), and the start is kept only when its Ising energy is no worse than the MMSE guess's; otherwise that
problem anneals from the plain MMSE start in index order.

Everything runs on the device through the C ABI: features (arp_warm_features), the three layers and their
backward products on the tensor cores (arp_gemm_bf16), the loss (arp_warm_loss), bias gradients
(arp_colsum_bf16), Adam (arp_adam), the warm start (arp_warm_start) and the warm anneal
(arp_anneal_first_accept_warm).  Labels are the plain MMSE-started annealer's decisions."""
import math

import numpy as np
import torch

from . import _lib, channel
from .detector import Detector, M32

NF, NH, NO = 16, 256, 16
EPI_F32, EPI_ACC, EPI_RELU_BF16, EPI_BIAS_F32, EPI_MASK_BF16 = range(5)


def gemm(A, a_mn, lda, B, b_mn, ldb, M, N, K, epi, C, ldc, bias=None, aux=None, ld_aux=0, status=None, stream=None):
    """C = A B^T on the tensor cores (arp_gemm_bf16); majors and epilogues as declared in the C header."""
    _lib.check(_lib.lib().arp_gemm_bf16(_lib.ptr(A), int(a_mn), lda, _lib.ptr(B), int(b_mn), ldb, M, N, K, epi,
                                        _lib.ptr(bias), _lib.ptr(aux), ld_aux, _lib.ptr(C), ldc, _lib.ptr(status),
                                        _lib.stream_ptr(stream)), 'gemm_bf16')


class WarmMLP:
    """16 features -> 256 -> 256 -> 16 logits (the first P + 1 used), ReLU, BF16 weights and activations, FP32
    accumulate and FP32 master weights with Adam.  Weights live in one flat buffer in the order of LAYOUT; W3t is
    the last layer stored as (in, out)."""
    LAYOUT = (('W1', (NH, NF)), ('b1', (NH,)), ('W2', (NH, NH)), ('b2', (NH,)), ('W3t', (NH, NO)), ('b3', (NO,)))

    def __init__(self, P=2, rows=0, device='cuda', seed=0):
        self.P, self.C = P, P + 1
        self.device = torch.device(device)
        self.offs, o = {}, 0
        for name, shp in self.LAYOUT:
            self.offs[name] = (o, shp)
            o += int(np.prod(shp))
        self.n = o
        g = torch.Generator().manual_seed(seed)
        w = torch.zeros(o, dtype=torch.float32)
        for name, fan in (('W1', NF), ('W2', NH), ('W3t', NH)):
            oo, shp = self.offs[name]
            std = math.sqrt((2.0 if name != 'W3t' else 1.0) / fan)
            w[oo:oo + int(np.prod(shp))] = torch.randn(int(np.prod(shp)), generator=g) * std
        self.w = w.to(self.device)
        self.wb = self.w.to(torch.bfloat16)
        self.w2p = torch.empty(NH * NH, dtype=torch.bfloat16, device=self.device)  # W2 in the fused kernel's order
        self.pack()
        self.grad = torch.zeros_like(self.w)
        self.m = torch.zeros_like(self.w)
        self.v = torch.zeros_like(self.w)
        self.steps = 0
        self.status = torch.zeros(1, dtype=torch.int32, device=self.device)
        self.loss = torch.zeros(1, dtype=torch.float32, device=self.device)
        self.correct = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._rows = 0
        self._train = False
        if rows:
            self.reserve(rows)

    def view(self, t, name):
        o, shp = self.offs[name]
        return t[o:o + int(np.prod(shp))].view(*shp)

    def reserve(self, rows, train=False):
        """Activation buffers for up to `rows` rows (no allocation afterwards for smaller calls)."""
        rows = -(-rows // 128) * 128
        if rows <= self._rows and (self._train or not train):
            return
        rows = max(rows, self._rows)
        dev, b16 = self.device, torch.bfloat16
        self.H1 = torch.empty(rows, NH, dtype=b16, device=dev)
        self.H2 = torch.empty(rows, NH, dtype=b16, device=dev)
        self.Z = torch.empty(rows, NO, dtype=torch.float32, device=dev)
        if train or self._train:
            self.dZ3 = torch.empty(rows, NO, dtype=b16, device=dev)
            self.dZ2 = torch.empty(rows, NH, dtype=b16, device=dev)
            self.dZ1 = torch.empty(rows, NH, dtype=b16, device=dev)
            self._train = True
        self._rows = rows

    def forward(self, X, rows, stream=None):
        """logits (rows, 16) float32 of features X (rows, 16) bf16, layer by layer with the hidden activations
        kept for backward (the training path); stream-ordered and allocation-free after reserve."""
        self.reserve(rows)
        H1, H2, Z = self.H1, self.H2, self.Z
        wb, st = self.wb, self.status
        gemm(X, 0, NF, self.view(wb, 'W1'), 0, NF, rows, NH, NF, EPI_RELU_BF16, H1, NH,
             bias=self.view(self.w, 'b1'), status=st, stream=stream)
        gemm(H1, 0, NH, self.view(wb, 'W2'), 0, NH, rows, NH, NH, EPI_RELU_BF16, H2, NH,
             bias=self.view(self.w, 'b2'), status=st, stream=stream)
        gemm(H2, 0, NH, self.view(wb, 'W3t'), 1, NO, rows, NO, NH, EPI_BIAS_F32, Z, NO,
             bias=self.view(self.w, 'b3'), status=st, stream=stream)
        return Z[:rows]

    def pack(self, stream=None):
        """Refreshes the packed copy of W2 that the fused forward streams (after every weight change)."""
        _lib.check(_lib.lib().arp_mlp_pack_w2(_lib.ptr(self.view(self.wb, 'W2')), _lib.ptr(self.w2p),
                                              _lib.stream_ptr(stream)), 'mlp_pack_w2')

    def infer(self, X, rows, Z, stream=None):
        """logits Z (rows, 16) float32 of features X (rows, 16) bf16 in one fused persistent launch
        (arp_mlp_forward): the hidden activations stay on chip; same roundings and summation order as forward()."""
        wb, w = self.wb, self.w
        _lib.check(_lib.lib().arp_mlp_forward(_lib.ptr(X), rows, _lib.ptr(self.view(wb, 'W1')),
                                              _lib.ptr(self.view(w, 'b1')), _lib.ptr(self.w2p),
                                              _lib.ptr(self.view(w, 'b2')), _lib.ptr(self.view(wb, 'W3t')),
                                              _lib.ptr(self.view(w, 'b3')), _lib.ptr(Z), _lib.ptr(self.status),
                                              _lib.stream_ptr(stream)), 'mlp_forward')
        return Z[:rows]

    def backward(self, X, labels, rows, stream=None):
        """Summed softmax cross-entropy over the rows' labels (< 0: ignored) and its gradients into self.grad
        (zeroed first); the forward pass must have run on the same X.  rows: a multiple of 16."""
        if rows % 16:
            raise ValueError('rows must be a multiple of 16')
        L = _lib.lib()
        sp = _lib.stream_ptr(stream)
        st = self.status
        self.grad.zero_()
        _lib.check(L.arp_warm_loss(_lib.ptr(self.Z), NO, _lib.ptr(labels), rows, self.C, _lib.ptr(self.dZ3), NO,
                                   _lib.ptr(self.loss), _lib.ptr(self.correct), sp), 'warm_loss')
        g = self.grad
        gemm(self.H2, 1, NH, self.dZ3, 1, NO, NH, NO, rows, EPI_ACC, self.view(g, 'W3t'), NO, status=st,
             stream=stream)
        _lib.check(L.arp_colsum_bf16(_lib.ptr(self.dZ3), rows, NO, NO, _lib.ptr(self.view(g, 'b3')), sp), 'colsum')
        gemm(self.dZ3, 0, NO, self.view(self.wb, 'W3t'), 0, NO, rows, NH, NO, EPI_MASK_BF16, self.dZ2, NH,
             aux=self.H2, ld_aux=NH, status=st, stream=stream)
        gemm(self.dZ2, 1, NH, self.H1, 1, NH, NH, NH, rows, EPI_ACC, self.view(g, 'W2'), NH, status=st,
             stream=stream)
        _lib.check(L.arp_colsum_bf16(_lib.ptr(self.dZ2), rows, NH, NH, _lib.ptr(self.view(g, 'b2')), sp), 'colsum')
        gemm(self.dZ2, 0, NH, self.view(self.wb, 'W2'), 1, NH, rows, NH, NH, EPI_MASK_BF16, self.dZ1, NH,
             aux=self.H1, ld_aux=NH, status=st, stream=stream)
        gemm(self.dZ1, 1, NH, X, 1, NF, NH, NF, rows, EPI_ACC, self.view(g, 'W1'), NF, status=st, stream=stream)
        _lib.check(L.arp_colsum_bf16(_lib.ptr(self.dZ1), rows, NH, NH, _lib.ptr(self.view(g, 'b1')), sp), 'colsum')

    def adam(self, scale, lr=1e-3, beta1=0.9, beta2=0.999, eps=1e-8, stream=None):
        self.steps += 1
        _lib.check(_lib.lib().arp_adam(_lib.ptr(self.w), _lib.ptr(self.wb), _lib.ptr(self.grad), _lib.ptr(self.m),
                                       _lib.ptr(self.v), self.n, float(lr), float(beta1), float(beta2), float(eps),
                                       self.steps, float(scale), _lib.stream_ptr(stream)), 'adam')
        self.pack(stream)

    def train_step(self, X, labels, rows, lr=1e-3, stream=None):
        """Forward, backward and one Adam step on the mean loss over `rows` rows (a multiple of 16)."""
        self.reserve(rows, train=True)
        self.forward(X, rows, stream)
        self.backward(X, labels, rows, stream)
        self.adam(1.0 / rows, lr, stream=stream)

    def check(self):
        _lib.check(int(self.status.item()), 'warm MLP')

    def state_dict(self):
        return {'w': self.w.cpu().numpy(), 'P': self.P, 'steps': self.steps}

    def load_state_dict(self, d):
        self.w.copy_(torch.as_tensor(np.asarray(d['w'], dtype=np.float32)))
        self.wb.copy_(self.w.to(torch.bfloat16))
        self.pack()
        self.steps = int(d.get('steps', 0))

    def numpy_params(self):
        return {name: self.view(self.w, name).cpu().numpy() for name, _ in self.LAYOUT}


class WarmDetector(Detector):
    """One-stage dDI detector (16/64-QAM or QPSK, K = 1, integer fields, Arpeggio first accept) whose anneals start
    from the MLP's warm start in its flip-test order; problems whose warm start is worse than the MMSE guess
    anneal from the plain MMSE start ('bal') in index order.  With tau set, anneal 0 starts from the argmax and
    every other warm anneal draws its start from softmax(tau z) of the network's logits (a different start per
    anneal, from the anneal's own Philox counters).  With conf_min also set, problems whose kept start has
    confidence sum_j log max_c p_jc above conf_min run only r_easy anneals (default 8), the others all R, and the
    warm anneal's blocks are r_easy warps wide (the largest power of two up to 8), so an easy problem fills one.  With mlp=None it is the plain MMSE-started detector that also records the
    features' inputs (used to make training labels)."""

    def __init__(self, B, nt, nr=None, M=16, anneals=32, sweeps=None, mlp=None, T0=None, T1=None, q=None,
                 device='cuda', warm_anneals=None, tau=None, conf_min=None, r_easy=8):
        super().__init__(B, nt, nr, M, 'arpeggio', anneals, 1, sweeps=sweeps, T0=T0, T1=T1, q=q, start='bal',
                         precision='int', device=device)
        dev = self.device
        B, D = self.B, self.D
        self.mlp = mlp
        self.warm_anneals = anneals if warm_anneals is None else warm_anneals  # the rest start from the guess
        self.zs = torch.empty(B, D, dtype=torch.float32, device=dev)
        self.X = torch.empty(B * D, NF, dtype=torch.bfloat16, device=dev)
        self.m0 = torch.zeros(B, D, dtype=torch.int8, device=dev)
        self.perm = torch.empty(B, D, dtype=torch.uint8, device=dev)
        self.e0 = torch.zeros(B, dtype=torch.int64, device=dev)
        self.kept = torch.zeros(B, dtype=torch.int32, device=dev)
        self.snr_db = torch.zeros(B, dtype=torch.float32, device=dev)
        self.Z = torch.empty(B * D, NO, dtype=torch.float32, device=dev) if mlp is not None else None
        self.tau = tau
        self.cdf = torch.empty(B, D, 2, dtype=torch.int32, device=dev) if tau is not None else None
        if conf_min is not None and tau is None:
            raise ValueError('per-problem anneal counts need the sampled start (tau)')
        self.conf_min, self.r_easy = conf_min, min(r_easy, anneals)
        self.ra = torch.full((B,), anneals, dtype=torch.int32, device=dev) if conf_min is not None else None
        if self.ra is not None:
            # an easy problem's anneals fill its block: the warm anneal runs blocks of the largest power of two
            # <= r_easy warps (at most 8; arp_anneal_tune, per coordinate-slot count, results unchanged)
            w = 1
            while w * 2 <= min(self.r_easy, 8):
                w *= 2
            _lib.check(_lib.lib().arp_anneal_tune(self.D, 2, 2, 0, w), 'anneal_tune')

    def set_noise(self, snr_db=None, N0=None, n=None):
        super().set_noise(snr_db, N0, n)
        n = self.B if n is None else n
        if N0 is None:
            s = torch.as_tensor(snr_db, dtype=torch.float64).reshape(-1)
        else:
            s = 10 * torch.log10(self.nt / torch.as_tensor(N0, dtype=torch.float64).reshape(-1))
        self.snr_db[:n].copy_(s.float().expand(n) if s.numel() == 1 else s.float(), non_blocking=True)

    def run(self, H, y, seed, n=None, inst0=0, stream=None, events=None, off=0, warm=True, inst=None):
        """Stream-ordered detection of uses off .. off+n-1 (instance numbers inst0 + off + i, or the device int32
        tensor `inst` (n,)): map with the MMSE soft estimate, then (warm and an MLP present) features -> MLP ->
        warm start -> warm anneal, else the plain MMSE-started anneal, then the readout.  events: 4 CUDA events
        (before map, anneal, readout, after) or 5 (before map, warm start, anneal, readout, after).  Returns
        views (bits, levels, dist)."""
        n = self.B - off if n is None else n
        if off < 0 or n < 0 or off + n > self.B:
            raise ValueError('slots %d..%d outside the detector batch %d' % (off, off + n, self.B))
        ev = (lambda i: events[i].record(stream)) if events is not None else (lambda i: None)
        e5 = events is not None and len(events) == 5
        key = (inst0, 0, self.B)
        if inst is not None:
            with torch.cuda.stream(stream if stream is not None else torch.cuda.current_stream()):
                self.inst[off:off + n].copy_(inst[:n], non_blocking=True)
            self._inst_base = None
        elif self._inst_base != key:  # every slot's instance number at once: pieces find theirs in place
            iv = (np.arange(inst0, inst0 + self.B, dtype=np.int64) & M32).astype(np.uint32).view(np.int32)
            with torch.cuda.stream(stream if stream is not None else torch.cuda.current_stream()):
                self.inst.copy_(torch.from_numpy(iv))
            self._inst_base = key
        L = _lib.lib()
        sp = _lib.stream_ptr(stream)
        D, NR2, P, R = self.D, self.NR2, self.P, self.R
        sl = slice(off, off + n)
        G, h, xq, sc, zs = self.G[sl], self.h[sl], self.xq[sl], self.scale[sl], self.zs[sl]
        spins, de, st, inst = self.spins[sl], self.de[sl], self.st[sl], self.inst[sl]
        ev(0)
        _lib.check(L.arp_map_dd_soft(_lib.ptr(H), _lib.ptr(y), _lib.ptr(self.sigma2[sl]), n, NR2, D, self.M, 1,
                                     _lib.ptr(G), _lib.ptr(h), _lib.ptr(xq), _lib.ptr(sc), _lib.ptr(zs),
                                     _lib.ptr(self.status), sp), 'map_soft')
        k0, k1 = seed & M32, (seed >> 32) & M32
        Lt = int(self.T.shape[0])
        outs = (_lib.ptr(spins), _lib.ptr(de), _lib.ptr(st), _lib.ptr(self.status), sp)
        if e5:
            ev(1)
        if warm and self.mlp is not None:
            X = self.X[off * D:(off + n) * D]
            _lib.check(L.arp_warm_features(_lib.ptr(G), _lib.ptr(h), _lib.ptr(xq), _lib.ptr(zs),
                                           _lib.ptr(self.snr_db[sl]), n, D, self.M, P, 1, _lib.ptr(X), None, None, sp),
                       'warm_features')
            Z = self.mlp.infer(X, n * D, self.Z[off * D:(off + n) * D], stream)
            starts = (_lib.ptr(self.m0[sl]), _lib.ptr(self.perm[sl]), _lib.ptr(self.e0[sl]), _lib.ptr(self.kept[sl]))
            if self.tau is None:
                _lib.check(L.arp_warm_start(_lib.ptr(Z), NO, _lib.ptr(G), _lib.ptr(h), _lib.ptr(xq), n, D, P, self.M, 1,
                                            *starts, sp), 'warm_start')
            else:
                ra = _lib.ptr(self.ra[sl]) if self.ra is not None else None
                cm = float(self.conf_min) if self.conf_min is not None else 0.0
                _lib.check(L.arp_warm_start_sampled(_lib.ptr(Z), NO, _lib.ptr(G), _lib.ptr(h), _lib.ptr(xq), n, D, P,
                                                    self.M, 1, *starts, float(self.tau), _lib.ptr(self.cdf[sl]), cm,
                                                    int(self.r_easy), R, ra, sp), 'warm_start')
            ev(2 if e5 else 1)
            if self.tau is None:
                rc = L.arp_anneal_first_accept_warm_mix(_lib.ptr(G), _lib.ptr(h), _lib.ptr(self.T), Lt, int(self.q), P,
                                                        R, D, n, _lib.ptr(inst), k0, k1, _lib.ptr(self.m0[sl]),
                                                        _lib.ptr(self.perm[sl]), int(self.warm_anneals), *outs)
            else:
                rc = L.arp_anneal_first_accept_warm_sampled(_lib.ptr(G), _lib.ptr(h), _lib.ptr(self.T), Lt,
                                                            int(self.q), P, R, D, n, _lib.ptr(inst), k0, k1,
                                                            _lib.ptr(self.m0[sl]), _lib.ptr(self.cdf[sl]),
                                                            _lib.ptr(self.perm[sl]), int(self.warm_anneals),
                                                            _lib.ptr(self.ra[sl]) if self.ra is not None else None,
                                                            *outs)
        else:
            ev(2 if e5 else 1)
            rc = L.arp_anneal_first_accept(_lib.ptr(G), _lib.ptr(h), _lib.ptr(self.T), Lt, int(self.q), P, R, D, n,
                                           _lib.ptr(inst), k0, k1, 1, *outs)
        _lib.check(rc, 'anneal')
        ev(3 if e5 else 2)
        levels, bits, dist, pick = self.levels[sl], self.bits[sl], self.dist[sl], self.pick[sl]
        whole = None if (off == 0 and n == self.B) else sl
        _lib.check(L.arp_readout_dd(_lib.ptr(H), _lib.ptr(y), _lib.ptr(xq), _lib.ptr(spins), n, NR2, D, P, R, self.M,
                                    _lib.ptr(levels), self._out_ptr(0, whole), self._out_ptr(1, whole), _lib.ptr(pick),
                                    sp), 'readout')
        ev(4 if e5 else 3)
        return bits, levels, dist

    def energies(self):
        """Final Ising energies per anneal relative to the MMSE guess (best energy change of the anneal plus the
        warm start's energy), in the integer problem's units; int64 (B, R)."""
        return self.de + self.e0[:, None]

    def labels(self, labels, stream=None):
        """Training labels (B*D) int8 of the last run: the class (level - guess)/2 + P/2 of each coordinate of
        the selected candidate; also (re)writes the features X of the run."""
        _lib.check(_lib.lib().arp_warm_features(_lib.ptr(self.G), _lib.ptr(self.h), _lib.ptr(self.xq),
                                                _lib.ptr(self.zs), _lib.ptr(self.snr_db), self.B, self.D, self.M, self.P,
                                                1, _lib.ptr(self.X), _lib.ptr(self.levels), _lib.ptr(labels),
                                                _lib.stream_ptr(stream)), 'warm_features')
        return labels


def train(mlp, nt=32, M=16, instances=2_000_000, batch=16384, snr=(8.0, 20.0), anneals=32, sweeps=None,
          rows_per_step=32768, lr=1e-3, lr_end=1e-4, seed=7, device='cuda', log=None):
    """Trains the warm-start MLP on the GPU: each generation batch of `batch` seeded Rayleigh instances (SNR
    uniform in `snr`) is detected by the plain MMSE-started annealer at the full budget, its decisions become
    per-coordinate labels, and the batch's rows are consumed in steps of `rows_per_step`.  Learning rate decays
    geometrically from lr to lr_end.  Returns a list of (instances seen, mean loss, accuracy) per batch."""
    plain = WarmDetector(batch, nt, M=M, anneals=anneals, sweeps=sweeps, mlp=None, device=device)
    D = plain.D
    rows = batch * D
    labels = torch.empty(rows, dtype=torch.int8, device=plain.device)
    mlp.reserve(min(rows, rows_per_step), train=True)
    nb = max(1, instances // batch)
    total_steps = nb * (-(-rows // rows_per_step))
    hist = []
    g = torch.Generator().manual_seed(seed)
    step = 0
    for bi in range(nb):
        snr_b = snr[0] + (snr[1] - snr[0]) * torch.rand(batch, generator=g)
        d = channel.draw_device(seed * 1000003 + bi, snr_b, batch, nt, M, dev=plain.device)
        plain.set_noise(N0=d['N0'])
        plain.run(d['H'], d['y'], seed=(seed << 20) + bi, warm=False)
        plain.labels(labels)
        mlp.loss.zero_()
        mlp.correct.zero_()
        for r0 in range(0, rows, rows_per_step):
            nr = min(rows_per_step, rows - r0)
            frac = step / max(1, total_steps - 1)
            mlp.train_step(plain.X[r0:r0 + nr], labels[r0:r0 + nr], nr, lr * (lr_end / lr) ** frac)
            step += 1
        hist.append((int((bi + 1) * batch), float(mlp.loss.item()) / rows, float(mlp.correct.item()) / rows))
        if log:
            log('batch %d/%d loss %.4f acc %.4f' % (bi + 1, nb, hist[-1][1], hist[-1][2]))
    plain.check()
    mlp.check()
    return hist


def _profile_main(argv):
    """python -m arpeggio_b200.warm profile --batch B [--sweeps S --T T --tau TAU --conf C --snr DB]: trains a
    network briefly (--train instances, default 262144), then runs three warm detections of B seeded 32-user
    uses (32 anneals x S sweeps, default 16; optional temperature, sampled starts and per-problem anneal counts
    with confidence threshold C, one SNR) and prints their stage times."""
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument('mode', choices=['profile'])
    ap.add_argument('--batch', type=int, default=16384)
    ap.add_argument('--train', type=int, default=262144)
    ap.add_argument('--sweeps', type=int, default=16)
    ap.add_argument('--T', type=float, default=None)
    ap.add_argument('--tau', type=float, default=None)
    ap.add_argument('--conf', type=float, default=None)
    ap.add_argument('--snr', type=float, default=None, help='one SNR (dB) for every use; default 10/14/18/22')
    a = ap.parse_args(argv)
    mlp = WarmMLP(P=2, seed=0)
    train(mlp, nt=32, instances=a.train, batch=min(a.train, 16384), anneals=32, sweeps=32, seed=11)
    B = a.batch
    snr = (torch.full((B,), a.snr) if a.snr is not None else
           torch.tensor([float(v) for v in np.repeat([10, 14, 18, 22], -(-B // 4))[:B]]))
    d = channel.draw_device(5, snr, B, 32, 16)
    det = WarmDetector(B, 32, anneals=32, sweeps=a.sweeps, mlp=mlp, T0=a.T, T1=a.T, tau=a.tau, conf_min=a.conf)
    det.set_noise(N0=d['N0'])
    for i in range(2):
        det.run(d['H'], d['y'], seed=i)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
    det.run(d['H'], d['y'], seed=9, events=ev)
    torch.cuda.synchronize()
    det.check()
    print('stages ms (map, warm start, anneal, readout):', [round(ev[i].elapsed_time(ev[i + 1]), 3) for i in range(4)])


def _gemm_main(argv):
    """python -m arpeggio_b200.warm gemm --rows R --width W [--reps N]: times the network's three large training
    products at R rows and hidden width W -- forward (H W^T, bias + ReLU to bf16), input gradient (dY W, ReLU mask)
    and weight gradient (dY^T H, split-K accumulation) -- each replayed N times in a CUDA graph; prints the device
    time and TFLOP/s of each."""
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument('mode', choices=['gemm'])
    ap.add_argument('--rows', type=int, default=32768)
    ap.add_argument('--width', type=int, default=512)
    ap.add_argument('--reps', type=int, default=20)
    a = ap.parse_args(argv)
    g = torch.Generator().manual_seed(0)
    R, W = a.rows, a.width
    X = (torch.randn(R, W, generator=g) * 0.5).to(torch.bfloat16).cuda()
    Wt = (torch.randn(W, W, generator=g) * 0.05).to(torch.bfloat16).cuda()
    dY = (torch.randn(R, W, generator=g) * 0.5).to(torch.bfloat16).cuda()
    bias = torch.randn(W, generator=g).cuda()
    H = torch.empty(R, W, dtype=torch.bfloat16, device='cuda')
    Gw = torch.zeros(W, W, device='cuda')
    st = torch.zeros(1, dtype=torch.int32, device='cuda')
    cases = [('forward', lambda: gemm(X, 0, W, Wt, 0, W, R, W, W, EPI_RELU_BF16, H, W, bias=bias, status=st)),
             ('input gradient', lambda: gemm(dY, 0, W, Wt, 1, W, R, W, W, EPI_MASK_BF16, H, W, aux=X, ld_aux=W,
                                             status=st)),
             ('weight gradient', lambda: gemm(dY, 1, W, X, 1, W, W, W, R, EPI_ACC, Gw, W, status=st))]
    for name, f in cases:
        for _ in range(3):
            f()
        torch.cuda.synchronize()
        s = torch.cuda.Stream()
        gr = torch.cuda.CUDAGraph()
        with torch.cuda.graph(gr, stream=s):
            for _ in range(a.reps):
                f()
        gr.replay()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        gr.replay()
        e1.record()
        torch.cuda.synchronize()
        if int(st.item()) != 0:
            raise _lib.ArpError('gemm status %d' % int(st.item()))
        us = 1e3 * e0.elapsed_time(e1) / a.reps
        print('%-16s %d x %d x %d: %8.1f us  %6.1f TFLOP/s' % (name, R, W, W, us, 2.0 * R * W * W / us / 1e6))


if __name__ == '__main__':
    import sys
    if sys.argv[1:2] == ['gemm']:
        _gemm_main(sys.argv[1:])
    else:
        _profile_main(sys.argv[1:])
