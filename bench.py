#!/usr/bin/env python3
"""Benchmark of the delta-encoded Ising MIMO detector path on B200.

Workload (one step = one pass of the hot path over one batch): 32 users x 32 antennas, 16-QAM, 65536 seeded
i.i.d. Rayleigh channel uses with SNR 6-22 dB in 2 dB steps (round robin over the batch), one-stage dDI
(K = 1, 128 spins) around the hard MMSE guess, 32 anneals per use, Arpeggio first-accept in fixed point at
the reference's x32 budget (abl_far_32_0.1_0.1_0_rand_8: 32 sweeps x 2 passes, T 0.1, q 0, random start),
then the distance readout: map (Gram + MMSE + quantise) -> anneal -> readout, three launches.

metric: detections/s (whole job, all ranks), inputs resident in HBM (1.07 GB of channels per rank: larger
than L2, no flush needed).  e2e: the same through Detector with pinned host buffers (H, y copied in, bits and
distances copied out, inside the timed region).  Under torchrun each rank detects its own batch (weak
scaling, no collective on the data path).  --impl reference times the CPU restatement of the reference's
chain (oracle) on this box's host cores on a bounded sample per step."""
import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402

WORKLOAD = dict(nt=32, nr=32, M=16, batch=65536, snrs=list(range(6, 23, 2)), anneals=32, K=1, policy='arpeggio',
                precision='int', sweeps=32, T0=0.1, T1=0.1, q=0.0, start='rand')
METRIC = 'detections/s (16-QAM 32x32, 32 anneals, Arpeggio fixed point)'


def config(args):
    w = WORKLOAD
    return {'workload': 'x32 one-stage dDI detection: %d users x %d antennas 16-QAM, %d channels/rank, SNR %d-%d dB '
                        'step 2, %d anneals, Arpeggio first-accept fixed point S=%d T=%g q=%g start=%s, K=%d (128 spins)'
                        % (w['nt'], w['nr'], args.batch, w['snrs'][0], w['snrs'][-1], args.anneals, w['sweeps'],
                           w['T0'], w['q'], w['start'], w['K']),
            'batch_per_rank': args.batch, 'anneals': args.anneals, 'users': w['nt'], 'antennas': w['nr'],
            'modulation': '16-QAM', 'policy': w['policy'], 'fields': 'int32 fixed point (Q=4096)',
            'l2': 'inputs larger than L2 (H is %.2f GB per rank), no flush' % (args.batch * 4 * 64 * 64 / 1e9),
            'parallelism': 'replicas x%d' % args.world}


# ---------------------------------------------------------------- clocks
class Clocks:
    Q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,'
         'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,'
         'clocks_event_reasons.sw_power_cap')

    def __init__(self, gpu):
        self.gpu, self.p, self.f = gpu, None, None

    def start(self):
        try:
            self.f = tempfile.NamedTemporaryFile('w+', suffix='.csv', delete=False)
            self.p = subprocess.Popen(['nvidia-smi', '-i', str(self.gpu), '--query-gpu=' + self.Q,
                                       '--format=csv,noheader,nounits', '-lms', '200'], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        rows = [r.split(', ') for r in open(self.f.name).read().strip().splitlines() if r.strip()]
        os.unlink(self.f.name)
        sm = [float(r[1]) for r in rows if len(r) >= 9 and r[1].replace('.', '').isdigit()]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and r[2].replace('.', '').isdigit()]
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        reasons = sorted({n for r in rows if len(r) >= 9 for n, v in zip(names, r[5:9]) if v.strip() == 'Active'})
        return {'sm_mhz': statistics.median(sm) if sm else None, 'sm_max_mhz': max(mx) if mx else None,
                'reasons': reasons, 'samples': len(sm)}


# ---------------------------------------------------------------- CPU chain (oracle restatement of the reference)
def cpu_chain(H, y, N0, R, seed, nthreads):
    """Float64 MMSE guess + dDI mapping + to_fixed/compress (numpy), the oracle's first-accept anneal on all
    threads, then select: the reference's chain restated on the CPU (test infrastructure, timed as baseline)."""
    from oracle import oracle as O
    from arpeggio_b200.detector import arpeggio_schedule
    w = WORKLOAD
    B = H.shape[0]
    lv = np.asarray([-3, -1, 1, 3], dtype=np.float64)
    el2 = float((lv ** 2).mean())
    Hd = H.astype(np.float64)
    Gm = np.einsum('bki,bkj->bij', Hd, Hd)
    A = Gm + ((N0 / 2) / el2)[:, None, None] * np.eye(Hd.shape[-1])
    z = np.linalg.solve(A, np.einsum('bki,bk->bi', Hd, y.astype(np.float64))[..., None])[..., 0]
    mu = np.diagonal(np.linalg.solve(A, Gm), axis1=-2, axis2=-1)
    xq = O.quantize_levels(z / mu, 16)
    Gf, hf, _ = O.ising_delta_compressed(H, y, xq)
    G, h = O.quantize_compressed(Gf, hf)
    T, q, _ = arpeggio_schedule(w['sweeps'], w['T0'], w['T1'], w['q'], w['K'])
    s, _, _ = O.anneal_dd(G, h, 2 * w['K'], R, T, q, np.arange(B), seed, w['start'], nthreads=nthreads)
    cand = O.spins_to_levels_delta(s, xq, w['K'], 16)
    sel, _ = O.select(H, y, cand, xq)
    return O.levels_to_bits(sel, 16)


def cpu_sample(args, nthreads, target_s):
    """Sized sample of the same workload for the CPU chain: returns (detections/s, sample description)."""
    import torch
    from arpeggio_b200 import channel
    w = WORKLOAD
    n = 32
    rate = None
    while True:
        snr = torch.tensor([w['snrs'][i % len(w['snrs'])] for i in range(n)], dtype=torch.float32)
        d = channel.draw_device(4321, snr, n, w['nt'], w['M'], dev='cpu')
        H, y, N0 = d['H'].numpy(), d['y'].numpy(), d['N0'].double().numpy()
        t0 = time.perf_counter()
        cpu_chain(H, y, N0, args.anneals, 7, nthreads)
        dt = time.perf_counter() - t0
        rate = n / dt
        if dt >= 0.5 * target_s or n >= args.batch:
            return rate, n, dt
        n = int(min(args.batch, max(2 * n, rate * target_s)))


def chord_engine_baseline(det, stream, target_s):
    """Chord's solver alone, both sides on the detector's own integer problems (G, h), schedule, instance numbers
    and key: this library's anneal over the whole batch on the GPU (CUDA events) against the reference's C++
    engine model (engine_model.cpp engine_solve_batch, Philox numbers, all host threads) on a bounded sample,
    whose outputs must equal the GPU's bit for bit."""
    import torch
    from arpeggio_b200 import arpeggiofx
    from oracle import ref_engine
    if not ref_engine.available():
        return {'unavailable': 'oracle/_ref/libape.so not built (make -C oracle ref needs the reference tree)'}
    B, R, P, D = det.B, det.R, det.P, det.D
    key = 12
    args = (det.G, det.h, P, R, det.T, det.q, det.inst, key, 'rand', 'chord', det.c)
    arpeggiofx.anneal(*args)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    s, de, st, status = arpeggiofx.anneal(*args)
    e1.record(stream)
    torch.cuda.synchronize()
    arpeggiofx.check_status(status)
    ms = e0.elapsed_time(e1)
    T = det.schedule['T']
    c = det.schedule['c'] if det.schedule['c'] is not None else [0] * len(T)
    nthreads = os.cpu_count() or 1
    n, rate, dt = 16, None, 0.0
    while True:
        G = det.G[:n].cpu().numpy()
        h = det.h[:n].cpu().numpy()
        inst = det.inst[:n].cpu().numpy().view(np.uint32)
        t0 = time.perf_counter()
        es, ede, cyc, est = ref_engine.solve_batch(G, h, P, R, T, c, det.q, inst, key, nthreads=nthreads)
        dt = time.perf_counter() - t0
        rate = n / dt
        if dt >= 0.5 * target_s or n >= B:
            break
        n = int(min(B, max(2 * n, rate * target_s)))
    equal = bool(np.array_equal(es, s[:n].cpu().numpy()) and np.array_equal(ede, de[:n].cpu().numpy()))
    return {'gpu_anneal_only': {'value': B / (ms / 1e3), 'unit': 'detections/s', 'ms': ms, 'uses': B},
            'cpu_baseline': {'value': rate, 'unit': 'detections/s', 'cores': nthreads, 'kind': 'reference',
                             'sample': '%d channel uses x %d anneals x %d steps through the reference\'s C++ Chord '
                                       'engine model (4 contexts, Philox numbers), %.1f s' % (n, R, len(T), dt)},
            'equal_to_gpu_on_sample': equal,
            'engine_cycles_per_use': float(cyc.mean()),
            'engine_cycles_model': 'Engine::cycle() clock edges from the first coupling row to idle, 4 contexts'}


# ---------------------------------------------------------------- cross-rank timing
def max_over_ranks(values, world, device='cpu'):
    """Per-rank device times (ms) -> their maximum over all ranks (every rank takes part, same order)."""
    import torch
    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t]


def job_throughput(uses_per_rank, world, ms_max):
    """Whole-job detections/s: every rank's uses over the slowest rank's time (weak scaling)."""
    return world * uses_per_rank / (ms_max / 1e3)


# ---------------------------------------------------------------- learned warm start vs plain
def frame_latency(det, f, stream, n):
    """Device time per replay of a captured one-frame graph (pinned H, y in; bits, distance out), with the
    detector's frame buffers (H and y side by side: one copy in, one copy out)."""
    import torch
    Hh1, yh1, Hd1, yd1, bo1, do1 = det.frame_buffers()
    Hh1.copy_(f['H'].cpu())
    yh1.copy_(f['y'].cpu())
    g = det.capture(Hh1, yh1, 5, bo1, do1, Hd1, yd1)
    for _ in range(50):
        g.replay()
    torch.cuda.synchronize()
    le = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
    for i in range(n):
        le[i][0].record(stream)
        g.replay()
        le[i][1].record(stream)
    torch.cuda.synchronize()
    det.check()
    us = sorted(1e3 * a_.elapsed_time(b_) for a_, b_ in le)
    return {'frames': n, 'p50_us': us[n // 2], 'p99_us': us[min(n - 1, int(0.99 * n))], 'max_us': us[-1]}


# Warm-start operating points: sweeps, temperature, sampling sharpness tau, confidence threshold per coordinate
# (problems whose kept start has sum_j log max_c p_jc > -CONF_PER_COORD * D run R_EASY anneals) -- chosen on
# separate seeded draws, not on the bench's instances.
CONF_PER_COORD = 5.0 / 64
WARM_POINTS = {32: {'warm': dict(sweeps=24, T=0.085, tau=0.8, counts=True, r_easy=4),
                    'warm_fast': dict(sweeps=20, T=0.085, tau=0.8, counts=True, r_easy=4),
                    # the configuration's own comparison: warm at half the plain cycle budget (16 of 32 sweeps)
                    'warm_half': dict(sweeps=16, T=0.085, tau=0.6, counts=True, r_easy=4),
                    'warm_argmax': dict(sweeps=24, T=0.085, tau=None, counts=False)},
               64: {'warm': dict(sweeps=24, T=0.07, tau=0.8, counts=True),
                    'warm_fast': dict(sweeps=32, T=0.07, tau=0.8, counts=True, per_coord=1.6 * CONF_PER_COORD,
                                      r_easy=16),
                    'warm_argmax': dict(sweeps=24, T=0.07, tau=None, counts=False)}}
R_EASY = 8


def warm_vs_plain(args, dev, stream, rank):
    """Trains the warm-start MLP on the GPU (plain MMSE-started Arpeggio at the full budget labels seeded 32-user
    16-QAM instances, SNR uniform 8-20 dB), then detects fresh 32-user and 64-user batches around the 1e-3 BER
    operating point with: the plain MMSE-started annealer at the reference's budget (its pick: T 0.1, 32 / 64
    sweeps); at 64 users also the plain annealer retuned (T 0.07, 48 sweeps), which matches that BER faster; the
    warm detector (sampled starts: anneal 0 from the network's argmax, the others drawn from softmax(0.8 z);
    per-problem anneal counts from the start's confidence; fewer sweeps) at two budgets; and the argmax-only warm
    start without counts at the warm budget.  Per variant: detections/s, stage times, BER per SNR point with the
    paired BER ratio to plain and its bootstrap interval (arpeggio_b200.stats.boot_ratio), mean final energy, and
    the one-frame latency at 32 users."""
    import torch
    from arpeggio_b200 import channel, stats, warm
    mlp = warm.WarmMLP(P=2, seed=0)
    t0 = time.time()
    hist = warm.train(mlp, nt=32, instances=args.warm_train, batch=16384, anneals=32, sweeps=32,
                      rows_per_step=65536, lr=2e-3, lr_end=1e-4, seed=11 + rank, device=dev)
    torch.cuda.synchronize()
    out = {'training': {'instances': args.warm_train, 'seconds': time.time() - t0, 'final_loss': hist[-1][1],
                        'final_accuracy': hist[-1][2], 'labels': 'plain MMSE-started Arpeggio, 32 anneals x 32 sweeps',
                        'optimizer': 'Adam, lr 2e-3 -> 1e-4, 65536 rows per step'},
           'plain': 'MMSE-started (bal) Arpeggio first accept, fixed point, the reference budget (T 0.1, full sweeps)',
           'plain_tuned': 'the same annealer at T 0.07 and 48 sweeps (64 users)',
           'warm': 'MLP warm start kept only where its energy is no worse than the MMSE guess, learned flip-test '
                   'order; anneal 0 from the argmax class, anneals 1..R-1 drawn per coordinate from softmax(0.8 z) '
                   '(Philox word 1 of the start block); problems whose kept start has confidence sum_j log max_c '
                   'p_jc above -%.4f D run 4 anneals at 32 users (one per warp of the anneal block), %d at 64 users '
                   '(warm_fast at 64 users: above -%.4f D, 16 anneals), the others all R'
                   % (CONF_PER_COORD, R_EASY, 1.6 * CONF_PER_COORD),
           'warm_half': 'the warm detector at half the plain budget (16 of 32 sweeps, softmax(0.6 z) starts), the '
                        'configuration\'s own comparison (32 users)',
           'warm_argmax': 'every anneal from the argmax class, all R anneals, at the warm budget',
           'points': {'x%d' % k: v for k, v in WARM_POINTS.items()}}
    for nt, B, snrs, full, R in ((32, args.batch, [18, 20, 22, 24], 32, 32),
                                 (64, args.batch, [16, 18, 20, 22], 64, 64)):
        snr = torch.tensor([float(snrs[i % len(snrs)]) for i in range(B)])
        d = channel.draw_device(9000 + nt + rank, snr, B, nt, 16, dev=dev)
        bt = channel.levels_to_bits(d['l'], 16)
        res = {}
        base_err = None
        variants = [('plain', dict(sweeps=full, T=None, tau=None, counts=False), None)]
        if nt == 64:
            variants.append(('plain_tuned', dict(sweeps=48, T=0.07, tau=None, counts=False), None))
        variants += [(k, v, mlp) for k, v in WARM_POINTS[nt].items()]
        for name, pt, net in variants:
            S = pt['sweeps']
            kw = dict(anneals=R, sweeps=S, mlp=net, device=dev, T0=pt['T'], T1=pt['T'], tau=pt['tau'])
            if pt['counts']:
                kw.update(conf_min=-pt.get('per_coord', CONF_PER_COORD) * 2 * nt, r_easy=pt.get('r_easy', R_EASY))
            det = warm.WarmDetector(B, nt, **kw)
            det.set_noise(N0=d['N0'])
            for i in range(2):
                det.run(d['H'], d['y'], seed=20 + i)
            torch.cuda.synchronize()
            ev = [[torch.cuda.Event(enable_timing=True) for _ in range(5)] for _ in range(3)]
            x0, x1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            x0.record(stream)
            for i in range(3):
                det.run(d['H'], d['y'], seed=30 + i, events=ev[i])
            x1.record(stream)
            torch.cuda.synchronize()
            det.check()
            ms = x0.elapsed_time(x1) / 3
            st = [sum(ev[i][s].elapsed_time(ev[i][s + 1]) for i in range(3)) / 3 for s in range(4)]
            err = (det.bits != bt).sum(-1).cpu().numpy()
            sn = snr.numpy()
            nb = bt.shape[1]
            r = {'sweeps': S, 'anneals': R, 'T': pt['T'] or 0.1, 'value': B / (ms / 1e3), 'unit': 'detections/s',
                 'ms_per_step': ms, 'stages_ms': {'map': st[0], 'warm_start': st[1], 'anneal': st[2], 'readout': st[3]},
                 'mean_final_energy': float(det.energies().min(1).values.clamp(max=0).double().mean()),
                 'ber': {'%d dB' % v: float(err[sn == v].sum()) / ((sn == v).sum() * nb) for v in snrs}}
            if net is not None:
                r['kept_fraction'] = float(det.kept.float().mean())
            if det.ra is not None:
                r['reduced_anneal_fraction'] = float((det.ra < R).float().mean())
            if base_err is None:
                base_err = err
            else:
                r['ber_ratio_vs_plain'] = {}
                for v in snrs:
                    m = sn == v
                    rr, lo, hi = stats.boot_ratio(err[m], base_err[m], B=1000)
                    r['ber_ratio_vs_plain']['%d dB' % v] = [rr, lo, hi]
                r['speedup_vs_plain'] = r['value'] / res['plain']['value']
            if nt == 32 and args.latency_frames > 0 and name != 'warm_argmax':
                f = channel.draw_device(77 + rank, 22.0, 1, nt, 16, dev=dev)
                d1 = warm.WarmDetector(1, nt, **kw)
                d1.set_noise(N0=f['N0'])
                r['frame_latency'] = frame_latency(d1, f, stream, min(args.latency_frames, 1000))
                del d1
            res[name] = r
            del det
        out['x%d' % nt] = res
    return out


def mixed_batch(args, dev, rank):
    """1 M detections (per rank) drawn uniformly over the 54 size classes users {8..64} x antennas {1, 1.5, 2} x
    {QPSK, 16-QAM, 64-QAM}, SNR uniform 5-25 dB, plain MMSE-started Arpeggio at the picks' budgets with 32 anneals,
    launch widths chosen by the autotuner, all classes in one captured CUDA graph on 8 forked streams."""
    import torch
    from arpeggio_b200 import mixed
    total = args.mixed
    counts = mixed.mixed_counts(total, seed=1 + rank)
    mb = mixed.MixedBatch(counts, anneals=32, streams=8, device=dev)
    mb.draw(7 + rank)
    tuner = mixed.Autotuner()
    t0 = time.time()
    mb.tune(tuner, precisions=('int', 'f32'))
    tune_s = time.time() - t0
    g = mb.capture(seed=3)
    ms = mixed.timed_replay(g, reps=3)
    mb.check()
    ber = mb.ber()
    bits = {c: d.bits.clone() for c, d in mb.dets.items()}
    del g
    # the same batch with every class's anneals in the persistent grids (blocks pulling problems from a device work
    # counter): same outputs, one anneal launch per slot count instead of one per class
    mb.persistent = True
    g = mb.capture(seed=3)
    ms_p = mixed.timed_replay(g, reps=3)
    mb.check()
    same = all(torch.equal(bits[c], d.bits) for c, d in mb.dets.items())
    g = None
    mb.persistent = False
    rebuilt = mb.apply_precision(tuner)  # sizes whose FP32-field anneal was faster, if any
    ms_t = None
    if rebuilt:
        g = mb.capture(seed=3)
        ms_t = mixed.timed_replay(g, reps=3)
        mb.check()
    out = {'value': total / (ms / 1e3), 'unit': 'detections/s', 'detections': total, 'classes': len(counts),
           'ms_per_replay': ms, 'ber': ber, 'tune_seconds': tune_s,
           'tuned_warps_per_block': {'D=%d' % k[0]: v['warps'] for k, v in tuner.table.items() if k[3] == 0},
           'tuned_precision': {'D=%d' % k[0]: {'pick': v['precision'],
                                               'anneal_ms': {p: round(t, 3) for p, t in v['precision_ms'].items()}}
                               for k, v in tuner.table.items() if k[3] == 0},
           'classes_rebuilt_for_precision': len(rebuilt),
           'value_with_tuned_precision': None if ms_t is None else total / (ms_t / 1e3),
           'persistent': {'value': total / (ms_p / 1e3), 'unit': 'detections/s', 'ms_per_replay': ms_p,
                          'bits_equal_to_per_class_graph': same,
                          'path': 'classes grouped by slot count, one stream per group: its maps, one persistent '
                                  'anneal grid for all its classes (arp_anneal_first_accept_mixed, blocks pulling '
                                  'problems from a device work counter), its readouts'},
           'config': 'users {8,16,24,32,48,64} x antennas {1,1.5,2}x users x {QPSK,16-QAM,64-QAM}, SNR U[5,25] dB, '
                     'MMSE-started Arpeggio first accept, 32 anneals, one CUDA graph (8 streams)'}
    tuner.reset()
    del g, mb
    torch.cuda.empty_cache()
    return out


def equal_budget(args, dev, rank, nt=64, snrs=tuple(range(10, 25, 2)), R=64):
    """Both flip policies at equal modelled cycle budgets (the reference's model F: steps or tests plus flips per
    anneal) at 64 users x 64 antennas 16-QAM: default Chord (128 steps per copy pair, T 0.3, q 0.4, random start)
    sets the budget; Arpeggio (MMSE start, T 0.1, q 0) takes the largest sweep count whose cost stays within it,
    chosen on the first 2048 uses; then both detect the whole batch (one-stage dDI, int32 fields)."""
    import torch
    from arpeggio_b200 import channel, detector, stats
    B = max(2048, args.x64_batch)
    snr = torch.tensor([float(snrs[i % len(snrs)]) for i in range(B)])
    d = channel.draw_device(6000 + rank, snr, B, nt, 16, dev=dev)
    bt = channel.levels_to_bits(d['l'], 16)

    def make(policy, n, sweeps=None):
        det = (detector.Detector(n, nt, nt, 16, 'chord', R, 1, precision='int', device=dev) if policy == 'chord' else
               detector.Detector(n, nt, nt, 16, 'arpeggio', R, 1, sweeps=sweeps, T0=0.1, T1=0.1, q=0.0, start='bal',
                                 precision='int', device=dev))
        det.set_noise(N0=d['N0'][:n])
        return det

    def cost(det):
        st = det.st.double()
        return float((st[..., 0] + st[..., 1]).mean())  # flips + (steps | tests) per anneal
    nt_ = 2048
    ch = make('chord', nt_)
    ch.run(d['H'][:nt_], d['y'][:nt_], seed=1)
    torch.cuda.synchronize()
    budget = cost(ch)
    grid, xs = (8, 12, 16, 24, 32, 48, 64, 96, 128), {}
    for S in grid:
        a = make('arpeggio', nt_, S)
        a.run(d['H'][:nt_], d['y'][:nt_], seed=1)
        torch.cuda.synchronize()
        xs[S] = cost(a) / budget
    ok = [S for S in grid if xs[S] <= 1.0]
    S_star = max(ok) if ok else grid[0]
    out = {'users': nt, 'uses': B, 'anneals': R, 'chord_cost_per_anneal': budget,
           'arpeggio_cost_ratio_by_sweeps': xs, 'arpeggio_sweeps': S_star}
    errs = {}
    for name, det in (('chord', make('chord', B)), ('arpeggio', make('arpeggio', B, S_star))):
        det.run(d['H'], d['y'], seed=2)
        torch.cuda.synchronize()
        x0, x1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        x0.record()
        for i in range(2):
            det.run(d['H'], d['y'], seed=3 + i)
        x1.record()
        torch.cuda.synchronize()
        det.check()
        e = (det.bits != bt).sum(-1).cpu().numpy()
        errs[name] = e
        sn = snr.numpy()
        out[name] = {'value': B / (x0.elapsed_time(x1) / 2 / 1e3), 'unit': 'detections/s',
                     'cost_per_anneal': cost(det),
                     'ber': {'%d dB' % v: float(e[sn == v].sum()) / ((sn == v).sum() * bt.shape[1]) for v in snrs}}
        del det
    sn = snr.numpy()
    out['ber_ratio_arpeggio_vs_chord'] = {'%d dB' % v: list(stats.boot_ratio(errs['arpeggio'][sn == v],
                                                                             errs['chord'][sn == v], B=1000))
                                          for v in snrs}
    return out


SERVE_CLASSES = [(8, 16, 4), (16, 16, 16), (24, 36, 64), (32, 32, 16), (48, 72, 4), (64, 64, 16)]


def serving(args, dev, rank, mlp=None):
    """Mixed-size frames (users x antennas x constellation as SERVE_CLASSES, SNR uniform 5-25 dB) arriving as
    Poisson streams at each offered rate, served by the continuous-batching loop (arpeggio_b200.serve.Server,
    2 lanes per class, 32 anneals at each class's Arpeggio budget, plain MMSE start unless an MLP is given):
    per-class p50/p99 latency (arrival to completion seen by the loop) and the achieved frames/s."""
    import torch
    from arpeggio_b200 import channel, serve
    out = {'classes': ['%d users x %d antennas %d-QAM' % c for c in SERVE_CLASSES],
           'start': 'warm (MLP)' if mlp is not None else 'plain MMSE start', 'rates': {}}
    for rate, seconds in ((1e5, 0.2), (1e6, 0.05)):
        rng = np.random.default_rng(17 + rank)
        n_all = int(rate * seconds)
        share = rng.multinomial(n_all, [1.0 / len(SERVE_CLASSES)] * len(SERVE_CLASSES))
        srv = serve.Server(SERVE_CLASSES, mlp=mlp, anneals=32, slots=4096, inflight=2, hbm_budget=24 << 30,
                           device=dev)
        t_all = serve.poisson_arrivals(n_all, rate, rng)
        cls_of = rng.integers(0, len(SERVE_CLASSES), n_all)
        for ci, cls in enumerate(SERVE_CLASSES):
            nt, nr, M = cls
            t = t_all[cls_of == ci]
            n = len(t)
            if n == 0:
                continue
            snr = torch.tensor(rng.uniform(5, 25, n), dtype=torch.float32)
            d = channel.draw_device(500 + ci, snr, n, nt, M, nr=nr, dev=dev)
            srv.open(cls, d['H'].cpu().pin_memory(), d['y'].cpu().pin_memory(), d['N0'].cpu(), t,
                     np.arange(n) + (ci << 24))
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        st = srv.serve(timeout=300)
        wall = time.perf_counter() - t0
        out['rates']['%.0e frames/s' % rate] = {'frames': n_all, 'seconds_offered': float(t_all[-1]),
                                                'seconds_to_drain': wall,
                                                'achieved_frames_per_s': n_all / wall, 'per_class': st}
        if rate == 1e5:  # the same arrivals through the library's loop (arp_serve_run)
            for cls, s_ in srv.streams.items():
                s_['done'][:] = np.nan
                s_['next'] = 0
                s_['batches'] = 0
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            st = srv.serve(timeout=300, native=True)
            wall = time.perf_counter() - t0
            out['rates']['%.0e frames/s' % rate]['native'] = {'seconds_to_drain': wall,
                                                              'achieved_frames_per_s': n_all / wall, 'per_class': st}
        del srv
        torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------- our arm
def run_ours(args):
    import torch
    import torch.distributed as dist
    from arpeggio_b200 import _lib, channel, detector
    rank, world, local = args.rank, args.world, args.local
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    w = WORKLOAD
    B = args.batch
    snr = torch.tensor([w['snrs'][i % len(w['snrs'])] for i in range(B)], dtype=torch.float32)
    data = channel.draw_device(1234 + rank, snr, B, w['nt'], w['M'], dev=dev)
    det = detector.Detector(B, w['nt'], w['nr'], w['M'], w['policy'], args.anneals, w['K'], sweeps=w['sweeps'],
                            T0=w['T0'], T1=w['T1'], q=w['q'], start=w['start'], precision=w['precision'], device=dev)
    det.set_noise(N0=data['N0'])
    H, y = data['H'], data['y']
    stream = torch.cuda.current_stream()

    def barrier():
        if world > 1:
            dist.barrier()

    for i in range(args.warmup):
        det.run(H, y, seed=1000 + i)
    torch.cuda.synchronize()
    det.check()
    barrier()
    K = args.steps
    evs = [[torch.cuda.Event(enable_timing=True) for _ in range(4)] for _ in range(K)]
    clocks = Clocks(local)
    clocks.start()
    barrier()
    torch.cuda.synchronize()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    t_start.record(stream)
    for i in range(K):
        det.run(H, y, seed=2000 + i, events=evs[i])
    t_end.record(stream)
    torch.cuda.synchronize()
    barrier()
    ck = clocks.stop()
    det.check()
    ms = t_start.elapsed_time(t_end) / K
    stage = [sum(evs[i][s].elapsed_time(evs[i][s + 1]) for i in range(K)) / K for s in range(3)]
    st = det.st.sum((0, 1)).tolist()  # flips, tests of the last step

    # ---- end to end through the public API with pinned host buffers
    Hh = H.cpu().pin_memory()
    yh = y.cpu().pin_memory()
    bits_h = torch.empty(det.bits.shape, dtype=torch.int8).pin_memory()
    dist_h = torch.empty(B, dtype=torch.float32).pin_memory()
    def e2e_step(seed):  # the detector's two staging buffers: the next step's copy overlaps this step's detection
        det.run_host(Hh, yh, seed, bits_h, dist_h, chunks=args.chunks, stream=stream)

    for i in range(max(1, args.warmup // 2)):
        e2e_step(3000 + i)
    torch.cuda.synchronize()
    barrier()
    Ke = K  # the same steps as the device-timed loop (the first step's copy in is the only one not overlapped)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for i in range(Ke):
        e2e_step(4000 + i)
    e1.record(stream)
    torch.cuda.synchronize()
    det.check()
    ms_e2e = e0.elapsed_time(e1) / Ke

    # ---- per-frame latency: one 32-user channel use, host buffers in and out, replayed CUDA graph
    lat = None
    if args.latency_frames > 0:
        f = channel.draw_device(77 + rank, float(w['snrs'][len(w['snrs']) // 2]), 1, w['nt'], w['M'], dev=dev)
        det1 = detector.Detector(1, w['nt'], w['nr'], w['M'], w['policy'], args.anneals, w['K'], sweeps=w['sweeps'],
                                 T0=w['T0'], T1=w['T1'], q=w['q'], start=w['start'], precision=w['precision'],
                                 device=dev)
        det1.set_noise(N0=f['N0'])
        Hh1, yh1, Hd1, yd1, bo1, do1 = det1.frame_buffers()
        Hh1.copy_(f['H'].cpu())
        yh1.copy_(f['y'].cpu())
        g = det1.capture(Hh1, yh1, 5, bo1, do1, Hd1, yd1)
        for _ in range(50):
            g.replay()
        torch.cuda.synchronize()
        n = args.latency_frames
        le = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n)]
        for i in range(n):
            le[i][0].record(stream)
            g.replay()
            le[i][1].record(stream)
        torch.cuda.synchronize()
        det1.check()
        us = sorted(1e3 * a_.elapsed_time(b_) for a_, b_ in le)
        lat = {'frame': 'one %d-user x %d-antenna 16-QAM channel use at %g dB, %d anneals, H/y from pinned host '
                        'memory, bits and distance into pinned host memory, one replayed CUDA graph (copy in, map, '
                        'anneal, readout writing straight into the mapped pinned outputs); device time per replay'
                        % (w['nt'], w['nr'], float(w['snrs'][len(w['snrs']) // 2]), args.anneals),
               'frames': n, 'p50_us': us[n // 2], 'p99_us': us[min(n - 1, int(0.99 * n))], 'max_us': us[-1]}

    # ---- BER of the last timed step per SNR point (the detection itself, and its MMSE guess for reference)
    ber = None
    if rank == 0:
        bt = channel.levels_to_bits(data['l'], w['M'])
        err = (det.bits != bt).float().mean(-1)
        errq = (channel.levels_to_bits(det.xq.float(), w['M']) != bt).float().mean(-1)
        ber = {'%d dB' % v: {'ber': float(err[snr == v].mean()), 'ber_mmse_guess': float(errq[snr == v].mean())}
               for v in w['snrs']}

    # ---- the other policy and the 64-user workload, same kernels (reported beside the headline)
    extra = {}
    if args.extras:
        for name, kw, Bx, ntx, snrs in (
                ('chord_x32', dict(policy='chord', sweeps=None, T0=0.3, T1=0.3, q=0.4, start='rand'), B, 32,
                 w['snrs']),
                ('arpeggio_x64', dict(policy='arpeggio', sweeps=64, T0=0.1, T1=0.1, q=0.0, start='bal'),
                 args.x64_batch, 64,
                 list(range(10, 25, 2)))):
            sx = torch.tensor([snrs[i % len(snrs)] for i in range(Bx)], dtype=torch.float32)
            dx = data if ntx == 32 else channel.draw_device(5678 + rank, sx, Bx, ntx, w['M'], dev=dev)
            anx = args.anneals if ntx == 32 else 64
            dtx = detector.Detector(Bx, ntx, ntx, w['M'], anneals=anx, K=1, precision='int', device=dev, **kw)
            dtx.set_noise(N0=dx['N0'])
            for i in range(2):
                dtx.run(dx['H'], dx['y'], seed=i)
            x0, x1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            x0.record(stream)
            for i in range(3):
                dtx.run(dx['H'], dx['y'], seed=10 + i)
            x1.record(stream)
            torch.cuda.synchronize()
            dtx.check()
            msx = x0.elapsed_time(x1) / 3
            btx = channel.levels_to_bits(dx['l'], w['M'])
            extra[name] = {'value': Bx / (msx / 1e3), 'unit': 'detections/s', 'ms_per_step': msx, 'uses': Bx,
                           'users': ntx, 'anneals': anx, 'policy': kw['policy'],
                           'budget': 'S=%s T0=%g T1=%g q=%g start=%s' % (kw['sweeps'] or '128 steps/copy pair',
                                                                           kw['T0'], kw['T1'], kw['q'], kw['start']),
                           'ber': float((dtx.bits != btx).float().mean()),
                           'flips_per_anneal': float(dtx.st[..., 0].float().mean()),
                           'tests_per_anneal': float(dtx.st[..., 1].float().mean())}
            if name == 'chord_x32' and world == 1 and not args.no_cpu:
                extra[name]['solver_vs_reference_engine'] = chord_engine_baseline(dtx, stream, 6.0)
            del dtx

    # ---- the reference's full chain: multi-stage MDI at its recorded x16 point (16 x 16, 20 dB, Ns 32,
    #      abl_far_64_0.1_0.1_0_rand_32; 267.9 detections/s recorded on a B200 with a 4-thread CPU wrapper)
    mdi_line = None
    if args.mdi_batch > 0:
        from arpeggio_b200 import mdi
        bm = channel.draw_device(4242 + rank, 20.0, args.mdi_batch, 16, 16, dev=dev)
        mdi.detect(bm['H'][:256], bm['y'][:256], 16 / 100.0, 16, 1, 'abl_far_64_0.1_0.1_0_rand_32')
        torch.cuda.synchronize()
        m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        m0.record(stream)
        lv_m, ann_m, cnt_m, _ = mdi.detect(bm['H'], bm['y'], 16 / 100.0, 16, 2, 'abl_far_64_0.1_0.1_0_rand_32')
        m1.record(stream)
        torch.cuda.synchronize()
        ms_m = m0.elapsed_time(m1)
        mdi_line = {'value': args.mdi_batch / (ms_m / 1e3), 'unit': 'detections/s', 'uses': args.mdi_batch,
                    'ms': ms_m, 'anneals_per_use': float(ann_m.mean()),
                    'config': 'MDI-MIMO (MMSE + SIC guesses, radius rule, K=1..3, up to 8 stages), 16 x 16 16-QAM, '
                              '20 dB, Ns 32, Arpeggio fixed point S=64 T=0.1 q=0 rand; device time incl. the host '
                              'walk over groups',
                    'reference_recorded': 267.9,
                    'reference_recorded_source': 'data/results/a513_fixed/x16/arpeggiofx_64_0.1_0.1_0_rand_32/'
                                                 'snr_20.00 (B200 anneal + 4 CPU threads)'}

    # ---- learned warm start against the plain MMSE-started annealer (the metric's "warm vs plain")
    warm_line = None
    if args.warm_train > 0:
        warm_line = warm_vs_plain(args, dev, stream, rank)
    serve_line = serving(args, dev, rank) if args.serve else None
    mixed_line = mixed_batch(args, dev, rank) if args.mixed > 0 else None
    budget_line = equal_budget(args, dev, rank) if args.extras else None

    # ---- integer-issue peak (calibration kernel) and the anneal kernel's algorithmic work
    L = _lib.lib()
    buf = torch.zeros(1, dtype=torch.int32, device=dev)
    nb, nth, it = 148 * 16, 256, 256
    L.arp_philox_rate(_lib.ptr(buf), nb, nth, 8, _lib.stream_ptr())
    c0, c1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c0.record(stream)
    _lib.check(L.arp_philox_rate(_lib.ptr(buf), nb, nth, it, _lib.stream_ptr()), 'philox_rate')
    c1.record(stream)
    torch.cuda.synchronize()
    peak_blocks = nb * nth * it / (c0.elapsed_time(c1) / 1e3)

    agg = max_over_ranks([ms, ms_e2e] + stage, world, dev)
    ms, ms_e2e = agg[0], agg[1]
    stage = agg[2:]
    if rank != 0:
        return None
    D, P, R = 2 * w['nt'], 2 * w['K'], args.anneals
    Lp = len(det.schedule['T'])
    nquad = -(-Lp // (4 * P))
    blocks = B * R * (P * D * nquad + (P * D if w['start'] == 'rand' else D))
    ops = 100.0 * blocks + 5.0 * B * R * D * Lp + 3.0 * D * st[0]
    t_anneal = stage[1] / 1e3
    peak_ops = 100.0 * peak_blocks
    traffic, inst_per_anneal = None, None
    tf = os.path.join(ROOT, 'profiles', 'traffic.json')
    if os.path.exists(tf):
        tj = json.load(open(tf)).get('anneal_first_accept_x32')
        if tj:
            traffic = tj['bytes_per_detection'] * B
            inst_per_anneal = tj.get('warp_instructions_per_anneal')
    alg_bytes = B * (D * D * 4 + D * 4) + B * R * (P * D + 24)
    peaks = {}
    pf = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    if os.path.exists(pf):
        peaks = json.load(open(pf))
    hbm_peak = peaks.get('hbm_gbs', 6650.0)
    smem_bytes = 4.0 * D * st[0] + 4.0 * st[1]
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    sm_mhz = (ck or {}).get('sm_mhz') or 1965.0
    smem_peak = 128.0 * sms * sm_mhz * 1e6 / 1e9
    line = {
        'metric': METRIC, 'value': job_throughput(B, world, ms), 'unit': 'detections/s', 'n_gpus': world,
        'steps': K, 'warmup': args.warmup, 'ms_per_step': ms, 'higher_is_better': True, 'scaling': 'weak',
        'vs_baseline': None, 'dtype': 'int32', 'data': 'synthetic (seeded Rayleigh draws on the device)',
        'config': config(args),
        'e2e': {'value': job_throughput(B, world, ms_e2e), 'unit': 'detections/s',
                'h2d_bytes_per_step': int(H.numel() * 4 + y.numel() * 4),
                'd2h_bytes_per_step': int(det.bits.numel() + B * 4), 'ms_per_step': ms_e2e, 'steps': Ke,
                'path': 'Detector.run_host: pinned host H, y in; bits, distances out; %d pipelined pieces; '
                        'alternate staging buffers, so a step\'s copy in overlaps the previous step\'s detection'
                        % args.chunks},
        'stages_ms': {'map': stage[0], 'anneal': stage[1], 'readout': stage[2]},
        'roofline': {'bound': 'int_issue', 'achieved': ops / t_anneal / 1e9, 'peak': peak_ops / 1e9,
                     'unit': 'Gop/s', 'frac': ops / t_anneal / peak_ops, 'traffic': traffic,
                     'kernel': 'k_anneal_int<2, 2, first accept, cached Philox>',
                     'ops_model': '100 per Philox4x32-10 block + 5 per lane decision + 3 per field update',
                     'peak_source': 'measured in this run: arp_philox_rate (chained Philox blocks, all SMs); '
                                    'MEASURED_PEAKS.json has no integer peak'},
        'roofline_hbm': {'bound': 'hbm', 'achieved': alg_bytes / t_anneal / 1e9, 'peak': hbm_peak, 'unit': 'GB/s',
                         'frac': alg_bytes / t_anneal / 1e9 / hbm_peak,
                         'peak_source': 'MEASURED_PEAKS.json hbm_gbs (of measured)' if peaks else 'fallback'},
        'roofline_issue': None if inst_per_anneal is None else {
            'bound': 'issue', 'achieved': inst_per_anneal * B * R / t_anneal / 1e9,
            'peak': 4.0 * sms * sm_mhz * 1e6 / 1e9, 'unit': 'G warp-instructions/s',
            'frac': inst_per_anneal * B * R / t_anneal / (4.0 * sms * sm_mhz * 1e6),
            'source': 'warp-instructions per anneal from the ncu capture of profiles/anneal_first_accept_x32.md '
                      '(profiles/traffic.json) x the anneals of this run over the measured anneal time; peak: one '
                      'issue per clock per SM sub-partition, 4 x %d SMs x the sampled median SM clock' % sms},
        'roofline_smem': {'bound': 'smem', 'achieved': smem_bytes / t_anneal / 1e9, 'peak': smem_peak, 'unit': 'GB/s',
                          'frac': smem_bytes / t_anneal / 1e9 / smem_peak,
                          'bytes_model': 'flips x D x 4 (a flipped coordinate\'s int32 row of G, read by the rank-1 '
                                         'field update) + tests x 4',
                          'peak_source': 'nominal: 128 B per clock per SM x %d SMs x the sampled median SM clock' % sms},
        'anneal_counters': {'flips': int(st[0]), 'tests': int(st[1]), 'anneals': B * R, 'philox_blocks': blocks},
        'latency': lat,
        'ber': ber,
        'mdi_x16': mdi_line,
        'warm_vs_plain': warm_line,
        'serving': serve_line,
        'mixed': mixed_line,
        'equal_budget_x64': budget_line,
        'extra': extra,
        'gpu_launches': 3 * K,
        'clocks': ck,
    }
    if world == 1 and not args.no_cpu:
        nthreads = os.cpu_count() or 1
        rate, n, dt = cpu_sample(args, nthreads, 12.0)
        line['cpu_baseline'] = {'value': rate, 'unit': 'detections/s', 'cores': nthreads, 'kind': 'port',
                                'sample': '%d channel uses of the same workload (same SNR mix, 32 anneals), full CPU '
                                          'chain (float64 MMSE + mapping, oracle first-accept anneal on %d threads, '
                                          'select), %.1f s' % (n, nthreads, dt)}
    line['summary'] = summary(line)
    return line


def _r(x, n=3):
    return None if x is None else float('%.*g' % (n, x))


def summary(line):
    """The metric's other halves in a few hundred bytes, as the line's last key: warm vs plain (speed-up and the
    paired BER-ratio intervals per SNR point), frame latency p50/p99, serving p99 per class at 1e5 frames/s."""
    out = {'det_per_s': _r(line['value'], 4), 'e2e_det_per_s': _r(line['e2e']['value'], 4),
           'roofline_frac': _r(line['roofline']['frac']),
           'issue_frac': _r((line.get('roofline_issue') or {}).get('frac')),
           'cpu_det_per_s': _r((line.get('cpu_baseline') or {}).get('value'), 4)}
    lat = line.get('latency') or {}
    out['frame_us_plain_p50_p99'] = [_r(lat.get('p50_us')), _r(lat.get('p99_us'))]
    wv = line.get('warm_vs_plain') or {}
    for wl in ('x32', 'x64'):
        blk = wv.get(wl)
        if not blk:
            continue
        o = {}
        for name, v in blk.items():
            if not isinstance(v, dict) or 'value' not in v:
                continue
            e = {'det_per_s': _r(v['value'], 4)}
            if 'speedup_vs_plain' in v:
                e['x_plain'] = _r(v['speedup_vs_plain'])
            if name in ('warm_argmax', 'warm_fast') and wl == 'x64':
                continue  # ablations and the second budget: in the full line only
            if 'ber_ratio_vs_plain' in v and name != 'warm_argmax':  # the ablation: speed-up only
                e['ber_ratio_ci'] = {k.replace(' ', ''): [_r(c) for c in ci] for k, ci in v['ber_ratio_vs_plain'].items()}
            if 'frame_latency' in v and name in ('plain', 'warm'):
                e['frame_us_p50_p99'] = [_r(v['frame_latency']['p50_us']), _r(v['frame_latency']['p99_us'])]
            o[name] = e
        out['warm_vs_plain_' + wl] = o
    sv = line.get('serving') or {}
    r5 = (sv.get('rates') or {}).get('1e+05 frames/s')
    if r5:
        out['serving_1e5'] = {'frames_per_s': _r(r5['achieved_frames_per_s']),
                              'p99_ms': {k: _r(v['p99_us'] / 1e3) for k, v in r5['per_class'].items()}}
        if r5.get('native'):
            out['serving_1e5']['native_p50_p99_ms'] = {k: [_r(v['p50_us'] / 1e3), _r(v['p99_us'] / 1e3)]
                                                      for k, v in r5['native']['per_class'].items()}
    mx = line.get('mixed') or {}
    if mx.get('value'):
        out['mixed_det_per_s'] = _r(mx['value'])
        if mx.get('persistent'):
            out['mixed_persistent_det_per_s'] = _r(mx['persistent']['value'])
    return out


def run_reference(args):
    """CPU restatement of the reference's chain, rank 0 only, each step a bounded sample of the workload."""
    if args.rank != 0:
        return None
    nthreads = os.cpu_count() or 1
    rate, n, dt = cpu_sample(args, nthreads, 4.0)
    import torch
    from arpeggio_b200 import channel
    w = WORKLOAD
    snr = torch.tensor([w['snrs'][i % len(w['snrs'])] for i in range(n)], dtype=torch.float32)
    d = channel.draw_device(999, snr, n, w['nt'], w['M'], dev='cpu')
    H, y, N0 = d['H'].numpy(), d['y'].numpy(), d['N0'].double().numpy()
    for i in range(args.warmup):
        cpu_chain(H[:max(1, n // 8)], y[:max(1, n // 8)], N0[:max(1, n // 8)], args.anneals, i, nthreads)
    t0 = time.perf_counter()
    for i in range(args.steps):
        cpu_chain(H, y, N0, args.anneals, 100 + i, nthreads)
    dt = (time.perf_counter() - t0) / args.steps
    v = n / dt
    return {'impl': 'reference', 'metric': METRIC, 'value': v, 'unit': 'detections/s', 'n_gpus': args.world,
            'steps': args.steps, 'warmup': args.warmup, 'ms_per_step': dt * 1e3, 'higher_is_better': True,
            'scaling': 'weak', 'vs_baseline': None, 'dtype': 'int32', 'data': 'synthetic', 'config': config(args),
            'cpu_baseline': {'value': v, 'unit': 'detections/s', 'cores': nthreads, 'kind': 'port',
                             'sample': '%d channel uses per step of the same workload' % n},
            'e2e': {'value': v, 'unit': 'detections/s', 'h2d_bytes_per_step': 0, 'd2h_bytes_per_step': 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=10)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='ours', choices=['ours', 'reference'])
    ap.add_argument('--batch', type=int, default=WORKLOAD['batch'])
    ap.add_argument('--anneals', type=int, default=WORKLOAD['anneals'])
    ap.add_argument('--no-cpu', action='store_true', help='skip the CPU baseline sample')
    ap.add_argument('--chunks', type=int, default=4, help='pipelined pieces of the end-to-end step')
    ap.add_argument('--latency-frames', type=int, default=2000, help='single-frame replays for p50/p99 latency')
    ap.add_argument('--mdi-batch', type=int, default=16384, help='uses of the multi-stage (MDI) line; 0 skips it')
    ap.add_argument('--x64-batch', type=int, default=262144,
                    help='uses of the 64-user lines (the 64 x 64 configuration: 262144 channels)')
    ap.add_argument('--no-extras', dest='extras', action='store_false', help='skip the Chord and 64-user lines')
    ap.add_argument('--no-serve', dest='serve', action='store_false', help='skip the serving-loop block')
    ap.add_argument('--mixed', type=int, default=1_000_000, help='detections of the mixed-size graph block; 0 skips')
    ap.add_argument('--warm-train', type=int, default=2_000_000,
                    help='training instances of the warm-start MLP for the warm-vs-plain block; 0 skips it')
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    args.rank = int(os.environ.get('RANK', 0))
    args.world = int(os.environ.get('WORLD_SIZE', 1))
    args.local = int(os.environ.get('LOCAL_RANK', 0))
    if args.impl == 'reference':
        line = run_reference(args)
    else:
        if args.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            torch.cuda.set_device(args.local)
            dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=120))
        line = run_ours(args)
        if args.world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()
    if line is not None:
        print(json.dumps(line), flush=True)


if __name__ == '__main__':
    main()
