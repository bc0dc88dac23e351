#!/usr/bin/env python3
"""Generates the golden fixtures in this folder by importing the reference (skethz/Arpeggio) itself.

Run in a container that has the reference tree (read-only; no bytecode is written there):
    python tests/golden/make_golden.py "$ARPEGGIO_REFERENCE"

Fixtures (all small, numpy .npz):
  golden_philox.npz   Random123 KATs (arpeggio/mimo/chordfx.py:53-56) and 256 further counter/key
                      words pushed through chordfx.philox (chordfx.py:39-49).
  golden_arpeggio.npz integer anneals on compressed dDI problems built by the reference's own chain
                      (arpx.draw -> mimo.mmse -> mimo.ising_delta_at -> chordfx.to_fixed ->
                      chord_ref.compress), answered by arpeggio_ref59.anneal
                      (rtl/cycle_checks/rtl_a59/src/arpeggio_ref59.py:41-85), modes 'arpeggio' and 'par'.
  golden_chord.npz    chordfx.chord_fx (chordfx.py:80-118) on the cases of arpeggio/mimo/test_kernel.py:213-221
                      (CPU generator, fewer instances), modes 'chains' and 'best'.
  golden_mapping.npz  the float chain: draws, MMSE guess, ising_delta_at scale, to_fixed/compress
                      integers, spins_to_levels_delta, dist, select and list_llr (mimo.py:434-462, clip 1e4,
                      as softlib.detect_llr) on fixed spin sets.
  golden_a513_b0.npz  batch 0 of the recorded B200 runs data/results/a513_fixed/{x16,x32}: per-use bit
                      errors, anneals per use, per-K [flips, tests, anneals] (`... "$ARPEGGIO_REFERENCE" a513`).
  golden_a513_points.npz  every recorded batch's per-use bit errors at the three recorded points
                      (x16 20 dB, x32 22 dB, x64 22 dB) for the BER-inside-CI gate (`... "$ARPEGGIO_REFERENCE" a513_points`).
  golden_stats.npz    stats_chord.boot_ber (sim/stats_chord.py:58-66), a56an.boot_ratio and a56an.mcnemar
                      (sim/a56an.py:74-108) on seeded per-use error vectors (`... "$ARPEGGIO_REFERENCE" stats`).
  golden_trajectory.npz  mimo.trajectory_llr (mimo.py:397-413) on seeded trajectory minima, 16-QAM and QPSK
                      (`... "$ARPEGGIO_REFERENCE" trajectory`).
  golden_cycles.json  the recorded single-lane engine latencies per K (data/results/a59/A59.json) and the x16 MDI
                      point's model-F cost with its counters (data/results/a513/analysis.json P1)
                      (`... "$ARPEGGIO_REFERENCE" cycles`).
"""
import math
import os
import random
import sys

sys.dont_write_bytecode = True
REF = os.path.abspath(sys.argv[1] if len(sys.argv) > 1 else os.environ['ARPEGGIO_REFERENCE'])
OUT = os.path.dirname(os.path.abspath(__file__))
for sub in ('arpeggio/mimo', 'arpeggio/sim', 'arpeggio/sim/x3model', 'arpeggio/sim/local_code_a513'):
    sys.path.insert(0, os.path.join(REF, sub))

import numpy as np  # noqa: E402
import torch  # noqa: E402

torch.set_num_threads(4)
import mimo  # noqa: E402
import chordfx  # noqa: E402
import chord_ref  # noqa: E402
import arpx  # noqa: E402

M64 = 0xFFFFFFFFFFFFFFFF


def load_ref59():
    """Exec-load arpeggio_ref59.py without its command-line tail, as gate_a513.load_ref does."""
    path = os.path.join(REF, 'arpeggio/rtl/cycle_checks/rtl_a59/src/arpeggio_ref59.py')
    src = open(path).read()
    cut = src.index("\nif sys.argv[1] == 'gen':")
    ns = {'__name__': 'arpeggio_ref59'}
    exec(compile(src[:cut], path, 'exec'), ns)
    return ns


def philox_fixture():
    kat_in = np.array([list(c) + list(k) for c, k, _ in chordfx.KAT], dtype=np.uint32)
    kat_out = np.array([list(w) for _, _, w in chordfx.KAT], dtype=np.uint32)
    rnd = np.random.default_rng(7).integers(0, 2 ** 32, size=(256, 6), dtype=np.uint64)
    t = [torch.tensor(rnd[:, i].astype(np.int64)) for i in range(4)]
    outs = []
    for i in range(256):
        o = chordfx.philox(*[x[i:i + 1] for x in t], int(rnd[i, 4]), int(rnd[i, 5]))
        outs.append([int(v) for v in o])
    np.savez_compressed(os.path.join(OUT, 'golden_philox.npz'), kat_in=kat_in, kat_out=kat_out,
                        rnd_in=rnd.astype(np.uint32), rnd_out=np.array(outs, dtype=np.uint32))
    print('philox: 3 KATs, 256 random words')


def dd_problem(nt, snr, K, B, seed, bi=0, M=16):
    """A batch of compressed integer dDI sub-problems from the reference's own chain, around the MMSE guess."""
    b = arpx.draw(seed, snr, bi, B, nt, M, dev='cpu')
    z, _, _ = mimo.mmse(b)
    lm = mimo.quantize_levels(z / mimo._mu(b, z), M)
    I = mimo.ising_delta_at(b, lm, K)
    F = chordfx.to_fixed(I, 8 * 2 * K, 0.3, 0.3, 0.4, 0.0)
    G, h = chord_ref.compress(F, K)
    return G.numpy().astype(np.int32), h.numpy().astype(np.int32)


def sched(S, T0, T1, q, K):
    Q = chordfx.QSCALE
    Tsw = [int(round(v * Q)) for v in mimo.geom(T0, T1, S, 'cpu').double().tolist()]
    return [t for t in Tsw for _ in range(2 * K)], int(round(q * Q))


def arpeggio_fixture():
    ns = load_ref59()
    rnd = random.Random(513)
    cases = [  # name, (nt, snr, K, B, seed), R, (S, T0, T1, q), start, key, inst base
        ('x16_K1_pick_rand', (16, 20.0, 1, 4, 9600), 3, (64, 0.1, 0.1, 0.0), 'rand', rnd.getrandbits(64), 0),
        ('x16_K1_hot_bal', (16, 12.0, 1, 3, 9601), 2, (8, 1.2, 0.1, 0.2), 'bal', 0x1234567890ABCDEF, 2 ** 32 - 2),
        ('x16_K2_pick_bal', (16, 20.0, 2, 3, 9602), 2, (16, 0.1, 0.1, 0.0), 'bal', rnd.getrandbits(64), 1000),
        ('x16_K3_hot_rand', (16, 16.0, 3, 2, 9603), 2, (8, 1.2, 0.1, 0.2), 'rand', rnd.getrandbits(64), 3000),
        ('x32_K1_pick_rand', (32, 22.0, 1, 3, 9604), 2, (32, 0.1, 0.1, 0.0), 'rand', rnd.getrandbits(64), 7),
        ('x32_K2_hot_bal', (32, 14.0, 2, 2, 9605), 2, (6, 0.8, 0.1, 0.1), 'bal', rnd.getrandbits(64), 50),
        ('x64_K1_pick_bal', (64, 22.0, 1, 2, 9606), 2, (16, 0.1, 0.1, 0.0), 'bal', rnd.getrandbits(64), 0),
        ('x10_K1_ragged_rand', (10, 10.0, 1, 3, 9607), 3, (20, 0.6, 0.05, 0.1), 'rand', rnd.getrandbits(64), 11),
        ('x50_K1_ragged_bal', (50, 18.0, 1, 2, 9608), 2, (8, 0.5, 0.1, 0.0), 'bal', rnd.getrandbits(64), 99),
        ('x40_K3_ragged_rand', (40, 20.0, 3, 1, 9609), 2, (3, 0.3, 0.1, 0.0), 'rand', rnd.getrandbits(64), 5),
    ]
    out = {}
    for name, (nt, snr, K, B, seed), R, (S, T0, T1, q), start, key, ib in cases:
        G, h = dd_problem(nt, snr, K, B, seed)
        P = 2 * K
        D = G.shape[1]
        T, qi = sched(S, T0, T1, q, K)
        inst = np.array([(ib + b) & 0xFFFFFFFF for b in range(B)], dtype=np.int64)
        ns['SEED'] = key
        for mode in ('arpeggio', 'par'):
            sp = np.zeros((B, R, P * D), dtype=np.int8)
            de = np.zeros((B, R), dtype=np.int64)
            st = np.zeros((B, R, 2), dtype=np.int64)
            for b in range(B):
                Gl, hl = [[int(v) for v in row] for row in G[b]], [int(v) for v in h[b]]
                for r in range(R):
                    a = ns['anneal'](Gl, hl, P, T, qi, r, int(inst[b]), start, mode)
                    for p in range(P):
                        bits = a['bs'][p]
                        for j in range(D):
                            sp[b, r, p * D + j] = 1 if bits[D - 1 - j] == '1' else -1
                    de[b, r] = a['best']
                    st[b, r, 0] = len(a['acc'])
                    st[b, r, 1] = sum(a['tests'])
            k = '%s/%s' % (name, mode)
            out[k + '/spins'], out[k + '/de'], out[k + '/st'] = sp, de, st
        out[name + '/G'], out[name + '/h'] = G, h
        out[name + '/T'] = np.array(T, dtype=np.int32)
        out[name + '/meta'] = np.array([P, R, qi, key & 0xFFFFFFFF, key >> 32, 0 if start == 'rand' else 1], dtype=np.int64)
        out[name + '/inst'] = inst
        print('arpeggio', name, 'D', D, 'P', P, 'passes', len(T), 'flips', int(out[name + '/arpeggio/st'][..., 0].sum()))
    out['names'] = np.array([c[0] for c in cases])
    np.savez_compressed(os.path.join(OUT, 'golden_arpeggio.npz'), **out)


def chord_fixture():
    cases = [  # name, (Nt, M, snr, B, kind, K), R, S, t0, t1, q, kappa, P, seed, inst0 (test_kernel.py:213-221)
        ('16x16_QPSK_RI', (16, 4, 10.0, 6, 'ri', 1), 16, 128, 0.7, 0.5, 0.6, 0.0, 1, 7, 0),
        ('16x16_QPSK_RI_kappa', (16, 4, 10.0, 6, 'ri', 1), 16, 128, 2.0, 0.05, 0.5, 0.3, 1, 8, 1000),
        ('16x16_16QAM_dDI_K1', (16, 16, 20.0, 6, 'ddi', 1), 16, 256, 0.3, 0.3, 0.4, 0.0, 2, 9, 0),
        ('32x32_16QAM_dDI_K1_kappa', (32, 16, 22.0, 3, 'ddi', 1), 8, 128, 0.3, 0.2, 0.4, 0.3, 2, 10, 77),
        ('16x16_16QAM_dDI_K3', (16, 16, 18.0, 3, 'ddi', 3), 4, 96, 0.3, 0.3, 0.4, 0.0, 6, 11, 5),
        ('64x64_16QAM_dDI_K1', (64, 16, 24.0, 2, 'ddi', 1), 3, 32, 0.3, 0.3, 0.4, 0.0, 2, 12, 0),
        ('16x16_QPSK_RI_40anneals', (16, 4, 12.0, 3, 'ri', 1), 40, 64, 0.7, 0.5, 0.6, 0.0, 1, 2 ** 40 + 3, 123456),
    ]
    out = {}
    for name, (Nt, M, snr, B, kind, K), R, S, t0, t1, q, kappa, P, seed, inst0 in cases:
        g = torch.Generator(device='cpu')
        g.manual_seed(seed + 100)
        b = mimo.make_batch(B, Nt, Nt, M, snr, g, device='cpu')
        z, Ai, _ = mimo.mmse(b)
        I = mimo.ising(b, z) if kind == 'ri' else mimo.ising_delta_at(b, mimo.mmse_hard(b, z, Ai), K)
        F = chordfx.to_fixed(I, S, t0, t1, q, kappa)
        rs, re = chordfx.chord_fx(F, R, seed, P=P, inst0=inst0)
        bs, be = chordfx.chord_fx(F, R, seed, P=P, inst0=inst0, mode='best')
        for k, v in (('J', F['J']), ('h', F['h']), ('h0', F['h0']), ('T', F['T']), ('c', F['c']),
                     ('chains_s', rs), ('chains_e', re), ('best_s', bs), ('best_e', be)):
            out[name + '/' + k] = v.numpy()
        out[name + '/meta'] = np.array([F['q'], S, P, R, seed & 0xFFFFFFFF, seed >> 32, inst0], dtype=np.int64)
        print('chord', name, 'N', F['h'].shape[1], 'best e', be.tolist()[:3])
    out['names'] = np.array([c[0] for c in cases])
    np.savez_compressed(os.path.join(OUT, 'golden_chord.npz'), **out)


def mapping_fixture():
    out = {}
    rng = np.random.default_rng(11)
    for nt, snr, B, seed in ((16, 12.0, 16, 9700), (32, 16.0, 8, 9701), (64, 20.0, 4, 9702)):
        tag = 'x%d' % nt
        b = arpx.draw(seed, snr, 0, B, nt, 16, dev='cpu')
        z, Ai, _ = mimo.mmse(b)
        mu = mimo._mu(b, z)
        lm = mimo.quantize_levels(z / mu, 16)
        out[tag + '/H'], out[tag + '/y'], out[tag + '/l'] = b['H'].numpy(), b['y'].numpy(), b['l'].numpy()
        out[tag + '/N0'] = np.array([b['N0']])
        out[tag + '/z'], out[tag + '/mu'], out[tag + '/xq'] = z.numpy(), mu.numpy(), lm.numpy()
        for K in (1, 2):
            I = mimo.ising_delta_at(b, lm, K)
            F = chordfx.to_fixed(I, 8 * 2 * K, 0.3, 0.3, 0.4, 0.0)
            G, h = chord_ref.compress(F, K)
            out['%s/K%d/scale' % (tag, K)] = I['scale'].numpy()
            out['%s/K%d/G' % (tag, K)] = G.numpy().astype(np.int32)
            out['%s/K%d/h' % (tag, K)] = h.numpy().astype(np.int32)
            S = torch.from_numpy(rng.choice([-1.0, 1.0], size=(B, 5, 2 * K * 2 * nt)).astype(np.float32))
            Lc = mimo.spins_to_levels_delta(S, I, 16)
            dd = mimo.dist(b, Lc)
            lh, allc, dsel = mimo.select(b, Lc, lm)
            out['%s/K%d/llr' % (tag, K)] = mimo.list_llr(b, allc, dsel, lh, clip=1e4).numpy()
            out['%s/K%d/S' % (tag, K)] = S.numpy().astype(np.int8)
            out['%s/K%d/Lc' % (tag, K)] = Lc.numpy().astype(np.int8)
            out['%s/K%d/dist' % (tag, K)] = dd.numpy()
            out['%s/K%d/sel' % (tag, K)] = lh.numpy().astype(np.int8)
            out['%s/K%d/bits' % (tag, K)] = mimo.levels_to_bits(lh, 16).numpy()
        print('mapping', tag)
    np.savez_compressed(os.path.join(OUT, 'golden_mapping.npz'), **out)


def a513_fixture():
    """Batch 0 of the recorded B200 runs (data/results/a513_fixed): per-use bit errors, anneals per use and the
    per-K counters [flips, tests, anneals] of info.cnt, for the on-device MDI parity test."""
    import json
    pts = {'x16': ('x16/arpeggiofx_64_0.1_0.1_0_rand_32/snr_20.00', 16, 20.0, 102, 'abl_far_64_0.1_0.1_0_rand_32'),
           'x32': ('x32/arpeggiofx_32_0.1_0.1_0_rand_8/snr_22.00', 32, 22.0, 102, 'abl_far_32_0.1_0.1_0_rand_8')}
    out = {}
    for tag, (rel, nt, snr, seed, pick) in pts.items():
        z = np.load(os.path.join(REF, 'data/results/a513_fixed', rel, 'b00000.npz'))
        info = json.loads(str(z['info']))
        out[tag + '/biterr'] = z['biterr']
        out[tag + '/anneals'] = z['anneals']
        out[tag + '/cnt'] = np.array([info['cnt'][str(K)] for K in (1, 2, 3)], dtype=np.int64)
        out[tag + '/meta'] = np.array([nt, snr, seed, info['m']], dtype=np.float64)
        out[tag + '/pick'] = np.array(pick)
        print('a513', tag, int(z['biterr'].sum()), 'bit errors over', info['m'], 'uses')
    np.savez_compressed(os.path.join(OUT, 'golden_a513_b0.npz'), **out)


def a513_points_fixture():
    """Every recorded batch of the three recorded B200 points (data/results/a513_fixed/{x16,x32,x64}): the per-use
    bit errors, for the gate "BER inside the reference's bootstrap CI" on the same draws."""
    import glob
    import json
    pts = {'x16': ('x16/arpeggiofx_64_0.1_0.1_0_rand_32/snr_20.00', 16, 20.0, 102, 'abl_far_64_0.1_0.1_0_rand_32'),
           'x32': ('x32/arpeggiofx_32_0.1_0.1_0_rand_8/snr_22.00', 32, 22.0, 102, 'abl_far_32_0.1_0.1_0_rand_8'),
           'x64': ('x64/arpeggiofx_64_0.1_0.1_0_bal_8/snr_22.00', 64, 22.0, 344, 'abl_far_64_0.1_0.1_0_bal_8')}
    out = {}
    for tag, (rel, nt, snr, seed, pick) in pts.items():
        files = sorted(glob.glob(os.path.join(REF, 'data/results/a513_fixed', rel, 'b*.npz')))
        be = []
        for i, f in enumerate(files):
            assert os.path.basename(f) == 'b%05d.npz' % i
            z = np.load(f)
            be.append(z['biterr'].astype(np.uint8))
        m = int(json.loads(str(np.load(files[0])['info']))['m'])
        out[tag + '/biterr'] = np.stack(be)  # (batches, uses)
        out[tag + '/meta'] = np.array([nt, snr, seed, m], dtype=np.float64)
        out[tag + '/pick'] = np.array(pick)
        print('a513 points', tag, len(files), 'batches', int(out[tag + '/biterr'].sum()), 'bit errors')
    np.savez_compressed(os.path.join(OUT, 'golden_a513_points.npz'), **out)


def stats_fixture():
    """stats_chord.boot_ber, a56an.boot_ratio and a56an.mcnemar on seeded per-use error vectors."""
    import importlib.util
    import stats_chord

    spec = importlib.util.spec_from_file_location('a56an_ref', os.path.join(REF, 'arpeggio/sim/a56an.py'))
    a56 = importlib.util.module_from_spec(spec)
    try:
        spec.loader.exec_module(a56)
    except SystemExit:
        pass
    rng = np.random.default_rng(99)
    a = (rng.random(3000) < 0.02) * rng.integers(1, 4, 3000)
    b = (rng.random(3000) < 0.03) * rng.integers(1, 4, 3000)
    lo, hi, _ = stats_chord.boot_ber(a, 64, B=500)
    r0, rlo, rhi = a56.boot_ratio(a, b, B=800)
    p, x, y = a56.mcnemar(a, b)
    np.savez_compressed(os.path.join(OUT, 'golden_stats.npz'), a=a, b=b,
                        boot_ber=np.array([lo, hi]), boot_ratio=np.array([r0, rlo, rhi]), mcnemar=np.array([p, x, y]))
    print('stats', lo, hi, r0, rlo, rhi, p)


def trajectory_fixture():
    """mimo.trajectory_llr (mimo.py:397-413, with list_llr :434-462) on seeded inputs shaped as chord_soft returns
    them: best levels with their distances, per-bit trajectory minima m0/m1 (some bits never seen with one of their
    values: +inf), the MMSE decision; 16-QAM and QPSK, scalar N0, clip 1e4 (softlib.BIG)."""
    import mimo
    out = {}
    for M, nt in ((16, 8), (4, 16)):
        b = arpx.draw(901 + M, 10.0, 0, 24, nt, M, dev='cpu')
        B, D = b['H'].shape[0], b['H'].shape[2]
        g = torch.Generator().manual_seed(31 + M)
        lv = torch.tensor(mimo.PAM[M]['levels'], dtype=torch.float32)
        best_l = lv[torch.randint(0, len(lv), (B, D), generator=g)]
        mm = lv[torch.randint(0, len(lv), (B, D), generator=g)]
        mm = torch.where(torch.rand(B, D, generator=g) < 0.7, best_l, mm)
        best_d = mimo.dist(b, best_l[:, None, :])[:, 0]
        nbits = D * mimo.PAM[M]['bits']
        m0 = best_d[:, None] * (1 + 2 * torch.rand(B, nbits, generator=g))
        m1 = best_d[:, None] * (1 + 2 * torch.rand(B, nbits, generator=g))
        m0 = torch.where(torch.rand(B, nbits, generator=g) < 0.15, torch.full_like(m0, float('inf')), m0)
        m1 = torch.where(torch.rand(B, nbits, generator=g) < 0.15, torch.full_like(m1, float('inf')), m1)
        l_hat, llr = mimo.trajectory_llr(b, best_l, best_d, m0, m1, mm, clip=1e4)
        tag = 'M%d' % M
        for k, v in (('H', b['H']), ('y', b['y']), ('best_l', best_l), ('best_d', best_d), ('m0', m0), ('m1', m1),
                     ('mmse', mm), ('l_hat', l_hat), ('llr', llr)):
            out['%s/%s' % (tag, k)] = v.numpy()
        out[tag + '/N0'] = np.array([float(b['N0'])])
    np.savez_compressed(os.path.join(OUT, 'golden_trajectory.npz'), **out)
    print('trajectory', {k: v.shape for k, v in out.items() if k.endswith('llr')})


def cycles_fixture():
    """The reference's recorded engine latencies and counters behind the cost models: data/results/a59/A59.json
    (per K, RTL runs of both single-lane engines at A = 1: first-accept tests, flips and latency; Chord steps L,
    flips, n1 and latency) and the model-F cost per anneal of its x16 MDI point P1 with the counters it was computed
    from (data/results/a513/analysis.json: counters_fx, cost_per_anneal.fx)."""
    import json
    a59 = json.load(open(os.path.join(REF, 'data/results/a59/A59.json')))
    keep = ('arpeggio_tests', 'arpeggio_F', 'arpeggio_lat', 'chord_L', 'chord_F', 'chord_n1', 'chord_lat')
    out = {'a59': {pt: {K: {k: v[k] for k in keep} for K, v in a59[pt]['A1']['per_K'].items()} for pt in ('p1', 'p2')}}
    a513 = json.load(open(os.path.join(REF, 'data/results/a513/analysis.json')))['points']['P1']
    out['a513_P1'] = {'counters_fx': a513['counters_fx'], 'cost_per_anneal_fx': a513['cost_per_anneal']['fx']}
    json.dump(out, open(os.path.join(OUT, 'golden_cycles.json'), 'w'), indent=1, sort_keys=True)
    print('cycles', out['a513_P1']['cost_per_anneal_fx'])


if __name__ == '__main__':
    if len(sys.argv) > 2:
        {'stats': stats_fixture, 'a513': a513_fixture, 'mapping': mapping_fixture,
         'a513_points': a513_points_fixture, 'cycles': cycles_fixture,
         'trajectory': trajectory_fixture}[sys.argv[2]]()
        sys.exit(0)
    a513_fixture()
    a513_points_fixture()
    stats_fixture()
    philox_fixture()
    arpeggio_fixture()
    chord_fixture()
    mapping_fixture()
