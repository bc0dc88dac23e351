"""GPU parity of the learned warm start: the tcgen05 GEMM against a plain PyTorch fp32 product of the same bf16
operands (every operand major and epilogue), the MLP's forward pass and gradients against the CPU oracle's
restatement, the features and the warm start exactly against the oracle, the warm anneal bit for bit against the
oracle's anneal of the relabelled problem, and the trained network's gain over the plain MMSE start at the same
budget."""
import os

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu
NTH = max(1, min(16, os.cpu_count() or 1))
# fp32 accumulation of bf16 products: the tensor core and torch sum in different orders
RTOL, ATOL = 2e-3, 2e-3


def _bf(shape, g, scale=1.0):
    return (torch.randn(*shape, generator=g) * scale).to(torch.bfloat16).cuda()


@pytest.mark.parametrize('a_mn,b_mn', [(0, 0), (0, 1), (1, 0), (1, 1)])
@pytest.mark.parametrize('M,N,K', [(256, 512, 512), (200, 48, 80), (128, 16, 16), (384, 256, 64), (136, 128, 1024),
                                   (328, 208, 1008)])
def test_gemm_matches_torch_fp32(a_mn, b_mn, M, N, K):
    from arpeggio_b200 import warm
    if a_mn and M % 8:
        pytest.skip('MN-major A needs M % 8 == 0')
    g = torch.Generator().manual_seed(M * 7 + N * 3 + K + 11 * a_mn + 5 * b_mn)
    A = _bf((K, M) if a_mn else (M, K), g)
    B = _bf((K, N) if b_mn else (N, K), g)
    Af = (A.float().t() if a_mn else A.float())
    Bf = (B.float() if b_mn else B.float().t())
    ref = Af @ Bf
    C = torch.full((M, N), float('nan'), device='cuda')
    st = torch.zeros(1, dtype=torch.int32, device='cuda')
    warm.gemm(A, a_mn, M if a_mn else K, B, b_mn, N if b_mn else K, M, N, K, warm.EPI_F32, C, N, status=st)
    torch.cuda.synchronize()
    assert int(st.item()) == 0
    torch.testing.assert_close(C, ref, rtol=RTOL, atol=ATOL * K ** 0.5)


def test_gemm_epilogues():
    from arpeggio_b200 import warm
    g = torch.Generator().manual_seed(5)
    M, N, K = 384, 512, 256
    A, B = _bf((M, K), g), _bf((N, K), g)
    bias = torch.randn(N, generator=g).cuda()
    ref = A.float() @ B.float().t()
    out = torch.empty(M, N, dtype=torch.bfloat16, device='cuda')
    warm.gemm(A, 0, K, B, 0, K, M, N, K, warm.EPI_RELU_BF16, out, N, bias=bias)
    torch.testing.assert_close(out.float(), torch.relu(ref + bias).to(torch.bfloat16).float(), rtol=1e-2, atol=2e-2)
    f = torch.empty(M, N, device='cuda')
    warm.gemm(A, 0, K, B, 0, K, M, N, K, warm.EPI_BIAS_F32, f, N, bias=bias)
    torch.testing.assert_close(f, ref + bias, rtol=RTOL, atol=ATOL * K ** 0.5)
    aux = _bf((M, N), g)
    mk = torch.empty(M, N, dtype=torch.bfloat16, device='cuda')
    warm.gemm(A, 0, K, B, 0, K, M, N, K, warm.EPI_MASK_BF16, mk, N, aux=aux, ld_aux=N)
    torch.testing.assert_close(mk.float(), torch.where(aux.float() > 0, ref, 0).to(torch.bfloat16).float(),
                               rtol=1e-2, atol=2e-2)
    # split-K accumulation onto an existing value (long K, few output tiles)
    M2, N2, K2 = 512, 512, 8192
    A2, B2 = _bf((K2, M2), g), _bf((K2, N2), g)
    acc = torch.ones(M2, N2, device='cuda')
    warm.gemm(A2, 1, M2, B2, 1, N2, M2, N2, K2, warm.EPI_ACC, acc, N2)
    torch.cuda.synchronize()
    torch.testing.assert_close(acc, 1 + A2.float().t() @ B2.float(), rtol=RTOL, atol=ATOL * K2 ** 0.5)


def test_gemm_rejects_bad_shapes():
    from arpeggio_b200 import _lib
    L = _lib.lib()
    x = torch.zeros(64, 64, dtype=torch.bfloat16, device='cuda')
    p = _lib.ptr(x)
    assert L.arp_gemm_bf16(p, 0, 64, p, 0, 64, 64, 24, 64, 0, None, None, 0, p, 64, None, None) == 1  # N % 16
    assert L.arp_gemm_bf16(p, 0, 64, p, 0, 64, 64, 16, 40, 0, None, None, 0, p, 64, None, None) == 1  # K % 16
    assert L.arp_gemm_bf16(p, 0, 64, p, 0, 64, 64, 16, 64, 2, None, None, 0, p, 64, None, None) == 3  # no bias
    assert L.arp_gemm_bf16(p, 0, 64, p, 0, 64, 64, 16, 64, 9, None, None, 0, p, 64, None, None) == 3  # epilogue


def _problems(B, nt, snr, seed):
    from arpeggio_b200 import channel, warm
    d = channel.draw_device(seed, snr, B, nt, 16)
    det = warm.WarmDetector(B, nt, anneals=8, sweeps=8)
    det.set_noise(N0=d['N0'])
    det.run(d['H'], d['y'], seed=seed, warm=False)
    torch.cuda.synchronize()
    det.check()
    return d, det


def test_features_and_labels_match_oracle():
    d, det = _problems(96, 32, 14.0, 3)
    lab = torch.empty(96 * 64, dtype=torch.int8, device='cuda')
    det.labels(lab)
    torch.cuda.synchronize()
    X = det.X.float().cpu().numpy()
    Xo, lo = O.warm_features(det.G.cpu().numpy(), det.h.cpu().numpy(), det.xq.cpu().numpy(), det.zs.cpu().numpy(),
                             det.snr_db.cpu().numpy(), 16, 2, det.levels.cpu().numpy())
    Xr = O.bf16(Xo)
    np.testing.assert_allclose(X[:, :9], Xr[:, :9], rtol=1e-2, atol=1e-3)
    # the Jacobi refinements round a continuous move: a half-way tie may fall either side in float32 vs float64
    close = np.isclose(X[:, 9:11], Xr[:, 9:11], rtol=1e-2, atol=1e-2).all(1)
    assert close.mean() >= 0.995, close.mean()
    assert np.array_equal(lab.cpu().numpy(), lo)
    # MMSE soft estimate: its nearest level is the guess
    zs, xq = det.zs.cpu().numpy(), det.xq.cpu().numpy()
    assert np.array_equal(O.quantize_levels(zs, 16), xq)


def test_mlp_forward_and_gradients_match_oracle():
    from arpeggio_b200 import warm
    d, det = _problems(16, 32, 12.0, 9)
    rows = 16 * 64
    lab = torch.empty(rows, dtype=torch.int8, device='cuda')
    det.labels(lab)
    lab[::7] = -1  # ignored rows
    mlp = warm.WarmMLP(P=2, seed=4)
    mlp.reserve(rows, train=True)
    mlp.forward(det.X, rows)
    mlp.backward(det.X, lab, rows)
    torch.cuda.synchronize()
    mlp.check()
    p = mlp.numpy_params()
    X = det.X.float().cpu().numpy()
    H1, H2, Z = O.mlp_forward(X, p['W1'], p['b1'], p['W2'], p['b2'], p['W3t'], p['b3'])
    np.testing.assert_allclose(mlp.Z[:rows].cpu().numpy(), Z, rtol=2e-2, atol=2e-2)
    gr = O.mlp_backward(X, lab.cpu().numpy(), 3, p['W1'], p['W2'], p['W3t'], H1, H2, Z)
    got = {name: mlp.view(mlp.grad, name).cpu().numpy() for name, _ in warm.WarmMLP.LAYOUT}
    for name in ('W1', 'b1', 'W2', 'b2', 'W3t', 'b3'):
        ref = gr[name]
        err = np.abs(got[name] - ref).max() / (np.abs(ref).max() + 1e-6)
        assert err < 3e-2, (name, err)
    assert abs(float(mlp.loss.item()) - gr['loss']) <= 1e-3 * abs(gr['loss']) + 1e-2


def test_training_is_bit_reproducible():
    """Split-K weight gradients and bias gradients reduce in a fixed order: two backward passes give identical
    gradients, and two short trainings from the same seed give identical weights."""
    from arpeggio_b200 import warm
    d, det = _problems(640, 32, 12.0, 19)
    rows = 640 * 64
    lab = torch.empty(rows, dtype=torch.int8, device='cuda')
    det.labels(lab)
    mlp = warm.WarmMLP(P=2, seed=5)
    mlp.reserve(rows, train=True)
    grads = []
    for _ in range(2):
        mlp.forward(det.X, rows)
        mlp.backward(det.X, lab, rows)
        torch.cuda.synchronize()
        grads.append(mlp.grad.clone())
    assert torch.equal(grads[0], grads[1])
    ws = []
    for _ in range(2):
        m = warm.WarmMLP(P=2, seed=6)
        m.reserve(rows // 2, train=True)
        for r0 in (0, rows // 2):
            m.train_step(det.X[r0:r0 + rows // 2], lab[r0:r0 + rows // 2], rows // 2, lr=1e-3)
        torch.cuda.synchronize()
        m.check()
        ws.append(m.w.clone())
    assert torch.equal(ws[0], ws[1])


@pytest.mark.parametrize('rows', [64, 128, 1000, 4096, 40000])
def test_fused_forward_equals_the_layer_by_layer_forward(rows):
    """One persistent launch (hidden activations on chip) against the three GEMM launches of the training path:
    same bf16 roundings and summation order, so the logits agree to the last bit."""
    from arpeggio_b200 import warm
    g = torch.Generator().manual_seed(rows)
    mlp = warm.WarmMLP(P=2, seed=rows)
    X = (torch.randn(rows, 16, generator=g) * 2).to(torch.bfloat16).cuda()
    ref = mlp.forward(X, rows).clone()
    Z = torch.full((rows, 16), float('nan'), device='cuda')
    mlp.infer(X, rows, Z)
    torch.cuda.synchronize()
    mlp.check()
    torch.testing.assert_close(Z, ref, rtol=0, atol=0)


def test_warm_start_and_warm_anneal_match_oracle():
    from arpeggio_b200 import _lib, warm
    d, det = _problems(64, 32, 16.0, 21)
    mlp = warm.WarmMLP(P=2, seed=1)
    # an untrained network gives arbitrary starts: some kept, some falling back
    w = warm.WarmDetector(64, 32, anneals=8, sweeps=8, mlp=mlp)
    w.set_noise(N0=d['N0'])
    w.run(d['H'], d['y'], seed=77)
    torch.cuda.synchronize()
    w.check()
    Z = w.Z[:64 * 64].cpu().numpy()
    G, h, xq = w.G.cpu().numpy(), w.h.cpu().numpy(), w.xq.cpu().numpy()
    m0, perm, e0, kept = O.warm_start(Z, G, h, xq, 2, 16)
    assert np.array_equal(w.m0.cpu().numpy(), m0)
    assert np.array_equal(w.perm.cpu().numpy(), perm)
    assert np.array_equal(w.kept.cpu().numpy(), kept)
    assert np.array_equal(w.e0.cpu().numpy(), e0)
    T, q = w.schedule['T'], w.schedule['q']
    s, de, st = O.anneal_dd_warm(G, h, 2, 8, T, q, np.arange(64), 77, m0, perm, nthreads=NTH)
    assert np.array_equal(w.spins.cpu().numpy(), s)
    assert np.array_equal(w.de.cpu().numpy(), de)
    assert np.array_equal(w.st.cpu().numpy(), st)
    # logits that point at the plain annealer's decisions (so most starts are kept and reordered)
    cls = (det.levels.long() - det.xq.long()) // 2 + 1
    Zc = torch.randn(64 * 64, 16, generator=torch.Generator().manual_seed(3)).cuda()
    Zc[torch.arange(64 * 64), cls.reshape(-1).clamp(0, 2)] += 4.0
    m0c, pc = torch.empty(64, 64, dtype=torch.int8, device='cuda'), torch.empty(64, 64, dtype=torch.uint8,
                                                                                  device='cuda')
    e0c, kc = torch.empty(64, dtype=torch.int64, device='cuda'), torch.empty(64, dtype=torch.int32, device='cuda')
    _lib.check(_lib.lib().arp_warm_start(_lib.ptr(Zc), 16, _lib.ptr(det.G), _lib.ptr(det.h), _lib.ptr(det.xq), 64, 64,
                                         2, 16, 1, _lib.ptr(m0c), _lib.ptr(pc), _lib.ptr(e0c), _lib.ptr(kc),
                                         _lib.stream_ptr()), 'warm_start')
    torch.cuda.synchronize()
    m0o, po, e0o, ko = O.warm_start(Zc.cpu().numpy(), det.G.cpu().numpy(), det.h.cpu().numpy(), det.xq.cpu().numpy(),
                                    2, 16)
    assert ko.sum() > 32
    assert np.array_equal(m0c.cpu().numpy(), m0o) and np.array_equal(pc.cpu().numpy(), po)
    assert np.array_equal(e0c.cpu().numpy(), e0o) and np.array_equal(kc.cpu().numpy(), ko)
    # a forced start and order on every problem (not only the ones the network keeps)
    g = np.random.default_rng(5)
    m0f = (2 * g.integers(-1, 2, size=(64, 64))).astype(np.int8)
    permf = np.stack([g.permutation(64) for _ in range(64)]).astype(np.uint8)
    so = torch.empty(64, 8, 128, dtype=torch.int8, device='cuda')
    deo = torch.empty(64, 8, dtype=torch.int64, device='cuda')
    sto = torch.empty(64, 8, 2, dtype=torch.int64, device='cuda')
    stat = torch.zeros(1, dtype=torch.int32, device='cuda')
    inst = torch.arange(64, dtype=torch.int32, device='cuda')
    Tt = torch.tensor(T, dtype=torch.int32, device='cuda')
    L = _lib.lib()
    m0d, permd = torch.from_numpy(m0f).cuda(), torch.from_numpy(permf).cuda()  # held: the kernel reads them
    _lib.check(L.arp_anneal_first_accept_warm(_lib.ptr(w.G), _lib.ptr(w.h), _lib.ptr(Tt), len(T), int(q), 2, 8, 64, 64,
                                              _lib.ptr(inst), 123, 456, _lib.ptr(m0d), _lib.ptr(permd), _lib.ptr(so),
                                              _lib.ptr(deo), _lib.ptr(sto), _lib.ptr(stat), _lib.stream_ptr()),
               'warm anneal')
    torch.cuda.synchronize()
    assert int(stat.item()) == 0
    s2, de2, st2 = O.anneal_dd_warm(G, h, 2, 8, T, q, np.arange(64), 123 | (456 << 32), m0f, permf, nthreads=NTH)
    assert np.array_equal(so.cpu().numpy(), s2)
    assert np.array_equal(deo.cpu().numpy(), de2)
    assert np.array_equal(sto.cpu().numpy(), st2)
    # an entry outside 0..D-1 is reported, not dereferenced
    bad = permd.clone()
    bad[3, 5] = 200
    _lib.check(L.arp_anneal_first_accept_warm(_lib.ptr(w.G), _lib.ptr(w.h), _lib.ptr(Tt), len(T), int(q), 2, 8, 64, 64,
                                              _lib.ptr(inst), 123, 456, _lib.ptr(m0d), _lib.ptr(bad), _lib.ptr(so),
                                              _lib.ptr(deo), _lib.ptr(sto), _lib.ptr(stat), _lib.stream_ptr()),
               'warm anneal')
    torch.cuda.synchronize()
    assert int(stat.item()) == 2


def test_identity_warm_start_is_the_plain_mmse_start():
    """m0 = 0 in index order is exactly the plain 'bal' (MMSE-started) anneal."""
    from arpeggio_b200 import _lib
    d, det = _problems(32, 32, 12.0, 5)
    L = _lib.lib()
    T = torch.tensor(det.schedule['T'], dtype=torch.int32, device='cuda')
    out = [torch.empty(32, 8, 128, dtype=torch.int8, device='cuda'), torch.empty(32, 8, dtype=torch.int64,
           device='cuda'), torch.empty(32, 8, 2, dtype=torch.int64, device='cuda')]
    m0 = torch.zeros(32, 64, dtype=torch.int8, device='cuda')
    perm = torch.arange(64, dtype=torch.uint8, device='cuda').repeat(32, 1).contiguous()
    inst = torch.arange(32, dtype=torch.int32, device='cuda')
    st = torch.zeros(1, dtype=torch.int32, device='cuda')
    _lib.check(L.arp_anneal_first_accept_warm(_lib.ptr(det.G), _lib.ptr(det.h), _lib.ptr(T), T.numel(), 0, 2, 8, 64, 32,
                                              _lib.ptr(inst), 5, 0, _lib.ptr(m0), _lib.ptr(perm), *map(_lib.ptr, out),
                                              _lib.ptr(st), _lib.stream_ptr()), 'warm')
    torch.cuda.synchronize()
    assert np.array_equal(out[0].cpu().numpy(), det.spins.cpu().numpy())
    assert np.array_equal(out[1].cpu().numpy(), det.de.cpu().numpy())
    assert np.array_equal(out[2].cpu().numpy(), det.st.cpu().numpy())


def test_trained_network_beats_the_plain_start_at_the_same_budget():
    """A short training run on the GPU; on fresh instances at half the x32 budget the warm start reaches lower
    final energies (relative to the MMSE guess) and no more bit errors than the plain MMSE start."""
    from arpeggio_b200 import channel, warm
    mlp = warm.WarmMLP(P=2, seed=0)
    hist = warm.train(mlp, nt=32, instances=65536, batch=8192, anneals=16, sweeps=32, rows_per_step=32768,
                      lr=2e-3, lr_end=2e-4, seed=11)
    assert hist[-1][1] < hist[0][1]  # the loss falls
    B = 4096
    snr = torch.tensor([float(v) for v in np.repeat([10, 14, 18], B // 3 + 1)[:B]])
    d = channel.draw_device(99, snr, B, 32, 16)
    res = {}
    for name, net in (('plain', None), ('warm', mlp)):
        det = warm.WarmDetector(B, 32, anneals=16, sweeps=16, mlp=net)
        det.set_noise(N0=d['N0'])
        det.run(d['H'], d['y'], seed=5)
        torch.cuda.synchronize()
        det.check()
        bt = channel.levels_to_bits(d['l'], 16)
        e = det.energies().min(1).values.clamp(max=0)  # the guess (0) is always a candidate
        res[name] = (float(e.double().mean()), int((det.bits != bt).sum()))
    assert res['warm'][0] < res['plain'][0], res
    assert res['warm'][1] <= res['plain'][1] * 1.02, res


@pytest.mark.parametrize('zero_copy', [True, False])
@pytest.mark.parametrize('warm_start', [False, True])
def test_frame_graph_with_one_copy_each_way_equals_run(warm_start, zero_copy):
    """A captured frame whose H and y sit side by side (one copy in) and whose bits and distances leave in one copy
    (or are written by the readout straight into the mapped pinned outputs) gives the detector's own results."""
    from arpeggio_b200 import channel, warm
    mlp = warm.WarmMLP(P=2, seed=2) if warm_start else None
    f = channel.draw_device(31, 12.0, 4, 32, 16)
    det = warm.WarmDetector(4, 32, anneals=16, sweeps=8, mlp=mlp)
    det.set_noise(N0=f['N0'])
    bits, _, dist = det.run(f['H'], f['y'], 5)
    ref_bits, ref_dist = bits.clone(), dist.clone()
    Hh, yh, Hd, yd, bo, do = det.frame_buffers()
    Hh.copy_(f['H'].cpu())
    yh.copy_(f['y'].cpu())
    g = det.capture(Hh, yh, 5, bo, do, Hd, yd, zero_copy=zero_copy)
    det.bits.zero_()
    bo.zero_()
    do.zero_()
    g.replay()
    torch.cuda.synchronize()
    assert torch.equal(bo, ref_bits.cpu()) and torch.equal(do, ref_dist.cpu())


def test_warm_start_mix_matches_oracle():
    """Only anneals r < warm_r start from the given spin sums; the rest start from the MMSE guess in the same
    order: bit-exact against the oracle."""
    from arpeggio_b200 import _lib
    d, det = _problems(48, 32, 15.0, 8)
    g = np.random.default_rng(9)
    m0 = (2 * g.integers(-1, 2, size=(48, 64))).astype(np.int8)
    perm = np.stack([g.permutation(64) for _ in range(48)]).astype(np.uint8)
    m0d, pd = torch.from_numpy(m0).cuda(), torch.from_numpy(perm).cuda()
    T = det.schedule['T']
    Tt = torch.tensor(T, dtype=torch.int32, device='cuda')
    inst = torch.arange(48, dtype=torch.int32, device='cuda')
    so = torch.empty(48, 8, 128, dtype=torch.int8, device='cuda')
    deo = torch.empty(48, 8, dtype=torch.int64, device='cuda')
    sto = torch.empty(48, 8, 2, dtype=torch.int64, device='cuda')
    stat = torch.zeros(1, dtype=torch.int32, device='cuda')
    for wr in (0, 3, 8):
        _lib.check(_lib.lib().arp_anneal_first_accept_warm_mix(
            _lib.ptr(det.G), _lib.ptr(det.h), _lib.ptr(Tt), len(T), 0, 2, 8, 64, 48, _lib.ptr(inst), 99, 1,
            _lib.ptr(m0d), _lib.ptr(pd), wr, _lib.ptr(so), _lib.ptr(deo), _lib.ptr(sto), _lib.ptr(stat),
            _lib.stream_ptr()), 'warm mix')
        torch.cuda.synchronize()
        s, de, st = O.anneal_dd_warm(det.G.cpu().numpy(), det.h.cpu().numpy(), 2, 8, T, 0, np.arange(48),
                                     99 | (1 << 32), m0, perm, nthreads=NTH, warm_r=wr)
        assert np.array_equal(so.cpu().numpy(), s) and np.array_equal(deo.cpu().numpy(), de), wr
        assert np.array_equal(sto.cpu().numpy(), st), wr


def test_sampled_warm_starts_match_oracle():
    """Sampled starts: the thresholds of softmax(tau z) against a float64 restatement (within 4096 / 2^32), and
    the anneal that draws anneal r's start (0 < r < warm_r) from them bit for bit against the oracle fed the
    device's thresholds."""
    from arpeggio_b200 import _lib
    B, D, R, wr, tau = 64, 64, 8, 6, 0.5
    d, det = _problems(B, 32, 14.0, 31)
    cls = (det.levels.long() - det.xq.long()) // 2 + 1
    Zc = torch.randn(B * D, 16, generator=torch.Generator().manual_seed(4)).cuda()
    Zc[torch.arange(B * D), cls.reshape(-1).clamp(0, 2)] += 3.0
    m0 = torch.empty(B, D, dtype=torch.int8, device='cuda')
    perm = torch.empty(B, D, dtype=torch.uint8, device='cuda')
    e0 = torch.empty(B, dtype=torch.int64, device='cuda')
    kept = torch.empty(B, dtype=torch.int32, device='cuda')
    cdf = torch.empty(B, D, 2, dtype=torch.int32, device='cuda')
    L = _lib.lib()
    _lib.check(L.arp_warm_start_sampled(_lib.ptr(Zc), 16, _lib.ptr(det.G), _lib.ptr(det.h), _lib.ptr(det.xq), B, D,
                                        2, 16, 1, _lib.ptr(m0), _lib.ptr(perm), _lib.ptr(e0), _lib.ptr(kept), tau,
                                        _lib.ptr(cdf), 0.0, 1, R, None, _lib.stream_ptr()), 'warm start sampled')
    torch.cuda.synchronize()
    G, h, xq = det.G.cpu().numpy(), det.h.cpu().numpy(), det.xq.cpu().numpy()
    m0o, po, e0o, ko = O.warm_start(Zc.cpu().numpy(), G, h, xq, 2, 16)
    assert ko.sum() > 16 and ko.sum() < B
    assert np.array_equal(m0.cpu().numpy(), m0o) and np.array_equal(perm.cpu().numpy(), po)
    assert np.array_equal(e0.cpu().numpy(), e0o) and np.array_equal(kept.cpu().numpy(), ko)
    cd = cdf.cpu().numpy().view(np.uint32)
    co = O.warm_cdf(Zc.cpu().numpy(), xq, 2, 16, tau, ko)
    assert np.abs(cd.astype(np.int64) - co.astype(np.int64)).max() <= 4096
    T = det.schedule['T']
    Tt = torch.tensor(T, dtype=torch.int32, device='cuda')
    inst = torch.arange(B, dtype=torch.int32, device='cuda')
    so = torch.empty(B, R, 128, dtype=torch.int8, device='cuda')
    deo = torch.empty(B, R, dtype=torch.int64, device='cuda')
    sto = torch.empty(B, R, 2, dtype=torch.int64, device='cuda')
    stat = torch.zeros(1, dtype=torch.int32, device='cuda')
    _lib.check(L.arp_anneal_first_accept_warm_sampled(
        _lib.ptr(det.G), _lib.ptr(det.h), _lib.ptr(Tt), len(T), 0, 2, R, D, B, _lib.ptr(inst), 17, 3, _lib.ptr(m0),
        _lib.ptr(cdf), _lib.ptr(perm), wr, None, _lib.ptr(so), _lib.ptr(deo), _lib.ptr(sto), _lib.ptr(stat),
        _lib.stream_ptr()), 'warm anneal sampled')
    torch.cuda.synchronize()
    assert int(stat.item()) == 0
    s, de, st = O.anneal_dd_warm(G, h, 2, R, T, 0, np.arange(B), 17 | (3 << 32), m0o, po, nthreads=NTH, warm_r=wr,
                                 cdf=cd)
    assert np.array_equal(so.cpu().numpy(), s) and np.array_equal(deo.cpu().numpy(), de)
    assert np.array_equal(sto.cpu().numpy(), st)
    # the sampled anneals explore: their results are not all anneal 0's
    sd = so.cpu().numpy().reshape(B, R, 2, D).sum(2)
    assert (sd[ko.astype(bool), 1:wr] != sd[ko.astype(bool), :1]).any()


def test_per_problem_anneal_counts_match_oracle():
    """Per-problem anneal counts from the start's confidence: counts against the float64 restatement (away from
    the threshold), the anneal with counts bit for bit against the oracle, each kept anneal identical to the
    full run's, skipped anneals reporting the guess (zero spin sums, INT64_MAX, no statistics)."""
    from arpeggio_b200 import _lib
    B, D, R, tau = 64, 64, 16, 0.5
    d, det = _problems(B, 32, 20.0, 41)
    cls = (det.levels.long() - det.xq.long()) // 2 + 1
    Zc = torch.randn(B * D, 16, generator=torch.Generator().manual_seed(6)).cuda()
    Zc[torch.arange(B * D), cls.reshape(-1).clamp(0, 2)] += 3.0 + 3.0 * torch.rand(B * D, generator=torch.Generator()
                                                                                    .manual_seed(7)).cuda()
    m0 = torch.empty(B, D, dtype=torch.int8, device='cuda')
    perm = torch.empty(B, D, dtype=torch.uint8, device='cuda')
    e0 = torch.empty(B, dtype=torch.int64, device='cuda')
    kept = torch.empty(B, dtype=torch.int32, device='cuda')
    cdf = torch.empty(B, D, 2, dtype=torch.int32, device='cuda')
    ra = torch.empty(B, dtype=torch.int32, device='cuda')
    G, h, xq = det.G.cpu().numpy(), det.h.cpu().numpy(), det.xq.cpu().numpy()
    _, _, _, ko = O.warm_start(Zc.cpu().numpy(), G, h, xq, 2, 16)
    _, conf = O.warm_counts(Zc.cpu().numpy(), 2, ko, 0.0, 4, R)
    cmin = float(np.median(conf[ko.astype(bool)]))
    L = _lib.lib()
    _lib.check(L.arp_warm_start_sampled(_lib.ptr(Zc), 16, _lib.ptr(det.G), _lib.ptr(det.h), _lib.ptr(det.xq), B, D,
                                        2, 16, 1, _lib.ptr(m0), _lib.ptr(perm), _lib.ptr(e0), _lib.ptr(kept), tau,
                                        _lib.ptr(cdf), cmin, 4, R, _lib.ptr(ra), _lib.stream_ptr()), 'warm start')
    torch.cuda.synchronize()
    rao, conf = O.warm_counts(Zc.cpu().numpy(), 2, ko, cmin, 4, R)
    rd = ra.cpu().numpy()
    far = np.abs(conf - cmin) > 1e-3
    assert np.array_equal(rd[far], rao[far])
    assert (rd == 4).sum() >= 8 and (rd == R).sum() >= 8
    T = det.schedule['T']
    Tt = torch.tensor(T, dtype=torch.int32, device='cuda')
    inst = torch.arange(B, dtype=torch.int32, device='cuda')
    outs = [(torch.empty(B, R, 128, dtype=torch.int8, device='cuda'), torch.empty(B, R, dtype=torch.int64, device='cuda'),
             torch.empty(B, R, 2, dtype=torch.int64, device='cuda')) for _ in range(2)]
    stat = torch.zeros(1, dtype=torch.int32, device='cuda')
    for (so, deo, sto), counts in zip(outs, (ra, None)):
        _lib.check(L.arp_anneal_first_accept_warm_sampled(
            _lib.ptr(det.G), _lib.ptr(det.h), _lib.ptr(Tt), len(T), 0, 2, R, D, B, _lib.ptr(inst), 5, 9, _lib.ptr(m0),
            _lib.ptr(cdf), _lib.ptr(perm), R, _lib.ptr(counts) if counts is not None else None, _lib.ptr(so),
            _lib.ptr(deo), _lib.ptr(sto), _lib.ptr(stat), _lib.stream_ptr()), 'warm anneal counts')
    torch.cuda.synchronize()
    assert int(stat.item()) == 0
    cd = cdf.cpu().numpy().view(np.uint32)
    s, de, st = O.anneal_dd_warm(G, h, 2, R, T, 0, np.arange(B), 5 | (9 << 32), m0.cpu().numpy(), perm.cpu().numpy(),
                                 nthreads=NTH, cdf=cd, ra=rd)
    (so, deo, sto), (sf, def_, stf) = [[x.cpu().numpy() for x in o] for o in outs]
    assert np.array_equal(so, s) and np.array_equal(deo, de) and np.array_equal(sto, st)
    for b in range(B):
        k = int(rd[b])
        assert np.array_equal(so[b, :k], sf[b, :k]) and np.array_equal(deo[b, :k], def_[b, :k])
        assert (so[b, k:] == 0).all() and (deo[b, k:] == np.iinfo(np.int64).max).all() and (sto[b, k:] == 0).all()


@pytest.mark.parametrize('nt', [8, 32, 64])
def test_block_per_problem_kernels_equal_the_warp_kernels(nt):
    """Batches of at most 2048 problems take the block-per-problem features and start kernels (G staged in
    shared memory); their outputs are bit-identical to the warp-per-problem kernels' on the same problems."""
    from arpeggio_b200 import _lib
    Bb, Bs = 2100, 64
    d, det = _problems(Bb, nt, 16.0, 50 + nt)
    D = 2 * nt
    L = _lib.lib()
    snr = torch.full((Bb,), 16.0, device='cuda')
    Xb = torch.empty(Bb * D, 16, dtype=torch.bfloat16, device='cuda')
    Xs = torch.empty(Bs * D, 16, dtype=torch.bfloat16, device='cuda')
    lb = torch.empty(Bb * D, dtype=torch.int8, device='cuda')
    ls = torch.empty(Bs * D, dtype=torch.int8, device='cuda')
    for B, X, lab in ((Bb, Xb, lb), (Bs, Xs, ls)):
        _lib.check(L.arp_warm_features(_lib.ptr(det.G), _lib.ptr(det.h), _lib.ptr(det.xq), _lib.ptr(det.zs),
                                       _lib.ptr(snr), B, D, 16, 2, 1, _lib.ptr(X), _lib.ptr(det.levels), _lib.ptr(lab),
                                       _lib.stream_ptr()), 'features')
    torch.cuda.synchronize()
    assert torch.equal(Xb[:Bs * D].view(torch.int16), Xs.view(torch.int16))
    assert torch.equal(lb[:Bs * D], ls)
    cls = (det.levels.long() - det.xq.long()) // 2 + 1
    g = torch.Generator().manual_seed(nt)
    Zc = torch.randn(Bb * D, 16, generator=g).cuda()
    Zc[torch.arange(Bb * D), cls.reshape(-1).clamp(0, 2)] += 2.0 + 4.0 * torch.rand(Bb * D, generator=g).cuda()

    def start(B, sampled):
        o = (torch.empty(B, D, dtype=torch.int8, device='cuda'), torch.empty(B, D, dtype=torch.uint8, device='cuda'),
             torch.empty(B, dtype=torch.int64, device='cuda'), torch.empty(B, dtype=torch.int32, device='cuda'),
             torch.empty(B, D, 2, dtype=torch.int32, device='cuda'), torch.empty(B, dtype=torch.int32, device='cuda'))
        args = [_lib.ptr(Zc), 16, _lib.ptr(det.G), _lib.ptr(det.h), _lib.ptr(det.xq), B, D, 2, 16, 1] + \
            [_lib.ptr(t) for t in o[:4]]
        if sampled:
            _lib.check(L.arp_warm_start_sampled(*args, 0.8, _lib.ptr(o[4]), -5.0 * D / 64, 8, 32, _lib.ptr(o[5]),
                                                _lib.stream_ptr()), 'start')
        else:
            _lib.check(L.arp_warm_start(*args, _lib.stream_ptr()), 'start')
        torch.cuda.synchronize()
        return o if sampled else o[:4]

    for sampled in (False, True):
        big, small = start(Bb, sampled), start(Bs, sampled)
        assert int(big[3].sum()) > 0 and int(big[3].sum()) < Bb
        for a, b in zip(big, small):
            assert torch.equal(a[:Bs], b)
        if sampled:
            assert 0 < int((big[5] == 8).sum()) < Bb


def test_host_device_pointer_refuses_unmapped_memory():
    """Only mapped pinned memory has a device address: pageable host memory and device memory are refused with
    ARP_ERR_ARG (the host-side query fails; nothing runs on the device)."""
    import ctypes
    from arpeggio_b200 import _lib
    L = _lib.lib()
    pinned = torch.empty(64, dtype=torch.int8).pin_memory()
    d = ctypes.c_void_p()
    assert L.arp_host_device_pointer(ctypes.c_void_p(pinned.data_ptr()), ctypes.byref(d)) == 0 and d.value
    pageable = np.zeros(64, dtype=np.int8)
    dev = torch.empty(64, dtype=torch.int8, device='cuda')
    for ptr in (pageable.ctypes.data, dev.data_ptr()):
        d = ctypes.c_void_p(1)
        assert L.arp_host_device_pointer(ctypes.c_void_p(ptr), ctypes.byref(d)) == 3  # ARP_ERR_ARG
        assert not d.value
    assert L.arp_host_device_pointer(None, ctypes.byref(d)) == 3
