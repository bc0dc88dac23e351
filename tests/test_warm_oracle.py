"""CPU checks of the warm-start oracle and of the serving / mixed-batch host logic (no GPU): the oracle's MLP
gradients against finite differences of its own loss, the warm anneal of an identity order and zero start
against the plain 'bal' anneal, a relabelled problem against the same problem, the warm start's fallback rule,
and the admission arithmetic of the server."""
import numpy as np

from oracle import oracle as O


def _mlp(seed, scale=0.3):
    r = np.random.default_rng(seed)
    return {'W1': r.normal(0, scale, (O.NH, O.NF)).astype(np.float32), 'b1': r.normal(0, 0.1, O.NH).astype(np.float32),
            'W2': r.normal(0, scale / 8, (O.NH, O.NH)).astype(np.float32),
            'b2': r.normal(0, 0.1, O.NH).astype(np.float32),
            'W3t': r.normal(0, scale / 8, (O.NH, O.NO)).astype(np.float32),
            'b3': r.normal(0, 0.1, O.NO).astype(np.float32)}


def _loss64(X, lab, p, C=3):
    """The same loss in float64 without bf16 roundings (the quantity the gradients differentiate)."""
    H1 = np.maximum(X @ p['W1'].T.astype(np.float64) + p['b1'], 0)
    H2 = np.maximum(H1 @ p['W2'].T.astype(np.float64) + p['b2'], 0)
    Z = (H2 @ p['W3t'].astype(np.float64) + p['b3'])[:, :C]
    zm = Z.max(1, keepdims=True)
    lse = np.log(np.exp(Z - zm).sum(1)) + zm[:, 0]
    v = lab >= 0
    return float((lse - Z[np.arange(len(lab)), np.maximum(lab, 0)])[v].sum())


def test_oracle_mlp_gradients_match_finite_differences():
    r = np.random.default_rng(0)
    X = O.bf16(r.normal(0, 1, (24, O.NF)).astype(np.float32))
    lab = r.integers(-1, 3, 24)
    p = {k: O.bf16(v) for k, v in _mlp(1).items()}
    H1, H2, Z = O.mlp_forward(X, p['W1'], p['b1'], p['W2'], p['b2'], p['W3t'], p['b3'])
    g = O.mlp_backward(X, lab, 3, p['W1'], p['W2'], p['W3t'], H1, H2, Z)
    pd = {k: v.astype(np.float64) for k, v in p.items()}
    eps = 1e-4
    for name, idx in (('b3', (1,)), ('W3t', (5, 2)), ('b2', (7,)), ('W2', (3, 11)), ('W1', (9, 4)), ('b1', (2,))):
        hi, lo = {k: v.copy() for k, v in pd.items()}, {k: v.copy() for k, v in pd.items()}
        hi[name][idx] += eps
        lo[name][idx] -= eps
        fd = (_loss64(X, lab, hi) - _loss64(X, lab, lo)) / (2 * eps)
        # the oracle keeps the device's bf16 roundings of dZ and the hidden activations: agreement to ~1 %
        assert abs(g[name][idx] - fd) <= 0.02 * abs(fd) + 2e-3, (name, g[name][idx], fd)


def _problem(B, D, seed):
    r = np.random.default_rng(seed)
    A = r.normal(0, 1, (B, D, D))
    G = np.round(np.einsum('bij,bkj->bik', A, A) / D * 600).astype(np.int32)
    h = np.round(r.normal(0, 800, (B, D))).astype(np.int32)
    return G, h


def test_oracle_warm_anneal_identity_is_the_bal_anneal():
    G, h = _problem(6, 40, 2)
    T = [400] * 16
    s0, de0, st0 = O.anneal_dd(G, h, 2, 4, T, 0, np.arange(6), 99, 'bal')
    s1, de1, st1 = O.anneal_dd_warm(G, h, 2, 4, T, 0, np.arange(6), 99, np.zeros((6, 40), np.int8),
                                    np.tile(np.arange(40, dtype=np.uint8), (6, 1)))
    assert np.array_equal(s0, s1) and np.array_equal(de0, de1) and np.array_equal(st0, st1)


def test_oracle_warm_anneal_is_the_anneal_of_the_relabelled_problem():
    G, h = _problem(4, 33, 3)
    T = [300] * 12
    r = np.random.default_rng(4)
    perm = np.stack([r.permutation(33) for _ in range(4)]).astype(np.uint8)
    m0 = (2 * r.integers(-1, 2, (4, 33))).astype(np.int8)
    s, de, st = O.anneal_dd_warm(G, h, 2, 3, T, 0, np.arange(4), 7, m0, perm)
    # relabel by hand and anneal with the identity order: the same trajectories, spins relabelled back
    bi = np.arange(4)[:, None]
    Gp = G[bi[:, :, None], perm[:, :, None].astype(np.int64), perm[:, None, :].astype(np.int64)]
    hp = h[bi, perm.astype(np.int64)]
    mp = m0[bi, perm.astype(np.int64)]
    ident = np.tile(np.arange(33, dtype=np.uint8), (4, 1))
    s2, de2, st2 = O.anneal_dd_warm(Gp, hp, 2, 3, T, 0, np.arange(4), 7, mp, ident)
    assert np.array_equal(de, de2) and np.array_equal(st, st2)
    s2 = s2.reshape(4, 3, 2, 33)
    back = np.empty_like(s2)
    for b in range(4):
        back[b][..., perm[b].astype(np.int64)] = s2[b]
    assert np.array_equal(s, back.reshape(4, 3, 66))


def test_oracle_warm_start_falls_back_when_worse_than_the_guess():
    G, h = _problem(3, 16, 5)
    logits = np.zeros((3 * 16, 16), np.float32)
    logits[:, 2] = 5.0  # every coordinate up by one level step
    xq = np.full((3, 16), -1, np.int8)
    h = -np.abs(h)  # the guess is a strict minimiser along +moves: moving up costs energy
    m0, perm, e0, kept = O.warm_start(logits, G, h, xq, 2, 16)
    assert (kept == 0).all() and (m0 == 0).all() and (e0 == 0).all()
    assert np.array_equal(perm, np.tile(np.arange(16, dtype=np.uint8), (3, 1)))
    m0, perm, e0, kept = O.warm_start(logits, G, -h, xq, 2, 16)  # now the move is downhill along h
    assert kept.dtype == np.int32


def test_oracle_sampled_starts():
    """Thresholds exclude the classes that leave the constellation and fall back to m = 0 for dropped problems;
    thresholds that always give m = 0 make the sampled anneal the warm anneal with warm_r = 1; thresholds that
    always give m0's class make it the warm anneal with every anneal from m0."""
    r = np.random.default_rng(8)
    xq = r.integers(-3, 4, (5, 24)).astype(np.int8)
    xq[0, :4] = [-3, 3, -1, 1]
    logits = r.normal(0, 2, (5 * 24, 16)).astype(np.float32)
    kept = np.array([1, 1, 1, 1, 0], np.int32)
    c = O.warm_cdf(logits, xq, 2, 16, 0.5, kept)
    assert c[0, 0, 0] == 0 and c[0, 1, 1] == 0xFFFFFFFF
    assert (c[..., 0] <= c[..., 1]).all()
    assert (c[4, :, 0] == 0).all() and (c[4, :, 1] == 0xFFFFFFFF).all()
    G, h = _problem(5, 24, 6)
    T = [300] * 10
    m0 = (2 * r.integers(-1, 2, (5, 24))).astype(np.int8)
    perm = np.stack([r.permutation(24) for _ in range(5)]).astype(np.uint8)
    zero = np.zeros((5, 24, 2), np.uint32)
    zero[..., 1] = 0xFFFFFFFF
    a = O.anneal_dd_warm(G, h, 2, 4, T, 0, np.arange(5), 21, m0, perm, warm_r=4, cdf=zero)
    b = O.anneal_dd_warm(G, h, 2, 4, T, 0, np.arange(5), 21, m0, perm, warm_r=1)
    assert all(np.array_equal(u, v) for u, v in zip(a, b))
    same = np.where(m0[..., None] < 0, [0xFFFFFFFF, 0xFFFFFFFF], np.where(m0[..., None] > 0, [0, 0],
                                                                          [0, 0xFFFFFFFF])).astype(np.uint32)
    a = O.anneal_dd_warm(G, h, 2, 4, T, 0, np.arange(5), 21, m0, perm, warm_r=4, cdf=same)
    b = O.anneal_dd_warm(G, h, 2, 4, T, 0, np.arange(5), 21, m0, perm, warm_r=4)
    assert all(np.array_equal(u, v) for u, v in zip(a, b))


def test_serving_admission_and_mixed_classes():
    from arpeggio_b200 import mixed, serve
    cls = mixed.mixed_classes()
    assert len(cls) == 54 and (64, 128, 64) in cls and (8, 12, 4) in cls
    n = mixed.mixed_counts(1_000_000, seed=1)
    assert sum(n.values()) == 1_000_000
    # every class of the mix fits the kernels' shared memory; a 96-user class does not (D > 128)
    assert all(serve.shared_bytes(c, 32) <= 227 * 1024 for c in cls)
    assert serve.shared_bytes((64, 128, 16), 32) > serve.shared_bytes((64, 64, 16), 32)
    arrivals = serve.poisson_arrivals(10000, 1e5, np.random.default_rng(0))
    assert np.all(np.diff(arrivals) > 0) and abs(arrivals[-1] - 0.1) < 0.01
    # the library loop's graph sizes: powers of two to 64, then steps of about a quarter, at most 32 sizes; a batch
    # of k requests pads to the next size by at most ~25 % beyond 64
    for slots in (1, 5, 64, 100, 4096, 100000):
        sz = serve.native_sizes(slots)
        assert sz[0] == 1 and len(sz) <= 32 and all(b > a for a, b in zip(sz, sz[1:])) and sz[-1] <= slots
        assert sz[-1] == slots or len(sz) == 32 or slots < 64  # below 64: the largest power of two
        for k in range(65, sz[-1] + 1, 97):
            kb = next(v for v in sz if v >= k)
            assert kb <= max(k + 32, 1.25 * k + 32)


def test_oracle_anneal_counts_skip_exactly_the_late_anneals():
    """Anneal counts keep anneals r < ra[b] as in the full run and report the guess for the rest."""
    G, h = _problem(4, 20, 9)
    T = [300] * 8
    r = np.random.default_rng(10)
    m0 = (2 * r.integers(-1, 2, (4, 20))).astype(np.int8)
    perm = np.stack([r.permutation(20) for _ in range(4)]).astype(np.uint8)
    ra = np.array([1, 3, 6, 0], np.int32)  # 0 is clamped to 1
    full = O.anneal_dd_warm(G, h, 2, 6, T, 0, np.arange(4), 3, m0, perm)
    part = O.anneal_dd_warm(G, h, 2, 6, T, 0, np.arange(4), 3, m0, perm, ra=ra)
    for b, k in enumerate(np.maximum(ra, 1)):
        for f, p in zip(full, part):
            assert np.array_equal(f[b, :k], p[b, :k])
        assert (part[0][b, k:] == 0).all() and (part[1][b, k:] == np.iinfo(np.int64).max).all()
        assert (part[2][b, k:] == 0).all()
    logits = np.zeros((2 * 20, 16), np.float32)
    logits[:20, 1] = 9.0  # problem 0 confident, problem 1 uniform (confidence 20 log(1/3))
    counts, conf = O.warm_counts(logits, 2, np.array([1, 1]), -1.0, 4, 16)
    assert list(counts) == [4, 16] and abs(conf[1] - 20 * np.log(1 / 3)) < 1e-9
