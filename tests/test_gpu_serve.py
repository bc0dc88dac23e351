"""The serving loop: continuous batching of mixed-size frames (users, antennas, constellations) arriving as a
Poisson stream; every request's bits and distance equal those of the same request detected alone."""
import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

CLASSES = [(8, 16, 4), (24, 36, 64), (32, 32, 16)]


def _streams(n, seed, burst=False):
    from arpeggio_b200 import channel, serve
    rng = np.random.default_rng(seed)
    out = {}
    for ci, (nt, nr, M) in enumerate(CLASSES):
        snr = torch.tensor(rng.uniform(5, 25, n), dtype=torch.float32)
        d = channel.draw_device(seed * 10 + ci, snr, n, nt, M, nr=nr, dev='cpu')
        t = np.zeros(n) if burst else serve.poisson_arrivals(n, 2e4, rng)
        rid = 1000 * (ci + 1) + np.arange(n)
        out[(nt, nr, M)] = (d['H'].pin_memory(), d['y'].pin_memory(), d['N0'], t, rid)
    return out


@pytest.mark.parametrize('warm_start,slots,burst', [(False, 64, False), (True, 64, False), (False, 256, True)])
def test_each_result_is_the_same_alone_and_in_the_mix(warm_start, slots, burst):
    """Poisson arrivals (small batches: captured graphs) or one burst (a 256-use batch on the direct path, then
    the rest)."""
    from arpeggio_b200 import serve, warm
    mlp = warm.WarmMLP(P=2, seed=3) if warm_start else None
    srv = serve.Server(CLASSES, mlp=mlp, anneals=8, sweeps=8, slots=slots, inflight=2, hbm_budget=1 << 30)
    streams = _streams(300, 5, burst)
    for cls, (H, y, N0, t, rid) in streams.items():
        srv.open(cls, H, y, N0, t, rid)
    stats = srv.serve()
    for cls, (H, y, N0, t, rid) in streams.items():
        st = srv.streams[cls]
        key = '%dx%d %d-QAM' % cls
        assert stats[key]['requests'] == 300
        assert stats[key]['batches'] > 1  # continuous batching, not one batch
        assert not np.isnan(st['done']).any()
        nt, nr, M = cls
        alone = warm.WarmDetector(1, nt, nr, M, anneals=8, sweeps=8, mlp=mlp)
        for i in np.random.default_rng(1).choice(300, 40, replace=False):
            alone.set_noise(N0=N0[i:i + 1])
            inst = torch.tensor([int(rid[i])], dtype=torch.int32, device='cuda')
            bits, _, dist = alone.run(H[i:i + 1].cuda(), y[i:i + 1].cuda(), srv.key, n=1, inst=inst)
            torch.cuda.synchronize()
            assert torch.equal(bits[0].cpu(), st['bits'][i]), (cls, i)
            assert float(dist[0]) == float(st['dist'][i]), (cls, i)


@pytest.mark.parametrize('slots,burst', [(64, False), (256, True)])
def test_native_loop_equals_the_python_loop(slots, burst):
    """The library's loop (arp_serve_run) and this module's step() loop give every request the same bits and
    distance, and both finish every request: Poisson arrivals (small batches), and one burst that the library
    loop takes in batches up to 256 (its graphs beyond 64 uses)."""
    from arpeggio_b200 import serve
    streams = _streams(200 if not burst else 600, 9, burst)
    res = {}
    for native in (True, False):
        srv = serve.Server(CLASSES, anneals=8, sweeps=8, slots=slots, inflight=2, hbm_budget=1 << 30)
        for cls, (H, y, N0, t, rid) in streams.items():
            srv.open(cls, H, y, N0, t, rid)
        stats = srv.serve(native=native)
        for cls in streams:
            st = srv.streams[cls]
            assert stats['%dx%d %d-QAM' % cls]['requests'] == (200 if not burst else 600)
            assert not np.isnan(st['done']).any()
        res[native] = {cls: (srv.streams[cls]['bits'].clone(), srv.streams[cls]['dist'].clone()) for cls in streams}
        del srv
    for cls in streams:
        assert torch.equal(res[True][cls][0], res[False][cls][0]), cls
        assert torch.equal(res[True][cls][1], res[False][cls][1]), cls
    with pytest.raises(ValueError):
        serve.Server(CLASSES[:1], anneals=8, sweeps=8, slots=4).serve(clock=lambda: 0.0, native=True)
    # requests that arrive after the time limit: the library loop gives up and reports it, with nothing in flight
    srv = serve.Server(CLASSES[:1], anneals=8, sweeps=8, slots=4)
    H, y, N0, t, rid = streams[CLASSES[0]]
    srv.open(CLASSES[0], H, y, N0, t + 1e6, rid)
    with pytest.raises(TimeoutError):
        srv.serve(native=True, timeout=0.05)


def test_server_rejects_classes_beyond_shared_memory():
    from arpeggio_b200 import serve
    with pytest.raises(ValueError):
        serve.Server([(96, 96, 16)], anneals=8, sweeps=8, slots=16)
