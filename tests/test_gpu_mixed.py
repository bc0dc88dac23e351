"""Mixed-size batches in one captured CUDA graph, and the anneal-width autotuner: every class's result equals the
class detected alone, whatever launch width the tuner installs."""
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('persistent', [False, True])
def test_graph_of_mixed_classes_equals_each_class_alone(persistent):
    """Per-class launches on forked streams, or the persistent anneal grids (problems from a device work counter):
    every class's bits, distances, anneal spins, energies and counters equal the class detected alone."""
    from arpeggio_b200 import detector, mixed
    counts = {(8, 16, 4): 40, (16, 24, 64): 33, (24, 24, 16): 50, (32, 48, 16): 64, (48, 48, 4): 20, (64, 96, 64): 17,
              (8, 8, 16): 1, (48, 72, 16): 301}
    mb = mixed.MixedBatch(counts, anneals=8, streams=6, persistent=persistent)  # more streams than slot groups
    mb.draw(3)
    g = mb.capture(seed=11)
    for _ in range(2):
        g.replay()
    torch.cuda.synchronize()
    mb.check()
    for cls, n in counts.items():
        nt, nr, M = cls
        alone = detector.Detector(n, nt, nr, M, 'arpeggio', 8, 1, start='bal')
        alone.sigma2.copy_(mb.dets[cls].sigma2)
        bits, _, dist = alone.run(mb.H[cls], mb.y[cls], 11)
        torch.cuda.synchronize()
        assert torch.equal(bits, mb.dets[cls].bits), cls
        assert torch.equal(dist, mb.dets[cls].dist), cls
        for name in ('spins', 'de', 'st'):
            assert torch.equal(getattr(alone, name), getattr(mb.dets[cls], name)), (cls, name)


def test_autotuned_width_does_not_change_results():
    from arpeggio_b200 import _lib, detector, mixed
    counts = {(32, 32, 16): 300, (64, 64, 16): 100}
    mb = mixed.MixedBatch(counts, anneals=16, streams=2)
    mb.draw(5)
    out = {}
    L = _lib.lib()
    for w in (1, 8):
        for cls in counts:
            _lib.check(L.arp_anneal_tune(2 * cls[0], 2, 0, 0, w), 'tune')
        mb.run(seed=7)
        torch.cuda.synchronize()
        out[w] = {cls: (mb.dets[cls].bits.clone(), mb.dets[cls].de.clone()) for cls in counts}
    tuner = mixed.Autotuner()
    table = mb.tune(tuner)
    assert set(k[0] for k in table) == {64, 128}
    assert all(v['warps'] in (1, 2, 4, 8) for v in table.values())
    mb.run(seed=7)
    torch.cuda.synchronize()
    for cls in counts:
        for w in (8,):
            assert torch.equal(out[1][cls][0], out[w][cls][0]) and torch.equal(out[1][cls][1], out[w][cls][1])
        assert torch.equal(out[1][cls][0], mb.dets[cls].bits)
    tuner.reset()
    assert L.arp_anneal_tune(64, 2, 0, 0, 3) == 3  # not a width


def test_mixed_entry_checks_its_arguments():
    """arp_anneal_first_accept_mixed refuses bad class tables on the host, before any launch."""
    import ctypes
    from arpeggio_b200 import _lib
    L = _lib.lib()
    cnt = torch.zeros(4, dtype=torch.int32, device='cuda')
    assert L.arp_anneal_first_accept_mixed(None, 0, 2, 0, 0, 0, _lib.ptr(cnt), None, None) == 0
    tab = (_lib.MixedClass * 1)()
    tab[0].D, tab[0].B, tab[0].L, tab[0].R = 129, 1, 1, 1
    assert L.arp_anneal_first_accept_mixed(tab, 1, 2, 0, 0, 0, _lib.ptr(cnt), None, None) == 1  # D > 128
    tab[0].D = 32
    assert L.arp_anneal_first_accept_mixed(tab, 1, 2, 0, 0, 0, _lib.ptr(cnt), None, None) == 3  # null pointers
    assert L.arp_anneal_first_accept_mixed(tab, 1, 4, 0, 0, 0, _lib.ptr(cnt), None, None) == 1  # P = 2 only
    assert L.arp_anneal_first_accept_mixed(tab, 65, 2, 0, 0, 0, _lib.ptr(cnt), None, None) == 1  # too many classes
    assert ctypes.sizeof(_lib.MixedClass) == 88
