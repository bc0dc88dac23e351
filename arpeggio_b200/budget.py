"""Modelled cost budgets for comparing the two flip policies at equal work (the reference's "model F").

  cost per anneal     (tests, or Chord steps) + flips                  (arpeggio/sim/a58_plan.py:51-62)
  ref_cost[K]         default Chord's L_K + F_K: 256 K steps + flips   (a58_plan.py:51-57)
  x                   mean over K of cost_K / ref_cost[K]              (arpeggio/sim/a519_plan.py:68-71)
  first-accept cycles 3 tests + 2 flips (the single-lane engine, data/results/a59/RESULT.txt: "cycles = 3 tests + 2 F")
`match_sweeps` picks Arpeggio's sweep count S* for a budget the way the reference's S* rule does: measure the
counters on a tuning batch for each S of a grid and take the largest S whose x does not exceed the target."""
import torch

from . import mdi as _mdi


def cost_per_anneal(counters):
    """counters {K: [flips, tests_or_steps, anneals]} -> {K: (tests + flips) / anneals}."""
    return {str(K): (v[1] + v[0]) / v[2] for K, v in counters.items() if v[2]}


def ref_cost_chord(counters):
    """Default Chord's L_K + F_K from its counters (L_K = its steps per anneal)."""
    return cost_per_anneal(counters)


def x_of(counters, ref):
    xs = [c / ref[K] for K, c in cost_per_anneal(counters).items() if K in ref]
    return sum(xs) / len(xs) if xs else None


def cycles_first_accept(tests, flips):
    """Single-lane first-accept engine cycles (3 per comparator pass, 2 per flip)."""
    return 3 * tests + 2 * flips


@torch.no_grad()
def counters_of(H, y, N0, M, seed, pick, policy='arpeggio', **kw):
    """Per-K [flips, tests_or_steps, anneals] of one MDI run (the reference's info.cnt)."""
    cnt = {}
    _mdi.detect(H, y, N0, M, seed, pick, policy=policy, counters=cnt, **kw)
    return cnt


def match_sweeps(H, y, N0, M, seed, chord_pick, grid, T0=0.1, T1=0.1, q=0.0, start='bal', Ns=None, target=1.0):
    """Largest Arpeggio sweep count S in `grid` whose model-F cost stays within `target` x the Chord budget measured
    on the same tuning batch.  Returns (S*, {S: x}, ref_cost)."""
    ref = ref_cost_chord(counters_of(H, y, N0, M, seed, chord_pick, policy='chord'))
    Ns = chord_pick['Ns'] if Ns is None else Ns
    xs = {}
    for S in sorted(grid):
        pk = dict(S=S, T0=T0, T1=T1, q=q, start=start, Ns=Ns)
        xs[S] = x_of(counters_of(H, y, N0, M, seed, pk), ref)
    ok = [S for S in sorted(grid) if xs[S] is not None and xs[S] <= target]
    return (max(ok) if ok else None), xs, ref

