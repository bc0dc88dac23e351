"""Modelled cost budgets for comparing the two flip policies at equal work.

Two cost models, both per anneal:
  model F   (tests, or Chord steps) + flips                     (arpeggio/sim/a58_plan.py:51-62; the reference's
            per-K cost_per_anneal in data/results/a513/analysis.json, written by local_code_a513/analyze_a513.py:94)
  cycles    the single-lane engines' latencies measured on their RTL (data/results/a59/A59.json, A = 1):
            first accept 3 tests + 2 flips  ("PASS cycles = 3 tests + 2 F", data/results/a59/RESULT.txt),
            Chord round 3 L + F + n1 with n1 the rounds that flip  (chord_lat_over_3LFn1 = 1.0 at every K)
  ref_cost[K]   default Chord's cost at K (its steps 256 K, flips and n1 measured on the same batch)
  x             mean over K of cost_K / ref_cost[K]             (arpeggio/sim/a519_plan.py:68-71)
`match_sweeps` picks Arpeggio's sweep count S* for a budget the way the reference's S* rule does: measure the
counters on a tuning batch for each S of a grid and take the largest S whose x does not exceed the target."""
import torch

from . import mdi as _mdi


def cycles_first_accept(tests, flips):
    """Single-lane first-accept engine cycles (3 per comparator pass, 2 per flip)."""
    return 3 * tests + 2 * flips


def cycles_chord(steps, flips, n1):
    """Single-lane Chord engine cycles: 3 per round, 1 per flip, 1 per round that flips."""
    return 3 * steps + flips + n1


def cost_per_anneal(counters, cost='F', policy='arpeggio'):
    """counters {K: [flips, tests_or_steps, anneals(, n1)]} -> {K: cost per anneal} in model F or in engine cycles
    (cost='cycles'; the Chord round needs the n1 counter)."""
    out = {}
    for K, v in counters.items():
        if not v[2]:
            continue
        if cost == 'F':
            c = v[1] + v[0]
        elif policy == 'arpeggio':
            c = cycles_first_accept(v[1], v[0])
        else:
            if len(v) < 4:
                raise ValueError('Chord cycles need the n1 counter (integer Chord round)')
            c = cycles_chord(v[1], v[0], v[3])
        out[str(K)] = c / v[2]
    return out


def ref_cost_chord(counters, cost='F'):
    """Default Chord's per-K cost from its counters."""
    return cost_per_anneal(counters, cost, policy='chord')


def x_of(counters, ref, cost='F', policy='arpeggio'):
    xs = [c / ref[K] for K, c in cost_per_anneal(counters, cost, policy).items() if K in ref]
    return sum(xs) / len(xs) if xs else None


@torch.no_grad()
def counters_of(H, y, N0, M, seed, pick, policy='arpeggio', **kw):
    """Per-K [flips, tests_or_steps, anneals(, n1)] of one MDI run (the reference's info.cnt)."""
    cnt = {}
    _mdi.detect(H, y, N0, M, seed, pick, policy=policy, counters=cnt, **kw)
    return cnt


def match_sweeps(H, y, N0, M, seed, chord_pick, grid, T0=0.1, T1=0.1, q=0.0, start='bal', Ns=None, target=1.0,
                 cost='F'):
    """Largest Arpeggio sweep count S in `grid` whose cost (model F, or engine cycles with cost='cycles') stays
    within `target` x the Chord budget measured on the same tuning batch.  Returns (S*, {S: x}, ref_cost)."""
    ref = ref_cost_chord(counters_of(H, y, N0, M, seed, chord_pick, policy='chord'), cost)
    Ns = chord_pick['Ns'] if Ns is None else Ns
    xs = {}
    for S in sorted(grid):
        pk = dict(S=S, T0=T0, T1=T1, q=q, start=start, Ns=Ns)
        xs[S] = x_of(counters_of(H, y, N0, M, seed, pk), ref, cost)
    ok = [S for S in sorted(grid) if xs[S] is not None and xs[S] <= target]
    return (max(ok) if ok else None), xs, ref
