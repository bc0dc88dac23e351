"""BER statistics for detector runs: the gates "BER inside the reference's bootstrap CI" and paired
comparisons, restated from the reference's analysis code.

  boot_ber    cluster bootstrap of BER over channel uses (arpeggio/sim/stats_chord.py:58-66)
  cp_interval Clopper-Pearson interval (stats_chord.py:50-55)
  boot_ratio  paired cluster bootstrap of sum(a)/sum(b) over uses, exact on the uses with errors
              (arpeggio/sim/a56an.py:74-95)
  mcnemar     exact two-sided McNemar test on per-use error indicators (a56an.py:98-108)
Same random-number order and seeds as the reference, so the intervals agree to the last bit."""
import math

import numpy as np


def boot_ber(biterr, bits_per_use, B=2000, rng=None):
    """biterr (n,) per-use bit errors -> (lo, hi, replicates) of the 95% percentile interval."""
    rng = rng or np.random.default_rng(12345)
    biterr = np.asarray(biterr)
    n = len(biterr)
    reps = np.empty(B)
    for k in range(B):
        idx = rng.integers(0, n, n)
        reps[k] = biterr[idx].sum() / (n * bits_per_use)
    return np.percentile(reps, 2.5), np.percentile(reps, 97.5), reps


def cp_interval(err, bits, alpha=0.05):
    from scipy.stats import beta
    lo = 0.0 if err == 0 else beta.ppf(alpha / 2, err, bits - err + 1)
    hi = 1.0 if err == bits else beta.ppf(1 - alpha / 2, err + 1, bits - err)
    return lo, hi


def boot_ratio(a, b, B=4000, seed=12345):
    """Paired bootstrap of sum(a)/sum(b); returns (ratio, lo, hi)."""
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    U = len(a)
    if U == 0:
        return None, None, None
    nz = np.nonzero((a > 0) | (b > 0))[0]
    sa, sb = a.sum(), b.sum()
    r0 = sa / sb if sb > 0 else (float('inf') if sa > 0 else 1.0)
    if len(nz) == 0:
        return 1.0, 1.0, 1.0
    rng = np.random.default_rng(seed)
    x, y = a[nz], b[nz]
    rs = np.empty(B)
    for i in range(B):
        n = rng.binomial(U, len(nz) / U)
        w = np.bincount(rng.integers(0, len(nz), n), minlength=len(nz))
        ya, yb = float((w * x).sum()), float((w * y).sum())
        rs[i] = ya / yb if yb > 0 else (float('inf') if ya > 0 else 1.0)
    rs.sort()
    return float(r0), float(rs[int(0.025 * (B - 1))]), float(rs[int(math.ceil(0.975 * (B - 1)))])


def mcnemar(a, b):
    """Exact two-sided McNemar on per-use errors: (p, a-only, b-only)."""
    a, b = np.asarray(a), np.asarray(b)
    x, y = int(((a > 0) & (b == 0)).sum()), int(((a == 0) & (b > 0)).sum())
    n = x + y
    if n == 0:
        return 1.0, x, y
    k = min(x, y)
    p = sum(math.comb(n, i) for i in range(k + 1)) / 2 ** n
    return min(1.0, 2 * p), x, y


def ber_inside(biterr, bits_per_use, ref_lo, ref_hi):
    """The gate: this run's BER lies inside the reference's interval [ref_lo, ref_hi]."""
    ber = float(np.asarray(biterr).sum()) / (len(biterr) * bits_per_use)
    return ref_lo <= ber <= ref_hi, ber
