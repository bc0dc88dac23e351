#!/usr/bin/env python3
"""Pins the CPU oracle against the reference's recorded B200 runs (data/results/a513_fixed).

The reference's own A5.13 driver (arpeggio/sim/local_code_a513/run_a513.py:90-130, `detect`) is run
unchanged on batch 0 of a recorded point, with its GPU solver `arpeggiofx.solve`
(arpeggio/sim/arpeggiofx.py:22-44) swapped for oracle.anneal_dd (same contract).  The recorded
per-K counters [flips, tests, anneals] (info.cnt) and per-use bit errors of b00000.npz were
produced by arpeggio_fx.cu on a B200; equality pins the oracle to the reference kernel on
tens of thousands of real sub-problems.  Host float effects (CPU BLAS last bits, see
arpeggio/sim/arpx.py:40-42) can move a few uses, so differing uses are reported, not hidden.

    python tests/golden/pin_a513.py "$ARPEGGIO_REFERENCE" x16 [x32 x64]
Writes tests/golden/pin_a513.json.
"""
import json
import os
import sys
import time

sys.dont_write_bytecode = True
REF = os.path.abspath(sys.argv[1])
HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for sub in ('arpeggio/mimo', 'arpeggio/sim', 'arpeggio/sim/x3model', 'arpeggio/sim/local_code_a513'):
    sys.path.insert(0, os.path.join(REF, sub))
sys.path.insert(0, ROOT)

import numpy as np  # noqa: E402
import torch  # noqa: E402

torch.set_num_threads(4)
import arpx  # noqa: E402
import arpeggiofx  # noqa: E402
import run_a513  # noqa: E402
from oracle import oracle as O  # noqa: E402

POINTS = {'x16': (16, 20.0, 'x16/arpeggiofx_64_0.1_0.1_0_rand_32/snr_20.00', 'abl_far_64_0.1_0.1_0_rand_32', 102, 2000),
          'x32': (32, 22.0, 'x32/arpeggiofx_32_0.1_0.1_0_rand_8/snr_22.00', 'abl_far_32_0.1_0.1_0_rand_8', 102, 1000),
          'x64': (64, 22.0, 'x64/arpeggiofx_64_0.1_0.1_0_bal_8/snr_22.00', 'abl_far_64_0.1_0.1_0_bal_8', 344, 500)}


def oracle_solve(G, h, P, R, T, q, inst, key, start):
    return O.anneal_dd(np.asarray(G), np.asarray(h), P, R, T, q, inst, key, start, nthreads=os.cpu_count())


def main():
    arpeggiofx.solve = oracle_solve
    path = os.path.join(HERE, 'pin_a513.json')
    res = json.load(open(path)) if os.path.exists(path) else {}
    for tag in sys.argv[2:]:
        nt, snr, rel, pick, seed, B = POINTS[tag]
        rec = np.load(os.path.join(REF, 'data/results/a513_fixed', rel, 'b00000.npz'))
        info = json.loads(str(rec['info']))
        assert info['m'] == B and info['seed'] == seed
        t0 = time.time()
        b = arpx.draw(seed, snr, 0, B, nt, 16, dev='cpu')
        lh, ann, cnt, cs = run_a513.detect(b, nt, 16, arpx.draw_seed(seed, snr, 0), run_a513.parse_pick(pick), 'arpeggiofx', 4)
        bev = arpx.biterr_per_use(b, lh).numpy()
        got = {k: [int(x) for x in v] for k, v in cnt.items()}
        want = info['cnt']
        res[tag] = dict(record=rel + '/b00000.npz', uses=B, wall_s=round(time.time() - t0, 1),
                        counters_equal=got == want, counters_oracle=got, counters_b200=want,
                        biterr_equal=bool(np.array_equal(bev, rec['biterr'])),
                        uses_differing=int((bev != rec['biterr']).sum()),
                        bit_errors_oracle=int(bev.sum()), bit_errors_b200=int(rec['biterr'].sum()),
                        anneals_equal=bool(np.array_equal(ann.astype(np.float32), rec['anneals'])))
        print(tag, json.dumps(res[tag]), flush=True)
    json.dump(res, open(path, 'w'), indent=1)


if __name__ == '__main__':
    main()
