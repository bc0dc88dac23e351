"""Per-batch detection records in the reference's format (arpeggio/sim/local_code_a513/run_a513.py:151-165):
one NPZ per batch with per-use bit errors (uint8), the indices of the uses in error (int32), their decided
levels (int8), anneals per use (float32) and an `info` JSON string; written to a temporary name and renamed,
and a batch already on disk is skipped on resume (sim/runner.py:139)."""
import json
import os

import numpy as np


def batch_path(root, tag, method, snr, bi):
    return os.path.join(root, tag, method, 'snr_%05.2f' % snr, 'b%05d.npz' % bi)


def write_batch(path, biterr, levels, anneals, info):
    """biterr (n,) per-use bit errors; levels (n, D) decided levels; anneals (n,); info: dict -> JSON."""
    biterr = np.asarray(biterr)
    err = np.nonzero(biterr > 0)[0]
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = os.path.join(os.path.dirname(path), '.tmp_' + os.path.basename(path))
    np.savez_compressed(tmp, biterr=biterr.astype(np.uint8), err_idx=err.astype(np.int32),
                        xhat=np.asarray(levels)[err].astype(np.int8),
                        anneals=np.asarray(anneals, dtype=np.float32), info=np.array(json.dumps(info)))
    os.replace(tmp if tmp.endswith('.npz') else tmp + '.npz', path)


def read_batch(path):
    z = np.load(path, allow_pickle=False)
    return dict(biterr=z['biterr'], err_idx=z['err_idx'], xhat=z['xhat'], anneals=z['anneals'],
                info=json.loads(str(z['info'])))


def done(path):
    return os.path.exists(path)


def point_biterr(root, tag, method, snr):
    """All batches of one point, in batch order: concatenated per-use bit errors."""
    d = os.path.dirname(batch_path(root, tag, method, snr, 0))
    files = sorted(f for f in os.listdir(d) if f.startswith('b') and f.endswith('.npz'))
    return np.concatenate([read_batch(os.path.join(d, f))['biterr'] for f in files])
