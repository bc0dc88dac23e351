"""arpeggio_b200: the delta-encoded Ising MIMO detector path of skethz/Arpeggio on B200 (sm_100a).

Hand-written CUDA kernels behind a C ABI (include/arpeggio_b200.h, libarpeggio_b200.so), with Python host
modules that keep the reference's interfaces:
  arpeggiofx  -- solve(G, h, P, R, T, q, inst, key, start) (arpeggio/sim/arpeggiofx.py) and the device form;
  chordfx     -- to_fixed and Kernel.chord / Kernel.philox_kat (arpeggio/mimo/chordfx.py);
  detector    -- the detector call (H, y, constellation, SNR, policy, anneals, budget, seed -> bits, energies)
                 and the solver(I, na, K) protocol of the reference's MDI wrapper;
  mdi         -- the multi-stage (MDI) detector on the device;
  warm        -- the learned warm start (network training and inference on the tensor cores);
  serve       -- continuous batching of mixed-size frames;
  mixed       -- mixed-size batches in one captured CUDA graph and the launch-width autotuner.
"""
from . import _lib  # noqa: F401

__all__ = ['arpeggiofx', 'chordfx', 'detector', 'channel', 'mdi', 'warm', 'serve', 'mixed', 'stats', 'records',
           'budget']
