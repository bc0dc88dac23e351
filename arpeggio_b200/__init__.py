"""arpeggio_b200: the delta-encoded Ising MIMO detector path of skethz/Arpeggio on B200 (sm_100a).

Hand-written CUDA kernels behind a C ABI (include/arpeggio_b200.h, libarpeggio_b200.so), with Python host
modules that keep the reference's interfaces:
  arpeggiofx  -- solve(G, h, P, R, T, q, inst, key, start) (arpeggio/sim/arpeggiofx.py) and the device form;
  chordfx     -- to_fixed and Kernel.chord / Kernel.philox_kat (arpeggio/mimo/chordfx.py);
  detector    -- the detector call (H, y, constellation, SNR, policy, anneals, budget, seed -> bits, energies)
                 and the solver(I, na, K) protocol of the reference's MDI wrapper.
"""
from . import _lib  # noqa: F401

__all__ = ['arpeggiofx', 'chordfx', 'detector', 'channel']
