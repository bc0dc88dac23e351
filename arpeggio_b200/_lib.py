"""ctypes binding of the in-tree C-ABI library libarpeggio_b200.so (declarations: include/arpeggio_b200.h).

There is no fallback: if the library is missing or a call fails, an exception is raised."""
import ctypes
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, 'libarpeggio_b200.so')

_P = ctypes.c_void_p
_I = ctypes.c_int
_U = ctypes.c_uint32
_F = ctypes.c_float

# name -> argtypes, in the order of include/arpeggio_b200.h
SIGNATURES = {
    'arp_version': [],
    'arp_status_string': [_I],
    'arp_host_device_pointer': [_P, _P],
    'arp_philox_kat': [_P, _P, _I, _P],
    'arp_philox_rate': [_P, _I, _I, _I, _P],
    'arp_anneal_first_accept': [_P, _P, _P, _I, _I, _I, _I, _I, _I, _P, _U, _U, _I, _P, _P, _P, _P, _P],
    'arp_anneal_chord_dd': [_P, _P, _P, _P, _I, _I, _I, _I, _I, _I, _P, _U, _U, _I, _P, _P, _P, _P, _P],
    'arp_anneal_chord_dd_n1': [_P, _P, _P, _P, _I, _I, _I, _I, _I, _I, _P, _U, _U, _I, _P, _P, _P, _P, _P, _P],
    'arp_anneal_chord_engine': [_P, _P, _P, _P, _I, _I, _I, _I, _I, _I, _P, _U, _U, _P, _P, _P, _P, _P],
    'arp_anneal_dd_f32': [_I, _P, _P, _P, _P, _I, _F, _I, _I, _I, _I, _P, _U, _U, _I, _P, _P, _P, _P, _P],
    'arp_anneal_chord': [_P, _P, _P, _P, _P, _I, _I, _I, _I, _I, _I, _U, _U, _U, _I, _I, _P, _P, _P, _P, _P],
    'arp_map_dd': [_P, _P, _P, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P],
    'arp_readout_dd': [_P, _P, _P, _P, _I, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P],
    'arp_map_ri': [_P, _P, _P, _I, _I, _I, _I, _F, _P, _P, _P, _P, _P, _P, _P],
    'arp_anneal_full_f32': [_I, _P, _P, _P, _P, _P, _I, _F, _I, _I, _I, _I, _P, _U, _U, _P, _P, _P, _P],
    'arp_readout_ri': [_P, _P, _P, _P, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P],
    'arp_readout_llr_dd': [_P, _P, _P, _P, _I, _I, _I, _I, _I, _I, _P, _F, _P, _P, _P, _P, _P, _P],
    'arp_detect_dd': [_P, _P, _P, _I, _I, _I, _I, _I, _I, _I, _I, _P, _P, _I, ctypes.c_double, _U, _U, _U, _I, _P,
                      ctypes.c_size_t, _P, _P, _P, _P, _P, _P],
    'arp_detect_dd_workspace': [_I, _I, _I, _I, _I, _P],
    'arp_mdi_guesses': [_P, _P, _P, _I, _I, _I, _I, _P, _P, _P],
    'arp_mdi_radius': [_P, _P, _P, _I, _I, _I, _I, _I, _I, _P, _P, _P],
    'arp_mdi_map': [_P, _P, _P, _I, _I, _I, _I, _P, _I, _I, _I, _P, _P, _P, _P, _P, _P],
    'arp_mdi_update': [_P, _P, _P, _I, _I, _I, _I, _I, _I, _P, _I, _I, _P, _P, _P, _P],
    'arp_mdi_select': [_P, _P, _I, _I, _I, _I, _P, _P, _P],
    'arp_soft_trajectory': [_P, _P, _P, _P, _P, _P, _P, _F, _I, _I, _I, _I, _I, _P, _U, _U, _P, _P, _P, _P, _P],
    'arp_anneal_tune': [_I, _I, _I, _I, _I],
    'arp_anneal_first_accept_mixed': [_P, _I, _I, _U, _U, _I, _P, _P, _P],
    'arp_map_dd_soft': [_P, _P, _P, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P, _P, _P],
    'arp_gemm_bf16': [_P, _I, _I, _P, _I, _I, _I, _I, _I, _I, _P, _P, _I, _P, _I, _P, _P],
    'arp_warm_features': [_P, _P, _P, _P, _P, _I, _I, _I, _I, _I, _P, _P, _P, _P],
    'arp_warm_loss': [_P, _I, _P, _I, _I, _P, _I, _P, _P, _P],
    'arp_colsum_bf16': [_P, _I, _I, _I, _P, _P],
    'arp_adam': [_P, _P, _P, _P, _P, _I, _F, _F, _F, _F, _I, _F, _P],
    'arp_warm_start': [_P, _I, _P, _P, _P, _I, _I, _I, _I, _I, _P, _P, _P, _P, _P],
    'arp_mlp_pack_w2': [_P, _P, _P],
    'arp_mlp_forward': [_P, _I, _P, _P, _P, _P, _P, _P, _P, _P, _P],
    'arp_anneal_first_accept_warm': [_P, _P, _P, _I, _I, _I, _I, _I, _I, _P, _U, _U, _P, _P, _P, _P, _P, _P, _P],
    'arp_anneal_first_accept_warm_mix': [_P, _P, _P, _I, _I, _I, _I, _I, _I, _P, _U, _U, _P, _P, _I, _P, _P, _P, _P,
                                         _P],
    'arp_warm_start_sampled': [_P, _I, _P, _P, _P, _I, _I, _I, _I, _I, _P, _P, _P, _P, _F, _P, _F, _I, _I, _P, _P],
    'arp_anneal_first_accept_warm_sampled': [_P, _P, _P, _I, _I, _I, _I, _I, _I, _P, _U, _U, _P, _P, _P, _I, _P, _P,
                                             _P, _P, _P, _P],
    'arp_serve_run': [_P, _I, _P, _I, ctypes.c_double, _P],
    'arp_detect_dd_static': [_P, _P, _P, _I, _I, _I, _I, _I, _I, _I, _I, _P, _P, _I, ctypes.c_double, _U, _U, _U,
                             _I, _P, _P, _P, _P, _P, _P],
}

_lib = None


class MixedClass(ctypes.Structure):
    """arp_mixed_class: one size class of arp_anneal_first_accept_mixed (layout of include/arpeggio_b200.h)."""
    _fields_ = [('Gt', _P), ('h', _P), ('T', _P), ('L', _I), ('q', _I), ('R', _I), ('D', _I), ('B', _I),
                ('inst', _P), ('start', _I), ('out_s', _P), ('out_de', _P), ('out_st', _P)]


class ServeStream(ctypes.Structure):
    """arp_serve_stream: one size class's request stream for arp_serve_run."""
    _fields_ = [('H', _P), ('y', _P), ('s2', _P), ('snr', _P), ('rid', _P), ('t_arrival', _P), ('n', _I),
                ('h_elems', _I), ('y_elems', _I), ('bits_per', _I), ('bits', _P), ('dist', _P), ('done', _P)]


class ServeLane(ctypes.Structure):
    """arp_serve_lane: one lane (stream, graphs per power-of-two batch, device buffers) for arp_serve_run."""
    _fields_ = [('cls', _I), ('stream', _P), ('ngraphs', _I), ('sizes', _I * 32), ('graphs', _P * 32), ('Hd', _P), ('yd', _P),
                ('s2d', _P), ('snrd', _P), ('instd', _P), ('bitsd', _P), ('distd', _P)]


class ArpError(RuntimeError):
    pass


def lib():
    """Loads the library (building it first when only the sources are present)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            from . import build
            build.build()
        if not os.path.exists(LIB):
            raise ArpError('libarpeggio_b200.so is missing; run python -m arpeggio_b200.build')
        L = ctypes.CDLL(LIB)
        for name, argt in SIGNATURES.items():
            f = getattr(L, name)
            f.argtypes = argt
            f.restype = (ctypes.c_char_p if name in ('arp_version', 'arp_status_string') else
                         ctypes.c_size_t if name.endswith('_workspace') else ctypes.c_int)
        _lib = L
    return _lib


def check(rc, what):
    if rc != 0:
        raise ArpError('%s failed: %s (code %d)' % (what, lib().arp_status_string(rc).decode(), rc))


def ptr(t):
    """Device pointer of a torch tensor (None -> NULL)."""
    return None if t is None else ctypes.c_void_p(t.data_ptr())


def host_device_ptr(t):
    """Device address of a pinned (mapped) host tensor, for kernels that write results straight into it."""
    d = ctypes.c_void_p()
    check(lib().arp_host_device_pointer(ctypes.c_void_p(t.data_ptr()), ctypes.byref(d)), 'host_device_pointer')
    return d


def stream_ptr(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)
