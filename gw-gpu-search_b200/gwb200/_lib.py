"""ctypes binding of libgwb200.so, the C ABI declared in include/gwb200.h.

The library is built in-tree (gw-gpu-search_b200/build.py) and loaded from gwb200/lib. There is no fallback: if the
library is missing or a call returns a non-zero status, the caller gets an exception."""
import ctypes
import os

import torch

_LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), 'lib', 'libgwb200.so')
_lib = None

GWB_OK = 0
GWB_ERR_SHAPE = 1
GWB_ERR_NOT_POW2 = 2
GWB_ERR_EDGE_ORDER = 3
GWB_ERR_ALLOC = 4
GWB_ERR_CUFFT = 5
GWB_ERR_TIMEOUT = 6
GWB_ERR_CUDA = 7
GWB_ERR_ARG = 8
GWB_ERR_NOT_IMPLEMENTED = 9
GWB_ERR_ALIGN = 10
GWB_ERR_CAPACITY = 11

_P = ctypes.c_void_p
_I = ctypes.c_int
_LL = ctypes.c_longlong
_F = ctypes.c_float
_D = ctypes.c_double

# name -> argument types (all entry points return int status)
SIGNATURES = {
    'gwb_device_error': [_P, _P, _P, _P, _I],
    'gwb_create': [_P],
    'gwb_destroy': [_P],
    'gwb_fft_c2c': [_P, _P, _P, _LL, _I, _LL, _LL, _I, _P],
    'gwb_fft_r2c': [_P, _P, _P, _LL, _I, _LL, _LL, _P],
    'gwb_fft_c2r': [_P, _P, _P, _LL, _I, _LL, _LL, _P],
    'gwb_window_peaks': [_P, _LL, _I, _LL, _I, _I, _P, _P, _P],
    'gwb_fused_peaks_f16': [_P, _P, _LL, _P, _LL, _I, _I, _LL, _I, _P, _P, _LL, _P],
    'gwb_fused_peaks_bf16x3': [_P, _P, _P, _P, _LL, _P, _P, _LL, _I, _I, _LL, _I, _P, _P, _LL, _P],
    'gwb_fused_peaks_f32': [_P, _P, _LL, _P, _LL, _I, _I, _LL, _I, _P, _P, _LL, _P],
    'gwb_f32_set_async': [_I],
    'gwb_fused_peaks_cplx': [_I, _P, _P, _LL, _P, _P, _LL, _I, _I, _LL, _I, _P, _P, _LL, _P, _P, _LL, _P],
    'gwb_fused_peaks_cplx_work_bytes': [_I],
    'gwb_gemm_set_config': [_I, _I, _I, _I, _I],
    'gwb_gemm_clear_configs': [],
    'gwb_basis_premul': [_P, _LL, _I, _P, _LL, _I, _P, _LL, _P, _LL, _P],
    'gwb_basis_scale': [_P, _LL, _I, _LL, _LL, _P, _I, _P, _P, _P],
    'gwb_fft_twiddles': [_LL, _P, _P],
    'gwb_fourstep_order': [_P, _LL, _I, _P, _LL, _LL, _P, _LL, _P],
    'gwb_basis_fused': [_P, _LL, _I, _P, _LL, _P, _P, _I, _LL, _LL, _I, _P, _P, _LL, _I, _I, _I, _P, _LL, _P, _P, _P,
                        _P, _LL, _P],
    'gwb_basis_fused_ring': [_P, _LL, _I, _P, _LL, _P, _P, _I, _LL, _LL, _I, _P, _P, _LL, _I, _I, _P, _LL, _P, _P, _P,
                             _LL, _P, _LL, _P],
    'gwb_basis_ring_set_config': [_I, _I, _I],
    'gwb_basis_ring_rows': [],
    'gwb_basis_set_pass2_columns': [_I, _I],
    'gwb_basis_pass2_columns': [_I],
    'gwb_basis_set_pass2_pairs': [_I],
    'gwb_basis_ring_sync_ints': [_I],
    'gwb_basis_pack': [_P, _LL, _I, _I, _I, _LL, _LL, _P, _I, _P, _P, _LL, _P],
    'gwb_stacked_a': [_P, _LL, _I, _I, _P, _LL, _D, _P, _I, _I, _I, _P, _P, _P, _P, _LL, _P],
    'gwb_stacked_a8': [_P, _LL, _I, _I, _P, _LL, _D, _P, _I, _P, _LL, _P, _P],
    'gwb_select_windows': [_P, _P, _LL, _I, _I, _F, _F, _F, _LL, _I, _I, _P, _P, _P, _P, _LL, _P, _P, _LL, _I, _I, _I,
                           _P, _P, _I, _P, _I, _P, _I, _P, _I, _P, _P],
    'gwb_snr_grad': [_P, _I, _P, _LL, _P, _LL, _I, _D, _I, _D, _I, _I, _P, _LL, _P],
    'gwb_phase_metric': [_P, _I, _P, _LL, _I, _D, _I, _D, _P, _P],
    'gwb_refine_step': [_P, _P, _LL, _P, _P, _I, _P, _P],
    'gwb_edges': [_P, _P, _I, _P, _LL, _P, _LL, _P, _P, _I, _I, _I, _P, _P],
    'gwb_bin_sums': [_P, _P, _I, _P, _P, _P, _I, _P, _P, _LL, _P, _LL, _I, _I, _LL, _P, _P],
    'gwb_exact_finalize': [_P, _P, _I, _P, _P, _I, _P, _I, _I, _P, _P, _LL, _D, _P, _P],
    'gwb_exact_chunks': [_I, _I],
    'gwb_bin_sums_ordered': [_P, _P, _I, _P, _P, _P, _I, _P, _I, _P, _LL, _P, _LL, _I, _I, _LL, _P, _LL, _P, _P, _P],
    'gwb_bin_sums_work_bytes': [_I, _I],
    'gwb_exact_set_staging': [_I],
    'gwb_append_results': [_P, _P, _P, _I, _I, _P, _P, _P, _P, _I, _P, _P, _P],
    'gwb_filter_step_work_bytes': [_P, _I, _I, _I, _LL, _I, _I, _P],
    'gwb_filter_batch_work_bytes': [_P, _I, _I, _I, _LL, _P, _P],
    'gwb_filter_batch': [_P, _P, _LL, _I, _LL, _P, _P, _I, _P, _LL, _I, _P, _P, _P, _P, _P, _LL, _P, _P, _P, _P, _P, _P,
                         _P],
    'gwb_filter_step': [_P, _I, _P, _LL, _I, _P, _P, _I, _D, _P, _P, _LL, _LL, _I, _P, _LL, _I, _P, _P, _LL, _P, _P, _P,
                        _P, _P],
    'gwb_select_top': [_P, _P, _P, _P, _I, _I, _I, _F, _F, _P, _P, _P, _P, _P, _I, _P, _LL, _P],
    'gwb_select_top_work_bytes': [_I, _I],
    'gwb_search_expand': [_P, _P, _P, _I, _LL, _I, _P, _I, _P, _P, _P, _P],
    'gwb_search_best': [_P, _I, _I, _P, _P],
    'gwb_sigma2': [_P, _LL, _I, _P, _LL, _I, _I, _I, _D, _P, _LL, _P, _LL, _P],
    'gwb_sigma2_noalloc': [_P, _LL, _I, _P, _LL, _I, _I, _I, _D, _P, _LL, _P],
    'gwb_gram': [_P, _LL, _I, _P, _I, _I, _P, _LL, _P, _P],
    'gwb_eigh_jacobi_sweep': [_P, _P, _P, _I, _I, _I, _D, _D, _P, _P],
    'gwb_eigh_values': [_P, _P, _I, _I, _P, _P],
    'gwb_basis_vh': [_P, _LL, _I, _I, _P, _LL, _P, _I, _I, _P, _LL, _P],
    'gwb_taylorf2': [_P, _P, _P, _P, _P, _P, _I, _D, _I, _I, _D, _P, _LL, _P],
    'gwb_frames': [_P, _LL, _I, _LL, _LL, _P, _I, _I, _P, _P, _LL, _P],
    'gwb_welch_avg': [_P, _LL, _I, _I, _I, _F, _I, _D, _F, _P, _LL, _P],
    'gwb_interp': [_P, _LL, _I, _I, _D, _D, _I, _P, _LL, _P],
    'gwb_ist_pre': [_P, _LL, _I, _I, _I, _P, _LL, _P],
    'gwb_ist_mid': [_P, _LL, _I, _I, _F, _I, _P, _P],
    'gwb_ist_post': [_P, _LL, _I, _I, _F, _P, _LL, _P],
    'gwb_d_ip': [_P, _LL, _I, _P, _LL, _P, _I, _I, _F, _P, _LL, _P, _LL, _P],
    'gwb_sw': [_P, _LL, _I, _I, _P, _P, _P],
    'gwb_taper_pad': [_P, _LL, _I, _LL, _LL, _P, _P, _P],
    'gwb_whiten': [_P, _I, _P, _F, _F, _P],
    'gwb_above': [_P, _LL, _LL, _I, _F, _F, _P, _P, _I, _P, _P],
    'gwb_apply_gates': [_P, _LL, _P, _I, _P],
    'gwb_consolidate': [_I, _I, _P, _P, _P, _P, _P, _I, _D, _D, _F, _F, _D, _I, _F, _P, _I, _D, _I, _P, _I, _P, _I,
                        _P, _LL, _P, _P, _P],
    'gwb_consolidate_work_bytes': [_I, _I],
    'gwb_highpass': [],
    'gwb_resample': [],
}


class GwbError(RuntimeError):
    def __init__(self, name, status, msg):
        super().__init__('%s failed with status %d (%s): %s' % (name, status, _status_string(status), msg))
        self.status = status


def lib_path():
    return _LIB_PATH


def load():
    """Load the shared library once; raise if it is not built."""
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            raise ImportError('libgwb200.so is not built (%s); run gw-gpu-search_b200/build.py' % _LIB_PATH)
        lib = ctypes.CDLL(_LIB_PATH)
        lib.gwb_version.restype = ctypes.c_int
        lib.gwb_status_string.restype = ctypes.c_char_p
        lib.gwb_status_string.argtypes = [_I]
        lib.gwb_last_error.restype = ctypes.c_char_p
        lib.gwb_num_sms.restype = ctypes.c_int
        for name, args in SIGNATURES.items():
            f = getattr(lib, name)
            f.argtypes = args
            f.restype = ctypes.c_int
        lib.gwb_consolidate_work_bytes.restype = ctypes.c_longlong
        lib.gwb_bin_sums_work_bytes.restype = ctypes.c_longlong
        lib.gwb_fused_peaks_cplx_work_bytes.restype = ctypes.c_longlong
        lib.gwb_select_top_work_bytes.restype = ctypes.c_longlong
        lib.gwb_filter_step_work_bytes.restype = ctypes.c_longlong
        lib.gwb_filter_batch_work_bytes.restype = ctypes.c_longlong
        _lib = lib
    return _lib


def _status_string(status):
    try:
        return load().gwb_status_string(int(status)).decode()
    except Exception:
        return '?'


def call(name, *args):
    """Call an entry point; raise GwbError on a non-zero status."""
    lib = load()
    st = getattr(lib, name)(*args)
    if st != GWB_OK:
        raise GwbError(name, st, lib.gwb_last_error().decode())
    return st


def stream_ptr(device=None):
    """The caller's current torch stream as the void* the C ABI takes."""
    return ctypes.c_void_p(torch.cuda.current_stream(device).cuda_stream)


def ptr(t):
    """Device pointer of a tensor (None -> NULL)."""
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


def row_stride(t):
    """Row stride (elements) of a 2-D tensor whose rows are contiguous; a single row may carry any stride in torch
    (a size-1 dimension's stride is free), so its row length is passed instead."""
    return t.stride(0) if t.shape[0] > 1 else t.shape[1]


def device_error(clear=True):
    """(code, where, info0, info1) from the current device's error word (a synchronous read)."""
    c, w, i0, i1 = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
    call('gwb_device_error', ctypes.byref(c), ctypes.byref(w), ctypes.byref(i0), ctypes.byref(i1), int(clear))
    return c.value, w.value, i0.value, i1.value


def check_device_error():
    """Raise if a kernel recorded an error (bounded wait gave up, failed self-check)."""
    code, where, i0, i1 = device_error(clear=True)
    if code:
        raise GwbError('device', code, 'site %d info %d %d' % (where, i0, i1))


def require_cuda(*tensors):
    """The product path runs on the GPU only: every tensor argument must be a CUDA tensor."""
    for t in tensors:
        if t is not None and not t.is_cuda:
            raise TypeError('gwb200 kernels take CUDA tensors (got a %s tensor)' % t.device)


_handles = {}


def handle(device=None):
    """The per-device library handle (owns cached cuFFT plans), created on first use."""
    dev = torch.cuda.current_device() if device is None else torch.device(device).index
    h = _handles.get(dev)
    if h is None:
        p = ctypes.c_void_p()
        with torch.cuda.device(dev):
            call('gwb_create', ctypes.byref(p))
        h = _handles[dev] = p
    return h
