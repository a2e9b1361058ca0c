"""Per-window peak picking: drop-in for pipeline/peak_kernel.py (window_peaks, :41-47).

For each (row, window) the maximum |z|^2 over the window's cw samples and its offset in the window; the first offset
wins ties (numpy argmax order), as the reference's win_peak kernel (peak_kernel.py:10-36)."""
import torch

from . import _lib

THREADS = 128


def window_peaks(z, a0, cw, nwin):
    """z: (rows, N) complex64 CUDA tensor. Returns (max |z|^2, argmax within window), each (rows, nwin)."""
    _lib.require_cuda(z)
    assert z.dtype == torch.complex64 and z.is_contiguous()
    rows = z.shape[0]
    pmax = torch.empty((rows, nwin), dtype=torch.float32, device=z.device)
    pidx = torch.empty((rows, nwin), dtype=torch.int32, device=z.device)
    _lib.call('gwb_window_peaks', _lib.ptr(z), int(z.shape[1]), int(rows), int(a0), int(cw), int(nwin),
              _lib.ptr(pmax), _lib.ptr(pidx), _lib.stream_ptr(z.device))
    return pmax, pidx
