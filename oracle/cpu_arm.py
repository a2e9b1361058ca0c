"""The CPU arm of the benchmark: one (chunk, tile) sample of the C2 workload on the host cores (test infrastructure,
the oracle used as the timed CPU baseline; never part of the library).

The reference has no CPU path for the compressed filter itself (its GEMM is Triton on a GPU); its numpy code covers
the conditioning (pipeline/gpu_prep.py gpu_stage2 with xp = numpy), the chi-squared edges
(pipeline/multi_filter.py:264-282) and the dense exact stage (pipeline/exact_stage.py:425-439, numpy backend).
This arm runs the oracle's restatements of those (pinned to the reference's own outputs by the golden fixtures) and
the reference's tile pass (pipeline/fp_filter.py:597-621, 741-853) in the precision the reference computes it:
complex64 basis series by scipy.fft with every host core as a worker, complex64 products by the multi-threaded
BLAS, float32 window maxima, then the float64 exact stage spread over the host cores by threads (numpy releases the
GIL inside its array operations)."""
import os
import time
from concurrent.futures import ThreadPoolExecutor

import numpy as np

from . import chisq, filt, prep

try:
    import scipy.fft as _sfft
except ImportError:         # pragma: no cover - scipy is part of the image
    _sfft = None


def cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:   # pragma: no cover
        return os.cpu_count() or 1


def ifft_rows(q, workers):
    """Inverse DFT along rows with norm='forward' (sum without 1/N), complex64 in and out."""
    if _sfft is not None:
        return _sfft.ifft(q, axis=1, norm='forward', workers=workers)
    return (np.fft.ifft(q, axis=1) * q.shape[1]).astype(np.complex64)


def basis_series_c64(Vh, Dw, a0, Tn, tlen, workers, batch=64):
    """fp_filter.py:597-613 in complex64: ifft(conj(Vh) Dw zero-padded to tlen)[a0:a0 + Tn], unscaled."""
    r, flen = Vh.shape
    zb = np.empty((r, Tn), np.complex64)
    q = np.zeros((min(batch, r), tlen), np.complex64)
    for j0 in range(0, r, batch):
        j1 = min(r, j0 + batch)
        q[:j1 - j0, :flen] = np.conj(Vh[j0:j1]) * Dw[None, :]
        zb[j0:j1] = ifft_rows(q[:j1 - j0], workers)[:, a0:a0 + Tn]
    return zb


def window_maxima(As, zb, cw, block_windows=16):
    """|As zb|^2 maxima and first argmax per window of cw samples (the fused GEMM + window reduction,
    fp_filter.py:744-747), complex64 products, blocks of windows to bound the memory."""
    n = As.shape[0]
    nw = zb.shape[1] // cw
    vw = np.empty((n, nw), np.float32)
    iw = np.empty((n, nw), np.int64)
    for w0 in range(0, nw, block_windows):
        w1 = min(nw, w0 + block_windows)
        zt = As @ zb[:, w0 * cw:w1 * cw]
        p = (zt.real * zt.real + zt.imag * zt.imag).reshape(n, w1 - w0, cw)
        j = p.argmax(2)
        iw[:, w0:w1] = j
        vw[:, w0:w1] = np.take_along_axis(p, j[..., None], 2)[..., 0]
    return vw, iw


def exact_threaded(H, nbins, kmin, kmax, D, IP, df, tlen, rows, samples, workers):
    """chisq.exact_dense over the candidates, split into contiguous slices run by a thread pool."""
    n = len(rows)
    if n == 0:
        return chisq.exact_dense(H, nbins, kmin, kmax, D, IP, df, tlen, rows, samples)
    parts = np.array_split(np.arange(n), min(workers, n))
    with ThreadPoolExecutor(len(parts)) as ex:
        res = list(ex.map(lambda ix: chisq.exact_dense(H, nbins, kmin, kmax, D, IP, df, tlen, rows[ix],
                                                       samples[ix]), parts))
    return tuple(np.concatenate([r_[k] for r_ in res]) for k in range(4))


def condition(x, sr, seg_len, start_pad, end_pad, f_low, psd_len, psd_stride, psd_nseg, max_filter_len):
    """gpu_stage2 with xp = numpy (the oracle's restatement, oracle/prep.py): D and IP of one chunk."""
    out = prep.stage2(x, sr, 0, seg_len, start_pad, end_pad, f_low, psd_len, psd_stride, psd_nseg, max_filter_len)
    return out['D'][0], out['IP'][0]


def tile_pass(H, nbins, kmin, kmax, A, Vh, D, IP, isw, df, tlen, a0, Tn, cw, thr, margin, workers):
    """One tile against one chunk: norms (float64), basis series, rebuilt SNR window maxima, candidates above
    (thr (1 - margin))^2, float64 exact stage on every candidate, snr / chisq. Returns (n candidates, n kept)."""
    sig, _ = filt.sigma2(H, IP[None], df)
    norm = 4.0 * df / np.sqrt(sig[:, 0])
    zb = basis_series_c64(Vh, (D * isw).astype(np.complex64), a0, Tn, tlen, workers)
    As = (A * norm[:, None]).astype(np.complex64)
    vw, iw = window_maxima(As, zb, cw)
    del zb
    tb, wb = np.nonzero(vw > (thr * (1 - margin)) ** 2)
    samp = a0 + wb * cw + iw[tb, wb]
    z, pw, fpk, E = exact_threaded(H, nbins, kmin, kmax, D, IP, df, tlen, tb, samp, workers)
    snr, chi, dof = filt.finalize(z, pw, norm[tb], np.asarray(nbins)[tb])
    return len(tb), int((snr > thr).sum())


def timed(fn, *args):
    t0 = time.perf_counter()
    out = fn(*args)
    return out, time.perf_counter() - t0
