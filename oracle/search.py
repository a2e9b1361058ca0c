"""End-to-end oracle of one (tile, segment) pass of the compressed filter (test infrastructure only).

Follows pipeline/fp_filter.py:741-853 for one tile and one segment: basis series (float64 transform), stacked A, the
rebuilt SNR series and its per-window maxima (the fused GEMM + window reduction, :744-747), candidates above
(thr (1 - margin))^2, the exact stage on every candidate (exact_snr = 0: exact everywhere, :769) and the final
snr / chisq / newsnr (:837-853)."""
import numpy as np

from . import chisq, filt


def tile_segment(H, nbins, kmin, kmax, r, A, Vh, D, IP, isw, sig_col, df, tlen, a0, Tn, cw, thr, margin):
    """Returns dict of candidates (row, window, sample, approx) and exact values (z, pw, snr, chisq, dof, newsnr)."""
    zb = filt.basis_series_complex(Vh, D * isw, a0, Tn, tlen)          # (r, Tn) complex128
    norm = 4.0 * df / np.sqrt(sig_col)
    zt = (A.astype(np.complex128) @ zb) * norm[:, None]                 # rebuilt complex SNR (n, Tn)
    p = zt.real ** 2 + zt.imag ** 2
    nw = Tn // cw
    pw = p[:, :nw * cw].reshape(len(p), nw, cw)
    iw = pw.argmax(2)
    vw = np.take_along_axis(pw, iw[..., None], 2)[..., 0]
    thr2 = (thr * (1 - margin)) ** 2
    tb, wb = np.nonzero(vw > thr2)
    samp = a0 + wb * cw + iw[tb, wb]
    approx = np.sqrt(vw[tb, wb])
    z, pwr, fpk, E = chisq.exact_dense(H, nbins, kmin, kmax, D, IP, df, tlen, tb, samp)
    snr, chi, dof = filt.finalize(z, pwr, norm[tb], np.asarray(nbins)[tb])
    ns = filt.newsnr(snr, chi / np.maximum(dof, 1))
    return dict(row=tb, window=wb, sample=samp, approx=approx, vw=vw, z=z, pw=pwr, snr=snr, chisq=chi, dof=dof,
                newsnr=ns, fpeak=fpk)


def tile_segment_lean(H, nbins, kmin, kmax, r, A, Vh, D, IP, isw, sig_col, df, tlen, a0, Tn, cw, thr, margin,
                      chunk_windows=32):
    """tile_segment with the rebuilt SNR formed a block of windows at a time (bounded memory), complex64 products
    (BLAS) for the rebuilt series; same outputs."""
    zb = filt.basis_series_complex(Vh, D * isw, a0, Tn, tlen).astype(np.complex64)
    norm = 4.0 * df / np.sqrt(sig_col)
    As = (A * norm[:, None]).astype(np.complex64)
    nw = Tn // cw
    vw = np.empty((len(A), nw), np.float32)
    iw = np.empty((len(A), nw), np.int64)
    for w0 in range(0, nw, chunk_windows):
        w1 = min(nw, w0 + chunk_windows)
        zt = As @ zb[:, w0 * cw:w1 * cw]
        p = (zt.real ** 2 + zt.imag ** 2).reshape(len(A), w1 - w0, cw)
        j = p.argmax(2)
        iw[:, w0:w1] = j
        vw[:, w0:w1] = np.take_along_axis(p, j[..., None], 2)[..., 0]
    thr2 = (thr * (1 - margin)) ** 2
    tb, wb = np.nonzero(vw > thr2)
    samp = a0 + wb * cw + iw[tb, wb]
    z, pwr, fpk, E = chisq.exact_dense(H, nbins, kmin, kmax, D, IP, df, tlen, tb, samp)
    snr, chi, dof = filt.finalize(z, pwr, norm[tb], np.asarray(nbins)[tb])
    return dict(row=tb, window=wb, sample=samp, approx=np.sqrt(vw[tb, wb]), z=z, pw=pwr, snr=snr, chisq=chi, dof=dof)
