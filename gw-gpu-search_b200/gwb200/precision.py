"""Precision of the filter's arithmetic forms against float64 on one (tile, segment): the window maxima of the SNR
that the fused GEMM of a form produces, against the same maxima of a float64 SNR series.

The float64 series follows the reference's math without rounding: the basis series zb = ifft(conj(Vh) D isw) over
the analysed span (fp_filter.py:597-613, norm='forward', zero-padded half spectrum), z = A zb (the product the
stacked GEMM forms, fp_filter.py:615-621, fp_gemm.py:14-33) and snr = |z| 4 df / sqrt(sigma^2) (fp_filter.py:710-714).
Windows are the filter's cluster windows over the analysed span; the index is the first maximum, as the GEMM's.
"""
import numpy as np
import torch

from . import fp_filter


def fp64_window_snr(sv, D_seg, isw, sig_col, df, tlen, a0, Tn, cw, batch=32):
    """float64 window maxima (n, nw) of the SNR of one tile against one segment, and their samples (relative to a0).
    sv: the tile's SVD entry (A (n, r), Vh (r, flen)); D_seg (flen,) complex64; isw (flen,); sig_col (n,) float64."""
    dev = D_seg.device
    Vh = sv['Vh'].to(torch.complex128)
    A = sv['A'].to(torch.complex128)
    r, flen = Vh.shape
    n = A.shape[0]
    dw = D_seg.to(torch.complex128) * isw.to(torch.float64)
    zb = torch.empty((r, Tn), dtype=torch.complex128, device=dev)
    for j0 in range(0, r, batch):
        j1 = min(r, j0 + batch)
        q = torch.zeros((j1 - j0, tlen), dtype=torch.complex128, device=dev)
        q[:, :flen] = torch.conj(Vh[j0:j1]) * dw
        zb[j0:j1] = torch.fft.ifft(q, norm='forward')[:, a0:a0 + Tn]
        del q
    z = A @ zb
    del zb
    norm = 4.0 * df / torch.sqrt(sig_col.to(torch.float64))
    snr = z.abs() * norm[:, None]
    del z
    nw = Tn // cw
    v, i = snr[:, :nw * cw].reshape(n, nw, cw).max(2)
    i = i + torch.arange(nw, device=dev)[None, :] * cw
    return v.cpu().numpy(), i.cpu().numpy()


def form_window_snr(mf, t, D, isw, sig, seg):
    """Window maxima of the SNR (n, nw) and their samples from the fused GEMM of mf's form, for tile t against
    segment seg (rows of D). Resets mf's candidate counters (the diagnostic call's candidates are not kept)."""
    if mf.fused:
        mf.Dp = fp_filter.fourstep_order(D, mf.tlen, isw)
    mf.counters.zero_()
    mf.tile_segment(t, D, isw, sig, seg)
    torch.cuda.synchronize()
    mf.counters.zero_()
    n = len(mf.bank.tiles[t])
    v = mf.V[:n].double().clamp_min(0).sqrt().cpu().numpy()
    return v, mf.I[:n].cpu().numpy().astype(np.int64)


def compare(v, i, v64, i64, thr):
    """Differences of one form's window maxima from float64's: |delta SNR| (max, median), relative (max, median),
    argmax agreement (exact, and within 2 samples: the series is smooth, so a 16-bit form may pick a neighbour of
    an almost equal maximum), and the windows above thr in one but not the other (all, and those more than 1e-3 thr
    away from the threshold in float64)."""
    d = np.abs(v - v64)
    rel = d / np.maximum(v64, 1e-30)
    above, above64 = v > thr, v64 > thr
    flip = above ^ above64
    return dict(max_abs_dsnr=float(d.max()), median_abs_dsnr=float(np.median(d)), max_rel=float(rel.max()),
                median_rel=float(np.median(rel)), argmax_agree=float(np.mean(i == i64)),
                argmax_within2=float(np.mean(np.abs(i - i64) <= 2)), windows=int(v.size),
                above_fp64=int(above64.sum()), set_diff=int(flip.sum()),
                set_diff_away=int((flip & (np.abs(v64 - thr) > 1e-3 * thr)).sum()))
