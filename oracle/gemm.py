"""Oracle for the reconstruction GEMM, window reduction and window peaks (test infrastructure only).

gemm_absmax follows pipeline/fp_gemm.py:14-33 (Triton gemm_absmax): acc_r = Are @ Z, acc_i = Aim @ Z with fp32
accumulation, pw = acc_r^2 + acc_i^2, columns >= Tn set to -1, max and first argmax per BN = 128 columns.
window_reduce follows pipeline/fp_filter.py:745-747 (V.view(n, nw, cw/BN).max(2), gather of I, threshold).
window_peaks follows pipeline/peak_kernel.py:10-36 (max |z|^2 per window, first offset on ties)."""
import numpy as np

BN = 128


def gemm_absmax(Are, Aim, Z, M, Tn, bn=BN):
    """Returns V (M, nblk) float32 and I (M, nblk) int32. Inputs of any float dtype; products summed in float32
    (float64 would differ from the fp32 kernels only below float32 resolution)."""
    Are = np.asarray(Are, np.float32)[:M]
    Aim = np.asarray(Aim, np.float32)[:M]
    Z = np.asarray(Z, np.float32)[:, :Tn]
    nblk = -(-Tn // bn)
    zr = Are @ Z
    zi = Aim @ Z
    pw = zr * zr + zi * zi
    pad = nblk * bn - Tn
    if pad:
        pw = np.concatenate([pw, np.full((M, pad), -1.0, np.float32)], axis=1)
    pw = pw.reshape(M, nblk, bn)
    I = pw.argmax(axis=2).astype(np.int64)
    V = np.take_along_axis(pw, I[..., None], 2)[..., 0]
    I = I + np.arange(nblk)[None, :] * bn
    return V.astype(np.float32), I.astype(np.int32)


def group_reduce(V, I, group):
    """Reduce `group` consecutive blocks per output: max and the first block's index on ties (torch.max(dim))."""
    M, nblk = V.shape
    nout = -(-nblk // group)
    pad = nout * group - nblk
    Vp = np.concatenate([V, np.full((M, pad), -np.inf, np.float32)], 1) if pad else V
    Ip = np.concatenate([I, np.zeros((M, pad), I.dtype)], 1) if pad else I
    j = Vp.reshape(M, nout, group).argmax(2)
    return (np.take_along_axis(Vp.reshape(M, nout, group), j[..., None], 2)[..., 0],
            np.take_along_axis(Ip.reshape(M, nout, group), j[..., None], 2)[..., 0])


def window_reduce(V, I, n, nw, cw, thr2):
    """fp_filter.py:745-747: per-window max over cw/BN blocks, its sample, and the candidates above thr2 = (thr(1-m))^2.
    Returns vw (n, nw), iw (n, nw), (tb, wb) candidate (row, window) pairs in row-major order."""
    g = cw // BN
    vw = V[:, :nw * g].reshape(n, nw, g)
    jj = vw.argmax(2)
    iw = np.take_along_axis(I[:, :nw * g].reshape(n, nw, g), jj[..., None], 2)[..., 0]
    vw = np.take_along_axis(vw, jj[..., None], 2)[..., 0]
    tb, wb = np.nonzero(vw > thr2)
    return vw, iw, tb, wb


def window_peaks(z, a0, cw, nwin):
    """z (rows, N) complex64 -> (pmax float32, pidx int32), each (rows, nwin)."""
    z = np.asarray(z, np.complex64)
    seg = z[:, a0:a0 + nwin * cw].reshape(z.shape[0], nwin, cw)
    p = seg.real * seg.real + seg.imag * seg.imag
    idx = p.argmax(axis=2)
    return np.take_along_axis(p, idx[..., None], 2)[..., 0].astype(np.float32), idx.astype(np.int32)
