"""Oracle for the compressed filter: SVD metric, template norms, tile SVD, basis series, stacked A, rebuilt z and the
SNR / chi-squared finalisation (test infrastructure only).

Restates the closures of pipeline/fp_filter.py (derive :354-370, svd_tile :576-593, basis_series :597-613,
stacked_A :615-621, rebuilt z :760-764, finalisation :837-853) and newsnr (pipeline/coinc_rank.py:39-46) in numpy.
The reference computes in torch on the GPU with complex64 GEMMs; here the Gram matrix and sigma^2 are float64, the
precision the B200 build uses for them."""
import numpy as np

CH = 1 << 16   # fp_filter.py:42
RB = 64        # fp_filter.py:43


def derive_sw(IPall):
    """fp_filter.py:363-364: sw = sqrt(mean over segments of IP) (float64 mean, cast to float32); isw = 1/sw or 0."""
    sw = np.sqrt(IPall.astype(np.float64).mean(0)).astype(np.float32)
    isw = np.where(sw > 0, 1.0 / np.maximum(sw, np.float32(1e-30)), 0.0).astype(np.float32)
    return sw, isw


def sigma2(H, IPall, df):
    """fp_filter.py:710-714 in float64: sig[i, s] = 4 df sum_k |H_ik|^2 IP_sk; norm = 4 df / sqrt(sig)."""
    P = H.real.astype(np.float64) ** 2 + H.imag.astype(np.float64) ** 2
    sig = (4.0 * df) * (P @ IPall.astype(np.float64).T)
    return sig, (4.0 * df) / np.sqrt(sig)


def gram(H, sw, kmin):
    """G = sum_k (H sw)(H sw)^H over k >= kmin, float64 (fp_filter.py:578-581)."""
    Hw = H[:, kmin:].astype(np.complex128) * sw[kmin:].astype(np.float64)
    return Hw @ Hw.conj().T


def svd_tile(H, sw, kmin, eps):
    """fp_filter.py:576-593 (Gram in float64). Returns r, A (n, r) complex64, Vh (r, flen) complex64, worst lost power,
    and the eigen-decomposition (lam descending, W) for checks."""
    n, flen = H.shape
    G = gram(H, sw, kmin)
    nrm = np.sqrt(np.maximum(G.diagonal().real, 1e-30))
    lam, W = np.linalg.eigh(G / (nrm[:, None] * nrm[None, :]))
    lam, W = np.maximum(lam[::-1], 0), W[:, ::-1]
    worst = (1 - ((np.abs(W) ** 2) * lam[None, :]).cumsum(1)).max(0)
    r = min(int((worst > eps).sum()) + 1, n)
    Wr = W[:, :r]
    s_r = np.sqrt(np.maximum(lam[:r], 1e-12 * lam[0]))
    Bm = (Wr.conj().T / s_r[:, None]) / nrm[None, :]
    Vh = np.zeros((r, flen), np.complex64)
    Vh[:, kmin:] = (Bm @ (H[:, kmin:].astype(np.complex128) * sw[kmin:])).astype(np.complex64)
    A = ((Wr * s_r[None, :]).conj() * nrm[:, None]).astype(np.complex64)
    return r, A, Vh, float(worst[r - 1]), lam, W


def kp_of(r):
    """fp_filter.py:601: K padded to a multiple of 64 for 2 r real rows."""
    return ((2 * r + 63) // 64) * 64


def basis_series_complex(Vh, Dws, a0, Tn, tlen):
    """The complex basis series before scaling: ifft(conj(Vh) Dws zero-padded to tlen, norm='forward')[a0:a0+Tn]
    (fp_filter.py:605-608), complex128."""
    r, flen = Vh.shape
    q = np.zeros((r, tlen), np.complex128)
    q[:, :flen] = np.conj(Vh.astype(np.complex128)) * Dws.astype(np.complex128)
    zb = np.fft.ifft(q, axis=1) * tlen
    return zb[:, a0:a0 + Tn]


def basis_series(Vh, Dws, a0, Tn, tlen, dtype=np.float16):
    """fp_filter.py:597-613. Z (Kp, Tn): rows 0..r-1 real, r..2r-1 imaginary parts divided by scale, the rms of the
    first RB-row batch; returns Z (as dtype) and scale."""
    r = Vh.shape[0]
    zb = basis_series_complex(Vh, Dws, a0, Tn, tlen)
    first = zb[:min(RB, r)]
    scale = float(np.sqrt((first.real ** 2 + first.imag ** 2).mean() / 2))
    Z = np.zeros((kp_of(r), Tn), np.float32)
    Z[:r] = zb.real / scale
    Z[r:2 * r] = zb.imag / scale
    return Z.astype(dtype), scale


def stacked_A(A, nrm_s, scale, Kp, dtype=np.float16):
    """fp_filter.py:615-621: As = A (norm scale); Are = [Re As, -Im As], Aim = [Im As, Re As], zero-padded to Kp."""
    r = A.shape[1]
    As = A.astype(np.complex128) * (np.asarray(nrm_s, np.float64) * scale)[:, None]
    Are = np.zeros((A.shape[0], Kp), np.float32)
    Aim = np.zeros_like(Are)
    Are[:, :r] = As.real
    Are[:, r:2 * r] = -As.imag
    Aim[:, :r] = As.imag
    Aim[:, r:2 * r] = As.real
    return Are.astype(dtype), Aim.astype(dtype)


def rebuilt_z(Are, Aim, Z, rows, cols):
    """fp_filter.py:760-764: the complex SNR the GEMM rebuilt at (row, column), float32 sums."""
    Zs = Z[:, cols].T.astype(np.float32)
    zr = (Are[rows].astype(np.float32) * Zs).sum(1)
    zi = (Aim[rows].astype(np.float32) * Zs).sum(1)
    return (zr + 1j * zi).astype(np.complex64)


def newsnr(snr, rchisq):
    """pipeline/coinc_rank.py:39-46."""
    ns = np.array(snr, dtype=np.float64)
    m = rchisq > 1
    ns[m] = snr[m] / ((1 + rchisq[m] ** 3) / 2.0) ** (1.0 / 6)
    return ns


def finalize(z, pw, norm, nbins):
    """fp_filter.py:837-853: snr = |z| norm; chisq = (nb pw - |z|^2) norm^2; dof = 2 nb - 2."""
    z = np.asarray(z, np.complex128)
    snr = np.abs(z) * norm
    chisq = (nbins * np.asarray(pw, np.float64) - np.abs(z) ** 2) * norm ** 2
    dof = 2 * np.asarray(nbins) - 2
    return snr, chisq, dof
