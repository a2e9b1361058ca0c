"""Oracle for the differentiation form (test infrastructure only): the SNR, chi-squared and newSNR of a TaylorF2
template against one trigger's data as float64 numpy functions of theta = (Mc, q, chi1z, chi2z, e0, t_c, phi_c), whose
central finite differences check the CUDA gradients.

Parity unpinned: the reference has no gradients and no TaylorF2 (its templates come from PyCBC). The quantities follow
its definitions: z and sigma^2 as the matched filter's inner products (fp_filter.py:710-714, 837-853), chi-squared
over equal-power bins (multi_filter.py:264-282 with the pipeline's edge rule), newsnr (coinc_rank.py:39-46); the
template is the phase of synth.taylorf2 (3.5PN TaylorF2 with the aligned-spin and eccentric terms)."""
import numpy as np

from . import synth


def masses(mc, q):
    """(m1, m2) from chirp mass and q = m2 / m1 <= 1."""
    eta = q / (1.0 + q) ** 2
    M = mc * eta ** -0.6
    return M / (1.0 + q), q * M / (1.0 + q)


def kmax(mc, q, df, flen):
    m1, m2 = masses(mc, q)
    return int(min(np.floor(synth.f_isco(m1, m2) / df) + 1, flen - 1))


def template(theta, flen, df, kmin, f_ecc=10.0):
    """h_k = f^-7/6 exp(-i (Psi(f) - pi/4 + 2 pi f t_c - phi_c)) on kmin <= k < kmax; complex128 (flen,)."""
    mc, q, c1, c2, e0, tc, phic = theta
    m1, m2 = masses(mc, q)
    k1 = kmax(mc, q, df, flen)
    h = np.zeros(flen, np.complex128)
    f = np.arange(kmin, k1) * df
    ph = synth.taylorf2_phase(f, m1, m2, c1, c2, e0, f_ecc) - np.pi / 4 + 2 * np.pi * f * tc - phic
    h[kmin:k1] = f ** (-7.0 / 6.0) * np.exp(-1j * ph)
    return h, k1


def edges(IP, df, kmin, k1, nb):
    """Equal-power edges of |h|^2 IP = f^-7/3 IP on [kmin, k1): edge j = first k with inclusive cumsum > (j/nb) total."""
    w = (np.arange(kmin, k1) * df) ** (-7.0 / 3.0) * IP[kmin:k1].astype(np.float64)
    cs = np.cumsum(w)
    e = [kmin]
    for j in range(1, nb):
        e.append(kmin + int(np.argmax(cs > j / nb * cs[-1])))
    e.append(k1)
    return np.array(e)


def snr_chisq(theta, D, IP, df, kmin, nb=16, f_ecc=10.0):
    """(snr, chisq, newsnr) in float64 for one trigger."""
    flen = len(D)
    h, k1 = template(theta, flen, df, kmin, f_ecc)
    e = edges(IP, df, kmin, k1, nb)
    q = 4 * df * np.conj(h) * D.astype(np.complex128)
    sig2 = 4 * df * np.sum(np.abs(h) ** 2 * IP.astype(np.float64))
    zj = np.array([q[e[j]:e[j + 1]].sum() for j in range(nb)])
    z = zj.sum()
    snr = abs(z) / np.sqrt(sig2)
    chisq = (nb * np.sum(np.abs(zj) ** 2) - abs(z) ** 2) / sig2
    rc = chisq / (2 * nb - 2)
    ns = snr if rc <= 1 else snr / ((1 + rc ** 3) / 2) ** (1.0 / 6.0)
    return snr, chisq, ns


def fd_grad(theta, D, IP, df, kmin, nb=16, f_ecc=10.0, rel=1e-6):
    """Central differences of (snr, chisq, newsnr) with step rel max(|theta_p|, scale_p) per parameter; (3, 7)."""
    scale = np.array([1.0, 1.0, 1.0, 1.0, 0.1, 1e-3, 1.0])
    th = np.asarray(theta, np.float64)
    g = np.zeros((3, 7))
    for p in range(7):
        hstep = rel * max(abs(th[p]), scale[p])
        a, b = th.copy(), th.copy()
        a[p] += hstep
        b[p] -= hstep
        g[:, p] = (np.array(snr_chisq(a, D, IP, df, kmin, nb, f_ecc)) -
                   np.array(snr_chisq(b, D, IP, df, kmin, nb, f_ecc))) / (2 * hstep)
    return g
