"""Oracle for the chi-squared bin edges, the power chi-squared at peaks and the dense exact stage (test infrastructure
only).

edges_per_template restates pipeline/multi_filter.py:264-282 (float64 cumulative |h|^2 IP, first k whose normalised
cumsum exceeds j/nb, clipped to [kmin, k1], padded with k1). bin_sums is the float64 definition the reference's
kernels are tested against (tests/test_chisq_kernel_gpu.py:17-23, exact_stage._dense_sums_numpy :425-439):
Z_j(t) = sum_{k in bin j} conj(h_k) D_k exp(2 pi i ((k t) mod N) / N), z = sum_j Z_j, pw = sum_j |Z_j|^2.
exact_dense follows ExactStage.evaluate for the dense tile (exact_stage.py:173-191, _plan :221-233,
_fpeak :236-238)."""
import numpy as np


def edges_per_template(rows, nb_, kmin, k1, Hd, ips):
    """multi_filter.py:264-282. rows: per-peak row index into Hd; nb_, k1 per peak. Returns int64 (npk, B + 1)."""
    rows = np.asarray(rows)
    nb_ = np.asarray(nb_)
    k1 = np.asarray(k1)
    ur, inv = np.unique(rows, return_inverse=True)
    B = int(nb_.max())
    h = Hd[ur]
    cs = np.cumsum((h.real.astype(np.float64) ** 2 + h.imag.astype(np.float64) ** 2) * ips[None, :].astype(np.float64),
                   axis=1)
    k1u = k1[np.unique(inv, return_index=True)[1]]
    tot = cs[np.arange(len(ur)), k1u - 1]
    F = cs.shape[1]
    flat = (cs / tot[:, None] + np.arange(len(ur), dtype=np.float64)[:, None]).ravel()
    j = np.arange(B)[None, :]
    target = inv[:, None] + j / nb_[:, None]
    e = np.searchsorted(flat, target.ravel(), side='right').reshape(target.shape) - inv[:, None] * F
    e = np.clip(e, kmin, k1[:, None])
    e = np.where(j < nb_[:, None], e, k1[:, None])
    return np.concatenate([e, k1[:, None]], axis=1)


def bin_sums(q_row, t, e, N):
    """Z_j for one peak: q_row (complex, indexed by k), sample t, edges e (nb + 1), time length N. float64."""
    k = np.arange(e[0], e[-1], dtype=np.int64)
    x = q_row[e[0]:e[-1]].astype(np.complex128) * np.exp(2j * np.pi * ((k * int(t)) % N) / N)
    b = np.searchsorted(e, k, side='right') - 1
    nb = len(e) - 1
    return np.bincount(b, x.real, nb) + 1j * np.bincount(b, x.imag, nb)


def bin_power_sums(q, rows, times, edges, want_z=False, d=None, n_time=None):
    """chisq_kernel.bin_power_sums semantics (chisq_kernel.py:85-121) in float64: q (nrows, N) complex, or the
    template rows H with d (fused mode, q = conj(H) d). Returns pw (and z) in input order."""
    N = q.shape[1] if d is None else n_time
    pw = np.empty(len(rows))
    z = np.empty(len(rows), np.complex128)
    for i, (r, t) in enumerate(zip(rows, times)):
        row = q[r] if d is None else np.conj(q[r].astype(np.complex128)) * d.astype(np.complex128)
        Zj = bin_sums(row, t, np.asarray(edges[i]), N)
        pw[i] = (np.abs(Zj) ** 2).sum()
        z[i] = Zj.sum()
    return (pw, z) if want_z else pw


def fpeak(E, nb, df):
    """exact_stage.py:236-238: sine-Gaussian reference frequency (2 e[nb-1] - e[nb-2]) df."""
    r = np.arange(len(E))
    return (2 * E[r, np.maximum(nb - 1, 0)] - E[r, np.maximum(nb - 2, 0)]) * df


def exact_dense(H, nbins, kmin, kmax, D, IP, df, tlen, rows, samples):
    """ExactStage(TemplateTile(H, nbins, kmin, kmax)).evaluate(SegmentData(D, IP, df, tlen), PeakRequest(rows,
    samples)) on the dense path: returns z (complex128), pw (float64), fpeak, edges per peak."""
    rows = np.asarray(rows, np.int64)
    samples = np.asarray(samples, np.int64)
    if len(rows) == 0:
        return np.zeros(0, np.complex128), np.zeros(0), np.zeros(0), np.zeros((0, 2), np.int64)
    nbins = np.asarray(nbins, np.int64)
    kmax = np.asarray(kmax, np.int64)
    ru = np.unique(rows)
    nbe = np.maximum(nbins[ru], 1)
    E = np.asarray(edges_per_template(ru, nbe, kmin, kmax[ru], H, IP), np.int64)
    E[nbins[ru] == 0, 0] = kmin
    u = np.searchsorted(ru, rows)
    Ep = E[u]
    z = np.empty(len(rows), np.complex128)
    pw = np.empty(len(rows))
    for i in range(len(rows)):
        e = Ep[i, :nbe[u[i]] + 1]
        row = np.conj(H[rows[i]].astype(np.complex128)) * D.astype(np.complex128)
        Zj = bin_sums(row, samples[i], e, tlen)
        z[i] = Zj.sum()
        pw[i] = (np.abs(Zj) ** 2).sum()
    return z, pw, fpeak(Ep, nbins[rows], df), Ep
