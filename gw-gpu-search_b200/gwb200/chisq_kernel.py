"""Power chi-squared at peaks: drop-in for pipeline/chisq_kernel.py (bin_power_sums, :85-121).

For each peak, Z_j(t) = sum over bin j of q_k exp(2 pi i k t / N); returns sum_j |Z_j|^2 and optionally
z = sum_j Z_j. Fused mode forms q = conj(H) d in registers. Peaks are grouped as the reference groups them (up to 8
peaks of one row per work item, edges taken from the group's row); the sums run in libgwb200 (csrc/chisq.cu)."""
import numpy as np
import torch

from . import _exact, _lib

P = _exact.MAX_PEAKS


def bin_power_sums(q, rows, times, edges_per_peak, want_z=False, d=None, n_time=None):
    """q: (nrows, N) complex64 CUDA tensor (or the template rows H with d (flen,) in fused mode, n_time the time
    length). rows, times: int arrays per peak; edges_per_peak: (npeaks, nedge) bin edges. Returns host arrays in
    input order: pw (float32), and z (complex64) when want_z."""
    _lib.require_cuda(q, d)
    N = q.shape[1] if d is None else n_time
    assert N & (N - 1) == 0, 'N must be a power of two'
    assert q.dtype == torch.complex64 and q.is_contiguous()
    rows = np.asarray(rows)
    times = np.asarray(times)
    E = np.asarray(edges_per_peak)
    npk = len(rows)
    if npk == 0:
        return (np.zeros(0, np.float32), np.zeros(0, np.complex64)) if want_z else np.zeros(0, np.float32)
    order, rows_u, cands, groups, units = _exact.plan(rows, times)
    # edges depend on the row only: take each row's edges from its first peak in sorted order
    first = np.r_[0, np.flatnonzero(np.diff(rows[order])) + 1]
    Eu = E[order[first]].astype(np.int32)
    nb_u = Eu.shape[1] - 1
    # the kernels index nbins by row: give every row the full edge count
    nb_rows = torch.full((int(rows_u.max()) + 1,), nb_u, dtype=torch.int32, device=q.device)
    kmin = int(Eu[:, 0].min())
    kend = int(Eu[:, -1].max())
    units['row'] = rows_u
    E_d = torch.from_numpy(Eu).to(q.device)
    flen = max(kend, kmin + 1)
    pk = _exact.run_sums(cands, groups, units, E_d, nb_u, nb_rows, q, d, kmin, flen, N)
    pw = np.empty(npk, np.float32)
    pw[order] = pk['pw']
    if not want_z:
        return pw
    z = np.empty(npk, np.complex64)
    z[order] = pk['zr'] + 1j * pk['zi']
    return pw, z
