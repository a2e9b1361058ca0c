"""Host-side planning and kernel runners shared by the chi-squared / exact-stage drop-ins.

Record layouts match the C structs of include/gwb200.h (GwbCand, GwbGroup, GwbUnit, GwbPeak). The planning follows
the reference's: peaks sorted by (row, sample), cut into items of at most 8 peaks of one row (exact_stage._plan,
pipeline/exact_stage.py:221-233; chisq_kernel.bin_power_sums, pipeline/chisq_kernel.py:96-107)."""
import numpy as np
import torch

from . import _lib

MAX_PEAKS = 8

CAND = np.dtype([('row', '<i4'), ('seg', '<i4'), ('sample', '<i4'), ('window', '<i4'), ('approx', '<f4'),
                 ('zr', '<f4'), ('zi', '<f4'), ('unit', '<i4')])
GROUP = np.dtype([('unit', '<i4'), ('first', '<i4'), ('count', '<i4'), ('pad', '<i4')])
UNIT = np.dtype([('row', '<i4'), ('seg', '<i4'), ('first', '<i4'), ('count', '<i4')])
PEAK = np.dtype([('zr', '<f4'), ('zi', '<f4'), ('pw', '<f4'), ('snr', '<f4'), ('chisq', '<f4'), ('newsnr', '<f4'),
                 ('fpeak', '<f4'), ('dof', '<i4')])


def to_dev(rec, device='cuda'):
    """A numpy record array as a flat byte tensor on the device."""
    b = torch.from_numpy(np.ascontiguousarray(rec).view(np.uint8).reshape(-1).copy())
    return b.to(device)


def from_dev(t, dtype, n):
    return t[:n * dtype.itemsize].cpu().numpy().view(dtype)


def plan(rows, samples, seg=0):
    """Sort peaks by (row, sample) and group them: returns (order, rows_u, cands, groups, units) where cands are in
    sorted order, units are the distinct rows (ascending), and groups cut each row's run into items of <= 8."""
    rows = np.asarray(rows, np.int64)
    samples = np.asarray(samples, np.int64)
    order = np.lexsort((samples, rows))
    rs, ss = rows[order], samples[order]
    rows_u, peak_u = np.unique(rs, return_inverse=True)
    n = len(rs)
    cands = np.zeros(n, CAND)
    cands['row'] = rs
    cands['seg'] = seg
    cands['sample'] = ss
    cands['unit'] = peak_u
    units = np.zeros(len(rows_u), UNIT)
    units['row'] = rows_u
    units['seg'] = seg
    if n:
        run_end = np.r_[np.flatnonzero(np.diff(rs)) + 1, n]
        run_start = np.r_[0, run_end[:-1]]
        units['first'] = run_start
        units['count'] = run_end - run_start
        g = []
        for u, (a, b) in enumerate(zip(run_start, run_end)):
            for f in range(a, b, MAX_PEAKS):
                g.append((u, f, min(MAX_PEAKS, b - f), 0))
        groups = np.array(g, GROUP)
    else:
        groups = np.zeros(0, GROUP)
    return order, rows_u, cands, groups, units


def run_edges(units, H, IP, nbins_row, kmax_row, kmin, B, offset_mode):
    """Edges for each unit: (len(units), B + 1) int32 device tensor. nbins_row, kmax_row: int32 device arrays indexed
    by the units' row field; IP (nseg, flen) indexed by the seg field."""
    nu = len(units)
    E = torch.empty((max(nu, 1), B + 1), dtype=torch.int32, device=H.device)
    if nu == 0:
        return E[:0]
    ud = to_dev(units, H.device)
    _lib.call('gwb_edges', _lib.ptr(ud), None, nu, _lib.ptr(H), H.stride(0), _lib.ptr(IP), IP.stride(0),
              _lib.ptr(nbins_row), _lib.ptr(kmax_row), int(kmin), int(B), int(offset_mode), _lib.ptr(E),
              _lib.stream_ptr(H.device))
    return E


def run_sums(cands, groups, units, E, B, nbins_row, H, D, kmin, flen, tlen, sig=None, df=1.0):
    """Binned sums and finalisation; returns the GwbPeak records (host), in the order of cands."""
    nc = len(cands)
    if nc == 0:
        return np.zeros(0, PEAK)
    dev = H.device
    nchunk = _lib.load().gwb_exact_chunks(int(flen), int(kmin))
    slots = torch.zeros((nc, nchunk, B, 2), dtype=torch.float32, device=dev)
    cd, gd, ud = to_dev(cands, dev), to_dev(groups, dev), to_dev(units, dev)
    s = _lib.stream_ptr(dev)
    _lib.call('gwb_bin_sums', _lib.ptr(gd), None, len(groups), _lib.ptr(ud), _lib.ptr(cd), _lib.ptr(E), int(B),
              _lib.ptr(nbins_row), _lib.ptr(H), H.stride(0), _lib.ptr(D), 0 if D is None else D.stride(0) if D.dim() > 1
              else D.shape[0], int(kmin), int(flen), int(tlen), _lib.ptr(slots), s)
    out = torch.empty(nc * PEAK.itemsize, dtype=torch.uint8, device=dev)
    _lib.call('gwb_exact_finalize', _lib.ptr(cd), None, nc, _lib.ptr(ud), _lib.ptr(E), int(B), _lib.ptr(nbins_row),
              int(kmin), int(flen), _lib.ptr(slots), _lib.ptr(sig), 0 if sig is None else sig.stride(0), float(df),
              _lib.ptr(out), s)
    return from_dev(out, PEAK, nc)
