"""Consolidation of peaks on the device and the peak-file records (the downstream step after the exact stage).

The reference consolidates each dataset's peaks on the host after every tile (consolidate, pipeline/fp_filter.py:
629-661: gate veto, newsnr cut with SNR-exempt peaks, keep the keep_loudest_num loudest by newsnr per
keep_loudest_interval window, ties to the earlier peak) and pre-filters rebuilt candidates on the GPU (pre_keep,
:663-695). Here both run in csrc/consolidate.cu (gwb_consolidate); `PeakStore` keeps one dataset's peaks on the
device and consolidates them as they arrive, and `peak_table` / `write_peaks` give write_one's datasets
(fp_filter.py:910-934)."""
import numpy as np
import torch

from . import _lib


def _nwin(ti, interval, sr, n_samples):
    if n_samples is None:
        n_samples = int(ti.max().item()) + 1 if ti.numel() else 1
    return int(np.floor(n_samples / (interval * sr))) + 2


def _gates_dev(gates, device):
    g = np.array([tuple(map(float, x)) for x in gates], np.float64).reshape(-1, 3)
    return torch.from_numpy(g).to(device), len(g)


def _run(mode, snr, chisq, dof, ti, order, use_chisq, gps_start, sr, exact_cut, thr, newsnr_threshold, exempt_snr,
         gates, keep_loudest_interval, keep_loudest_num, floor_in, want_floor, n_samples, check):
    _lib.require_cuda(snr, ti)
    dev = snr.device
    n = snr.numel()
    assert snr.dtype == torch.float32 and ti.dtype == torch.int64 and snr.is_contiguous() and ti.is_contiguous()
    if mode == 0 and use_chisq:
        assert chisq.dtype == torch.float32 and dof.dtype == torch.int32
    if order is not None:
        assert order.dtype == torch.int64 and order.is_contiguous()
    interval = float(keep_loudest_interval or 0.0)
    nwin = _nwin(ti, interval, sr, n_samples) if interval > 0 else 0
    g, ng = _gates_dev(gates, dev)
    wb = _lib.load().gwb_consolidate_work_bytes(n, nwin)
    work = torch.empty(max(wb, 16), dtype=torch.uint8, device=dev)
    keep = torch.empty(n, dtype=torch.uint8, device=dev)
    status = torch.empty(1, dtype=torch.int32, device=dev)
    floor = torch.empty(nwin, dtype=torch.float64, device=dev) if (want_floor and interval > 0) else None
    fl_in = floor_in.contiguous() if floor_in is not None else None
    _lib.call('gwb_consolidate', mode, n, _lib.ptr(snr), _lib.ptr(chisq), _lib.ptr(dof), _lib.ptr(ti),
              _lib.ptr(order), 1 if use_chisq else 0, float(gps_start), float(sr), float(exact_cut), float(thr),
              float(newsnr_threshold or 0.0), 0 if exempt_snr is None else 1,
              float(exempt_snr if exempt_snr is not None else 0.0), _lib.ptr(g), ng, interval,
              int(keep_loudest_num or 0), _lib.ptr(fl_in), 0 if fl_in is None else fl_in.numel(), _lib.ptr(floor), nwin,
              _lib.ptr(work), work.numel(), _lib.ptr(keep), _lib.ptr(status), _lib.stream_ptr())
    if check and int(status.item()):
        raise _lib.GwbError('gwb_consolidate', _lib.GWB_ERR_CAPACITY, 'a peak lies outside the %d windows' % nwin)
    return keep.bool(), floor


def consolidate(snr, chisq, dof, ti, gates, gps_start, sr, newsnr_threshold=None, keep_loudest_interval=None,
                keep_loudest_num=None, exempt_snr=None, use_chisq=True, order=None, want_floor=False,
                n_samples=None, check=True):
    """Keep mask (bool CUDA tensor) of one dataset's peaks by the reference's consolidate. snr, chisq float32, dof
    int32, ti int64 (samples since the dataset's start: the peak time is gps_start + ti / sr), gates a list of
    (gps, width, taper). order: int64 keys giving the reference's append order (ties go to the smaller key); None =
    the array order. Returns (keep, floor): floor (float64, one per window) when want_floor, else None."""
    return _run(0, snr, chisq, dof, ti, order, use_chisq, gps_start, sr, 0.0, 0.0, newsnr_threshold, exempt_snr,
                gates, keep_loudest_interval, keep_loudest_num, None, want_floor, n_samples, check)


def pre_keep(ti, apx, gates, gps_start, sr, exact_snr, margin, thr, exempt_snr=None, newsnr_threshold=None,
             keep_loudest_interval=None, keep_loudest_num=None, floor=None, order=None, n_samples=None, check=True):
    """Mask (bool CUDA tensor) over one part's candidates by the reference's pre_keep: apx float32 rebuilt SNRs,
    ti int64 samples since the dataset's start. Candidates with apx >= exact_snr (1 - margin) are kept; the others
    that consolidate would drop are not."""
    cut = np.float32(exact_snr * (1 - margin))
    return _run(1, apx, None, None, ti, order, False, gps_start, sr, cut, np.float32(thr), newsnr_threshold,
                exempt_snr, gates, keep_loudest_interval, keep_loudest_num, floor, False, n_samples, check)[0]


def newsnr(snr, rchisq):
    """PyCBC's newsnr (float64 numpy), for the records: snr (0.5 (1 + r^3))^(-1/6) where r > 1."""
    ns = np.array(snr, dtype=np.float64, ndmin=1)
    r = np.array(rchisq, dtype=np.float64, ndmin=1)
    m = r > 1.0
    ns[m] *= (0.5 * (1.0 + r[m] ** 3.0)) ** (-1.0 / 6.0)
    return ns


FIELDS = ('tid', 'ti', 'snr', 'phase', 'peak_sigmasq', 'exact', 'chisq', 'dof', 'order')


class PeakStore:
    """One dataset's peaks on the device (tid, ti, snr, phase, peak_sigmasq, exact, chisq, dof and the order key),
    consolidated after every add as the reference does after every tile: the loudest of a union are among the loudest
    of its parts, so the result equals one consolidation of everything (ties by order key)."""

    def __init__(self, gps_start, sr, n_samples, gates=(), newsnr_threshold=None, keep_loudest_interval=None,
                 keep_loudest_num=None, exempt_snr=None, use_chisq=True, device='cuda'):
        self.gps_start, self.sr, self.n_samples = gps_start, sr, n_samples
        self.gates = list(gates)
        self.kw = dict(newsnr_threshold=newsnr_threshold, keep_loudest_interval=keep_loudest_interval,
                       keep_loudest_num=keep_loudest_num, exempt_snr=exempt_snr, use_chisq=use_chisq)
        self.device = device
        self.d = None
        self.n_in = 0

    def add(self, **part):
        n = part['snr'].numel()
        self.n_in += n
        if self.d is None:
            self.d = {k: part[k] for k in FIELDS}
        else:
            self.d = {k: torch.cat([self.d[k], part[k]]) for k in FIELDS}
        d = self.d
        keep, _ = consolidate(d['snr'].contiguous(), d['chisq'].contiguous(), d['dof'].contiguous(),
                              d['ti'].contiguous(), self.gates, self.gps_start, self.sr, order=d['order'].contiguous(),
                              n_samples=self.n_samples, **self.kw)
        self.d = {k: v[keep] for k, v in d.items()}

    def __len__(self):
        return 0 if self.d is None else self.d['snr'].numel()

    def host(self):
        if self.d is None:
            return {k: np.zeros(0) for k in FIELDS}
        return {k: v.cpu().numpy() for k, v in self.d.items()}


def peak_table(h, gates, gps_start, sr, sigmasq=None, hashes=None):
    """write_one's datasets (fp_filter.py:910-934) from a PeakStore's host arrays: the gate veto, rows sorted by
    (template id, end time), newsnr from snr and chisq / max(dof, 1), the gates."""
    t = gps_start + np.asarray(h['ti'], np.int64) / sr
    tid = np.asarray(h['tid'], np.int64)
    keep = np.ones(len(t), bool)
    for g_t, g_w, g_taper in gates:
        keep &= np.abs(t - g_t) > g_w + g_taper + 0.5
    sel = np.nonzero(keep)[0][np.lexsort((t[keep], tid[keep]))]
    chi = np.asarray(h['chisq'], np.float32)[sel]
    dof = np.asarray(h['dof'], np.int32)[sel]
    snr = np.asarray(h['snr'], np.float32)[sel]
    gt = np.array([tuple(map(float, x)) for x in gates], np.float64).reshape(-1, 3)
    out = {'template_id': tid[sel], 'snr': snr, 'end_time': t[sel],
           'coa_phase': np.asarray(h['phase'], np.float32)[sel],
           'peak_sigmasq': np.asarray(h['peak_sigmasq'], np.float64)[sel], 'exact': np.asarray(h['exact'], bool)[sel],
           'chisq': chi, 'chisq_dof': dof, 'newsnr': newsnr(snr, chi / np.maximum(dof, 1)),
           'gates/time': gt[:, 0], 'gates/width': gt[:, 1], 'gates/taper': gt[:, 2]}
    if sigmasq is not None:
        out['sigmasq'] = sigmasq
    if hashes is not None:
        out['template_hash'] = np.asarray(hashes)[tid[sel]]
    return out


def write_peaks(path, table, attrs=None):
    """One peak file: HDF5 (the reference's layout, gzip + shuffle above 1000 elements) when h5py is importable,
    else a numpy .npz with the same dataset names."""
    try:
        import h5py
    except ImportError:
        h5py = None
    if h5py is None:
        np.savez(path if path.endswith('.npz') else path + '.npz', **table)
        return
    with h5py.File(path, 'w') as f:
        for k, v in table.items():
            v = np.asarray(v)
            f.create_dataset(k, data=v, **(dict(compression='gzip', compression_opts=4, shuffle=True)
                                           if v.size > 1000 else {}))
        f.attrs['n_gates'] = len(table.get('gates/time', ()))
        for k, v in (attrs or {}).items():
            f.attrs[k] = v
