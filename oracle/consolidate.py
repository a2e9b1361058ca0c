"""Oracle for the downstream consolidation (test infrastructure only): numpy restatements of the reference's
consolidate and pre_keep closures (pipeline/fp_filter.py:629-661 and 663-695), of the peak-file assembly in write_one
(fp_filter.py:910-934), and of the newsnr that fp_filter.py:250 imports from PyCBC (pycbc.events.ranking.newsnr,
PyCBC 2.8.3 as pinned by the reference's environment/requirements.txt:7; not installed here).

Pinned by tests/golden/consolidate.npz: the reference's own consolidate and pre_keep source, run on seeded cases by
tests/golden/make_golden.py with newsnr below standing in for PyCBC's.

Arithmetic follows the reference's types: float32 SNRs compare with Python-float thresholds in float32 (numpy and
torch cast the scalar to the array's type); times, windows and newsnr are float64. Ties in the ranking go to the
earlier position (the reference's sorts are stable); `order` gives that position when the arrays are not already in
the reference's append order."""
import numpy as np


def newsnr(snr, rchisq, q=6.0, n=2.0):
    """PyCBC's re-weighted SNR: snr (0.5 (1 + rchisq^(q/n)))^(-1/q) where rchisq > 1, else snr; float64."""
    ns = np.array(snr, dtype=np.float64, ndmin=1)
    r = np.array(rchisq, dtype=np.float64, ndmin=1)
    m = r > 1.0
    ns[m] *= (0.5 * (1.0 + r[m] ** (q / n))) ** (-1.0 / q)
    return ns


def _gate_ok(t, gates):
    ok = np.ones(len(t), bool)
    for g_t, g_w, g_taper in gates:
        ok &= np.abs(t - g_t) > g_w + g_taper + 0.5
    return ok


def _windows(t, gps_start, sr, interval):
    """Keep-loudest window of each time: trunc(round((t - gps_start) sr) / (interval sr))."""
    ti = np.round((t - gps_start) * sr)
    return (ti / (interval * sr)).astype(np.int64)


def _top(stat, wt, pos, num):
    """Mask of the num first items of each window by (stat descending, pos ascending); and the sorted view."""
    od = np.lexsort((pos, -stat, wt))
    wt_s = wt[od]
    first = np.r_[0, np.nonzero(np.diff(wt_s))[0] + 1] if len(od) else np.zeros(0, np.int64)
    sizes = np.diff(np.r_[first, len(od)])
    rank = np.arange(len(od)) - np.repeat(first, sizes)
    top = np.zeros(len(stat), bool)
    top[od[rank < num]] = True
    return top, od, wt_s, first, sizes


def consolidate(snr, chisq, dof, t, gates, gps_start, sr, newsnr_threshold=None, keep_loudest_interval=None,
                keep_loudest_num=None, exempt_snr=None, use_chisq=True, want_floor=False, order=None):
    """fp_filter.py:629-661: keep mask of one dataset's peaks (t float64 GPS times). Returns (keep, floor), floor the
    keep_loudest_num-th newsnr of every full window (-inf elsewhere; length max window + 1) when want_floor."""
    snr = np.asarray(snr, np.float32)
    n = len(snr)
    ns = newsnr(snr, np.asarray(chisq, np.float32) / np.maximum(np.asarray(dof, np.int32), 1)) if use_chisq else snr
    exempt = snr >= np.float32(exempt_snr) if exempt_snr is not None else np.zeros(n, bool)
    keep = (ns >= (newsnr_threshold or 0)) | exempt
    keep &= _gate_ok(t, gates)
    floor = None
    if keep_loudest_interval:
        idx = np.nonzero(keep & ~exempt)[0]
        wt = _windows(t[idx], gps_start, sr, keep_loudest_interval)
        pos = idx if order is None else np.asarray(order)[idx]
        top, od, wt_s, first, sizes = _top(np.asarray(ns, np.float64)[idx], wt, pos, keep_loudest_num)
        gated = keep.copy()
        keep = np.zeros(n, bool)
        keep[idx[top]] = True
        keep |= gated & exempt
        if want_floor:
            full = sizes >= keep_loudest_num
            floor = np.full(int(wt_s[-1]) + 1 if len(wt_s) else 1, -np.inf)
            floor[wt_s[first[full]]] = np.asarray(ns, np.float64)[idx[od[first[full] + keep_loudest_num - 1]]]
    return keep, floor


def pre_keep(ti, apx, gates, gps_start, sr, exact_snr, margin, thr, exempt_snr=None, newsnr_threshold=None,
             keep_loudest_interval=None, keep_loudest_num=None, floor=None, order=None):
    """fp_filter.py:663-695: mask over one part's candidates (ti: samples since the dataset's start, apx float32
    rebuilt SNRs). Exact candidates (apx >= exact_snr (1 - margin)) are all kept; the rest pass the newsnr cut (newsnr
    of a rebuilt peak = its SNR), the gate veto, the floor and the keep-loudest ranking."""
    apx = np.asarray(apx, np.float32)
    n = len(apx)
    ex = apx >= np.float32(exact_snr * (1 - margin))
    ok = ~ex & (apx > np.float32(thr))
    t = gps_start + np.asarray(ti, np.int64).astype(np.float64) / sr
    exempt = ok & (apx >= np.float32(exempt_snr)) if exempt_snr is not None else np.zeros(n, bool)
    ok &= (apx >= np.float32(newsnr_threshold or 0)) | exempt
    ok &= _gate_ok(t, gates)
    idx = np.nonzero(ok & ~exempt)[0]
    if keep_loudest_interval and len(idx):
        wt = _windows(t[idx], gps_start, sr, keep_loudest_interval)
        if floor is not None:
            fl = np.asarray(floor, np.float64)
            bar = np.where(wt < len(fl), fl[np.minimum(wt, len(fl) - 1)], -np.inf)
            above = apx[idx].astype(np.float64) > bar
            ok[idx[~above]] = False
            idx, wt = idx[above], wt[above]
        pos = idx if order is None else np.asarray(order)[idx]
        top, *_ = _top(apx[idx].astype(np.float64), wt, pos, keep_loudest_num)
        t_ok = np.zeros(n, bool)
        t_ok[idx[top]] = True
        ok = t_ok | (ok & exempt)
    return ex | ok


def peak_table(tid, t, snr, phase, peak_sigmasq, exact, chisq, dof, gates, sigmasq, hashes=None):
    """write_one's datasets (fp_filter.py:910-934) as a dict: the gate veto once more, then rows sorted by (template
    id, time); newsnr from snr and chisq / max(dof, 1)."""
    tid = np.asarray(tid, np.int64)
    keep = _gate_ok(t, gates)
    srt = np.lexsort((t[keep], tid[keep]))
    sel = np.nonzero(keep)[0][srt]
    chi, dof_ = np.asarray(chisq, np.float32)[sel], np.asarray(dof, np.int32)[sel]
    gt = np.array(gates, np.float64).reshape(-1, 3)
    out = {'template_id': tid[sel], 'snr': np.asarray(snr)[sel], 'end_time': np.asarray(t, np.float64)[sel],
           'sigmasq': sigmasq, 'coa_phase': np.asarray(phase, np.float32)[sel],
           'peak_sigmasq': np.asarray(peak_sigmasq, np.float64)[sel], 'exact': np.asarray(exact, bool)[sel],
           'chisq': chi, 'chisq_dof': dof_, 'newsnr': newsnr(np.asarray(snr)[sel], chi / np.maximum(dof_, 1)),
           'gates/time': gt[:, 0], 'gates/width': gt[:, 1], 'gates/taper': gt[:, 2]}
    if hashes is not None:
        out['template_hash'] = np.asarray(hashes)[tid[sel]]
    return out
