"""Oracle for strain conditioning: PSD estimate, interpolation, inverse spectrum truncation, autogating, segments,
D = stilde / psd and IP = 1 / psd (test infrastructure only).

A numpy restatement of pipeline/gpu_prep.py (itself PyCBC's conditioning step for step), function by function, with
the same precisions and scale factors. GPS times are carried as integer nanoseconds where the reference uses
lal.LIGOTimeGPS (gpu_prep.py:178, 208-209, 214-226)."""
import numpy as np

DYN_RANGE_FAC = 5.9029581035870565e+20   # gpu_prep.py:21


def median_bias(n):
    """gpu_prep.py:47-53."""
    if n >= 1000:
        return np.log(2)
    b = 1.0
    for i in range(1, (n - 1) // 2 + 1):
        b += 1.0 / (2 * i + 1) - 1.0 / (2 * i)
    return b


def welch_segments(n, seg_len, seg_stride, num_segments=None):
    """Segment count and start of the used span (gpu_prep.py:92-101)."""
    if num_segments is None:
        num_segments = int(n // seg_stride)
        if (num_segments - 1) * seg_stride + seg_len > n:
            num_segments -= 1
    used = (num_segments - 1) * seg_stride + seg_len
    start = 0
    if used < n:
        d = n - used
        start = d // 2 + (d % 2)
    assert used <= n
    return num_segments, start


def welch(x, seg_len, seg_stride, dt, num_segments=None, avg='median'):
    """gpu_prep.py:87-125: Hann-windowed periodograms (float32 FFT products), median / bias (or mean), PyCBC scale
    2 df L / sum(w^2). x: (n,) or (rows, n) float32. Returns (psd, delta_f)."""
    single = x.ndim == 1
    X = x[None] if single else x
    n = X.shape[1]
    nseg, start = welch_segments(n, seg_len, seg_stride, num_segments)
    X = X[:, start:start + (nseg - 1) * seg_stride + seg_len]
    w = np.hanning(seg_len).astype(X.dtype)
    idx = (np.arange(nseg) * seg_stride)[:, None] + np.arange(seg_len)[None, :]
    ctype = np.complex64 if X.dtype == np.float32 else np.complex128
    out = []
    for row in X:
        st = (np.fft.rfft(row[idx] * w, axis=1) * X.dtype.type(dt)).astype(ctype)
        p = (st.real * st.real + st.imag * st.imag).astype(X.dtype)
        p[:, 0] /= 2
        p[:, -1] /= 2
        if avg == 'median':
            b = median_bias(nseg)
            q = np.median(p, axis=0)
            q = q.astype(np.float64) / float(b) if isinstance(b, np.floating) else q / b
        else:
            q = np.mean(p, axis=0)
        out.append(q)
    df = 1.0 / dt / seg_len
    fac = 2 * df * seg_len / (w * w).sum()
    res = (np.stack(out) * (float(fac) if out[0].dtype == np.float64 else fac)).astype(X.dtype)
    return (res[0] if single else res), df


def interpolate(psd, df_old, df_new, length=None):
    """gpu_prep.py:128-135: np.interp in float64 onto k df_new, cast back."""
    new_n = (psd.shape[-1] - 1) * df_old / df_new + 1 if length is None else length
    fs = np.arange(0, np.rint(new_n)) * df_new
    fo = np.arange(psd.shape[-1]) * df_old
    P = psd[None] if psd.ndim == 1 else psd
    out = np.stack([np.interp(fs, fo, r.astype(np.float64)) for r in P]).astype(psd.dtype)
    return out[0] if psd.ndim == 1 else out


def inverse_spectrum_truncation(psd, df, max_filter_len, low_frequency_cutoff, trunc_method=None):
    """gpu_prep.py:138-158: 1/sqrt(psd) -> irfft (times df) -> keep max_filter_len/2 taps at each end (optional Hann)
    -> rfft / (df N) -> 1 / |.|^2."""
    P = psd[None] if psd.ndim == 1 else psd
    flen = P.shape[1]
    N = (flen - 1) * 2
    ctype = np.complex64 if P.dtype == np.float32 else np.complex128
    kmin = int(low_frequency_cutoff / df) if low_frequency_cutoff else 1
    inv = np.zeros(P.shape, ctype)
    inv[:, kmin:N // 2] = (1.0 / P[:, kmin:N // 2]) ** 0.5
    q = np.fft.irfft(inv, n=N, axis=1, norm='forward').astype(P.dtype) * P.dtype.type(df)
    ts, te = max_filter_len // 2, N - max_filter_len // 2
    if trunc_method == 'hann':
        tw = np.hanning(max_filter_len).astype(P.dtype)
        q[:, 0:ts] *= tw[-ts:]
        q[:, te:N] *= tw[0:max_filter_len // 2]
    if ts < te:
        q[:, ts:te] = 0
    pt = np.fft.rfft(q, axis=1).astype(ctype) * P.dtype.type(1.0 / (df * N))
    out = (1.0 / np.abs(pt * pt.conj())).astype(P.dtype)
    return out[0] if psd.ndim == 1 else out


def cluster_over_window(idx, vals, window):
    """gpu_prep.py:161-172 (findchirp cluster): keep the loudest of samples closer than window to the kept one."""
    if len(idx) == 0:
        return np.zeros(0, dtype=int)
    keep = [0]
    for i in range(1, len(idx)):
        if idx[i] < idx[keep[-1]] + window:
            if vals[i] > vals[keep[-1]]:
                keep[-1] = i
        else:
            keep.append(i)
    return np.array(keep)


def _ns(t):
    """float seconds (or int) -> integer nanoseconds, rounded as LIGOTimeGPS does from a float."""
    return int(round(float(t) * 1e9))


def whitened_magnitude(strain, sr, low_freq_cutoff, corrupt_time, psd_duration=4., psd_stride=2.):
    """The whitened |x| that detect_loud_glitches thresholds (gpu_prep.py:179-202)."""
    dt = 1.0 / sr
    s = strain.copy()
    n = len(s)
    cl = int(corrupt_time * sr)
    w = (np.arange(cl) / float(cl)).astype(s.dtype)
    s[0:cl] *= w
    s[n - cl:] *= w[::-1]
    L = 1 << n.bit_length()
    pad_start = int(L / 2 - n / 2)
    sp = np.zeros(L, dtype=s.dtype)
    sp[pad_start:pad_start + n] = s
    psd, pdf = welch(s[cl:n - cl], int(psd_duration * sr), int(psd_stride * sr), dt)
    df = 1. / (L * dt)
    psd = interpolate(psd, pdf, df)
    psd = inverse_spectrum_truncation(psd, df, int(psd_duration * sr), low_freq_cutoff, 'hann')
    psd[0:int(low_freq_cutoff / df)] = np.inf
    norm = sr / 2. - low_freq_cutoff
    ct = np.complex64 if s.dtype == np.float32 else np.complex128
    st = np.fft.rfft(sp).astype(ct) * s.dtype.type(dt)
    st *= (psd * norm) ** (-0.5)
    wt = np.fft.irfft(st, n=L, norm='forward').astype(s.dtype) * s.dtype.type(df)
    mag = np.abs(wt[pad_start:pad_start + n])
    mag[0:cl] = 0
    mag[n - cl:] = 0
    return mag


def detect_loud_glitches(strain, sr, start_gps, threshold, cluster_window, low_freq_cutoff, corrupt_time,
                         psd_duration=4., psd_stride=2.):
    """gpu_prep.py:175-209. Returns the glitch times as integer GPS nanoseconds."""
    mag = whitened_magnitude(strain, sr, low_freq_cutoff, corrupt_time, psd_duration, psd_stride)
    ind = np.nonzero(mag > threshold)[0]
    keep = cluster_over_window(ind.astype(np.int32), mag[ind], int(cluster_window * sr))
    t0 = _ns(start_gps)
    r = int(sr)
    # i / sr seconds to the nearest nanosecond, halves rounded up (a float offset added to a GPS time)
    return [t0 + (2 * int(i) * 1000000000 + r) // (2 * r) for i in ind[keep]]


def gate_window(sr, gw, pw):
    """The inverted-Tukey gate of gpu_prep.py:222-225: cos tapers of pw s around 2 (gw + pw) s, zeros inside."""
    win_samples = int(2 * sr * (gw + pw))
    pad_samples = int(sr * pw)
    pad = 0.5 * (1. + np.cos(np.pi * np.arange(pad_samples) / pad_samples))
    return np.concatenate((pad, np.zeros(win_samples - 2 * pad_samples), pad[::-1]))


def gate_taper(x, sr, start_gps_ns, gates):
    """gpu_prep.py:212-231, in place. gates: (time_ns, width s, taper s); offsets in integer nanoseconds (sr an
    integer rate)."""
    duration_ns = int(round(len(x) / sr * 1e9))
    for gt, gw, pw in gates:
        half = int(round((gw + pw) * 1e9))
        t_start = gt - half - start_gps_ns
        t_end = gt + half - start_gps_ns
        if t_start > duration_ns or t_end < 0:
            continue
        window = gate_window(sr, gw, pw)
        offset = (t_start * int(sr)) // 1000000000        # floor, as int() of a normalised GPS time
        i1, i2 = max(0, -offset), min(len(window), len(x) - offset)
        sl = slice(i1 + offset, i2 + offset)
        x[sl] = (x[sl].astype(np.float64) * window[i1:i2]).astype(x.dtype)
    return x


def segment_slices(n, sr, start_gps, seg_len, start_pad, end_pad, trig_start=0, trig_end=0):
    """gpu_prep.py:234-271 (PyCBC StrainSegments index arithmetic)."""
    end_gps = start_gps + n / sr
    if not trig_start:
        trig_start = int(start_gps) + start_pad
    if not trig_end:
        trig_end = int(end_gps) - end_pad
    seg_width = seg_len - start_pad - end_pad
    analyzable = trig_end - trig_start
    data_start = (trig_start - start_pad) - int(start_gps)
    data_end = trig_end + end_pad - int(start_gps)
    data_dur = data_end - data_start
    data_start, data_end = data_start * sr, data_end * sr
    num_segs = int(np.ceil(float(analyzable) / float(seg_width)))
    seg_offset = int(np.ceil(analyzable / float(num_segs)))
    segs, anas = [], []
    for k in range(num_segs - 1):
        s0 = int(data_start + (k * seg_offset) * sr)
        segs.append((s0, int(s0 + seg_len * sr)))
        a0 = int(start_pad * sr)
        anas.append((a0, int(a0 + seg_offset * sr)))
    s1 = int(data_end)
    segs.append((int(s1 - seg_len * sr), s1))
    remaining = data_dur - ((num_segs - 1) * seg_offset + start_pad)
    anas.append((int((seg_len - remaining) * sr), int((seg_len - end_pad) * sr)))
    ts_i = (trig_start - int(start_gps)) * sr
    te_i = (trig_end - int(start_gps)) * sr
    out = []
    for (s0, s1), (a0, a1) in zip(segs, anas):
        if ts_i > a0 + s0:
            a0 += ts_i - (a0 + s0)
        if te_i < a1 + s0:
            a1 -= (a1 + s0) - te_i
        if a0 < a1:
            assert s0 >= 0 and s1 <= n
            out.append(((s0, s1), (a0, a1)))
    return out


def overlapping_psd_spans(n, seg_len, seg_stride, num_segments):
    """gpu_prep.py:274-282."""
    psd_len = (num_segments - 1) * seg_stride + seg_len
    assert n >= psd_len
    if n == psd_len:
        return [(0, n)]
    m = int(2 * (n - 1) / psd_len)
    stride = int((n - psd_len) / m)
    return [(n - psd_len, n) if i == m - 1 else (stride * i, psd_len + stride * i) for i in range(m)]


def pick_psd(seg, spans):
    """Largest overlap, first wins ties (gpu_prep.py:439-446)."""
    pick = []
    for (a, b), _ in seg:
        best, ov = None, 0
        for j, (c, e) in enumerate(spans):
            o = min(b, e) - max(a, c)
            if o > 0 and o > ov:
                best, ov = j, o
        pick.append(best)
    return pick


def stage2(s, sr, gps_start, seg_len_s, start_pad, end_pad, flow, psd_seg_len, psd_seg_stride, psd_num_segments,
           psd_inverse_length, trunc_method=None, avg='median', trig_start=0, trig_end=0):
    """gpu_stage2 (gpu_prep.py:405-454) on a float32 strain s with the padding already removed."""
    n = len(s)
    seg = segment_slices(n, sr, gps_start, seg_len_s, start_pad, end_pad, trig_start, trig_end)
    tlen = int(seg_len_s * sr)
    flen = tlen // 2 + 1
    df = 1.0 / seg_len_s
    idx = np.array([a for (a, _), _ in seg])[:, None] + np.arange(tlen)[None, :]
    stilde = np.fft.rfft(s[idx], axis=1).astype(np.complex64) * np.float32(1.0 / sr)
    pl, ps = int(psd_seg_len * sr), int(psd_seg_stride * sr)
    spans = overlapping_psd_spans(n, pl, ps, psd_num_segments)
    parts = np.stack([s[a:b] for a, b in spans])
    psd, pdf = welch(parts, int(psd_seg_len * sr + 0.5), int(psd_seg_stride * sr + 0.5), 1.0 / sr,
                     num_segments=psd_num_segments, avg=avg)
    if pdf != df:
        psd = interpolate(psd, pdf, df, flen)
    if psd_inverse_length:
        psd = inverse_spectrum_truncation(psd, df, int(psd_inverse_length * sr), flow, trunc_method)
    psd = psd.astype(np.float32)
    pick = pick_psd(seg, spans)
    P = psd[np.array(pick)].astype(np.float64)
    kmin = int(flow / df)
    ip = np.where(P > 0, 1.0 / np.where(P > 0, P, 1.0), 0.0)
    ip[:, :kmin] = 0
    D = (stilde * ip).astype(np.complex64)
    return dict(D=D, IP=ip.astype(np.float32), flen=flen, tlen=tlen, df=df, sr=float(sr),
                analyze=[a for _, a in seg], seg_start=[s0 for (s0, _), _ in seg], psd=psd, pick=pick)
