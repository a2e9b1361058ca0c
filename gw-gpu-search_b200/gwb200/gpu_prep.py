"""Strain conditioning on the B200: drop-in for pipeline/gpu_prep.py (PyCBC's conditioning step for step).

Same function names, arguments and results as the reference. `xp` is accepted for call compatibility; arrays are
torch CUDA tensors here (numpy inputs are copied to the device), and every transform and streaming step runs in
libgwb200 (cuFFT plus the kernels of csrc/prep.cu). Host-side logic that the reference also runs on the host stays
in Python: argument parsing, segment index arithmetic, clustering of glitch samples and GPS-time arithmetic (integer
nanoseconds here, where the reference uses lal.LIGOTimeGPS).

Not provided: the store read and the two lal IIR highpasses (cpu_stage1 / cpu_stage2, gpu_prep.py:314-334, 396-402)
and the ldas resampler (:67-84); calls to them raise NotImplementedError. Synthetic inputs are generated at the
analysis sample rate already high-passed, so the path starts at gpu_stage1's DYN_RANGE_FAC scaling."""
import argparse
import time

import numpy as np
import torch

from . import _lib

DYN_RANGE_FAC = 5.9029581035870565e+20      # pipeline/gpu_prep.py:21


def parser():
    """The reference's option parser (gpu_prep.py:24-44), same options and refusals."""
    p = argparse.ArgumentParser(add_help=False)
    a = p.add_argument
    a('--hdf-store'); a('--channel-name'); a('--gps-start-time', type=int); a('--gps-end-time', type=int)
    a('--pad-data', type=int, default=0); a('--strain-high-pass', type=float); a('--sample-rate', type=float)
    a('--low-frequency-cutoff', type=float); a('--segment-length', type=int)
    a('--segment-start-pad', type=int); a('--segment-end-pad', type=int)
    a('--trig-start-time', type=int, default=0); a('--trig-end-time', type=int, default=0)
    a('--psd-estimation'); a('--psd-segment-length', type=float); a('--psd-segment-stride', type=float)
    a('--psd-num-segments', type=int); a('--psd-inverse-length', type=float); a('--invpsd-trunc-method')
    a('--autogating-threshold', type=float); a('--autogating-cluster', type=float, default=5.0)
    a('--autogating-width', type=float, default=0.25); a('--autogating-taper', type=float, default=0.25)
    a('--autogating-pad', type=float, default=16); a('--autogating-max-iterations', type=int, default=1)
    a('--gating-method', default='taper')
    a('--injection-file'); a('--injection-scale-factor', type=float, default=1); a('--injection-sample-rate', type=float)
    for k in ('--gating-file', '--zpk-z', '--normalize-strain', '--strain-low-pass', '--taper-data', '--witness-frame-type',
              '--sgburst-injection-file', '--psd-model', '--psd-file', '--asd-file', '--fake-strain', '--filter-inj-only',
              '--allow-zero-padding', '--frame-files', '--frame-cache', '--frame-type'):
        a(k, dest='unsupported_' + k[2:].replace('-', '_'))
    return p


def options(argv):
    opt, _ = parser().parse_known_args(argv)
    bad = [k for k, v in vars(opt).items() if k.startswith('unsupported_') and v]
    assert not bad, f'gpu_prep does not implement {bad}'
    assert opt.psd_estimation in ('median', 'mean') and opt.gating_method == 'taper'
    return opt


def median_bias(n):
    """PyCBC's median bias (gpu_prep.py:47-53)."""
    if n >= 1000:
        return np.log(2)
    ans = 1
    for i in range(1, (n - 1) // 2 + 1):
        ans += 1.0 / (2 * i + 1) - 1.0 / (2 * i)
    return ans


class GPS:
    """A GPS time in integer nanoseconds (stands in for lal.LIGOTimeGPS in the gating arithmetic)."""
    __slots__ = ('ns',)

    def __init__(self, t=0, ns=None):
        if ns is not None:
            self.ns = int(ns)
        elif isinstance(t, GPS):
            self.ns = t.ns
        elif isinstance(t, (int, np.integer)):
            self.ns = int(t) * 1000000000
        else:
            self.ns = int(np.floor(float(t) * 1e9 + 0.5))

    def __float__(self):
        return self.ns / 1e9

    def __repr__(self):
        return 'GPS(%d.%09d)' % divmod(self.ns, 1000000000)

    def __eq__(self, o):
        return isinstance(o, GPS) and o.ns == self.ns

    def __hash__(self):
        return hash(self.ns)


def _dev(x, dtype=None):
    if isinstance(x, torch.Tensor):
        t = x if x.is_cuda else x.cuda()
    else:
        t = torch.as_tensor(np.asarray(x)).cuda()
    if dtype is not None and t.dtype != dtype:
        t = t.to(dtype)
    return t.contiguous()


def _s():
    return _lib.stream_ptr()


def _rfft_rows(x, n):
    """Batched real FFT of the rows of x (rows, n) float32 -> (rows, n/2 + 1) complex64."""
    rows = x.shape[0]
    out = torch.empty((rows, n // 2 + 1), dtype=torch.complex64, device=x.device)
    _lib.call('gwb_fft_r2c', _lib.handle(), _lib.ptr(x), _lib.ptr(out), n, rows, x.stride(0), out.stride(0), _s())
    return out


def _irfft_rows(X, n):
    """Unnormalised inverse real FFT of rows of X (rows, n/2 + 1) -> (rows, n) float32. X is consumed."""
    rows = X.shape[0]
    out = torch.empty((rows, n), dtype=torch.float32, device=X.device)
    _lib.call('gwb_fft_c2r', _lib.handle(), _lib.ptr(X), _lib.ptr(out), n, rows, X.stride(0), out.stride(0), _s())
    return out


def _welch_layout(n, seg_len, seg_stride, num_segments):
    if num_segments is None:
        num_segments = int(n // seg_stride)
        if (num_segments - 1) * seg_stride + seg_len > n:
            num_segments -= 1
    data_len = (num_segments - 1) * seg_stride + seg_len
    start = 0
    if data_len < n:
        diff = n - data_len
        start = diff // 2 + (diff % 2)
    assert data_len <= n, 'Incorrect choice of segmentation parameters'
    return num_segments, start


def welch(xp, x, seg_len, seg_stride, dt, num_segments=None, avg='median'):
    """pycbc.psd.welch (Hann window), for one series or a batch of rows (gpu_prep.py:87-125). float32 input."""
    x = _dev(x, torch.float32)
    single = x.dim() == 1
    X = x[None] if single else x
    n = X.shape[1]
    nseg, start = _welch_layout(n, seg_len, seg_stride, num_segments)
    w = np.hanning(seg_len).astype(np.float32)
    frames = torch.empty((X.shape[0] * nseg, seg_len), dtype=torch.float32, device=X.device)
    _lib.call('gwb_frames', _lib.ptr(X), X.stride(0), X.shape[0], start, int(seg_stride), None, nseg, seg_len,
              _lib.ptr(_dev(w)), _lib.ptr(frames), frames.stride(0), _s())
    F = _rfft_rows(frames, seg_len)
    nbin = seg_len // 2 + 1
    delta_f = 1. / dt / seg_len
    fac = np.float32(2 * delta_f * seg_len / (w * w).sum())
    out = torch.empty((X.shape[0], nbin), dtype=torch.float32, device=X.device)
    b = median_bias(nseg)
    _lib.call('gwb_welch_avg', _lib.ptr(F), F.stride(0), X.shape[0], nseg, nbin, float(np.float32(dt)),
              int(avg == 'median'), float(b), float(fac), _lib.ptr(out), out.stride(0), _s())
    return (out[0] if single else out), delta_f


def interpolate(xp, psd, df_old, df_new, length=None):
    """pycbc.psd.interpolate: np.interp in float64, cast back (gpu_prep.py:128-135)."""
    psd = _dev(psd, torch.float32)
    P = psd[None] if psd.dim() == 1 else psd
    new_n = (P.shape[-1] - 1) * df_old / df_new + 1 if length is None else length
    nnew = int(np.rint(new_n))
    out = torch.empty((P.shape[0], nnew), dtype=torch.float32, device=P.device)
    _lib.call('gwb_interp', _lib.ptr(P), P.stride(0), P.shape[0], P.shape[1], float(df_old), float(df_new), nnew,
              _lib.ptr(out), out.stride(0), _s())
    return out[0] if psd.dim() == 1 else out


def inverse_spectrum_truncation(xp, psd, df, max_filter_len, low_frequency_cutoff, trunc_method=None):
    """pycbc.psd.inverse_spectrum_truncation (gpu_prep.py:138-158), float32 rows."""
    psd = _dev(psd, torch.float32)
    P = psd[None] if psd.dim() == 1 else psd
    rows, flen = P.shape
    N = (flen - 1) * 2
    kmin = int(low_frequency_cutoff / df) if low_frequency_cutoff else 1
    inv = torch.empty((rows, flen), dtype=torch.complex64, device=P.device)
    _lib.call('gwb_ist_pre', _lib.ptr(P), P.stride(0), rows, flen, kmin, _lib.ptr(inv), inv.stride(0), _s())
    q = _irfft_rows(inv, N)
    tw = None
    if trunc_method == 'hann':
        tw = _dev(np.hanning(max_filter_len).astype(np.float32))
    _lib.call('gwb_ist_mid', _lib.ptr(q), q.stride(0), rows, N, float(np.float32(df)), int(max_filter_len),
              _lib.ptr(tw), _s())
    pt = _rfft_rows(q, N)
    out = torch.empty((rows, flen), dtype=torch.float32, device=P.device)
    _lib.call('gwb_ist_post', _lib.ptr(pt), pt.stride(0), rows, flen, float(np.float32(1.0 / (df * N))), _lib.ptr(out),
              out.stride(0), _s())
    return out[0] if psd.dim() == 1 else out


def cluster_over_window(idx, vals, window):
    """pycbc.events.findchirp_cluster_over_window (gpu_prep.py:161-172); host loop, as in the reference."""
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


def whitened_above(strain, sr, threshold, low_freq_cutoff, corrupt_time, psd_duration=4., psd_stride=2., cap=1 << 20):
    """The device part of detect_loud_glitches: indices (sorted) and values of whitened |x| > threshold."""
    return above_collect(*whitened_above_queue(strain, sr, threshold, low_freq_cutoff, corrupt_time, psd_duration,
                                               psd_stride, cap))


def above_collect(idx, val, cnt, tapered, cap):
    """Host side of whitened_above_queue's result (synchronises on its count): sorted indices, values, tapered."""
    c = int(cnt.item())
    if c > cap:
        raise _lib.GwbError('gwb_above', _lib.GWB_ERR_CAPACITY, '%d samples above threshold, capacity %d' % (c, cap))
    ih, vh = idx[:c].cpu().numpy(), val[:c].cpu().numpy()
    o = np.argsort(ih, kind='stable')
    return ih[o], vh[o], tapered


def whitened_above_queue(strain, sr, threshold, low_freq_cutoff, corrupt_time, psd_duration=4., psd_stride=2.,
                         cap=1 << 20):
    """whitened_above's device work, queued without a host synchronisation: returns (idx, val, cnt, tapered, cap)
    device tensors for above_collect (so many segments can be queued before one synchronisation)."""
    s = _dev(strain, torch.float32)
    dt = 1.0 / sr
    n = s.shape[0]
    cl = int(corrupt_time * sr)
    L = 1 << n.bit_length()
    pad_start = int(L / 2 - n / 2)
    tapered = torch.empty_like(s)
    sp = torch.empty((1, L), dtype=torch.float32, device=s.device)
    _lib.call('gwb_taper_pad', _lib.ptr(s), n, cl, L, pad_start, _lib.ptr(tapered), _lib.ptr(sp), _s())
    psd, pdf = welch(None, s[cl:n - cl], int(psd_duration * sr), int(psd_stride * sr), dt)
    df = 1. / (L * dt)
    psd = interpolate(None, psd, pdf, df)
    psd = inverse_spectrum_truncation(None, psd, df, int(psd_duration * sr), low_freq_cutoff, 'hann')
    psd[0:int(low_freq_cutoff / df)] = float('inf')
    norm = sr / 2. - low_freq_cutoff
    st = _rfft_rows(sp, L)
    _lib.call('gwb_whiten', _lib.ptr(st), st.shape[1], _lib.ptr(psd), float(np.float32(dt)), float(np.float32(norm)),
              _s())
    wt = _irfft_rows(st, L)
    idx = torch.empty(cap, dtype=torch.int32, device=s.device)
    val = torch.empty(cap, dtype=torch.float32, device=s.device)
    cnt = torch.zeros(1, dtype=torch.int32, device=s.device)
    _lib.call('gwb_above', _lib.ptr(wt), pad_start, n, cl, float(np.float32(df)), float(threshold), _lib.ptr(idx),
              _lib.ptr(val), cap, _lib.ptr(cnt), _s())
    return idx, val, cnt, tapered, cap


def detect_loud_glitches(xp, strain, sr, start_gps, threshold, cluster_window, low_freq_cutoff, corrupt_time,
                         psd_duration=4., psd_stride=2.):
    """pycbc.strain.detect_loud_glitches (gpu_prep.py:175-209). Returns GPS times (integer nanoseconds)."""
    ind, v, _ = whitened_above(strain, sr, threshold, low_freq_cutoff, corrupt_time, psd_duration, psd_stride)
    return glitch_times(ind, v, sr, start_gps, cluster_window)


def glitch_times(ind, v, sr, start_gps, cluster_window):
    """The host end of detect_loud_glitches (gpu_prep.py:199-209): clustering over the window, GPS times."""
    keep = cluster_over_window(ind.astype(np.int32), v, int(cluster_window * sr))
    t0 = GPS(start_gps)
    r = int(sr)
    return [GPS(ns=t0.ns + (2 * int(i) * 1000000000 + r) // (2 * r)) for i in ind[keep]]


def gate_table(n, sr, start_gps, gates):
    """Host GPS arithmetic of gate_taper (gpu_prep.py:217-227): per applied gate (offset, window samples, taper
    samples, i1, i2), in nanoseconds, with int() of a GPS time taken as the floor."""
    t0 = GPS(start_gps).ns
    duration_ns = int(round(n / sr * 1e9))
    rows = []
    for gt, gw, pw in gates:
        g = GPS(gt).ns
        half = int(round((gw + pw) * 1e9))
        t_start, t_end = g - half - t0, g + half - t0
        if t_start > duration_ns or t_end < 0:
            continue
        win = int(2 * sr * (gw + pw))
        pad = int(sr * pw)
        off = (t_start * int(sr)) // 1000000000
        i1, i2 = max(0, -off), min(win, n - off)
        rows.append((off, win, pad, i1, i2))
    return np.array(rows, np.int64).reshape(-1, 5)


def gate_taper(xp, x, sr, start_gps, gates):
    """pycbc.strain.gate_data (inverted Tukey), in place on a float32 CUDA tensor (gpu_prep.py:212-231)."""
    _lib.require_cuda(x)
    tab = gate_table(x.shape[0], sr, start_gps, gates)
    if len(tab):
        g = _dev(tab)
        _lib.call('gwb_apply_gates', _lib.ptr(x), x.shape[0], _lib.ptr(g), len(tab), _s())
    return x


def segment_slices(n, sr, start_gps, seg_len, start_pad, end_pad, trig_start, trig_end):
    """pycbc.strain.StrainSegments index arithmetic (gpu_prep.py:234-271); host."""
    end_gps = start_gps + n / sr
    if not trig_start:
        trig_start = int(start_gps) + start_pad
    if not trig_end:
        trig_end = int(end_gps) - end_pad
    assert trig_start >= int(start_gps) + start_pad and trig_end <= int(end_gps) - end_pad
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
            assert s0 >= 0 and s1 <= n, 'segment outside the data needs zero padding (not supported)'
            out.append(((s0, s1), (a0, a1)))
    return out


def overlapping_psd_spans(n, seg_len, seg_stride, num_segments):
    """pycbc.psd.generate_overlapping_psds spans (gpu_prep.py:274-282); host."""
    psd_len = (num_segments - 1) * seg_stride + seg_len
    assert n >= psd_len
    if n == psd_len:
        return [(0, n)]
    m = int(2 * (n - 1) / psd_len)
    stride = int((n - psd_len) / m)
    return [(n - psd_len, n) if i == m - 1 else (stride * i, psd_len + stride * i) for i in range(m)]


class _Laps:
    """Per-stage seconds with a device sync at each lap (gpu_prep.py:296-303)."""

    def __init__(self):
        self.T, self.t = {}, time.perf_counter()

    def __call__(self, k):
        torch.cuda.synchronize()
        self.T[k] = round(time.perf_counter() - self.t, 4)
        self.t = time.perf_counter()


def highpass_cpu(*a, **k):
    raise NotImplementedError('the lal IIR highpass (pipeline/gpu_prep.py:56-64) is outside this library')


def resample_ldas(*a, **k):
    raise NotImplementedError('the ldas FIR resampler (pipeline/gpu_prep.py:67-84) is outside this library')


def cpu_stage1(argv):
    raise NotImplementedError('store read and IIR highpass (pipeline/gpu_prep.py:314-334) are outside this library')


def cpu_stage2(h, argv):
    raise NotImplementedError('the second IIR highpass (pipeline/gpu_prep.py:396-402) is outside this library')


def gpu_stage1(xp, x, argv, inj=None):
    """x DYN_RANGE_FAC to float32, injections, autogating (gpu_prep.py:362-393). x must already be at the analysis
    sample rate (the ldas resampler is not provided). Returns (gated float32 strain, gates, timing)."""
    L = _Laps()
    opt = options(argv)
    t0 = opt.gps_start_time - opt.pad_data
    sr = opt.sample_rate
    sr0 = len(x) / (opt.gps_end_time - opt.gps_start_time + 2 * opt.pad_data)
    if int(round(sr0 / sr)) != 1:
        resample_ldas()
    xg = _dev(x, torch.float64)
    if inj is not None:
        xg = xg + _dev(inj, torch.float64)
        L('injections')
    s = (xg * DYN_RANGE_FAC).to(torch.float32)
    del xg
    gates = []
    if opt.autogating_threshold is not None:
        for _ in range(opt.autogating_max_iterations):
            gt = detect_loud_glitches(xp, s, sr, t0, opt.autogating_threshold, opt.autogating_cluster,
                                      opt.strain_high_pass, opt.pad_data + opt.autogating_pad)
            gp = [(g_, opt.autogating_width, opt.autogating_taper) for g_ in gt]
            gates += gp
            gate_taper(xp, s, sr, t0, gp)
            if not gt:
                break
    L('autogating')
    return s, [(float(g), w, tp) for g, w, tp in gates], L.T


def gpu_stage2(xp, h, argv):
    """Remove padding, segment FFTs, overlapping PSDs, interpolation, truncation, D and IP (gpu_prep.py:405-454).
    Returns dict(D, IP as CUDA tensors, flen, tlen, df, sr, gps_start, analyze, seg_start, timing)."""
    L = _Laps()
    opt = options(argv)
    sr, pad = opt.sample_rate, opt.pad_data
    s = _dev(h, torch.float32)
    if pad:
        s = s[int(pad * sr):int(len(s) - sr * pad)].contiguous()
    n = len(s)
    gps_start = opt.gps_start_time
    seg = segment_slices(n, sr, gps_start, opt.segment_length, opt.segment_start_pad, opt.segment_end_pad,
                         opt.trig_start_time, opt.trig_end_time)
    tlen = int(opt.segment_length * sr)
    flen = tlen // 2 + 1
    df = 1.0 / opt.segment_length
    starts = _dev(np.array([a for (a, _), _ in seg], np.int64))
    frames = torch.empty((len(seg), tlen), dtype=torch.float32, device=s.device)
    _lib.call('gwb_frames', _lib.ptr(s[None]), n, 1, 0, 0, _lib.ptr(starts), len(seg), tlen, None, _lib.ptr(frames),
              tlen, _s())
    stilde = _rfft_rows(frames, tlen)
    del frames
    L('segment_fft')
    pl, ps = int(opt.psd_segment_length * sr), int(opt.psd_segment_stride * sr)
    spans = overlapping_psd_spans(n, pl, ps, opt.psd_num_segments)
    parts = torch.stack([s[a:b] for a, b in spans])
    psd, pdf = welch(xp, parts, int(opt.psd_segment_length * sr + 0.5), int(opt.psd_segment_stride * sr + 0.5),
                     1.0 / sr, num_segments=opt.psd_num_segments, avg=opt.psd_estimation)
    del parts
    if pdf != df:
        psd = interpolate(xp, psd, pdf, df, flen)
    L('psd_welch')
    if opt.psd_inverse_length:
        psd = inverse_spectrum_truncation(xp, psd, df, int(opt.psd_inverse_length * sr), opt.low_frequency_cutoff,
                                          opt.invpsd_trunc_method)
    L('psd_truncation')
    pick = []
    for (a, b), _ in seg:
        best, ov = None, 0
        for j, (c, e) in enumerate(spans):
            o = min(b, e) - max(a, c)
            if o > 0 and o > ov:
                best, ov = j, o
        pick.append(best)
    kmin = int(opt.low_frequency_cutoff / df)
    D = torch.empty((len(seg), flen), dtype=torch.complex64, device=s.device)
    IP = torch.empty((len(seg), flen), dtype=torch.float32, device=s.device)
    _lib.call('gwb_d_ip', _lib.ptr(stilde), stilde.stride(0), len(seg), _lib.ptr(psd), psd.stride(0),
              _lib.ptr(_dev(np.array(pick, np.int32))), flen, kmin, float(np.float32(1.0 / sr)), _lib.ptr(D),
              D.stride(0), _lib.ptr(IP), IP.stride(0), _s())
    L('output')
    return dict(D=D, IP=IP, flen=flen, tlen=tlen, df=df, sr=float(sr), gps_start=float(gps_start),
                analyze=[a for _, a in seg], seg_start=[s0 for (s0, _), _ in seg], timing=L.T)


def prep(argv, xp, inj=None, strain=None):
    """Condition one dataset (gpu_prep.py:457-470). The store read and highpasses are outside this library, so the
    (already high-passed, analysis-rate) strain must be given; stage 1 and stage 2 then run on the device."""
    if strain is None:
        cpu_stage1(argv)
    s, gates, T1 = gpu_stage1(xp, strain, argv, inj)
    out = gpu_stage2(xp, s, argv)
    out['gates'] = gates
    out['timing'] = {**T1, **out['timing']}
    return out


class BatchConditioner:
    """gpu_stage2 for many datasets of equal length that each hold exactly one analysis segment and one PSD span
    (a dataset as long as the segment and the Welch span, as the synthetic 512 s chunks are), batched: one set of
    transforms and kernels for every dataset at once. Output rows are the datasets' D and IP (gpu_prep.py:405-454).
    Buffers are allocated once for the batch shape, so repeated calls allocate nothing and can be graph-captured."""

    def __init__(self, nds, n, sr, flow, psd_seg_len, psd_seg_stride, psd_num_segments, psd_inverse_length,
                 trunc_method=None, avg='median', device='cuda'):
        self.nds, self.n, self.sr, self.flow = nds, n, sr, flow
        self.tlen = n
        self.flen = n // 2 + 1
        self.df = sr / n
        self.kmin = int(flow / self.df)
        self.L = int(psd_seg_len * sr + 0.5)
        self.stride = int(psd_seg_stride * sr + 0.5)
        nseg, start = _welch_layout(n, self.L, self.stride, psd_num_segments)
        assert start == 0 and (nseg - 1) * self.stride + self.L == n, 'one PSD span per dataset'
        self.nfr = nseg
        self.median = avg == 'median'
        self.bias = median_bias(nseg)
        w = np.hanning(self.L).astype(np.float32)
        self.w = torch.from_numpy(w).to(device)
        # the Welch scale 2 / (dt sum w^2) with dt = 1 / sr, the window's float values squared and summed in double
        # (gwb_filter_batch forms the same number)
        self.fac = float(np.float32(2.0 * sr / np.sum(w.astype(np.float64) ** 2)))
        self.pdf = 1. / (1. / sr) / self.L
        self.mfl = int(psd_inverse_length * sr) if psd_inverse_length else 0
        self.tw = torch.from_numpy(np.hanning(self.mfl).astype(np.float32)).to(device) if trunc_method == 'hann' else None
        nb = self.L // 2 + 1
        self.frames = torch.empty((nds * nseg, self.L), dtype=torch.float32, device=device)
        self.F = torch.empty((nds * nseg, nb), dtype=torch.complex64, device=device)
        self.psd_w = torch.empty((nds, nb), dtype=torch.float32, device=device)
        self.psd = torch.empty((nds, self.flen), dtype=torch.float32, device=device)
        self.inv = torch.empty((nds, self.flen), dtype=torch.complex64, device=device)
        self.q = torch.empty((nds, n), dtype=torch.float32, device=device)
        self.pt = torch.empty((nds, self.flen), dtype=torch.complex64, device=device)
        self.st = torch.empty((nds, self.flen), dtype=torch.complex64, device=device)
        self.pick = torch.arange(nds, dtype=torch.int32, device=device)
        self.D = torch.empty((nds, self.flen), dtype=torch.complex64, device=device)
        self.IP = torch.empty((nds, self.flen), dtype=torch.float32, device=device)
        self.launches = 0

    def __call__(self, x):
        """x: (nds, n) float32 strain (DYN_RANGE_FAC units). Returns (D, IP), each (nds, flen)."""
        assert tuple(x.shape) == (self.nds, self.n) and x.dtype == torch.float32 and x.is_contiguous()
        h, s = _lib.handle(), _s()
        nds, n, L, flen = self.nds, self.n, self.L, self.flen
        _lib.call('gwb_frames', _lib.ptr(x), n, nds, 0, self.stride, None, self.nfr, L, _lib.ptr(self.w),
                  _lib.ptr(self.frames), L, s)
        _lib.call('gwb_fft_r2c', h, _lib.ptr(self.frames), _lib.ptr(self.F), L, nds * self.nfr, L, self.F.stride(0), s)
        _lib.call('gwb_welch_avg', _lib.ptr(self.F), self.F.stride(0), nds, self.nfr, L // 2 + 1,
                  float(np.float32(1.0 / self.sr)), int(self.median), float(self.bias), self.fac, _lib.ptr(self.psd_w),
                  self.psd_w.stride(0), s)
        _lib.call('gwb_interp', _lib.ptr(self.psd_w), self.psd_w.stride(0), nds, L // 2 + 1, float(self.pdf),
                  float(self.df), flen, _lib.ptr(self.psd), flen, s)
        self.launches += 3          # this library's kernels; the transforms are cuFFT's
        P = self.psd
        if self.mfl:
            _lib.call('gwb_ist_pre', _lib.ptr(self.psd), flen, nds, flen, self.kmin, _lib.ptr(self.inv), flen, s)
            _lib.call('gwb_fft_c2r', h, _lib.ptr(self.inv), _lib.ptr(self.q), n, nds, flen, n, s)
            _lib.call('gwb_ist_mid', _lib.ptr(self.q), n, nds, n, float(np.float32(self.df)), self.mfl,
                      _lib.ptr(self.tw), s)
            _lib.call('gwb_fft_r2c', h, _lib.ptr(self.q), _lib.ptr(self.pt), n, nds, n, flen, s)
            _lib.call('gwb_ist_post', _lib.ptr(self.pt), flen, nds, flen, float(np.float32(1.0 / (self.df * n))),
                      _lib.ptr(self.psd), flen, s)
            self.launches += 3
        _lib.call('gwb_fft_r2c', h, _lib.ptr(x), _lib.ptr(self.st), n, nds, n, flen, s)
        _lib.call('gwb_d_ip', _lib.ptr(self.st), flen, nds, _lib.ptr(P), flen, _lib.ptr(self.pick), flen, self.kmin,
                  float(np.float32(1.0 / self.sr)), _lib.ptr(self.D), flen, _lib.ptr(self.IP), flen, s)
        self.launches += 1
        return self.D, self.IP
