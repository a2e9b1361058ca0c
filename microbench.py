"""Micro-benchmarks of single kernels on synthetic operands (used for profiling; prints one JSON line per case).

    python microbench.py gemm  [--r 128] [--n 256] [--tn 917504] [--form f16] [--reps 20]
    python microbench.py basis [--r 128] [--tlen 1048576] [--form f16] [--reps 5] [--wrows 0,4,8]
    python microbench.py exact [--groups 512] [--peaks 1] [--tlen 1048576] [--reps 5]
    python microbench.py adjoint [--triggers 4096] [--reps 5]
    python microbench.py c4 [--segments 300] [--batch 32] [--form f16] [--no-graph] [--production]

Run from the repository root. Operand sizes default to one (tile, chunk) of the C2 workload; inputs are larger than
L2 where the real ones are. The measurement harness lives here, outside the library package gwb200."""
import argparse
import json
import os
import sys

import numpy as np
import torch

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), 'gw-gpu-search_b200'))
from gwb200 import _exact, _lib, fp_filter  # noqa: E402


def _time(fn, reps):
    for _ in range(2):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def gemm(a):
    n, r, Tn = a.n, a.r, a.tn
    code = {'f16': 0, 'bf16': 1, 'bf16x3': 2, 'fp8': 3, 'f16x2': 6}[a.form]
    Kh = fp_filter.kh_of(r, a.form)
    g = torch.Generator(device='cuda').manual_seed(0)
    A = torch.randn((n, 2 * Kh), generator=g, device='cuda')
    Z = torch.randn((2 * Kh, Tn), generator=g, device='cuda')
    if code == 3:
        A, Z = A.to(torch.float8_e4m3fn).view(torch.uint8), Z.to(torch.float8_e4m3fn).view(torch.uint8)
    else:
        dt = torch.float16 if a.form in ('f16', 'f16x2') else torch.bfloat16
        A, Z = A.to(dt), Z.to(dt)
    rs = torch.ones(n, device='cuda')
    lo = (A.clone(), Z.clone()) if code == 2 else ((A.clone(), None) if code == 6 else (None, None))
    nw = Tn // 2048
    V = torch.empty((n, nw), dtype=torch.float32, device='cuda')
    I = torch.empty((n, nw), dtype=torch.int32, device='cuda')
    work = torch.empty(_lib.load().gwb_fused_peaks_cplx_work_bytes(n), dtype=torch.uint8, device='cuda')
    wk = None if a.no_split else work

    def f():
        _lib.call('gwb_fused_peaks_cplx', code, _lib.ptr(A), _lib.ptr(lo[0]), A.stride(0), _lib.ptr(Z), _lib.ptr(lo[1]),
                  Z.stride(0), n, Kh, Tn, 16, _lib.ptr(V), _lib.ptr(I), V.stride(0), _lib.ptr(rs), _lib.ptr(wk),
                  0 if wk is None else wk.numel(), _lib.stream_ptr())
    useful = 8.0 * n * r * Tn
    issued = {2: 3, 6: 2}.get(code, 1) * 4.0 * n * 2 * Kh * Tn
    zbytes = 2 * Kh * Tn * (1 if code == 3 else 2) * (2 if code == 2 else 1)
    out = dict(kernel='umma_cplx_kernel', form=a.form, n=n, r=r, Kh=Kh, Tn=Tn)
    # launch configurations (gwb_gemm_set_config): pair x stages x order; results must not depend on them
    ref = None
    for pair in [int(x) for x in a.pair.split(',')]:
        for st in [int(x) for x in a.stages.split(',')]:
            for order in [int(x) for x in a.orders.split(',')]:
                _lib.call('gwb_gemm_set_config', code, Kh, pair, st, order)
                ms = _time(f, a.reps)
                if ref is None:
                    ref = (V.clone(), I.clone())
                same = bool(torch.equal(ref[0], V) and torch.equal(ref[1], I))
                out['p%d_s%d_o%d' % (pair, st, order)] = dict(ms=ms, useful_tflops=useful / ms / 1e9,
                                                              issued_tflops=issued / ms / 1e9,
                                                              z_gbs=zbytes / ms / 1e6, same_output=same)
    _lib.call('gwb_gemm_clear_configs')
    return out


def basis(a):
    r, tlen = a.r, a.tlen
    flen = tlen // 2 + 1
    ws = fp_filter.BasisWorkspace(tlen, flen)
    g = torch.Generator(device='cuda').manual_seed(0)
    Vh = torch.randn((r, flen), generator=g, device='cuda', dtype=torch.complex64)
    D = torch.randn(flen, generator=g, device='cuda', dtype=torch.complex64)
    isw = torch.rand(flen, generator=g, device='cuda')
    a0, Tn = tlen * 3 // 32, tlen * 28 // 32
    Kh = fp_filter.kh_of(r, a.form)
    Z = torch.zeros((2 * Kh, Tn), dtype=fp_filter._z_dtype(a.form), device='cuda')
    Zlo = torch.zeros_like(Z) if a.form == 'bf16x3' else None
    Dp = fp_filter.fourstep_order(D, tlen, isw)
    Vp = fp_filter.fourstep_order(Vh, tlen)
    out = dict(kernel='basis_series', form=a.form, r=r, tlen=tlen)
    if a.form != 'fp8':            # the cuFFT path has no fp8 pack
        ms = _time(lambda: fp_filter.basis_series_into(ws, Vh, D, isw, a0, Tn, Z, Zlo, a.form, im_off=Kh), a.reps)
        out.update(ms_cufft_path=ms, us_per_row_cufft=ms * 1e3 / r)
    zb = 2 * Tn * {'f16': 2, 'bf16': 2, 'fp8': 1}.get(a.form, 4)
    first = None
    runs = [(c, p) for c in [int(x) for x in a.pass2_cols.split(',')]
            for p in ([int(x) for x in a.pass2_pairs.split(',')] if c == 16 else [1])]
    for cols, pairs in runs:
        _lib.call('gwb_basis_set_pass2_columns', -1, cols)
        _lib.call('gwb_basis_set_pass2_pairs', pairs)
        for wr in [int(x) for x in a.wrows.split(',')]:
            fws = fp_filter.FusedBasisWorkspace(tlen, flen, r, wrows=wr or None, ring=False)
            msf = _time(lambda: fp_filter.basis_series_fused(fws, Vp, Dp, a0, Tn, Z, Zlo, a.form, im_off=Kh), a.reps)
            tag = f'w{fws.wrows}_c{cols}' + ('' if pairs else '_unpaired')
            # HBM bytes of the fused form when W stays in L2: Vh read and Z written (D isw stays in L2)
            out['us_per_row_fused_' + tag] = msf * 1e3 / r
            out['hbm_gbs_' + tag] = r * (8 * flen + zb) / msf / 1e6
            got = [Z.clone()] + ([Zlo.clone()] if Zlo is not None else [])
            if first is None:
                first = got
            else:
                out['bit_identical_' + tag] = all(torch.equal(x, y) for x, y in zip(got, first))
    _lib.call('gwb_basis_set_pass2_columns', -1, 16)
    _lib.call('gwb_basis_set_pass2_pairs', 1)
    full = (lambda: Z.double() + Zlo.double()) if Zlo is not None else (lambda: Z.double())
    if tlen == fp_filter.RING_N and a.ring_cfgs:
        ref = full() * fws.scale.double()
        for rc in [tuple(int(v) for v in x.split(':')) for x in a.ring_cfgs.split(',')]:
            _lib.call('gwb_basis_ring_set_config', *rc)
            rws = fp_filter.FusedBasisWorkspace(tlen, flen, r, ring=True)
            msr = _time(lambda: fp_filter.basis_series_fused(rws, Vp, Dp, a0, Tn, Z, Zlo, a.form, im_off=Kh),
                        a.reps)
            tag = 'ring_%d_%d_%d' % rc
            out['us_per_row_' + tag] = msr * 1e3 / r
            # the ring form's scale comes from pc rows instead of 64: compare the series times their scales
            got = full() * rws.scale.double()
            out['max_rel_vs_two_pass_' + tag] = float(((got - ref).abs().max() / ref.abs().max()).item())
            del rws
        _lib.call('gwb_basis_ring_set_config', 2, 3, 1)
    return out


def exact(a):
    tlen = a.tlen
    flen = tlen // 2 + 1
    kmin = tlen // 100
    nrow = 64
    g = torch.Generator(device='cuda').manual_seed(0)
    H = torch.randn((nrow, flen), generator=g, device='cuda', dtype=torch.complex64)
    D = torch.randn((1, flen), generator=g, device='cuda', dtype=torch.complex64)
    rng = np.random.default_rng(0)
    rows = np.repeat(rng.integers(0, nrow, a.groups), a.peaks)
    samples = rng.integers(0, tlen, len(rows))
    order, rows_u, cands, groups, units = _exact.plan(rows, samples)
    B = 16
    edges = np.linspace(kmin, flen - 2, B + 1).astype(np.int32)
    E = torch.from_numpy(np.tile(edges, (len(units), 1))).cuda()
    nb = torch.full((nrow,), B, dtype=torch.int32, device='cuda')
    nchunk = _lib.load().gwb_exact_chunks(flen, kmin)
    slots = torch.empty((len(cands), nchunk, B, 2), dtype=torch.float32, device='cuda')
    cd, gd, ud = _exact.to_dev(cands), _exact.to_dev(groups), _exact.to_dev(units)

    def f():
        _lib.call('gwb_bin_sums', _lib.ptr(gd), None, len(groups), _lib.ptr(ud), _lib.ptr(cd), _lib.ptr(E), B,
                  _lib.ptr(nb), _lib.ptr(H), H.stride(0), _lib.ptr(D), D.stride(0), kmin, flen, tlen, _lib.ptr(slots),
                  _lib.stream_ptr())
    ms = _time(f, a.reps)
    nbins = int(edges[-1] - edges[0])
    return dict(kernel='binsum_kernel', groups=len(groups), peaks_per_group=a.peaks, ms=ms,
                gbs=len(groups) * nbins * 16 / ms / 1e6)


def adjoint(a):
    """C5: n triggers of 16 s (flen 16,385) with random C2-like parameters against synthetic whitened data: gradient of
    SNR / newSNR (fp32 and fp64 sums), the 7 x 7 phase metric of 10,000 bank points, and 20 refinement steps."""
    from gwb200 import adjoint as adj
    n, tlen = a.triggers, 1 << 15
    flen, df = tlen // 2 + 1, 2048.0 / tlen
    kmin = int(20.0 / df)
    g = torch.Generator(device='cuda').manual_seed(0)
    th = torch.empty((n, 7), dtype=torch.float64, device='cuda')
    th[:, 0] = 5.0 + 30.0 * torch.rand(n, generator=g, device='cuda', dtype=torch.float64)
    th[:, 1] = 0.3 + 0.7 * torch.rand(n, generator=g, device='cuda', dtype=torch.float64)
    th[:, 2:4] = 1.8 * torch.rand((n, 2), generator=g, device='cuda', dtype=torch.float64) - 0.9
    th[:, 4] = 0.3 * torch.rand(n, generator=g, device='cuda', dtype=torch.float64)
    th[:, 5] = 0.0
    th[:, 6] = 0.0
    D = torch.randn((n, flen), generator=g, device='cuda', dtype=torch.complex64)
    f = torch.arange(flen, device='cuda', dtype=torch.float64) * df
    IP = torch.where(f >= 20.0, (f / 200.0) ** 4.0 / (1 + (f / 200.0) ** 4), torch.zeros_like(f)).float()
    out = {}
    for fp64 in (False, True):
        out['ms_grad_fp64' if fp64 else 'ms_grad_fp32'] = _time(lambda: adj.snr_grad(th, D, IP, df, kmin, fp64=fp64),
                                                                a.reps)
    bank = th[:min(n, 10000)]
    if n < 10000:
        bank = th.repeat(-(-10000 // n), 1)[:10000].contiguous()
    out['ms_metric_10000'] = _time(lambda: adj.phase_metric(bank, IP, flen, df, kmin), a.reps)
    out['ms_refine_20_steps'] = _time(lambda: adj.refine(th, D, IP, df, kmin, steps=20), 1)
    bins = float((adj.snr_grad(th, D, IP, df, kmin)['kmax'] - kmin).clamp_min(0).sum())   # bins below each ISCO
    return dict(kernel='snr_grad_kernel / phase_metric_kernel / refine', triggers=n, flen=flen,
                triggers_per_s_fp32=n / out['ms_grad_fp32'] * 1e3, bins=bins, bins_per_ns_fp32=bins / out['ms_grad_fp32'] / 1e6,
                **out)


def c4(a):
    """C4: science segments with lengths log-uniform in [64, 4096] s at 2048 Hz over two detectors, coloured noise
    (the analytic PSD with 60/120/180 Hz lines), TaylorF2 injections (SNR 6-30, about one per 290 s), sine-Gaussian
    glitches (Q = 10, f0 30-300 Hz, SNR 20-200) in 2% of the segments; the C2 bank of 5,880 templates in 512 s chunks.
    Times filter_segments (autogating, chunking, graph-replayed batches, results) end to end on the device."""
    import time
    import numpy as np
    from gwb200 import pipeline, segments as sg, templates
    sr, L = 2048.0, 512.0
    tlen = int(L * sr)
    flen, df = tlen // 2 + 1, 1.0 / L
    rng = np.random.default_rng(a.seed)
    lens = np.floor(np.exp(rng.uniform(np.log(64.0), np.log(4096.0), a.segments))).astype(int)
    dyn = 5.9029581035870565e+20

    def psd(f):
        x = np.maximum(f, 15.0) / 215.0
        p_ = 1e-49 * (x ** -4.14 - 5.0 * x ** -2 + 111.0 * (1.0 - x ** 2 + 0.5 * x ** 4) / (1.0 + 0.5 * x ** 2))
        p_ = np.where(f < 15.0, 1e4 * p_, p_)
        for f0, h, w in ((60.0, 1e3, 0.02), (120.0, 1e3, 0.02), (180.0, 1e3, 0.02)):
            p_ = p_ * (1.0 + h / (1.0 + ((f - f0) / w) ** 2))
        return p_ * dyn ** 2

    rb = np.random.default_rng(0)
    m = rb.uniform(3.0, 100.0, (4612, 2))
    mt, q, e0 = rb.uniform(45.0, 100.0, 1268), rb.uniform(1.0, 3.0, 1268), rb.uniform(0.0, 0.3, 1268)
    bank = dict(mass1=np.r_[m.max(1), mt * q / (1 + q)], mass2=np.r_[m.min(1), mt / (1 + q)],
                spin1z=np.r_[rb.uniform(-0.9, 0.9, 4612), np.zeros(1268)],
                spin2z=np.r_[rb.uniform(-0.9, 0.9, 4612), np.zeros(1268)], ecc=np.r_[np.zeros(4612), e0])
    segs, inj, glitches = [], [], []
    gps = 1000000000
    for i, n_s in enumerate(lens):
        n = int(n_s * sr)
        fl = n // 2 + 1
        f = np.arange(fl) * (sr / n)
        g = torch.Generator(device='cuda').manual_seed(a.seed * 7919 + i)
        X = torch.fft.rfft(torch.randn(n, generator=g, device='cuda', dtype=torch.float64))
        X *= torch.from_numpy(np.sqrt(psd(f) * sr / 2.0)).cuda()
        X[0] = 0
        ps = torch.from_numpy(psd(f)).cuda()
        fk = torch.from_numpy(f).cuda()
        kmin = int(20.0 * n / sr)
        for _ in range(rng.poisson(n_s / 290.0)):
            row, t0, snr = int(rng.integers(0, 5880)), rng.uniform(48.0, n_s - 16.0), rng.uniform(6.0, 30.0)
            h, _ = templates.generate(bank, [row], fl, sr / n, 20.0, device='cuda')
            h = h[0].to(torch.complex128)
            h = h * (snr / torch.sqrt(4 * (sr / n) * (h[kmin:].abs() ** 2 / ps[kmin:]).sum()))
            X += h * torch.exp(-2j * np.pi * fk * t0) * sr
            inj.append((i, t0, row, snr))
        x = torch.fft.irfft(X, n)
        if rng.uniform() < 0.02:
            f0, snr, tg = rng.uniform(30.0, 300.0), rng.uniform(20.0, 200.0), rng.uniform(20.0, n_s - 20.0)
            tau = 10.0 / (np.sqrt(2.0) * np.pi * f0)
            t = torch.arange(n, device='cuda', dtype=torch.float64) / sr - tg
            sgx = torch.exp(-(t / tau) ** 2) * torch.sin(2 * np.pi * f0 * t)
            G = torch.fft.rfft(sgx) / sr
            rho = torch.sqrt(4 * (sr / n) * (G[kmin:].abs() ** 2 / ps[kmin:]).sum())
            x += sgx * (snr / rho)
            glitches.append((i, tg, f0, snr))
        segs.append(dict(x=x.to(torch.float32).contiguous(), start_gps=gps, det=i % 2))
        gps += int(n_s) + 100
    tune = bool(getattr(a, 'autotune', False))
    cfg = pipeline.FilterConfig(form=a.form, autotune=tune)
    co = None
    if a.production:
        # production's selection (threshold 4, exact stage above 5.5 (1 - margin), the rest rebuilt) and
        # consolidation (newsnr 4, 30 loudest per 1.072 s, SNR >= 5 exempt): ops/run_prod_o4a.sh's flags
        cfg = pipeline.FilterConfig(form=a.form, snr_threshold=4.0, exact_snr=5.5, rebuilt_cap=1 << 24, autotune=tune)
        co = sg.Consolidation()
    # SVD metric of the run from a first batch of chunks, then the bank (as bench.py builds it)
    from gwb200 import gpu_prep
    first = [s for s in segs if s['x'].shape[0] >= tlen][:a.batch]
    Xb = torch.stack([s['x'][:tlen] for s in first] + [first[0]['x'][:tlen]] * (a.batch - len(first)))
    cond = gpu_prep.BatchConditioner(a.batch, tlen, sr, 20.0, 16.0, 8.0, 63, 16.0)
    _, IPb = cond(Xb.contiguous())
    sw, isw = fp_filter.derive_sw(IPb)
    sw, isw = sw.clone(), isw.clone()
    del cond
    torch.cuda.synchronize()
    t_b = time.perf_counter()
    if getattr(a, 'bank_obj', None) is not None:
        # a bank built by the caller for the same chunk length (the C2 bank of bench.py), with its own SVD metric
        B, isw = a.bank_obj, a.isw
    else:
        B = pipeline.Bank(bank, flen, df, sw, cfg)
    torch.cuda.synchronize()
    bank_s = time.perf_counter() - t_b
    F = sg.SegmentFilter(B, cfg, batch=a.batch, isw=isw, graph=not a.no_graph, consolidation=co)
    one_graph = co is None and not a.no_graph and not getattr(a, 'per_batch', False)
    prep_s = None
    if one_graph:
        # the whole run (every batch: chunk copies, conditioning, filter step, result append) captured as one graph
        # before the timed region; the timed region gates the segments, replays it once and copies the results back
        prep_s = F.prepare(segs)
    else:
        F.run(first[:1], gate=False)       # warm-up on one chunk (captures the batch graph outside the timed run)
    torch.cuda.synchronize()
    e0_, e1_ = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.perf_counter()
    e0_.record()
    res = F.run_graph() if one_graph else F.run(segs)
    e1_.record()
    torch.cuda.synchronize()
    wall = time.perf_counter() - t0
    ms = e0_.elapsed_time(e1_)
    # injections in analysed time recovered: a kept peak within 0.1 s of the injection in its segment
    kept = res['keep']
    c, segi, ch = res['cands'][kept], res['segment'][kept], res['chunk'][kept]
    t_peak = (np.array([res['plan'][k][1][0] for k in ch]) + c['sample']) / sr if len(c) else np.zeros(0)
    n_inj_an, found = 0, 0
    for (i, t_inj, row, snr) in inj:
        if lens[i] < L or snr < 8.0:
            continue
        n_inj_an += 1
        found += int(np.any((segi == i) & (np.abs(t_peak - t_inj) < 0.1)))
    gated = sum(1 for (i, *_rest) in glitches if res['gates'][i])
    weeks = res['analysed_s'] / (2 * 604800.0)
    extra = {}
    if co is not None:
        found_t = 0
        for (i, t_inj, row, snr) in inj:
            if lens[i] < L or snr < 8.0 or i not in res['tables']:
                continue
            found_t += int(np.any(np.abs(res['tables'][i]['end_time'] - (segs[i]['start_gps'] + t_inj)) < 0.1))
        extra = dict(selection='threshold 4, exact above 5.28, rebuilt below; consolidated (newsnr 4, 30 per '
                               '1.072 s, exempt 5)', peaks_before_consolidation=res['n_peaks_in'],
                     peaks_after_consolidation=res['n_peaks_out'], injections_found_in_tables=found_t)
    return dict(workload='C4: %d segments, log-uniform 64-4096 s, 2 detectors, %d injections, %d glitches; 5880 '
                         'templates, %s' % (a.segments, len(inj), len(glitches), a.form),
                value=weeks / (ms / 1e3 / 3600.0), unit='2-det weeks / hour', ms=ms, wall_s=wall,
                analysed_s=res['analysed_s'], skipped_s=res['skipped_s'], skipped_segments=len(res['skipped']),
                total_s=float(lens.sum()), chunks=res['n_chunks'], batches=res['batches'], graph=not a.no_graph,
                kept=int(kept.sum()), candidates=len(res['cands']), glitches=len(glitches), glitches_gated=gated,
                injections_snr8_in_analysed=n_inj_an, injections_found=found,
                gates=sum(len(g) for g in res['gates']), bank_setup_s=bank_s, seed=a.seed,
                one_graph=one_graph, graph_capture_s=prep_s, **extra)


# ---- precision of the arithmetic forms against float64 -------------------------------------------------------------
# Precision of the filter's arithmetic forms against float64 on one (tile, segment): the window maxima of the SNR
# that the fused GEMM of a form produces, against the same maxima of a float64 SNR series.
#
# The float64 series follows the reference's math without rounding: the basis series zb = ifft(conj(Vh) D isw) over
# the analysed span (fp_filter.py:597-613, norm='forward', zero-padded half spectrum), z = A zb (the product the
# stacked GEMM forms, fp_filter.py:615-621, fp_gemm.py:14-33) and snr = |z| 4 df / sqrt(sigma^2) (fp_filter.py:710-714).
# Windows are the filter's cluster windows over the analysed span; the index is the first maximum, as the GEMM's.


def fp64_window_snr(sv, D_seg, isw, sig_col, df, tlen, a0, Tn, cw, batch=32):
    """float64 window maxima (n, nw) of the SNR of one tile against one segment, and their samples (relative to a0).
    sv: the tile's SVD entry (A (n, r), Vh (r, flen)); D_seg (flen,) complex64; isw (flen,); sig_col (n,) float64."""
    dev = D_seg.device
    Vh = sv['Vh'].to(torch.complex128)
    A = sv['A'].to(torch.complex128)
    r, flen = Vh.shape
    n = A.shape[0]
    dw = D_seg.to(torch.complex128) * isw.to(torch.float64)
    zb = torch.empty((r, Tn), dtype=torch.complex128, device=dev)
    for j0 in range(0, r, batch):
        j1 = min(r, j0 + batch)
        q = torch.zeros((j1 - j0, tlen), dtype=torch.complex128, device=dev)
        q[:, :flen] = torch.conj(Vh[j0:j1]) * dw
        zb[j0:j1] = torch.fft.ifft(q, norm='forward')[:, a0:a0 + Tn]
        del q
    z = A @ zb
    del zb
    norm = 4.0 * df / torch.sqrt(sig_col.to(torch.float64))
    snr = z.abs() * norm[:, None]
    del z
    nw = Tn // cw
    v, i = snr[:, :nw * cw].reshape(n, nw, cw).max(2)
    i = i + torch.arange(nw, device=dev)[None, :] * cw
    return v.cpu().numpy(), i.cpu().numpy()


def form_window_snr(mf, t, D, isw, sig, seg):
    """Window maxima of the SNR (n, nw) and their samples from the fused GEMM of mf's form, for tile t against
    segment seg (rows of D). Resets mf's candidate counters (the diagnostic call's candidates are not kept)."""
    if mf.fused:
        mf.Dp = fp_filter.fourstep_order(D, mf.tlen, isw)
    mf.counters.zero_()
    mf.tile_segment(t, D, isw, sig, seg)
    torch.cuda.synchronize()
    mf.counters.zero_()
    n = len(mf.bank.tiles[t])
    v = mf.V[:n].double().clamp_min(0).sqrt().cpu().numpy()
    return v, mf.I[:n].cpu().numpy().astype(np.int64)


def compare(v, i, v64, i64, thr):
    """Differences of one form's window maxima from float64's: |delta SNR| (max, median), relative (max, median),
    argmax agreement (exact, and within 2 samples: the series is smooth, so a 16-bit form may pick a neighbour of
    an almost equal maximum), and the windows above thr in one but not the other (all, and those more than 1e-3 thr
    away from the threshold in float64)."""
    d = np.abs(v - v64)
    rel = d / np.maximum(v64, 1e-30)
    above, above64 = v > thr, v64 > thr
    flip = above ^ above64
    return dict(max_abs_dsnr=float(d.max()), median_abs_dsnr=float(np.median(d)), max_rel=float(rel.max()),
                median_rel=float(np.median(rel)), argmax_agree=float(np.mean(i == i64)),
                argmax_within2=float(np.mean(np.abs(i - i64) <= 2)), windows=int(v.size),
                above_fp64=int(above64.sum()), set_diff=int(flip.sum()),
                set_diff_away=int((flip & (np.abs(v64 - thr) > 1e-3 * thr)).sum()))


def fp64_exact_at(H, rows, samples, D_seg, IP_seg, kmin, kmax, nbins, sig, df, tlen, batch=16):
    """The exact stage in float64 at (row, sample) pairs: equal-power edges as multi_filter.edges_per_template
    (pipeline/multi_filter.py:264-282: first k whose cumulative |h|^2 IP exceeds j / nb of the total below kmax,
    clipped to [kmin, kmax]), bin sums Z_j = sum_{k in bin j} conj(h_k) D_k e^{2 pi i (k t mod N) / N}
    (pipeline/chisq_kernel.py:17-82), then snr = |z| 4 df / sqrt(sig) and chisq = (nb pw - |z|^2) norm^2
    (pipeline/fp_filter.py:837-853). H (rows of the bank) complex64, D_seg / IP_seg one segment, kmax / nbins per bank
    row (int), sig per bank row (float64 of this segment). Returns (snr, chisq) float64 numpy arrays."""
    dev = H.device
    flen = H.shape[1]
    rh = np.asarray(rows, np.int64)
    assert rh.size == 0 or (rh.min() >= 0 and rh.max() < min(H.shape[0], len(kmax), len(nbins), len(sig))), \
        'rows index the bank: kmax, nbins and sig are per bank row'
    assert len(samples) == len(rh)
    rows = torch.as_tensor(rh, device=dev)
    samples = torch.as_tensor(np.asarray(samples, np.int64), device=dev)
    kmax = torch.as_tensor(np.asarray(kmax, np.int64), device=dev)
    nbins = torch.as_tensor(np.asarray(nbins, np.int64), device=dev)
    sig = torch.as_tensor(sig, device=dev).to(torch.float64)
    k = torch.arange(flen, device=dev, dtype=torch.int64)
    ip = IP_seg.to(torch.float64)
    Dd = D_seg.to(torch.complex128)
    B = int(nbins.max()) if len(rows) else 1
    snr_o, chi_o = [], []
    for b0 in range(0, len(rows), batch):
        r = rows[b0:b0 + batch]
        t = samples[b0:b0 + batch]
        h = H[r].to(torch.complex128)
        nb, k1 = nbins[r], kmax[r]
        cs = torch.cumsum((h.real ** 2 + h.imag ** 2) * ip, 1)
        tot = cs.gather(1, (k1 - 1)[:, None])
        j = torch.arange(B, device=dev, dtype=torch.float64)[None, :]
        e = torch.searchsorted((cs / tot).contiguous(), (j / nb[:, None]).contiguous(), right=True)
        e = torch.minimum(torch.maximum(e, torch.full_like(e, kmin)), k1[:, None])
        e = torch.where(j < nb[:, None], e, k1[:, None])
        edges = torch.cat([e, k1[:, None]], 1)                              # (b, B + 1)
        q = torch.conj(h) * Dd
        ph = ((k[None, :] * t[:, None]) % tlen).to(torch.float64) * (2.0 * np.pi / tlen)
        x = q * torch.polar(torch.ones_like(ph), ph)
        inb = (k[None, :] >= edges[:, :1]) & (k[None, :] < edges[:, -1:])
        bidx = torch.searchsorted(edges.contiguous(), k[None, :].expand(len(r), flen).contiguous(), right=True) - 1
        bidx = bidx.clamp(0, B - 1)
        x = torch.where(inb, x, torch.zeros_like(x))
        Z = torch.zeros((len(r), B), dtype=torch.complex128, device=dev)
        Z.real.scatter_add_(1, bidx, x.real.contiguous())
        Z.imag.scatter_add_(1, bidx, x.imag.contiguous())
        z = Z.sum(1)
        pw = (Z.real ** 2 + Z.imag ** 2).sum(1)
        norm = 4.0 * df / torch.sqrt(sig[r])
        snr_o.append((z.abs() * norm).cpu().numpy())
        chi_o.append(((nb.to(torch.float64) * pw - z.abs() ** 2) * norm ** 2).cpu().numpy())
        del h, cs, q, ph, x, bidx, inb
    if not snr_o:
        return np.zeros(0), np.zeros(0)
    return np.concatenate(snr_o), np.concatenate(chi_o)


def _stats(x):
    x = np.asarray(x, np.float64)
    if x.size == 0:
        return dict(n=0)
    return dict(n=int(x.size), max=float(x.max()), median=float(np.median(x)), p99=float(np.percentile(x, 99)))


def precision_c2(B, cond, x, isw, forms, form_config, g, seg=0, n_chisq=256, seed=0):
    """Precision of each form against float64 over every tile of one segment (seg) of a C2 step:
    windows: the window maxima of the rebuilt SNR from the form's fused GEMM against the float64 series' (all tiles);
    kept: the peaks kept after the form's exact stage (one step of every tile against seg) against the float64
      exact stage's: float64 transform and product, window argmax, float64 exact SNR at that sample for every window
      whose float64 window maximum is above 0.95 of the threshold (the rebuilt and exact SNR differ by about 1%),
      kept when above the threshold. Set agreement (away = beyond 3% of the threshold in the float64 exact SNR),
      relative exact-SNR error at the common windows, and relative chi-squared error against the float64 exact stage
      at the float64 argmax for up to n_chisq sampled common windows (the loudest 32 always among them), and at the
      form's own sample (the exact stage's own error).
    form_config(form): the FilterConfig of a form. g: dict(df, tlen, a0, an (analysed span), cw, thr)."""
    from gwb200 import pipeline
    Dd, IPd = cond(x)
    rep = dict(segment=seg, tiles=len(B.tiles), reference='float64 transform, product and exact stage (torch '
               'complex128 on the device; checked against the numpy oracle in tests/test_precision_gpu.py)')
    mf0 = pipeline.MatchedFilter(B, g['tlen'], g['a0'], g['an'], pipeline.FilterConfig(form=forms[0]))
    sig = mf0.norms(IPd)
    Tn, cw = mf0.Tn, mf0.cw
    del mf0
    v64, i64 = [], []
    for t in range(len(B.tiles)):
        r0, n = B.row0[t], len(B.tiles[t])
        v, i = fp64_window_snr(B.svd[t], Dd[seg], isw, sig[r0:r0 + n, seg], g['df'], g['tlen'], g['a0'], Tn, cw)
        v64.append(v)
        i64.append(i)
    V64, I64 = np.concatenate(v64), np.concatenate(i64)                     # (M, nw), bank rows in tile order
    thr = g['thr']
    sig_seg = sig[:, seg].double()
    kmax = B.kmax_h
    nbins = np.full(B.M, B.cfg.nbins)
    # the float64 exact stage: exact SNR at the float64 argmax of every window near or above the threshold
    near = np.argwhere(V64 > 0.95 * thr)
    ex_snr, _ = fp64_exact_at(B.H, near[:, 0], g['a0'] + I64[near[:, 0], near[:, 1]], Dd[seg], IPd[seg], B.kmin, kmax,
                              nbins, sig_seg, g['df'], g['tlen'], batch=64)
    EX64 = {(int(r_), int(w_)): float(v_) for (r_, w_), v_ in zip(near.tolist(), ex_snr)}
    set64 = {p for p, v_ in EX64.items() if v_ > thr}
    rep['fp64_exact'] = dict(windows_evaluated=len(EX64), kept=len(set64),
                             rebuilt_vs_exact=_stats(np.abs(ex_snr - V64[near[:, 0], near[:, 1]]) / ex_snr)
                             if len(ex_snr) else None)
    AWAY = 0.03
    rng = np.random.default_rng(seed)
    for form in forms:
        cfg = form_config(form)
        mf = pipeline.MatchedFilter(B, g['tlen'], g['a0'], g['an'], cfg)
        # window maxima of every tile
        vf, if_ = [], []
        for t in range(len(B.tiles)):
            v, i = form_window_snr(mf, t, Dd, isw, sig, seg)
            vf.append(v)
            if_.append(i)
        Vf, If = np.concatenate(vf), np.concatenate(if_)
        win = compare(Vf, If, V64, I64, thr)
        # the peaks the form keeps after its exact stage, one step over every tile against seg
        mf.step(Dd, IPd, isw, seg_ids=[seg])
        torch.cuda.synchronize()
        res = mf.results()
        kc, kp = res['cands'][res['keep']], res['peaks'][res['keep']]
        kept = {(int(r_), int(w_)): (float(s_), float(c_), int(t_))
                for r_, w_, s_, c_, t_ in zip(kc['row'], kc['window'], kp['snr'], kp['chisq'], kc['sample'])}
        ks = set(kept)
        only64, onlyf = set64 - ks, ks - set64
        common = sorted(ks & set64)
        rel_snr = [abs(kept[p][0] - EX64[p]) / EX64[p] for p in common]
        # chi-squared against float64 at a sample of the common windows
        chi = dict(n=0)
        if common:
            loud = sorted(common, key=lambda p: -V64[p])[:32]
            rest = [p for p in common if p not in set(loud)]
            pick = loud + [rest[j] for j in rng.choice(len(rest), min(len(rest), max(0, n_chisq - len(loud))),
                                                       replace=False)]
            rows = np.array([p[0] for p in pick])
            s64 = np.array([g['a0'] + I64[p] for p in pick])
            sf = np.array([kept[p][2] for p in pick])
            snr_a, chi_a = fp64_exact_at(B.H, rows, s64, Dd[seg], IPd[seg], B.kmin, kmax, nbins, sig_seg, g['df'],
                                         g['tlen'])
            snr_b, chi_b = fp64_exact_at(B.H, rows, sf, Dd[seg], IPd[seg], B.kmin, kmax, nbins, sig_seg, g['df'],
                                         g['tlen'])
            cf = np.array([kept[p][1] for p in pick])
            snf = np.array([kept[p][0] for p in pick])
            chi = dict(n=len(pick), rel_vs_fp64_argmax=_stats(np.abs(cf - chi_a) / np.maximum(np.abs(chi_a), 1e-30)),
                       rel_vs_fp64_same_sample=_stats(np.abs(cf - chi_b) / np.maximum(np.abs(chi_b), 1e-30)),
                       snr_rel_vs_fp64_same_sample=_stats(np.abs(snf - snr_b) / snr_b),
                       fp64_series_vs_fp64_exact_snr=_stats(np.abs(snr_a - np.array([V64[p] for p in pick])) /
                                                            snr_a),
                       sample_agree=float(np.mean(s64 == sf)))
        rep[form] = dict(windows=win, kept=dict(
            fp64=len(set64), form=len(ks), both=len(common), only_fp64=len(only64), only_form=len(onlyf),
            only_fp64_away=sum(EX64[p] > thr * (1 + AWAY) for p in only64),
            only_form_away=sum(EX64.get(p, 0.0) < thr * (1 - AWAY) for p in onlyf),
            snr_rel_common=_stats(rel_snr)), chisq=chi)
        del mf
        torch.cuda.empty_cache()
    return rep


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('what', choices=['gemm', 'basis', 'exact', 'adjoint', 'c4'])
    ap.add_argument('--segments', type=int, default=300)
    ap.add_argument('--batch', type=int, default=32)
    ap.add_argument('--seed', type=int, default=4)
    ap.add_argument('--no-graph', action='store_true')
    ap.add_argument('--production', action='store_true')
    ap.add_argument('--no-split', action='store_true', help='gemm: whole windows per CTA (no partial-window merge)')
    ap.add_argument('--triggers', type=int, default=4096)
    ap.add_argument('--r', type=int, default=128)
    ap.add_argument('--n', type=int, default=256)
    ap.add_argument('--tn', type=int, default=917504)
    ap.add_argument('--tlen', type=int, default=1 << 20)
    ap.add_argument('--form', default='f16')
    ap.add_argument('--groups', type=int, default=512)
    ap.add_argument('--peaks', type=int, default=1)
    ap.add_argument('--reps', type=int, default=10)
    ap.add_argument('--wrows', default='0', help='basis: comma list of W row batches (0: all rows at once)')
    ap.add_argument('--pass2-cols', default='16,8', help='basis: comma list of columns per pass-2 CTA (8, 16)')
    ap.add_argument('--pass2-pairs', default='1,0',
                    help='basis: comma list of Z store modes of the 16-column pass 2 (1 paired, 0 per sample)')
    ap.add_argument('--pair', default='1', help='gemm: comma list, 1 CTA pairs, 0 one CTA per M block')
    ap.add_argument('--stages', default='0', help='gemm: comma list of Z ring depths (0: the most that fit)')
    ap.add_argument('--orders', default='0', help='gemm: comma list of MMA orders of the CTA-pair kernel (0-3)')
    ap.add_argument('--ring-cfgs', default='2:3:1,2:4:2,4:2:1,2:3:0,2:2:0,4:2:0,1:4:0',
                    help='basis: comma list of rows:slots:lookahead of the persistent ring form (2^20; empty: '
                         'none)')
    a = ap.parse_args()
    print(json.dumps({'gemm': gemm, 'basis': basis, 'exact': exact, 'adjoint': adjoint, 'c4': c4}[a.what](a)))


if __name__ == '__main__':
    main()
