"""Throughput of the B200 matched-filter hot path on the two-detector production workload.

Workload (name: "C2"): two detectors (H, L) with independent noise, 64 chunks of 512 s at 2048 Hz each (2^20
samples, one analysis segment per chunk with 48 s / 16 s pads, so 448 s analysed per chunk), Gaussian noise coloured
by the analytic broadband PSD with narrow lines at 60/120/180 Hz, 200 TaylorF2 injections at SNR 6-30; bank of 5,880
templates (4,612 aligned-spin TaylorF2, 1,268 eccentric), SVD-compressed per tile of 256 with eps = 1e-3; 16
chi-squared bins, 1 s windows, candidates above SNR 5.5 (1 - 0.04), exact stage on every candidate. All inputs are
synthetic (seeded); there is no dataset.

One step = the whole hot path over all 128 chunks: conditioning (segment FFT, median-Welch PSD, interpolation,
inverse spectrum truncation, D and IP), template norms, then for every (tile, chunk): basis series, stacked A, the
fused reconstruction GEMM with |z|^2 and windowed argmax, and candidate selection; then the exact stage over every
candidate (edges, binned sums, snr / chisq / newsnr). The bank (templates and tile SVDs) is built once before timing
and reported as bank_setup_s. Metric: two-detector weeks of data filtered per GPU-hour.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--form bf16x3|f16|f32] [--impl reference]
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path[:0] = [os.path.join(ROOT, 'gw-gpu-search_b200'), ROOT]

SR = 2048.0
CHUNK_S = 512
TLEN = int(CHUNK_S * SR)
FLEN = TLEN // 2 + 1
DF = SR / TLEN
START_PAD, END_PAD = 48, 16
A0, A1 = int(START_PAD * SR), int((CHUNK_S - END_PAD) * SR)
F_LOW = 20.0
WEEK2 = 2 * 604800.0
METRIC = "2-det weeks filtered per GPU-hour, 5,880 templates, SNR err<=1e-3: FP32 vs BF16"
DYN = 5.9029581035870565e+20
LINES = ((60.0, 1e3, 0.02), (120.0, 1e3, 0.02), (180.0, 1e3, 0.02))


def psd_model(f):
    """Analytic broadband PSD (strain^2/Hz): 1e-49 [x^-4.14 - 5 x^-2 + 111 (1 - x^2 + x^4/2) / (1 + x^2/2)],
    x = f / 215 Hz; below 15 Hz, 1e4 x its 15 Hz value; narrow lines at 60/120/180 Hz; times DYN_RANGE_FAC^2."""
    f = np.asarray(f, np.float64)
    x = np.maximum(f, 15.0) / 215.0
    s = 1e-49 * (x ** -4.14 - 5.0 * x ** -2 + 111.0 * (1.0 - x ** 2 + 0.5 * x ** 4) / (1.0 + 0.5 * x ** 2))
    s = np.where(f < 15.0, 1e4 * s, s)
    for f0, h, w in LINES:
        s = s * (1.0 + h / (1.0 + ((f - f0) / w) ** 2))
    return s * DYN ** 2


def make_bank(n_aligned=4612, n_ecc=1268, seed=0):
    rng = np.random.default_rng(seed)
    m = rng.uniform(3.0, 100.0, (n_aligned, 2))
    m1, m2 = m.max(1), m.min(1)
    s1, s2 = rng.uniform(-0.9, 0.9, n_aligned), rng.uniform(-0.9, 0.9, n_aligned)
    mt = rng.uniform(45.0, 100.0, n_ecc)
    q = rng.uniform(1.0, 3.0, n_ecc)
    e0 = rng.uniform(0.0, 0.3, n_ecc)
    return dict(mass1=np.r_[m1, mt * q / (1 + q)], mass2=np.r_[m2, mt / (1 + q)], spin1z=np.r_[s1, np.zeros(n_ecc)],
                spin2z=np.r_[s2, np.zeros(n_ecc)], ecc=np.r_[np.zeros(n_aligned), e0])


def make_data(nchunk, bank, n_inj, seed, device):
    """(nchunk, TLEN) float32 strain on the device: coloured noise (seed per chunk) plus injections."""
    import torch
    from gwb200 import templates
    f = np.arange(FLEN) * DF
    amp = torch.from_numpy(np.sqrt(psd_model(f) * SR / 2.0)).to(device)
    rng = np.random.default_rng(seed)
    inj_chunk = rng.integers(0, nchunk, n_inj)
    inj_row = rng.integers(0, len(bank['mass1']), n_inj)
    inj_t = rng.uniform(START_PAD + 2, CHUNK_S - END_PAD - 2, n_inj)
    inj_snr = rng.uniform(6.0, 30.0, n_inj)
    x = torch.empty((nchunk, TLEN), dtype=torch.float32, device=device)
    kmin = int(F_LOW / DF)
    psd_t = torch.from_numpy(psd_model(f)).to(device)
    fk = torch.from_numpy(f).to(device)
    for c in range(nchunk):
        g = torch.Generator(device=device).manual_seed(seed * 100003 + c)
        w = torch.randn(TLEN, generator=g, device=device, dtype=torch.float64)
        X = torch.fft.rfft(w) * amp
        X[0] = 0
        for i in np.flatnonzero(inj_chunk == c):
            h, km = templates.generate(bank, [inj_row[i]], FLEN, DF, F_LOW, device=device)
            h = h[0].to(torch.complex128)
            rho = torch.sqrt(4 * DF * (h[kmin:].abs() ** 2 / psd_t[kmin:]).sum())
            h = h * (inj_snr[i] / rho) * torch.exp(-2j * np.pi * fk * inj_t[i])
            X = X + h * SR                                  # DFT of the time series = h(f) / dt
        x[c] = torch.fft.irfft(X, TLEN).to(torch.float32)
    return x, dict(chunk=inj_chunk, row=inj_row, t=inj_t, snr=inj_snr)


class Clocks:
    """nvidia-smi clock and throttle samples during the timed region."""

    def __init__(self, index):
        self.index, self.lines, self.proc = index, [], None

    def __enter__(self):
        q = ('index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,'
             'clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,'
             'clocks_event_reasons.sw_power_cap')
        try:
            self.proc = subprocess.Popen(['nvidia-smi', '-i', str(self.index), '--query-gpu=' + q,
                                          '--format=csv,noheader,nounits', '-lms', '200'], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ['hw_slowdown', 'hw_thermal_slowdown', 'sw_thermal_slowdown', 'sw_power_cap']
        for l in self.lines:
            p = [x.strip() for x in l.split(',')]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = max(mx, float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower() == 'active':
                    reasons.add(nm)
        return dict(sm_mhz=statistics.median(sm) if sm else None, sm_max_mhz=mx or None, reasons=sorted(reasons),
                    samples=len(sm))


def peaks_file():
    p = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), 'measured'
    return dict(hbm_gbs=6650.0, bf16_tflops=1590.0), 'fallback'


def cpu_reference(bank, n_tiles_sample=1, seed=5):
    """The CPU (numpy) arm: conditioning of one chunk and the full per-(tile, segment) pass with exact stage for
    `n_tiles_sample` tiles of 256, timed with all host threads; returns seconds per chunk for the full bank."""
    from oracle import prep as op, search as osr, filt as of, synth
    rng = np.random.default_rng(seed)
    x = np.fft.irfft(synth.coloured_noise(TLEN, SR, rng, synth.LINES_C2), TLEN).astype(np.float32)
    t0 = time.perf_counter()
    out = op.stage2(x, SR, 0, CHUNK_S, START_PAD, END_PAD, F_LOW, 16, 8, 63, 16)
    t_cond = time.perf_counter() - t0
    D, IP = out['D'][0], out['IP'][0]
    sw, isw = of.derive_sw(out['IP'])
    order = np.argsort(synth.tau0(bank['mass1'], bank['mass2']), kind='stable')
    tiles = [order[b:b + 256] for b in range(0, len(order), 256)]
    kmin = int(F_LOW / DF)
    t_tiles = 0.0
    for t in np.linspace(0, len(tiles) - 1, n_tiles_sample).astype(int):
        ids = tiles[t]
        H = np.stack([synth.taylorf2(FLEN, DF, bank['mass1'][i], bank['mass2'][i], bank['spin1z'][i],
                                     bank['spin2z'][i], bank['ecc'][i]) for i in ids]).astype(np.complex64)
        kmax = np.array([min(int(np.floor(synth.f_isco(bank['mass1'][i], bank['mass2'][i]) / DF)) + 1, FLEN - 1)
                         for i in ids])
        for j, k in enumerate(kmax):
            H[j, k:] = 0
        t1 = time.perf_counter()
        sig, _ = of.sigma2(H, IP[None], DF)
        r, A, Vh, worst, _, _ = of.svd_tile(H, sw, kmin, 1e-3)
        osr.tile_segment_lean(H, np.full(len(ids), 16), kmin, kmax, r, A, Vh, D, IP, isw, sig[:, 0], DF, TLEN, A0,
                              (A1 - A0) // 2048 * 2048, 2048, 5.5, 0.04)
        t_tiles += time.perf_counter() - t1
    per_chunk = t_cond + t_tiles / n_tiles_sample * len(tiles)
    return per_chunk, dict(cond_s=t_cond, tile_s=t_tiles / n_tiles_sample, n_tiles=len(tiles))


def run_reference(a):
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return
    bank = make_bank()
    cores = os.cpu_count()
    per = []
    info = None
    for _ in range(max(1, a.steps)):
        s, info = cpu_reference(bank)
        per.append(s)
    per_chunk = float(np.median(per))
    val = ((A1 - A0) / SR / WEEK2) / (per_chunk / 3600.0)
    print(json.dumps(dict(metric=METRIC, impl='reference', value=val, unit='2-det weeks / hour', n_gpus=a.gpus,
                          steps=a.steps, warmup=a.warmup, ms_per_step=per_chunk * 1e3, higher_is_better=True,
                          scaling='weak', vs_baseline=None, dtype='f32/f64', data='synthetic',
                          config=dict(workload='C2 sample: 1 chunk x 1 of 23 tiles, extrapolated to the bank'),
                          cpu_baseline=dict(value=val, unit='2-det weeks / hour', cores=cores, kind='port',
                                            sample='one 512 s chunk: conditioning + one tile of 256 templates '
                                                   '(tile pass incl. SVD, exact stage), scaled to 23 tiles', **info),
                          e2e=dict(value=val, unit='2-det weeks / hour', h2d_bytes_per_step=0, d2h_bytes_per_step=0))))


def top_peak_sets(kept, thr):
    """Each form's kept peaks (exact stage) against the plain fp32 form's: windows kept by both, by one only, and by
    one only with an exact SNR more than 3% above the threshold (a real disagreement, not a threshold straddle)."""
    if 'f32' not in kept:
        return None
    ref = kept['f32']
    out = {}
    for f, k in kept.items():
        if f == 'f32':
            continue
        only, only_ref = k.keys() - ref.keys(), ref.keys() - k.keys()
        out[f] = dict(kept=len(k), kept_f32=len(ref), both=len(k.keys() & ref.keys()), only_this=len(only),
                      only_f32=len(only_ref), only_this_away=sum(k[x] > 1.03 * thr for x in only),
                      only_f32_away=sum(ref[x] > 1.03 * thr for x in only_ref))
    return out


def traffic_ratios():
    """Measured DRAM bytes over algorithmic bytes, from the committed ncu summaries (lines 'traffic_ratio: X')."""
    out = {}
    for key, name in (('basis', 'basis_passes_c2_r128.md'), ('gemm', 'umma_cplx2_kernel_c2_r128.md')):
        try:
            for ln in open(os.path.join(os.path.dirname(os.path.abspath(__file__)), 'profiles', name)):
                if ln.startswith('traffic_ratio:'):
                    out[key] = float(ln.split(':')[1])
        except OSError:
            pass
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=3)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='gwb')
    ap.add_argument('--form', default='bf16x3', choices=['bf16x3', 'f16', 'f32'])
    ap.add_argument('--chunks', type=int, default=64, help='chunks per detector')
    ap.add_argument('--templates', type=int, default=5880)
    ap.add_argument('--no-cpu', action='store_true', help='skip the CPU baseline sample')
    ap.add_argument('--no-precision', action='store_true', help='skip the float64 precision comparison')
    ap.add_argument('--forms', default='f16,bf16,fp8,f32', help='forms timed (the first gives value)')
    ap.add_argument('--slow-steps', type=int, default=1,
                    help='timed steps (and warm-up steps) for the plain fp32 form, which is many times slower')
    a = ap.parse_args()
    if a.impl == 'reference':
        run_reference(a)
        return
    import torch
    import torch.distributed as dist
    from gwb200 import _lib, gpu_prep, pipeline, fp_filter
    from gwb200 import dist as gdist
    world = int(os.environ.get('WORLD_SIZE', '1'))
    rank = int(os.environ.get('RANK', '0'))
    local = int(os.environ.get('LOCAL_RANK', '0'))
    torch.cuda.set_device(local)
    dev = torch.device('cuda', local)
    if world > 1:
        import datetime
        dist.init_process_group('nccl', timeout=datetime.timedelta(seconds=300))

    def barrier():
        if world > 1:
            dist.barrier()

    bank = make_bank()
    if a.templates < len(bank['mass1']):
        sel = np.random.default_rng(1).choice(len(bank['mass1']), a.templates, replace=False)
        bank = {k: v[sel] for k, v in bank.items()}
    nch = 2 * a.chunks
    n_inj = int(round(200 * a.chunks / 64))
    x, inj = make_data(nch, bank, n_inj, seed=1000 + rank, device=dev)
    x_host = x.cpu().pin_memory()
    cond = gpu_prep.BatchConditioner(nch, TLEN, SR, F_LOW, 16, 8, 63, 16, device=dev)
    D, IP = cond(x)
    sw, isw = fp_filter.derive_sw(IP)
    sw, isw = sw.clone(), isw.clone()
    forms = a.forms.split(',')
    results = {}
    kept_sets = {}
    torch.cuda.synchronize()
    t_b = time.perf_counter()
    cfg0 = pipeline.FilterConfig(form=forms[0])
    B = pipeline.Bank(bank, FLEN, DF, sw, cfg0, device=dev)
    torch.cuda.synchronize()
    bank_setup = time.perf_counter() - t_b
    analysed = nch * (A1 - A0) / SR
    for form in forms:
        cfg = pipeline.FilterConfig(form=form)
        mf = pipeline.MatchedFilter(B, TLEN, A0, A1 - A0, cfg, device=dev)

        def step():
            Dd, IPd = cond(x)
            mf.step(Dd, IPd, isw)

        nsteps, nwarm = (a.slow_steps, a.slow_steps) if form == 'f32' else (a.steps, a.warmup)
        for _ in range(nwarm):
            step()
        torch.cuda.synchronize()
        res0 = mf.results()
        # kept peaks of the step after the exact stage: (row, segment, window) -> exact SNR
        kc, kp = res0['cands'][res0['keep']], res0['peaks'][res0['keep']]
        kept_sets[form] = dict(zip(zip(kc['row'].tolist(), kc['seg'].tolist(), kc['window'].tolist()),
                                   kp['snr'].tolist()))
        l0c, l0m = cond.launches, mf.kernel_launches
        barrier()
        torch.cuda.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with Clocks(local) as clk:
            ev0.record()
            for _ in range(nsteps):
                step()
            ev1.record()
            torch.cuda.synchronize()
        barrier()
        ms = ev0.elapsed_time(ev1) / nsteps
        launches = (cond.launches - l0c + mf.kernel_launches - l0m) // nsteps
        ms = gdist.max_over_ranks(ms, dev)
        # end to end through the public API: strain from pinned host memory, results back to the host
        res_bytes = 0
        torch.cuda.synchronize()
        barrier()
        e0 = time.perf_counter()
        ee0, ee1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ee0.record()
        for _ in range(nsteps):
            x.copy_(x_host, non_blocking=True)
            step()
            r = mf.results()
            res_bytes = r['n_candidates'] * (32 + 32) + 16
        ee1.record()
        torch.cuda.synchronize()
        barrier()
        ms_e2e = ee0.elapsed_time(ee1) / nsteps
        ms_e2e = gdist.max_over_ranks(ms_e2e, dev)
        # dominant kernel: the fused reconstruction GEMM, each launch bracketed by events in one extra step
        mf.profile = {}
        ec = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        ec[0].record()
        Dd, IPd = cond(x)
        ec[1].record()
        mf.step(Dd, IPd, isw)
        ep = torch.cuda.Event(enable_timing=True)
        ep.record()
        torch.cuda.synchronize()
        L = mf.profile['launches']
        g_ms = [e[1].elapsed_time(e[2]) for e, n, r, kp in L]
        b_ms = [e[0].elapsed_time(e[3]) for e, n, r, kp in L]
        # where the profiled step goes (CUDA events; the events themselves add a little)
        split = dict(conditioning=ec[0].elapsed_time(ec[1]), basis_series=float(np.sum(b_ms)),
                     stacked_a=float(np.sum([e[3].elapsed_time(e[1]) for e, n, r, kp in L])),
                     gemm=float(np.sum(g_ms)))
        sel = [L[i][0][2].elapsed_time(L[i + 1][0][0]) for i in range(len(L) - 1)]
        split['selection'] = float(np.sum(sel))
        for name, (a_, b_) in mf.profile['parts']:
            split[name] = a_.elapsed_time(b_)
        split['total'] = ec[0].elapsed_time(ep)
        split = {k: round(v, 3) for k, v in split.items()}
        # algorithmic HBM bytes of one basis-series call (both passes): Vp read (tlen/2 + 1 complex per row), W
        # written and read back (tlen complex per row), Z written (re + im over Tn, one or two 16-bit planes or fp32)
        zb = {'bf16x3': 8, 'f16': 4, 'bf16': 4, 'f32': 8, 'fp8': 2}[form]
        b_bytes = [r * (8 * (mf.tlen // 2 + 1) + 16 * mf.tlen + zb * mf.Tn) for e, n, r, kp in L]
        useful = [8.0 * n * r * mf.Tn for e, n, r, kp in L]
        nprod = {'bf16x3': 3, 'f16': 1, 'bf16': 1, 'f32': 1, 'fp8': 1}[form]
        issued = [nprod * 4.0 * n * kp * mf.Tn for e, n, r, kp in L]
        mf.profile = None
        val = world * (analysed / WEEK2) / (ms / 1e3 / 3600.0)
        val_e2e = world * (analysed / WEEK2) / (ms_e2e / 1e3 / 3600.0)
        results[form] = dict(value=val, ms=ms, e2e=val_e2e, ms_e2e=ms_e2e, launches=launches, clocks=clk.summary(),
                             n_candidates=res0['n_candidates'], n_kept=int(res0['keep'].sum()),
                             h2d=x.numel() * 4, d2h=res_bytes, gemm_ms=float(np.mean(g_ms)),
                             gemm_total_ms=float(np.sum(g_ms)), basis_total_ms=float(np.sum(b_ms)),
                             basis_ms=float(np.mean(b_ms)), basis_bytes=float(np.mean(b_bytes)),
                             z_bytes=float(np.mean([2 * kp * mf.Tn * {'f32': 4, 'fp8': 1}.get(form, 2) *
                                                    (2 if form == 'bf16x3' else 1) for e, n, r, kp in L])),
                             useful=float(np.mean(useful)), issued=float(np.mean(issued)), n_gemm=len(L),
                             split_ms=split)
        del mf
        torch.cuda.empty_cache()
    # precision of every form against float64 on one (tile, chunk) (after the timed regions; the split bf16 form
    # needs r <= 128, so the tile is the one with the largest such rank)
    precision_rep = None
    if not a.no_precision and rank == 0:
        from gwb200 import precision
        t_p = max((i for i, s_ in enumerate(B.svd) if s_['r'] <= 128), key=lambda i: B.svd[i]['r'])
        seg_p = 0
        Dd, IPd = cond(x)
        precision_rep = dict(tile=t_p, r=B.svd[t_p]['r'], segment=seg_p,
                             reference='float64 transform and product (gwb200.precision)')
        ref = None
        for form in ('f32', 'bf16x3', 'f16', 'bf16', 'fp8'):
            cfg = pipeline.FilterConfig(form=form)
            mf = pipeline.MatchedFilter(B, TLEN, A0, A1 - A0, cfg, device=dev)
            sig = mf.norms(IPd)
            if ref is None:
                r0, n = B.row0[t_p], len(B.tiles[t_p])
                ref = precision.fp64_window_snr(B.svd[t_p], Dd[seg_p], isw, sig[r0:r0 + n, seg_p], DF, TLEN, A0,
                                                mf.Tn, mf.cw)
            v, i = precision.form_window_snr(mf, t_p, Dd, isw, sig, seg_p)
            precision_rep[form] = precision.compare(v, i, ref[0], ref[1], cfg.snr_threshold)
            del mf
            torch.cuda.empty_cache()
    main_form = forms[0]
    R = results[main_form]
    peaks, kind = peaks_file()
    ratios = traffic_ratios()
    # dominant kernel: the fused basis series (basis_pass1_w + basis_pass2_p, one call per (tile, segment)), HBM-bound
    hbm = peaks.get('hbm_gbs', 6650.0)
    b_ach = R['basis_bytes'] / (R['basis_ms'] / 1e3) / 1e9
    b_tr = ratios.get('basis') and ratios['basis'] * R['basis_bytes']
    roof = dict(kernel='basis series: basis_pass1_w + basis_pass2_p (%s)' % main_form, bound='hbm', achieved=b_ach,
                peak=hbm, unit='GB/s', frac=b_ach / hbm, traffic=b_tr, bytes_per_call=R['basis_bytes'],
                avg_call_ms=R['basis_ms'], calls=R['n_gemm'], share_of_step=R['basis_total_ms'] / R['ms'],
                peak_kind='%s hbm copy' % kind,
                traffic_source='profiles/basis_passes_c2_r128.md (dram bytes / algorithmic bytes, scaled)')
    ach = R['useful'] / (R['gemm_ms'] / 1e3) / 1e12
    pk = peaks.get('bf16_tflops', 1590.0) if main_form != 'f32' else None
    g_tr = ratios.get('gemm') and ratios['gemm'] * R['z_bytes']
    gname = {'f16': 'umma_cplx2_kernel (f16, CTA pairs)', 'bf16': 'umma_cplx2_kernel (bf16, CTA pairs)',
             'f32': 'simt_absmax_kernel'}.get(main_form, 'umma_cplx_kernel (%s)' % main_form)
    roof_gemm = dict(kernel=gname,
                     bound='tensor', achieved=ach, peak=pk, unit='TFLOP/s', frac=(ach / pk) if pk else None,
                     traffic=g_tr, flops_per_launch_useful=R['useful'], flops_per_launch_issued=R['issued'],
                     issued_tflops=R['issued'] / (R['gemm_ms'] / 1e3) / 1e12, avg_launch_ms=R['gemm_ms'],
                     launches=R['n_gemm'], share_of_step=R['gemm_total_ms'] / R['ms'],
                     peak_kind='%s burst bf16' % kind,
                     traffic_source='profiles/umma_cplx2_kernel_c2_r128.md (dram bytes / Z bytes, scaled)')
    line = dict(metric=METRIC, value=R['value'], unit='2-det weeks / GPU-hour', n_gpus=world, steps=a.steps,
                warmup=a.warmup, ms_per_step=R['ms'], higher_is_better=True, scaling='weak', vs_baseline=None,
                dtype={'bf16x3': 'bf16 hi+lo (fp32 accumulate)', 'f16': 'f16 (fp32 accumulate)',
                       'bf16': 'bf16 (fp32 accumulate)', 'f32': 'f32',
                       'fp8': 'fp8 e4m3 screen (fp32 accumulate) + float64 exact stage'}[main_form],
                data='synthetic (seeded noise, TaylorF2 bank and injections)',
                config=dict(workload='C2: 2 det x %d chunks x 512 s at 2048 Hz, %d TaylorF2 templates in tiles of 256, '
                                     'eps 1e-3, 16 chi-squared bins' % (a.chunks, len(bank['mass1'])),
                            form=main_form, analysed_s_per_step=analysed, r_over_n=B.r_over_n,
                            r_per_tile=[s_['r'] for s_ in B.svd],
                            l2='inputs larger than L2 (strain 512 MiB, bank 24.7 GB)', parallelism='dp%d' % world),
                e2e=dict(value=R['e2e'], unit='2-det weeks / GPU-hour', h2d_bytes_per_step=R['h2d'],
                         d2h_bytes_per_step=R['d2h']),
                gpu_launches=R['launches'], clocks=R['clocks'], bank_setup_s=bank_setup, roofline=roof,
                roofline_gemm=roof_gemm, precision=precision_rep, top_peak_sets=top_peak_sets(kept_sets, 5.5),
                forms={k: dict(value=v['value'], ms_per_step=v['ms'], e2e=v['e2e'], n_candidates=v['n_candidates'],
                               n_kept=v['n_kept'], gemm_ms_per_launch=v['gemm_ms'], gemm_share=v['gemm_total_ms'] / v['ms'],
                               basis_share=v['basis_total_ms'] / v['ms'], split_ms=v['split_ms'])
                       for k, v in results.items()},
                peaks_source=kind)
    if rank == 0:
        if not a.no_cpu:
            try:
                per_chunk, info = cpu_reference(bank)
                cval = ((A1 - A0) / SR / WEEK2) / (per_chunk / 3600.0)
                line['cpu_baseline'] = dict(value=cval, unit='2-det weeks / hour', cores=os.cpu_count(), kind='port',
                                            sample='one 512 s chunk: conditioning + one tile of 256 templates, '
                                                   'scaled to the full bank', **info)
            except MemoryError as ex:
                line['cpu_baseline'] = dict(value=None, error=repr(ex))
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == '__main__':
    main()
