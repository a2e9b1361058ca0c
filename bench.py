"""Throughput of the B200 matched-filter hot path on the two-detector production workload.

Workload c2 (the default): two detectors (H, L) with independent noise, 64 chunks of 512 s at 2048 Hz each (2^20
samples, one analysis segment per chunk with 48 s / 16 s pads, so 448 s analysed per chunk), Gaussian noise coloured
by the analytic broadband PSD with narrow lines at 60/120/180 Hz, 200 TaylorF2 injections at SNR 6-30; bank of 5,880
templates (4,612 aligned-spin TaylorF2, 1,268 eccentric), SVD-compressed per tile of 256 with eps = 1e-3; 16
chi-squared bins, 1 s windows, candidates above SNR 5.5 (1 - 0.04), exact stage on every candidate. All inputs are
synthetic (seeded); there is no dataset.

One step = the whole hot path over all 128 chunks: conditioning (segment FFT, median-Welch PSD, interpolation,
inverse spectrum truncation, D and IP), template norms, then for every (tile, chunk): basis series, stacked A, the
fused reconstruction GEMM with |z|^2 and windowed argmax, and candidate selection; then the exact stage over every
candidate (edges, binned sums, snr / chisq / newsnr). The bank (templates and tile SVDs) is built once before timing
and reported as bank_setup_s. Metric: two-detector weeks of data filtered per hour of the job (per GPU-hour at one
GPU). The first form of --forms gives the line's value; every other form is timed too (fewer steps) and reported
under `forms`, with the precision of each against float64 over every tile of one chunk. The default first form is
split bf16 (hi + lo, three products, fp32 accumulation): of the mixed forms it is the one whose window SNR maxima stay
within 1e-3 of float64 over every tile and whose kept peaks equal the fp32 form's; fp16 (the reference's own GEMM
precision) comes second.

Workload c4: the batched form (300 science segments of uneven length, gating, graph-replayed batches); c5: the
differentiation form (SNR gradients of 4,096 triggers, the 7 x 7 match metric, 20-step refinement).

The reference arm (--impl reference) times the CPU arm (oracle/cpu_arm.py: the reference's numpy conditioning and
exact stage as restated by the oracle, its tile pass in its own float32 precision with scipy.fft and BLAS over all
host cores) on the same workload, one step = one chunk's conditioning plus one tile of 256 templates against it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--workload c2|c4|c5] [--forms f16,...] [--impl reference]
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
N_TEMPLATES = 5880
METRIC = "2-det weeks filtered per GPU-hour, 5,880 templates, SNR err\u22641e-3: FP32 vs BF16"
UNIT = '2-det weeks / hour'
DYN = 5.9029581035870565e+20
LINES = ((60.0, 1e3, 0.02), (120.0, 1e3, 0.02), (180.0, 1e3, 0.02))
CW = 2048
THR, MARGIN = 5.5, 0.04
DTYPES = {'bf16x3': 'bf16 hi+lo, 3 products (fp32 accumulate)', 'f16': 'f16 (fp32 accumulate)',
          'f16x2': 'f16, A as f16 hi+lo, 2 products (fp32 accumulate)',
          'bf16': 'bf16 (fp32 accumulate)', 'f32': 'f32',
          'fp8': 'fp8 e4m3 screen (fp32 accumulate) + float64 exact stage'}


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


def _plain(o):
    """JSON for the numpy scalars and arrays a report may hold."""
    if isinstance(o, np.generic):
        return o.item()
    if isinstance(o, np.ndarray):
        return o.tolist()
    raise TypeError('not JSON serialisable: %r' % type(o))


def peaks_file():
    p = os.path.join(ROOT, 'MEASURED_PEAKS.json')
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), 'measured'
    return dict(hbm_gbs=6650.0, bf16_tflops=1590.0, bf16_tflops_sustained=1400.0), 'fallback'


# ---------------------------------------------------------------------------------------------------------------------
# CPU arm: one (chunk, tile) sample per step, on every host core
# ---------------------------------------------------------------------------------------------------------------------
CPU_TILES = (0, 11, 22)          # shortest, middle and longest templates of the chirp-time-sorted bank


def cpu_setup(bank, tiles=CPU_TILES, seed=5):
    """The sample tiles (templates, ISCO cut, SVD; bank set-up, not timed) and one chunk of strain."""
    from oracle import cpu_arm, filt, synth
    rng = np.random.default_rng(seed)
    x = np.fft.irfft(synth.coloured_noise(TLEN, SR, rng, synth.LINES_C2), TLEN).astype(np.float32)
    D, IP = cpu_arm.condition(x, SR, CHUNK_S, START_PAD, END_PAD, F_LOW, 16, 8, 63, 16)
    sw, isw = filt.derive_sw(IP[None])
    kmin = int(F_LOW / DF)
    order = np.argsort(synth.tau0(bank['mass1'], bank['mass2']), kind='stable')
    prepared = []
    for t in tiles:
        ids = order[t * 256:(t + 1) * 256]
        H = np.stack([synth.taylorf2(FLEN, DF, bank['mass1'][i], bank['mass2'][i], bank['spin1z'][i],
                                     bank['spin2z'][i], bank['ecc'][i]) for i in ids]).astype(np.complex64)
        kmax = np.array([min(int(np.floor(synth.f_isco(bank['mass1'][i], bank['mass2'][i]) / DF)) + 1, FLEN - 1)
                         for i in ids])
        for j, k in enumerate(kmax):
            H[j, k:] = 0
        r, A, Vh, worst, _, _ = filt.svd_tile(H, sw, kmin, 1e-3)
        prepared.append(dict(tile=t, H=H, kmax=kmax, r=r, A=A, Vh=Vh, n=len(ids)))
    return dict(x=x, isw=isw, kmin=kmin, tiles=prepared, workers=cpu_arm.cores())


def cpu_step(S, i):
    """Step i of the CPU arm: conditioning of the chunk, then sample tile i mod 3 against it (norms, basis series,
    rebuilt SNR window maxima, candidates, float64 exact stage). Returns (seconds, templates filtered)."""
    from oracle import cpu_arm
    T = S['tiles'][i % len(S['tiles'])]
    t0 = time.perf_counter()
    D, IP = cpu_arm.condition(S['x'], SR, CHUNK_S, START_PAD, END_PAD, F_LOW, 16, 8, 63, 16)
    cpu_arm.tile_pass(T['H'], np.full(T['n'], 16), S['kmin'], T['kmax'], T['A'], T['Vh'], D, IP, S['isw'], DF, TLEN,
                      A0, (A1 - A0) // CW * CW, CW, THR, MARGIN, S['workers'])
    return time.perf_counter() - t0, T['n']


def cpu_rate(times, templates):
    """2-det weeks per hour of the CPU samples: each step filtered (A1 - A0) / SR analysed seconds of one chunk
    against `templates` of the N_TEMPLATES-template bank."""
    weeks = sum((A1 - A0) / SR / WEEK2 * (n / N_TEMPLATES) for n in templates)
    return weeks / (sum(times) / 3600.0)


def cpu_sample_desc(S, k):
    return ('%d steps; each: conditioning of one 512 s chunk + one tile of 256 templates (tiles %s of 23 in turn, '
            'r = %s) against it (norms, basis series, rebuilt-SNR window maxima, float64 exact stage); throughput '
            'weighted by the tile\'s share of the %d-template bank' %
            (k, ', '.join(str(t['tile']) for t in S['tiles']), ', '.join(str(t['r']) for t in S['tiles']),
             N_TEMPLATES))


def run_reference(a):
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return
    S = cpu_setup(make_bank())
    for i in range(a.warmup):
        cpu_step(S, i)
    times, tmpl = [], []
    for i in range(a.steps):
        t, n = cpu_step(S, i)
        times.append(t)
        tmpl.append(n)
    val = cpu_rate(times, tmpl)
    desc = cpu_sample_desc(S, a.steps)
    print(json.dumps(dict(metric=METRIC, impl='reference', value=val, unit=UNIT, n_gpus=a.gpus, steps=a.steps,
                          warmup=a.warmup, ms_per_step=float(np.mean(times)) * 1e3, higher_is_better=True,
                          scaling='weak', vs_baseline=None, dtype='f32 (complex64 transforms and products), '
                          'f64 norms and exact stage', data='synthetic (seeded noise, TaylorF2 bank)',
                          config=dict(workload='C2 per-(chunk, tile) sample on the host cores', sample=desc),
                          cpu_baseline=dict(value=val, unit=UNIT, cores=S['workers'], kind='port', sample=desc),
                          e2e=dict(value=val, unit=UNIT, h2d_bytes_per_step=0, d2h_bytes_per_step=0))), flush=True)


# ---------------------------------------------------------------------------------------------------------------------
# C2 on the GPU
# ---------------------------------------------------------------------------------------------------------------------
def top_peak_sets(kept, thr):
    """Each form's kept peaks (exact stage) over the whole step against the plain fp32 form's: windows kept by both,
    by one only, and by one only with an exact SNR more than 3% above the threshold."""
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


# the committed ncu summaries of each form's two dominant kernels (DRAM bytes over algorithmic bytes)
PROFILES = {'basis': {'bf16x3': 'basis_passes_c2_r128_bf16x3.md'},
            'gemm': {'bf16x3': 'umma_cplx2_kernel_c2_r192_bf16x3.md', 'f16': 'umma_cplx_kernel_c2_r128.md',
                     'bf16': 'umma_cplx_kernel_c2_r128.md'}}
BASIS_DEFAULT = 'basis_passes_c2_r128.md'


def traffic_ratios(form):
    """Measured DRAM bytes over algorithmic bytes of the form's basis series and GEMM, from the committed ncu
    summaries (lines 'traffic_ratio: X'); returns ({kernel: ratio}, {kernel: summary file})."""
    out, src = {}, {}
    names = dict(basis=PROFILES['basis'].get(form, BASIS_DEFAULT), gemm=PROFILES['gemm'].get(form))
    for key, name in names.items():
        if name is None:
            continue
        try:
            for ln in open(os.path.join(ROOT, 'profiles', name)):
                if ln.startswith('traffic_ratio:'):
                    out[key] = float(ln.split(':')[1])
                    src[key] = 'profiles/' + name
        except OSError:
            pass
    return out, src


def form_config(form, autotune=False):
    """The filter configuration of a form: the fp8 screen with its exact-stage local search (+-2 samples around the
    screened argmax) and a candidate list for its wider margin."""
    from gwb200 import pipeline
    if form == 'fp8':
        return pipeline.FilterConfig(form=form, screen_search=2, autotune=autotune)
    return pipeline.FilterConfig(form=form, autotune=autotune)


def run_c2(a):
    import torch
    import torch.distributed as dist
    from gwb200 import gpu_prep, pipeline, fp_filter
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
    tunings = {}
    torch.cuda.synchronize()
    t_b = time.perf_counter()
    B = pipeline.Bank(bank, FLEN, DF, sw, pipeline.FilterConfig(form=forms[0]), device=dev)
    torch.cuda.synchronize()
    bank_setup = time.perf_counter() - t_b
    analysed = nch * (A1 - A0) / SR
    for fi, form in enumerate(forms):
        cfg = form_config(form, autotune=not a.no_autotune)
        mf = pipeline.MatchedFilter(B, TLEN, A0, A1 - A0, cfg, device=dev)
        tunings[form] = mf.tuning

        def step():
            Dd, IPd = cond(x)
            mf.step(Dd, IPd, isw)

        # the headline form runs --steps timed steps after --warmup; the comparison forms --form-steps after one
        head = fi == 0
        nsteps = a.steps if head else max(1, min(a.form_steps, a.steps))
        nwarm = a.warmup if head else 1
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
        launches = cond.launches - l0c + mf.kernel_launches - l0m
        ms = gdist.max_over_ranks(ms, dev)
        ms_e2e, res_bytes = None, 0
        if head:
            # end to end through the public API: strain from pinned host memory, results back to the host
            torch.cuda.synchronize()
            barrier()
            ee0, ee1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            ee0.record()
            for _ in range(nsteps):
                x.copy_(x_host, non_blocking=True)
                step()
                r = mf.results()
                res_bytes = r["n_candidates"] * (32 + 32) + 24   # counters, status word, candidates and peaks
            ee1.record()
            torch.cuda.synchronize()
            barrier()
            ms_e2e = gdist.max_over_ranks(ee0.elapsed_time(ee1) / nsteps, dev)
        # one extra step with CUDA events around every (tile, segment) call: where the step goes, and the two
        # dominant kernels (basis series, fused GEMM) per call
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
        # written and read back (tlen complex per row), Z written (re + im over Tn, one or two 16-bit planes, fp32 or
        # fp8)
        zb = {'bf16x3': 8, 'f16': 4, 'f16x2': 4, 'bf16': 4, 'f32': 8, 'fp8': 2}[form]
        b_bytes = [r * (8 * (mf.tlen // 2 + 1) + 16 * mf.tlen + zb * mf.Tn) for e, n, r, kp in L]
        useful = [8.0 * n * r * mf.Tn for e, n, r, kp in L]
        nprod = {'bf16x3': 3, 'f16x2': 2}.get(form, 1)
        issued = [nprod * 4.0 * n * kp * mf.Tn for e, n, r, kp in L]
        mf.profile = None
        val = world * (analysed / WEEK2) / (ms / 1e3 / 3600.0)
        results[form] = dict(value=val, ms=ms, steps=nsteps, warmup=nwarm, launches=launches, clocks=clk.summary(),
                             n_candidates=res0['n_candidates'], n_kept=int(res0['keep'].sum()),
                             h2d=x.numel() * 4, d2h=res_bytes, gemm_ms=float(np.mean(g_ms)),
                             gemm_total_ms=float(np.sum(g_ms)), basis_total_ms=float(np.sum(b_ms)),
                             basis_ms=float(np.mean(b_ms)), basis_bytes=float(np.mean(b_bytes)),
                             z_bytes=float(np.mean([2 * kp * mf.Tn * {'f32': 4, 'fp8': 1}.get(form, 2) *
                                                    (2 if form == 'bf16x3' else 1) for e, n, r, kp in L])),
                             useful=float(np.mean(useful)), issued=float(np.mean(issued)), n_gemm=len(L),
                             split_ms=split)
        if ms_e2e is not None:
            results[form].update(e2e=world * (analysed / WEEK2) / (ms_e2e / 1e3 / 3600.0), ms_e2e=ms_e2e)
        if head:
            # the exact stage with direct loads instead of its bands staged in shared memory by bulk copies (TMA)
            from gwb200 import _lib as glib
            glib.call('gwb_exact_set_staging', 0)
            mf.profile = {}
            Dd, IPd = cond(x)
            mf.step(Dd, IPd, isw)
            torch.cuda.synchronize()
            results[form]['exact_ms_direct'] = [a_.elapsed_time(b_) for nm, (a_, b_) in mf.profile['parts']
                                                if nm == 'exact'][0]
            results[form]['exact_ms_bulk'] = split.get('exact')
            mf.profile = None
            glib.call('gwb_exact_set_staging', 1)
        del mf
        torch.cuda.empty_cache()
    precision_rep = None
    if not a.no_precision and rank == 0:
        import microbench
        precision_rep = microbench.precision_c2(B, cond, x, isw, forms, form_config,
                                                dict(df=DF, tlen=TLEN, a0=A0, an=A1 - A0,
                                                                               cw=CW, thr=THR))
    main_form = forms[0]
    R = results[main_form]
    peaks, kind = peaks_file()
    ratios, rsrc = traffic_ratios(main_form)
    # dominant kernel: the fused basis series (pass 1 + pass 2, one call per (tile, segment)), HBM-bound
    hbm = peaks.get('hbm_gbs', 6650.0)
    b_ach = R['basis_bytes'] / (R['basis_ms'] / 1e3) / 1e9
    b_tr = ratios.get('basis') and ratios['basis'] * R['basis_bytes']
    # the pass-2 kernel the headline form ran with: its tuned column count (the library default, 16, untuned)
    tb = tunings.get(main_form)
    cols = ((tb or {}).get('basis') or {}).get('best', {}).get('pass2_cols') or 16
    p2 = 'basis_pass2_w' if cols == 16 else 'basis_pass2 (per row)' if main_form == 'bf16x3' else 'basis_pass2_p'
    roof = dict(kernel='basis series: basis_pass1_w + %s (%s)' % (p2, main_form), bound='hbm', achieved=b_ach,
                peak=hbm, unit='GB/s', frac=b_ach / hbm, traffic=b_tr, bytes_per_call=R['basis_bytes'],
                avg_call_ms=R['basis_ms'], calls=R['n_gemm'], share_of_step=R['basis_total_ms'] / R['ms'],
                peak_kind='%s hbm copy' % kind,
                traffic_source='%s (dram bytes / algorithmic bytes, scaled)' % rsrc.get('basis'))
    # the fused GEMM, timed inside a seconds-long step: against the sustained bf16 peak (the burst one beside it).
    # Algorithmic flop of a launch: 8 n r Tn per product (the split form computes three), without the K padding
    nprod = {'bf16x3': 3, 'f16x2': 2}.get(main_form, 1)
    ach = nprod * R['useful'] / (R['gemm_ms'] / 1e3) / 1e12
    pk = peaks.get('bf16_tflops_sustained', peaks.get('bf16_tflops', 1590.0)) if main_form != 'f32' else None
    pkb = peaks.get('bf16_tflops') if main_form != 'f32' else None
    g_tr = ratios.get('gemm') and ratios['gemm'] * R['z_bytes']
    gname = {'f32': 'simt_absmax_kernel'}.get(main_form, 'umma_cplx_kernel / umma_cplx2_kernel (%s, the launch '
                                                         'shape the autotuner picked per Kh)' % main_form)
    roof_gemm = dict(kernel=gname,
                     bound='tensor', achieved=ach, peak=pk, unit='TFLOP/s', frac=(ach / pk) if pk else None,
                     frac_of_burst=(ach / pkb) if pkb else None,
                     traffic=g_tr, products=nprod, flops_per_launch_algorithmic=nprod * R['useful'],
                     flops_per_launch_useful=R['useful'], flops_per_launch_issued=R['issued'],
                     useful_tflops=R['useful'] / (R['gemm_ms'] / 1e3) / 1e12,
                     issued_tflops=R['issued'] / (R['gemm_ms'] / 1e3) / 1e12, avg_launch_ms=R['gemm_ms'],
                     launches=R['n_gemm'], share_of_step=R['gemm_total_ms'] / R['ms'],
                     peak_kind='%s sustained bf16 (cuBLAS loop under the power cap)' % kind,
                     traffic_source='%s (dram bytes / Z bytes, scaled)' % rsrc.get('gemm'))
    fp32 = results.get('f32')
    line = dict(metric=METRIC, value=R['value'], unit=UNIT, n_gpus=world, steps=a.steps,
                warmup=a.warmup, ms_per_step=R['ms'], higher_is_better=True, scaling='weak', vs_baseline=None,
                dtype=DTYPES[main_form],
                data='synthetic (seeded noise, TaylorF2 bank and injections)',
                config=dict(workload='C2: 2 det x %d chunks x 512 s at 2048 Hz, %d TaylorF2 templates in tiles of 256, '
                                     'eps 1e-3, 16 chi-squared bins' % (a.chunks, len(bank['mass1'])),
                            form=main_form, analysed_s_per_step=analysed, r_over_n=B.r_over_n,
                            r_per_tile=[s_['r'] for s_ in B.svd], unit_note='per GPU-hour at n_gpus = 1',
                            l2='inputs larger than L2 (strain 512 MiB, bank 24.7 GB)', parallelism='dp%d' % world),
                e2e=dict(value=R['e2e'], unit=UNIT, h2d_bytes_per_step=R['h2d'], d2h_bytes_per_step=R['d2h']),
                gpu_launches=R['launches'], gpu_launches_per_step=R['launches'] // max(1, R['steps']),
                clocks=R['clocks'], bank_setup_s=bank_setup, roofline=roof,
                roofline_gemm=roof_gemm, precision=precision_rep, top_peak_sets=top_peak_sets(kept_sets, THR),
                mixed_over_fp32={k: v['value'] / fp32['value'] for k, v in results.items() if k != 'f32'}
                if fp32 else None,
                forms={k: dict(value=v['value'], ms_per_step=v['ms'], steps=v['steps'], warmup=v['warmup'],
                               e2e=v.get('e2e'), n_candidates=v['n_candidates'], n_kept=v['n_kept'],
                               gemm_ms_per_launch=v['gemm_ms'], gemm_share=v['gemm_total_ms'] / v['ms'],
                               basis_share=v['basis_total_ms'] / v['ms'], clocks=v['clocks'], split_ms=v['split_ms'],
                               exact_ms_direct=v.get('exact_ms_direct'), exact_ms_bulk=v.get('exact_ms_bulk'))
                       for k, v in results.items()},
                peaks_source=kind,
                autotune={f: (None if t is None else dict(gemm={str(k): v['best'] for k, v in t['gemm'].items()},
                                                            basis=t['basis'] and t['basis']['best']))
                          for f, t in tunings.items()})
    if rank == 0 and world == 1 and not a.no_c4:
        # the batched form (300 uneven segments, autogating, the whole run as one graph) on the same bank and GPU
        import microbench
        try:
            ns = argparse.Namespace(segments=300, batch=32, seed=4, no_graph=False, production=False,
                                    form='bf16x3', bank_obj=B, isw=isw, autotune=not a.no_autotune)
            r4 = microbench.c4(ns)
            line['c4'] = {k: r4[k] for k in ('workload', 'value', 'unit', 'ms', 'analysed_s', 'chunks', 'batches',
                                             'one_graph', 'graph_capture_s', 'glitches', 'glitches_gated',
                                             'injections_snr8_in_analysed', 'injections_found')}
        except Exception as ex:     # reported in the line; the C2 measurement above stands
            line['c4'] = dict(error=repr(ex)[:300])
        torch.cuda.empty_cache()
    if rank == 0 and world == 1 and not a.no_cpu:
        S = cpu_setup(bank if len(bank['mass1']) == N_TEMPLATES else make_bank())
        cpu_step(S, 0)
        times, tmpl = [], []
        for i in range(a.cpu_steps):
            t, n = cpu_step(S, i)
            times.append(t)
            tmpl.append(n)
        line['cpu_baseline'] = dict(value=cpu_rate(times, tmpl), unit=UNIT, cores=S['workers'], kind='port',
                                    sample=cpu_sample_desc(S, a.cpu_steps) + ' (after one untimed step)',
                                    ms_per_step=float(np.mean(times)) * 1e3)
    if rank == 0:
        print(json.dumps(line, default=_plain), flush=True)
    if world > 1:
        dist.destroy_process_group()


# ---------------------------------------------------------------------------------------------------------------------
# C4 (batched segments) and C5 (differentiation)
# ---------------------------------------------------------------------------------------------------------------------
def run_c4(a):
    import microbench
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return
    # the batched form's configuration names the split-bf16 GEMM; --forms overrides it
    form = a.forms.split(',')[0] if a.forms_given else 'bf16x3'
    ns = argparse.Namespace(segments=300, batch=32, seed=4, no_graph=False, production=a.production, form=form,
                            autotune=not a.no_autotune)
    r = microbench.c4(ns)
    print(json.dumps(dict(metric=METRIC, value=r['value'], unit=UNIT, n_gpus=1, steps=1, warmup=1,
                          ms_per_step=r['ms'], higher_is_better=True, scaling='weak', vs_baseline=None,
                          dtype=DTYPES[ns.form], data='synthetic (seeded noise, TaylorF2 bank and injections, '
                          'sine-Gaussian glitches)', config=dict(workload=r['workload']), c4=r)), flush=True)


def run_c5(a):
    import microbench
    rank = int(os.environ.get('RANK', '0'))
    if rank != 0:
        return
    ns = argparse.Namespace(triggers=4096, reps=max(3, a.steps))
    r = microbench.adjoint(ns)
    print(json.dumps(dict(metric='SNR gradients per second (7 parameters, 16 s triggers)',
                          value=r['triggers_per_s_fp32'], unit='triggers / s', n_gpus=1, steps=ns.reps, warmup=2,
                          ms_per_step=r['ms_grad_fp32'], higher_is_better=True, scaling='weak', vs_baseline=None,
                          dtype='f32 sums, f64 phase', data='synthetic', config=dict(workload='C5: 4,096 triggers '
                          'x 16 s at 2048 Hz'), c5=r)), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--gpus', type=int, default=1)
    ap.add_argument('--steps', type=int, default=3)
    ap.add_argument('--warmup', type=int, default=3)
    ap.add_argument('--impl', default='gwb', choices=['gwb', 'reference'])
    ap.add_argument('--workload', default='c2', choices=['c2', 'c4', 'c5'])
    ap.add_argument('--chunks', type=int, default=64, help='chunks per detector')
    ap.add_argument('--templates', type=int, default=N_TEMPLATES)
    ap.add_argument('--no-cpu', action='store_true', help='skip the CPU baseline sample')
    ap.add_argument('--cpu-steps', type=int, default=3, help='timed steps of the CPU baseline sample')
    ap.add_argument('--no-precision', action='store_true', help='skip the float64 precision comparison')
    ap.add_argument('--forms', default='bf16x3,f16x2,f16,bf16,fp8,f32', help='forms timed (the first gives value)')
    ap.add_argument('--form-steps', type=int, default=3, help='timed steps of each form after the first')
    ap.add_argument('--production', action='store_true', help='c4: production selection and consolidation')
    ap.add_argument('--no-autotune', action='store_true', help='c2, c4: default launch shapes instead of tuned ones')
    ap.add_argument('--no-c4', action='store_true', help='c2: skip the batched-form run reported under "c4"')
    a = ap.parse_args()
    a.forms_given = any(x == '--forms' or x.startswith('--forms=') for x in sys.argv[1:])
    if a.impl == 'reference':
        run_reference(a)
    elif a.workload == 'c2':
        run_c2(a)
    elif a.workload == 'c4':
        run_c4(a)
    else:
        run_c5(a)


if __name__ == '__main__':
    main()
