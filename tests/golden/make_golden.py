"""Writes the golden fixtures in this directory by running the reference's own code on seeded inputs.

Run from the repository root on a machine where the reference checkout is present (it is read, never modified);
its location is given with --ref or the GWB_REFERENCE environment variable:

    python tests/golden/make_golden.py --ref PATH_TO_REFERENCE [--only NAME ...]

Each fixture holds the inputs and the reference's outputs for one call. The reference functions used:
  fp_gemm_*.npz      pipeline/fp_gemm.py fused_peaks (the Triton kernel under TRITON_INTERPRET=1, on the CPU)
  prep_stage2.npz    pipeline/gpu_prep.py gpu_stage2 with xp = numpy (welch, interpolate, truncation, D, IP)
  prep_gating.npz    pipeline/gpu_prep.py detect_loud_glitches + gate_taper with xp = numpy; lal is absent here, so
                     LIGOTimeGPS is replaced by _GPS below (integer nanoseconds, halves rounded up, int() = floor)
  filt_tile.npz      pipeline/fp_filter.py closures svd_tile, basis_series, stacked_A (source text run with exec in a
                     prepared namespace, as the reference's tests/test_prekeep.py does), torch on the CPU
  edges_exact.npz    pipeline/multi_filter.py edges_per_template, pipeline/chisq_edges.py edges_blocked (numpy) and
                     pipeline/exact_stage.py ExactStage.evaluate on the dense numpy backend
  consolidate.npz    pipeline/fp_filter.py closures consolidate and pre_keep (source text run with exec, torch on the
                     CPU); PyCBC is absent here, so its newsnr is the oracle's restatement (oracle/consolidate.py)
The tests compare the oracle (oracle/) against these files on the CPU, and the CUDA kernels against the oracle and
the files on the GPU. Nothing at test time reads the reference."""
import argparse
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_REF = {}


def _ref_path(ref):
    p = os.path.join(ref, 'pipeline')
    if not os.path.isdir(p):
        raise SystemExit('reference pipeline not found at %s' % p)
    if p not in sys.path:
        sys.path.insert(0, p)
    sys.modules.setdefault('h5py', types.ModuleType('h5py'))   # multi_filter imports h5py at module level
    _REF['pipeline'] = p
    return p


def gen_fp_gemm():
    os.environ['TRITON_INTERPRET'] = '1'
    import torch
    import fp_gemm
    cases = {
        'fp_gemm_a': dict(M=64, K=64, Tn=1024, cfg=(64, 32, 4, 2), seed=1, kind='normal'),
        'fp_gemm_ragged': dict(M=150, K=128, Tn=1000, cfg=(64, 64, 4, 2), seed=2, kind='normal'),
        'fp_gemm_ties': dict(M=64, K=64, Tn=640, cfg=(64, 64, 4, 2), seed=3, kind='ints'),
    }
    for name, c in cases.items():
        rng = np.random.default_rng(c['seed'])
        if c['kind'] == 'ints':
            # small integers: every product and sum is exact in fp32, so ties are real and the first index must win
            Are = rng.integers(-2, 3, (c['M'], c['K'])).astype(np.float16)
            Aim = rng.integers(-2, 3, (c['M'], c['K'])).astype(np.float16)
            Z = rng.integers(-1, 2, (c['K'], c['Tn'])).astype(np.float16)
        else:
            Are = rng.standard_normal((c['M'], c['K'])).astype(np.float16)
            Aim = rng.standard_normal((c['M'], c['K'])).astype(np.float16)
            Z = rng.standard_normal((c['K'], c['Tn'])).astype(np.float16)
        V, I = fp_gemm.fused_peaks(torch.from_numpy(Are), torch.from_numpy(Aim), torch.from_numpy(Z), c['M'], c['Tn'],
                                   c['cfg'])
        np.savez_compressed(os.path.join(HERE, name + '.npz'), Are=Are, Aim=Aim, Z=Z, V=V.numpy(), I=I.numpy(),
                            M=c['M'], Tn=c['Tn'])
        print(name, V.shape)


class _GPS:
    """Stand-in for lal.LIGOTimeGPS in the reference's gating code: integer nanoseconds."""

    def __init__(self, t=0, ns=None):
        self.ns = int(ns) if ns is not None else (t.ns if isinstance(t, _GPS) else self._from_float(t))

    @staticmethod
    def _from_float(t):
        if isinstance(t, (int, np.integer)):
            return int(t) * 1000000000
        return int(np.floor(float(t) * 1e9 + 0.5))

    def _o(self, x):
        return x.ns if isinstance(x, _GPS) else self._from_float(x)

    def __add__(self, x):
        return _GPS(ns=self.ns + self._o(x))

    __radd__ = __add__

    def __sub__(self, x):
        return _GPS(ns=self.ns - self._o(x))

    def __rsub__(self, x):
        return _GPS(ns=self._o(x) - self.ns)

    def __mul__(self, x):
        return _GPS(ns=int(np.floor(self.ns * float(x) + 0.5)))

    __rmul__ = __mul__

    def __int__(self):
        return self.ns // 1000000000

    def __float__(self):
        return self.ns / 1e9

    def __gt__(self, x):
        return self.ns > self._o(x)

    def __lt__(self, x):
        return self.ns < self._o(x)


def _lal_stub():
    lal = types.ModuleType('lal')
    lal.LIGOTimeGPS = _GPS
    sys.modules['lal'] = lal


def _prep_argv(gps0, dur):
    return ['--hdf-store', 'none', '--gps-start-time', str(gps0), '--gps-end-time', str(gps0 + dur), '--pad-data', '0',
            '--sample-rate', '2048', '--low-frequency-cutoff', '20', '--segment-length', '32',
            '--segment-start-pad', '4', '--segment-end-pad', '4', '--psd-estimation', 'median',
            '--psd-segment-length', '4', '--psd-segment-stride', '2', '--psd-num-segments', '15',
            '--psd-inverse-length', '4', '--strain-high-pass', '15', '--autogating-threshold', '50']


def gen_prep():
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from oracle import synth
    _lal_stub()
    import gpu_prep
    sr, dur, gps0 = 2048, 64, 1000000000
    rng = np.random.default_rng(10)
    n = sr * dur
    X = synth.coloured_noise(n, sr, rng, synth.LINES_C2)
    s = np.fft.irfft(X, n).astype(np.float32)
    argv = _prep_argv(gps0, dur)
    out = gpu_prep.gpu_stage2(np, s.copy(), argv)
    np.savez_compressed(os.path.join(HERE, 'prep_stage2.npz'), strain=s, argv=np.array(argv), D=out['D'],
                        IP=out['IP'], analyze=np.array(out['analyze']), seg_start=np.array(out['seg_start']),
                        flen=out['flen'], tlen=out['tlen'], df=out['df'])
    print('prep_stage2', out['D'].shape)
    # gating: two loud sine-Gaussians, one near the edge of the corrupt zone, on 64 s of noise
    g = s.copy()
    for tc, f0, a in ((20.3, 80.0, 40.0), (41.77, 150.0, 25.0)):
        g += synth.sine_gaussian(n, sr, tc, f0, 10.0, a).astype(np.float32)
    gates_t = gpu_prep.detect_loud_glitches(np, g, sr, gps0, 50.0, 0.5, 15.0, 0.0 + 16, 4.0, 2.0)
    gates = [(t, 0.25, 0.25) for t in gates_t]
    gated = gpu_prep.gate_taper(np, g.copy(), sr, gps0, gates)
    np.savez_compressed(os.path.join(HERE, 'prep_gating.npz'), strain=g, gated=gated, sr=sr, gps0=gps0,
                        gate_ns=np.array([t.ns for t in gates_t], np.int64))
    print('prep_gating', len(gates_t), 'gates')


def _small_tile(seed=20, n=16, tlen=1 << 14, sr=2048.0, mrange=(8.0, 30.0)):
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from oracle import synth
    rng = np.random.default_rng(seed)
    flen = tlen // 2 + 1
    df = sr / tlen
    m = rng.uniform(mrange[0], mrange[1], (n, 2))
    m1, m2 = m.max(1), m.min(1)
    H = np.stack([synth.taylorf2(flen, df, a, b, f_low=20.0) for a, b in zip(m1, m2)]).astype(np.complex64)
    f = np.arange(flen) * df
    psd = synth.analytic_psd(f, synth.LINES_C2)
    kmin = int(20.0 / df)
    IP = np.zeros(flen, np.float32)
    IP[kmin:] = (1.0 / psd[kmin:]).astype(np.float32)
    X = synth.coloured_noise(tlen, sr, rng, synth.LINES_C2) / sr      # stilde = rfft(x) dt
    sig = 4 * df * (np.abs(H.astype(np.complex128)) ** 2 @ IP.astype(np.float64))
    t0 = 0.6 * tlen / sr
    X = X + 12.0 / np.sqrt(sig[3]) * H[3].astype(np.complex128) * np.exp(-2j * np.pi * f * t0)
    D = (X * IP).astype(np.complex64)
    kend = np.minimum((synth.f_isco(m1, m2) / df).astype(np.int64), flen - 1)
    return dict(H=H, IP=IP, D=D, df=df, tlen=tlen, flen=flen, kmin=kmin, kmax=kend, m1=m1, m2=m2, t0=t0)


def _fp_filter_closures(ns):
    src = open(os.path.join(_REF['pipeline'], 'fp_filter.py')).read().splitlines()
    a = next(i for i, l in enumerate(src) if l.strip().startswith('def svd_tile(H):'))
    b = next(i for i, l in enumerate(src) if l.strip().startswith('cons_pool = ThreadPoolExecutor(1)'))
    import textwrap
    exec(textwrap.dedent('\n'.join(src[a:b])), ns)
    return ns


def gen_filt():
    import torch
    T = _small_tile(mrange=(9.0, 11.0))
    sw = np.sqrt(T['IP'].astype(np.float64)).astype(np.float32)   # one segment: sw = sqrt(IP)
    isw = np.where(sw > 0, 1.0 / np.maximum(sw, 1e-30), 0.0).astype(np.float32)
    ns = dict(torch=torch, dev='cpu', kmin=T['kmin'], flen=T['flen'], tlen=T['tlen'], CH=1 << 16, RB=64,
              sw=torch.from_numpy(sw), eps_b=1e-3)
    _fp_filter_closures(ns)
    H = torch.from_numpy(T['H'])
    r, A, Vh, worst = ns['svd_tile'](H)
    a0, Tn = 2048, 2048 * 5
    Dws = torch.from_numpy(T['D']) * torch.from_numpy(isw)
    Z, scale = ns['basis_series'](Vh, Dws, a0, Tn)
    sig = 4 * T['df'] * (np.abs(T['H'].astype(np.complex128)) ** 2 @ T['IP'].astype(np.float64))
    nrm_s = torch.from_numpy((4 * T['df'] / np.sqrt(sig)).astype(np.float32))
    Are, Aim = ns['stacked_A'](A, nrm_s, scale, Z.shape[0])
    np.savez_compressed(os.path.join(HERE, 'filt_tile.npz'), H=T['H'], IP=T['IP'], D=T['D'], sw=sw, isw=isw,
                        kmin=T['kmin'], tlen=T['tlen'], df=T['df'], r=r, A=A.numpy(), Vh=Vh.numpy(), worst=worst,
                        a0=a0, Tn=Tn, Z=Z.numpy(), scale=scale, nrm_s=nrm_s.numpy(), Are=Are.numpy(),
                        Aim=Aim.numpy(), eps=1e-3, t0=T['t0'])
    print('filt_tile r', r, 'worst', worst, 'scale', scale)


def gen_edges_exact():
    import multi_filter
    import chisq_edges
    import exact_stage
    T = _small_tile(seed=21)
    n = T['H'].shape[0]
    rng = np.random.default_rng(22)
    nbins = rng.integers(2, 20, n)
    nbins[5] = 0                      # a template without chi-squared bins (one bin over the band)
    rows = np.arange(n)
    E_full = multi_filter.edges_per_template(np, rows, np.maximum(nbins, 1), T['kmin'], T['kmax'], T['H'], T['IP'])
    E_blk = chisq_edges.edges_blocked(np, rows, np.maximum(nbins, 1), T['kmin'], T['kmax'], T['H'], T['IP'])
    assert np.array_equal(E_full, E_blk)
    tile = exact_stage.TemplateTile(T['H'], nbins, T['kmin'], T['kmax'])
    stage = exact_stage.ExactStage(tile)
    seg = exact_stage.SegmentData(T['D'], T['IP'], T['df'], T['tlen'])
    counts = [1, 2, 3, 8, 9, 12, 1, 5, 4, 7, 2, 3, 6, 1, 10, 2]
    prow, psamp = [], []
    for r_, c in zip(rows, counts):
        prow += [r_] * c
        psamp += list(rng.integers(0, T['tlen'], c))
    prow += [0, 1, 1, 3]
    psamp += [psamp[0], 0, T['tlen'] - 1, int(T['t0'] * 2048)]
    perm = rng.permutation(len(prow))
    prow, psamp = np.array(prow)[perm], np.array(psamp)[perm]
    pv = stage.evaluate(seg, exact_stage.PeakRequest(prow, psamp))
    np.savez_compressed(os.path.join(HERE, 'edges_exact.npz'), H=T['H'], IP=T['IP'], D=T['D'], df=T['df'],
                        tlen=T['tlen'], kmin=T['kmin'], kmax=T['kmax'], nbins=nbins, E=E_full, rows=prow,
                        samples=psamp, z=pv.z, pw=pv.pw, fpeak=pv.fpeak)
    print('edges_exact', E_full.shape, len(prow), 'peaks')


def _closure(name):
    """Source of one closure of fp_filter.py's main (indentation-delimited), dedented."""
    import textwrap
    src = open(os.path.join(_REF['pipeline'], 'fp_filter.py')).read().splitlines()
    i = next(k for k, l in enumerate(src) if l.strip().startswith('def %s(' % name))
    ind = len(src[i]) - len(src[i].lstrip())
    out = [src[i]]
    for l in src[i + 1:]:
        if l.strip() and len(l) - len(l.lstrip()) <= ind:
            break
        out.append(l)
    return textwrap.dedent('\n'.join(out))


def gen_consolidate():
    """Seeded cases of the reference's consolidate (keep mask, floor) and pre_keep (mask): SNRs rounded to 0.01 so
    that ties are frequent, windows crowded (20 s spans) or sparse (800 s), 0-3 gates, exempt SNR 5 or none, keep
    1-6 or 30 loudest per 1.072 s window or no ranking, with and without chi-squared."""
    import time
    import torch
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from oracle.consolidate import newsnr
    src_c, src_p = _closure('consolidate'), _closure('pre_keep')
    rng = np.random.default_rng(30)
    sr, gps0 = 2048.0, 1380077576.0
    seg_start = [0, 1636352]
    out = {}
    nc = npk = 0
    for trial in range(60):
        interval = None if trial % 7 == 3 else 1.072
        num = int(rng.choice([1, 2, 3, 5, 6, 30]))
        exempt = [5.0, None][trial % 2]
        do_chisq = trial % 11 != 5
        a = types.SimpleNamespace(pre_consolidate=True, exact_snr=5.5, margin=0.04, consolidate_exempt_snr=exempt)
        klo = types.SimpleNamespace(newsnr_threshold=4.0, keep_loudest_interval=interval, keep_loudest_num=num,
                                    keep_loudest_stat='newsnr')
        g = dict(time=time, a=a, klo=klo, sr=sr, thr=4.0, T={}, dev='cpu', torch=torch, np=np, newsnr=newsnr,
                 do_chisq=do_chisq)
        exec(src_c, g)
        exec(src_p, g)
        gates = [(gps0 + float(rng.uniform(0, 1500)), 0.25, 0.25) for _ in range(int(rng.integers(0, 4)))]
        span = float(rng.choice([20.0, 800.0]))
        # consolidate: peaks of one dataset, rebuilt (dof 0) and exact (dof 30) mixed
        n = int(rng.choice([0, 1, 7, 300, 3000]))
        ti = rng.integers(0, int(span * sr), n) + seg_start[int(rng.integers(0, 2))]
        t = gps0 + ti / sr
        snr = np.round(rng.uniform(3.84, 9.0, n), 2).astype(np.float32)
        isex = rng.uniform(size=n) < 0.4
        chi = np.where(isex, np.round(rng.uniform(0, 80, n), 1), 0).astype(np.float32)
        dof = np.where(isex, 30, 0).astype(np.int32)
        m = dict(gps_start=gps0, gates=gates,
                 out=dict(snr=[snr], chi=[chi], dof=[dof], t=[t], idx=[np.arange(n)]))
        g['consolidate'](m)
        kept = np.concatenate(m['out']['idx']) if m['out']['idx'] else np.zeros(0, np.int64)
        keep = np.zeros(n, bool)
        keep[kept] = True
        floor = m['floor'].numpy() if 'floor' in m else np.zeros(0)
        pre = 'c%d_' % nc
        nc += 1
        out.update({pre + 'ti': ti, pre + 'snr': snr, pre + 'chi': chi, pre + 'dof': dof,
                    pre + 'gates': np.array(gates, np.float64).reshape(-1, 3),
                    pre + 'par': np.array([interval or 0.0, num, -1.0 if exempt is None else exempt, do_chisq,
                                           4.0]),
                    pre + 'keep': keep, pre + 'floor': floor})
        # pre_keep on a new part of the same dataset, against the floor that consolidate left
        s = int(rng.integers(0, 2))
        k = int(rng.choice([0, 5, 500, 3000]))
        samp = rng.integers(0, int(span * sr), k).astype(np.int32)
        apx = np.round(rng.uniform(3.84, 7.0, k), 2).astype(np.float32)
        mp = dict(gps_start=gps0, seg_start=seg_start, gates=gates)
        if 'floor' in m and trial % 3:
            mp['floor'] = m['floor']
        kp = g['pre_keep'](mp, s, torch.from_numpy(samp), torch.from_numpy(apx)).numpy()
        pre = 'p%d_' % npk
        npk += 1
        out.update({pre + 'ti': samp.astype(np.int64) + seg_start[s], pre + 'apx': apx,
                    pre + 'gates': np.array(gates, np.float64).reshape(-1, 3),
                    pre + 'par': np.array([interval or 0.0, num, -1.0 if exempt is None else exempt, 5.5, 0.04, 4.0,
                                           4.0]),
                    pre + 'floor': mp['floor'].numpy() if 'floor' in mp else np.zeros(0), pre + 'has_floor':
                    np.array('floor' in mp), pre + 'keep': kp})
    out.update(n_cons=nc, n_pre=npk, sr=sr, gps0=gps0)
    np.savez_compressed(os.path.join(HERE, 'consolidate.npz'), **out)
    print('consolidate', nc, 'consolidate cases,', npk, 'pre_keep cases')


GENERATORS = {'fp_gemm': gen_fp_gemm, 'prep': gen_prep, 'filt': gen_filt, 'edges_exact': gen_edges_exact,
              'consolidate': gen_consolidate}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument('--ref', default=os.environ.get('GWB_REFERENCE'),
                    help='root of the reference checkout (the directory holding pipeline/); default $GWB_REFERENCE')
    ap.add_argument('--only', nargs='*')
    a = ap.parse_args()
    if not a.ref:
        ap.error('the reference checkout is required: --ref PATH or GWB_REFERENCE=PATH')
    _ref_path(a.ref)
    for name, fn in GENERATORS.items():
        if a.only and name not in a.only:
            continue
        fn()


if __name__ == '__main__':
    main()
