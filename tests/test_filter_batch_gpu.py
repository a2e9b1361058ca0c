"""gwb_filter_batch (gwb200.cstep.CBatch): raw chunks conditioned and filtered in one C call give the D, IP,
candidates and exact values of the Python conditioning (gpu_prep.BatchConditioner) followed by the C step."""
import numpy as np
import pytest
import torch

from oracle import synth

pytestmark = pytest.mark.gpu

SR = 2048.0
TLEN = 1 << 18
FLEN = TLEN // 2 + 1
DF = SR / TLEN
A0, A1 = 24 * 2048, TLEN - 8 * 2048


def _chunks(bank, seed=3):
    """Two 128 s chunks of noise coloured by the analytic PSD, the first with an SNR 12 injection of row 5."""
    rng = np.random.default_rng(seed)
    f = np.arange(FLEN) * DF
    psd = synth.analytic_psd(f)
    kmin = int(20.0 / DF)
    out = []
    for c in range(2):
        X = np.fft.rfft(rng.standard_normal(TLEN)) * np.sqrt(psd * SR / 2.0)
        X[0] = 0
        if c == 0:
            h = synth.taylorf2(FLEN, DF, bank['mass1'][5], bank['mass2'][5], t0=70.0)
            h[f > synth.f_isco(bank['mass1'][5], bank['mass2'][5])] = 0
            X = X + 12.0 / synth.optimal_snr(h, psd, DF, kmin) * h * SR
        out.append(np.fft.irfft(X, TLEN).astype(np.float32))
    return torch.from_numpy(np.stack(out)).cuda().contiguous()


@pytest.mark.parametrize('form', ['f16', 'bf16x3'])
def test_filter_batch_matches_conditioning_then_step(form):
    from gwb200 import cstep, fp_filter, gpu_prep, pipeline
    bank = synth.random_bank_c1(48, 3)
    x = _chunks(bank)
    cond = gpu_prep.BatchConditioner(2, TLEN, SR, 20.0, 16.0, 8.0, 15, 16.0)
    D, IP = cond(x)
    D, IP = D.clone(), IP.clone()
    sw, isw = fp_filter.derive_sw(IP)
    cfg = pipeline.FilterConfig(tile=24, form=form, snr_threshold=5.0, cand_cap=1 << 16)
    B = pipeline.Bank(bank, FLEN, DF, sw, cfg)
    cs = cstep.CStep(B, TLEN, A0, A1 - A0, 2, cfg)
    sig_s = cs.step(D, IP, isw).clone()
    torch.cuda.synchronize()
    r_s = cs.results()
    cb = cstep.CBatch(B, TLEN, A0, A1 - A0, 2, cfg, psd_seg_len=16.0, psd_seg_stride=8.0, psd_inverse_length=16.0)
    sig_b = cb.batch(x, isw)
    torch.cuda.synchronize()
    r_b = cb.results()
    # the conditioning: the same float32 arithmetic up to the window's last bits
    ip_s, ip_b = IP.double(), cb.IP.double()
    assert ((ip_b - ip_s).abs() <= 1e-6 * ip_s.abs().max()).all()
    assert ((cb.D - D).abs() <= 1e-6 * D.abs().max()).all()
    assert torch.allclose(sig_b, sig_s, rtol=1e-6, atol=0)
    # the step: the same candidates away from the threshold, the same exact values within float32 rounding
    thr2 = (cfg.snr_threshold * (1 - cfg.margin))

    def keyed(r):
        return {(int(c['row']), int(c['seg']), int(c['window'])): (float(c['approx']), float(p['snr']),
                                                                     float(p['chisq']))
                for c, p in zip(r['cands'], r['peaks'])}
    ks, kb = keyed(r_s), keyed(r_b)
    assert len(ks) > 0
    for k in ks.keys() ^ kb.keys():
        v = (ks.get(k) or kb.get(k))[0]
        assert abs(v - thr2) < 1e-3 * thr2, (k, v)
    for k in ks.keys() & kb.keys():
        a, b = ks[k], kb[k]
        assert abs(a[1] - b[1]) <= 1e-4 * a[1] and abs(a[2] - b[2]) <= 1e-3 * max(abs(a[2]), 1.0), (k, a, b)
    # the injection (row 5 of the bank, 70 s into the first chunk) is among the kept peaks of chunk 0
    rows = np.asarray(B.order)[r_b['cands']['row']]
    t = r_b['cands']['sample'] / SR
    near = (rows == 5) & (r_b['cands']['seg'] == 0) & (np.abs(t - 70.0) < 0.1) & r_b['keep']
    assert near.any()
