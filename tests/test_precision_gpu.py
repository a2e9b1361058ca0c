"""Precision of each arithmetic form against float64 (microbench.py) on the small pipeline case: window maxima of
the SNR from the fused GEMM against the float64 series (float64 transform and product)."""
import pytest
import torch

from test_pipeline_gpu import A0, A1, DF, FLEN, TLEN, _case

pytestmark = pytest.mark.gpu

# bound on the relative SNR error of each form (operand rounding: fp16 11 bits, bf16 8, split bf16 about 16, fp32 24)
TOL = {'f32': 1e-4, 'bf16x3': 2e-4, 'f16': 3e-3, 'bf16': 2e-2}


def test_forms_against_float64():
    import microbench as precision
    from gwb200 import fp_filter, pipeline
    bank, D, IP, kmin, inj = _case()
    Dd, IPd = torch.from_numpy(D).cuda(), torch.from_numpy(IP).cuda()
    sw, isw = fp_filter.derive_sw(IPd)
    B = pipeline.Bank(bank, FLEN, DF, sw, pipeline.FilterConfig(tile=24, form='f16'))
    t, seg = 0, inj['seg']
    ref = None
    for form in ('f32', 'bf16x3', 'f16', 'bf16'):
        cfg = pipeline.FilterConfig(tile=24, form=form)
        mf = pipeline.MatchedFilter(B, TLEN, A0, A1 - A0, cfg)
        sig = mf.norms(IPd)
        if ref is None:
            r0, n = B.row0[t], len(B.tiles[t])
            ref = precision.fp64_window_snr(B.svd[t], Dd[seg], isw, sig[r0:r0 + n, seg], DF, TLEN, A0, mf.Tn, mf.cw)
        v, i = precision.form_window_snr(mf, t, Dd, isw, sig, seg)
        c = precision.compare(v, i, ref[0], ref[1], cfg.snr_threshold)
        assert c['max_rel'] < TOL[form], (form, c)
        assert c['set_diff_away'] == 0, (form, c)
        if form in ('f32', 'bf16x3'):
            assert c['argmax_agree'] > 0.98, (form, c)
        else:
            assert c['argmax_within2'] > 0.9, (form, c)


def test_fp64_exact_reference_matches_the_oracle():
    """The float64 exact stage the precision report compares against (microbench.fp64_exact_at, torch complex128 on
    the device) equals the oracle's dense exact stage (oracle/chisq.py exact_dense + oracle/filt.py finalize) at the
    same (row, sample) pairs, to float64 rounding."""
    import numpy as np
    import microbench
    from oracle import chisq as oc
    from oracle import filt as of
    from gwb200 import fp_filter, pipeline
    bank, D, IP, kmin, inj = _case()
    Dd, IPd = torch.from_numpy(D).cuda(), torch.from_numpy(IP).cuda()
    sw, isw = fp_filter.derive_sw(IPd)
    B = pipeline.Bank(bank, FLEN, DF, sw, pipeline.FilterConfig(tile=24, form='f16'))
    mf = pipeline.MatchedFilter(B, TLEN, A0, A1 - A0, pipeline.FilterConfig(tile=24, form='f16'))
    sig = mf.norms(IPd).cpu().numpy()
    rng = np.random.default_rng(7)
    seg = inj['seg']
    rows = rng.integers(0, B.M, 40)
    samples = rng.integers(0, TLEN, 40)
    nb = np.full(B.M, 16)
    snr, chi = microbench.fp64_exact_at(B.H, rows, samples, Dd[seg], IPd[seg], B.kmin, B.kmax_h, nb, sig[:, seg],
                                        DF, TLEN)
    H = B.H.cpu().numpy()
    z, pw, _, _ = oc.exact_dense(H, nb, B.kmin, B.kmax_h, D[seg], IP[seg], DF, TLEN, rows, samples)
    snr_o, chi_o, _ = of.finalize(z, pw, 4.0 * DF / np.sqrt(sig[rows, seg]), nb[rows])
    np.testing.assert_allclose(snr, snr_o, rtol=1e-9)
    np.testing.assert_allclose(chi, chi_o, rtol=1e-8, atol=1e-9 * np.abs(chi_o).max())
