"""The autotuner (gwb200.autotune) and the drop-in pick_cfg: every launch configuration they choose between gives the
same V and I (so tuning changes speed only), the chosen one is written into the library's launch table, and a
MatchedFilter built with autotune=True finds the same candidates and exact values as one without."""
import numpy as np
import pytest
import torch

from oracle import gemm as og

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize('form,r', [('f16', 100), ('bf16', 150), ('bf16x3', 150), ('fp8', 96)])
def test_every_gemm_configuration_gives_the_same_output(form, r):
    from gwb200 import _lib, autotune, fp_filter
    rng = np.random.default_rng(r)
    M, Tn, group = 256, 2048 * 10, 16
    Kh = fp_filter.kh_of(r, form)
    code = autotune.FORM_CODE[form]
    A = torch.from_numpy(rng.integers(-3, 4, (M, 2 * Kh)).astype(np.float32)).cuda()
    Z = torch.from_numpy(rng.integers(-3, 4, (2 * Kh, Tn)).astype(np.float32)).cuda()
    if form == 'fp8':
        A8, Z8 = A.to(torch.float8_e4m3fn).view(torch.uint8), Z.to(torch.float8_e4m3fn).view(torch.uint8)
        ops = (A8, None, Z8, None)
    else:
        dt = torch.float16 if form == 'f16' else torch.bfloat16
        lo = lambda x: torch.zeros_like(x.to(dt)) if form == 'bf16x3' else None
        ops = (A.to(dt), lo(A), Z.to(dt), lo(Z))
    rs = torch.ones(M, device='cuda')
    nout = -(-(Tn // 128) // group)
    work = torch.empty(_lib.load().gwb_fused_peaks_cplx_work_bytes(M), dtype=torch.uint8, device='cuda')
    An = A.cpu().numpy()
    Are = np.concatenate([An[:, :Kh], -An[:, Kh:]], 1)
    Aim = np.concatenate([An[:, Kh:], An[:, :Kh]], 1)
    Vr, Ir = og.group_reduce(*og.gemm_absmax(Are, Aim, Z.cpu().numpy(), M, Tn), group)
    for cand in autotune.gemm_space(form):
        _lib.call('gwb_gemm_set_config', code, Kh, *cand)
        V = torch.full((M, nout), -7.0, device='cuda')
        I = torch.zeros((M, nout), dtype=torch.int32, device='cuda')
        try:
            _lib.call('gwb_fused_peaks_cplx', code, _lib.ptr(ops[0]), _lib.ptr(ops[1]), ops[0].stride(0),
                      _lib.ptr(ops[2]), _lib.ptr(ops[3]), ops[2].stride(0), M, Kh, Tn, group, _lib.ptr(V),
                      _lib.ptr(I), V.stride(0), _lib.ptr(rs), _lib.ptr(work), work.numel(), _lib.stream_ptr())
        except _lib.GwbError:
            continue                       # a ring deeper than this shape fits is refused before any launch
        assert np.array_equal(V.cpu().numpy(), Vr), cand
        assert np.array_equal(I.cpu().numpy(), Ir), cand
    _lib.call('gwb_gemm_clear_configs')


def test_tune_gemm_sets_the_table_and_caches():
    from gwb200 import autotune
    best, res = autotune.tune_gemm('f16', 256, 128, 2048 * 40)
    assert best in res and isinstance(res[best], float)
    again = autotune.tune_gemm('f16', 256, 128, 2048 * 40)
    assert again[0] == best


def test_pick_cfg_returns_a_config_that_runs():
    from gwb200 import fp_gemm
    cfg, res = fp_gemm.pick_cfg('cuda', 256, 128, 2048 * 16)
    assert cfg[0] == 'umma' and isinstance(res[str(cfg)], float)


def test_matched_filter_with_autotune_matches_without():
    from gwb200 import fp_filter, pipeline
    from test_pipeline_gpu import A0, A1, DF, FLEN, TLEN, _case
    bank, D, IP, kmin, inj = _case()
    Dd, IPd = torch.from_numpy(D).cuda(), torch.from_numpy(IP).cuda()
    sw, isw = fp_filter.derive_sw(IPd)
    out = {}
    for tune in (False, True):
        cfg = pipeline.FilterConfig(tile=24, form='f16', snr_threshold=5.0, cand_cap=1 << 16, autotune=tune)
        B = pipeline.Bank(bank, FLEN, DF, sw, cfg)
        mf = pipeline.MatchedFilter(B, TLEN, A0, A1 - A0, cfg)
        mf.step(Dd, IPd, isw)
        torch.cuda.synchronize()
        res = mf.results()
        out[tune] = {(int(c['row']), int(c['seg']), int(c['window'])): (int(c['sample']), float(p['snr']))
                     for c, p in zip(res['cands'], res['peaks'])}
        if tune:
            assert mf.tuning['gemm'] and mf.tuning['basis']
    # the basis-series form may differ (its scale then comes from another number of rows, which moves the 16-bit
    # rounding of Z): the same windows away from the threshold, the same exact values up to a near-tie sample
    for a, b in ((False, True), (True, False)):
        for k, (s, v) in out[a].items():
            if v > 5.0 * 1.05:
                assert k in out[b], (k, v)
                assert abs(out[b][k][1] - v) <= 2e-3 * v, (k, v, out[b][k])
