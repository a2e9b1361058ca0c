"""The batched form (gwb200.segments.filter_segments) on a small case: segments of 300 s (an injection), 200 s (a loud
sine-Gaussian glitch) and 100 s (shorter than the 128 s chunks: skipped), a 48-template bank. The glitch is gated, the
injection is found at its time, and the graph-replayed run gives the same peaks as the direct one."""
import numpy as np
import pytest
import torch

from oracle import synth

pytestmark = pytest.mark.gpu

SR, L, SP, EP = 2048.0, 128.0, 24.0, 8.0
TLEN = int(L * SR)
FLEN, DF = TLEN // 2 + 1, 1.0 / L


def _segment(n_s, rng, bank=None, inj=None, glitch=None):
    n = int(n_s * SR)
    f = np.arange(n // 2 + 1) * (SR / n)
    psd = synth.analytic_psd(f)
    X = np.fft.rfft(rng.standard_normal(n)) * np.sqrt(psd * SR / 2.0)
    X[0] = 0
    kmin = int(20.0 * n / SR)
    if inj is not None:
        i, t0, snr = inj
        h = synth.taylorf2(n // 2 + 1, SR / n, bank['mass1'][i], bank['mass2'][i], t0=t0)
        h[f > synth.f_isco(bank['mass1'][i], bank['mass2'][i])] = 0
        X = X + snr / synth.optimal_snr(h, psd, SR / n, kmin) * h * SR
    x = np.fft.irfft(X, n)
    if glitch is not None:
        tg, f0, snr = glitch
        g = synth.sine_gaussian(n, SR, tg, f0, 10.0)
        G = np.fft.rfft(g) / SR
        x = x + g * snr / np.sqrt(4 * (SR / n) * np.sum(np.abs(G[kmin:]) ** 2 / psd[kmin:]))
    return torch.from_numpy(x.astype(np.float32)).cuda()          # analytic_psd is in DYN_RANGE_FAC units


def test_filter_segments_gates_finds_and_replays():
    from gwb200 import fp_filter, gpu_prep, pipeline, segments
    rng = np.random.default_rng(11)
    bank = synth.random_bank_c1(48, 3)
    segs = [dict(x=_segment(300, rng, bank, inj=(7, 150.0, 15.0)), start_gps=1000000000, det=0),
            dict(x=_segment(200, rng, glitch=(100.0, 120.0, 200.0)), start_gps=1000001000, det=1),
            dict(x=_segment(100, rng), start_gps=1000002000, det=0)]
    cond = gpu_prep.BatchConditioner(4, TLEN, SR, 20.0, 16.0, 8.0, 15, 16.0)
    _, IP = cond(torch.stack([segs[0]['x'][:TLEN]] * 4).contiguous())
    sw, isw = fp_filter.derive_sw(IP)
    cfg = pipeline.FilterConfig(tile=24, form='f16', snr_threshold=5.5, cand_cap=1 << 16)
    B = pipeline.Bank(bank, FLEN, DF, sw.clone(), cfg)
    out = {}
    for graph in (False, True):
        sg = [dict(s, x=s['x'].clone()) for s in segs]
        F = segments.SegmentFilter(B, cfg, seg_len=L, start_pad=SP, end_pad=EP, batch=4, psd=(16.0, 8.0, 15, 16.0),
                                   isw=isw.clone(), graph=graph)
        out[graph] = F.run(sg)
    r = out[True]
    assert r['skipped'] == [2]
    assert r['analysed_s'] == pytest.approx((300 - SP - EP) + (200 - SP - EP))
    assert len(r['gates'][1]) >= 1 and abs(r['gates'][1][0][0] - (1000001000 + 100.0)) < 0.5
    assert r['gates'][0] == []
    keep = r['keep']
    t_peak = np.array([r['plan'][k][1][0] for k in r['chunk'][keep]]) + r['cands']['sample'][keep]
    hit = (r['segment'][keep] == 0) & (np.abs(t_peak / SR - 150.0) < 0.1)
    assert hit.any()
    assert abs(r['peaks']['snr'][keep][hit].max() - 15.0) < 3.0
    # the glitch leaves no loud peak after gating
    g_snr = r['peaks']['snr'][keep][r['segment'][keep] == 1]
    assert g_snr.size == 0 or g_snr.max() < 12.0
    # graph replay = direct run
    key = lambda x: sorted(zip(x['segment'].tolist(), x['chunk'].tolist(), x['cands']['sample'].tolist(),
                               np.round(x['peaks']['snr'], 4).tolist()))
    assert key(out[True]) == key(out[False])


def test_filter_segments_consolidated_tables():
    """Production's selection (threshold 4, exact stage above 5.5 (1 - margin), the rest rebuilt) with consolidation
    (newsnr 4, 3 loudest per 1.072 s, SNR >= 5 exempt): each segment's table equals the oracle's consolidation of
    the run's raw peaks in the reference's append order, followed by write_one's assembly."""
    from gwb200 import fp_filter, gpu_prep, pipeline, segments
    from oracle import consolidate as oc
    rng = np.random.default_rng(12)
    bank = synth.random_bank_c1(48, 3)
    segs = [dict(x=_segment(300, rng, bank, inj=(7, 150.0, 15.0)), start_gps=1000000000, det=0),
            dict(x=_segment(200, rng, glitch=(100.0, 120.0, 200.0)), start_gps=1000001000, det=1)]
    cond = gpu_prep.BatchConditioner(4, TLEN, SR, 20.0, 16.0, 8.0, 15, 16.0)
    _, IP = cond(torch.stack([segs[0]['x'][:TLEN]] * 4).contiguous())
    sw, isw = fp_filter.derive_sw(IP)
    cfg = pipeline.FilterConfig(tile=24, form='f16', snr_threshold=4.0, exact_snr=5.5, cand_cap=1 << 18)
    B = pipeline.Bank(bank, FLEN, DF, sw.clone(), cfg)
    co = segments.Consolidation(4.0, 1.072, 3, 5.0)
    F = segments.SegmentFilter(B, cfg, seg_len=L, start_pad=SP, end_pad=EP, batch=4, psd=(16.0, 8.0, 15, 16.0),
                               isw=isw.clone(), consolidation=co)
    r = F.run(segs, keep_raw=True)
    assert r['n_peaks_in'] > r['n_peaks_out'] > 0
    for i, tab in r['tables'].items():
        h = r['raw'][i]
        gps = segs[i]['start_gps']
        t = gps + h['ti'] / SR
        keep, _ = oc.consolidate(h['snr'], h['chisq'], h['dof'], t, r['gates'][i], gps, SR, 4.0, 1.072, 3, 5.0,
                                 order=h['order'])
        ref = oc.peak_table(h['tid'][keep], t[keep], h['snr'][keep], h['phase'][keep], h['peak_sigmasq'][keep],
                            h['exact'][keep], h['chisq'][keep], h['dof'][keep], r['gates'][i], tab['sigmasq'])
        for k, v in ref.items():
            assert np.array_equal(tab[k], v), (i, k)
        assert len(np.unique(h['order'])) == len(h['order'])
        assert tab['exact'].any() and (~tab['exact']).any()
    # the injection is among the consolidated peaks of its segment
    t0 = r['tables'][0]
    near = np.abs(t0['end_time'] - (1000000000 + 150.0)) < 0.1
    assert near.any() and abs(t0['snr'][near].max() - 15.0) < 3.0


def test_whole_run_graph_matches_the_direct_run():
    """The whole run captured as one graph (SegmentFilter.prepare, then run_graph: batched gating, one replay, one
    copy of the run-wide result list) gives the same gates and the same peaks as the direct batch-by-batch run."""
    from gwb200 import fp_filter, gpu_prep, pipeline, segments
    rng = np.random.default_rng(11)
    bank = synth.random_bank_c1(48, 3)
    segs = [dict(x=_segment(300, rng, bank, inj=(7, 150.0, 15.0)), start_gps=1000000000, det=0),
            dict(x=_segment(200, rng, glitch=(100.0, 120.0, 200.0)), start_gps=1000001000, det=1),
            dict(x=_segment(100, rng), start_gps=1000002000, det=0),
            dict(x=_segment(420, rng), start_gps=1000003000, det=1)]
    cond = gpu_prep.BatchConditioner(4, TLEN, SR, 20.0, 16.0, 8.0, 15, 16.0)
    _, IP = cond(torch.stack([segs[0]['x'][:TLEN]] * 4).contiguous())
    sw, isw = fp_filter.derive_sw(IP)
    cfg = pipeline.FilterConfig(tile=24, form='f16', snr_threshold=5.5, cand_cap=1 << 16)
    B = pipeline.Bank(bank, FLEN, DF, sw.clone(), cfg)
    out = {}
    for mode in ('direct', 'graph'):
        sg = [dict(s, x=s['x'].clone()) for s in segs]
        F = segments.SegmentFilter(B, cfg, seg_len=L, start_pad=SP, end_pad=EP, batch=4, psd=(16.0, 8.0, 15, 16.0),
                                   isw=isw.clone(), graph=False)
        if mode == 'graph':
            F.prepare(sg)
            out[mode] = F.run_graph()
            assert out[mode]['graph_launches'] == 1 and out[mode]['batches'] >= 2
        else:
            out[mode] = F.run(sg)
    a, b = out['direct'], out['graph']
    assert a['gates'] == b['gates'] and a['skipped'] == b['skipped'] and a['analysed_s'] == b['analysed_s']
    key = lambda x: sorted(zip(x['segment'].tolist(), x['chunk'].tolist(), x['cands']['row'].tolist(),
                               x['cands']['sample'].tolist(), np.round(x['peaks']['snr'], 4).tolist()))
    assert key(a) == key(b)
    assert np.array_equal(np.sort(a['keep']), np.sort(b['keep']))
