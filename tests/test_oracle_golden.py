"""Pins the oracle to the reference: every oracle stage against the golden fixtures made from the reference's own
code (tests/golden/make_golden.py). CPU only."""
import numpy as np

from oracle import chisq, filt, prep


def _argv_opts(argv):
    a = list(argv)
    g = lambda k: a[a.index(k) + 1]
    return dict(gps0=int(g('--gps-start-time')), sr=float(g('--sample-rate')), seg=int(g('--segment-length')),
                sp=int(g('--segment-start-pad')), ep=int(g('--segment-end-pad')), flow=float(g('--low-frequency-cutoff')),
                pl=float(g('--psd-segment-length')), ps=float(g('--psd-segment-stride')),
                pn=int(g('--psd-num-segments')), pinv=float(g('--psd-inverse-length')))


def test_stage2_matches_reference(golden):
    g = golden('prep_stage2')
    o = _argv_opts(g['argv'])
    out = prep.stage2(g['strain'], o['sr'], o['gps0'], o['seg'], o['sp'], o['ep'], o['flow'], o['pl'], o['ps'], o['pn'],
                      o['pinv'])
    assert out['D'].shape == g['D'].shape
    assert [list(a) for a in out['analyze']] == g['analyze'].tolist()
    assert list(out['seg_start']) == g['seg_start'].tolist()
    rel = np.linalg.norm(out['D'] - g['D'], axis=1) / np.linalg.norm(g['D'], axis=1)
    assert rel.max() < 1e-6
    rel = np.linalg.norm(out['IP'] - g['IP'], axis=1) / np.linalg.norm(g['IP'], axis=1)
    assert rel.max() < 1e-6
    kmin = int(o['flow'] * o['seg'])
    assert (out['IP'][:, :kmin] == 0).all()


def test_gating_matches_reference(golden):
    g = golden('prep_gating')
    sr, gps0 = int(g['sr']), int(g['gps0'])
    times = prep.detect_loud_glitches(g['strain'].copy(), sr, gps0, 50.0, 0.5, 15.0, 16.0, 4.0, 2.0)
    assert times == g['gate_ns'].tolist() and len(times) >= 2
    x = prep.gate_taper(g['strain'].copy(), sr, gps0 * 10 ** 9, [(t, 0.25, 0.25) for t in times])
    assert np.array_equal(x, g['gated'])


def test_svd_tile_matches_reference(golden):
    g = golden('filt_tile')
    r, A, Vh, worst, lam, W = filt.svd_tile(g['H'], g['sw'], int(g['kmin']), float(g['eps']))
    assert r == int(g['r'])
    assert abs(worst - float(g['worst'])) < 2e-5
    # A conj(Vh) is independent of the eigenvector phases: compare the compressed templates themselves
    rec = A.astype(np.complex128) @ Vh.astype(np.complex128)
    rec_ref = g['A'].astype(np.complex128) @ g['Vh'].astype(np.complex128)
    rel = np.linalg.norm(rec - rec_ref, axis=1) / np.linalg.norm(rec_ref, axis=1)
    assert rel.max() < 2e-5


def test_basis_series_and_stacked_A_match_reference(golden):
    g = golden('filt_tile')
    r, A, Vh, worst, lam, W = filt.svd_tile(g['H'], g['sw'], int(g['kmin']), float(g['eps']))
    Dws = g['D'] * g['isw']
    a0, Tn, tlen = int(g['a0']), int(g['Tn']), int(g['tlen'])
    Z, scale = filt.basis_series(Vh, Dws, a0, Tn, tlen, np.float32)
    assert abs(scale - float(g['scale'])) < 1e-5 * float(g['scale'])
    Are, Aim = filt.stacked_A(A, g['nrm_s'], scale, Z.shape[0], np.float32)
    # the rebuilt complex SNR series (phase-convention free) against the reference's fp16 pipeline
    zr, zi = Are @ Z, Aim @ Z
    zr_ref = g['Are'].astype(np.float32) @ g['Z'].astype(np.float32)
    zi_ref = g['Aim'].astype(np.float32) @ g['Z'].astype(np.float32)
    snr, snr_ref = np.hypot(zr, zi), np.hypot(zr_ref, zi_ref)
    assert np.abs(snr - snr_ref).max() < 3e-3 * snr_ref.max()      # fp16 rounding of the reference's operands
    # the injection (row 3 at t0) is recovered at the same sample with SNR ~ 12
    t = int(float(g['t0']) * 2048) - a0
    assert np.argmax(snr[3]) == np.argmax(snr_ref[3]) and abs(np.argmax(snr[3]) - t) <= 2
    assert 10 < snr[3].max() < 14


def test_edges_match_reference_exactly(golden):
    g = golden('edges_exact')
    nb = np.maximum(g['nbins'], 1)
    rows = np.arange(len(nb))
    E = chisq.edges_per_template(rows, nb, int(g['kmin']), g['kmax'], g['H'], g['IP'])
    assert np.array_equal(E, g['E'])


def test_exact_dense_matches_reference(golden):
    g = golden('edges_exact')
    z, pw, fpk, _ = chisq.exact_dense(g['H'], g['nbins'], int(g['kmin']), g['kmax'], g['D'], g['IP'], float(g['df']),
                                      int(g['tlen']), g['rows'], g['samples'])
    np.testing.assert_allclose(z, g['z'], rtol=1e-6, atol=1e-9 * np.abs(g['z']).max())
    np.testing.assert_allclose(pw, g['pw'], rtol=1e-6)
    assert np.array_equal(fpk, g['fpeak'])
