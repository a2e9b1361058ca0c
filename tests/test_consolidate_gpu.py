"""GPU consolidation (gwb200.consolidate, csrc/consolidate.cu) against the reference's consolidate and pre_keep
(tests/golden/consolidate.npz) and the oracle (oracle/consolidate.py): identical keep masks, floors equal to 1e-15
relative (newsnr goes through CUDA's pow), at the fixtures' sizes, with explicit order keys, with windows larger than
one shared-memory tile, and at two million peaks."""
import numpy as np
import pytest
import torch

from oracle import consolidate as oc
from test_consolidate_cpu import _cases

pytestmark = pytest.mark.gpu


def _d(x):
    return torch.from_numpy(np.ascontiguousarray(x)).cuda()


def _floor_eq(a, b):
    a, b = np.asarray(a), np.asarray(b)
    n = max(len(a), len(b))
    pa = np.full(n, -np.inf)
    pb = np.full(n, -np.inf)
    pa[:len(a)], pb[:len(b)] = a, b
    fin = np.isfinite(pb)
    assert np.array_equal(np.isfinite(pa), fin)
    np.testing.assert_allclose(pa[fin], pb[fin], rtol=1e-15)


def test_consolidate_matches_reference(golden):
    from gwb200 import consolidate as gc
    g = golden('consolidate')
    sr, gps0 = float(g['sr']), float(g['gps0'])
    for c in _cases(g, 'c'):
        interval, num, exempt, do_chisq, nthr = c['par']
        keep, floor = gc.consolidate(_d(c['snr']), _d(c['chi']), _d(c['dof']), _d(c['ti'].astype(np.int64)),
                                     [tuple(x) for x in c['gates']], gps0, sr, nthr, interval or None, int(num),
                                     None if exempt < 0 else exempt, use_chisq=bool(do_chisq), want_floor=True,
                                     n_samples=int(c['ti'].max()) + 1 if len(c['ti']) else 1)
        assert np.array_equal(keep.cpu().numpy(), c['keep'])
        if interval:
            _floor_eq(floor.cpu().numpy(), c['floor'])


def test_pre_keep_matches_reference(golden):
    from gwb200 import consolidate as gc
    g = golden('consolidate')
    sr, gps0 = float(g['sr']), float(g['gps0'])
    for c in _cases(g, 'p'):
        interval, num, exempt, exact_snr, margin, thr, nthr = c['par']
        fl = _d(c['floor']) if bool(c['has_floor']) else None
        keep = gc.pre_keep(_d(c['ti'].astype(np.int64)), _d(c['apx']), [tuple(x) for x in c['gates']], gps0, sr,
                           exact_snr, margin, thr, None if exempt < 0 else exempt, nthr, interval or None, int(num),
                           floor=fl)
        assert np.array_equal(keep.cpu().numpy(), c['keep'])


def _synthetic(n, span_s, seed, tie_step=0.01):
    rng = np.random.default_rng(seed)
    ti = rng.integers(0, int(span_s * 2048), n).astype(np.int64)
    snr = np.round(rng.uniform(3.9, 12.0, n) / tie_step) * tie_step
    snr = snr.astype(np.float32)
    isex = rng.uniform(size=n) < 0.5
    chi = np.where(isex, np.round(rng.uniform(0, 90, n), 1), 0).astype(np.float32)
    dof = np.where(isex, 30, 0).astype(np.int32)
    return ti, snr, chi, dof


@pytest.mark.parametrize('n,span,num,seed', [(2_000_000, 4096.0, 30, 1), (20_000, 2.0, 7, 2), (50_000, 8.0, 3000, 3)])
def test_consolidate_at_scale_against_oracle(n, span, num, seed):
    """Two million peaks over 4096 s (production's 30 per 1.072 s), and crowded windows of ~7,000-10,000 peaks (more
    than one shared-memory tile) with small and large keep counts; order keys a random permutation."""
    from gwb200 import consolidate as gc
    ti, snr, chi, dof = _synthetic(n, span, seed)
    gps0, sr = 1380077576.0, 2048.0
    gates = [(gps0 + span * 0.3, 0.25, 0.25), (gps0 + span * 0.71, 0.25, 0.25)]
    order = np.random.default_rng(seed + 10).permutation(n).astype(np.int64)
    t = gps0 + ti / sr
    ref, fl_ref = oc.consolidate(snr, chi, dof, t, gates, gps0, sr, 4.0, 1.072, num, 5.0, want_floor=True,
                                 order=order)
    keep, fl = gc.consolidate(_d(snr), _d(chi), _d(dof), _d(ti), gates, gps0, sr, 4.0, 1.072, num, 5.0,
                              order=_d(order), want_floor=True, n_samples=int(span * sr))
    k = keep.cpu().numpy()
    assert np.array_equal(k, ref), (k.sum(), ref.sum(), np.nonzero(k != ref)[0][:10])
    _floor_eq(fl.cpu().numpy(), fl_ref)


def test_window_outside_range_raises():
    from gwb200 import _lib, consolidate as gc
    ti, snr, chi, dof = _synthetic(1000, 10.0, 4)
    with pytest.raises(_lib.GwbError):
        gc.consolidate(_d(snr), _d(chi), _d(dof), _d(ti), [], 1e9, 2048.0, 4.0, 1.072, 3, n_samples=2048)


def test_peak_store_equals_one_consolidation():
    """Consolidating after every part (the reference's per-tile calls) equals one call over the union."""
    from gwb200 import consolidate as gc
    n = 60_000
    ti, snr, chi, dof = _synthetic(n, 30.0, 5, tie_step=0.05)
    gps0, sr = 1e9, 2048.0
    order = np.arange(n, dtype=np.int64)
    store = gc.PeakStore(gps0, sr, int(30 * sr), [(gps0 + 12.0, 0.25, 0.25)], 4.0, 1.072, 4, 5.0)
    for a, b in ((0, 7000), (7000, 7001), (7001, 40000), (40000, n)):
        store.add(tid=_d(np.arange(a, b, dtype=np.int64)), ti=_d(ti[a:b]), snr=_d(snr[a:b]),
                  phase=_d(np.zeros(b - a, np.float32)), peak_sigmasq=_d(np.ones(b - a)),
                  exact=_d(dof[a:b] > 0), chisq=_d(chi[a:b]), dof=_d(dof[a:b]), order=_d(order[a:b]))
    ref, _ = oc.consolidate(snr, chi, dof, gps0 + ti / sr, [(gps0 + 12.0, 0.25, 0.25)], gps0, sr, 4.0, 1.072, 4, 5.0)
    h = store.host()
    assert sorted(h['tid'].tolist()) == np.nonzero(ref)[0].tolist()
    tab = gc.peak_table(h, [(gps0 + 12.0, 0.25, 0.25)], gps0, sr)
    ref_tab = oc.peak_table(h['tid'], gps0 + h['ti'] / sr, h['snr'], h['phase'], h['peak_sigmasq'], h['exact'],
                            h['chisq'], h['dof'], [(gps0 + 12.0, 0.25, 0.25)], None)
    for key, v in ref_tab.items():
        if v is not None:
            assert np.array_equal(tab[key], v), key
