"""The consolidation oracle (oracle/consolidate.py) against the reference's own consolidate and pre_keep closures
(tests/golden/consolidate.npz): identical keep masks and floors on every case, ties included."""
import numpy as np

from oracle import consolidate as oc


def _cases(g, kind):
    n = int(g['n_cons' if kind == 'c' else 'n_pre'])
    for i in range(n):
        pre = '%s%d_' % (kind, i)
        yield {k[len(pre):]: v for k, v in g.items() if k.startswith(pre)}


def test_consolidate_oracle_matches_reference(golden):
    g = golden('consolidate')
    sr, gps0 = float(g['sr']), float(g['gps0'])
    n_ties = 0
    for c in _cases(g, 'c'):
        interval, num, exempt, do_chisq, nthr = c['par']
        t = gps0 + c['ti'] / sr
        keep, floor = oc.consolidate(c['snr'], c['chi'], c['dof'], t, [tuple(x) for x in c['gates']], gps0, sr,
                                     nthr, interval or None, int(num), None if exempt < 0 else exempt,
                                     use_chisq=bool(do_chisq), want_floor=True)
        assert np.array_equal(keep, c['keep'])
        if interval:
            assert np.array_equal(floor, c['floor'])
        n_ties += len(c['snr']) - len(np.unique(c['snr']))
    assert n_ties > 1000          # the cases exercise the tie rule


def test_pre_keep_oracle_matches_reference(golden):
    g = golden('consolidate')
    sr, gps0 = float(g['sr']), float(g['gps0'])
    for c in _cases(g, 'p'):
        interval, num, exempt, exact_snr, margin, thr, nthr = c['par']
        keep = oc.pre_keep(c['ti'], c['apx'], [tuple(x) for x in c['gates']], gps0, sr, exact_snr, margin, thr,
                           None if exempt < 0 else exempt, nthr, interval or None, int(num),
                           floor=c['floor'] if bool(c['has_floor']) else None)
        assert np.array_equal(keep, c['keep'])


def test_order_keys_replace_positions():
    """Ranking by an explicit order key gives the masks of the arrays permuted into that order."""
    rng = np.random.default_rng(3)
    n = 2000
    ti = rng.integers(0, 20 * 2048, n)
    t = 1e9 + ti / 2048.0
    snr = np.round(rng.uniform(4, 6, n), 1).astype(np.float32)
    chi, dof = np.zeros(n, np.float32), np.zeros(n, np.int32)
    perm = rng.permutation(n)
    k0, _ = oc.consolidate(snr, chi, dof, t, [], 1e9, 2048.0, 4.0, 1.072, 3)
    k1, _ = oc.consolidate(snr[perm], chi[perm], dof[perm], t[perm], [], 1e9, 2048.0, 4.0, 1.072, 3, order=perm)
    assert np.array_equal(k1, k0[perm])


def test_peak_table_and_file_match_the_oracle(tmp_path):
    """write_one's datasets (fp_filter.py:910-934) from the library's host assembly equal the oracle's, and the file
    written without h5py (.npz) holds the same datasets."""
    from gwb200 import consolidate as gc
    rng = np.random.default_rng(9)
    n, gps0, sr = 5000, 1380077576.0, 2048.0
    h = dict(tid=rng.integers(0, 300, n).astype(np.int64), ti=rng.integers(0, 600 * 2048, n).astype(np.int64),
             snr=rng.uniform(4, 12, n).astype(np.float32), phase=rng.uniform(-3, 3, n).astype(np.float32),
             peak_sigmasq=rng.uniform(1, 2, n), exact=rng.uniform(size=n) < 0.4,
             chisq=rng.uniform(0, 80, n).astype(np.float32))
    h['dof'] = np.where(h['exact'], 30, 0).astype(np.int32)
    gates = [(gps0 + 100.0, 0.25, 0.25), (gps0 + 412.5, 0.25, 0.25)]
    sig = rng.uniform(1, 2, (300, 3))
    hashes = np.array(['h%04d' % i for i in range(300)])
    tab = gc.peak_table(h, gates, gps0, sr, sigmasq=sig, hashes=hashes)
    ref = oc.peak_table(h['tid'], gps0 + h['ti'] / sr, h['snr'], h['phase'], h['peak_sigmasq'], h['exact'], h['chisq'],
                        h['dof'], gates, sig, hashes=hashes)
    assert sorted(tab) == sorted(ref)
    for k, v in ref.items():
        assert np.array_equal(tab[k], v), k
    assert len(tab['snr']) < n                              # the gates removed some peaks
    path = str(tmp_path / 'H1-peaks')
    gc.write_peaks(path, tab)
    try:
        import h5py
    except ImportError:
        h5py = None
    if h5py is None:
        with np.load(path + '.npz') as z:
            for k, v in tab.items():
                assert np.array_equal(z[k], v), k
    else:
        with h5py.File(path, 'r') as f:
            for k, v in tab.items():
                assert np.array_equal(f[k][()].astype(v.dtype), v), k
