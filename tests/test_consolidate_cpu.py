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
