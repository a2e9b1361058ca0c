"""Exact-stage selection by rank (gwb_select_top) through the C ABI against a numpy statement of the rule: per segment
the candidates whose rebuilt SNR is at least the k-th largest of the segment (ties kept) stay exact-stage candidates
(units and groups of <= 8 rebuilt, candidate order kept within each unit), the others above rthr become rebuilt peaks
after the selection's own, the rest are dropped."""
import numpy as np
import pytest
import torch

from gwb200 import _exact

pytestmark = pytest.mark.gpu


def _lists(rng, nseg, nrow):
    cands, units, groups = [], [], []
    for row in range(nrow):
        for seg in range(nseg):
            m = int(rng.integers(0, 12))
            if m == 0:
                continue
            u = len(units)
            first = len(cands)
            for w in range(m):
                a = float(np.float32(rng.choice([5.3, 5.6, 6.0, 7.5]) if rng.uniform() < 0.2 else rng.uniform(5.2, 9.0)))
                cands.append((row, seg, 1000 + w * 2048, w, a, a * 0.6, a * 0.8, u))
            units.append((row, seg, first, m))
            for g0 in range(0, m, 8):
                groups.append((u, first + g0, min(8, m - g0), 0))
    return (np.array(cands, _exact.CAND), np.array(units, _exact.UNIT), np.array(groups, _exact.GROUP))


@pytest.mark.parametrize('top_n,frac', [(10, 0.0), (3, 0.0), (0, 0.01), (0, 0.25), (1000, 0.0)])
def test_select_top_against_numpy(top_n, frac):
    from gwb200 import _lib
    rng = np.random.default_rng(top_n * 7 + int(frac * 100))
    nseg, nrow, cap, rthr = 5, 60, 1 << 14, np.float32(5.5)
    cands, units, groups = _lists(rng, nseg, nrow)
    dev = lambda rec, n: torch.cat([_exact.to_dev(rec), torch.zeros(n * rec.dtype.itemsize - rec.nbytes,
                                                                      dtype=torch.uint8, device='cuda')])
    ci, ui, gi = dev(cands, cap), dev(units, cap), dev(groups, cap)
    n_reb0 = 7                                            # the selection's own rebuilt peaks come first
    cnt_in = torch.tensor([len(cands), len(groups), len(units), 0, n_reb0], dtype=torch.int32, device='cuda')
    co = torch.zeros(cap * 32, dtype=torch.uint8, device='cuda')
    go = torch.zeros(cap * 16, dtype=torch.uint8, device='cuda')
    uo = torch.zeros(cap * 16, dtype=torch.uint8, device='cuda')
    rb = torch.zeros(cap * 32, dtype=torch.uint8, device='cuda')
    cnt = torch.zeros(5, dtype=torch.int32, device='cuda')
    lib = _lib.load()
    work = torch.empty(lib.gwb_select_top_work_bytes(nseg, cap), dtype=torch.uint8, device='cuda')
    _lib.call('gwb_select_top', _lib.ptr(ci), _lib.ptr(gi), _lib.ptr(ui), _lib.ptr(cnt_in), cap, nseg, top_n, frac,
              float(rthr), _lib.ptr(co), _lib.ptr(go), _lib.ptr(uo), _lib.ptr(cnt), _lib.ptr(rb), cap, _lib.ptr(work),
              work.numel(), _lib.stream_ptr())
    torch.cuda.synchronize()
    c = cnt.cpu().numpy()
    assert c[3] == 0
    out_c = _exact.from_dev(co, _exact.CAND, int(c[0]))
    out_u = _exact.from_dev(uo, _exact.UNIT, int(c[2]))
    out_g = _exact.from_dev(go, _exact.GROUP, int(c[1]))
    out_r = _exact.from_dev(rb, _exact.CAND, int(c[4]))[n_reb0:]
    # numpy statement of the rule
    tau = np.zeros(nseg, np.float32)
    for s in range(nseg):
        a = np.sort(cands['approx'][cands['seg'] == s])[::-1]
        k = top_n if top_n > 0 else int(np.ceil(np.float32(frac) * np.float32(len(a))))
        k = max(k, 1)
        tau[s] = a[k - 1] if len(a) > k else 0.0
    keep = cands['approx'] >= tau[cands['seg']]
    reb = ~keep & (cands['approx'] > rthr)
    key = lambda x: sorted(zip(x['row'].tolist(), x['seg'].tolist(), x['window'].tolist()))
    assert key(out_c) == key(cands[keep])
    assert key(out_r) == key(cands[reb]) and np.all(out_r['unit'] == -1)
    np.testing.assert_array_equal(np.sort(out_r['zr']), np.sort(cands['zr'][reb]))
    # units: one per input unit with kept candidates, contiguous runs in input order, groups of <= 8 covering them
    assert len(out_u) == len({(r, s) for r, s in zip(cands['row'][keep], cands['seg'][keep])})
    covered = np.zeros(len(out_c), int)
    for g in out_g:
        u = out_u[g['unit']]
        assert u['first'] <= g['first'] and g['first'] + g['count'] <= u['first'] + u['count'] and g['count'] <= 8
        covered[g['first']:g['first'] + g['count']] += 1
    assert np.all(covered == 1)
    for i, u in enumerate(out_u):
        run = out_c[u['first']:u['first'] + u['count']]
        assert np.all(run['row'] == u['row']) and np.all(run['seg'] == u['seg']) and np.all(run['unit'] == i)
        assert np.all(np.diff(run['window']) > 0)
