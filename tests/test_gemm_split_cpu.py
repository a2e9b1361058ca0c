"""Index arithmetic of the GEMM's tile-granular CTA ranges (csrc/gemm_cplx.cu), restated on the CPU: CTA c owns
tiles [c ntiles / g, (c + 1) ntiles / g); a window cut by a range boundary is written by each covering CTA into slot
0 (the window began before the CTA's range) or 1 (it goes on after it), and window_merge_kernel reads, for each CTA
from cta_of_tile(first tile) to cta_of_tile(last tile), slot 0 when the CTA's range begins after the window's first
tile, else slot 1. Every slot read must be written by exactly that CTA, and every other window written directly by
exactly one CTA."""
import itertools


def _ranges(ntiles, g):
    return [(c * ntiles // g, (c + 1) * ntiles // g) for c in range(g)]


def _cta_of_tile(t, ntiles, g):
    # the kernel's search: an estimate then steps to the CTA whose range holds t
    c = t * g // ntiles
    while c + 1 < g and (c + 1) * ntiles // g <= t:
        c += 1
    while c > 0 and c * ntiles // g > t:
        c -= 1
    return c


def test_every_merged_slot_is_written_once_by_its_cta():
    for ntiles, g, group in itertools.product([1, 5, 16, 51, 320, 7168, 7169], [1, 2, 7, 51, 74, 148],
                                              [1, 4, 16, 17]):
        g_ = min(g, ntiles)
        nout = -(-ntiles // group)
        ranges = _ranges(ntiles, g_)
        writes, direct = {}, {}
        for c, (tb, te) in enumerate(ranges):
            for t in range(tb, te):
                last = (t + 1) % group == 0 or t == ntiles - 1 or t == te - 1
                if not last:
                    continue
                o = t // group
                w0, w1 = o * group, min(o * group + group, ntiles)
                if tb > w0 or te < w1:
                    key = (c, 0 if tb > w0 else 1)
                    assert key not in writes
                    writes[key] = o
                else:
                    assert o not in direct
                    direct[o] = c
        for o in range(nout):
            w0, w1 = o * group, min(o * group + group, ntiles)
            ca, cb = _cta_of_tile(w0, ntiles, g_), _cta_of_tile(w1 - 1, ntiles, g_)
            assert ranges[ca][0] <= w0 < ranges[ca][1] and ranges[cb][0] <= w1 - 1 < ranges[cb][1]
            if ca == cb:
                assert direct.get(o) == ca, (ntiles, g_, group, o)
                continue
            assert o not in direct
            for c in range(ca, cb + 1):
                slot = 0 if ranges[c][0] > w0 else 1
                assert writes.get((c, slot)) == o, (ntiles, g_, group, o, c, slot)
