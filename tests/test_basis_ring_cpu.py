"""CPU model of the persistent basis-series kernel's work order (basis_persist in csrc/fft_basis.cu): the ticket order
of its P1 / P2 items, their waits, and the W ring's buffer bounds.

Checked: every item of every chunk appears exactly once in the ticket order; each item waits only on items earlier
in that order (so the earliest unfinished item can always proceed); under random interleavings of a grid of CTAs
that take tickets in order and block on their waits, every run completes; no P1 item overwrites a W slot that a P2
item of an older chunk has not finished reading; and the kernel's index arithmetic stays inside its buffers."""
import numpy as np
import pytest

PC, PSLOT, PG = 2, 3, 128          # rows per chunk, W slots, items per chunk and pass (csrc/fft_basis.cu)
N = 1 << 20
N1 = N2 = 1024
TB = 8


def persist_item(t, nch):
    """persist_item() of the kernel: (type, chunk, column group) of ticket t, or None past the end."""
    if t < PG:
        return (1, 0, t) if nch > 0 else None
    t -= PG
    j, o = divmod(t, 2 * PG)
    if j >= nch:
        return None
    if j + 1 < nch:
        return (1, j + 1, o) if o < PG else (2, j, o - PG)
    if o >= PG:
        return None
    return (2, j, o)


def deps(item):
    """What the item waits for: (type, chunk) whose PG items must all be done."""
    typ, c, _ = item
    if typ == 1:
        return [(2, c - PSLOT)] if c >= PSLOT else []
    return [(1, 0), (1, c)]


def order(nch):
    out, t = [], 0
    while True:
        it = persist_item(t, nch)
        if it is None:
            return out
        out.append(it)
        t += 1


@pytest.mark.parametrize('rows', [1, 2, 3, 5, 6, 7, 64, 78, 128, 192, 255])
def test_ticket_order_covers_every_item_once_and_waits_backwards(rows):
    nch = (rows + PC - 1) // PC
    seq = order(nch)
    assert len(seq) == 2 * PG * nch
    assert sorted(seq) == sorted([(1, c, g) for c in range(nch) for g in range(PG)] +
                                 [(2, c, g) for c in range(nch) for g in range(PG)])
    pos = {it: i for i, it in enumerate(seq)}
    last = {}
    for i, it in enumerate(seq):
        last[it[:2]] = i
    for i, it in enumerate(seq):
        for d in deps(it):
            assert last[d] < i, (it, d)


@pytest.mark.parametrize('rows,ctas,seed', [(128, 296, 0), (192, 296, 1), (7, 296, 2), (78, 17, 3), (40, 1, 4)])
def test_random_interleavings_complete_and_respect_the_ring(rows, ctas, seed):
    """CTAs take the next ticket when free, wait until their dependencies are complete, then finish after a random
    number of scheduler steps; a P1 item of chunk c writes slot c % PSLOT, which no unfinished P2 item of another
    chunk may be reading."""
    rng = np.random.default_rng(seed)
    nch = (rows + PC - 1) // PC
    seq = order(nch)
    done = {}
    t = 0
    running = []                    # [item, remaining steps or None while waiting]
    free = ctas
    steps = 0
    while t < len(seq) or running:
        steps += 1
        assert steps < 10 ** 6, 'no progress'
        while free and t < len(seq):
            running.append([seq[t], None])
            t += 1
            free -= 1
        rng.shuffle(running)
        for r in running:
            if r[1] is None and all(done.get(d, 0) == PG for d in deps(r[0])):
                r[1] = int(rng.integers(1, 5))
                if r[0][0] == 1:        # starting to write a slot: its previous chunk's readers are all done
                    c = r[0][1]
                    for o in running:
                        if o[0][0] == 2 and o[1] is not None and o[0][1] != c and o[0][1] % PSLOT == c % PSLOT:
                            raise AssertionError(('slot overwritten while read', r[0], o[0]))
        for r in list(running):
            if r[1] is not None:
                r[1] -= 1
                if r[1] == 0:
                    k = r[0][:2]
                    done[k] = done.get(k, 0) + 1
                    running.remove(r)
                    free += 1
    assert all(done[(ty, c)] == PG for ty in (1, 2) for c in range(nch))


def test_index_arithmetic_stays_inside_the_buffers():
    """The W writes of P1 (blocks of 8 t1), the W tile reads of P2, the basis-filter / D reads and the shared-memory
    regions of basis_persist, at the extreme indices."""
    R, H = 32, N1 // 2
    # P1: W offset of (lane, vv, k2) inside one row of the slot
    lane, vv, k2 = np.meshgrid(np.arange(32), np.arange(R), np.arange(N2), indexing='ij')
    off = (lane >> 3) * (N2 * 8) + k2 * 8 + (lane & 7) + 4 * vv * (N2 * 8)
    assert off.min() == 0 and off.max() == N - 1
    assert len(np.unique(off)) == N                      # every W element of the row written once
    # P1 reads: Vp segment k2 H .. k2 H + H (4 KB) and D at k2 H + R q + lane
    assert (N2 - 1) * H + H <= N // 2
    assert (N2 - 1) * H + R * (R // 2 - 1) + 31 < N // 2 + 1
    # P2: tile of block b (N2 TB complex, contiguous) inside the row; 512 discarded lines of 128 bytes
    assert (N1 // TB - 1) * (N2 * TB) + N2 * TB == N
    assert N2 * TB * 8 == 512 * 128
    # ring: slot c % PSLOT, row j - j0 < PC
    assert (PSLOT - 1) * PC * N + (PC - 1) * N + N == PSLOT * PC * N
    # shared memory: the twiddle table, then P1's per-warp tiles or P2's exchange tile
    WS = R * (R + 1) + R + H
    p1 = N1 + 8 * WS
    SB = 33
    SC = 32 * SB + ((2 - (32 * SB) % 16) + 16) % 16
    p2 = N1 + TB * SC
    assert p2 <= p1 and p1 * 8 == 110592
