"""CPU model of the persistent basis-series kernel's work order (basis_persist in csrc/fft_basis.cu): the ticket order
of its P1 / P2 items for a ring of (pc rows per chunk, nslot W slots, lookahead L), their waits, and the W ring's
buffer bounds.

Checked: every item of every chunk appears exactly once in the ticket order; each item waits only on items earlier
in that order (so the earliest unfinished item can always proceed); under random interleavings of a grid of CTAs
that take tickets in order and block on their waits, every run completes; no P1 item overwrites a W slot that a P2
item of another chunk has not finished reading; and the kernel's index arithmetic stays inside its buffers."""
import numpy as np
import pytest

PG = 128                          # items per chunk and pass (csrc/fft_basis.cu)
N = 1 << 20
N1 = N2 = 1024
TB = 8
CONFIGS = [(2, 3, 1), (2, 4, 2), (1, 4, 2), (1, 6, 3), (4, 2, 1), (3, 3, 2)]   # shared-ticket rings (look >= 1)


def persist_item(t, nch, look):
    """persist_item() of the kernel: (type, chunk, column group) of ticket t, or None past the end."""
    pre = min(look, nch)
    if t < pre * PG:
        return (1, t // PG, t % PG)
    t -= pre * PG
    full = max(0, nch - look)
    if t < full * 2 * PG:
        j, o = divmod(t, 2 * PG)
        return (1, j + look, o) if o < PG else (2, j, o - PG)
    t -= full * 2 * PG
    j = full + t // PG
    if j >= nch:
        return None
    return (2, j, t % PG)


def deps(item, nslot):
    """What the item waits for: (type, chunk) whose PG items must all be done."""
    typ, c, _ = item
    if typ == 1:
        return [(2, c - nslot)] if c >= nslot else []
    return [(1, 0), (1, c)]


def order(nch, look):
    out, t = [], 0
    while True:
        it = persist_item(t, nch, look)
        if it is None:
            return out
        out.append(it)
        t += 1


@pytest.mark.parametrize('cfg', CONFIGS)
@pytest.mark.parametrize('rows', [1, 2, 3, 5, 6, 7, 64, 78, 128, 192, 255])
def test_ticket_order_covers_every_item_once_and_waits_backwards(rows, cfg):
    pc, nslot, look = cfg
    assert nslot > look
    nch = (rows + pc - 1) // pc
    seq = order(nch, look)
    assert len(seq) == 2 * PG * nch
    assert sorted(seq) == sorted([(1, c, g) for c in range(nch) for g in range(PG)] +
                                 [(2, c, g) for c in range(nch) for g in range(PG)])
    last = {}
    for i, it in enumerate(seq):
        last[it[:2]] = i
    for i, it in enumerate(seq):
        for d in deps(it, nslot):
            assert last[d] < i, (it, d)


@pytest.mark.parametrize('rows,ctas,seed,cfg', [(128, 296, 0, (2, 3, 1)), (192, 296, 1, (2, 4, 2)),
                                                 (7, 296, 2, (1, 6, 3)), (78, 17, 3, (4, 2, 1)),
                                                 (40, 1, 4, (3, 3, 2)), (99, 64, 5, (1, 4, 2))])
def test_random_interleavings_complete_and_respect_the_ring(rows, ctas, seed, cfg):
    """CTAs take the next ticket when free, wait until their dependencies are complete, then finish after a random
    number of scheduler steps; a P1 item of chunk c writes slot c % nslot, which no unfinished P2 item of another
    chunk may be reading."""
    pc, nslot, look = cfg
    rng = np.random.default_rng(seed)
    nch = (rows + pc - 1) // pc
    seq = order(nch, look)
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
            if r[1] is None and all(done.get(d, 0) == PG for d in deps(r[0], nslot)):
                r[1] = int(rng.integers(1, 5))
                if r[0][0] == 1:        # starting to write a slot: its previous chunk's readers are all done
                    c = r[0][1]
                    for o in running:
                        if o[0][0] == 2 and o[1] is not None and o[0][1] != c and o[0][1] % nslot == c % nslot:
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
    lane, vv, k2 = np.meshgrid(np.arange(32), np.arange(R), np.arange(N2), indexing='ij')
    off = (lane >> 3) * (N2 * 8) + k2 * 8 + (lane & 7) + 4 * vv * (N2 * 8)
    assert off.min() == 0 and off.max() == N - 1
    assert len(np.unique(off)) == N                      # every W element of the row written once
    assert (N2 - 1) * H + H <= N // 2
    assert (N2 - 1) * H + R * (R // 2 - 1) + 31 < N // 2 + 1
    assert (N1 // TB - 1) * (N2 * TB) + N2 * TB == N
    assert N2 * TB * 8 == 512 * 128
    for pc, nslot, look in CONFIGS:
        # ring: slot c % nslot, row j - j0 < pc, inside pc x nslot rows; the fp8 row scales use warps 1..pc of 8
        assert (nslot - 1) * pc * N + (pc - 1) * N + N == nslot * pc * N
        assert 1 <= pc <= 4
    WS = R * (R + 1) + R + H
    p1 = N1 + 8 * WS
    SB = 33
    SC = 32 * SB + ((2 - (32 * SB) % 16) + 16) % 16
    p2 = N1 + TB * SC
    assert p2 <= p1 and p1 * 8 == 110592


@pytest.mark.parametrize('rows,ctas,seed,pc,nslot', [(128, 148, 0, 2, 3), (192, 148, 1, 2, 2), (7, 148, 2, 1, 4),
                                                      (78, 3, 3, 4, 2), (40, 1, 4, 3, 3)])
def test_split_roles_complete_and_respect_the_ring(rows, ctas, seed, pc, nslot):
    """look = 0: half the grid takes pass-1 items in chunk order from one ticket, the other half pass-2 items from a
    second ticket; a pass-1 item of chunk c waits for the pass-2 items of chunk c - nslot, a pass-2 item for the
    pass-1 items of its chunk (and of chunk 0). Random interleavings complete and no slot is overwritten while read."""
    rng = np.random.default_rng(seed)
    nch = (rows + pc - 1) // pc
    queues = {1: [(1, c, g) for c in range(nch) for g in range(PG)], 2: [(2, c, g) for c in range(nch) for g in range(PG)]}
    done, running, steps = {}, [], 0
    free = {1: ctas, 2: ctas}
    pos = {1: 0, 2: 0}
    while any(pos[k] < len(queues[k]) for k in (1, 2)) or running:
        steps += 1
        assert steps < 10 ** 6, 'no progress'
        for k in (1, 2):
            while free[k] and pos[k] < len(queues[k]):
                running.append([queues[k][pos[k]], None])
                pos[k] += 1
                free[k] -= 1
        rng.shuffle(running)
        for r in running:
            if r[1] is None and all(done.get(d, 0) == PG for d in deps(r[0], nslot)):
                r[1] = int(rng.integers(1, 5))
                if r[0][0] == 1:
                    c = r[0][1]
                    for o in running:
                        if o[0][0] == 2 and o[1] is not None and o[0][1] != c and o[0][1] % nslot == c % nslot:
                            raise AssertionError(('slot overwritten while read', r[0], o[0]))
        for r in list(running):
            if r[1] is not None:
                r[1] -= 1
                if r[1] == 0:
                    k = r[0][:2]
                    done[k] = done.get(k, 0) + 1
                    running.remove(r)
                    free[r[0][0]] += 1
    assert all(done[(ty, c)] == PG for ty in (1, 2) for c in range(nch))
