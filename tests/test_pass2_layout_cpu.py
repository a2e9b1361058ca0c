"""Index arithmetic of the 16-column pass 2 of the basis series (basis_pass2_w, csrc/fft_basis.cu) for N2 = 1024,
checked on the CPU: every thread's (column, b) and (column, u) pairs cover the tile once, every shared-memory index
stays inside the buffer, each half-warp's 64-bit accesses hit 16 distinct bank pairs, and a warp's Z stores form
two runs of 16 consecutive samples."""
import numpy as np

R1 = R2 = 32
N2 = N1 = 1024
TB, TBW = 8, 16
NT = TBW * R2
SB = ((R1 + 15) // 16) * 16 + 1
SC = R2 * SB + ((2 - (R2 * SB) % 16) + 16) % 16
BUF = TBW * SC                       # float2 words of the tile / exchange buffer


def _maps():
    t = np.arange(NT)
    c = (t & 7) + 8 * ((t >> 4) & 1)
    lo, hi = (t >> 3) & 1, t >> 5
    return t, c, lo + 2 * hi, lo + 2 * hi      # c, b (step 1), u (step 2)


def test_thread_maps_are_bijective():
    t, c, b, u = _maps()
    assert SC >= N2 and SC % 16 == 2
    assert len(set(zip(c.tolist(), b.tolist()))) == NT and b.max() == R2 - 1 and c.max() == TBW - 1
    assert len(set(zip(c.tolist(), u.tolist()))) == NT and u.max() == R1 - 1


def test_tile_reads_cover_the_copied_tile():
    t, c, b, u = _maps()
    cblk = (c >> 3) * (N2 * TB) + (c & 7)
    idx = np.concatenate([cblk + (R2 * a + b) * TB for a in range(R1)])
    assert np.array_equal(np.sort(idx), np.arange(TBW * N2))     # the 128 KB copied by the 16 x 512 cp.async
    assert idx.max() < BUF and (15 * NT + NT) * 16 <= BUF * 8


def _conflict_free(words):
    """64-bit accesses of one half-warp: 16 distinct bank pairs."""
    banks = (2 * np.asarray(words)) % 32
    return len(set(banks.tolist())) == 16


def test_shared_accesses_are_conflict_free():
    t, c, b, u = _maps()
    cblk = (c >> 3) * (N2 * TB) + (c & 7)
    for half in range(NT // 16):
        s = slice(16 * half, 16 * half + 16)
        for a in range(R1):
            assert _conflict_free(cblk[s] + (R2 * a + b[s]) * TB)               # step 1 tile reads
        for k in range(R1):
            w = c[s] * SC + b[s] * SB + k                                    # exchange writes (u = k)
            assert _conflict_free(w) and w.max() < BUF
            r = c[s] * SC + k * SB + u[s]                                    # exchange reads (bb = k)
            assert _conflict_free(r) and r.max() < BUF


def test_warp_stores_are_two_runs_of_sixteen():
    t, c, b, u = _maps()
    for w in range(NT // 32):
        s = slice(32 * w, 32 * w + 32)
        samples = np.sort(c[s] + N1 * u[s])
        runs = np.split(samples, np.flatnonzero(np.diff(samples) != 1) + 1)
        assert [len(x) for x in runs] == [16, 16]
