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


def _byte_perm(x, y, s):
    """__byte_perm(x, y, s): byte i of the result is byte (s >> 4 i) & 7 of the 8 bytes {y:x}."""
    b = (int(x) | (int(y) << 32)).to_bytes(8, 'little')
    return int.from_bytes(bytes(b[(s >> (4 * i)) & 7] for i in range(4)), 'little')


def _bf16_bits(v):
    """Round-to-nearest-even bf16 bits of float32 values."""
    u = np.asarray(v, np.float32).view(np.uint32).astype(np.uint64)
    return ((u + 0x7FFF + ((u >> 16) & 1)) >> 16).astype(np.uint32)


def test_paired_z_stores_place_every_sample():
    """The paired stores of pass 2 (PairStore in csrc/fft_basis.cu), emulated on the CPU for a lane pair (c even and
    odd, samples t and t + 1): the even lane's word holds the two real parts, the odd lane's the two imaginary parts,
    for 16-bit Z (selector 0x5410 / 0x3276) and for split bf16 (hi 0x5410 / 0x3254, lo 0x7610 / 0x3276, sent word
    0x7632 / 0x5410), the same bits as one 16-bit store per plane and sample."""
    rng = np.random.default_rng(3)
    for _ in range(200):
        x = rng.standard_normal(4).astype(np.float32)          # (re, im) of sample t, then of sample t + 1
        hr = _bf16_bits(x)                                     # hi of re_t, im_t, re_t1, im_t1
        back = (hr.astype(np.uint64) << 16).astype(np.uint32).view(np.float32)
        lo = _bf16_bits(x - back)
        H = [int(hr[0]) | int(hr[1]) << 16, int(hr[2]) | int(hr[3]) << 16]     # lane even, lane odd
        L = [int(lo[0]) | int(lo[1]) << 16, int(lo[2]) | int(lo[3]) << 16]
        # 16-bit forms: each lane sends its packed (re, im) word
        R = [H[1], H[0]]
        w_even = _byte_perm(H[0], R[0], 0x5410)
        w_odd = _byte_perm(H[1], R[1], 0x3276)
        assert w_even == int(hr[0]) | int(hr[2]) << 16                           # re of t, t + 1
        assert w_odd == int(hr[1]) | int(hr[3]) << 16                            # im of t, t + 1
        # split bf16: even sends (im hi, im lo), odd sends (re hi, re lo)
        S = [_byte_perm(H[0], L[0], 0x7632), _byte_perm(H[1], L[1], 0x5410)]
        R = [S[1], S[0]]
        assert _byte_perm(H[0], R[0], 0x5410) == int(hr[0]) | int(hr[2]) << 16   # re hi plane
        assert _byte_perm(L[0], R[0], 0x7610) == int(lo[0]) | int(lo[2]) << 16   # re lo plane
        assert _byte_perm(H[1], R[1], 0x3254) == int(hr[1]) | int(hr[3]) << 16   # im hi plane
        assert _byte_perm(L[1], R[1], 0x3276) == int(lo[1]) | int(lo[3]) << 16   # im lo plane
