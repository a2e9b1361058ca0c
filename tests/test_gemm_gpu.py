"""GPU parity of the fused reconstruction GEMM (+|z|^2 +argmax) and of the window-peak kernel.

References: the reference's own Triton kernel outputs (tests/golden/fp_gemm_*.npz) and the numpy oracle
(oracle/gemm.py, itself checked against those fixtures on the CPU). Peak indices must be identical wherever the
block's maximum is not a near-tie (two values within the accumulation-order rounding), and bit-identical, ties
included, when every product and sum is exact (integer operands)."""
import numpy as np
import pytest
import torch

from oracle import gemm as og

pytestmark = pytest.mark.gpu

RTOL = 2e-5   # fp32 accumulation in a different order than numpy / Triton


def _near_tie_mask(Are, Aim, Z, M, Tn, I_ref, rel=1e-5):
    """True where the reference block's winner is within rel of another column (argmax legitimately ambiguous)."""
    zr = Are[:M].astype(np.float32) @ Z[:, :Tn].astype(np.float32)
    zi = Aim[:M].astype(np.float32) @ Z[:, :Tn].astype(np.float32)
    pw = zr * zr + zi * zi
    nblk = I_ref.shape[1]
    pad = nblk * 128 - Tn
    if pad:
        pw = np.concatenate([pw, np.full((M, pad), -1.0, np.float32)], 1)
    pw = pw.reshape(M, nblk, 128)
    s = np.sort(pw, axis=2)
    return (s[..., -1] - s[..., -2]) <= rel * np.abs(s[..., -1])


def _grouped(Vb, Ib, tie, group):
    """Group the block results as the kernel does; a group's winner is ambiguous where a block inside it is, or where
    two block maxima of the group nearly tie."""
    M, nblk = Vb.shape
    Vr, Ir = og.group_reduce(Vb, Ib, group)
    nout = Vr.shape[1]
    pad = nout * group - nblk
    t = np.pad(tie, ((0, 0), (0, pad))).reshape(M, nout, group).any(2)
    s = np.sort(np.pad(Vb, ((0, 0), (0, pad)), constant_values=-1).reshape(M, nout, group), 2)
    if group > 1:
        t |= (s[..., -1] - s[..., -2]) <= 1e-5 * np.abs(s[..., -1])
    return Vr, Ir, t


def _dev(a, dt):
    return torch.from_numpy(np.ascontiguousarray(a)).to('cuda', dt)


def _check(V, I, Vr, Ir, tie):
    np.testing.assert_allclose(V, Vr, rtol=RTOL, atol=1e-6)
    bad = (I != Ir) & ~tie
    assert not bad.any(), 'index mismatch away from near-ties at %s' % (np.argwhere(bad)[:5],)


@pytest.mark.parametrize('name', ['fp_gemm_a', 'fp_gemm_ragged', 'fp_gemm_ties'])
def test_f16_matches_reference_triton_kernel(golden, name):
    from gwb200 import fp_gemm
    g = golden(name)
    M, Tn, K = int(g['M']), int(g['Tn']), g['Are'].shape[1]
    Z = g['Z']
    ldz = -(-Tn // 8) * 8   # TMA wants the row stride a multiple of 16 bytes
    Zp = np.zeros((K, ldz), np.float16)
    Zp[:, :Tn] = Z
    V, I = fp_gemm.fused_peaks(_dev(g['Are'], torch.float16), _dev(g['Aim'], torch.float16),
                               _dev(Zp, torch.float16)[:, :Tn], M, Tn, (64, 64, 4, 2))
    V, I = V.cpu().numpy(), I.cpu().numpy()
    if name == 'fp_gemm_ties':
        assert np.array_equal(V, g['V']) and np.array_equal(I, g['I'])
    else:
        _check(V, I, g['V'], g['I'], _near_tie_mask(g['Are'], g['Aim'], Z, M, Tn, g['I']))


@pytest.mark.parametrize('M,K,Tn,group', [(256, 64, 131072, 1), (256, 64, 131072, 16), (300, 128, 40000, 1),
                                          (100, 64, 2048 * 7 + 640, 16), (128, 128, 8192, 4)])
def test_f16_random_against_oracle(M, K, Tn, group):
    from gwb200 import fp_gemm
    rng = np.random.default_rng(M + K + Tn)
    Are = rng.standard_normal((M, K)).astype(np.float16)
    Aim = rng.standard_normal((M, K)).astype(np.float16)
    Z = rng.standard_normal((K, Tn)).astype(np.float16)
    V, I = fp_gemm.fused_peaks(_dev(Are, torch.float16), _dev(Aim, torch.float16), _dev(Z, torch.float16), M, Tn,
                               group=group)
    Vr, Ir = og.gemm_absmax(Are, Aim, Z, M, Tn)
    tie = _near_tie_mask(Are, Aim, Z, M, Tn, Ir)
    if group > 1:
        Vr, Ir, tie = _grouped(Vr, Ir, tie, group)
    _check(V.cpu().numpy(), I.cpu().numpy(), Vr, Ir, tie)


def test_f16_integer_operands_bit_exact_with_ties():
    from gwb200 import fp_gemm
    rng = np.random.default_rng(7)
    M, K, Tn = 256, 64, 128 * 300 + 16
    Are = rng.integers(-2, 3, (M, K)).astype(np.float16)
    Aim = rng.integers(-2, 3, (M, K)).astype(np.float16)
    Z = rng.integers(-1, 2, (K, Tn)).astype(np.float16)
    V, I = fp_gemm.fused_peaks(_dev(Are, torch.float16), _dev(Aim, torch.float16), _dev(Z, torch.float16), M, Tn)
    Vr, Ir = og.gemm_absmax(Are, Aim, Z, M, Tn)
    assert np.array_equal(V.cpu().numpy(), Vr)
    assert np.array_equal(I.cpu().numpy(), Ir)


@pytest.mark.parametrize('M,K,Tn,group', [(256, 64, 32768, 1), (130, 40, 5000, 16), (70, 37, 3001, 4)])
def test_f32_form_against_oracle(M, K, Tn, group):
    from gwb200 import fp_gemm
    rng = np.random.default_rng(11)
    Are = rng.standard_normal((M, K)).astype(np.float32)
    Aim = rng.standard_normal((M, K)).astype(np.float32)
    Z = rng.standard_normal((K, Tn)).astype(np.float32)
    V, I = fp_gemm.fused_peaks(_dev(Are, torch.float32), _dev(Aim, torch.float32), _dev(Z, torch.float32), M, Tn,
                               group=group)
    Vr, Ir = og.gemm_absmax(Are, Aim, Z, M, Tn)
    tie = _near_tie_mask(Are, Aim, Z, M, Tn, Ir)
    if group > 1:
        Vr, Ir, tie = _grouped(Vr, Ir, tie, group)
    _check(V.cpu().numpy(), I.cpu().numpy(), Vr, Ir, tie)


@pytest.mark.parametrize('M,K,Tn,group', [(256, 384, 40000, 16), (200, 72, 4998, 3), (64, 16, 130, 1)])
def test_f32_async_kernel_bit_identical(M, K, Tn, group):
    """The fp32 form's cp.async kernel (the default where K, lda, ldz are multiples of 4) gives the same V and I bits
    as the synchronous kernel (gwb_f32_set_async(0)): the same fp32 sums in the same K order, samples past Tn (inside
    the last 16-byte copy and past it) ignored."""
    from gwb200 import _lib, fp_gemm
    rng = np.random.default_rng(K + Tn)
    Are = _dev(rng.standard_normal((M, K)).astype(np.float32), torch.float32)
    Aim = _dev(rng.standard_normal((M, K)).astype(np.float32), torch.float32)
    ldz = -(-Tn // 4) * 4
    Zf = torch.zeros((K, ldz), dtype=torch.float32, device='cuda')
    Zf[:, :Tn] = _dev(rng.standard_normal((K, Tn)).astype(np.float32), torch.float32)
    Zf[:, Tn:] = float('nan')                    # never read as a sample: NaN there would show in V
    Z = Zf[:, :Tn]
    out = {}
    try:
        for mode in (0, 1):
            _lib.call('gwb_f32_set_async', mode)
            out[mode] = [x.cpu() for x in fp_gemm.fused_peaks(Are, Aim, Z, M, Tn, group=group)]
    finally:
        _lib.call('gwb_f32_set_async', 1)
    assert torch.equal(out[0][0].view(torch.int32), out[1][0].view(torch.int32))
    assert torch.equal(out[0][1], out[1][1])
    assert torch.isfinite(out[1][0]).all()


def test_bf16x3_form_close_to_fp32():
    from gwb200 import fp_gemm
    rng = np.random.default_rng(5)
    M, K, Tn = 256, 64, 65536
    Are = rng.standard_normal((M, K)).astype(np.float32)
    Aim = rng.standard_normal((M, K)).astype(np.float32)
    Z = rng.standard_normal((K, Tn)).astype(np.float32)

    def split(x):
        t = torch.from_numpy(x).cuda()
        hi = t.to(torch.bfloat16)
        lo = (t - hi.float()).to(torch.bfloat16)
        return hi.contiguous(), lo.contiguous()
    (rh, rl), (ih, il), (zh, zl) = split(Are), split(Aim), split(Z)
    V, I = fp_gemm.fused_peaks_split(rh, rl, ih, il, zh, zl, M, Tn)
    Vr, Ir = og.gemm_absmax(Are, Aim, Z, M, Tn)
    V = V.cpu().numpy()
    rel = np.abs(V - Vr) / Vr
    assert rel.max() < 1e-4, rel.max()
    assert (I.cpu().numpy() == Ir).mean() > 0.995


def test_window_peaks_bit_exact():
    from gwb200 import peak_kernel
    rng = np.random.default_rng(3)
    rows, N, a0, cw, nwin = 37, 3 * 2048 + 500, 300, 2048, 3
    z = (rng.standard_normal((rows, N)) + 1j * rng.standard_normal((rows, N))).astype(np.complex64)
    z[5, a0 + 10] = z[5, a0 + 900] = 10 + 0j          # a planted tie: the first offset must win
    p, i = peak_kernel.window_peaks(torch.from_numpy(z).cuda(), a0, cw, nwin)
    pr, ir = og.window_peaks(z, a0, cw, nwin)
    assert np.array_equal(p.cpu().numpy(), pr)
    assert np.array_equal(i.cpu().numpy(), ir)
    assert i[5, 0].item() == 10


def _compact(rng, M, r, Kh, Tn, dtype):
    """Random complex As (M, r) and zb (r, Tn) in the compact layout, plus the reference's stacked layout."""
    As = (rng.standard_normal((M, r)) + 1j * rng.standard_normal((M, r))).astype(np.complex64)
    zb = (rng.standard_normal((r, Tn)) + 1j * rng.standard_normal((r, Tn))).astype(np.complex64)
    A = np.zeros((M, 2 * Kh), np.float32)
    A[:, :r], A[:, Kh:Kh + r] = As.real, As.imag
    Z = np.zeros((2 * Kh, Tn), np.float32)
    Z[:r], Z[Kh:Kh + r] = zb.real, zb.imag
    A, Z = A.astype(dtype).astype(np.float32), Z.astype(dtype).astype(np.float32)   # the values the kernel sees
    Are = np.concatenate([A[:, :Kh], -A[:, Kh:]], 1)
    Aim = np.concatenate([A[:, Kh:], A[:, :Kh]], 1)
    return A, Z, Are, Aim


@pytest.mark.parametrize('M,r,Tn,group', [(256, 60, 2048 * 20, 16), (256, 190, 2048 * 6, 16), (300, 100, 40000, 1),
                                          (100, 17, 2048 * 3 + 384, 4)])
@pytest.mark.parametrize('split', [False, True])
def test_cplx_f16_against_oracle(M, r, Tn, group, split):
    from gwb200 import _lib
    work = torch.empty(_lib.load().gwb_fused_peaks_cplx_work_bytes(M), dtype=torch.uint8, device='cuda') if split \
        else None
    rng = np.random.default_rng(r + M)
    Kh = -(-r // 16) * 16
    A, Z, Are, Aim = _compact(rng, M, r, Kh, Tn, np.float16)
    Ad, Zd = _dev(A, torch.float16), _dev(Z, torch.float16)
    nout = -(-(-(-Tn // 128)) // group)
    V = torch.empty((M, nout), dtype=torch.float32, device='cuda')
    I = torch.empty((M, nout), dtype=torch.int32, device='cuda')
    _lib.call('gwb_fused_peaks_cplx', 0, _lib.ptr(Ad), None, Ad.stride(0), _lib.ptr(Zd), None, Zd.stride(0), M, Kh, Tn,
              group, _lib.ptr(V), _lib.ptr(I), V.stride(0), None, _lib.ptr(work), 0 if work is None else work.numel(),
              _lib.stream_ptr())
    Vr, Ir = og.gemm_absmax(Are, Aim, Z, M, Tn)
    tie = _near_tie_mask(Are, Aim, Z, M, Tn, Ir)
    if group > 1:
        Vr, Ir, tie = _grouped(Vr, Ir, tie, group)
    _check(V.cpu().numpy(), I.cpu().numpy(), Vr, Ir, tie)


_PAIR_CFGS = [None, (1, 0), (1, 2), (1, 0, 1)]


def _with_config(form, Kh, cfg, fn):
    """Runs fn with the launch table entry (pair, stages[, order]) for (form, Kh), or the default without one."""
    from gwb200 import _lib
    if cfg is None:
        return fn()
    _lib.call('gwb_gemm_set_config', form, Kh, cfg[0], cfg[1], cfg[2] if len(cfg) > 2 else 0)
    try:
        return fn()
    finally:
        _lib.call('gwb_gemm_clear_configs')


@pytest.mark.parametrize('form,r,cfg', [(1, 120, None)] +
                         [(2, r, c) for r in (40, 120, 150, 192, 250) for c in _PAIR_CFGS])
def test_cplx_bf16_forms_against_oracle(form, r, cfg):
    """bf16 and split bf16 (Kh <= 128: A hi and lo resident; beyond: A hi resident, A lo streamed with Z) against
    the float64 stacked product, with whole windows per CTA and with tile-granular ranges (merged windows); the split
    form also on CTA pairs (launch table pair 1; A lo resident or streamed, the most stages or two)."""
    _with_config(form, -(-r // 16) * 16, cfg, lambda: _bf16_forms_case(form, r))


def _bf16_forms_case(form, r):
    from gwb200 import _lib
    rng = np.random.default_rng(form * 100 + r)
    M, Tn, group = 256, 2048 * 8, 16
    Kh = -(-r // 16) * 16
    As = (rng.standard_normal((M, r)) + 1j * rng.standard_normal((M, r))).astype(np.complex64)
    zb = (rng.standard_normal((r, Tn)) + 1j * rng.standard_normal((r, Tn))).astype(np.complex64)
    A = np.zeros((M, 2 * Kh), np.float32)
    A[:, :r], A[:, Kh:Kh + r] = As.real, As.imag
    Z = np.zeros((2 * Kh, Tn), np.float32)
    Z[:r], Z[Kh:Kh + r] = zb.real, zb.imag
    At, Zt = torch.from_numpy(A).cuda(), torch.from_numpy(Z).cuda()
    Ah, Zh = At.to(torch.bfloat16), Zt.to(torch.bfloat16)
    Al, Zl = (At - Ah.float()).to(torch.bfloat16), (Zt - Zh.float()).to(torch.bfloat16)
    nout = -(-(Tn // 128) // group)
    V = torch.empty((M, nout), dtype=torch.float32, device='cuda')
    I = torch.empty((M, nout), dtype=torch.int32, device='cuda')
    Are = np.concatenate([A[:, :Kh], -A[:, Kh:]], 1)
    Aim = np.concatenate([A[:, Kh:], A[:, :Kh]], 1)
    Vr, Ir = og.group_reduce(*og.gemm_absmax(Are, Aim, Z, M, Tn), group)
    work = torch.empty(_lib.load().gwb_fused_peaks_cplx_work_bytes(M), dtype=torch.uint8, device='cuda')
    for wk in (None, work):
        V.fill_(-7.0)
        _lib.call('gwb_fused_peaks_cplx', form, _lib.ptr(Ah), _lib.ptr(Al if form == 2 else None), Ah.stride(0),
                  _lib.ptr(Zh), _lib.ptr(Zl if form == 2 else None), Zh.stride(0), M, Kh, Tn, group, _lib.ptr(V),
                  _lib.ptr(I), V.stride(0), None, _lib.ptr(wk), 0 if wk is None else wk.numel(), _lib.stream_ptr())
        rel = np.abs(V.cpu().numpy() - Vr) / Vr
        # split bf16 carries ~16 bits per operand; one bf16 product ~8 bits, averaged over K terms
        assert rel.max() < (5e-5 if form == 2 else 2e-2), rel.max()
        assert (I.cpu().numpy() == Ir).mean() > (0.99 if form == 2 else 0.8)


@pytest.mark.parametrize('r', [40, 120, 150, 192])
@pytest.mark.parametrize('cfg', _PAIR_CFGS)
def test_cplx_f16_split_a_against_oracle(r, cfg):
    """fp16 Z with A split into fp16 hi + lo (form 6: two products; A hi and lo resident for Kh <= 128, A lo streamed
    with Z beyond) against the float64 product of the fp16 Z values with the unrounded A; also on CTA pairs."""
    _with_config(6, -(-r // 16) * 16, cfg, lambda: _f16_split_a_case(r))


def _f16_split_a_case(r):
    from gwb200 import _lib
    rng = np.random.default_rng(600 + r)
    M, Tn, group = 256, 2048 * 8, 16
    Kh = -(-r // 16) * 16
    As = (rng.standard_normal((M, r)) + 1j * rng.standard_normal((M, r))).astype(np.complex64)
    zb = (rng.standard_normal((r, Tn)) + 1j * rng.standard_normal((r, Tn))).astype(np.complex64)
    A = np.zeros((M, 2 * Kh), np.float32)
    A[:, :r], A[:, Kh:Kh + r] = As.real, As.imag
    Z = np.zeros((2 * Kh, Tn), np.float32)
    Z[:r], Z[Kh:Kh + r] = zb.real, zb.imag
    Z = Z.astype(np.float16).astype(np.float32)                # the Z values the kernel sees
    At = torch.from_numpy(A).cuda()
    Ah = At.to(torch.float16)
    Al = (At - Ah.float()).to(torch.float16)
    Zh = torch.from_numpy(Z).cuda().to(torch.float16)
    nout = -(-(Tn // 128) // group)
    V = torch.empty((M, nout), dtype=torch.float32, device='cuda')
    I = torch.empty((M, nout), dtype=torch.int32, device='cuda')
    Are = np.concatenate([A[:, :Kh], -A[:, Kh:]], 1)
    Aim = np.concatenate([A[:, Kh:], A[:, :Kh]], 1)
    Vr, Ir = og.group_reduce(*og.gemm_absmax(Are, Aim, Z, M, Tn), group)
    work = torch.empty(_lib.load().gwb_fused_peaks_cplx_work_bytes(M), dtype=torch.uint8, device='cuda')
    for wk in (None, work):
        V.fill_(-7.0)
        _lib.call('gwb_fused_peaks_cplx', 6, _lib.ptr(Ah), _lib.ptr(Al), Ah.stride(0), _lib.ptr(Zh), None,
                  Zh.stride(0), M, Kh, Tn, group, _lib.ptr(V), _lib.ptr(I), V.stride(0), None, _lib.ptr(wk),
                  0 if wk is None else wk.numel(), _lib.stream_ptr())
        rel = np.abs(V.cpu().numpy() - Vr) / Vr
        # A carries ~22 bits (hi + lo); Z's own rounding is in the oracle's operands
        assert rel.max() < 5e-5, rel.max()
        assert (I.cpu().numpy() == Ir).mean() > 0.99


def test_cplx_rejects_oversized_kh():
    from gwb200 import _lib
    with pytest.raises(_lib.GwbError, match='shared memory'):
        # Kh = 336: A hi alone (11 swizzle tiles of 16 KB) and two stages exceed the 227 KB of a CTA
        x = torch.zeros((256, 672), dtype=torch.bfloat16, device='cuda')
        z = torch.zeros((672, 4096), dtype=torch.bfloat16, device='cuda')
        V = torch.empty((256, 2), dtype=torch.float32, device='cuda')
        I = torch.empty((256, 2), dtype=torch.int32, device='cuda')
        _lib.call('gwb_fused_peaks_cplx', 2, _lib.ptr(x), _lib.ptr(x), 672, _lib.ptr(z), _lib.ptr(z), 4096, 256, 336,
                  4096, 16, _lib.ptr(V), _lib.ptr(I), 2, None, None, 0, _lib.stream_ptr())


@pytest.mark.parametrize('r', [96, 150])
def test_cplx_fp8_integer_operands_exact(r):
    """fp8 e4m3 form: integer operands in [-4, 4] are exact in e4m3 and every sum is exact in fp32, so V (times the
    per-row scale squared) and the first-index argmax equal the float64 reference exactly."""
    from gwb200 import _lib
    rng = np.random.default_rng(r)
    M, Tn, group = 256, 2048 * 8, 16
    Kh = -(-r // 32) * 32
    A = np.zeros((M, 2 * Kh), np.float32)
    A[:, :r] = rng.integers(-4, 5, (M, r))
    A[:, Kh:Kh + r] = rng.integers(-4, 5, (M, r))
    Z = np.zeros((2 * Kh, Tn), np.float32)
    Z[:r] = rng.integers(-4, 5, (r, Tn))
    Z[Kh:Kh + r] = rng.integers(-4, 5, (r, Tn))
    rs = (1 + np.arange(M) % 3).astype(np.float32)
    A8 = torch.from_numpy(A).to(torch.float8_e4m3fn).view(torch.uint8).cuda()
    Z8 = torch.from_numpy(Z).to(torch.float8_e4m3fn).view(torch.uint8).cuda()
    rsd = torch.from_numpy(rs).cuda()
    nout = -(-(Tn // 128) // group)
    V = torch.empty((M, nout), dtype=torch.float32, device='cuda')
    I = torch.empty((M, nout), dtype=torch.int32, device='cuda')
    Are = np.concatenate([A[:, :Kh], -A[:, Kh:]], 1)
    Aim = np.concatenate([A[:, Kh:], A[:, :Kh]], 1)
    Vr, Ir = og.group_reduce(*og.gemm_absmax(Are, Aim, Z, M, Tn), group)
    work = torch.empty(_lib.load().gwb_fused_peaks_cplx_work_bytes(M), dtype=torch.uint8, device='cuda')
    for wk in (None, work):          # whole windows per CTA, and tile-granular ranges with merged windows
        V.fill_(-7.0)
        _lib.call('gwb_fused_peaks_cplx', 3, _lib.ptr(A8), None, A8.stride(0), _lib.ptr(Z8), None, Z8.stride(0), M, Kh,
                  Tn, group, _lib.ptr(V), _lib.ptr(I), V.stride(0), _lib.ptr(rsd), _lib.ptr(wk),
                  0 if wk is None else wk.numel(), _lib.stream_ptr())
        assert np.array_equal(V.cpu().numpy(), (Vr * rs[:, None] ** 2).astype(np.float32))
        assert np.array_equal(I.cpu().numpy(), Ir)
