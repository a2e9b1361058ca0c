"""GPU parity of the bank and tile steps: TaylorF2 templates, sigma^2 (float64), sw, the tile SVD, basis series and
stacked A, against the oracle and the reference's own closures (tests/golden/filt_tile.npz)."""
import numpy as np
import pytest
import torch

from oracle import filt as of
from oracle import synth

pytestmark = pytest.mark.gpu


def test_taylorf2_matches_oracle():
    from gwb200 import templates
    flen, df = (1 << 17) + 1, 1 / 64.
    bank = dict(mass1=np.array([30.0, 5.0, 60.0, 12.0]), mass2=np.array([25.0, 3.2, 40.0, 9.0]),
                spin1z=np.array([0.0, 0.5, -0.8, 0.3]), spin2z=np.array([0.0, -0.2, 0.4, 0.0]),
                ecc=np.array([0.0, 0.0, 0.2, 0.1]))
    H, km = templates.generate(bank, np.arange(4), flen, df)
    H = H.cpu().numpy()
    for i in range(4):
        ref = synth.taylorf2(flen, df, bank['mass1'][i], bank['mass2'][i], bank['spin1z'][i], bank['spin2z'][i],
                             bank['ecc'][i])
        ref[km[i]:] = 0                        # the bin at f_ISCO itself may fall on either side; compare below kend
        k = np.arange(int(20 / df), km[i])
        rel = np.abs(H[i, k] - ref[k]) / np.abs(ref[k])
        assert rel.max() < 2e-5, (i, rel.max())
        assert (H[i, :int(20 / df)] == 0).all() and (H[i, km[i]:] == 0).all()


def test_sigma2_and_sw_match_oracle(golden):
    from gwb200 import fp_filter
    g = golden('filt_tile')
    H = torch.from_numpy(g['H']).cuda()
    IP = np.stack([g['IP'], g['IP'] * 0.5, g['IP'] * 2]).astype(np.float32)
    sig, norm = fp_filter.sigma2(H, torch.from_numpy(IP).cuda(), float(g['df']))
    sref, _ = of.sigma2(g['H'], IP, float(g['df']))
    np.testing.assert_allclose(sig.cpu().numpy(), sref, rtol=1e-12)
    sw, isw = fp_filter.derive_sw(torch.from_numpy(IP).cuda())
    swr, iswr = of.derive_sw(IP)
    assert np.array_equal(sw.cpu().numpy(), swr) and np.array_equal(isw.cpu().numpy(), iswr)


def test_svd_tile_matches_reference(golden):
    from gwb200 import fp_filter
    g = golden('filt_tile')
    H = torch.from_numpy(g['H']).cuda()
    sw = torch.from_numpy(g['sw']).cuda()
    G = fp_filter.gram(H, sw, int(g['kmin'])).cpu().numpy()
    Gr = of.gram(g['H'], g['sw'], int(g['kmin']))
    np.testing.assert_allclose(G, Gr, rtol=1e-10, atol=1e-12 * np.abs(Gr).max())
    r, A, Vh, worst = fp_filter.svd_tile(H, sw, int(g['kmin']), float(g['eps']))
    assert r == int(g['r'])
    assert abs(worst - float(g['worst'])) < 2e-5
    # the reconstruction conj(A) Vh = W W^H H' is independent of the eigenvectors' phases (the device solver's differ
    # from LAPACK's); the filter uses A with conj(Vh) (fp_filter.py:592)
    rec = A.cpu().numpy().astype(np.complex128).conj() @ Vh.cpu().numpy().astype(np.complex128)
    rec_ref = g['A'].astype(np.complex128).conj() @ g['Vh'].astype(np.complex128)
    assert (np.linalg.norm(rec - rec_ref, axis=1) / np.linalg.norm(rec_ref, axis=1)).max() < 2e-5


@pytest.mark.parametrize('form', ['f16', 'f32', 'bf16x3'])
def test_basis_series_and_gemm_rebuild_the_reference_snr(golden, form):
    """Basis series + stacked A + fused GEMM (per-sample max over 128 blocks) rebuild the reference's SNR series."""
    from gwb200 import fp_filter, fp_gemm
    g = golden('filt_tile')
    H = torch.from_numpy(g['H']).cuda()
    sw = torch.from_numpy(g['sw']).cuda()
    cl = fp_filter.make_closures(int(g['kmin']), H.shape[1], int(g['tlen']), sw, float(g['eps']), form=form)
    r, A, Vh, worst = cl.svd_tile(H)
    Dws = torch.from_numpy(g['D'] * g['isw']).cuda()
    a0, Tn = int(g['a0']), int(g['Tn'])
    Z, scale = cl.basis_series(Vh, Dws, a0, Tn)
    assert abs(scale - float(g['scale'])) < 1e-5 * float(g['scale'])
    Are, Aim = cl.stacked_A(A, torch.from_numpy(g['nrm_s']).cuda(), scale, fp_filter.kp_of(r))
    if form == 'bf16x3':
        V, I = fp_gemm.fused_peaks_split(Are[0], Are[1], Aim[0], Aim[1], Z[0], Z[1], H.shape[0], Tn)
        zf = (Z[0].float() + Z[1].float()).cpu().numpy()
        ar = (Are[0].float() + Are[1].float()).cpu().numpy()
        ai = (Aim[0].float() + Aim[1].float()).cpu().numpy()
    else:
        V, I = fp_gemm.fused_peaks(Are, Aim, Z, H.shape[0], Tn)
        zf, ar, ai = Z.float().cpu().numpy(), Are.float().cpu().numpy(), Aim.float().cpu().numpy()
    # the SNR series these operands define, against the reference's fp16 operands
    snr = np.hypot(ar @ zf, ai @ zf)
    snr_ref = np.hypot(g['Are'].astype(np.float32) @ g['Z'].astype(np.float32),
                       g['Aim'].astype(np.float32) @ g['Z'].astype(np.float32))
    tol = 3e-3 if form == 'f16' else 2e-3          # the reference's own operands are fp16
    assert np.abs(snr - snr_ref).max() < tol * snr_ref.max()
    # the GEMM's block maxima are the maxima of that series
    Vr = (snr ** 2).reshape(snr.shape[0], -1, 128).max(2)
    np.testing.assert_allclose(V.cpu().numpy(), Vr, rtol=1e-4)
    t = int(float(g['t0']) * 2048) - a0
    assert abs(int(I[3].cpu().numpy()[np.argmax(V[3].cpu().numpy())]) - t) <= 2


@pytest.mark.parametrize('tlen,flen', [(1 << 12, None), (1 << 13, 3000), (1 << 15, None), (1 << 20, None)])
def test_fourstep_order(tlen, flen):
    """P[k2 (N1/2) + k1] = X[N2 k1 + k2] isw for k1 < N1/2, P[N/2] = X[N/2] isw, zero from flen on."""
    from gwb200 import fp_filter
    rng = np.random.default_rng(7)
    flen = tlen // 2 + 1 if flen is None else flen
    X = (rng.standard_normal((3, flen)) + 1j * rng.standard_normal((3, flen))).astype(np.complex64)
    isw = rng.uniform(0.5, 2, flen).astype(np.float32)
    P = fp_filter.fourstep_order(torch.from_numpy(X).cuda(), tlen, torch.from_numpy(isw).cuda()).cpu().numpy()
    p = (tlen.bit_length() - 1 + 1) // 2
    N1, N2 = 1 << p, tlen >> p
    full = np.zeros((3, tlen // 2 + 1), np.complex64)
    full[:, :flen] = X * isw
    ref = np.empty_like(full)
    ref[:, :tlen // 2] = full[:, :tlen // 2].reshape(3, N1 // 2, N2).transpose(0, 2, 1).reshape(3, -1)
    ref[:, tlen // 2] = full[:, tlen // 2]
    assert np.array_equal(P, ref)


@pytest.mark.parametrize('tlen,wrows,ring', [(1 << 12, None, False), (1 << 13, 32, False), (1 << 15, None, False),
                                             (1 << 16, 32, False), (1 << 20, 8, False), (1 << 20, None, False),
                                             (1 << 20, None, True)])
def test_fused_basis_series_matches_float64_transform(tlen, wrows, ring):
    """The fused basis series (fp32 output) times its scale equals ifft(conj(Vh) D isw) over the span: two passes with
    the rows in batches of wrows through W, or (2^20) the persistent ring form with W in L2."""
    from gwb200 import fp_filter
    rng = np.random.default_rng(tlen % 1000)
    flen = tlen // 2 + 1
    r = 70
    Vh = (rng.standard_normal((r, flen)) + 1j * rng.standard_normal((r, flen))).astype(np.complex64)
    D = (rng.standard_normal(flen) + 1j * rng.standard_normal(flen)).astype(np.complex64)
    isw = rng.uniform(0.5, 2, flen).astype(np.float32)
    Dw = D * isw
    a0, Tn = tlen // 16, tlen - tlen // 8
    ws = fp_filter.FusedBasisWorkspace(tlen, flen, r, wrows=wrows, ring=ring)
    Z = torch.zeros((2 * r, Tn), dtype=torch.float32, device='cuda')
    Vp = fp_filter.fourstep_order(torch.from_numpy(Vh).cuda(), tlen)
    Dp = fp_filter.fourstep_order(torch.from_numpy(D).cuda(), tlen, torch.from_numpy(isw).cuda())
    sc = fp_filter.basis_series_fused(ws, Vp, Dp, a0, Tn, Z, None, 'f32', im_off=r)
    scale = float(sc.item())
    zb = of.basis_series_complex(Vh, Dw, a0, Tn, tlen)
    got = (Z[:r].double() + 1j * Z[r:].double()).cpu().numpy() * scale
    err = np.abs(got - zb).max() / np.abs(zb).max()
    assert err < 2e-5, err
    # Parseval scale over the first min(64, wrows) rows (the ring form: the first chunk of two rows)
    nf = 2 if ring else min(64, ws.wrows)
    q = np.conj(Vh[:nf].astype(np.complex128)) * Dw
    assert abs(scale - np.sqrt((np.abs(q) ** 2).sum() / nf / 2)) < 1e-5 * scale


@pytest.mark.parametrize('tlen,wrows,ring', [(1 << 13, None, False), (1 << 16, 32, False), (1 << 20, 8, False),
                                             (1 << 20, None, True)])
def test_fused_basis_series_fp8_rows(tlen, wrows, ring):
    """fp8 form: rowscale[j] = sqrt(sum_k |q_jk|^2 / 2) / 16 (Parseval), and Z row j holds z_j / rowscale[j] rounded to
    e4m3 (3 mantissa bits: within 2^-4 relative, or half the smallest subnormal step for the smallest values), plus
    the float32 transform's own error (which can move a value across a rounding midpoint)."""
    from gwb200 import fp_filter
    rng = np.random.default_rng(tlen % 997)
    flen = tlen // 2 + 1
    r = 40
    Vh = (rng.standard_normal((r, flen)) + 1j * rng.standard_normal((r, flen))).astype(np.complex64)
    Vh *= np.linspace(0.2, 3.0, r, dtype=np.float32)[:, None]      # rows of different power
    D = (rng.standard_normal(flen) + 1j * rng.standard_normal(flen)).astype(np.complex64)
    isw = rng.uniform(0.5, 2, flen).astype(np.float32)
    Dw = D * isw
    a0, Tn = tlen // 16, tlen - tlen // 8
    ws = fp_filter.FusedBasisWorkspace(tlen, flen, r, wrows=wrows, ring=ring)
    Kh = fp_filter.kh_of(r, 'fp8')
    Z = torch.zeros((2 * Kh, -(-Tn // 16) * 16), dtype=torch.uint8, device='cuda')
    Vp = fp_filter.fourstep_order(torch.from_numpy(Vh).cuda(), tlen)
    Dp = fp_filter.fourstep_order(torch.from_numpy(D).cuda(), tlen, torch.from_numpy(isw).cuda())
    fp_filter.basis_series_fused(ws, Vp, Dp, a0, Tn, Z, None, 'fp8', im_off=Kh)
    rs = ws.rowscale[:r].double().cpu().numpy()
    q = np.conj(Vh.astype(np.complex128)) * Dw
    rs_ref = np.sqrt((np.abs(q) ** 2).sum(1) / 2) / 16
    np.testing.assert_allclose(rs, rs_ref, rtol=1e-5)
    dec = Z.view(torch.float8_e4m3fn).float().double().cpu().numpy()
    got = (dec[:r, :Tn] + 1j * dec[Kh:Kh + r, :Tn])
    ref = of.basis_series_complex(Vh, Dw, a0, Tn, tlen) / rs[:, None]
    for part_got, part_ref in ((got.real, ref.real), (got.imag, ref.imag)):
        err = np.abs(part_got - part_ref)
        bound = np.maximum(2.0 ** -4 * np.abs(part_ref), 2.0 ** -10) + 1e-5 * np.abs(ref).max()
        assert (err <= bound).all(), (err - bound).max()
    assert np.abs(ref).max() < 448                                   # no saturation at this scale


@pytest.mark.parametrize('form', ['f16', 'bf16', 'bf16x3'])
def test_ring_basis_series_16bit_forms(form):
    """The persistent ring form (N = 2^20) packing 16-bit Z: fp16 and bf16 within their rounding of the float64
    transform, split bf16 (hi + lo) within 2^-16 relative to the series' maximum, against the same scale."""
    from gwb200 import fp_filter
    tlen = 1 << 20
    rng = np.random.default_rng(5)
    flen = tlen // 2 + 1
    r = 9
    Vh = (rng.standard_normal((r, flen)) + 1j * rng.standard_normal((r, flen))).astype(np.complex64)
    D = (rng.standard_normal(flen) + 1j * rng.standard_normal(flen)).astype(np.complex64)
    isw = rng.uniform(0.5, 2, flen).astype(np.float32)
    a0, Tn = tlen // 16, tlen - tlen // 8
    ws = fp_filter.FusedBasisWorkspace(tlen, flen, r, ring=True)
    Kh = fp_filter.kh_of(r, form)
    dt = fp_filter._z_dtype(form)
    Z = torch.zeros((2 * Kh, Tn), dtype=dt, device='cuda')
    Zlo = torch.zeros_like(Z) if form == 'bf16x3' else None
    Vp = fp_filter.fourstep_order(torch.from_numpy(Vh).cuda(), tlen)
    Dp = fp_filter.fourstep_order(torch.from_numpy(D).cuda(), tlen, torch.from_numpy(isw).cuda())
    scale = float(fp_filter.basis_series_fused(ws, Vp, Dp, a0, Tn, Z, Zlo, form, im_off=Kh).item())
    zf = Z.double() + (Zlo.double() if Zlo is not None else 0)
    got = (zf[:r] + 1j * zf[Kh:Kh + r]).cpu().numpy() * scale
    zb = of.basis_series_complex(Vh, D * isw, a0, Tn, tlen)
    err = np.abs(got - zb) / np.abs(zb).max()
    assert err.max() < {'f16': 1e-3, 'bf16': 8e-3, 'bf16x3': 3e-5}[form], err.max()


@pytest.mark.parametrize('form', ['f16', 'bf16', 'bf16x3', 'f32', 'fp8'])
@pytest.mark.parametrize('da0,dtn', [(8, -24), (9, -23)])
def test_pass2_sixteen_columns_bit_identical(form, da0, dtn):
    """The 16-column pass 2 (gwb_basis_set_pass2_columns(form, 16)) writes the same Z bits as the 8-column kernels at
    N = 2^20, for every Z encoding, with rows that end mid-chunk (r = 11) and an analysed span that starts and ends
    inside a column block; with its paired stores (even a0 and Tn) and with per-sample stores
    (gwb_basis_set_pass2_pairs(0), and odd a0 and Tn, where pairs do not apply)."""
    from gwb200 import _lib, fp_filter
    tlen = 1 << 20
    rng = np.random.default_rng(8)
    flen = tlen // 2 + 1
    r = 11
    Vh = (rng.standard_normal((r, flen)) + 1j * rng.standard_normal((r, flen))).astype(np.complex64)
    D = (rng.standard_normal(flen) + 1j * rng.standard_normal(flen)).astype(np.complex64)
    isw = rng.uniform(0.5, 2, flen).astype(np.float32)
    a0, Tn = 98304 + da0, 917504 + dtn
    Kh = fp_filter.kh_of(r, form)
    dt = fp_filter._z_dtype(form)
    Vp = fp_filter.fourstep_order(torch.from_numpy(Vh).cuda(), tlen)
    Dp = fp_filter.fourstep_order(torch.from_numpy(D).cuda(), tlen, torch.from_numpy(isw).cuda())
    out = {}
    try:
        for cols, pairs in ((8, 1), (16, 0), (16, 1)):
            _lib.call('gwb_basis_set_pass2_columns', -1, cols)
            _lib.call('gwb_basis_set_pass2_pairs', pairs)
            ws = fp_filter.FusedBasisWorkspace(tlen, flen, r)
            Z = torch.full((2 * Kh, -(-Tn // 16) * 16), 7 if dt == torch.uint8 else 3.0, dtype=dt, device='cuda')
            Zlo = torch.full_like(Z, 5.0) if form == 'bf16x3' else None
            fp_filter.basis_series_fused(ws, Vp, Dp, a0, Tn, Z, Zlo, form, im_off=Kh)
            out[cols, pairs] = [Z.cpu()] + ([Zlo.cpu()] if Zlo is not None else []) + [ws.scale.cpu()]
            if form == 'fp8':
                out[cols, pairs].append(ws.rowscale[:r].cpu())
    finally:
        _lib.call('gwb_basis_set_pass2_columns', -1, 16)
        _lib.call('gwb_basis_set_pass2_pairs', 1)
    for key in ((16, 0), (16, 1)):
        for x, y in zip(out[8, 1], out[key]):
            assert torch.equal(x.view(torch.uint8), y.view(torch.uint8)), key


@pytest.mark.parametrize('n,spread', [(64, 6), (248, 12), (256, 14)])
def test_device_jacobi_eigh_matches_lapack(n, spread):
    """The device's one-sided Jacobi (fp_filter.eigh_device, float64) against LAPACK on Hermitian positive
    semi-definite matrices with eigenvalues over `spread` decades: eigenvalues within 1e-12 of the largest, the
    projector onto the eigenvectors of the eigenvalues above 1e-4 of the largest within 1e-9, unitary eigenvectors."""
    from gwb200 import fp_filter
    rng = np.random.default_rng(n)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)) + 1j * rng.standard_normal((n, n)))
    lam = np.logspace(0, -spread, n)
    G = (Q * lam[None, :]) @ Q.conj().T
    G = (G + G.conj().T) / 2
    l_d, W_d = fp_filter.eigh_device(torch.from_numpy(G).cuda())
    l_h, W_h = np.linalg.eigh(G)
    l_h, W_h = l_h[::-1], W_h[:, ::-1]
    assert np.abs(l_d - l_h).max() < 1e-12 * l_h[0]
    k = int((l_h > 1e-4 * l_h[0]).sum())
    P_d = W_d[:, :k] @ W_d[:, :k].conj().T
    P_h = W_h[:, :k] @ W_h[:, :k].conj().T
    assert np.abs(P_d - P_h).max() < 1e-9
    assert np.abs(W_d.conj().T @ W_d - np.eye(n)).max() < 1e-11


def test_svd_tile_device_eigh_matches_host(golden):
    """svd_tile with the device eigendecomposition gives the same rank, worst lost power and reconstruction as with
    LAPACK on the host, on the reference's svd_tile fixture."""
    from gwb200 import fp_filter
    g = golden('filt_tile')
    H = torch.from_numpy(g['H']).cuda()
    sw = torch.from_numpy(g['sw']).cuda()
    out = {}
    for e in ('host', 'device'):
        r, A, Vh, worst = fp_filter.svd_tile(H, sw, int(g['kmin']), float(g['eps']), eigh=e)
        out[e] = (r, worst, (A.to(torch.complex128).conj() @ Vh.to(torch.complex128)).cpu().numpy())
    assert out['host'][0] == out['device'][0]
    assert abs(out['host'][1] - out['device'][1]) < 1e-9
    rec_h, rec_d = out['host'][2], out['device'][2]
    assert np.abs(rec_d - rec_h).max() < 1e-4 * np.abs(rec_h).max()
