"""The compressed filter's tile-level steps: drop-in for the closures of pipeline/fp_filter.py.

The reference defines these as closures inside its main loop (fp_filter.py:354-370 derive, :576-593 svd_tile,
:597-613 basis_series, :615-621 stacked_A, :710-714 template norms). Here
they are functions over explicit arguments, or made by make_closures(...) with the reference's closure variables, so
a caller can keep the reference's call sites. All array work runs in libgwb200; the one host step is the Hermitian
eigendecomposition of the tile's n x n Gram matrix (float64 LAPACK, n <= a few hundred), whose input (the Gram
matrix, O(n^2 flen)) and outputs (Vh, O(r n flen)) are computed on the device in float64 / fp32."""
from types import SimpleNamespace

import numpy as np
import torch

from . import _lib

CH = 1 << 16       # fp_filter.py:42 (kept for reference; the kernels do not chunk)
RB = 64            # basis rows per inverse-FFT batch (fp_filter.py:43)
# Z encodings of the basis-series and pack kernels; fp8 (e4m3 with per-row scales, the screening form) exists in the
# fused basis series and the compact GEMM only. f16x2: fp16 Z with A split into fp16 hi + lo (two GEMM products)
FORMS = {'f16': 0, 'f32': 1, 'bf16x3': 2, 'bf16': 3, 'fp8': 4, 'f16x2': 0}
# operand (A and Z) encodings of the stacked-A and selection kernels
A_FORMS = dict(FORMS, f16x2=5)


def _s():
    return _lib.stream_ptr()


def derive_sw(IPall):
    """fp_filter.py:363-364: sw = sqrt(mean over segments of IP) (float64 mean), isw = 1/sw (0 where sw = 0)."""
    _lib.require_cuda(IPall)
    IPall = IPall.contiguous()
    nseg, flen = IPall.shape
    sw = torch.empty(flen, dtype=torch.float32, device=IPall.device)
    isw = torch.empty_like(sw)
    _lib.call('gwb_sw', _lib.ptr(IPall), _lib.row_stride(IPall), nseg, flen, _lib.ptr(sw), _lib.ptr(isw), _s())
    return sw, isw


def sigma2(H, IPall, df, kmin=0):
    """Template norms (fp_filter.py:710-714) in float64: sig (n, nseg) = 4 df |H|^2 @ IP^T; norm = 4 df / sqrt(sig)."""
    _lib.require_cuda(H, IPall)
    n, flen = H.shape
    nseg = IPall.shape[0]
    part_elems = n * nseg * 64
    part = torch.empty(part_elems, dtype=torch.float64, device=H.device)
    sig = torch.empty((n, nseg), dtype=torch.float64, device=H.device)
    _lib.call('gwb_sigma2', _lib.ptr(H), H.stride(0), n, _lib.ptr(IPall), _lib.row_stride(IPall), nseg, int(kmin), flen,
              float(df), _lib.ptr(part), part_elems, _lib.ptr(sig), sig.stride(0), _s())
    return sig, (4.0 * df) / torch.sqrt(sig)


def gram(H, sw, kmin):
    """G = sum_{k >= kmin} (H sw)(H sw)^H in float64 (complex128, n x n)."""
    n, flen = H.shape
    part_elems = 2 * n * n * 128
    part = torch.empty(part_elems, dtype=torch.float64, device=H.device)
    G = torch.empty((n, n), dtype=torch.complex128, device=H.device)
    _lib.call('gwb_gram', _lib.ptr(H), H.stride(0), n, _lib.ptr(sw), int(kmin), flen, _lib.ptr(part), part_elems,
              _lib.ptr(G), _s())
    return G


# rotation threshold (cosine of a column pair), null-column floor (relative to the largest column of G), sweep limit
EIGH_TOL, EIGH_FLOOR, EIGH_SWEEPS = 1e-13, 1e-12, 40


def eigh_device(Gn):
    """Eigenvalues (descending, float64 numpy) and eigenvectors (columns, complex128 numpy) of a Hermitian positive
    semi-definite matrix (n <= 256, complex128 CUDA tensor) by the device's one-sided Jacobi in float64
    (gwb_eigh_jacobi_sweep: sweeps until one rotates no pair with cosine above EIGH_TOL; columns below EIGH_FLOOR of
    the largest column of G are numerically null and not rotated)."""
    n = Gn.shape[0]
    U = Gn.transpose(0, 1).contiguous()                 # column-major: U[j, i] = G[i, j]
    V = torch.empty_like(U)
    nv = torch.tensor([n], dtype=torch.int32, device=Gn.device)
    rot = torch.zeros(1, dtype=torch.int32, device=Gn.device)
    floor = EIGH_FLOOR * float(torch.linalg.vector_norm(Gn, dim=0).max().item())
    for sweep in range(EIGH_SWEEPS):
        _lib.call('gwb_eigh_jacobi_sweep', _lib.ptr(U), _lib.ptr(V), _lib.ptr(nv), 1, n, int(sweep == 0),
                  EIGH_TOL, floor, _lib.ptr(rot), _s())
        if int(rot.item()) == 0:
            break
    else:
        raise _lib.GwbError('eigh_jacobi_sweep', _lib.GWB_ERR_SHAPE,
                            'no convergence in %d sweeps (%d rotations in the last)' % (EIGH_SWEEPS, int(rot.item())))
    lam = torch.empty(n, dtype=torch.float64, device=Gn.device)
    _lib.call('gwb_eigh_values', _lib.ptr(U), _lib.ptr(nv), 1, n, _lib.ptr(lam), _s())
    lam, Vm = lam.cpu().numpy(), V.cpu().numpy().T       # Vm[:, j] = eigenvector j
    o = np.argsort(-lam, kind='stable')
    return lam[o], Vm[:, o]


def svd_tile(H, sw, kmin, eps, eigh='device'):
    """fp_filter.py:576-593: Gram matrix (float64, device), normalised, Hermitian eigendecomposition (float64 on the
    device by one-sided Jacobi, eigh_device; eigh='host' uses LAPACK on the host instead), rank r = smallest with worst
    lost power <= eps, basis filters Vh (device). Returns (r, A, Vh, worst) with A (n, r) and Vh (r, flen) complex64
    CUDA tensors."""
    _lib.require_cuda(H, sw)
    H = H.contiguous()
    n, flen = H.shape
    Gd = gram(H, sw, kmin)
    G = Gd.cpu().numpy()
    nrm = np.sqrt(np.maximum(G.diagonal().real, 1e-30))
    if eigh == 'host' or n > 256 or n < 2:
        lam, W = np.linalg.eigh(G / (nrm[:, None] * nrm[None, :]))
        lam, W = np.maximum(lam[::-1], 0), W[:, ::-1]
    else:
        nd = torch.from_numpy(nrm).to(H.device)
        lam, W = eigh_device(Gd / (nd[:, None] * nd[None, :]))
        lam = np.maximum(lam, 0)
    worst = (1 - ((np.abs(W) ** 2) * lam[None, :]).cumsum(1)).max(0)
    r = min(int((worst > eps).sum()) + 1, n)
    Wr = W[:, :r]
    s_r = np.sqrt(np.maximum(lam[:r], 1e-12 * lam[0]))
    Bm = ((Wr.conj().T / s_r[:, None]) / nrm[None, :]).astype(np.complex64)
    A = ((Wr * s_r[None, :]).conj() * nrm[:, None]).astype(np.complex64)
    Bm_d = torch.from_numpy(np.ascontiguousarray(Bm)).to(H.device)
    Vh = torch.empty((r, flen), dtype=torch.complex64, device=H.device)
    _lib.call('gwb_basis_vh', _lib.ptr(Bm_d), Bm_d.stride(0), r, n, _lib.ptr(H), H.stride(0), _lib.ptr(sw), int(kmin),
              flen, _lib.ptr(Vh), Vh.stride(0), _s())
    return r, torch.from_numpy(np.ascontiguousarray(A)).to(H.device), Vh, float(worst[r - 1])


def kp_of(r):
    """K padded to a multiple of 64 for 2 r real rows (fp_filter.py:601)."""
    return ((2 * r + 63) // 64) * 64


_TWIDDLES = {}


def twiddles(N, device='cuda'):
    """e^{2 pi i m / N}, m < N, complex64 on the device (cached per (N, device))."""
    key = (int(N), str(torch.device(device)))
    t = _TWIDDLES.get(key)
    if t is None:
        t = torch.empty(N, dtype=torch.complex64, device=device)
        _lib.call('gwb_fft_twiddles', int(N), _lib.ptr(t), _lib.stream_ptr(t.device))
        _TWIDDLES[key] = t
    return t


FUSED_MIN, FUSED_MAX = 1 << 12, 1 << 20     # transform lengths of the fused basis series


def fourstep_order(X, N, isw=None, out=None):
    """Rows of a half spectrum (rows, flen) complex64 in the four-step order of a length-N transform: P[j, k2 (N1/2) +
    k1] = X[j, N2 k1 + k2] (times isw), P[j, N/2] = X[j, N/2] (gwb_fourstep_order); the input layout of the fused
    basis series."""
    _lib.require_cuda(X)
    X2 = X if X.dim() == 2 else X[None]
    rows, flen = X2.shape
    if out is None:
        # rows padded to an even length: 16-byte aligned rows for the fused pass's asynchronous copies
        out = torch.empty((rows, N // 2 + 2), dtype=torch.complex64, device=X.device)[:, :N // 2 + 1]
    _lib.call('gwb_fourstep_order', _lib.ptr(X2), _lib.row_stride(X2), rows, _lib.ptr(isw), flen, int(N),
              _lib.ptr(out), _lib.row_stride(out), _lib.stream_ptr(X.device))
    return out if X.dim() == 2 else out[0]


RING_N = 1 << 20   # the transform length of the persistent ring form (gwb_basis_fused_ring)


class FusedBasisWorkspace:
    """Workspace of the fused basis series: the intermediate W, the twiddle table, the scale partials and ticket.
    ring (tlen = 2^20 only; the default there): one persistent launch with W in a ring of gwb_basis_ring_rows() rows
    kept in L2; else two passes with W of wrows x tlen complex (the rows go through it in batches of wrows)."""

    def __init__(self, tlen, flen, rows, device='cuda', wrows=None, ring=None):
        assert FUSED_MIN <= tlen <= FUSED_MAX and flen <= tlen // 2 + 1
        self.tlen, self.flen, self.rows = tlen, flen, rows
        self.ring = (tlen == RING_N) if ring is None else bool(ring)
        assert not self.ring or tlen == RING_N, 'the ring form is for tlen = 2^20'
        self.wrows = rows if wrows is None else max(1, min(int(wrows), rows))
        lib = _lib.load()
        wr = lib.gwb_basis_ring_rows() if self.ring else self.wrows
        self.W = torch.empty((wr, tlen), dtype=torch.complex64, device=device)
        self.sync = (torch.zeros(lib.gwb_basis_ring_sync_ints(rows), dtype=torch.int32, device=device)
                     if self.ring else None)
        self.tw = twiddles(tlen, device)
        self.partials = torch.empty(RB * max(1, tlen // 64), dtype=torch.float64, device=device)
        self.ticket = torch.zeros(1, dtype=torch.int32, device=device)
        self.scale = torch.empty(1, dtype=torch.float32, device=device)
        # fp8 form: one scale per basis row, and the per-row |q|^2 partial sums behind it (at most N2 per row)
        self.rowscale = torch.empty(rows, dtype=torch.float32, device=device)
        n2 = tlen >> ((tlen.bit_length() - 1 + 1) // 2)
        self.rowpart = torch.empty((rows if self.ring else self.wrows) * n2, dtype=torch.float32, device=device)


def basis_series_fused(ws, Vp, Dp, a0, Tn, Z, Zlo=None, form='f16', im_off=None):
    """Same Z as basis_series_into in two fused passes (gwb_basis_fused), from the basis filters Vp (r, tlen/2 + 1) and
    one segment's D isw Dp (tlen/2 + 1,), both in four-step order (fourstep_order). The scale is the whole-series rms
    of the first min(RB, wrows) rows by Parseval instead of the analysed-span rms (it cancels between Z and A).
    Returns the device scale; for form 'fp8' Z row j holds z_j / ws.rowscale[j] in e4m3 instead."""
    r = Vp.shape[0]
    assert r <= ws.rows and Vp.shape[1] >= ws.tlen // 2 + 1 and Dp.numel() >= ws.tlen // 2 + 1
    im_off = r if im_off is None else im_off
    if ws.ring:
        # one persistent launch, W in an L2-resident ring; the scale from the first two rows
        _lib.call('gwb_basis_fused_ring', _lib.ptr(Vp), Vp.stride(0), r, _lib.ptr(Dp), ws.tlen, _lib.ptr(ws.tw),
                  _lib.ptr(ws.W), ws.W.shape[0], int(a0), int(Tn), FORMS[form], _lib.ptr(Z), _lib.ptr(Zlo), Z.stride(0), int(im_off),
                  0, _lib.ptr(ws.partials), ws.partials.numel(), _lib.ptr(ws.scale), _lib.ptr(ws.rowscale),
                  _lib.ptr(ws.rowpart), ws.rowpart.numel(), _lib.ptr(ws.sync), ws.sync.numel(), _lib.stream_ptr())
        return ws.scale
    _lib.call('gwb_basis_fused', _lib.ptr(Vp), Vp.stride(0), r, _lib.ptr(Dp), ws.tlen, _lib.ptr(ws.tw),
              _lib.ptr(ws.W), ws.wrows, int(a0), int(Tn), FORMS[form], _lib.ptr(Z), _lib.ptr(Zlo), Z.stride(0),
              int(im_off), 0, min(RB, r), _lib.ptr(ws.partials), ws.partials.numel(), _lib.ptr(ws.ticket),
              _lib.ptr(ws.scale), _lib.ptr(ws.rowscale), _lib.ptr(ws.rowpart), ws.rowpart.numel(),
              _lib.stream_ptr())
    return ws.scale


class BasisWorkspace:
    """Device buffers of the basis series for one (tlen, batch) shape: the zero-padded transform input q, the
    transform output, the scale reduction's partials and ticket. q's upper half is zeroed once and never written."""

    def __init__(self, tlen, flen, rows=RB, device='cuda', npartials=1024):
        self.tlen, self.flen, self.rows = tlen, flen, rows
        self.q = torch.zeros((rows, tlen), dtype=torch.complex64, device=device)
        self.zb = torch.empty((rows, tlen), dtype=torch.complex64, device=device)
        self.partials = torch.empty(npartials, dtype=torch.float64, device=device)
        self.ticket = torch.zeros(1, dtype=torch.int32, device=device)
        self.scale = torch.empty(1, dtype=torch.float32, device=device)
        self.ones = torch.ones(flen, dtype=torch.float32, device=device)


def kh_of(r, form='f16'):
    """Half width of the compact operands: r rounded up to the MMA's K step (16; 32 for fp8)."""
    k = 32 if form == 'fp8' else 16
    return ((r + k - 1) // k) * k


def basis_series_into(ws, Vh, D, isw, a0, Tn, Z, Zlo=None, form='f16', im_off=None):
    """Z rows: real parts of the r basis series over [a0, a0+Tn) divided by the first batch's rms, then the imaginary
    parts from row im_off (r by default, the reference's layout; kh_of(r) for the compact one) (fp_filter.py:597-613),
    written into a preallocated Z (rows not written are left as they are). D: one segment's data (flen,) complex64;
    isw: 1/sw (or None when D is already divided by sw). Returns the device scale."""
    r, flen = Vh.shape
    im_off = r if im_off is None else im_off
    assert flen == ws.flen and Tn <= ws.tlen - a0
    f = FORMS[form]
    iw = ws.ones if isw is None else isw
    for c0 in range(0, r, ws.rows):
        nb = min(ws.rows, r - c0)
        _lib.call('gwb_basis_premul', _lib.ptr(Vh[c0:]), Vh.stride(0), nb, _lib.ptr(D), flen, 1, _lib.ptr(iw), flen,
                  _lib.ptr(ws.q), ws.q.stride(0), _s())
        _lib.call('gwb_fft_c2c', _lib.handle(), _lib.ptr(ws.q), _lib.ptr(ws.zb), ws.tlen, nb, ws.tlen, ws.tlen, 1, _s())
        if c0 == 0:
            _lib.call('gwb_basis_scale', _lib.ptr(ws.zb), ws.tlen, nb, int(a0), int(Tn), _lib.ptr(ws.partials),
                      ws.partials.numel(), _lib.ptr(ws.ticket), _lib.ptr(ws.scale), _s())
        _lib.call('gwb_basis_pack', _lib.ptr(ws.zb), ws.tlen, nb, im_off, c0, int(a0), int(Tn), _lib.ptr(ws.scale), f,
                  _lib.ptr(Z), _lib.ptr(Zlo), Z.stride(0), _s())
    return ws.scale


def _z_dtype(form):
    return {'f16': torch.float16, 'f32': torch.float32, 'bf16x3': torch.bfloat16, 'bf16': torch.bfloat16,
            'fp8': torch.uint8, 'f16x2': torch.float16}[form]


def stacked_A_into(A, nrm, scale, Kp, Are, Aim, Are_lo=None, Aim_lo=None, form='f16', df4=0.0, kh=0):
    """As = A (norm scale); Are = [Re As, -Im As], Aim = [Im As, Re As], zero-padded to Kp (fp_filter.py:615-621), or
    with kh > 0 the compact Are = [Re As | Im As] (Kp = 2 kh, Aim unused). nrm: float64 CUDA vector (a strided view is
    fine), the norms, or sigma^2 when df4 = 4 df is given; scale: device float32 scalar."""
    n, r = A.shape
    _lib.call('gwb_stacked_a', _lib.ptr(A), A.stride(0), n, r, _lib.ptr(nrm), nrm.stride(0), float(df4),
              _lib.ptr(scale), Kp, int(kh),
              A_FORMS[form], _lib.ptr(Are), _lib.ptr(Aim), _lib.ptr(Are_lo), _lib.ptr(Aim_lo), Are.stride(0), _s())


def stacked_A8_into(A, nrm, zscale, kh, A8, sa, df4):
    """fp8 screening form of the compact A: A8 row i = e4m3([Re As' | Im As'] / sa[i]) with As'_ij = A_ij norm_i
    zscale[j] (gwb_stacked_a8); sa (n,) float32 receives the row scales."""
    n, r = A.shape
    _lib.call('gwb_stacked_a8', _lib.ptr(A), A.stride(0), n, r, _lib.ptr(nrm), nrm.stride(0), float(df4),
              _lib.ptr(zscale), int(kh), _lib.ptr(A8), A8.stride(0), _lib.ptr(sa), _s())


def make_closures(kmin, flen, tlen, sw, eps_b, dev='cuda', form='f16'):
    """The reference's closures over (kmin, flen, tlen, sw, eps_b, RB, qz, dev) (fp_filter.py:576-621): returns an
    object with svd_tile(H), basis_series(Vh, Dws, a0, Tn) and stacked_A(A, nrm_s, scale, Kp), same arguments and
    results as the reference (CUDA tensors; scale a Python float, as the reference returns)."""
    ws = BasisWorkspace(tlen, flen, RB, dev)

    def _svd_tile(H):
        return svd_tile(H, sw, kmin, eps_b)

    def _basis_series(Vh, Dws, a0, Tn):
        r = Vh.shape[0]
        Kp = kp_of(r)
        Z = torch.zeros((Kp, Tn), dtype=_z_dtype(form), device=Dws.device)
        Zlo = torch.zeros_like(Z) if form == 'bf16x3' else None
        sc = basis_series_into(ws, Vh, Dws.contiguous(), None, a0, Tn, Z, Zlo, form)
        scale = float(sc.item())
        return (Z, scale) if Zlo is None else ((Z, Zlo), scale)

    def _stacked_A(A, nrm_s, scale, Kp):
        n = A.shape[0]
        dt = _z_dtype(form)
        Are = torch.empty((n, Kp), dtype=dt, device=A.device)
        Aim = torch.empty_like(Are)
        lo = (torch.empty_like(Are), torch.empty_like(Are)) if form == 'bf16x3' else (None, None)
        sc = torch.tensor([scale], dtype=torch.float32, device=A.device)
        nrm = torch.as_tensor(nrm_s, device=A.device).to(torch.float64)
        stacked_A_into(A.contiguous(), nrm, sc, Kp, Are, Aim, lo[0], lo[1], form)
        return (Are, Aim) if form != 'bf16x3' else ((Are, lo[0]), (Aim, lo[1]))

    return SimpleNamespace(svd_tile=_svd_tile, basis_series=_basis_series, stacked_A=_stacked_A, ws=ws)

