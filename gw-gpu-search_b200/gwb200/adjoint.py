"""Derivatives of the matched filter with respect to the template parameters (the differentiation form): SNR,
chi-squared and newSNR of a TaylorF2 template against each trigger's data, their gradients with respect to
(Mc, q, chi1z, chi2z, e0, t_c, phi_c), the phase metric of the match, and a damped Newton ascent that refines
triggers. The reference has no gradients (its template placement maximises the match numerically,
ecc_bank_place.py:79-89); everything here runs in the library's CUDA kernels (csrc/adjoint.cu).

Conventions: params (n, 7) float64 CUDA tensor, rows (Mc [M_sun], q = m2/m1 <= 1, chi1z, chi2z, e0 at f_ecc, t_c [s],
phi_c). D (n, flen) complex64 over-whitened data (stilde / PSD, as the pipeline's D), IP (n, flen) or (flen,) float32
inverse PSD. The template is the bank's TaylorF2 (templates.generate) with h -> h exp(-i (2 pi f t_c - phi_c)).
"""
import torch

from . import _lib

NPARAM = 7
NAMES = ('Mc', 'q', 'chi1z', 'chi2z', 'e0', 't_c', 'phi_c')
_NOUT = 7 + 3 * NPARAM


def _ip2(IP):
    return (IP, 0) if IP.dim() == 1 else (IP, IP.stride(0))


def snr_grad(params, D, IP, df, kmin, nbins=16, f_ecc=10.0, fp64=False, out=None):
    """SNR, newSNR and chi-squared of each trigger and their gradients. Returns a dict of CUDA tensors: snr, newsnr,
    chisq, sigma2 (n,), z (n,) complex128, kmax (n,) and dsnr, dnewsnr, dchisq (n, 7). fp64 selects float64 sums
    (float32 otherwise; the phase and its derivatives are float64 in both)."""
    _lib.require_cuda(params, D, IP)
    n, flen = D.shape
    assert params.shape == (n, NPARAM) and params.dtype == torch.float64 and params.is_contiguous()
    if out is None:
        out = torch.empty((n, _NOUT), dtype=torch.float64, device=D.device)
    ip, ldip = _ip2(IP)
    _lib.call('gwb_snr_grad', _lib.ptr(params), n, _lib.ptr(D), D.stride(0), _lib.ptr(ip), ldip, flen, float(df),
              int(kmin), float(f_ecc), int(nbins), 1 if fp64 else 0, _lib.ptr(out), out.stride(0), _lib.stream_ptr())
    return dict(snr=out[:, 0], newsnr=out[:, 1], chisq=out[:, 2], sigma2=out[:, 3],
                z=torch.complex(out[:, 4], out[:, 5]), kmax=out[:, 6], dsnr=out[:, 7:14], dnewsnr=out[:, 14:21],
                dchisq=out[:, 21:28], raw=out)


class _Stat(torch.autograd.Function):
    """SNR, newSNR or chi-squared of each trigger as a function of params, with the hand-written gradient of
    gwb_snr_grad as its backward (first order only)."""

    @staticmethod
    def forward(ctx, params, D, IP, df, kmin, nbins, f_ecc, fp64, which):
        r = snr_grad(params.detach().contiguous(), D, IP, df, kmin, nbins, f_ecc, fp64)
        ctx.save_for_backward(r['d' + which].clone())
        return r[which].clone()

    @staticmethod
    @torch.autograd.function.once_differentiable
    def backward(ctx, g):
        (d,) = ctx.saved_tensors
        return (g[:, None] * d,) + (None,) * 8


def stat(params, D, IP, df, kmin, nbins=16, f_ecc=10.0, fp64=False, which='snr'):
    """Differentiable (torch.autograd) SNR ('snr'), newSNR ('newsnr') or chi-squared ('chisq') of each trigger,
    (n,) float64; params (n, 7) float64 may require grad."""
    assert which in ('snr', 'newsnr', 'chisq')
    return _Stat.apply(params, D, IP, df, kmin, nbins, f_ecc, fp64, which)


def phase_metric(params, IP, flen, df, kmin, f_ecc=10.0):
    """(n, 7, 7) float64: g_ij = Cov_w(dPhi/dtheta_i, dPhi/dtheta_j), w = |h|^2 IP, so that the phase-maximised match
    of h(theta) and h(theta + d) is 1 - d^T g d / 2 to second order (the phi_c row is zero; project t_c out for the
    time-maximised match)."""
    _lib.require_cuda(params, IP)
    n = params.shape[0]
    g = torch.empty((n, NPARAM, NPARAM), dtype=torch.float64, device=params.device)
    ip, ldip = _ip2(IP)
    _lib.call('gwb_phase_metric', _lib.ptr(params), n, _lib.ptr(ip), ldip, int(flen), float(df), int(kmin),
              float(f_ecc), _lib.ptr(g), _lib.stream_ptr())
    return g


def refine(params, D, IP, df, kmin, steps=20, nbins=16, f_ecc=10.0, fp64=False, lam0=1.0):
    """Gradient ascent of each trigger's SNR over (Mc, q, chi1z, chi2z, e0, t_c): `steps` Levenberg-Marquardt steps
    with the phase metric as the curvature (gwb_refine_step). A step that raises a trigger's SNR is kept and its damping
    divided by 3 (down to 1e-4); one that does not is dropped and the damping multiplied by 10. Returns (params,
    history) with history (steps + 1, n) of SNRs."""
    n, flen = D.shape
    th = params.clone()
    lam = torch.full((n,), float(lam0), dtype=torch.float64, device=params.device)
    res = snr_grad(th, D, IP, df, kmin, nbins, f_ecc, fp64)['raw'].clone()
    hist = [res[:, 0].clone()]
    trial = torch.empty_like(th)
    for _ in range(steps):
        g = phase_metric(th, IP, flen, df, kmin, f_ecc)
        _lib.call('gwb_refine_step', _lib.ptr(th), _lib.ptr(res), res.stride(0), _lib.ptr(g), _lib.ptr(lam), n,
                  _lib.ptr(trial), _lib.stream_ptr())
        new = snr_grad(trial, D, IP, df, kmin, nbins, f_ecc, fp64)['raw']
        up = new[:, 0] > res[:, 0]
        th = torch.where(up[:, None], trial, th)
        res = torch.where(up[:, None], new, res)
        lam = torch.where(up, torch.clamp(lam * 0.3, min=1e-4), lam * 10.0)
        hist.append(res[:, 0].clone())
    return th, torch.stack(hist)
