"""The differentiation form (gwb200.adjoint): SNR / chi-squared / newSNR of TaylorF2 templates against 16 s data
stretches and their gradients, against the float64 numpy oracle (values and central finite differences), a plain
PyTorch float64 autograd reference, the float32 form, the phase metric's second-order match, and the ascent."""
import numpy as np
import pytest
import torch

from oracle import adjoint as oa
from oracle import synth

pytestmark = pytest.mark.gpu

SR, TLEN = 2048.0, 1 << 15          # 16 s stretches
FLEN = TLEN // 2 + 1
DF = SR / TLEN
KMIN = int(20.0 / DF)
NB = 16
# (Mc, q, chi1z, chi2z, e0, t_c, phi_c): aligned-spin and eccentric triggers
THETA = np.array([[12.0, 0.7, 0.3, -0.2, 0.0, 0.01, 0.4],
                  [25.0, 0.45, -0.6, 0.5, 0.0, -0.02, 1.1],
                  [6.5, 0.9, 0.1, 0.0, 0.0, 0.0, 2.0],
                  [30.0, 0.85, 0.0, 0.0, 0.2, 0.005, 0.3],
                  [38.0, 0.95, 0.0, 0.0, 0.12, -0.01, 2.7]])


def _data(theta_true, snr=15.0, seed=0, noise=True):
    rng = np.random.default_rng(seed)
    f = np.arange(FLEN) * DF
    psd = synth.analytic_psd(f)
    IP = np.zeros((len(theta_true), FLEN), np.float32)
    IP[:, KMIN:] = 1.0 / psd[KMIN:]
    D = np.zeros((len(theta_true), FLEN), np.complex64)
    for i, th in enumerate(theta_true):
        h, _ = oa.template(th, FLEN, DF, KMIN)
        a = snr / np.sqrt(4 * DF * np.sum(np.abs(h) ** 2 / psd))
        s = a * h
        if noise:
            sd = np.sqrt(psd / (4 * DF))
            s = s + sd * (rng.standard_normal(FLEN) + 1j * rng.standard_normal(FLEN))
        D[i] = (s * IP[i]).astype(np.complex64)
    return D, IP


def _gpu(*a):
    return [torch.from_numpy(np.ascontiguousarray(x)).cuda() for x in a]


def test_values_and_finite_differences():
    from gwb200 import adjoint
    D, IP = _data(THETA)
    th = THETA + np.array([0.01, 0.01, 0.02, -0.02, 0.01, 1e-4, 0.1])
    Dd, IPd, thd = _gpu(D, IP, th)
    r = adjoint.snr_grad(thd, Dd, IPd, DF, KMIN, NB, fp64=True)
    for i in range(len(th)):
        snr, chisq, ns = oa.snr_chisq(th[i], D[i], IP[i], DF, KMIN, NB)
        assert abs(r['snr'][i].item() - snr) <= 1e-8 * snr
        assert abs(r['chisq'][i].item() - chisq) <= 1e-7 * max(chisq, 1.0)
        assert abs(r['newsnr'][i].item() - ns) <= 1e-8 * ns
        fd = oa.fd_grad(th[i], D[i], IP[i], DF, KMIN, NB)
        for name, row in (('dsnr', 0), ('dchisq', 1), ('dnewsnr', 2)):
            got = r[name][i].cpu().numpy()
            ref = fd[row]
            scale = np.abs(ref).max()
            assert np.all(np.abs(got - ref) <= 2e-5 * np.abs(ref) + 1e-7 * scale), (i, name, got, ref)


def _torch_reference(th, D, IP, edges):
    """Plain PyTorch float64: the same snr / chisq / newsnr with autograd through the TaylorF2 phase."""
    th = torch.tensor(th, dtype=torch.float64, requires_grad=True)
    mc, q, c1, c2, e0, tc, phic = th
    eta = q / (1 + q) ** 2
    M = mc * eta ** -0.6
    m1, m2 = M / (1 + q), q * M / (1 + q)
    d1, d2 = m1 / M, m2 / M
    k1 = int(edges[-1])
    f = torch.arange(KMIN, k1, dtype=torch.float64) * DF
    Ms = M * synth.MTSUN_SI
    v = (np.pi * Ms * f) ** (1.0 / 3.0)
    pi = np.pi
    beta = 113.0 / 12.0 * (d1 * d1 * c1 + d2 * d2 * c2) + 6.25 * eta * (c1 + c2)
    sigma = eta * 474.0 / 48.0 * c1 * c2
    p2 = 20.0 / 9.0 * (743.0 / 336.0 + 11.0 / 4.0 * eta)
    p3 = -16.0 * pi + 4.0 * beta
    p4 = 10.0 * (3058673.0 / 7257600.0 + 5429.0 / 1008.0 * eta + 617.0 / 144.0 * eta ** 2) - 10.0 * sigma
    p5 = pi * (38645.0 / 756.0 - 65.0 / 9.0 * eta) * (1.0 + 3.0 * torch.log(v * np.sqrt(6.0)))
    p6 = (11583231236531.0 / 4694215680.0 - 640.0 / 3.0 * pi ** 2 - 6848.0 / 21.0 * synth.EULER_GAMMA
          + eta * (-15737765635.0 / 3048192.0 + 2255.0 / 12.0 * pi ** 2) + 76055.0 / 1728.0 * eta ** 2
          - 127825.0 / 1296.0 * eta ** 3 - 6848.0 / 21.0 * torch.log(4.0 * v))
    p7 = pi * (77096675.0 / 254016.0 + 378515.0 / 1512.0 * eta - 74045.0 / 756.0 * eta ** 2)
    series = 1.0 + v * v * (p2 + v * (p3 + v * (p4 + v * (p5 + v * (p6 + v * p7)))))
    v0 = (pi * Ms * 10.0) ** (1.0 / 3.0)
    series = series - 2355.0 / 1462.0 * e0 ** 2 * (v0 / v) ** (19.0 / 3.0)
    ph = 3.0 / (128.0 * eta * v ** 5) * series - pi / 4 + 2 * pi * f * tc - phic
    amp = f ** (-7.0 / 6.0)
    Dk = torch.from_numpy(D[KMIN:k1].astype(np.complex128))
    q_ = 4 * DF * amp * torch.exp(1j * ph) * Dk
    sig2 = 4 * DF * torch.sum(amp ** 2 * torch.from_numpy(IP[KMIN:k1].astype(np.float64)))
    zj = torch.stack([q_[int(edges[j]) - KMIN:int(edges[j + 1]) - KMIN].sum() for j in range(NB)])
    z = zj.sum()
    snr = torch.abs(z) / torch.sqrt(sig2)
    chisq = (NB * torch.sum(torch.abs(zj) ** 2) - torch.abs(z) ** 2) / sig2
    rc = chisq / (2 * NB - 2)
    ns = snr / ((1 + rc ** 3) / 2) ** (1.0 / 6.0) if rc.item() > 1 else snr
    out = []
    for y in (snr, chisq, ns):
        g, = torch.autograd.grad(y, th, retain_graph=True)
        out.append(g.numpy())
    return out


def test_against_torch_autograd():
    from gwb200 import adjoint
    D, IP = _data(THETA, seed=1)
    th = THETA + np.array([0.02, -0.01, 0.05, 0.03, 0.02, 2e-4, -0.3])
    Dd, IPd, thd = _gpu(D, IP, th)
    r = adjoint.snr_grad(thd, Dd, IPd, DF, KMIN, NB, fp64=True)
    for i in range(len(th)):
        k1 = oa.kmax(th[i][0], th[i][1], DF, FLEN)
        e = oa.edges(IP[i], DF, KMIN, k1, NB)
        ref = _torch_reference(th[i], D[i], IP[i], e)
        for name, g in zip(('dsnr', 'dchisq', 'dnewsnr'), ref):
            got = r[name][i].cpu().numpy()
            assert np.all(np.abs(got - g) <= 1e-8 * np.abs(g) + 1e-10 * np.abs(g).max()), (i, name, got, g)


def test_float32_form_against_float64():
    from gwb200 import adjoint
    D, IP = _data(THETA, seed=2)
    Dd, IPd, thd = _gpu(D, IP, THETA + 0.01 * np.array([1, 1, 1, 1, 1, 0.01, 1]))
    r64 = adjoint.snr_grad(thd, Dd, IPd, DF, KMIN, NB, fp64=True)
    r32 = adjoint.snr_grad(thd, Dd, IPd, DF, KMIN, NB, fp64=False)
    np.testing.assert_allclose(r32['snr'].cpu().numpy(), r64['snr'].cpu().numpy(), rtol=1e-4)
    for name in ('dsnr', 'dnewsnr'):
        a, b = r32[name].cpu().numpy(), r64[name].cpu().numpy()
        assert np.all(np.abs(a - b) <= 1e-3 * np.abs(b) + 1e-4 * np.abs(b).max(1, keepdims=True)), (name, a, b)


def test_phase_metric_predicts_the_match():
    from gwb200 import adjoint
    D, IP = _data(THETA, noise=False)           # D = a h(theta) IP: the SNR is proportional to the match
    Dd, IPd, thd = _gpu(D, IP, THETA)
    g = adjoint.phase_metric(thd, IPd, FLEN, DF, KMIN).cpu().numpy()
    assert np.allclose(g, np.transpose(g, (0, 2, 1)))
    assert np.all(g[:, 6, :] == 0) and np.all(g[:, :, 6] == 0)
    for gi in g:
        w = np.linalg.eigvalsh(gi)
        assert w.min() >= -1e-9 * w.max()
    r0 = adjoint.snr_grad(thd, Dd, IPd, DF, KMIN, NB, fp64=True)['snr'].cpu().numpy()
    rng = np.random.default_rng(5)
    for i in range(len(THETA)):
        for _ in range(3):
            d = rng.standard_normal(7) * np.array([1e-3, 1e-3, 1e-2, 1e-2, 1e-3, 1e-5, 0.0])
            if THETA[i, 4] == 0:
                d[4] = 0.0                       # e0 = 0 sits at the edge of its range
            # keep the total mass (and with it the ISCO cut-off bin) fixed: d ln Mc = 0.6 d ln eta
            q = THETA[i, 1]
            d[0] = THETA[i, 0] * 0.6 * (1 - q) / (q * (1 + q)) * d[1]
            d *= np.sqrt(2e-3 / (d @ g[i] @ d))  # a 1e-3 mismatch by the metric
            r1 = adjoint.snr_grad(torch.from_numpy((THETA[i] + d)[None]).cuda(), Dd[i:i + 1], IPd[i:i + 1], DF, KMIN,
                                  NB, fp64=True)['snr'].item()
            mism = 1 - r1 / r0[i]
            assert abs(mism - 1e-3) < 0.15e-3, (i, mism)


def test_refinement_climbs_to_the_signal():
    from gwb200 import adjoint
    D, IP = _data(THETA, snr=20.0, seed=3)
    start = THETA.copy()
    start[:, 0] *= 1.003
    start[:, 1] = np.clip(start[:, 1] - 0.03, 0.05, 1.0)
    start[:, 2] += 0.05
    start[:, 3] -= 0.05
    start[:, 5] += 2e-4
    Dd, IPd, thd = _gpu(D, IP, start)
    truth = adjoint.snr_grad(_gpu(THETA)[0], Dd, IPd, DF, KMIN, NB, fp64=True)['snr'].cpu().numpy()
    th, hist = adjoint.refine(thd, Dd, IPd, DF, KMIN, steps=20, nbins=NB, fp64=True)
    h = hist.cpu().numpy()
    assert np.all(np.diff(h, axis=0) >= -1e-12)                 # never worse
    assert np.all(h[-1] > h[0])
    # a local ascent: it reaches the maximum near the start (0.98 of the SNR at the true parameters, which the noise
    # need not make the global maximum)
    assert np.all(h[-1] >= 0.98 * truth), (h[0], h[-1], truth)


def test_autograd_function_carries_the_gradients():
    """adjoint.stat as a torch.autograd.Function: backward of a scalar loss gives the chain rule through the
    hand-written gradients, for snr, newsnr and chisq."""
    from gwb200 import adjoint
    D, IP = _data(THETA, seed=4)
    Dd, IPd, thd = _gpu(D, IP, THETA + 0.01)
    r = adjoint.snr_grad(thd, Dd, IPd, DF, KMIN, NB, fp64=True)
    for which in ('snr', 'newsnr', 'chisq'):
        th = thd.clone().requires_grad_(True)
        y = adjoint.stat(th, Dd, IPd, DF, KMIN, NB, fp64=True, which=which)
        assert torch.equal(y.detach(), r[which])
        (y ** 2).sum().backward()
        assert torch.allclose(th.grad, 2 * r[which][:, None] * r['d' + which], rtol=1e-14, atol=0)
