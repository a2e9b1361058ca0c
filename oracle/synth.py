"""Seeded synthetic inputs for the configurations (test infrastructure only): analytic PSD, coloured Gaussian noise,
TaylorF2 templates and injections, sine-Gaussian glitches.

The reference works on LIGO open data and PyCBC templates; there is no TaylorF2 code in it (only the SPAtmplt name in
its argv). These generators restate published formulas, named where they are used, so parity for the templates and
the PSD model is pinned by known-answer tests in tests/test_oracle_synth.py, not by the reference.

Units: strain is carried multiplied by DYN_RANGE_FAC (pipeline/gpu_prep.py:21), as the reference's conditioning does
before its float32 cast, so PSDs are in (DYN_RANGE_FAC x strain)^2 / Hz."""
import numpy as np

DYN_RANGE_FAC = 5.9029581035870565e+20
MTSUN_SI = 4.925490947641267e-06       # G M_sun / c^3 in seconds
EULER_GAMMA = 0.5772156649015329
F_CUT_LOW = 15.0                       # below this the PSD model is "very large"
LOW_WALL = 1e4                         # PSD below F_CUT_LOW = LOW_WALL x PSD(F_CUT_LOW)
LINES_C2 = ((60.0, 1e3, 0.02), (120.0, 1e3, 0.02), (180.0, 1e3, 0.02))   # (f0 Hz, height, half-width Hz)


def analytic_psd(f, lines=(), scaled=True):
    """S(f) = 1e-49 [x^-4.14 - 5 x^-2 + 111 (1 - x^2 + x^4/2) / (1 + x^2/2)], x = f / 215 Hz, for f >= 15 Hz; below,
    LOW_WALL x S(15 Hz). Narrow lines multiply by 1 + h / (1 + ((f - f0) / w)^2). scaled: times DYN_RANGE_FAC^2."""
    f = np.asarray(f, np.float64)
    fc = np.maximum(f, F_CUT_LOW)
    x = fc / 215.0
    s = 1e-49 * (x ** -4.14 - 5.0 * x ** -2 + 111.0 * (1.0 - x ** 2 + 0.5 * x ** 4) / (1.0 + 0.5 * x ** 2))
    s = np.where(f < F_CUT_LOW, LOW_WALL * s, s)
    for f0, h, w in lines:
        s = s * (1.0 + h / (1.0 + ((f - f0) / w) ** 2))
    return s * DYN_RANGE_FAC ** 2 if scaled else s


def coloured_noise(n, sr, rng, lines=()):
    """n samples at sr of Gaussian noise with one-sided PSD analytic_psd (scaled units), float64 spectrum."""
    w = rng.standard_normal(n)
    X = np.fft.rfft(w)
    f = np.arange(len(X)) * sr / n
    X *= np.sqrt(analytic_psd(f, lines) * sr / 2.0)
    X[0] = 0.0
    return X


def f_isco(m1, m2):
    return 1.0 / (6.0 ** 1.5 * np.pi * (m1 + m2) * MTSUN_SI)


def taylorf2_phase(f, m1, m2, chi1=0.0, chi2=0.0, e0=0.0, f_ecc=10.0):
    """Stationary-phase TaylorF2 phase Psi(f) (without the 2 pi f t_c - phi_c - pi/4 part), to 3.5PN in the
    non-spinning terms (Buonanno, Iyer, Ochsner, Pan & Sathyaprakash 2009, Eq. 3.18), with the aligned-spin
    spin-orbit term at 1.5PN (beta) and the leading spin1-spin2 term at 2PN (sigma), and the leading-order eccentric
    correction -2355/1462 e0^2 (v0/v)^(19/3) (Yunes & Arun 2009), e0 defined at f_ecc."""
    f = np.asarray(f, np.float64)
    M = m1 + m2
    eta = m1 * m2 / M ** 2
    Ms = M * MTSUN_SI
    v = np.cbrt(np.pi * Ms * f)
    d1, d2 = m1 / M, m2 / M
    beta = (113.0 / 12.0) * (d1 * d1 * chi1 + d2 * d2 * chi2) + 6.25 * eta * (chi1 + chi2)
    sigma = eta * (474.0 / 48.0) * chi1 * chi2
    pi = np.pi
    p2 = 20.0 / 9.0 * (743.0 / 336.0 + 11.0 / 4.0 * eta)
    p3 = -16.0 * pi + 4.0 * beta
    p4 = 10.0 * (3058673.0 / 7257600.0 + 5429.0 / 1008.0 * eta + 617.0 / 144.0 * eta ** 2) - 10.0 * sigma
    v_isco = 1.0 / np.sqrt(6.0)
    p5 = pi * (38645.0 / 756.0 - 65.0 / 9.0 * eta) * (1.0 + 3.0 * np.log(v / v_isco))
    p6 = (11583231236531.0 / 4694215680.0 - 640.0 / 3.0 * pi ** 2 - 6848.0 / 21.0 * EULER_GAMMA
          + eta * (-15737765635.0 / 3048192.0 + 2255.0 / 12.0 * pi ** 2) + 76055.0 / 1728.0 * eta ** 2
          - 127825.0 / 1296.0 * eta ** 3 - 6848.0 / 21.0 * np.log(4.0 * v))
    p7 = pi * (77096675.0 / 254016.0 + 378515.0 / 1512.0 * eta - 74045.0 / 756.0 * eta ** 2)
    series = 1.0 + v * v * (p2 + v * (p3 + v * (p4 + v * (p5 + v * (p6 + v * p7)))))
    if e0:
        v0 = np.cbrt(pi * Ms * f_ecc)
        series = series - 2355.0 / 1462.0 * e0 ** 2 * (v0 / v) ** (19.0 / 3.0)
    return 3.0 / (128.0 * eta * v ** 5) * series


def taylorf2(flen, df, m1, m2, chi1=0.0, chi2=0.0, e0=0.0, f_low=20.0, t0=0.0, amp=1.0):
    """complex128 (flen,) template amp f^-7/6 exp(-i (Psi(f) - pi/4)) exp(-2 pi i f t0) on k df for f_low <= f <= f_ISCO,
    zero elsewhere (t0 shifts the merger to sample time t0 seconds)."""
    k = np.arange(flen)
    f = k * df
    on = (f >= f_low) & (f <= f_isco(m1, m2))
    h = np.zeros(flen, np.complex128)
    fo = f[on]
    psi = taylorf2_phase(fo, m1, m2, chi1, chi2, e0) - np.pi / 4
    h[on] = amp * fo ** (-7.0 / 6.0) * np.exp(-1j * psi) * np.exp(-2j * np.pi * fo * t0)
    return h


def optimal_snr(h, psd, df, kmin=0):
    return float(np.sqrt(4.0 * df * np.sum(np.abs(h[kmin:]) ** 2 / psd[kmin:])))


def sine_gaussian(n, sr, t_c, f0, q, amp=1.0):
    """Time-domain sine-Gaussian: amp exp(-(t - t_c)^2 / tau^2) sin(2 pi f0 (t - t_c)), tau = Q / (sqrt(2) pi f0)."""
    t = np.arange(n) / sr - t_c
    tau = q / (np.sqrt(2.0) * np.pi * f0)
    return amp * np.exp(-(t / tau) ** 2) * np.sin(2 * np.pi * f0 * t)


def random_bank_c1(n=64, seed=0):
    """C1 bank: n non-spinning templates, m1 and m2 uniform in 5-50 M_sun."""
    rng = np.random.default_rng(seed)
    m = rng.uniform(5.0, 50.0, (n, 2))
    m1, m2 = m.max(1), m.min(1)
    z = np.zeros(n)
    return dict(mass1=m1, mass2=m2, spin1z=z, spin2z=z.copy(), ecc=z.copy())


def random_bank_c2(n_aligned=4612, n_ecc=1268, seed=0):
    """C2 bank: aligned-spin TaylorF2 (component masses 3-100, chi_z in [-0.9, 0.9]) plus eccentric templates (total
    mass 45-100, equal-ish mass ratio, e0 in [0, 0.3] at 10 Hz, non-spinning)."""
    rng = np.random.default_rng(seed)
    m = rng.uniform(3.0, 100.0, (n_aligned, 2))
    m1, m2 = m.max(1), m.min(1)
    s1, s2 = rng.uniform(-0.9, 0.9, n_aligned), rng.uniform(-0.9, 0.9, n_aligned)
    mt = rng.uniform(45.0, 100.0, n_ecc)
    q = rng.uniform(1.0, 3.0, n_ecc)
    em1, em2 = mt * q / (1 + q), mt / (1 + q)
    e0 = rng.uniform(0.0, 0.3, n_ecc)
    return dict(mass1=np.r_[m1, em1], mass2=np.r_[m2, em2], spin1z=np.r_[s1, np.zeros(n_ecc)],
                spin2z=np.r_[s2, np.zeros(n_ecc)], ecc=np.r_[np.zeros(n_aligned), e0])


def tau0(m1, m2, f_low=20.0):
    """Newtonian chirp time (s), used to sort templates into tiles (pipeline/fp_filter.py:419-420)."""
    M = (m1 + m2) * MTSUN_SI
    eta = m1 * m2 / (m1 + m2) ** 2
    return 5.0 / (256.0 * np.pi * f_low * eta) * (np.pi * M * f_low) ** (-5.0 / 3.0)
