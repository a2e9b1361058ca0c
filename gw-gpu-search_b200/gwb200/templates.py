"""TaylorF2 template bank on the device (the synthetic bank of the configurations).

The reference makes IMRPhenomD / SEOBNRv5EHM templates with PyCBC and pyseobnr (pipeline/imr_interp.py,
pipeline/ecc_templates.py); neither exists here, so the bank is stationary-phase TaylorF2 to 3.5PN with aligned-spin
terms to 2PN and the leading eccentric term, evaluated straight into the filter's frequency layout by
gwb_taylorf2 (csrc/bank.cu). Templates are ordered by Newtonian chirp time and cut into tiles, as fp_filter.py does
(:419-420, :448)."""
import numpy as np
import torch

from . import _lib

MTSUN_SI = 4.925490947641267e-06


def f_isco(m1, m2):
    return 1.0 / (6.0 ** 1.5 * np.pi * (np.asarray(m1) + np.asarray(m2)) * MTSUN_SI)


def tau0(m1, m2, f_low=20.0):
    m1, m2 = np.asarray(m1, np.float64), np.asarray(m2, np.float64)
    M = (m1 + m2) * MTSUN_SI
    eta = m1 * m2 / (m1 + m2) ** 2
    return 5.0 / (256.0 * np.pi * f_low * eta) * (np.pi * M * f_low) ** (-5.0 / 3.0)


def kend(m1, m2, df, flen):
    """Exclusive end bin of each template: the last bin at or below f_ISCO, plus one, capped at flen - 1 (the
    reference's kend never includes the Nyquist bin, fp_filter.py:520)."""
    return np.minimum(np.floor(f_isco(m1, m2) / df).astype(np.int64) + 1, flen - 1).astype(np.int32)


def generate(bank, rows, flen, df, f_low=20.0, f_ecc=10.0, out=None, device='cuda'):
    """Templates for bank rows `rows` (bank: dict of mass1, mass2, spin1z, spin2z, ecc arrays) as a complex64
    (len(rows), flen) CUDA tensor (or into `out`), and their kmax (int32 numpy)."""
    rows = np.asarray(rows)
    n = len(rows)
    kmin = int(f_low / df)
    col = lambda k: torch.from_numpy(np.ascontiguousarray(np.asarray(bank[k], np.float64)[rows])).to(device)
    m1, m2 = np.asarray(bank['mass1'])[rows], np.asarray(bank['mass2'])[rows]
    km = kend(m1, m2, df, flen)
    H = out if out is not None else torch.empty((n, flen), dtype=torch.complex64, device=device)
    km_d = torch.from_numpy(km).to(device)
    a = [col(k) for k in ('mass1', 'mass2', 'spin1z', 'spin2z', 'ecc')]
    _lib.call('gwb_taylorf2', *[_lib.ptr(t) for t in a], _lib.ptr(km_d), n, float(df), kmin, flen, float(f_ecc),
              _lib.ptr(H), H.stride(0), _lib.stream_ptr())
    return H, km


def tiles(bank, tile, f_low=20.0):
    """Bank rows sorted by chirp time (stable), cut into tiles of `tile` (fp_filter.py:419-420, 448)."""
    order = np.argsort(tau0(bank['mass1'], bank['mass2'], f_low), kind='stable')
    return [order[b0:b0 + tile] for b0 in range(0, len(order), tile)]
