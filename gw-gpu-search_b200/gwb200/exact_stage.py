"""Exact complex SNR numerator z and chi-squared bin power at candidate peaks of one template tile: drop-in for
pipeline/exact_stage.py (ExactStage, TemplateTile, SegmentData, PeakRequest, PeakValues, compare_values).

The dense path (coarse=None, the reference's --templates pycbc mode) runs on the device: edges per distinct row
from the float64 cumulative |H|^2 IP (multi_filter's rule, exact_stage._dense_edges :261-266), then the binned sums
over the dense rows with q = conj(H) D formed in registers (exact_stage._dense_sums_cuda :734-739). Results come back
to the host in request order, as the reference returns them (:186-188). The regenerating path (coarse nodes,
:446-731) is not built: a tile with coarse nodes raises NotImplementedError."""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import torch

from . import _exact, _lib

R = 32
MAX_PEAKS = _exact.MAX_PEAKS
CHECK_TOL = dict(edge_bins=1, edge_frac=1e-2, snr_rel=1e-4, phase_rad=1e-4, chisq_rel=1e-3)   # exact_stage.py:35


@dataclass(frozen=True, eq=False)
class TemplateTile:
    """One tile: H (n, flen) complex64 CUDA tensor, nbins per row (0 = no chi-squared, one bin), bins cover
    [kmin, kmax[row]) (exact_stage.py:97-117)."""
    H: object
    nbins: np.ndarray
    kmin: int
    kmax: np.ndarray
    coarse: object = None

    def __post_init__(self):
        n = self.H.shape[0]
        object.__setattr__(self, 'nbins', np.asarray(self.nbins, np.int64))
        object.__setattr__(self, 'kmax', np.asarray(self.kmax, np.int64))
        assert self.H.dim() == 2 and self.H.dtype == torch.complex64 and self.H.is_contiguous()
        assert self.nbins.shape == (n,) and self.kmax.shape == (n,)


@dataclass(frozen=True, eq=False)
class SegmentData:
    """One segment: D (flen,) complex64, IP (flen,) float32, both zero below kmin; tlen a power of two
    (exact_stage.py:120-133)."""
    D: object
    IP: object
    df: float
    tlen: int

    def __post_init__(self):
        flen = self.tlen // 2 + 1
        assert self.tlen & (self.tlen - 1) == 0
        assert tuple(self.D.shape) == (flen,) and self.D.dtype == torch.complex64
        assert tuple(self.IP.shape) == (flen,) and self.IP.dtype == torch.float32


@dataclass(frozen=True, eq=False)
class PeakRequest:
    """Peaks of one (tile, segment): tile row and sample index; duplicates allowed, results keep this order."""
    rows: np.ndarray
    samples: np.ndarray

    def __post_init__(self):
        object.__setattr__(self, 'rows', np.asarray(self.rows, np.int64))
        object.__setattr__(self, 'samples', np.asarray(self.samples, np.int64))
        assert self.rows.ndim == 1 and self.rows.shape == self.samples.shape


@dataclass(frozen=True, eq=False)
class PeakValues:
    """Per requested peak, in request order: z (complex64), pw (float32), fpeak (Hz, float64)."""
    z: np.ndarray
    pw: np.ndarray
    fpeak: np.ndarray


class ExactStage:
    """Exact z, pw and fpeak at requested peaks of one tile, segment after segment (exact_stage.py:157-203)."""

    def __init__(self, tile: TemplateTile):
        if tile.coarse is not None:
            raise NotImplementedError('the regenerating exact stage (coarse nodes) is not built; pass coarse=None')
        _lib.require_cuda(tile.H)
        self.tile = tile
        self.check = None
        dev = tile.H.device
        self._nb_rows = torch.from_numpy(tile.nbins.astype(np.int32)).to(dev)
        self._kmax_rows = torch.from_numpy(tile.kmax.astype(np.int32)).to(dev)

    def _edges_dev(self, seg, rows_u):
        units = np.zeros(len(rows_u), _exact.UNIT)
        units['row'] = rows_u
        B = int(np.maximum(self.tile.nbins[rows_u], 1).max()) if len(rows_u) else 1
        ip = seg.IP.reshape(1, -1).contiguous()
        return _exact.run_edges(units, self.tile.H, ip, self._nb_rows, self._kmax_rows, self.tile.kmin, B, 1), B

    def edges(self, seg: SegmentData, rows: np.ndarray) -> np.ndarray:
        """(len(rows), B + 1) int64 edges, padded with kmax beyond each row's bin count (exact_stage.py:167-171)."""
        rows_u, inv = np.unique(np.asarray(rows, np.int64), return_inverse=True)
        E, _ = self._edges_dev(seg, rows_u)
        return E.cpu().numpy().astype(np.int64)[inv]

    def evaluate(self, seg: SegmentData, req: PeakRequest) -> PeakValues:
        _lib.require_cuda(seg.D, seg.IP)
        n = self.tile.H.shape[0]
        rows, samples = req.rows, req.samples
        assert len(rows) == 0 or (0 <= rows.min() and rows.max() < n and 0 <= samples.min() and samples.max() < seg.tlen)
        npk = len(rows)
        if npk == 0:
            return PeakValues(np.zeros(0, np.complex64), np.zeros(0, np.float32), np.zeros(0))
        order, rows_u, cands, groups, units = _exact.plan(rows, samples)
        E, B = self._edges_dev(seg, rows_u)
        flen = seg.D.shape[0]
        pk = _exact.run_sums(cands, groups, units, E, B, self._nb_rows, self.tile.H, seg.D, self.tile.kmin, flen,
                             seg.tlen)
        z = np.empty(npk, np.complex64)
        pw = np.empty(npk, np.float32)
        z[order] = pk['zr'] + 1j * pk['zi']
        pw[order] = pk['pw']
        Eh = E.cpu().numpy().astype(np.int64)
        u_req = np.empty(npk, np.int64)
        u_req[order] = cands['unit']
        return PeakValues(z, pw, _fpeak(Eh[u_req], self.tile.nbins[rows], seg.df))


def _fpeak(E, nb, df):
    """exact_stage.py:236-238."""
    r = np.arange(len(E))
    return (2 * E[r, np.maximum(nb - 1, 0)] - E[r, np.maximum(nb - 2, 0)]) * df


def compare_values(z, pw, z_ref, pw_ref, nbins) -> dict:
    """Relative |z| error, phase error and relative chi-squared error, max and p99 (exact_stage.py:299-311)."""
    z = np.asarray(z, np.complex128)
    z_ref = np.asarray(z_ref, np.complex128)
    snr = np.abs(np.abs(z) - np.abs(z_ref)) / np.abs(z_ref)
    ph = np.abs(np.angle(z * np.conj(z_ref)))
    nb = np.asarray(nbins)
    m = nb > 0
    q = nb[m] * np.asarray(pw, np.float64)[m] - np.abs(z[m]) ** 2
    q_ref = nb[m] * np.asarray(pw_ref, np.float64)[m] - np.abs(z_ref[m]) ** 2
    chi = np.abs(q - q_ref) / np.abs(q_ref) if m.any() else np.zeros(1)
    return dict(snr_rel_max=float(snr.max()), snr_rel_p99=float(np.percentile(snr, 99)),
                phase_max=float(ph.max()), phase_p99=float(np.percentile(ph, 99)),
                chisq_rel_max=float(chi.max()), chisq_rel_p99=float(np.percentile(chi, 99)))
