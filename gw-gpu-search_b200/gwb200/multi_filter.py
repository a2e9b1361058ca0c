"""Chi-squared bin edges: drop-in for multi_filter.edges_per_template (pipeline/multi_filter.py:264-282).

Equal-power edges from each template's float64 cumulative |h|^2 / psd: the first k whose normalised cumulative sum
exceeds j / nb, clipped to [kmin, k1], padded with k1. The comparison keeps the reference's row offset (its rows are
flattened into one searchsorted), so rounding at near-ties follows it; the sums run in csrc/chisq.cu."""
import numpy as np
import torch

from . import _exact, _lib


def _edges(rows, nb_, kmin, k1, Hd, ips, offset_mode):
    _lib.require_cuda(Hd)
    rows = np.asarray(rows)
    nb_ = np.asarray(nb_)
    k1 = np.asarray(k1)
    ur, first, inv = np.unique(rows, return_index=True, return_inverse=True)
    B = int(nb_.max())
    units = np.zeros(len(ur), _exact.UNIT)
    units['row'] = ur
    n = int(ur.max()) + 1
    nb_rows = np.zeros(n, np.int32)
    nb_rows[ur] = nb_[first]
    k1_rows = np.zeros(n, np.int32)
    k1_rows[ur] = k1[first]
    ip = torch.as_tensor(ips, device=Hd.device).to(torch.float32).reshape(1, -1).contiguous()
    E = _exact.run_edges(units, Hd, ip, torch.from_numpy(nb_rows).to(Hd.device),
                         torch.from_numpy(k1_rows).to(Hd.device), kmin, B, offset_mode)
    return E.cpu().numpy().astype(np.int64)[inv]


def edges_per_template(xp, rows, nb_, kmin, k1, Hd, ips):
    """rows: per-peak row index into Hd (CUDA complex64); nb_, k1 per peak; ips 1/psd. Returns int64 (npk, B + 1)."""
    E = _edges(rows, nb_, kmin, k1, Hd, ips, 1)
    j = np.arange(E.shape[1] - 1)[None, :]
    nb_ = np.asarray(nb_)
    E[:, :-1] = np.where(j < nb_[:, None], E[:, :-1], np.asarray(k1)[:, None])
    return E
