"""Chi-squared bin edges without a float64 cumulative sum per bin: drop-in for pipeline/chisq_edges.py
(edges_blocked :47-87, edges_fused :92-143). Both run the one fused edges kernel (csrc/chisq.cu), which compares
as these two reference functions do (cs > (j / nb) tot), computed once per distinct row."""
import numpy as np

from .multi_filter import _edges

BL = 256


def edges_blocked(xp, rows, nb_, kmin, k1, Hd, ips):
    """(npk, B + 1) int64 edges, padded with k1 beyond each peak's own bin count."""
    E = _edges(rows, nb_, kmin, k1, Hd, ips, 0)
    j = np.arange(E.shape[1] - 1)[None, :]
    nb_ = np.asarray(nb_)
    E[:, :-1] = np.where(j < nb_[:, None], E[:, :-1], np.asarray(k1)[:, None])
    return E


def edges_fused(xp, rows, nb_, kmin, k1, Hd, ips):
    """Same output as edges_blocked (the reference's fused kernel takes one peak per row; any rows work here)."""
    return edges_blocked(xp, rows, nb_, kmin, k1, Hd, ips)
