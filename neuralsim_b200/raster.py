"""Raster utilities: per-neuron spike steps of a raster and nearest
matching of two rasters (spike-time error of one run against another)."""
import numpy as np


def spike_times(idx, off):
    """Per-neuron spike steps from a raster (idx, per-step offsets)."""
    off = np.asarray(off, np.int64)
    steps = np.repeat(np.arange(len(off) - 1), np.diff(off))
    order = np.lexsort((steps, np.asarray(idx, np.int64)))
    return np.asarray(idx, np.int64)[order], steps[order]


def match_spikes(a, b, window):
    """Matches spikes of raster b to raster a per neuron, nearest within
    `window` steps (each spike used once, in time order). Returns
    (abs step differences of matched pairs, unmatched in a, unmatched in b)."""
    ia, ta = spike_times(*a)
    ib, tb = spike_times(*b)
    diffs, ua, ub = [], 0, 0
    na = np.searchsorted(ia, np.arange(max(ia.max(initial=-1), ib.max(initial=-1)) + 2))
    nb = np.searchsorted(ib, np.arange(len(na)))
    for i in range(len(na) - 1):
        x, y = ta[na[i]:na[i + 1]], tb[nb[i]:nb[i + 1]]
        p = q = 0
        while p < len(x) and q < len(y):
            d = y[q] - x[p]
            if abs(d) <= window:
                diffs.append(abs(d)); p += 1; q += 1
            elif d < 0:
                ub += 1; q += 1
            else:
                ua += 1; p += 1
        ua += len(x) - p
        ub += len(y) - q
    return np.asarray(diffs, np.int64), ua, ub
