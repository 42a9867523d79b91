import numpy as np


def max_rel_err(a, b):
    """Max |a - b| / |b| over all entries (FP64)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    den = np.maximum(np.abs(b), np.finfo(np.float64).tiny)
    return float(np.max(np.abs(a - b) / den)) if a.size else 0.0
