import numpy as np


def relerr(a, b):
    """max |a-b| / max |b|: norm-wise relative error of a field."""
    a = np.asarray(a, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    den = np.max(np.abs(b)) if b.size else 0.0
    return float(np.max(np.abs(a - b)) / (den if den > 0 else 1.0)) if b.size else 0.0
