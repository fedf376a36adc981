"""Seeded synthetic connectomes standing in for the reference's packaged
connectomes (not available offline)."""
import numpy as np


def connectome(n, density, lo, hi, seed):
    """Symmetric lognormal(0, 1) weights on a random upper-triangle mask of the
    given density, normalised to max 1 with a zero diagonal, and symmetric
    uniform [lo, hi) tract lengths with a zero diagonal.  Returns (weights,
    tract_lengths) as float64 (n, n) arrays."""
    rng = np.random.default_rng(seed)
    w = rng.lognormal(0.0, 1.0, (n, n))
    mask = np.triu(rng.random((n, n)) < density, 1)
    w = np.triu(w * mask, 1)
    w = w + w.T
    w /= w.max()
    lengths = np.triu(rng.uniform(lo, hi, (n, n)), 1)
    lengths = lengths + lengths.T
    return w, lengths
