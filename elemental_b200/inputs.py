"""Seeded synthetic inputs with the shapes and distributions of the benchmark
configurations.  numpy's PCG64 generator (``numpy.random.default_rng(seed)``)
is the documented source of randomness; every matrix is float64 and
column-major (Fortran order), as Elemental's Matrix<F> stores it.

  spd_ggt(n, seed)          A = G G^T + n I,  G ~ N(0,1)       (Cholesky configs)
  uniform(m, n, seed)       A ~ U[-1, 1]                       (LU configs; the
                            reference's Uniform, core/random_impl.hpp:47-50)
  normal(m, n, seed)        B ~ N(0, 1)                        (right-hand sides)
  spd_spectrum(n, kappa, seed)   A = Q diag(s) Q^T, s log-spaced over [1, kappa],
                            Q the orthogonal factor of a seeded N(0,1) matrix
"""
from __future__ import annotations

import numpy as np


def rng(seed: int) -> np.random.Generator:
    return np.random.default_rng(seed)


def normal(m: int, n: int, seed: int) -> np.ndarray:
    return np.asfortranarray(rng(seed).standard_normal((m, n)))


def uniform(m: int, n: int, seed: int) -> np.ndarray:
    return np.asfortranarray(rng(seed).uniform(-1.0, 1.0, size=(m, n)))


def spd_ggt(n: int, seed: int) -> np.ndarray:
    g = rng(seed).standard_normal((n, n))
    a = g @ g.T
    a[np.diag_indices(n)] += n
    return np.asfortranarray(a)


def spd_spectrum(n: int, kappa: float, seed: int, device: str | None = None):
    """A = Q diag(s) Q^T.  With ``device`` set, the QR and products run in
    torch on that device (large n); returns a numpy array either way."""
    s = np.logspace(0.0, np.log10(kappa), n)
    if device is None:
        g = rng(seed).standard_normal((n, n))
        q, _ = np.linalg.qr(g)
        a = (q * s) @ q.T
        a = 0.5 * (a + a.T)
        return np.asfortranarray(a)
    import torch
    g = torch.from_numpy(rng(seed).standard_normal((n, n))).to(device)
    q, _ = torch.linalg.qr(g)
    a = (q * torch.from_numpy(s).to(device)) @ q.T
    a = 0.5 * (a + a.T)
    return np.asfortranarray(a.cpu().numpy())


def general_spectrum(n: int, kappa: float, seed: int) -> np.ndarray:
    """A nonsymmetric A = U diag(s) V^T (U, V orthogonal from the QR of two
    Gaussian matrices, s log-spaced from 1 to 1/kappa): 2-norm condition kappa."""
    r = rng(seed)
    u, _ = np.linalg.qr(r.standard_normal((n, n)))
    v, _ = np.linalg.qr(r.standard_normal((n, n)))
    s = np.logspace(0.0, -np.log10(kappa), n)
    return np.asfortranarray((u * s) @ v.T)


def spd_spectrum_torch(n: int, kappa: float, seed: int, device: str):
    """Same matrix as spd_spectrum(..., device=device), left on the device as a
    column-major torch tensor."""
    import torch
    s = torch.logspace(0.0, float(np.log10(kappa)), n, dtype=torch.float64, device=device)
    g = torch.from_numpy(rng(seed).standard_normal((n, n))).to(device)
    q, _ = torch.linalg.qr(g)
    a = (q * s) @ q.T
    a = 0.5 * (a + a.T)
    return a.t().contiguous().t()  # symmetric: column-major view of the same values
