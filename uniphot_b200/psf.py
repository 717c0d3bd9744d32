"""PSF descriptors accepted by the solver.

* ``PsfPolynomial`` -- the reference's pixelised PSFEx-style polynomial PSF
  (same fields as ``fit/grid_gpu/psf_polynomial.py:56-71``):
  ``stamp[i, j] = sum_t coefs[i, j, t] X^m Y^n`` with
  ``X = (x - x_origin) / x_scale``; render mode ``"reference"``.
* ``MogPsf`` -- the analytic PSF: K elliptical Gaussians whose sigma, e1, e2
  and weight are polynomials (same term order) in the normalised position;
  component covariance ``s^2 [[1+e1, e2], [e2, 1-e1]]``, weights normalised
  to unit sum; render mode ``"analytic"``.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

_ORDER_OF_NT = {1: 0, 3: 1, 6: 2, 10: 3, 15: 4, 21: 5}


def poly_terms(nt: int):
    """(m, n) exponents, low order first: 1, x, y, x^2, xy, y^2, ..."""
    if nt not in _ORDER_OF_NT:
        raise ValueError(f"n_terms must be one of {sorted(_ORDER_OF_NT)}; got {nt}")
    out = []
    for deg in range(_ORDER_OF_NT[nt] + 1):
        for n in range(deg + 1):
            out.append((deg - n, n))
    return out


def poly_basis_np(X, Y, nt: int) -> np.ndarray:
    """(..., nt) basis values for arrays X, Y."""
    X = np.asarray(X, np.float64)
    Y = np.asarray(Y, np.float64)
    return np.stack([X ** m * Y ** n for (m, n) in poly_terms(nt)], axis=-1)


@dataclass
class PsfPolynomial:
    coefs: np.ndarray          # (H_psf, W_psf, n_terms)
    x_origin: float
    x_scale: float
    y_origin: float
    y_scale: float
    H_psf: int
    W_psf: int

    def stamp_at(self, x: float, y: float) -> np.ndarray:
        X = (x - self.x_origin) / self.x_scale
        Y = (y - self.y_origin) / self.y_scale
        b = poly_basis_np(X, Y, self.coefs.shape[-1]).astype(np.float32)
        return np.tensordot(self.coefs.astype(np.float32), b, axes=([-1], [-1]))


@dataclass
class MogPsf:
    sigma: np.ndarray          # (K, n_terms)
    e1: np.ndarray
    e2: np.ndarray
    weight: np.ndarray
    x_origin: float
    x_scale: float
    y_origin: float
    y_scale: float

    @classmethod
    def constant(cls, sigma, e1, e2, weight, *, x_origin=0.0, x_scale=1.0,
                 y_origin=0.0, y_scale=1.0):
        col = lambda v: np.asarray(v, np.float64).reshape(-1, 1)  # noqa: E731
        return cls(col(sigma), col(e1), col(e2), col(weight),
                   float(x_origin), float(x_scale), float(y_origin), float(y_scale))

    @property
    def n_comp(self) -> int:
        return int(self.sigma.shape[0])

    @property
    def n_terms(self) -> int:
        return int(self.sigma.shape[1])

    def components_at(self, xs, ys):
        """Normalised weights (m, K) and covariances (m, K, 3) = (xx, yy, xy)."""
        X = (np.asarray(xs, np.float64) - self.x_origin) / self.x_scale
        Y = (np.asarray(ys, np.float64) - self.y_origin) / self.y_scale
        b = poly_basis_np(X, Y, self.n_terms)                # (m, nt)
        s = b @ self.sigma.T
        a1 = b @ self.e1.T
        a2 = b @ self.e2.T
        w = b @ self.weight.T
        w = w / w.sum(axis=1, keepdims=True)
        s2 = s * s
        cov = np.stack([s2 * (1 + a1), s2 * (1 - a1), s2 * a2], axis=-1)
        return w, cov


def _mog_stamp(psf: MogPsf, T: int, x: float, y: float, sub: int = 1):
    """Unit-sum stamp of the PSF at (x, y), centre pixel T//2; ``sub`` > 1
    integrates each pixel with sub x sub samples."""
    w, cov = psf.components_at([x], [y])
    c = T // 2
    o = (np.arange(sub) + 0.5) / sub - 0.5
    g = (np.arange(T) - c)[:, None] + o[None, :]
    xx = g.reshape(1, T, 1, sub) * np.ones((T, 1, sub, 1))
    yy = g.reshape(T, 1, sub, 1) * np.ones((1, T, 1, sub))
    img = np.zeros((T, T, sub, sub))
    for q in range(w.shape[1]):
        A, C, B = cov[0, q]
        det = A * C - B * B
        Q = (C * xx * xx - 2 * B * xx * yy + A * yy * yy) / det
        img += w[0, q] * np.exp(-0.5 * Q) / (2 * math.pi * math.sqrt(det))
    st = img.mean(axis=(2, 3))
    return st / st.sum()


def rasterize_mog_psf(psf: MogPsf, T: int, x: float, y: float,
                      sub: int = 8) -> PsfPolynomial:
    """Constant (n_terms = 1) pixel-integrated pixelised PSF at (x, y)."""
    st = _mog_stamp(psf, T, x, y, sub).astype(np.float32)
    return PsfPolynomial(st[:, :, None], psf.x_origin, psf.x_scale,
                         psf.y_origin, psf.y_scale, T, T)


def mog_to_poly_psf(psf: MogPsf, T: int, W: int, H: int, nt: int = 6,
                    grid: int = 7) -> PsfPolynomial:
    """Least-squares pixel-polynomial fit to centre-sampled MoG stamps on a
    grid x grid lattice of field positions (what a PSFEx model of this PSF
    would be)."""
    xs = np.linspace(0, W - 1, grid)
    ys = np.linspace(0, H - 1, grid)
    rows, stamps = [], []
    for yv in ys:
        for xv in xs:
            stamps.append(_mog_stamp(psf, T, xv, yv, 1).reshape(-1))
            rows.append(poly_basis_np((xv - psf.x_origin) / psf.x_scale,
                                      (yv - psf.y_origin) / psf.y_scale, nt))
    Amat = np.stack(rows)
    Y = np.stack(stamps)
    coef, *_ = np.linalg.lstsq(Amat, Y, rcond=None)          # (nt, T*T)
    return PsfPolynomial(coef.T.reshape(T, T, nt).astype(np.float32),
                         psf.x_origin, psf.x_scale, psf.y_origin, psf.y_scale,
                         T, T)
