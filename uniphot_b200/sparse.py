"""Per-grid, per-band sparse forced photometry on the GPU: the linear flux +
polynomial-background solve that runs on either side of the island solve
(``tract7dt/fit/grid_gpu/forced_phot_sparse.py``).

Mirrors the reference's entry points for point sources:

* ``GridBandInputs`` / ``SparseForcedPhotResult`` (``:65-116``),
* ``build_neighbor_list`` (``:272-330``) and ``stamp_top_left``
  (``:255-269``) on the host,
* ``make_bg_basis`` (``bg_polynomial.py:125-178``) on the host, for callers
  and tests (the device evaluates the same basis per pixel),
* ``solve_band_sparse`` (``:690-718``): every source's Lanczos-shifted,
  unit-sum PSF stamp at its fixed position, the weighted normal matrix of
  the stamps (diagonal, stamp-overlap pairs from the neighbour list, source
  x background, background x background over the whole grid), an element-
  wise ridge ``reg |diag|``, a float64 solve and the diagonal of the
  inverse -- all in the CUDA library (``uph_sparse_band_solve``).

Extended sources (EXP/DEV/SERSIC) take the reference's "fft" backend
(``source_model.py:304-318``): the Sersic mixture's Fourier transform times
the padded PSF's (``sersic_mog.py:153-194``), cropped to the stamp, plus the
core times the PSF, then the stars' Lanczos shift; with any extended source
no stamp is renormalised (the reference's mixed renderer).  The legacy
"direct" backend (``source_model.py:218-256, 298-303``) renders EXP sources
as the six-Gaussian exponential mixture (``data/exp_mog.npz``) at pixel
centres, convolved with the PSF stamp and renormalised to unit sum; it
accepts STAR and EXP sources only (DEV/SERSIC raise ``ValueError``, as the
reference's pipeline enforces upstream, pipeline.py:1582-1586).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

DEFAULT_K_MAX = 32
SOURCE_STAR = 0

# background polynomial terms (m, n) of X^m Y^n, low order first
# (bg_polynomial.py:25-37)
_TERMS = {0: ((0, 0),), 1: ((0, 0), (1, 0), (0, 1)),
          2: ((0, 0), (1, 0), (0, 1), (2, 0), (1, 1), (0, 2))}


_EXP_MOG = None


def exp_mixture():
    """(amp, var) float32 of the exponential profile's six-Gaussian mixture
    (source_model.py:56-75), from ``data/exp_mog.npz``."""
    global _EXP_MOG
    if _EXP_MOG is None:
        from pathlib import Path
        z = np.load(Path(__file__).with_name("data") / "exp_mog.npz")
        _EXP_MOG = (np.ascontiguousarray(z["amp"], np.float32),
                    np.ascontiguousarray(z["var"], np.float32))
    return _EXP_MOG


def n_terms_for_order(order: int) -> int:
    if order not in _TERMS:
        raise ValueError(f"bg_poly_order must be 0, 1 or 2, got {order}")
    return len(_TERMS[order])


@dataclass
class GridBandInputs:
    """One band of one grid: ``data``, ``invvar``, ``pix_good`` (band_h,
    band_w); source positions in FULL-image pixels; the band's polynomial
    PSF; the grid's top-left in the full image; the background polynomial's
    normalisation.  ``source_type`` may mark extended sources (rejected)."""
    data: np.ndarray
    invvar: np.ndarray
    pix_good: np.ndarray
    pos_x: np.ndarray
    pos_y: np.ndarray
    psf: object                  # uniphot_b200.psf.PsfPolynomial
    band_h: int
    band_w: int
    grid_x0: int
    grid_y0: int
    bg_x_origin: float
    bg_x_scale: float
    bg_y_origin: float
    bg_y_scale: float
    source_type: np.ndarray | None = None
    logre: np.ndarray | None = None
    ee1: np.ndarray | None = None
    ee2: np.ndarray | None = None
    sersic_n: np.ndarray | None = None
    render_backend: str = "direct"
    renorm: bool = True          # unit-sum stamps on the all-star path (the default)


@dataclass
class SparseForcedPhotResult:
    fluxes: np.ndarray           # (n_sources,)
    bg_coefs: np.ndarray         # (M,)
    flux_var: np.ndarray         # (n_sources,) diag of inv(AtWA)
    bg_var: np.ndarray           # (M,)
    converged: bool


def stamp_top_left(pos_x, pos_y, grid_x0: int, grid_y0: int, H_psf: int, W_psf: int):
    """Integer top-left of each stamp in grid coordinates: rint (half to
    even) of the grid-local position minus half the stamp."""
    x = np.asarray(pos_x, np.float32) - np.float32(grid_x0)
    y = np.asarray(pos_y, np.float32) - np.float32(grid_y0)
    return (np.rint(x).astype(np.int32) - W_psf // 2,
            np.rint(y).astype(np.int32) - H_psf // 2)


def build_neighbor_list(pos_x, pos_y, H_psf: int, W_psf: int, k_max: int = DEFAULT_K_MAX):
    """Fixed-width neighbour list: t is a neighbour of s when their stamps
    overlap (|dx| < W_psf and |dy| < H_psf); beyond k_max the closest are
    kept (ties as numpy's argsort orders them).  Returns (idx (n, k_max) int32 padded with
    -1, mask (n, k_max) bool)."""
    from scipy.spatial import cKDTree
    pos_x = np.asarray(pos_x, np.float64)
    pos_y = np.asarray(pos_y, np.float64)
    n = pos_x.size
    idx = np.full((n, k_max), -1, np.int32)
    mask = np.zeros((n, k_max), bool)
    fin = np.nonzero(np.isfinite(pos_x) & np.isfinite(pos_y))[0]
    if fin.size == 0:
        return idx, mask
    xy = np.column_stack([pos_x[fin], pos_y[fin]])
    cands = cKDTree(xy).query_ball_point(xy, r=float(np.hypot(W_psf, H_psf)))
    for a, s in enumerate(fin):
        c = fin[np.asarray(cands[a], np.int64)]
        c = c[c != s]
        if c.size == 0:
            continue
        c = c[(np.abs(pos_x[c] - pos_x[s]) < W_psf) & (np.abs(pos_y[c] - pos_y[s]) < H_psf)]
        if c.size > k_max:
            d2 = (pos_x[c] - pos_x[s]) ** 2 + (pos_y[c] - pos_y[s]) ** 2
            c = c[np.argsort(d2)[:k_max]]
        idx[s, :c.size] = c
        mask[s, :c.size] = True
    return idx, mask


def make_bg_basis(band_h: int, band_w: int, x0: int, y0: int, x_origin: float,
                  x_scale: float, y_origin: float, y_scale: float, order: int = 2):
    """(band_h * band_w, M) float32: X^m Y^n at every grid pixel, X = (x0 +
    column - x_origin) / x_scale (float64, rounded once)."""
    terms = _TERMS[order] if order in _TERMS else None
    if terms is None:
        raise ValueError(f"bg_poly_order must be 0, 1 or 2, got {order}")
    X = (np.arange(band_w, dtype=np.float64) + x0 - x_origin) / x_scale
    Y = (np.arange(band_h, dtype=np.float64) + y0 - y_origin) / y_scale
    cols = [(X[None, :] ** m * Y[:, None] ** n).reshape(-1) for m, n in terms]
    return np.stack(cols, axis=-1).astype(np.float32)


def solve_band_sparse(inputs: GridBandInputs, neighbor_idx, neighbor_mask,
                      reg: float = 1e-9, bg_poly_order: int = 2,
                      context=None, device: int = 0) -> SparseForcedPhotResult:
    """Fluxes and background coefficients of one band of one grid
    (forced_phot_sparse.py:690-718) on the GPU.  ``context`` is a
    ``uniphot_b200._lib.Context`` to reuse (one is created otherwise)."""
    from . import _lib
    if inputs.render_backend not in ("fft", "auto", "direct"):
        raise ValueError(f"unknown render_backend: {inputs.render_backend!r}")
    if inputs.source_type is not None and inputs.render_backend == "direct" and \
            np.any(np.asarray(inputs.source_type) > 1):
        raise ValueError("render_backend='direct' cannot render DEV/SERSIC sources; "
                         "use 'fft' or 'auto'")
    M = n_terms_for_order(bg_poly_order)
    ctx = context if context is not None else _lib.Context(device)
    return ctx.sparse_band_solve(inputs, np.asarray(neighbor_idx), np.asarray(neighbor_mask),
                                 float(reg), int(bg_poly_order), M)
