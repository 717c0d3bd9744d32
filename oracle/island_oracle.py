"""CPU restatement of uniphot's per-island VarPro-LM forced-photometry solve.

TEST INFRASTRUCTURE ONLY.  Nothing in the product path (``uniphot_b200``)
imports this module: it is the checker that the CUDA path is compared
against (``tests/``, ``__graft_entry__.smoke()``) and the timed CPU arm of
``bench.py`` (``cpu_baseline`` / ``--impl reference``).

Parity pin: the reference solver is JAX code and JAX is not installed.  The
host-side numpy modules it relies on (islands.py, island_plan.py,
psf_polynomial.py, the Sersic table) are imported from the reference to
generate the golden fixtures under ``tests/golden/``
(``tests/golden/make_golden.py``), and the reference's own ``island_fit``
is run with a float64 numpy stand-in for JAX
(``tests/golden/make_golden_solver.py``, ``tests/golden/jax_stand_in.py``)
to produce per-source results on seeded fields.  This restatement's float64
mode reproduces those: identical LM iteration counts and flags on every
island, positions within 1e-4 px, fluxes within 1e-5 relative or 1e-3 of
their error (``tests/test_golden_reference_solver.py``), besides the
known-answer tests (noise-free star, zero shift identity, table knots,
finite-difference Jacobians).

Algorithm followed (paths relative to the reference project ``tract7dt/``):

* PSF polynomial stamp ``sum_t coefs[i,j,t] X^m Y^n`` and its spatial basis:
  ``fit/grid_gpu/psf_polynomial.py:134-197``, term order
  ``fit/grid_gpu/bg_polynomial.py:31-100``.
* Lanczos-3 taps (f64, normalised, cast f32) and the separable zero-border
  correlate (x then y, fixed tap order):
  ``fit/optimize/gpu/kernels/lanczos.py:50-181``.
* Star stamp = PSF at (x, y) shifted by ``dx = x - x0 - rint(x - x0)``:
  ``fit/grid_gpu/island_solver.py:441-458``; placement at
  ``rint(x - x0) - T//2``: ``island_solver.py:469-478``.
* Galaxy stamp ("fft" backend): Sersic MoG table lookup
  ``fit/grid_gpu/sersic_mog.py:81-100``, ellipse covariance ``:108-150``,
  Fourier product ``irfft2(rfft2(psf_pad) * sum_k a_k exp(v_k expo))[:T,:T]
  + core * psf`` ``:153-194``, pad rule ``:197-207``; n <-> u logit
  ``fit/grid_gpu/source_model.py:38-54``.
* Per-band VarPro flux solve with ridge ``reg`` on real and 1.0 on padded
  slots, f64 solve: ``island_solver.py:570-590``; whitened residual
  ``:592-605``; chi2 ``:668-684``.
* Gauss-Newton (H, g) = sum_b J_b J_b^T, J_b r_b with J the exact derivative
  of the VarPro residual (AD through the f64 solve):
  ``island_solver.py:812-865``.  Here J is formed explicitly per pixel from
  the analytic stamp derivatives and the Golub-Pereyra formula.
* LM step (keep mask, damping, f64 solve, clips, bounds, accept/reject,
  three convergence prongs): ``island_solver.py:921-1002`` with constants
  ``:146-152`` and ``fit/grid_gpu/island_plan.py:55-74``.
* Step variants: trust-region scaled dogleg ``island_solver.py:1004-1116``
  (radius carried in the lam slot, seeded by the first Gauss-Newton step),
  "changed" stall counting ``:1118-1208``, "dlnp" convergence
  ``:1210-1333``; bound-pinned disclosure ``:1717-1728``.
* Post-hoc divergence probe ``island_solver.py:1335-1399``, plateau probe
  ``:1401-1465``, final fluxes and errors ``:1467-1482``, marginal
  covariance of the nonlinear parameters ``:1484-1547``, shape-marginalised
  flux-variance increment ``:1549-1613``, source metrics ``:1639-1715``,
  band-coadded residual ``:1615-1637``, Re profile ``:1779-1792``,
  good-pixel count
  ``:2690-2699``.

A second render mode, ``analytic``, is the north-star forward model (not in the
reference): the PSF is a mixture of elliptical Gaussians whose sigma, e1, e2
and weight are polynomials in the normalised position; galaxy MoG components
are convolved analytically (covariances add), sampled at pixel centres around
the integer-rounded position, then Lanczos-3 shifted exactly like the
reference's stars.

Two precisions:

* ``"f64"``: everything float64 (the FP64 oracle for flux-error metrics).
* ``"ref"``: the reference's arithmetic classes: f32 stamps / residuals /
  H, g; f64 flux and step solves; f32 LM state and chi2 (per-band sums formed
  exactly and rounded to f32, accumulated over bands in f32).
"""

from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

SOURCE_STAR, SOURCE_EXP, SOURCE_DEV, SOURCE_SERSIC = 0, 1, 2, 3
SERSIC_N_MIN, SERSIC_N_MAX = 0.29, 6.3

# LM constants (island_solver.py:146-152, island_plan.py:55-74)
STALL_REJECT_K = 4
SHAPE_STEP_MAX = 0.15
UN_STEP_MAX = 0.5
SHAPE_STEP_TOL = 0.01
LM_LAMBDA0 = 1e-3
LM_UP, LM_DOWN = 10.0, 0.1
LAM_MIN, LAM_MAX = 1e-9, 1e6
# trust-region radius update (island_solver.py:154-163): Nocedal & Wright
# Alg. 4.1 gain-ratio thresholds, shrink and expand factors
TR_ETA_LO, TR_ETA_HI = 0.25, 0.75
TR_SHRINK, TR_EXPAND = 0.25, 2.0

_ORDER_OF_NT = {1: 0, 3: 1, 6: 2, 10: 3, 15: 4, 21: 5}


def poly_terms(nt: int):
    """(m, n) exponent pairs in the low-order-first PSFEx order."""
    if nt not in _ORDER_OF_NT:
        raise ValueError(f"unsupported number of polynomial terms {nt}")
    order = _ORDER_OF_NT[nt]
    out = []
    for deg in range(order + 1):
        for n in range(deg + 1):
            out.append((deg - n, n))
    return out


def poly_basis(X: float, Y: float, nt: int):
    """Basis values and d/dX, d/dY (float64 arrays of length nt)."""
    b = np.empty(nt)
    bx = np.empty(nt)
    by = np.empty(nt)
    for t, (m, n) in enumerate(poly_terms(nt)):
        b[t] = X ** m * Y ** n
        bx[t] = m * X ** (m - 1) * Y ** n if m > 0 else 0.0
        by[t] = n * X ** m * Y ** (n - 1) if n > 0 else 0.0
    return b, bx, by


# ---------------------------------------------------------------------------
# Lanczos-3
# ---------------------------------------------------------------------------

def _l3(x: np.ndarray):
    """Lanczos-3 window value and derivative (float64)."""
    ax = np.abs(x)
    zero = ax < 1e-12
    out = ax >= 3.0
    xs = np.where(zero, 1.0, x)
    px = np.pi * xs
    s1, c1 = np.sin(px), np.cos(px)
    s3, c3 = np.sin(px / 3.0), np.cos(px / 3.0)
    val = 3.0 * s1 * s3 / (px * px)
    dval = 3.0 * (np.pi * c1 * s3 + (np.pi / 3.0) * s1 * c3) / (px * px) \
        - 6.0 * s1 * s3 / (np.pi * np.pi * xs ** 3)
    v = np.where(zero, 1.0, np.where(out, 0.0, val))
    dv = np.where(zero | out, 0.0, dval)
    return v, dv


def lanczos3_taps(d: float):
    """Normalised 7-tap weights at offsets -3..3 (+d) and d(weights)/dd."""
    x = np.arange(-3, 4, dtype=np.float64) + float(d)
    v, dv = _l3(x)
    s = v.sum()
    ds = dv.sum()
    return v / s, (dv * s - v * ds) / (s * s)


def correlate_x(img: np.ndarray, taps: np.ndarray) -> np.ndarray:
    """out[:, j] = sum_k taps[k] img[:, j + k - 3], zero border, k in order."""
    n = img.shape[1]
    pad = np.zeros((img.shape[0], n + 6), dtype=img.dtype)
    pad[:, 3:3 + n] = img
    out = taps[0] * pad[:, 0:n]
    for k in range(1, 7):
        out = out + taps[k] * pad[:, k:k + n]
    return out


def correlate_y(img: np.ndarray, taps: np.ndarray) -> np.ndarray:
    n = img.shape[0]
    pad = np.zeros((n + 6, img.shape[1]), dtype=img.dtype)
    pad[3:3 + n, :] = img
    out = taps[0] * pad[0:n, :]
    for k in range(1, 7):
        out = out + taps[k] * pad[k:k + n, :]
    return out


# ---------------------------------------------------------------------------
# Sersic MoG table and ellipse covariance
# ---------------------------------------------------------------------------

@dataclass
class SersicTable:
    n_knots: np.ndarray
    amps: np.ndarray
    log_vars: np.ndarray
    core_amp: np.ndarray
    n_min: float
    n_max: float

    @classmethod
    def load(cls, path):
        z = np.load(path)
        return cls(np.asarray(z["n_knots"], np.float64),
                   np.asarray(z["amps"], np.float64),
                   np.asarray(z["log_vars"], np.float64),
                   np.asarray(z["core_amp"], np.float64),
                   float(z["n_min"]), float(z["n_max"]))

    def lookup(self, n: float):
        """(amps, vars, core) and their d/dn (piecewise-linear interpolant)."""
        inside = self.n_min < n < self.n_max
        nc = min(max(n, self.n_min), self.n_max)
        K = self.n_knots.shape[0]
        i = int(np.searchsorted(self.n_knots, nc, side="right")) - 1
        i = min(max(i, 0), K - 2)
        n0, n1 = self.n_knots[i], self.n_knots[i + 1]
        if n1 > n0:
            t = (nc - n0) / (n1 - n0)
            dt = (1.0 / (n1 - n0)) if inside else 0.0
        else:
            t, dt = 0.0, 0.0
        a = (1 - t) * self.amps[i] + t * self.amps[i + 1]
        lv = (1 - t) * self.log_vars[i] + t * self.log_vars[i + 1]
        v = np.exp(lv)
        core = (1 - t) * self.core_amp[i] + t * self.core_amp[i + 1]
        da = dt * (self.amps[i + 1] - self.amps[i])
        dv = v * dt * (self.log_vars[i + 1] - self.log_vars[i])
        dcore = dt * (self.core_amp[i + 1] - self.core_amp[i])
        return a, v, core, da, dv, dcore


def u_to_n(u: float):
    """Sigmoid map u -> n and dn/du (source_model.py:50-54)."""
    e = math.exp(-u)
    n = SERSIC_N_MIN + (SERSIC_N_MAX - SERSIC_N_MIN) / (1.0 + e)
    dn = (SERSIC_N_MAX - SERSIC_N_MIN) * e / (1.0 + e) ** 2
    return n, dn


def cov_terms(lr: float, e1: float, e2: float):
    """(cxx, cyy, cxy) unit-variance covariance and d/d(lr, e1, e2).

    Returns (c (3,), dc (3 params, 3 terms)).  Restates
    sersic_mog._ellipse_cov_terms including the round-source nudge."""
    ex = math.exp(lr)
    re = min(max(ex, 0.1), 1000.0)
    dre = re if 0.1 < ex < 1000.0 else 0.0
    nudge = (e1 == 0.0) and (e2 == 0.0)
    e1n = 1e-4 if nudge else e1
    de1n = 0.0 if nudge else 1.0
    ee = math.hypot(e1n, e2)
    dee1 = e1n / ee * de1n
    dee2 = e2 / ee
    ex2 = math.exp(-ee)
    e = 1.0 - ex2
    de_dee = ex2
    if 1.0 - e > 1e-4:
        den, dden = 1.0 - e, -1.0
    else:
        den, dden = 1e-4, 0.0
    ibr = (1.0 + e) / den
    dibr = (den - (1.0 + e) * dden) / (den * den)
    if ibr < 1000.0:
        ib, dib = ibr, dibr
    else:
        ib, dib = 1000.0, 0.0
    th = 0.5 * math.atan2(e2, e1n)
    dth1 = -0.5 * e2 / (ee * ee) * de1n
    dth2 = 0.5 * e1n / (ee * ee)
    ct, st = math.cos(th), math.sin(th)
    s2 = 1.0 / (ib * ib)
    cxx = re * re * (ct * ct * s2 + st * st)
    cyy = re * re * (st * st * s2 + ct * ct)
    cxy = re * re * ct * st * (1.0 - s2)
    # partials w.r.t. (re, ib, th)
    d_re = np.array([2 * re * (ct * ct * s2 + st * st),
                     2 * re * (st * st * s2 + ct * ct),
                     2 * re * ct * st * (1.0 - s2)])
    d_ib = np.array([re * re * ct * ct * (-2.0 / ib ** 3),
                     re * re * st * st * (-2.0 / ib ** 3),
                     re * re * ct * st * (2.0 / ib ** 3)])
    d_th = np.array([2 * re * re * ct * st * (1.0 - s2),
                     -2 * re * re * ct * st * (1.0 - s2),
                     re * re * (ct * ct - st * st) * (1.0 - s2)])
    dib_dee = dib * de_dee
    dc = np.stack([
        d_re * dre,
        d_ib * dib_dee * dee1 + d_th * dth1,
        d_ib * dib_dee * dee2 + d_th * dth2,
    ])
    return np.array([cxx, cyy, cxy]), dc


def fft_pad_for(T: int) -> int:
    n = 1
    while n < T + T // 2:
        n <<= 1
    return n


# ---------------------------------------------------------------------------
# PSF models
# ---------------------------------------------------------------------------

@dataclass
class PolyPsfBand:
    """Pixelised polynomial PSF for one band, zero-padded to the tier T."""
    coefs: np.ndarray         # (T, T, nt) float32
    x_origin: float
    x_scale: float
    y_origin: float
    y_scale: float

    def stamp(self, x, y, dt):
        """PSF stamp and d/dx, d/dy at image position (x, y)."""
        f32 = np.float32
        X = float(f32((f32(x) - f32(self.x_origin)) / f32(self.x_scale)))
        Y = float(f32((f32(y) - f32(self.y_origin)) / f32(self.y_scale)))
        nt = self.coefs.shape[-1]
        b, bx, by = poly_basis(X, Y, nt)
        c = self.coefs.astype(np.float64)
        S = (c @ b).astype(dt)
        Sx = (c @ (bx / self.x_scale)).astype(dt)
        Sy = (c @ (by / self.y_scale)).astype(dt)
        return S, Sx, Sy, nt > 1


@dataclass
class MogPsfBand:
    """Analytic PSF: K elliptical Gaussians with polynomial parameters.

    Component q has ``Sigma = s^2 [[1+e1, e2], [e2, 1-e1]]`` and weight
    ``w_q / sum_q w_q``; s, e1, e2, w are polynomials (nt terms) in
    ``X = (x - x_origin)/x_scale``, ``Y = (y - y_origin)/y_scale``."""
    sigma: np.ndarray     # (K, nt)
    e1: np.ndarray        # (K, nt)
    e2: np.ndarray        # (K, nt)
    weight: np.ndarray    # (K, nt)
    x_origin: float
    x_scale: float
    y_origin: float
    y_scale: float

    def components(self, x, y):
        """Per-component weights (K,), covariances (K, 3) = (A, C, B) with
        A=Sxx, C=Syy, B=Sxy, and their d/dx, d/dy."""
        X = (x - self.x_origin) / self.x_scale
        Y = (y - self.y_origin) / self.y_scale
        nt = self.sigma.shape[1]
        b, bx, by = poly_basis(X, Y, nt)
        bx = bx / self.x_scale
        by = by / self.y_scale
        s, sx, sy = self.sigma @ b, self.sigma @ bx, self.sigma @ by
        a1, a1x, a1y = self.e1 @ b, self.e1 @ bx, self.e1 @ by
        a2, a2x, a2y = self.e2 @ b, self.e2 @ bx, self.e2 @ by
        wr, wrx, wry = self.weight @ b, self.weight @ bx, self.weight @ by
        W, Wx, Wy = wr.sum(), wrx.sum(), wry.sum()
        w = wr / W
        wx = (wrx * W - wr * Wx) / (W * W)
        wy = (wry * W - wr * Wy) / (W * W)
        s2 = s * s
        cov = np.stack([s2 * (1 + a1), s2 * (1 - a1), s2 * a2], axis=1)

        def dcov(sd, a1d, a2d):
            return np.stack([2 * s * sd * (1 + a1) + s2 * a1d,
                             2 * s * sd * (1 - a1) - s2 * a1d,
                             2 * s * sd * a2 + s2 * a2d], axis=1)
        return w, cov, wx, wy, dcov(sx, a1x, a2x), dcov(sy, a1y, a2y)


def _gauss(xx, yy, A, C, B):
    """Normalised 2-D Gaussian at offsets, its Mahalanobis distance and the
    covariance determinant."""
    det = A * C - B * B
    Q = (C * xx * xx - 2.0 * B * xx * yy + A * yy * yy) / det
    N = np.exp(-0.5 * Q) / (2.0 * np.pi * np.sqrt(det))
    return N, Q, det


def _gauss_and_dlog(xx, yy, A, C, B):
    """Normalised 2-D Gaussian at offsets and d ln N / d(A, C, B)."""
    N, Q, det = _gauss(xx, yy, A, C, B)
    dA = (Q * C - yy * yy - C) / (2.0 * det)
    dC = (Q * A - xx * xx - A) / (2.0 * det)
    dB = (xx * yy - B * Q + B) / det
    return N, dA, dC, dB


# ---------------------------------------------------------------------------
# Island context
# ---------------------------------------------------------------------------

@dataclass
class IslandInput:
    """Everything the per-island solve reads (one island of one class)."""
    B: int
    T: int
    data: np.ndarray         # (n_b, B, B) float32 window of data - bg
    w: np.ndarray            # (n_b, B, B) float32 inverse variance
    x0: float
    y0: float
    stype: np.ndarray        # (N,) int
    n_frozen: np.ndarray     # (N,) float32
    free_n: np.ndarray       # (N,) bool
    mmask: np.ndarray        # (N,) bool
    keep: np.ndarray         # (N, 6) bool
    p0: np.ndarray           # (N*6,) float32
    lower: np.ndarray        # (N*6,)
    upper: np.ndarray
    prior_mean: np.ndarray
    prior_inv_sigma: np.ndarray
    has_priors: bool
    psf: list                # per band PolyPsfBand | MogPsfBand
    table: SersicTable | None
    mode: str                # "reference" | "analytic"
    native: int = 0          # star support side (0 = the tier)
    bg_joint: bool = False   # planar background (1, X, Y) solved with the fluxes
    # cross-band GLS (island_solver.py:607-723, 867-919): {"rank": r,
    # "u": (r, n_b), "lam": (r,)} and the island's amplitude scale; None = off
    crossband: dict | None = None
    cb_scale: float = 1.0
    # galaxy render backend in the pixelised-PSF mode: "fft" (the Sersic
    # mixture's transform) or the legacy "direct" (EXP only: the
    # exponential mixture exp_mog = (amp, var) at pixel centres convolved
    # with the PSF, source_model.py:218-256, 298-303)
    render_backend: str = "fft"
    exp_mog: tuple | None = None


@dataclass
class SolverConfig:
    reg: float = 1e-9
    pos_step_max: float = 0.5
    ftol_rel: float = 1e-4
    step_tol: float = 0.1
    un_freeze_steps: int = 0
    precision: str = "ref"   # "ref" | "f64"
    # "proposals" (legacy) | "changed": a rejected step counts toward the
    # stall only when its proposal differs from the previous rejected one
    # (island_solver.py:1118-1208); identical-proposal runs of
    # STALL_REJECT_K set the sticky diverged flag in the loop
    stall_count_mode: str = "proposals"
    # "legacy" | "dlnp" (island_solver.py:1210-1333): chi2 carried in f64,
    # absolute sub-quantum ftol, quantum-gated step prong, distinct-proposal
    # stall counting with reject-exits at the lam cap or on a no-move
    # proposal; plateau-certified reject-exits count as converged
    convergence: str = "legacy"
    plateau_dlnp_tol: float = 0.5
    # "clip" | "trust_region" (island_solver.py:1004-1116): scaled dogleg
    # inside a radius carried in the lam slot; accept rule and the three
    # convergence prongs as in the clip step.  Callers pass "clip" for star
    # classes, which the reference exempts (island_solver.py:1910-1912).
    step_mode: str = "clip"


class IslandSolver:
    """Per-island VarPro-LM in the reference's legacy/clip/proposals mode."""

    def __init__(self, isl: IslandInput, cfg: SolverConfig):
        self.isl = isl
        self.cfg = cfg
        self.dt = np.float64 if cfg.precision == "f64" else np.float32
        self.N = isl.stype.shape[0]
        self.nP = 6 * self.N
        self.nb = isl.data.shape[0]
        self.clip = np.tile(np.array([cfg.pos_step_max, cfg.pos_step_max,
                                      SHAPE_STEP_MAX, SHAPE_STEP_MAX,
                                      SHAPE_STEP_MAX, UN_STEP_MAX]), self.N)
        self.not_un = np.tile(np.array([1, 1, 1, 1, 1, 0], bool), self.N)

    # ---------------- rendering ----------------
    def _frac(self, x, x0):
        f32 = np.float32
        if self.dt == np.float32:
            g = f32(f32(x) - f32(x0))
            r = np.round(g)
            return float(g - r), int(r)
        g = float(x) - float(x0)
        r = np.round(g)
        return g - r, int(r)

    def _star_unshifted(self, band, x, y):
        psf = self.isl.psf[band]
        T = self.isl.T
        if isinstance(psf, PolyPsfBand):
            S, Sx, Sy, var = psf.stamp(x, y, self.dt)
            return S, (Sx if var else None), (Sy if var else None)
        return self._analytic(band, x, y, None, True)[:3]

    def _analytic(self, band, x, y, gal, need=True):
        """Analytic stamp.  gal = None (star) or (amps, vars, core, da, dv,
        dcore, dn_du, c(3), dc(3,3)).  Returns S, Sx, Sy, S_shape(3), S_u.

        Components (PSF q x galaxy g) are evaluated together; a star is the
        PSF on its native stamp, zero beyond it (the reference zero-pads the
        native PSF to the tier)."""
        psf = self.isl.psf[band]
        T = self.isl.T
        c0 = T // 2
        hs = c0 if gal is not None else min((self.isl.native or T) // 2, c0)
        n = 2 * hs + 1
        off = np.arange(-hs, hs + 1, dtype=np.float64)
        xx = off[None, None, :]
        yy = off[None, :, None]
        wq, cq, wqx, wqy, dcx, dcy = psf.components(float(x), float(y))
        if gal is None:
            ga = np.array([1.0]); gv = np.zeros(1); gda = np.zeros(1); gdv = np.zeros(1)
            cgal = np.zeros(3)
            dcg = np.zeros((3, 3))
            dndu = 0.0
        else:
            amps, vars_, core, da, dv, dcore, dndu, cgal, dcg = gal
            sel = (amps != 0.0) | (da != 0.0)
            ga = np.concatenate([amps[sel], [core]])
            gv = np.concatenate([vars_[sel], [0.0]])
            gda = np.concatenate([da[sel], [dcore]])
            gdv = np.concatenate([dv[sel], [0.0]])
        K = wq.shape[0]
        G = ga.shape[0]
        A = (gv[None, :] * cgal[0] + cq[:, 0, None]).reshape(-1)[:, None, None]
        C = (gv[None, :] * cgal[1] + cq[:, 1, None]).reshape(-1)[:, None, None]
        Bc = (gv[None, :] * cgal[2] + cq[:, 2, None]).reshape(-1)[:, None, None]
        wa = (wq[:, None] * ga[None, :]).reshape(-1)[:, None, None]
        if need:
            N, lA, lC, lB = _gauss_and_dlog(xx, yy, A, C, Bc)
        else:
            N = _gauss(xx, yy, A, C, Bc)[0]
        Nw = wa * N
        Sfull = np.zeros((6, T, T))
        sub = (slice(c0 - hs, c0 + hs + 1), slice(c0 - hs, c0 + hs + 1))
        S = np.zeros((T, T))
        S[sub] = Nw.sum(0)
        Sx = np.zeros((T, T))
        Sy = np.zeros((T, T))
        Ssh = np.zeros((3, T, T))
        Su = np.zeros((T, T))
        if need:
            rep = lambda a: np.repeat(a, G, axis=0)  # noqa: E731  per (q, g)
            wxa = (wqx[:, None] * ga[None, :]).reshape(-1)[:, None, None]
            wya = (wqy[:, None] * ga[None, :]).reshape(-1)[:, None, None]
            dx_ = rep(dcx)[:, :, None, None]
            dy_ = rep(dcy)[:, :, None, None]
            Sx[sub] = (wxa * N + Nw * (lA * dx_[:, 0] + lC * dx_[:, 1]
                                       + lB * dx_[:, 2])).sum(0)
            Sy[sub] = (wya * N + Nw * (lA * dy_[:, 0] + lC * dy_[:, 1]
                                       + lB * dy_[:, 2])).sum(0)
            if gal is not None:
                v = np.tile(gv, K)[:, None, None]
                dvv = np.tile(gdv, K)[:, None, None]
                wda = (wq[:, None] * gda[None, :]).reshape(-1)[:, None, None]
                gA = (Nw * v * lA).sum(0)
                gC = (Nw * v * lC).sum(0)
                gB = (Nw * v * lB).sum(0)
                for s_ in range(3):
                    Ssh[s_][sub] = gA * dcg[s_, 0] + gC * dcg[s_, 1] + gB * dcg[s_, 2]
                Su[sub] = ((wda * N).sum(0) + (Nw * dvv * (
                    lA * cgal[0] + lC * cgal[1] + lB * cgal[2])).sum(0)) * dndu
        del Sfull
        dt = self.dt
        return (S.astype(dt), Sx.astype(dt), Sy.astype(dt),
                Ssh.astype(dt), Su.astype(dt))

    def _galaxy_fft(self, band, x, y, gal, need):
        """Reference 'fft' backend galaxy stamp (+ derivatives if need)."""
        T = self.isl.T
        dt = self.dt
        psf, psfx, psfy = self._star_unshifted(band, x, y)
        amps, vars_, core, da, dv, dcore, dndu, cg, dcg = gal
        pad = fft_pad_for(T)
        cdt = np.complex64 if dt == np.float32 else np.complex128

        def rf(img):
            z = np.zeros((pad, pad), dtype=dt)
            z[:T, :T] = img
            return np.fft.rfft2(z).astype(cdt)
        P = rf(psf)
        v = np.fft.rfftfreq(pad)[None, :]
        w = np.fft.fftfreq(pad)[:, None]
        vv, ww, vw = v * v, w * w, v * w
        expo = -2.0 * np.pi ** 2 * (cg[0] * vv + cg[1] * ww + 2.0 * cg[2] * vw)
        E = np.exp(vars_[:, None, None] * expo[None])
        F = np.tensordot(amps, E, axes=(0, 0))

        def irf(Q):
            return np.fft.irfft2(Q, s=(pad, pad))[:T, :T]
        psf64 = psf.astype(np.float64)
        S = (irf(P * F) + core * psf64).astype(dt)
        if not need:
            return S, None, None, None, None
        F1 = np.tensordot(amps * vars_, E, axes=(0, 0))
        Ssh = np.zeros((3, T, T))
        for s in range(3):
            dexpo = -2.0 * np.pi ** 2 * (dcg[s, 0] * vv + dcg[s, 1] * ww
                                         + 2.0 * dcg[s, 2] * vw)
            Ssh[s] = irf(P * (F1 * dexpo))
        dF = np.tensordot(da, E, axes=(0, 0)) + \
            np.tensordot(amps * dv, E, axes=(0, 0)) * expo
        Su = (irf(P * dF) + dcore * psf64) * dndu
        Sx = Sy = None
        if psfx is not None:
            Sx = (irf(rf(psfx) * F) + core * psfx.astype(np.float64)).astype(dt)
            Sy = (irf(rf(psfy) * F) + core * psfy.astype(np.float64)).astype(dt)
        return S, Sx, Sy, Ssh.astype(dt), Su.astype(dt)

    def _galaxy_direct(self, band, x, y, k, p, need):
        """Legacy 'direct' backend EXP stamp (source_model.py:218-256,
        298-303): the exponential mixture at pixel centres, normalised,
        convolved with the PSF stamp ("same") and renormalised to unit sum.
        Position partials through the PSF's spatial variation by the
        quotient rule; shape partials (log r_e, e1, e2) by float64 central
        differences of the whole stamp (step 1e-6); no Sersic-index row."""
        from .sparse_oracle import convolve_same, exp_profile_direct
        if self.isl.stype[k] != 1:
            raise ValueError("the direct backend renders STAR and EXP sources only")
        dt = self.dt
        amp, var = self.isl.exp_mog
        T = self.isl.T
        psf, psfx, psfy = self._star_unshifted(band, x, y)
        psf64 = np.asarray(psf, np.float64)
        lr, e1, e2 = (float(p[6 * k + 2]), float(p[6 * k + 3]), float(p[6 * k + 4]))

        def stamp(lr_, e1_, e2_):
            c = convolve_same(exp_profile_direct(T, T, lr_, e1_, e2_, amp, var), psf64)
            t = c.sum()
            return (c / t if t > 0 else c), c, t
        S, C, tot = stamp(lr, e1, e2)
        if not need:
            return S.astype(dt), None, None, None, None
        prof = exp_profile_direct(T, T, lr, e1, e2, amp, var)

        def dpos(dpsf):
            if dpsf is None or tot <= 0:
                return None
            dc = convolve_same(prof, np.asarray(dpsf, np.float64))
            return ((dc - S * dc.sum()) / tot).astype(dt)
        h = 1e-6
        Ssh = []
        for j in range(3):
            a = [lr, e1, e2]
            b = [lr, e1, e2]
            a[j] += h
            b[j] -= h
            Ssh.append(((stamp(*a)[0] - stamp(*b)[0]) / (2 * h)).astype(dt))
        return S.astype(dt), dpos(psfx), dpos(psfy), Ssh, np.zeros((T, T), dt)

    def _gal_params(self, k, p):
        isl = self.isl
        lr, e1, e2, u = (float(p[6 * k + 2]), float(p[6 * k + 3]),
                         float(p[6 * k + 4]), float(p[6 * k + 5]))
        if isl.free_n[k]:
            if self.dt == np.float32:
                uf = np.float32(u)
                n = float(np.float32(SERSIC_N_MIN) + np.float32(
                    SERSIC_N_MAX - SERSIC_N_MIN) / (np.float32(1.0) + np.exp(-uf)))
                _, dndu = u_to_n(u)
            else:
                n, dndu = u_to_n(u)
        else:
            n, dndu = float(isl.n_frozen[k]), 0.0
        amps, vars_, core, da, dv, dcore = isl.table.lookup(n)
        c, dc = cov_terms(lr, e1, e2)
        return (amps, vars_, core, da, dv, dcore, dndu, c, dc)

    def member_stamps(self, band, p, k, need):
        """Unit-flux stamp of member k (T, T) and derivative stamps for its
        live parameters (dict param_index -> (T, T)), all in self.dt."""
        isl = self.isl
        dt = self.dt
        x, y = float(p[6 * k]), float(p[6 * k + 1])
        dx, _ = self._frac(x, isl.x0)
        dy, _ = self._frac(y, isl.y0)
        is_star = isl.stype[k] == SOURCE_STAR
        if is_star:
            S, Sx, Sy = self._star_unshifted(band, x, y)
            Ssh = Su = None
        else:
            direct = isl.mode != "analytic" and isl.render_backend == "direct"
            gal = None if direct else self._gal_params(k, p)
            if isl.mode == "analytic":
                S, Sx, Sy, Ssh, Su = self._analytic(band, x, y, gal, need)
            elif isl.render_backend == "direct":
                S, Sx, Sy, Ssh, Su = self._galaxy_direct(band, x, y, k, p, need)
            else:
                S, Sx, Sy, Ssh, Su = self._galaxy_fft(band, x, y, gal, need)
        Lx, dLx = lanczos3_taps(dx)
        Ly, dLy = lanczos3_taps(dy)
        Lx, dLx, Ly, dLy = (a.astype(dt) for a in (Lx, dLx, Ly, dLy))
        sx = correlate_x(S, Lx)
        m = correlate_y(sx, Ly)
        if not need:
            return m, {}
        keep = isl.keep[k]
        D = {}
        shift = lambda img: correlate_y(correlate_x(img, Lx), Ly)  # noqa: E731
        if keep[0]:
            d = correlate_y(correlate_x(S, dLx), Ly)
            if Sx is not None:
                d = d + shift(Sx)
            D[0] = d
        if keep[1]:
            d = correlate_y(sx, dLy)
            if Sy is not None:
                d = d + shift(Sy)
            D[1] = d
        if not is_star:
            for s in range(3):
                if keep[2 + s]:
                    D[2 + s] = shift(Ssh[s])
            if keep[5]:
                D[5] = shift(Su)
        return m, D

    def place(self, stamp, ix_top, iy_top):
        B, T = self.isl.B, self.isl.T
        out = np.zeros((B, B), dtype=stamp.dtype)
        y0, x0 = max(iy_top, 0), max(ix_top, 0)
        y1, x1 = min(iy_top + T, B), min(ix_top + T, B)
        if y1 > y0 and x1 > x0:
            out[y0:y1, x0:x1] = stamp[y0 - iy_top:y1 - iy_top,
                                      x0 - ix_top:x1 - ix_top]
        return out

    def bg_basis(self):
        """(3, B, B) planar background basis over the island window:
        1, X = (x - c) / s, Y = (y - c) / s with c = (B - 1) / 2, s = B / 2
        (the per-tile plane of forced_phot_sparse.py:417-497 /
        bg_polynomial.py:125-178 at order 1, the island window as its
        tile), in the working precision."""
        B = self.isl.B
        c, sc = (B - 1) / 2.0, B / 2.0
        X = ((np.arange(B, dtype=np.float64) - c) / sc).astype(np.float32)
        P = np.zeros((3, B, B), dtype=self.dt)
        P[0] = 1.0
        P[1] = X[None, :]
        P[2] = X[:, None]
        return P

    @property
    def n_lin(self):
        return self.N + (3 if self.isl.bg_joint else 0)

    def models_band(self, band, p, need):
        """M (n_lin, B, B) placed unit models (+ the background basis when
        bg_joint) and derivative list [(k, j, (B,B))] for live params."""
        isl = self.isl
        N, B, T = self.N, isl.B, isl.T
        M = np.zeros((self.n_lin, B, B), dtype=self.dt)
        if isl.bg_joint:
            M[N:] = self.bg_basis()
        Ds = []
        for k in range(N):
            if not isl.mmask[k]:
                continue
            x, y = float(p[6 * k]), float(p[6 * k + 1])
            _, rx = self._frac(x, isl.x0)
            _, ry = self._frac(y, isl.y0)
            ixt, iyt = rx - T // 2, ry - T // 2
            m, D = self.member_stamps(band, p, k, need)
            M[k] = self.place(m, ixt, iyt)
            for j in sorted(D):
                Ds.append((k, j, self.place(D[j], ixt, iyt)))
        return M, Ds

    # ---------------- linear algebra ----------------
    def fluxes_band(self, M, d, w):
        """Linear solve of one band: fluxes (and background coefficients).
        Ridge: reg on real members, 1.0 on padded slots
        (island_solver.py:570-590); reg * |diag| on background rows (the
        element-wise ridge of forced_phot_sparse.py:474-489)."""
        nl = self.n_lin
        mm = np.concatenate([self.isl.mmask, np.ones(nl - self.N, bool)])
        w64 = w.astype(np.float64)
        M64 = M.reshape(nl, -1).astype(np.float64)
        wm = M64 * w64.reshape(1, -1)
        A = wm @ M64.T
        b = wm @ d.astype(np.float64).reshape(-1)
        if self.dt == np.float32:
            A = A.astype(np.float32).astype(np.float64)
            b = b.astype(np.float32).astype(np.float64)
        ridge = np.where(mm, self.cfg.reg, 1.0)
        ridge[self.N:] = self.cfg.reg * np.maximum(np.abs(np.diag(A)[self.N:]), 1e-30)
        A64 = A + np.diag(ridge)
        f64 = np.linalg.solve(A64, b)
        f = (f64.astype(self.dt) * mm).astype(self.dt)
        return f, f64, A64

    def chi2_band(self, M, d, w, f):
        model = np.tensordot(f.astype(self.dt), M, axes=(0, 0))
        r = np.sqrt(w.astype(self.dt)) * (d.astype(self.dt) - model)
        r64 = r.astype(np.float64)
        return float((r64 * r64).sum()), r

    def chi2_of64(self, p):
        """chi2 with the band sums accumulated in float64 and the prior
        penalty's float32 squares summed in float64
        (island_solver.py:741-758)."""
        c = 0.0
        resids = []
        for b in range(self.nb):
            M, _ = self.models_band(b, p, False)
            f, _, _ = self.fluxes_band(M, self.isl.data[b], self.isl.w[b])
            cb, r = self.chi2_band(M, self.isl.data[b], self.isl.w[b], f)
            c += cb
            resids.append(r)
        isl = self.isl
        if isl.crossband is not None:
            q, s_b, wk = self._cb_filters(p)
            c -= self._cb_chi2_corr(resids, q, s_b, wk)[0]
        if isl.has_priors:
            keep = (isl.keep & isl.mmask[:, None]).reshape(-1)
            t = (isl.prior_inv_sigma.astype(self.dt) * (p - isl.prior_mean).astype(self.dt))
            sq = (t * t).astype(self.dt).astype(np.float64)
            c += float(np.sum(np.where(keep, sq, 0.0)))
        return c

    def prior_pen(self, p):
        isl = self.isl
        if not isl.has_priors:
            return 0.0
        keep = (isl.keep & isl.mmask[:, None]).reshape(-1)
        t = isl.prior_inv_sigma * (p - isl.prior_mean)
        return float(np.sum(np.where(keep, t * t, 0.0)))

    def _cb_filters(self, p):
        """Cross-band GLS channels (island_solver.py:607-666): per band the
        filter q_b = rfft2 of the PSF at the members' mean position (zero-
        padded to, or centre-cropped to, B x B), the channel weights
        s_b = sqrt(lam) sqrt(max(cb_scale, 0)) u_b, and the rfft half-plane
        weights (2, with 1 on the zero and Nyquist columns)."""
        isl = self.isl
        cb = isl.crossband
        if isl.mode != "reference":
            raise ValueError("cross-band GLS needs the pixelised PSF (reference mode)")
        B, T = isl.B, isl.T
        pp = np.asarray(p, np.float32).reshape(self.N, 6)
        mm = isl.mmask.astype(np.float32)
        den = np.float32(max(float(mm.sum()), 1.0))
        cx = float(np.float32((pp[:, 0] * mm).sum()) / den)
        cy = float(np.float32((pp[:, 1] * mm).sum()) / den)
        u = np.asarray(cb["u"], np.float64)
        sl = np.sqrt(np.clip(np.asarray(cb["lam"], np.float64), 0.0, None))
        scale = math.sqrt(max(float(isl.cb_scale), 0.0))
        q = []
        for b in range(self.nb):
            st = isl.psf[b].stamp(cx, cy, np.float64)[0]
            if T <= B:
                z = np.zeros((B, B))
                z[:T, :T] = st
            else:
                o = (T - B) // 2
                z = st[o:o + B, o:o + B]
            q.append(np.fft.rfft2(z))
        wk = np.full((B, B // 2 + 1), 2.0)
        wk[:, 0] = 1.0
        if B % 2 == 0:
            wk[:, -1] = 1.0
        s_b = (sl * scale)[None, :] * u.T            # (n_b, r)
        return np.stack(q), s_b, wk

    def _cb_chi2_corr(self, resids, q, s_b, wk):
        """Woodbury correction (1/B^2) sum_k w_k z^H M^-1 z of the GLS chi2
        (island_solver.py:686-712)."""
        B = self.isl.B
        r_ = s_b.shape[1]
        z = np.zeros((r_,) + wk.shape, complex)
        Mc = np.zeros((r_, r_) + wk.shape)
        for b, rb in enumerate(resids):
            rh = np.fft.rfft2(rb.astype(np.float64).reshape(B, B))
            z += s_b[b][:, None, None] * (np.conj(q[b]) * rh)[None]
            Mc += s_b[b][:, None, None, None] * s_b[b][None, :, None, None] * \
                (np.abs(q[b]) ** 2)[None, None]
        Mk = np.moveaxis(Mc, (0, 1), (-2, -1)) + np.eye(r_)
        zk = np.moveaxis(z, 0, -1)
        sol = np.linalg.solve(Mk, zk[..., None])[..., 0]
        return float(np.sum(wk * np.real(np.sum(np.conj(zk) * sol, axis=-1)))) / (B * B), \
            Mk, zk

    def chi2_of(self, p):
        dt = self.dt
        c = dt(0.0)
        resids = []
        for b in range(self.nb):
            M, _ = self.models_band(b, p, False)
            f, _, _ = self.fluxes_band(M, self.isl.data[b], self.isl.w[b])
            cb, r = self.chi2_band(M, self.isl.data[b], self.isl.w[b], f)
            c = dt(c + dt(cb))
            resids.append(r)
        if self.isl.crossband is not None:
            q, s_b, wk = self._cb_filters(p)
            c = dt(c - dt(self._cb_chi2_corr(resids, q, s_b, wk)[0]))
        if self.isl.has_priors:
            c = dt(c + dt(self.prior_pen(p)))
        return c

    def hg(self, p, flux_jac=None):
        """Un-masked, un-damped Gauss-Newton (H, g) with the explicit
        VarPro Jacobian J_j = -sqrt(w)(f_k D_j + M^T c_j),
        c_j = A64^{-1}(e_k s_j - f_k u_j) = d f / d theta_j (the flux
        solution's sensitivity).  ``flux_jac``, a dict, receives per band
        (parameter indices, c rows (n_live, n_lin))."""
        dt = self.dt
        nP, N = self.nP, self.N
        H = np.zeros((nP, nP), dtype=dt)
        g = np.zeros(nP, dtype=dt)
        cbx = self.isl.crossband is not None
        cb_r, cb_J = [], []
        for b in range(self.nb):
            d, w = self.isl.data[b], self.isl.w[b]
            M, Ds = self.models_band(b, p, True)
            f, f64, A64 = self.fluxes_band(M, d, w)
            _, r = self.chi2_band(M, d, w, f)
            if cbx:
                cb_r.append(r)
                cb_J.append(np.zeros((nP, r.size)))
            if not Ds:
                continue
            w64 = w.astype(np.float64).reshape(-1)
            M64 = M.reshape(self.n_lin, -1).astype(np.float64)
            rt = d.astype(np.float64).reshape(-1) - f64 @ M64
            sw = np.sqrt(w.astype(dt).astype(np.float64)).reshape(-1)
            Ainv = np.linalg.inv(A64)
            rows = []
            idx = []
            cjs = []
            for (k, j, Dp) in Ds:
                D64 = Dp.astype(np.float64).reshape(-1)
                s = np.dot(D64 * w64, rt)
                u = M64 @ (D64 * w64)
                rhs = -f64[k] * u
                rhs[k] += s
                cj = Ainv @ rhs
                if dt == np.float32:
                    cj = cj.astype(np.float32).astype(np.float64)
                cjs.append(cj)
                J = -sw * (float(f[k]) * D64 + cj @ M64)
                if dt == np.float32:
                    J = J.astype(np.float32).astype(np.float64)
                rows.append(J)
                idx.append(6 * k + j)
            Jb = np.stack(rows)
            if cbx:
                cb_J[-1][np.array(idx)] = Jb
            if flux_jac is not None:
                flux_jac[b] = (np.array(idx), np.stack(cjs))
            Hb = Jb @ Jb.T
            gb = Jb @ r.astype(np.float64).reshape(-1)
            ii = np.array(idx)
            Hf = np.zeros((nP, nP))
            Hf[np.ix_(ii, ii)] = Hb
            gf = np.zeros(nP)
            gf[ii] = gb
            H = (H + Hf.astype(dt)).astype(dt)
            g = (g + gf.astype(dt)).astype(dt)
        if cbx:
            # Woodbury corrections of the GLS Gauss-Newton system
            # (island_solver.py:894-919): JZ_p = sum_b s_b conj(q_b) FFT(J_b,p)
            B = self.isl.B
            q, s_b, wk = self._cb_filters(p)
            _, Mk, zk = self._cb_chi2_corr(cb_r, q, s_b, wk)
            JZ = np.zeros((nP, s_b.shape[1]) + wk.shape, complex)
            for b in range(self.nb):
                Jh = np.fft.rfft2(cb_J[b].reshape(nP, B, B))
                JZ += s_b[b][None, :, None, None] * (np.conj(q[b])[None] * Jh)[:, None]
            JZk = np.moveaxis(JZ, (0, 1), (-2, -1))          # (B, Bh, nP, r)
            solz = np.linalg.solve(Mk, zk[..., None])[..., 0]
            solJ = np.linalg.solve(Mk, np.conj(np.swapaxes(JZk, -1, -2)))
            Hc2 = np.real(np.einsum("ab,abpr,abrq->pq", wk, JZk, solJ)) / (B * B)
            gc2 = np.real(np.einsum("ab,abpr,abr->p", wk, np.conj(JZk), solz)) / (B * B)
            H = (H - Hc2.astype(dt)).astype(dt)
            g = (g - gc2.astype(dt)).astype(dt)
        return H, g

    def _keep(self, nsteps):
        isl = self.isl
        keep = (isl.keep & isl.mmask[:, None]).reshape(-1)
        if self.cfg.un_freeze_steps > 0:
            keep = keep & (self.not_un | (nsteps < self.cfg.un_freeze_steps))
        return keep

    def propose(self, p, H, g, lam, keep):
        """Damped f64 step, clips and bounds (island_solver.py:932-967)."""
        dt = self.dt
        isl = self.isl
        nP = self.nP
        ko = keep[:, None] & keep[None, :]
        Hm = np.where(ko, H, dt(0)).astype(dt) + np.diag(
            np.where(keep, 0.0, 1.0)).astype(dt)
        gm = np.where(keep, g, dt(0)).astype(dt)
        if isl.has_priors:
            pi2 = (isl.prior_inv_sigma * isl.prior_inv_sigma).astype(dt)
            pdiag = np.where(keep, pi2, dt(0)).astype(dt)
            gm = (gm + np.where(keep, pi2 * (p - isl.prior_mean).astype(dt),
                                dt(0))).astype(dt)
            Hd = (Hm + dt(lam) * np.diag(np.diag(Hm)) + np.diag(pdiag)
                  + dt(1e-8) * np.eye(nP, dtype=dt)).astype(dt)
        else:
            Hd = (Hm + dt(lam) * np.diag(np.diag(Hm))
                  + dt(1e-8) * np.eye(nP, dtype=dt)).astype(dt)
        delta = -np.linalg.solve(Hd.astype(np.float64), gm.astype(np.float64))
        delta = delta.astype(dt)
        delta = np.where(keep, delta, dt(0)).astype(dt)
        delta = np.clip(delta, -self.clip.astype(dt), self.clip.astype(dt))
        p_try = np.clip((p + delta).astype(dt), isl.lower.astype(dt),
                        isl.upper.astype(dt)).astype(dt)
        return p_try

    def propose_tr(self, p, H, g, delta_r, keep):
        """Scaled dogleg step inside the trust radius (island_solver.py:
        1021-1078).  Returns (p_try, pred, Dr, Dmax, at_bnd): the predicted
        chi2 gain of the realised (box-clipped) step, the radius used (the
        first call seeds it with the Gauss-Newton step's scaled length), the
        radius cap and whether the step reached the boundary."""
        dt = self.dt
        isl = self.isl
        nP = self.nP
        ko = keep[:, None] & keep[None, :]
        Hm = np.where(ko, H, dt(0)).astype(dt) + np.diag(
            np.where(keep, 0.0, 1.0)).astype(dt)
        gm = np.where(keep, g, dt(0)).astype(dt)
        if isl.has_priors:
            pi2 = (isl.prior_inv_sigma * isl.prior_inv_sigma).astype(dt)
            pdiag = np.where(keep, pi2, dt(0)).astype(dt)
            gm = (gm + np.where(keep, pi2 * (p - isl.prior_mean).astype(dt),
                                dt(0))).astype(dt)
            Hm = (Hm + np.diag(pdiag) + dt(1e-8) * np.eye(nP, dtype=dt)).astype(dt)
        else:
            Hm = (Hm + dt(1e-8) * np.eye(nP, dtype=dt)).astype(dt)
        H64 = Hm.astype(np.float64)
        g64 = gm.astype(np.float64)
        dsc = np.sqrt(np.maximum(np.diag(H64), 1e-12))
        s_gn = dsc * -np.linalg.solve(H64, g64)
        n_gn = float(np.sqrt(s_gn @ s_gn))
        Dr = float(delta_r)
        if Dr <= 0.0:          # unset: the first Gauss-Newton step's length
            Dr = max(n_gn, 1e-6)
        gh = g64 / dsc
        Hgh = (H64 @ (gh / dsc)) / dsc
        ghHgh = float(gh @ Hgh)
        gg = float(gh @ gh)
        alpha = gg / max(ghHgh, 1e-30) if ghHgh > 0.0 else 1.0
        s_c = -alpha * gh
        ss = float(s_c @ s_c)
        n_c = math.sqrt(ss)
        diff = s_gn - s_c
        aa = float(diff @ diff)
        bb = 2.0 * float(s_c @ diff)
        cc = ss - Dr * Dr
        disc = max(bb * bb - 4.0 * aa * cc, 0.0)
        t = min(max((-bb + math.sqrt(disc)) / max(2.0 * aa, 1e-30), 0.0), 1.0)
        if n_gn <= Dr:
            s = s_gn
        elif n_c >= Dr:
            s = (Dr / max(n_c, 1e-30)) * s_c if n_c > 0.0 else s_c
        else:
            s = s_c + t * diff
        s_norm = float(np.sqrt(s @ s))
        delta = np.where(keep, (s / dsc).astype(dt), dt(0)).astype(dt)
        p_try = np.clip((p + delta).astype(dt), isl.lower.astype(dt),
                        isl.upper.astype(dt)).astype(dt)
        d = (p_try - p).astype(dt).astype(np.float64)
        pred = -(float(g64 @ d) + 0.5 * float(d @ (H64 @ d)))
        span = (isl.upper.astype(dt) - isl.lower.astype(dt)).astype(dt).astype(np.float64)
        v = dsc * span
        Dmax = float(np.sqrt(v @ v))
        return p_try, pred, Dr, Dmax, s_norm >= 0.99 * Dr

    def railed(self, p):
        """Any kept member parameter at its box bound (island_solver.py:
        1717-1728)."""
        isl = self.isl
        keep = (isl.keep & isl.mmask[:, None]).reshape(-1)
        dt = self.dt
        pp = np.asarray(p, dt).reshape(-1)
        return bool(np.any(keep & ((pp <= isl.lower.astype(dt))
                                   | (pp >= isl.upper.astype(dt)))))

    # ---------------- LM loop ----------------
    def run(self, max_steps, state=None):
        dt = self.dt
        isl = self.isl
        cfg = self.cfg
        dlnp = cfg.convergence == "dlnp"
        changed = cfg.stall_count_mode == "changed" or dlnp
        tr = cfg.step_mode == "trust_region"
        quantum = 2.0 * cfg.plateau_dlnp_tol
        div, n_same = False, 0
        prej = np.zeros(self.nP, dt)
        if state is None:
            p = isl.p0.astype(dt).copy()
            lam = dt(0.0) if tr else dt(LM_LAMBDA0)   # 0: radius unset
            chi2 = self.chi2_of64(p) if dlnp else self.chi2_of(p)
            consec = nrej = nst = 0
        else:
            p = np.asarray(state["p"], dt).reshape(-1).copy()
            lam = dt(state["lam"])
            chi2 = self.chi2_of64(p) if dlnp else dt(state["chi2"])
            consec, nrej, nst = (int(state["consec"]), int(state["nrej"]),
                                 int(state["nst"]))
            div = bool(state.get("diverged", False))
            n_same = int(state.get("n_same", 0))
            prej = np.asarray(state.get("prej", prej), dt).reshape(-1).copy()
        conv = False
        stall = False
        HG = None
        steps = 0
        N = self.N
        mmf = isl.mmask.astype(np.float64)
        for _ in range(int(max_steps)):
            if conv:
                break
            steps += 1
            if HG is None:
                HG = self.hg(p)
            H, g = HG
            keep = self._keep(nst)
            if tr:
                p_try, pred, Dr, Dmax, at_bnd = self.propose_tr(p, H, g, lam, keep)
            else:
                p_try = self.propose(p, H, g, lam, keep)
            chi2_try = self.chi2_of64(p_try) if dlnp else self.chi2_of(p_try)
            accept = bool(chi2_try < chi2)
            p_new = p_try if accept else p
            if tr:
                # gain ratio on the realised step; radius update of
                # Nocedal & Wright Alg. 4.1 (island_solver.py:1079-1092)
                actual = float(dt(chi2 - chi2_try))
                rho = actual / (pred if pred > 0.0 else 1e-30)
                if rho < TR_ETA_LO:
                    Dr_new = Dr * TR_SHRINK
                elif rho > TR_ETA_HI and at_bnd:
                    Dr_new = min(Dr * TR_EXPAND, Dmax)
                else:
                    Dr_new = Dr
                lam_new = dt(Dr_new)
            else:
                lam_new = dt(max(lam * dt(LM_DOWN), dt(LAM_MIN))) if accept \
                    else dt(min(lam * dt(LM_UP), dt(LAM_MAX)))
            se = (p_new - p).astype(np.float64).reshape(N, 6)
            pos_step = float(np.max(mmf * np.hypot(se[:, 0], se[:, 1])))
            shape_step = float(np.max(mmf[:, None] * np.abs(se[:, 2:6])))
            if dlnp:
                dchi2 = chi2 - chi2_try               # float64
                sub_q = dchi2 < quantum
                small = accept and sub_q
                step_small = accept and pos_step < cfg.step_tol \
                    and shape_step < SHAPE_STEP_TOL and sub_q
            else:
                dchi2 = dt(chi2 - chi2_try)
                small = accept and (dchi2 < dt(cfg.ftol_rel) * max(chi2, dt(1.0)))
                step_small = accept and pos_step < cfg.step_tol \
                    and shape_step < SHAPE_STEP_TOL
            consec = consec + 1 if small else (0 if accept else consec)
            if changed:
                # proposal identity (exact comparison) with the previous
                # rejected proposal (island_solver.py:1180-1192)
                prop_same = n_same > 0 and bool(np.all(p_try == prej))
                n_same = 0 if accept else (n_same + 1 if prop_same else 1)
                if not accept:
                    prej = p_try.astype(dt).copy()
                nrej = 0 if accept else (nrej if prop_same else nrej + 1)
                div = div or n_same >= STALL_REJECT_K
            else:
                nrej = 0 if accept else nrej + 1
            stall_now = nrej >= STALL_REJECT_K
            if dlnp and not accept and (lam >= dt(LAM_MAX) or bool(np.all(p_try == p))):
                stall_now = True     # no further information reachable
            conv = (consec >= 2) or step_small or stall_now
            stall = stall_now
            if accept:
                p = p_new
                chi2 = chi2_try if dlnp else dt(chi2_try)
                HG = None
            lam = lam_new
            nst += 1
        return dict(p=p, lam=lam, chi2=chi2, consec=consec, nrej=nrej,
                    nst=nst, conv=conv, stall=stall, steps=steps, HG=HG,
                    div=div, n_same=n_same, prej=prej)

    def diverged_probe(self, p, lam_final, nsteps_final, HG=None):
        """True iff the K rejected proposals of a stall were identical."""
        dt = self.dt
        H, g = HG if HG is not None else self.hg(p)
        props = []
        for j in range(STALL_REJECT_K):
            lam_j = dt(dt(lam_final) * dt(10.0 ** (j - STALL_REJECT_K)))
            keep = self._keep(nsteps_final - STALL_REJECT_K + j) \
                if self.cfg.un_freeze_steps > 0 else self._keep(0)
            props.append(self.propose(p, H, g, lam_j, keep))
        return all(np.array_equal(props[0], q) for q in props[1:])

    def plateau_probe(self, p, nsteps_final, HG=None):
        """min over the lam ladder 1e-9..1e6 of chi2(prop) - chi2(p)."""
        dt = self.dt
        c0 = self.chi2_of(p)
        H, g = HG if HG is not None else self.hg(p)
        keep = self._keep(nsteps_final)
        best = None
        for e in range(-9, 7):
            lam_j = dt(10.0 ** e)
            v = dt(self.chi2_of(self.propose(p, H, g, lam_j, keep)) - c0)
            best = v if best is None else min(best, v)
        return best

    def _posterior(self, p, flux_jac=None):
        """(H, keep, Hm, prior diagonal) at p with the static keep mask."""
        dt = self.dt
        isl = self.isl
        H, _ = self.hg(p, flux_jac)
        keep = (isl.keep & isl.mmask[:, None]).reshape(-1)
        Hm = np.where(keep[:, None] & keep[None, :], H, dt(0)).astype(dt) + np.diag(
            np.where(keep, 0.0, 1.0)).astype(dt)
        pdiag = None
        if isl.has_priors:
            pi2 = (isl.prior_inv_sigma * isl.prior_inv_sigma).astype(dt)
            pdiag = np.where(keep, pi2, dt(0)).astype(dt)
            Hm = (Hm + np.diag(pdiag)).astype(dt)
        return H, keep, Hm, pdiag

    def final_flux_marg(self, p):
        """Shape-marginalised flux-variance increment (island_solver.py:
        1549-1613): per band and extended member k, J_k Sigma J_k^T with J
        the flux solution's sensitivity to the extended members' kept
        parameters and Sigma the posterior covariance of final_errors;
        0 for star rows and padded slots.  (n_b, N) float32."""
        N = self.N
        isl = self.isl
        fj = {}
        _, keep, Hm, _ = self._posterior(p, fj)
        S = np.linalg.inv(Hm.astype(np.float64))
        ext = (isl.stype != 0) & isl.mmask
        marg = (keep.reshape(N, 6) & ext[:, None]).reshape(-1)
        out = np.zeros((self.nb, N), np.float32)
        for b, (idx, C) in fj.items():
            J = np.zeros((N, self.nP))
            J[:, idx] = C[:, :N].T          # member fluxes only
            J[:, ~marg] = 0.0
            dv = np.einsum("ka,ab,kb->k", J, S, J)
            out[b] = np.where(ext, np.maximum(dv, 0.0), 0.0)
        return out

    def source_metrics(self, p):
        """Per-member model-quality metrics at p (island_solver.py:1639-
        1715): rchisq (own-model-weighted chi2 per unit model flux),
        fracflux (neighbours' light under the member's profile), fracin
        (unit-model flux inside the window), fracmasked (unit-model flux on
        zero-weight pixels), combined over bands as the reference does
        (fin = clip(sum m, 0, 1) weights fracflux and fracmasked; fracin and
        rchisq are ratios of band sums); and the per-band window flux
        f * sum(m).  Returns ((N, 4), (n_b, N)) float32; padded slots give
        NaN (rchisq, fracin, window flux) or 0.  With a joint background the
        chi2 uses the full model (members and plane) and the neighbours'
        light the members only."""
        isl = self.isl
        N, nb = self.N, self.nb
        acc = np.zeros((8, N))
        fwin = np.zeros((nb, N))
        for b in range(nb):
            d = isl.data[b].astype(np.float64)
            w = isl.w[b].astype(np.float64)
            M, _ = self.models_band(b, p, False)
            f = self.fluxes_band(M, isl.data[b], isl.w[b])[0].astype(np.float64)
            mods = M[:N].astype(np.float64)
            model_m = np.tensordot(f[:N], mods, 1)
            full = model_m + (np.tensordot(f[N:], M[N:].astype(np.float64), 1)
                              if isl.bg_joint else 0.0)
            own = f[:N, None, None] * mods
            s_m = mods.sum(axis=(1, 2))
            fin = np.clip(s_m, 0.0, 1.0)
            bot = (own * own).sum(axis=(1, 2))
            top = ((model_m[None] - own) * own).sum(axis=(1, 2))
            ratio = np.where(bot > 0, top / np.where(bot > 0, bot, 1.0), 0.0)
            fm = np.clip(((w == 0)[None] * mods).sum(axis=(1, 2)), 0.0, 1.0)
            rc = (mods * (w * (d - full) ** 2)[None]).sum(axis=(1, 2))
            acc += np.stack([fin * ratio, fin, np.abs(s_m), np.ones(N), fin * fm, fin,
                             np.abs(rc), np.abs(s_m)])
            fwin[b] = f[:N] * s_m
        mm = isl.mmask

        def ratio_of(n, dd, fill):
            return np.where((dd > 0) & mm, n / np.where(dd > 0, dd, 1.0), fill)
        met = np.stack([ratio_of(acc[6], acc[7], np.nan), ratio_of(acc[0], acc[1], 0.0),
                        ratio_of(acc[2], acc[3], np.nan), ratio_of(acc[4], acc[5], 0.0)],
                       axis=1)
        fwin = np.where(mm[None, :], fwin, np.nan)
        return met.astype(np.float32), fwin.astype(np.float32)

    def re_profile(self, p, deltas):
        """chi2 along each member slot's log-radius (island_solver.py:
        1779-1792): chi2_of(p + dk e_{6n+2}) - chi2_of(p) for every slot n
        and offset dk (the parameter moved by a float add).  (N, K)
        float32."""
        dt = self.dt
        base = self.chi2_of(p)
        out = np.zeros((self.N, len(deltas)), np.float32)
        for n in range(self.N):
            for j, dk in enumerate(deltas):
                q = np.asarray(p, dt).copy()
                q[6 * n + 2] = dt(q[6 * n + 2] + dt(dk))
                out[n, j] = dt(self.chi2_of(q) - base)
        return out

    def residual_coadd(self, p):
        """Band-coadded residual (island_solver.py:1615-1637): per window
        pixel sum_b w (d - model) and sum_b w, float32 in band order; the
        model includes the plane when it is solved.  ((B, B), (B, B))."""
        isl = self.isl
        dt = np.float32
        R = np.zeros((isl.B, isl.B), dt)
        W = np.zeros((isl.B, isl.B), dt)
        for b in range(self.nb):
            M, _ = self.models_band(b, p, False)
            f = self.fluxes_band(M, isl.data[b], isl.w[b])[0].astype(dt)
            model = np.tensordot(f, M.astype(dt), 1).astype(dt)
            w = isl.w[b].astype(dt)
            R = (R + w * (isl.data[b].astype(dt) - model)).astype(dt)
            W = (W + w).astype(dt)
        return R, W

    def final_errors(self, p):
        """Marginal covariance of the nonlinear parameters at p
        (island_solver.py:1484-1547): the undamped Gauss-Newton matrix with
        the static keep mask (no annealing), plus the prior diagonal,
        inverted in float64.  Returns (N, 13) float32: var(x, y, logre,
        ee1, ee2, u), cov(ee1, ee2), the prior fractions
        pinv^2 / (H_kk + pinv^2) (0 where that sum is 0; NaN without
        priors)."""
        dt = self.dt
        N = self.N
        H, keep, Hm, pdiag = self._posterior(p)
        if pdiag is not None:
            hdiag = np.where(keep, np.diag(H), dt(0)).astype(dt)
            den = (hdiag + pdiag).astype(dt)
            with np.errstate(invalid="ignore", divide="ignore"):
                pf = np.where(den > 0, pdiag / np.where(den > 0, den, dt(1)), dt(0))
            pf6 = pf.reshape(N, 6).astype(np.float64)
        else:
            pf6 = np.full((N, 6), np.nan)
        S = np.linalg.inv(Hm.astype(np.float64))
        var6 = np.diag(S).reshape(N, 6)
        k6 = 6 * np.arange(N)
        cov = S[k6 + 3, k6 + 4]
        return np.concatenate([var6, cov[:, None], pf6], axis=1).astype(np.float32)

    def final_fluxes(self, p):
        """Fluxes and errors (n_b, N), and background coefficients and
        errors (n_b, 3; zero without bg_joint)."""
        nb, N = self.nb, self.N
        F = np.zeros((nb, N), np.float32)
        E = np.zeros((nb, N), np.float32)
        G = np.zeros((nb, 3), np.float32)
        GE = np.zeros((nb, 3), np.float32)
        for b in range(nb):
            M, _ = self.models_band(b, p, False)
            f, _, A64 = self.fluxes_band(M, self.isl.data[b], self.isl.w[b])
            Ainv = np.linalg.inv(A64)
            e = np.sqrt(np.maximum(np.diag(Ainv), 1e-30))
            F[b] = f[:N]
            E[b] = e[:N]
            if self.isl.bg_joint:
                G[b] = f[N:]
                GE[b] = e[N:]
        return F, E, G, GE


def solve_island(isl: IslandInput, cfg: SolverConfig, max_steps: int = 30,
                 state=None, param_errors: bool = False, flux_marg: bool = False,
                source_metrics: bool = False, re_profile=None,
                residual: bool = False):
    """Full per-island result (the row of run_class_chunk's dict)."""
    s = IslandSolver(isl, cfg)
    out = s.run(max_steps, state)
    changed = cfg.stall_count_mode == "changed" or cfg.convergence == "dlnp"
    div = bool(out["div"]) if changed else False
    sd = float("nan")
    if out["stall"]:
        if not changed:   # changed mode keeps the in-loop tracker's flag
            div = s.diverged_probe(out["p"], out["lam"], out["nst"], out["HG"])
        sd = float(s.plateau_probe(out["p"], out["nst"], out["HG"]))
    stall = bool(out["stall"])
    if cfg.convergence == "dlnp" and stall and np.isfinite(sd) \
            and sd > -2.0 * cfg.plateau_dlnp_tol:
        stall = False        # certified: converged on the plateau
    F, E, G, GE = s.final_fluxes(out["p"])
    n_good = int(np.sum(isl.w > 0))
    railed = s.railed(out["p"]) if cfg.step_mode == "trust_region" else False
    perr = s.final_errors(out["p"]) if param_errors else None
    femarg = s.final_flux_marg(out["p"]) if flux_marg else None
    smet, swin = s.source_metrics(out["p"]) if source_metrics else (None, None)
    reprof = s.re_profile(out["p"], re_profile) if re_profile is not None else None
    resid, resid_w = s.residual_coadd(out["p"]) if residual else (None, None)
    return dict(p=out["p"].reshape(s.N, 6).astype(np.float32),
                fluxes=F, ferr=E, bg=G, bg_err=GE, chi2=out["chi2"], conv=out["conv"],
                stall=stall, diverged=div, stall_dchi2=sd,
                nst=out["nst"], lam=out["lam"], consec=out["consec"],
                nrej=out["nrej"], n_good=n_good, steps=out["steps"],
                n_same=out["n_same"], prej=np.asarray(out["prej"], np.float32),
                railed=railed, perr=perr, femarg=femarg, smetrics=smet, swin=swin,
                reprof=reprof, resid=resid, resid_w=resid_w)


def island_inputs_from_host(host: dict, row: int, *, B: int, T: int,
                            dstack, wstack, psf: list, table, mode: str,
                            native: int = 0, bg_joint: bool = False):
    """Slice one island out of class host arrays + the padded stacks."""
    ox, oy = int(host["ox"][row]), int(host["oy"][row])
    N = host["mmask"].shape[1]
    return IslandInput(
        B=B, T=T,
        data=np.ascontiguousarray(dstack[:, oy:oy + B, ox:ox + B]),
        w=np.ascontiguousarray(wstack[:, oy:oy + B, ox:ox + B]),
        x0=float(host["x0b"][row]), y0=float(host["y0b"][row]),
        stype=host["st"][row], n_frozen=host["sn"][row],
        free_n=host["fn_flag"][row], mmask=host["mmask"][row],
        keep=host["keep"][row],
        p0=host["p0"][row].reshape(-1).astype(np.float32),
        lower=host["lower"][row].reshape(-1).astype(np.float32),
        upper=host["upper"][row].reshape(-1).astype(np.float32),
        prior_mean=host["prior_mean"][row].reshape(-1).astype(np.float32),
        prior_inv_sigma=host["prior_inv_sigma"][row].reshape(-1).astype(np.float32),
        has_priors=bool(host["has_priors"]),
        psf=psf, table=table, mode=mode, native=int(native), bg_joint=bool(bg_joint))
