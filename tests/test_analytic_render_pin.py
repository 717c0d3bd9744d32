"""Independent pin of the analytic render mode's member stamps.

The analytic mode (the headline workload's forward model) renders a member
as the PSF mixture convolved with the galaxy's Gaussian mixture, using the
closed form that the convolution of two Gaussians is a Gaussian whose
covariance is the sum of theirs, sampled at pixel centres around the
integer-rounded centre, then Lanczos-3 shifted.  The oracle restates that
closed form, and the CUDA kernels are held to the oracle.  This file checks
the oracle's stamps against a computation that does not use the closed form:
every (PSF component, galaxy component) convolution integral is evaluated
numerically, by tensor-product Gauss-Hermite quadrature over the narrower of
the two Gaussians (in its whitened coordinates), at every output pixel.  The
delta core of the Sersic mixture convolves to the PSF itself.

Derivative stamps (through the PSF's position dependence, the ellipse
parameters and the Sersic index) are checked against central differences of
the numerical convolution.

Cases: STAR (the PSF on its native stamp), EXP (n = 1), DEV (n = 4) and free
SERSIC near n = 0.5, 2 and 6, at an off-centre field position where the
PSF's order-2 variation matters.  Bar: stamps within 1e-9 of their peak (the
quadrature converges to ~1e-11 with 48 nodes a dimension), derivative stamps
within 1e-6 of their largest magnitude.
"""
from types import SimpleNamespace

import numpy as np
import pytest

from _common import TABLE

GH = 48          # Gauss-Hermite nodes per dimension


def _psf():
    from oracle.driver import psf_bands
    from uniphot_b200.synth import make_production_field
    f = make_production_field(4, side=320, n_bands=1, n_src=10, margin=40)
    return psf_bands(f.mog_psfs, 31, "analytic")[0]


def _gauss(dx, dy, A, C, B):
    det = A * C - B * B
    q = (C * dx * dx - 2.0 * B * dx * dy + A * dy * dy) / det
    return np.exp(-0.5 * q) / (2.0 * np.pi * np.sqrt(det))


def _gh_points():
    t, w = np.polynomial.hermite.hermgauss(GH)
    z1, z2 = np.meshgrid(np.sqrt(2.0) * t, np.sqrt(2.0) * t, indexing="ij")
    ww = np.outer(w, w) / np.pi
    return z1.ravel(), z2.ravel(), ww.ravel()


def _conv_pair(X, Y, cq, cg):
    """(N(.; cq) * N(.; cg)) at offsets (X, Y), by quadrature: the integral
    E_{u ~ N(0, S_n)}[N(x - u; S_w)] over the narrower covariance S_n."""
    def mat(c):
        return np.array([[c[0], c[2]], [c[2], c[1]]])
    Sq, Sg = mat(cq), mat(cg)
    if np.linalg.eigvalsh(Sg).max() <= np.linalg.eigvalsh(Sq).max():
        Sn, Sw = Sg, Sq
    else:
        Sn, Sw = Sq, Sg
    L = np.linalg.cholesky(Sn + 1e-300 * np.eye(2))
    z1, z2, ww = _gh_points()
    ux = L[0, 0] * z1
    uy = L[1, 0] * z1 + L[1, 1] * z2
    g = _gauss(X.ravel()[:, None] - ux[None, :], Y.ravel()[:, None] - uy[None, :],
               Sw[0, 0], Sw[1, 1], Sw[0, 1])
    return (g @ ww).reshape(X.shape)


def _brute(psf, x, y, gal, T, native):
    """Unshifted analytic stamp (T, T) by numerical convolution."""
    w, cov, *_ = psf.components(float(x), float(y))
    c0 = T // 2
    hs = c0 if gal is not None else min(native // 2, c0)
    off = np.arange(-hs, hs + 1, dtype=np.float64)
    X, Y = np.meshgrid(off, off)          # X varies along columns
    sub = np.zeros(X.shape)
    for q in range(w.shape[0]):
        A, C, B = cov[q]
        if gal is None:
            sub += w[q] * _gauss(X, Y, A, C, B)
            continue
        amps, vars_, core, cg = gal
        for g in range(amps.shape[0]):
            if amps[g] == 0.0:
                continue
            sub += w[q] * amps[g] * _conv_pair(X, Y, (A, C, B), vars_[g] * cg)
        sub += w[q] * core * _gauss(X, Y, A, C, B)
    S = np.zeros((T, T))
    S[c0 - hs:c0 + hs + 1, c0 - hs:c0 + hs + 1] = sub
    return S


def _gal(table, n, lr, e1, e2):
    from oracle.island_oracle import cov_terms
    amps, vars_, core, *_ = table.lookup(n)
    c, _ = cov_terms(lr, e1, e2)
    return amps, vars_, core, c


def _solver(psf, T, native):
    from oracle.island_oracle import IslandSolver
    s = IslandSolver.__new__(IslandSolver)
    s.isl = SimpleNamespace(psf=[psf], T=T, native=native)
    s.dt = np.float64
    return s


# free indices sit between the table's knots (at a knot the piecewise-linear
# table has no single slope, and a central difference averages the two)
CASES = [("star", None), ("exp", 1.0), ("dev", 4.0), ("sersic_0.5", 0.5137),
         ("sersic_2", 2.0719), ("sersic_6", 5.9431)]


@pytest.mark.parametrize("name,n", CASES)
def test_analytic_stamp_equals_numerical_convolution(name, n):
    from oracle.island_oracle import SersicTable, cov_terms, u_to_n
    table = SersicTable.load(TABLE)
    psf = _psf()
    T, native = 31, 31
    x, y = 281.3, 47.8                       # far from the PSF origin
    lr, e1, e2 = np.log(2.5), 0.35, -0.2
    s = _solver(psf, T, native)
    free = name.startswith("sersic")
    if n is None:
        S, Sx, Sy, _, _ = s._analytic(0, x, y, None, True)
        ref = _brute(psf, x, y, None, T, native)
    else:
        amps, vars_, core, da, dv, dcore = table.lookup(n)
        c, dc = cov_terms(lr, e1, e2)
        # a free index: n through the sigmoid of u (dn/du at that u)
        u = -np.log((6.3 - 0.29) / (n - 0.29) - 1.0) if free else 0.0
        dndu = u_to_n(u)[1] if free else 0.0
        gal = (amps, vars_, core, da, dv, dcore, dndu, c, dc)
        S, Sx, Sy, Ssh, Su = s._analytic(0, x, y, gal, True)
        ref = _brute(psf, x, y, _gal(table, n, lr, e1, e2), T, native)
    peak = np.abs(ref).max()
    assert np.abs(S - ref).max() <= 1e-9 * peak, np.abs(S - ref).max() / peak

    h = 2e-5

    def fd(fun):
        return (fun(+h) - fun(-h)) / (2 * h)

    def gal_at(nn, l_, a_, b_):
        return None if n is None else _gal(table, nn, l_, a_, b_)

    derivs = [("x", Sx, fd(lambda d: _brute(psf, x + d, y, gal_at(n, lr, e1, e2), T, native))),
              ("y", Sy, fd(lambda d: _brute(psf, x, y + d, gal_at(n, lr, e1, e2), T, native)))]
    if n is not None:
        derivs += [
            ("logre", Ssh[0], fd(lambda d: _brute(psf, x, y, _gal(table, n, lr + d, e1, e2),
                                                  T, native))),
            ("ee1", Ssh[1], fd(lambda d: _brute(psf, x, y, _gal(table, n, lr, e1 + d, e2),
                                                T, native))),
            ("ee2", Ssh[2], fd(lambda d: _brute(psf, x, y, _gal(table, n, lr, e1, e2 + d),
                                                T, native)))]
        if free:
            derivs.append(("u", Su, fd(lambda d: _brute(
                psf, x, y, _gal(table, u_to_n(u + d)[0], lr, e1, e2), T, native))))
    for what, got, want in derivs:
        scale = np.abs(want).max()
        assert scale > 0, what
        err = np.abs(got - want).max() / scale
        assert err <= 1e-6, f"{name} d/d{what}: {err:.2e} of the largest"


def test_shifted_member_stamp_is_the_lanczos_shift_of_the_convolution():
    """member_stamps: the numerical convolution at the rounded centre,
    Lanczos-3 shifted by the fractional offset (lanczos.py:50-181)."""
    from oracle.island_oracle import (SersicTable, correlate_x, correlate_y,
                                      lanczos3_taps)
    table = SersicTable.load(TABLE)
    psf = _psf()
    T, native = 31, 31
    s = _solver(psf, T, native)
    s.isl.x0, s.isl.y0 = 250.0, 20.0
    s.isl.stype = np.array([1])
    s.isl.mode = "analytic"
    s.isl.render_backend = "fft"
    s.isl.keep = np.ones((1, 6), bool)
    s.isl.free_n = np.array([False])
    s.isl.n_frozen = np.array([1.0])
    s.isl.table = table
    p = np.array([281.3, 47.8, np.log(2.5), 0.35, -0.2, 0.0])
    m, _ = s.member_stamps(0, p, 0, False)
    ref = _brute(psf, p[0], p[1], _gal(table, 1.0, p[2], p[3], p[4]), T, native)
    dx = (p[0] - s.isl.x0) - np.round(p[0] - s.isl.x0)
    dy = (p[1] - s.isl.y0) - np.round(p[1] - s.isl.y0)
    want = correlate_y(correlate_x(ref, lanczos3_taps(dx)[0]), lanczos3_taps(dy)[0])
    assert np.abs(m - want).max() <= 1e-9 * np.abs(want).max()
