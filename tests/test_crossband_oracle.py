"""CPU pins of the oracle's cross-band GLS restatement
(tract7dt/fit/grid_gpu/island_solver.py:607-723, 867-919).

The reference has no tests or golden vectors for this mode, so the pins
are the identity its comments state: with flat whitened residuals r_b and
an ambient covariance C = I + V V^T, V[(b, .), (i, .)] = s_bi Q_b (Q_b the
circular convolution by the band PSF placed in the B x B window), the GLS
chi2 r^T C^-1 r equals the per-band chi2 minus (1/B^2) sum_k z^H M^-1 z, and
the Gauss-Newton system is J^T C^-1 J, J^T C^-1 r.  The tests build C
densely on small windows and compare.
"""

import numpy as np
import pytest

from oracle import island_oracle as O
from tests.test_oracle_pins import _mini_island


def _conv_matrix(z):
    """Dense circular convolution by the B x B image z (acting on flattened
    B x B images)."""
    B = z.shape[0]
    cols = []
    for e in range(B * B):
        y = np.zeros(B * B)
        y[e] = 1.0
        cols.append(np.fft.irfft2(np.fft.rfft2(z) * np.fft.rfft2(y.reshape(B, B)),
                                  s=(B, B)).reshape(-1))
    return np.stack(cols, axis=1)


def _dense_V(zs, s_b):
    nb, r = s_b.shape
    B2 = zs[0].size
    V = np.zeros((nb * B2, r * B2))
    for b in range(nb):
        Q = _conv_matrix(zs[b])
        for i in range(r):
            V[b * B2:(b + 1) * B2, i * B2:(i + 1) * B2] = s_b[b, i] * Q
    return V


def _cinv(V, X):
    """C^-1 X with C = I + V V^T, by Woodbury on the small side."""
    K = np.eye(V.shape[1]) + V.T @ V
    return X - V @ np.linalg.solve(K, V.T @ X)


@pytest.mark.parametrize("B", [8, 9])
def test_woodbury_correction_equals_dense_gls(B):
    rng = np.random.default_rng(B)
    nb, r_ = 3, 2
    zs = [rng.normal(size=(B, B)) for _ in range(nb)]
    s_b = rng.normal(size=(nb, r_))
    resids = [rng.normal(size=(B, B)) for _ in range(nb)]
    s = O.IslandSolver.__new__(O.IslandSolver)
    s.isl = type("I", (), {"B": B})()
    q = np.stack([np.fft.rfft2(z) for z in zs])
    wk = np.full((B, B // 2 + 1), 2.0)
    wk[:, 0] = 1.0
    if B % 2 == 0:
        wk[:, -1] = 1.0
    corr, _, _ = s._cb_chi2_corr(resids, q, s_b, wk)
    rv = np.concatenate([x.reshape(-1) for x in resids])
    V = _dense_V(zs, s_b)
    dense = float(rv @ rv - rv @ _cinv(V, rv))
    assert corr == pytest.approx(dense, rel=1e-10)
    assert corr > 0.0


def _cb_island(rank=2, lam=(400.0, 90.0), cb_scale=0.7, seed=3, B=16, T=15):
    isl, flux = _mini_island("reference", n_src=2, seed=seed, B=B, T=T, nb=3)
    rng = np.random.default_rng(seed + 11)
    u = rng.normal(size=(rank, 3))
    u /= np.linalg.norm(u, axis=1, keepdims=True)
    isl.crossband = {"rank": rank, "u": u, "lam": np.asarray(lam[:rank])}
    isl.cb_scale = cb_scale
    return isl, flux


def test_filters_place_the_psf_at_the_member_mean():
    isl, _ = _cb_island()
    s = O.IslandSolver(isl, O.SolverConfig(precision="f64"))
    p = isl.p0.astype(np.float64)
    q, s_b, wk = s._cb_filters(p)
    pp = p.reshape(-1, 6)
    cx, cy = pp[:, 0].mean(), pp[:, 1].mean()
    st = isl.psf[1].stamp(cx, cy, np.float64)[0]
    z = np.zeros((isl.B, isl.B))
    z[:isl.T, :isl.T] = st
    np.testing.assert_allclose(q[1], np.fft.rfft2(z), rtol=1e-5, atol=1e-7)
    u = isl.crossband["u"]
    lam = isl.crossband["lam"]
    np.testing.assert_allclose(s_b, (np.sqrt(lam) * np.sqrt(0.7))[None, :] * u.T)
    assert wk[0, 0] == 1.0 and wk[0, 1] == 2.0 and wk[0, -1] == 1.0


def test_filters_crop_the_centre_when_the_tier_exceeds_the_window():
    isl, _ = _cb_island()
    s = O.IslandSolver(isl, O.SolverConfig(precision="f64"))
    isl.T = 21                                  # only the filter reads T here
    psf = isl.psf[0]
    big = O.PolyPsfBand(np.pad(psf.coefs, ((3, 3), (3, 3), (0, 0))), psf.x_origin,
                        psf.x_scale, psf.y_origin, psf.y_scale)
    isl.psf = [big] * 3
    p = isl.p0.astype(np.float64)
    q, _, _ = s._cb_filters(p)
    pp = p.reshape(-1, 6)
    st = big.stamp(pp[:, 0].mean(), pp[:, 1].mean(), np.float64)[0]
    np.testing.assert_allclose(q[0], np.fft.rfft2(st[2:18, 2:18]), rtol=1e-5, atol=1e-7)


def test_analytic_mode_rejects_crossband():
    isl, _ = _mini_island("analytic", n_src=1, gal=False)
    isl.crossband = {"rank": 1, "u": np.ones((1, 2)), "lam": np.ones(1)}
    s = O.IslandSolver(isl, O.SolverConfig(precision="f64"))
    with pytest.raises(ValueError):
        s.chi2_of(isl.p0.astype(np.float64))


def _resid_all(s, isl, p):
    out = []
    for b in range(isl.data.shape[0]):
        M, _ = s.models_band(b, p, False)
        f, _, _ = s.fluxes_band(M, isl.data[b], isl.w[b])
        _, r = s.chi2_band(M, isl.data[b], isl.w[b], f)
        out.append(r.reshape(-1).astype(np.float64))
    return np.concatenate(out)


def _dense_of(s, isl, p):
    q, s_b, _ = s._cb_filters(p)
    zs = [np.fft.irfft2(qb, s=(isl.B, isl.B)) for qb in q]
    return _dense_V(zs, s_b)


def test_chi2_is_the_dense_gls_form():
    isl, _ = _cb_island()
    s = O.IslandSolver(isl, O.SolverConfig(precision="f64"))
    p = isl.p0.astype(np.float64) + 0.05
    rv = _resid_all(s, isl, p)
    V = _dense_of(s, isl, p)
    gls = float(rv @ _cinv(V, rv))
    assert float(s.chi2_of(p)) == pytest.approx(gls, rel=1e-9)
    assert float(s.chi2_of64(p)) == pytest.approx(gls, rel=1e-9)
    plain = float(rv @ rv)
    assert gls < plain


def test_gauss_newton_system_is_the_dense_gls_form():
    """H = J^T C^-1 J and g = J^T C^-1 r with C at the current filters (the
    filters' own dependence on the positions is left out, as in the
    reference)."""
    isl, _ = _cb_island()
    s = O.IslandSolver(isl, O.SolverConfig(precision="f64"))
    p = isl.p0.astype(np.float64) + 0.05
    live = [j for j in range(p.size) if isl.keep.reshape(-1)[j]]
    Jn = []
    for j in live:
        h = 1e-5
        q1, q2 = p.copy(), p.copy()
        q1[j] += h
        q2[j] -= h
        Jn.append((_resid_all(s, isl, q1) - _resid_all(s, isl, q2)) / (2 * h))
    Jn = np.array(Jn)
    rv = _resid_all(s, isl, p)
    V = _dense_of(s, isl, p)
    CJ = _cinv(V, Jn.T)
    Hn = Jn @ CJ
    gn = CJ.T @ rv
    H, g = s.hg(p)
    idx = np.array(live)
    np.testing.assert_allclose(H[np.ix_(idx, idx)], Hn, rtol=2e-4,
                               atol=2e-4 * np.abs(Hn).max())
    np.testing.assert_allclose(g[idx], gn, rtol=2e-3, atol=2e-4 * np.abs(gn).max())


def test_zero_scale_reduces_to_the_band_solve():
    isl, _ = _cb_island(cb_scale=0.0)
    s = O.IslandSolver(isl, O.SolverConfig(precision="f64"))
    p = isl.p0.astype(np.float64) + 0.05
    H, g = s.hg(p)
    c = s.chi2_of(p)
    isl.crossband = None
    H0, g0 = s.hg(p)
    np.testing.assert_allclose(H, H0, rtol=1e-12, atol=1e-12 * np.abs(H0).max())
    np.testing.assert_allclose(g, g0, rtol=1e-12, atol=1e-12 * np.abs(g0).max())
    assert float(c) == pytest.approx(float(s.chi2_of(p)), rel=1e-12)


def test_noise_free_gls_fit_recovers_truth():
    isl, flux = _cb_island()
    isl.data[:] = 0.0
    s = O.IslandSolver(isl, O.SolverConfig(precision="f64"))
    truth = isl.p0.astype(np.float64)
    for b in range(3):
        M, _ = s.models_band(b, truth, False)
        isl.data[b] = np.tensordot(flux[b], M, axes=(0, 0)).astype(np.float32)
    isl.p0 = (truth + np.tile([0.2, -0.15, 0, 0, 0, 0], 2)).astype(np.float32)
    out = O.solve_island(isl, O.SolverConfig(precision="f64"), max_steps=30)
    np.testing.assert_allclose(out["p"].reshape(-1)[[0, 1, 6, 7]],
                               truth[[0, 1, 6, 7]], atol=2e-3)
    np.testing.assert_allclose(out["fluxes"], flux, rtol=2e-3)
