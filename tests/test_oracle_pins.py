"""Pins of the CPU oracle: the reference's numpy PSF evaluation, the Sersic
table, Lanczos taps, ellipse covariance and the VarPro Jacobian (finite
differences), plus known-answer fits."""
import hashlib
from pathlib import Path

import numpy as np
import pytest

from oracle import island_oracle as O
from uniphot_b200.sersic import load_table

GOLD = Path(__file__).resolve().parent / "golden"
ROOT = Path(__file__).resolve().parents[1]
TABLE = ROOT / "uniphot_b200" / "data" / "sersic_mog_table.npz"


@pytest.mark.parametrize("nt", [1, 3, 6, 10, 15])
def test_poly_psf_matches_reference_numpy_eval(nt):
    z = np.load(GOLD / "psf_poly_eval.npz")
    coefs, xy, stamps = z[f"nt{nt}_coefs"], z[f"nt{nt}_xy"], z[f"nt{nt}_stamps"]
    psf = O.PolyPsfBand(coefs, 1000.0, 900.0, 700.0, 650.0)
    for (x, y), ref in zip(xy, stamps):
        S, _, _, _ = psf.stamp(x, y, np.float64)
        np.testing.assert_allclose(S, ref, rtol=2e-5, atol=2e-5 * np.abs(ref).max())


def test_sersic_table_identical_to_reference():
    z = np.load(GOLD / "sersic_table_ref.npz")
    t = load_table()
    for k in ("n_knots", "amps", "log_vars", "core_amp"):
        a = np.ascontiguousarray(np.asarray(t[k], np.float64))
        assert hashlib.sha256(a.tobytes()).hexdigest() == str(z[f"{k}_sha256"])
        np.testing.assert_array_equal(a[z["rows"]], z[f"{k}_rows"])
    assert float(t["n_min"]) == float(z["n_min"]) and float(t["n_max"]) == float(z["n_max"])


def test_table_lookup_at_knots_returns_stored_rows():
    tb = O.SersicTable.load(TABLE)
    for i in (10, 148, 600, 1100):
        n = tb.n_knots[i]
        if tb.n_knots[i + 1] == n:       # duplicated boundary knot
            continue
        a, v, core, *_ = tb.lookup(n)
        j = int(np.searchsorted(tb.n_knots, n, side="right")) - 1
        np.testing.assert_allclose(a, tb.amps[j], rtol=1e-12)
        np.testing.assert_allclose(v, np.exp(tb.log_vars[j]), rtol=1e-12)


def test_lanczos_zero_shift_is_identity():
    L, dL = O.lanczos3_taps(0.0)
    np.testing.assert_allclose(L, [0, 0, 0, 1, 0, 0, 0], atol=1e-15)
    img = np.random.default_rng(0).normal(size=(9, 11))
    np.testing.assert_allclose(O.correlate_y(O.correlate_x(img, L), L), img, atol=1e-14)


@pytest.mark.parametrize("d", [-0.49, -0.2, 0.13, 0.37])
def test_lanczos_taps_normalised_and_derivative(d):
    L, dL = O.lanczos3_taps(d)
    assert abs(L.sum() - 1.0) < 1e-14 and abs(dL.sum()) < 1e-12
    h = 1e-6
    num = (O.lanczos3_taps(d + h)[0] - O.lanczos3_taps(d - h)[0]) / (2 * h)
    np.testing.assert_allclose(dL, num, atol=1e-7)


@pytest.mark.parametrize("p", [(0.3, 0.2, -0.1), (1.2, -0.5, 0.4), (-0.7, 1e-3, 2.0)])
def test_cov_terms_derivative(p):
    c, dc = O.cov_terms(*p)
    h = 1e-6
    for s in range(3):
        q1 = list(p)
        q2 = list(p)
        q1[s] += h
        q2[s] -= h
        num = (O.cov_terms(*q1)[0] - O.cov_terms(*q2)[0]) / (2 * h)
        np.testing.assert_allclose(dc[s], num, rtol=1e-5, atol=1e-8)


def test_cov_terms_round_source_nudge():
    """ee1 = ee2 = 0 is evaluated at ee1 = 1e-4 with a zero ee1 derivative
    (sersic_mog.py:135-136): finite, and identical to the nudged point."""
    c0, dc0 = O.cov_terms(0.5, 0.0, 0.0)
    c1, _ = O.cov_terms(0.5, 1e-4, 0.0)
    np.testing.assert_array_equal(c0, c1)
    np.testing.assert_array_equal(dc0[1], 0.0)
    assert np.all(np.isfinite(dc0))


def _mini_island(mode, n_src=2, seed=0, gal=True, B=32, T=31, nb=2, noise=True):
    """A small synthetic island for known-answer and Jacobian tests."""
    from uniphot_b200.psf import MogPsf, rasterize_mog_psf
    rng = np.random.default_rng(seed)
    mog = MogPsf(np.array([[1.3, 0.05, 0.0], [2.4, 0.0, 0.1]]),
                 np.array([[0.05, 0.01, 0.0], [-0.02, 0.0, 0.01]]),
                 np.array([[0.02, 0.0, 0.0], [0.0, 0.01, 0.0]]),
                 np.array([[0.8, 0.0, 0.0], [0.2, 0.0, 0.0]]), 100.0, 100.0, 100.0, 100.0)
    if mode == "analytic":
        psf = [O.MogPsfBand(mog.sigma, mog.e1, mog.e2, mog.weight, 100.0, 100.0,
                            100.0, 100.0) for _ in range(nb)]
    else:
        p = rasterize_mog_psf(mog, T, 100.0, 100.0)
        psf = [O.PolyPsfBand(p.coefs, 100.0, 100.0, 100.0, 100.0) for _ in range(nb)]
    N = n_src
    x0 = y0 = 84.0
    xs = x0 + B / 2 + rng.uniform(-4, 4, N)
    ys = y0 + B / 2 + rng.uniform(-4, 4, N)
    stype = np.zeros(N, np.int32)
    if gal and mode == "analytic":
        stype[-1] = 3
    keep = np.zeros((N, 6), bool)
    keep[:, :2] = True
    keep[stype != 0, 2:5] = True
    keep[stype == 3, 5] = True
    p0 = np.zeros((N, 6), np.float32)
    p0[:, 0], p0[:, 1] = xs, ys
    p0[:, 2] = 0.6
    p0[:, 3], p0[:, 4] = 0.2, -0.1
    p0[:, 5] = -0.5
    isl = O.IslandInput(
        B=B, T=T, data=np.zeros((nb, B, B), np.float32),
        w=np.full((nb, B, B), 0.01, np.float32), x0=x0, y0=y0, stype=stype,
        n_frozen=np.ones(N, np.float32), free_n=(stype == 3), mmask=np.ones(N, bool),
        keep=keep, p0=p0.reshape(-1), lower=(p0 - 5).reshape(-1),
        upper=(p0 + 5).reshape(-1), prior_mean=p0.reshape(-1),
        prior_inv_sigma=np.zeros(6 * N, np.float32), has_priors=False, psf=psf,
        table=O.SersicTable.load(TABLE), mode=mode, native=T)
    cfg = O.SolverConfig(precision="f64")
    s = O.IslandSolver(isl, cfg)
    flux = rng.uniform(2e3, 2e4, (nb, N))
    for b in range(nb):
        M, _ = s.models_band(b, isl.p0.astype(np.float64), False)
        isl.data[b] = np.tensordot(flux[b], M, axes=(0, 0)).astype(np.float32)
        if noise:
            isl.data[b] += rng.normal(0, 10.0, (B, B)).astype(np.float32)
    return isl, flux


@pytest.mark.parametrize("mode", ["reference", "analytic"])
def test_noise_free_fit_recovers_truth(mode):
    isl, flux = _mini_island(mode, n_src=2, noise=False)
    truth = isl.p0.copy()
    isl.p0 = truth + np.tile(np.array([0.2, -0.15, 0, 0, 0, 0], np.float32), 2)
    out = O.solve_island(isl, O.SolverConfig(precision="f64"), max_steps=30)
    np.testing.assert_allclose(out["p"].reshape(-1)[[0, 1, 6, 7]],
                               truth[[0, 1, 6, 7]], atol=2e-3)
    np.testing.assert_allclose(out["fluxes"], flux, rtol=2e-3)


@pytest.mark.parametrize("mode", ["reference", "analytic"])
def test_varpro_jacobian_matches_finite_differences(mode):
    isl, _ = _mini_island(mode, n_src=2)
    s = O.IslandSolver(isl, O.SolverConfig(precision="f64"))
    p = isl.p0.astype(np.float64)

    def resid(q, b):
        M, _ = s.models_band(b, q, False)
        f, _, _ = s.fluxes_band(M, isl.data[b], isl.w[b])
        _, r = s.chi2_band(M, isl.data[b], isl.w[b], f)
        return r.reshape(-1)
    live = [j for j in range(p.size) if isl.keep.reshape(-1)[j]]
    H, g = s.hg(p)
    Jn = []
    for j in live:
        h = 1e-5 if (j % 6) < 2 else 1e-5
        q1, q2 = p.copy(), p.copy()
        q1[j] += h
        q2[j] -= h
        Jn.append(np.concatenate([(resid(q1, b) - resid(q2, b)) / (2 * h)
                                  for b in range(isl.data.shape[0])]))
    Jn = np.array(Jn)
    r = np.concatenate([resid(p, b) for b in range(isl.data.shape[0])])
    Hn = Jn @ Jn.T
    gn = Jn @ r
    idx = np.array(live)
    np.testing.assert_allclose(H[np.ix_(idx, idx)], Hn, rtol=2e-4,
                               atol=2e-4 * np.abs(Hn).max())
    np.testing.assert_allclose(g[idx], gn, rtol=2e-3, atol=2e-4 * np.abs(gn).max())


def test_two_source_blend_flux_solve_is_normal_equations():
    isl, flux = _mini_island("analytic", n_src=2, gal=False, noise=False)
    s = O.IslandSolver(isl, O.SolverConfig(precision="f64"))
    M, _ = s.models_band(0, isl.p0.astype(np.float64), False)
    f, f64, A64 = s.fluxes_band(M, isl.data[0], isl.w[0])
    Mm = M.reshape(2, -1).astype(np.float64)
    w = isl.w[0].reshape(-1).astype(np.float64)
    A = (Mm * w) @ Mm.T + 1e-9 * np.eye(2)
    b = (Mm * w) @ isl.data[0].reshape(-1).astype(np.float64)
    np.testing.assert_allclose(f64, np.linalg.solve(A, b), rtol=1e-10)
    np.testing.assert_allclose(f64, flux[0], rtol=1e-5)


def test_stall_sets_probes():
    """A zero-weight island never improves: 4 rejects -> stalled, and the
    frozen proposals are identical (diverged)."""
    isl, _ = _mini_island("analytic", n_src=1, gal=False, noise=False)
    isl.w[:] = 0.0
    out = O.solve_island(isl, O.SolverConfig(precision="ref"), max_steps=30)
    assert out["stall"] and out["conv"] and out["nst"] == 4
    assert np.isfinite(out["stall_dchi2"])


def _with_plane(isl, coefs):
    """Add a known plane c0 + c1 X + c2 Y (window-normalised) per band."""
    isl.bg_joint = True
    s = O.IslandSolver(isl, O.SolverConfig(precision="f64"))
    P = s.bg_basis().astype(np.float64)
    for b in range(isl.data.shape[0]):
        isl.data[b] += np.tensordot(coefs[b], P, axes=(0, 0)).astype(np.float32)
    return isl


@pytest.mark.parametrize("mode", ["reference", "analytic"])
def test_joint_background_noise_free_recovers_fluxes_and_plane(mode):
    """Fluxes and a planar background solved together recover both exactly
    on noise-free data (forced_phot_sparse.py:417-497 semantics)."""
    isl, flux = _mini_island(mode, n_src=2, noise=False)
    coefs = np.array([[30.0, 4.0, -2.5], [12.0, -1.0, 3.0]])
    isl = _with_plane(isl, coefs)
    truth = isl.p0.copy()
    isl.p0 = truth + np.tile(np.array([0.2, -0.15, 0, 0, 0, 0], np.float32), 2)
    out = O.solve_island(isl, O.SolverConfig(precision="f64"), max_steps=30)
    np.testing.assert_allclose(out["p"].reshape(-1)[[0, 1, 6, 7]],
                               truth[[0, 1, 6, 7]], atol=2e-3)
    np.testing.assert_allclose(out["fluxes"], flux, rtol=2e-3)
    np.testing.assert_allclose(out["bg"], coefs, rtol=2e-3, atol=2e-2)


def test_joint_background_jacobian_matches_finite_differences():
    isl, _ = _mini_island("analytic", n_src=2)
    isl = _with_plane(isl, np.array([[20.0, 3.0, 1.0], [5.0, 0.5, -2.0]]))
    s = O.IslandSolver(isl, O.SolverConfig(precision="f64"))
    p = isl.p0.astype(np.float64)

    def resid(q, b):
        M, _ = s.models_band(b, q, False)
        f, _, _ = s.fluxes_band(M, isl.data[b], isl.w[b])
        _, r = s.chi2_band(M, isl.data[b], isl.w[b], f)
        return r.reshape(-1)
    live = [j for j in range(p.size) if isl.keep.reshape(-1)[j]]
    H, g = s.hg(p)
    Jn = []
    for j in live:
        q1, q2 = p.copy(), p.copy()
        q1[j] += 1e-5
        q2[j] -= 1e-5
        Jn.append(np.concatenate([(resid(q1, b) - resid(q2, b)) / 2e-5
                                  for b in range(isl.data.shape[0])]))
    Jn = np.array(Jn)
    r = np.concatenate([resid(p, b) for b in range(isl.data.shape[0])])
    idx = np.array(live)
    Hn = Jn @ Jn.T
    np.testing.assert_allclose(H[np.ix_(idx, idx)], Hn, rtol=2e-4,
                               atol=2e-4 * np.abs(Hn).max())
    gn = Jn @ r
    np.testing.assert_allclose(g[idx], gn, rtol=2e-3, atol=2e-4 * np.abs(gn).max())


def test_changed_mode_zero_weight_island_runs_out_diverged():
    """stall_count_mode='changed' (island_solver.py:1118-1208): a zero-
    weight island proposes the same step at every escalating damping, so
    the identical rejects never count toward the stall; the loop runs to
    max_steps and the sticky diverged flag is set."""
    isl, _ = _mini_island("analytic", n_src=1, gal=False, noise=False)
    isl.w[:] = 0.0
    out = O.solve_island(isl, O.SolverConfig(precision="ref", stall_count_mode="changed"),
                         max_steps=12)
    assert not out["stall"] and not out["conv"] and out["nst"] == 12
    assert out["diverged"] and out["n_same"] == 12 and out["nrej"] == 1


def test_changed_mode_matches_legacy_when_no_repeats():
    isl, _ = _mini_island("analytic", n_src=2, seed=3)
    a = O.solve_island(isl, O.SolverConfig(precision="ref"), max_steps=30)
    b = O.solve_island(isl, O.SolverConfig(precision="ref", stall_count_mode="changed"),
                       max_steps=30)
    assert a["nst"] == b["nst"] and a["conv"] == b["conv"]
    np.testing.assert_array_equal(a["p"], b["p"])


def test_dlnp_zero_weight_island_exits_at_once_and_certifies():
    """convergence='dlnp' (island_solver.py:1210-1333): a no-move proposal
    is a terminal reject-exit; the plateau certificate (dchi2 = 0 >
    -quantum) maps it to converged-on-plateau."""
    isl, _ = _mini_island("analytic", n_src=1, gal=False, noise=False)
    isl.w[:] = 0.0
    out = O.solve_island(isl, O.SolverConfig(precision="ref", convergence="dlnp"),
                         max_steps=30)
    assert out["nst"] == 1 and out["conv"] and not out["stall"]
    assert out["stall_dchi2"] == 0.0


def test_dlnp_converges_on_a_blend():
    isl, flux = _mini_island("analytic", n_src=2, seed=4)
    out = O.solve_island(isl, O.SolverConfig(precision="ref", convergence="dlnp"),
                         max_steps=30)
    assert out["conv"] and not out["stall"]
    np.testing.assert_allclose(out["fluxes"], flux, rtol=0.05)


def _tr_setup(seed=5):
    isl, flux = _mini_island("analytic", n_src=2, seed=seed)
    s = O.IslandSolver(isl, O.SolverConfig(precision="f64", step_mode="trust_region"))
    p = isl.p0.astype(np.float64)
    H, g = s.hg(p)
    return isl, s, p, H, g, s._keep(0)


def test_trust_region_first_step_is_gauss_newton():
    """An unset radius (0) is seeded with the scaled Gauss-Newton step's
    length, so the first proposal is the Gauss-Newton step
    (island_solver.py:1040-1044)."""
    isl, s, p, H, g, keep = _tr_setup()
    pt, pred, Dr, Dmax, at_bnd = s.propose_tr(p, H, g, 0.0, keep)
    Hm = np.where(keep[:, None] & keep[None, :], H, 0) + np.diag(np.where(keep, 0, 1.0))
    Hm = Hm + 1e-8 * np.eye(p.size)
    gn = -np.linalg.solve(Hm, np.where(keep, g, 0))
    np.testing.assert_allclose(pt - p, gn, rtol=1e-9, atol=1e-12)
    dsc = np.sqrt(np.diag(Hm))
    assert abs(Dr - np.linalg.norm(dsc * gn)) <= 1e-12 * Dr
    assert at_bnd and pred > 0 and Dmax > Dr


def test_trust_region_dogleg_respects_the_radius():
    """A radius below the Cauchy point's length scales the steepest-descent
    step to the boundary; one between it and the Gauss-Newton length takes
    the dogleg blend, again on the boundary |D delta| = Dr."""
    isl, s, p, H, g, keep = _tr_setup()
    _, _, D0, _, _ = s.propose_tr(p, H, g, 0.0, keep)
    Hm = np.where(keep[:, None] & keep[None, :], H, 0) + np.diag(np.where(keep, 0, 1.0))
    dsc = np.sqrt(np.diag(Hm + 1e-8 * np.eye(p.size)))
    gh = np.where(keep, g, 0) / dsc
    for frac in (1e-4, 0.5):
        Dr = frac * D0
        pt, pred, Dr_used, _, at_bnd = s.propose_tr(p, H, g, Dr, keep)
        step = dsc * (pt - p)
        assert Dr_used == Dr and at_bnd and pred > 0
        np.testing.assert_allclose(np.linalg.norm(step), Dr, rtol=1e-9)
        if frac == 1e-4:    # pure (scaled) steepest descent direction
            np.testing.assert_allclose(step / Dr, -gh / np.linalg.norm(gh), atol=1e-9)


def test_trust_region_solve_converges_and_matches_clip():
    isl, flux = _mini_island("analytic", n_src=2, seed=4)
    a = O.solve_island(isl, O.SolverConfig(precision="f64"), max_steps=30)
    b = O.solve_island(isl, O.SolverConfig(precision="f64", step_mode="trust_region"),
                       max_steps=30)
    assert b["conv"] and not b["stall"] and not b["railed"]
    assert b["lam"] > 0
    np.testing.assert_allclose(b["fluxes"], a["fluxes"], rtol=1e-3)
    np.testing.assert_allclose(b["p"][:, :2], a["p"][:, :2], atol=1e-2)


def test_trust_region_railed_flags_a_pinned_bound():
    """The bound-pinned disclosure (island_solver.py:1717-1728) is set when
    a kept parameter ends at its box bound."""
    isl, _ = _mini_island("analytic", n_src=2, seed=4)
    isl.upper = isl.upper.copy()
    isl.upper[8] = isl.p0[8]          # member 1's log-radius pinned at its seed
    out = O.solve_island(isl, O.SolverConfig(precision="ref", step_mode="trust_region"),
                         max_steps=30)
    assert out["railed"]
    out = O.solve_island(isl, O.SolverConfig(precision="ref"), max_steps=30)
    assert not out["railed"]      # clip mode reports none


def test_final_errors_of_a_star_match_the_projected_fisher_matrix():
    """Known answer for the covariance (island_solver.py:1484-1547): for a
    noise-free isolated star the (x, y) block is the inverse of
    sum_b w f_b^2 (D^T D - D^T m (m^T m)^-1 m^T D), D the unit model's
    position derivatives (flux marginalised by the projection)."""
    isl, flux = _mini_island("analytic", n_src=1, gal=False, noise=False)
    s = O.IslandSolver(isl, O.SolverConfig(precision="f64"))
    p = isl.p0.astype(np.float64)
    pe = s.final_errors(p)
    F = np.zeros((2, 2))
    for b in range(isl.data.shape[0]):
        m = s.models_band(b, p, False)[0][0].astype(np.float64).reshape(-1)
        D = []
        for j in range(2):
            h = 1e-4
            q1, q2 = p.copy(), p.copy()
            q1[j] += h
            q2[j] -= h
            D.append((s.models_band(b, q1, False)[0][0].astype(np.float64)
                      - s.models_band(b, q2, False)[0][0].astype(np.float64)).reshape(-1)
                     / (2 * h))
        D = np.array(D).T
        w = float(isl.w[b, 0, 0])
        P = D.T @ D - np.outer(D.T @ m, D.T @ m) / (m @ m)
        F += w * flux[b, 0] ** 2 * P
    np.testing.assert_allclose(pe[0, :2], np.diag(np.linalg.inv(F)), rtol=1e-4)
    np.testing.assert_array_equal(pe[0, 2:6], 1.0)     # frozen slots: unit rows
    assert pe[0, 6] == 0.0 and np.all(np.isnan(pe[0, 7:]))


def test_flux_sensitivities_match_finite_differences():
    """The Golub-Pereyra flux sensitivities c_j = A^-1 (e_k s_j - f_k u_j)
    that the Jacobian assembly and the marginalised flux error use are the
    derivatives of the flux solution (island_solver.py:570-590, 1549-1613)."""
    isl, _ = _mini_island("analytic", n_src=2, seed=6)
    s = O.IslandSolver(isl, O.SolverConfig(precision="f64"))
    p = isl.p0.astype(np.float64)
    fj = {}
    s.hg(p, fj)
    for b, (idx, C) in fj.items():
        for r, q in enumerate(idx):
            h = 1e-5
            q1, q2 = p.copy(), p.copy()
            q1[q] += h
            q2[q] -= h
            f1 = s.fluxes_band(s.models_band(b, q1, False)[0], isl.data[b], isl.w[b])[1]
            f2 = s.fluxes_band(s.models_band(b, q2, False)[0], isl.data[b], isl.w[b])[1]
            fd = (f1 - f2) / (2 * h)
            np.testing.assert_allclose(C[r], fd, rtol=2e-4, atol=1e-6 * np.abs(fd).max())


def test_flux_marg_is_zero_for_stars_and_the_quadratic_form_for_galaxies():
    isl, _ = _mini_island("analytic", n_src=2, seed=6)      # member 1 is a galaxy
    s = O.IslandSolver(isl, O.SolverConfig(precision="f64"))
    p = isl.p0.astype(np.float64)
    dv = s.final_flux_marg(p)
    assert dv.shape == (2, 2) and np.all(dv[:, 0] == 0.0) and np.all(dv[:, 1] > 0)
    fj = {}
    _, keep, Hm, _ = s._posterior(p, fj)
    S = np.linalg.inv(Hm.astype(np.float64))
    idx, C = fj[0]
    cols = [r for r, q in enumerate(idx) if q >= 6]          # the galaxy's parameters
    J = C[cols, 1]
    q = idx[cols]
    np.testing.assert_allclose(dv[0, 1], J @ S[np.ix_(q, q)] @ J, rtol=1e-5)


def test_source_metrics_known_answers():
    """Source metrics (island_solver.py:1639-1715): an isolated noise-free
    star has no neighbour light, no masked flux and zero chi2; masking a
    half-plane gives the unit model's flux there; a blend's fracflux is the
    neighbour's light under the member's profile."""
    isl, flux = _mini_island("analytic", n_src=1, gal=False, noise=False)
    s = O.IslandSolver(isl, O.SolverConfig(precision="f64"))
    p = isl.p0.astype(np.float64)
    met, fwin = s.source_metrics(p)
    m = s.models_band(0, p, False)[0][0].astype(np.float64)
    assert met[0, 1] == 0.0 and met[0, 3] == 0.0 and abs(met[0, 0]) < 1e-6
    np.testing.assert_allclose(met[0, 2], m.sum(), rtol=1e-6)
    np.testing.assert_allclose(fwin[:, 0], flux[:, 0] * m.sum(), rtol=1e-4)
    isl.w[:, :, :16] = 0.0
    met, _ = s.source_metrics(p)
    np.testing.assert_allclose(met[0, 3], m[:, :16].sum() / 1.0, rtol=1e-4)
    isl2, flux2 = _mini_island("analytic", n_src=2, gal=False, noise=False, seed=7)
    s2 = O.IslandSolver(isl2, O.SolverConfig(precision="f64"))
    p2 = isl2.p0.astype(np.float64)
    met2, _ = s2.source_metrics(p2)
    num = den = 0.0
    for b in range(2):
        M = s2.models_band(b, p2, False)[0].astype(np.float64)
        f = s2.fluxes_band(M, isl2.data[b], isl2.w[b])[0].astype(np.float64)
        own, other = f[0] * M[0], f[1] * M[1]
        fin = min(max(M[0].sum(), 0.0), 1.0)
        num += fin * (other * own).sum() / (own * own).sum()
        den += fin
    np.testing.assert_allclose(met2[0, 1], num / den, rtol=1e-5)


def test_re_profile_and_residual_known_answers():
    """Re profile (island_solver.py:1779-1792): 0 for a star slot, a
    positive bowl around a galaxy's converged log-radius; the band-coadded
    residual (:1615-1637) of a noise-free fit at the truth is ~0 and its
    weight is the band sum of w."""
    isl, flux = _mini_island("analytic", n_src=2, seed=8, noise=False)
    s = O.IslandSolver(isl, O.SolverConfig(precision="f64"))
    p = isl.p0.astype(np.float64)
    from uniphot_b200.plan import REPROF_DELTAS_LN
    prof = s.re_profile(p, REPROF_DELTAS_LN)
    assert np.all(prof[0] == 0.0)
    assert np.all(prof[1] > 0) and prof[1, 0] > prof[1, 5] and prof[1, -1] > prof[1, 6]
    R, W = s.residual_coadd(p)
    np.testing.assert_allclose(W, isl.w.sum(axis=0), rtol=1e-6)
    assert np.abs(R).max() <= 1e-3 * np.abs(isl.w * isl.data).sum(axis=0).max()


def test_re_profile_interval_interpolates_the_unit_crossing():
    """island_plan.py:913-952: the interval ends where the profile first
    reaches 1 on each side, linearly interpolated; a side that never does
    ends at its outermost offset."""
    from uniphot_b200.plan import REPROF_DELTAS_LN, re_profile_interval
    d = REPROF_DELTAS_LN.astype(np.float64)
    sig = 0.3
    prof = np.zeros((1, 2, d.size), np.float32)
    prof[0, 0] = (d / sig) ** 2
    prof[0, 0, d < 0] = 0.5               # never reaches 1 on the left
    res_p = np.zeros((1, 2, 6), np.float32)
    res_p[0, 0, 2] = np.log(4.0)
    is_ext = np.array([[True, False]])
    lo, hi = re_profile_interval(res_p, prof, d, np.array([0, 0]), np.array([0, 1]), is_ext)
    p0, p1 = (0.25 / sig) ** 2, (0.5 / sig) ** 2
    cross = 0.25 + (1 - p0) / (p1 - p0) * 0.25
    np.testing.assert_allclose(hi[0], 4.0 * np.exp(cross), rtol=1e-6)
    np.testing.assert_allclose(lo[0], 4.0 * np.exp(-2.5), rtol=1e-6)
    assert np.isnan(lo[1]) and np.isnan(hi[1])
