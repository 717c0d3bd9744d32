"""Per-grid sparse forced photometry, host side and oracle
(forced_phot_sparse.py): the background basis against the reference's own
``make_bg_basis`` (golden fixture), the neighbour list against a brute-force
predicate, and the oracle's solve on noise-free known answers."""
from pathlib import Path

import numpy as np
import pytest

from uniphot_b200.sparse import build_neighbor_list, make_bg_basis, stamp_top_left

GOLD = Path(__file__).resolve().parent / "golden" / "bg_basis_ref.npz"


def test_bg_basis_matches_the_reference_bit_for_bit():
    g = np.load(GOLD)
    for ci in range(3):
        h, w, x0, y0, xo, xs, yo, ys = g[f"case{ci}_geom"]
        for order in (0, 1, 2):
            got = make_bg_basis(int(h), int(w), int(x0), int(y0), xo, xs, yo, ys, order)
            np.testing.assert_array_equal(got, g[f"case{ci}_o{order}"])


def test_neighbor_list_is_the_stamp_overlap_predicate():
    rng = np.random.default_rng(0)
    x = rng.uniform(0, 200, 120)
    y = rng.uniform(0, 200, 120)
    idx, mask = build_neighbor_list(x, y, 21, 25, k_max=64)
    for s in range(x.size):
        want = {t for t in range(x.size) if t != s and abs(x[t] - x[s]) < 25
                and abs(y[t] - y[s]) < 21}
        assert set(idx[s][mask[s]].tolist()) == want
    # truncation keeps the k_max closest
    idx2, mask2 = build_neighbor_list(x, y, 21, 25, k_max=3)
    for s in range(x.size):
        full = idx[s][mask[s]]
        if full.size > 3:
            d2 = (x[full] - x[s]) ** 2 + (y[full] - y[s]) ** 2
            assert set(idx2[s][mask2[s]].tolist()) == set(full[np.argsort(d2)[:3]].tolist())


def test_stamp_top_left_rounds_half_to_even():
    ix, iy = stamp_top_left(np.array([10.5, 11.5, 3.2]), np.array([0.5, 1.5, 7.7]), 0, 0, 5, 7)
    np.testing.assert_array_equal(ix, [10 - 3, 12 - 3, 3 - 3])
    np.testing.assert_array_equal(iy, [0 - 2, 2 - 2, 8 - 2])


def _grid(seed=0, n=12, order=1, h=64, w=72, noise=0.0):
    from oracle import sparse_oracle as SO
    from uniphot_b200.psf import MogPsf, rasterize_mog_psf
    rng = np.random.default_rng(seed)
    mog = MogPsf(np.array([[1.4, 0.0, 0.0], [2.6, 0.0, 0.0]]),
                 np.array([[0.05, 0.0, 0.0], [0.0, 0.0, 0.0]]),
                 np.array([[0.0, 0.0, 0.0], [0.02, 0.0, 0.0]]),
                 np.array([[0.75, 0.0, 0.0], [0.25, 0.0, 0.0]]), 500.0, 500.0, 500.0, 500.0)
    psf = rasterize_mog_psf(mog, 15, 500.0, 500.0)
    gx0, gy0 = 400, 380
    px = (gx0 + rng.uniform(4, w - 4, n)).astype(np.float32)
    py = (gy0 + rng.uniform(4, h - 4, n)).astype(np.float32)
    flux = rng.uniform(200, 5000, n)
    S = SO.stamps(psf, px, py, gx0, gy0)
    ixt, iyt = stamp_top_left(px, py, gx0, gy0, 15, 15)
    img = np.zeros((h, w))
    for s in range(n):
        for ky in range(15):
            for kx in range(15):
                yy, xx = iyt[s] + ky, ixt[s] + kx
                if 0 <= yy < h and 0 <= xx < w:
                    img[yy, xx] += flux[s] * S[s, ky, kx]
    bn = (gx0 + w / 2.0, w / 2.0, gy0 + h / 2.0, h / 2.0)
    coef = np.array([20.0, 1.5, -0.8, 0.3, 0.1, -0.2])[:{0: 1, 1: 3, 2: 6}[order]]
    B = SO.bg_basis(h, w, gx0, gy0, *bn, order)
    img = img + B.astype(np.float64) @ coef
    img = img + rng.normal(0, noise, img.shape) if noise else img
    data = img.astype(np.float32)
    invvar = np.full((h, w), 0.04, np.float32)
    good = np.ones((h, w), bool)
    return dict(data=data, invvar=invvar, good=good, px=px, py=py, psf=psf, gx0=gx0,
                gy0=gy0, bn=bn, order=order, flux=flux, coef=coef)


@pytest.mark.parametrize("order", [0, 1, 2])
def test_oracle_recovers_noise_free_fluxes_and_background(order):
    from oracle import sparse_oracle as SO
    g = _grid(order=order)
    idx, mask = build_neighbor_list(g["px"], g["py"], 15, 15, k_max=32)
    f, b, fv, bv = SO.solve_band(g["data"], g["invvar"], g["good"], g["px"], g["py"],
                                 g["psf"], g["gx0"], g["gy0"], g["bn"], order, idx, mask,
                                 reg=1e-9)
    np.testing.assert_allclose(f, g["flux"], rtol=2e-4)
    np.testing.assert_allclose(b, g["coef"], rtol=2e-3, atol=2e-3)
    assert np.all(fv > 0) and np.all(bv > 0)


@pytest.mark.parametrize("stype,backend", [((0, 2, 0), "direct"), ((0, 3, 1), "direct"),
                                           ((0, 1, 0), "bogus")])
def test_direct_backend_rejects_dev_sersic_and_unknown_backends(stype, backend):
    """The "direct" backend renders STAR and EXP only (the reference's
    pipeline rejects DEV/SERSIC there, pipeline.py:1582-1586); checked on
    the host before any device call."""
    from uniphot_b200.sparse import GridBandInputs, solve_band_sparse
    g = _grid(n=3)
    h, w = g["data"].shape
    inp = GridBandInputs(data=g["data"], invvar=g["invvar"], pix_good=g["good"],
                         pos_x=g["px"], pos_y=g["py"], psf=g["psf"], band_h=h, band_w=w,
                         grid_x0=g["gx0"], grid_y0=g["gy0"], bg_x_origin=0.0, bg_x_scale=1.0,
                         bg_y_origin=0.0, bg_y_scale=1.0,
                         source_type=np.array(stype), render_backend=backend)
    with pytest.raises(ValueError):
        solve_band_sparse(inp, np.zeros((3, 4), np.int32), np.zeros((3, 4), bool))


def test_exp_mixture_data_matches_the_reference_constants():
    """``data/exp_mog.npz`` holds source_model.py:56-75's arrays: six
    components, amplitudes normalised to unit sum, the reference's fixture
    agreeing with the oracle through it."""
    from uniphot_b200.sparse import exp_mixture
    amp, var = exp_mixture()
    assert amp.dtype == np.float32 and var.dtype == np.float32
    assert amp.size == var.size == 6
    assert abs(float(amp.astype(np.float64).sum()) - 1.0) < 1e-6
    assert np.all(np.diff(var) > 0) and np.all(amp > 0)


def test_grid_galaxy_stamp_matches_the_island_fft_render():
    """The grid solve's "fft" galaxy stamp is the island solver's reference-
    mode galaxy render (sersic_mog.py:153-194) for the same PSF image."""
    import oracle.island_oracle as O
    from oracle import sparse_oracle as SO
    from test_oracle_pins import _mini_island
    isl, _ = _mini_island("reference", n_src=2, seed=3, T=55, B=48)
    isl.stype[:] = np.array([0, 3])
    isl.free_n[:] = [False, False]
    isl.n_frozen[:] = 2.5
    s = O.IslandSolver(isl, O.SolverConfig(precision="f64"))
    p = isl.p0.astype(np.float64)
    gal = s._gal_params(1, p)
    x, y = float(p[6]), float(p[7])
    S = s._galaxy_fft(0, x, y, gal, False)[0]
    psf = s._star_unshifted(0, x, y)[0]
    amps, vars_, core = isl.table.lookup(2.5)[:3]
    cg, _ = O.cov_terms(float(p[8]), float(p[9]), float(p[10]))
    np.testing.assert_allclose(SO.galaxy_fft(psf.astype(np.float64), amps, vars_, core, cg), S,
                               rtol=1e-9, atol=1e-12)


def test_neighbor_list_skips_non_finite_positions():
    x = np.array([0.0, 5.0, np.nan, 10.0])
    y = np.array([0.0, 3.0, 1.0, np.inf])
    idx, mask = build_neighbor_list(x, y, 15, 15, k_max=4)
    assert not mask[2].any() and not mask[3].any()
    assert set(idx[0][mask[0]].tolist()) == {1} and set(idx[1][mask[1]].tolist()) == {0}
