"""Per-grid sparse forced photometry on the GPU (uph_sparse_band_solve) vs
the oracle (forced_phot_sparse.py:342-562, 690-718).

Bar: fluxes within 1e-4 relative or 0.01 sigma, background coefficients
within 1e-4 relative or 0.01 of their sigma, variances within 1e-3
relative; both sides sum float32 products (the device in float64, the
oracle in float64) and solve in float64.
"""
import numpy as np
import pytest

from test_sparse_cpu import _grid
from uniphot_b200.sparse import GridBandInputs, build_neighbor_list, solve_band_sparse

pytestmark = pytest.mark.gpu


def _inputs(g):
    h, w = g["data"].shape
    return GridBandInputs(data=g["data"], invvar=g["invvar"], pix_good=g["good"],
                          pos_x=g["px"], pos_y=g["py"], psf=g["psf"], band_h=h, band_w=w,
                          grid_x0=g["gx0"], grid_y0=g["gy0"], bg_x_origin=g["bn"][0],
                          bg_x_scale=g["bn"][1], bg_y_origin=g["bn"][2],
                          bg_y_scale=g["bn"][3])


def _check(r, o):
    f, b, fv, bv = o
    sig = np.sqrt(np.maximum(fv, 1e-30))
    assert np.all((np.abs(r.fluxes - f) <= 1e-4 * np.abs(f)) | (np.abs(r.fluxes - f) <= 0.01 * sig))
    bs = np.sqrt(np.maximum(bv, 1e-30))
    assert np.all((np.abs(r.bg_coefs - b) <= 1e-4 * np.abs(b)) | (np.abs(r.bg_coefs - b) <= 0.01 * bs))
    np.testing.assert_allclose(r.flux_var, fv, rtol=1e-3)
    np.testing.assert_allclose(r.bg_var, bv, rtol=1e-3)
    assert r.converged


@pytest.fixture(scope="module")
def ctx():
    from uniphot_b200 import _lib
    return _lib.Context(0)


@pytest.mark.parametrize("order", [0, 1, 2])
def test_sparse_band_parity(ctx, order):
    from oracle import sparse_oracle as SO
    g = _grid(seed=order, n=20, order=order, noise=5.0)
    g["good"][10:14, :] = False                  # a masked band of rows
    g["px"][0] = g["gx0"] + 1.3                  # a stamp hanging over the edge
    idx, mask = build_neighbor_list(g["px"], g["py"], 15, 15, k_max=32)
    r = solve_band_sparse(_inputs(g), idx, mask, reg=1e-9, bg_poly_order=order, context=ctx)
    o = SO.solve_band(g["data"], g["invvar"], g["good"], g["px"], g["py"], g["psf"],
                      g["gx0"], g["gy0"], g["bn"], order, idx, mask, reg=1e-9)
    _check(r, o)


def test_sparse_band_crowded_truncated_neighbours(ctx):
    """60 sources on 64 x 72 pixels with k_max = 4: truncated (asymmetric)
    neighbour lists are scatter-added exactly as listed."""
    from oracle import sparse_oracle as SO
    g = _grid(seed=5, n=60, order=1, noise=5.0)
    idx, mask = build_neighbor_list(g["px"], g["py"], 15, 15, k_max=4)
    r = solve_band_sparse(_inputs(g), idx, mask, reg=1e-9, bg_poly_order=1, context=ctx)
    o = SO.solve_band(g["data"], g["invvar"], g["good"], g["px"], g["py"], g["psf"],
                      g["gx0"], g["gy0"], g["bn"], 1, idx, mask, reg=1e-9)
    _check(r, o)


def test_sparse_band_noise_free_known_answer_and_empty_grid(ctx):
    g = _grid(seed=2, n=12, order=2)
    idx, mask = build_neighbor_list(g["px"], g["py"], 15, 15)
    r = solve_band_sparse(_inputs(g), idx, mask, reg=1e-9, bg_poly_order=2, context=ctx)
    np.testing.assert_allclose(r.fluxes, g["flux"], rtol=2e-4)
    np.testing.assert_allclose(r.bg_coefs, g["coef"], rtol=2e-3, atol=2e-3)
    e = _inputs(g)
    e.pos_x = e.pos_x[:0]
    e.pos_y = e.pos_y[:0]
    r0 = solve_band_sparse(e, np.zeros((0, 8), np.int32), np.zeros((0, 8), bool),
                           bg_poly_order=0, context=ctx)
    assert r0.fluxes.size == 0 and r0.converged
    w = g["invvar"].astype(np.float64)
    np.testing.assert_allclose(r0.bg_coefs[0], (w * g["data"]).sum() / w.sum(), rtol=1e-5)


def test_sparse_band_with_galaxies_fft_backend(ctx):
    """Stars and EXP/DEV/SERSIC galaxies with the "fft" backend
    (source_model.py:304-318): galaxy stamps from the Sersic mixture's
    transform times the PSF's, no renormalisation on the mixed path."""
    from oracle import sparse_oracle as SO
    from oracle.island_oracle import SersicTable
    from _common import TABLE
    g = _grid(seed=7, n=16, order=1, noise=5.0)
    rng = np.random.default_rng(7)
    st = np.array([0, 1, 2, 3] * 4, np.int32)
    lr = rng.uniform(0.0, 1.2, 16).astype(np.float32)
    e1 = rng.uniform(-0.3, 0.3, 16).astype(np.float32)
    e2 = rng.uniform(-0.3, 0.3, 16).astype(np.float32)
    sn = np.where(st == 1, 1.0, np.where(st == 2, 4.0, rng.uniform(0.7, 5.0, 16))).astype(np.float32)
    idx, mask = build_neighbor_list(g["px"], g["py"], 15, 15, k_max=32)
    inp = _inputs(g)
    inp.source_type, inp.logre, inp.ee1, inp.ee2, inp.sersic_n = st, lr, e1, e2, sn
    inp.render_backend = "fft"
    r = solve_band_sparse(inp, idx, mask, reg=1e-9, bg_poly_order=1, context=ctx)
    o = SO.solve_band(g["data"], g["invvar"], g["good"], g["px"], g["py"], g["psf"],
                      g["gx0"], g["gy0"], g["bn"], 1, idx, mask, reg=1e-9,
                      gal=(st, lr, e1, e2, sn), table=SersicTable.load(TABLE))
    _check(r, o)


def test_sparse_band_exp_direct_backend(ctx):
    """Stars and EXP galaxies on the legacy "direct" backend
    (source_model.py:218-256, 298-303): the pixel-centre exponential mixture
    convolved with the PSF stamp and renormalised, then the stars' Lanczos
    shift.  Checked against the oracle and against the reference's own
    solve of the same grid (tests/golden/sparse_exp_direct.npz)."""
    import sys
    from pathlib import Path
    from oracle import sparse_oracle as SO
    from uniphot_b200.sparse import exp_mixture
    golden = Path(__file__).parent / "golden"
    sys.path.insert(0, str(golden))
    from make_golden_sparse import case_inputs
    g, idx, mask, order, gal, backend = case_inputs("exp_direct")
    assert backend == "direct"
    inp = _inputs(g)
    inp.source_type, inp.logre, inp.ee1, inp.ee2, inp.sersic_n = gal
    inp.render_backend = "direct"
    r = solve_band_sparse(inp, idx, mask, reg=1e-9, bg_poly_order=order, context=ctx)
    o = SO.solve_band(g["data"], g["invvar"], g["good"], g["px"], g["py"], g["psf"],
                      g["gx0"], g["gy0"], g["bn"], order, idx, mask, reg=1e-9, gal=gal,
                      backend="direct", exp_mog=exp_mixture())
    _check(r, o)
    ref = np.load(golden / "sparse_exp_direct.npz")
    _check(r, (ref["fluxes"], ref["bg_coefs"], ref["flux_var"], ref["bg_var"]))
