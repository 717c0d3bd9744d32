"""The oracle against the reference's own island solver.

``tests/golden/solver_<case>.npz`` hold the per-source results of the
reference's ``island_fit`` (island_solver.py:3233-3595), run on seeded
fields by ``tests/golden/make_golden_solver.py`` with a float64 numpy
stand-in for JAX.  Here the oracle solves the same classes in its float64
reference-render mode and the per-source rows (through the same unpacking
as ``island_fit``) must match: identical LM iteration counts and
converged / stalled / diverged flags on every island, positions within
1e-4 px, shapes within 1e-5, fluxes within 1e-5 relative or 1e-3 of their
error, flux errors within 1e-4 relative, and, where the case asked for
them, the parameter errors, prior fractions, source metrics and Re interval.
"""

from pathlib import Path

import numpy as np
import pytest

from _common import TABLE, field_classes
from uniphot_b200.plan import REPROF_DELTAS_LN, unpack_class_results

GOLDEN = Path(__file__).parent / "golden"

# case -> (field, oracle options, compared columns beyond the fit)
_POST_COLS = ("pos_x_err", "pos_y_err", "re_err", "ell_err", "theta_err", "sersic_n_err",
              "rchisq", "fracflux", "fracin", "fracmasked", "flux_win")
_PRIOR_COLS = ("pos_x_err", "pos_y_err", "re_err", "ell_err", "theta_err", "sersic_n_err",
               "pos_x_prior_frac", "pos_y_prior_frac", "re_prior_frac", "ell_prior_frac",
               "theta_prior_frac", "sersic_n_prior_frac")
CASES = {
    "small": ("small", dict(param_errors=True, source_metrics=True, re_profile=True),
              _POST_COLS + ("re_prof_lo", "re_prof_hi")),
    "small_priors": ("small", dict(param_errors=True, priors=True), _PRIOR_COLS),
    "small_changed": ("small", dict(stall_count_mode="changed"), ()),
    "small_dlnp": ("small", dict(convergence="dlnp"), ()),
    "small_direct": ("small", dict(render_backend="direct"), ()),
    "galaxies": ("galaxies", dict(param_errors=True, source_metrics=True), _POST_COLS),
    "galaxies_changed": ("galaxies", dict(stall_count_mode="changed"), ()),
    "galaxies_dlnp": ("galaxies", dict(convergence="dlnp"), ()),
    "galaxies_free_n": ("galaxies", dict(free_n="sersic"), ()),
    "galaxies_free_n_unfreeze": ("galaxies", dict(free_n="sersic", un_freeze_steps=3), ()),
    "blends": ("blends", dict(param_errors=True, source_metrics=True), _POST_COLS),
    "giants": ("giants", dict(param_errors=True, source_metrics=True), _POST_COLS),
    "large": ("large", dict(param_errors=True, source_metrics=True), _POST_COLS),
}


# The blends case holds 2-12 point sources at 0.3-1.5 FWHM separations and
# flux ratios up to 1e4; there the reference's own result moves by up to
# 6e-3 px between linearisation steps of 1e-7 and 1e-8 (relative) in the
# generator, so its error columns are compared at the 1e-3 level the
# stand-in's derivative supports.
# The large case's 14-member island stalls after 24 LM steps; along that
# trajectory the same derivative differences move one galaxy's ee2 by 1.5e-4
# and a theta error by 1.3e-4 relative, so its shapes are compared to 5e-4
# and its error columns to 1e-3.
ERR_RTOL = {c: (1e-3 if c in ("blends", "large") else 1e-4) for c in CASES}
# With a free Sersic index the fitted n goes through the table's piecewise-
# linear mixture, whose derivative the generator takes by differences; one
# index lands 1.75e-5 (1e-5 relative) from the oracle's, so the free-n cases
# compare shapes to 5e-5.
SHAPE_ATOL = {c: (5e-4 if c == "large" else 5e-5 if "free_n" in c else 1e-5) for c in CASES}


def _field(name):
    from uniphot_b200 import synth
    if name == "small":
        return synth.make_small_field(0)
    if name == "galaxies":
        return synth.make_production_field(4, side=320, n_bands=3, n_src=40, margin=40)
    if name == "giants":
        return synth.make_production_field(1, side=320, n_bands=3, n_src=40, margin=40)
    if name == "large":
        return synth.make_production_field(3, side=256, n_bands=3, n_src=30, margin=40)
    return synth.make_blend_field(0, n_islands=6, n_bands=3)


def _digest(f):
    import hashlib
    h = hashlib.sha256()
    for a in (f.data_minus_bg, f.invvar, f.pos_x, f.pos_y, f.source_type, f.logre, f.ee1,
              f.ee2, f.sersic_n, f.s1_flux, f.s1_flux_var):
        h.update(np.ascontiguousarray(a).tobytes())
    for p in f.poly_psfs:
        h.update(np.ascontiguousarray(p.coefs, np.float32).tobytes())
    return h.hexdigest()


def _oracle_rows(f, opts, precision="f64"):
    """Per-source rows of the oracle's solve (float64, or "ref": the
    reference's float32 render with float64 solves), sorted by source."""
    from oracle.driver import solve_chunk
    from uniphot_b200.plan import giant_seed_rows, plan_island_classes
    opts = dict(opts)
    if opts.get("render_backend") == "direct":
        z = np.load(Path(__file__).parents[1] / "uniphot_b200" / "data" / "exp_mog.npz")
        opts["exp_mog"] = (z["amp"], z["var"])
    priors = opts.pop("priors", False)
    re_prof = opts.pop("re_profile", False)
    # island_fit's free_n_override: here every SERSIC source
    free_n = (f.source_type == 3) if opts.pop("free_n", None) == "sersic" else None
    # the reference's island_fit uses its default tier ladder (111, 221)
    plans, hosts, PAD, ds, ws, psfs = field_classes(f, "reference", priors=priors,
                                                    tier_ladder=(111, 221), free_n=free_n)
    # islands in nsrc buckets above the joint cap (32) keep their seeds
    _, capped = plan_island_classes(f.island_set, f.buckets, f.source_type, f.logre,
                                    f.sersic_n, f.native, tier_ladder=(111, 221))
    giant_ids = np.concatenate([np.asarray(f.buckets.giant_ids, np.int64).ravel(),
                                np.asarray(capped, np.int64)])
    rows = []
    for p, h in zip(plans, hosts):
        o = solve_chunk(h, np.arange(p.n_islands), B=p.bbox_class, T=p.tier, dstack=ds,
                        wstack=ws, psfs=psfs, mode="reference", table_path=TABLE,
                        precision=precision, max_steps=30, native=f.native,
                        step_mode="clip", re_profile=REPROF_DELTAS_LN if re_prof else None,
                        **opts)
        rows.append(unpack_class_results(
            p, h, f.island_set, o["p"], o["fluxes"], o["ferr"], o["chi2"], o["conv"],
            o["stall"], o["nst"], res_pdchi2=o["stall_dchi2"], res_div=o["diverged"],
            res_ngood=o["n_good"], n_bands=ds.shape[0], res_perr=o["perr"],
            res_smetrics=o["smetrics"], res_swin=o["swin"], res_reprof=o["reprof"],
            reprof_deltas=REPROF_DELTAS_LN if re_prof else None))
    if giant_ids.size:
        rows.extend(giant_seed_rows(giant_ids, f.island_set, n_bands=ds.shape[0],
                                    pos_x=f.pos_x, pos_y=f.pos_y, logre=f.logre, ee1=f.ee1,
                                    ee2=f.ee2, sersic_n=f.sersic_n))
    cat = {k: np.concatenate([r[k] for r in rows]) for k in rows[0]}
    order = np.argsort(cat["src"])
    return {k: v[order] for k, v in cat.items()}


def _close(name, a, b, atol, rtol=0.0):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    np.testing.assert_array_equal(np.isnan(a), np.isnan(b), err_msg=f"{name}: NaN pattern")
    ok = ~np.isnan(a)
    np.testing.assert_allclose(a[ok], b[ok], atol=atol, rtol=rtol, err_msg=name)


@pytest.mark.parametrize("case", sorted(CASES))
def test_oracle_matches_reference_solver(case):
    path = GOLDEN / f"solver_{case}.npz"
    if not path.exists():
        pytest.skip(f"fixture {path.name} not generated")
    field_name, opts, cols = CASES[case]
    ref = dict(np.load(path))
    f = _field(field_name)
    assert str(ref.pop("digest")) == _digest(f), "synthetic field changed since the fixture"
    order = np.argsort(ref["source_idx"])
    ref = {k: v[order] for k, v in ref.items()}
    o = _oracle_rows(f, opts)
    np.testing.assert_array_equal(o["src"], ref["source_idx"])
    assert ref["island_giant"].any() == (case == "giants")
    np.testing.assert_array_equal(o["n_steps"], ref["n_steps"])
    for k in ("converged", "stalled", "diverged", "free_n", "island_id", "island_nsrc",
              "island_giant"):
        np.testing.assert_array_equal(o[k], ref[k], err_msg=k)
    _close("pos_x", o["pos_x"], ref["pos_x"], 1e-4)
    _close("pos_y", o["pos_y"], ref["pos_y"], 1e-4)
    for k in ("logre", "ee1", "ee2", "sersic_n"):
        _close(k, o[k], ref[k], SHAPE_ATOL[case])
    # fluxes within 1e-5 relative or 1e-3 of their error
    # (giant rows carry NaN fluxes on both sides)
    np.testing.assert_array_equal(np.isnan(o["fluxes"]), np.isnan(ref["fluxes"]))
    fin = ~np.isnan(ref["fluxes"])
    df = np.abs(o["fluxes"].astype(np.float64) - ref["fluxes"])[fin]
    bound = np.maximum(1e-5 * np.abs(ref["fluxes"]), 1e-3 * ref["flux_err"])[fin]
    assert np.all(df <= bound), f"fluxes: worst {np.max(df / bound):.3g} x the bound"
    _close("flux_err", o["flux_err"], ref["flux_err"], 0.0, ERR_RTOL[case])
    _close("chi2", o["chi2"], ref["chi2"], 1e-3, 1e-6)
    _close("chi2_nu", o["chi2_nu"], ref["chi2_nu"], 1e-6, 1e-6)
    # the stalled islands' plateau-probe certificate (island_solver.py:1401-1465)
    _close("stall_dchi2", o["stall_dchi2"], ref["stall_dchi2"], 1e-3, 1e-4)
    _close("re_upper_pix", o["re_upper_pix"], ref["re_upper_pix"], 0.0, 1e-6)
    for k in cols:
        _close(k, o[k], ref[k], 1e-5, ERR_RTOL[case])
