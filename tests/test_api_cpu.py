"""Host-side API behaviour that needs no GPU: option validation mirrors the
reference's ValueErrors; unsupported options fail loudly."""
import numpy as np
import pytest

from uniphot_b200 import solver
from uniphot_b200.plan import IslandClassPlan


def _plan(kind="star"):
    return IslandClassPlan(0, 32, 1, kind, 31, np.zeros(1, np.int64),
                           np.zeros((1, 1), np.int64), np.ones((1, 1), bool),
                           np.zeros((1, 4), np.int64), np.ones(1, np.int32))


KW = dict(render_backend="fft", reg=1e-9, pos_step_max_pix=0.5, chi2_ftol_rel=1e-4,
          step_tol_pix=0.1, un_freeze_steps=0)


@pytest.mark.parametrize("bad", [dict(stall_count_mode="x"), dict(step_mode="x"),
                                 dict(convergence="x"),
                                 dict(convergence="dlnp", step_mode="trust_region"),
                                 dict(convergence="dlnp", stall_count_mode="changed"),
                                 dict(step_mode="trust_region", stall_count_mode="changed"),
                                 dict(render_mode="x")])
def test_invalid_options_raise_valueerror(bad):
    with pytest.raises(ValueError):
        solver.make_class_kernels(_plan(), 3, 1, **KW, **bad)


@pytest.mark.parametrize("opt", [dict(crossband={"rank": 1})])
def test_unbuilt_options_raise(opt):
    with pytest.raises(ValueError, match="not supported"):
        solver.make_class_kernels(_plan("mixed"), 3, 1, **KW, **opt)


def test_dlnp_convergence_sets_the_descriptor():
    k = solver.make_class_kernels(_plan("mixed"), 3, 1, **KW, convergence="dlnp",
                                  plateau_dlnp_tol=0.25)
    assert k.desc.convergence_dlnp == 1 and k.step_protocol == "dlnp"
    assert abs(k.desc.plateau_dlnp_tol - 0.25) < 1e-7


def test_changed_stall_counting_sets_the_descriptor():
    k = solver.make_class_kernels(_plan("mixed"), 3, 1, **KW, stall_count_mode="changed")
    assert k.desc.stall_changed == 1 and k.step_protocol == "changed"
    k = solver.make_class_kernels(_plan("mixed"), 3, 1, **KW)
    assert k.desc.stall_changed == 0 and k.step_protocol == "proposals"


def test_class_descriptor_fields():
    k = solver.make_class_kernels(_plan(), 3, 1, **KW, native_stamp=31)
    assert (k.desc.bbox, k.desc.nsrc, k.desc.tier, k.desc.native_stamp) == (32, 1, 31, 31)
    assert k.desc.render_mode == 0


def test_run_class_chunk_rejects_post_convergence_options():
    k = solver.make_class_kernels(_plan(), 3, 1, **KW)
    with pytest.raises(ValueError):
        solver.run_class_chunk(k, None, {}, np.arange(1), 1, 30, None, None, 10,
                               compute_source_metrics=True)


def test_psf_tree_padding_keeps_centre():
    from uniphot_b200.psf import PsfPolynomial
    c = np.zeros((5, 5, 1), np.float32)
    c[2, 2, 0] = 1.0
    tree, nt = solver.build_psf_tree([PsfPolynomial(c, 0, 1, 0, 1, 5, 5)], 9)
    assert nt == 1 and tree.params.shape == (1, 9, 9, 1)
    assert tree.params[0, 4, 4, 0] == 1.0 and tree.params.sum() == 1.0


def test_trust_region_sets_the_descriptor_except_on_star_classes():
    """Star-only classes keep the clip step (island_solver.py:1910-1912)."""
    k = solver.make_class_kernels(_plan("mixed"), 3, 1, **KW, step_mode="trust_region")
    assert k.desc.step_tr == 1 and k.step_mode == "trust_region"
    k = solver.make_class_kernels(_plan("star"), 3, 1, **KW, step_mode="trust_region")
    assert k.desc.step_tr == 0 and k.step_mode == "clip"


def test_catalog_errors_propagate_to_the_catalog_frame():
    """Variances -> catalog-frame errors (island_plan.py:796-885): Re scales
    by exp(logre), ELL and THETA take the exact 2x2 quadratic forms with the
    ee1-ee2 covariance, Sersic n scales by dn/du on free-n members; non-kept
    slots and non-positive variances read NaN."""
    from uniphot_b200.plan import SERSIC_N_MAX, SERSIC_N_MIN, catalog_errors
    res_p = np.zeros((1, 2, 6), np.float32)
    res_p[0, 0] = [10, 12, np.log(3.0), 0.3, -0.4, 0.0]
    perr = np.zeros((1, 2, 13), np.float32)
    perr[0, 0, :7] = [0.04, 0.09, 0.01, 0.02, 0.03, 0.25, 0.005]
    perr[0, 0, 7:] = [0.5, 0.5, 0.2, 0.1, 0.3, 0.0]
    perr[0, 1, :6] = [-1.0, 0.0, 1.0, 1.0, 1.0, 1.0]
    keep = np.zeros((1, 2, 6), bool)
    keep[0, 0] = True
    keep[0, 1, :2] = True
    pinv = np.zeros((1, 2, 6), np.float32)
    pinv[0, 0, :5] = 1.0
    host = dict(keep=keep, fn_flag=np.array([[True, False]]), prior_inv_sigma=pinv)
    nfin = np.array([[2.0, 1.0]], np.float32)
    e = catalog_errors(res_p, perr, host, np.array([0, 0]), np.array([0, 1]), nfin)
    np.testing.assert_allclose(e["pos_x_err"][0], 0.2, rtol=1e-6)
    np.testing.assert_allclose(e["re_err"][0], 3.0 * 0.1, rtol=1e-6)
    e1, e2, v1, v2, c = 0.3, -0.4, 0.02, 0.03, 0.005
    r = np.hypot(e1, e2)
    q = np.exp(-r)
    g = 2 * q / (2 - q) ** 2 * np.array([e1, e2]) / r
    S = np.array([[v1, c], [c, v2]])
    np.testing.assert_allclose(e["ell_err"][0], np.sqrt(g @ S @ g), rtol=1e-5)
    gt = (90 / np.pi) * np.array([e2, -e1]) / r ** 2
    np.testing.assert_allclose(e["theta_err"][0], np.sqrt(gt @ S @ gt), rtol=1e-5)
    dndu = (2.0 - SERSIC_N_MIN) * (SERSIC_N_MAX - 2.0) / (SERSIC_N_MAX - SERSIC_N_MIN)
    np.testing.assert_allclose(e["sersic_n_err"][0], 0.5 * dndu, rtol=1e-6)
    assert np.isnan(e["pos_x_err"][1]) and np.isnan(e["pos_y_err"][1])
    assert np.isnan(e["re_err"][1]) and np.isnan(e["sersic_n_err"][1])
    np.testing.assert_allclose(e["pos_x_prior_frac"][0], 0.5)
    np.testing.assert_allclose(e["ell_prior_frac"][0], (e1**2 * 0.1 + e2**2 * 0.3) / r**2,
                               rtol=1e-6)
    assert np.isnan(e["sersic_n_prior_frac"][0]) and np.isnan(e["pos_x_prior_frac"][1])


def test_direct_backend_sets_the_descriptor_in_reference_mode():
    """render_backend="direct" selects the legacy EXP backend for the
    pixelised-PSF render (the device checks the members are STAR or EXP);
    the analytic render has no backend choice."""
    k = solver.make_class_kernels(_plan("mixed"), 3, 1, **dict(KW, render_backend="direct"),
                                  render_mode="reference")
    assert k.desc.render_mode == 0 and k.desc.render_direct == 1
    k = solver.make_class_kernels(_plan("star"), 3, 1, **dict(KW, render_backend="direct"),
                                  render_mode="reference")
    assert k.desc.render_mode == 0 and k.desc.render_direct == 1
    k = solver.make_class_kernels(_plan("mixed"), 3, 1, **dict(KW, render_backend="fft"),
                                  render_mode="reference")
    assert k.desc.render_direct == 0
    k = solver.make_class_kernels(_plan("mixed"), 3, 1, **dict(KW, render_backend="direct"),
                                  render_mode="analytic")
    assert k.desc.render_direct == 0


def test_scene_subtract_sets_the_descriptor_and_needs_s1_fluxes():
    k = solver.make_class_kernels(_plan("mixed"), 3, 1, **KW, scene_subtract=True)
    assert k.desc.scene_subtract == 1
    host = dict(ox=[0], oy=[0], x0b=[0.0], y0b=[0.0], st=np.zeros((1, 1)), sn=np.ones((1, 1)),
                fn_flag=np.zeros((1, 1), bool), mmask=np.ones((1, 1), bool),
                keep=np.ones((1, 1, 6), bool), p0=np.zeros((1, 1, 6)),
                lower=np.zeros((1, 1, 6)), upper=np.ones((1, 1, 6)),
                prior_mean=np.zeros((1, 1, 6)), prior_inv_sigma=np.zeros((1, 1, 6)),
                member_s1_flux=None)
    with pytest.raises(ValueError, match="member_s1_flux"):
        solver._slice_host(host, np.arange(1), scene_subtract=True)


def test_re_profile_interval_edges():
    """A side whose profile never reaches 1 ends at its outermost offset; a
    non-finite profile value counts as beyond 1 (island_plan.py:913-952)."""
    from uniphot_b200.plan import REPROF_DELTAS_LN, re_profile_interval
    d = REPROF_DELTAS_LN.astype(np.float64)
    prof = np.full((1, 1, d.size), 0.2, np.float32)
    prof[0, 0, d == 0.25] = np.nan                 # +0.25 counts as >= 1
    res_p = np.zeros((1, 1, 6), np.float32)
    lo, hi = re_profile_interval(res_p, prof, d, np.array([0]), np.array([0]),
                                 np.array([[True]]))
    np.testing.assert_allclose(lo[0], np.exp(-2.5), rtol=1e-6)
    # crossing between 0.1 (profile 0.2) and 0.25 (infinite): t = 0.8 / inf -> 0
    np.testing.assert_allclose(hi[0], np.exp(0.1), rtol=1e-6)


def test_catalog_errors_round_source_and_degenerate_variances():
    from uniphot_b200.plan import catalog_errors
    res_p = np.zeros((1, 1, 6), np.float32)          # ee = 0: direction undefined
    perr = np.zeros((1, 1, 13), np.float32)
    perr[0, 0, :6] = [np.inf, -1.0, 0.04, 0.01, 0.01, 0.0]
    host = dict(keep=np.ones((1, 1, 6), bool), fn_flag=np.array([[False]]),
                prior_inv_sigma=np.zeros((1, 1, 6), np.float32))
    e = catalog_errors(res_p, perr, host, np.array([0]), np.array([0]),
                       np.ones((1, 1), np.float32))
    assert np.isnan(e["pos_x_err"][0]) and np.isnan(e["pos_y_err"][0])
    np.testing.assert_allclose(e["re_err"][0], 0.2, rtol=1e-6)
    assert np.isnan(e["ell_err"][0]) and np.isnan(e["theta_err"][0])
    assert np.isnan(e["sersic_n_err"][0]) and np.isnan(e["pos_x_prior_frac"][0])


def test_superseded_device_field_is_refused():
    """A DeviceField records the upload it came from; after another field is
    uploaded to the same context it refuses to bind new chunks (the chunks
    already added keep their own buffers).  A stand-in context holds only
    the upload counter the check reads."""
    class Ctx:
        field_gen = 0

        def upload_field_unpadded(self, d, w, pad):
            self.field_gen += 1
    ctx = Ctx()
    d = np.zeros((2, 8, 8), np.float32)
    a = solver.DeviceField.from_unpadded(d, d, 3, context=ctx)
    a.check_current()
    b = solver.DeviceField.from_unpadded(d, d, 3, context=ctx)
    b.check_current()
    with pytest.raises(ValueError, match="superseded"):
        a.check_current()
    assert b.shape == (2, 14, 14) and b.pad == 3
