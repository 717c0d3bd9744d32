"""Joint planar background: each band's plane (1, X, Y over the island
window) solved with the fluxes in the inner linear step, CUDA path vs the
oracle on the same inputs.

Bar (plain form, the reference's arithmetic): identical LM iteration counts
and flags, fluxes and plane coefficients within 1e-4 relative or 0.01 sigma,
positions within 1e-3 px.
"""
import numpy as np
import pytest

from _common import compare, field_classes, run_gpu, run_oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def planed():
    """The small field with a residual plane per band (what a frozen
    background leaves behind when it is off by a tilt)."""
    from uniphot_b200.synth import make_small_field
    f = make_small_field(0)
    nb, H, W = f.data_minus_bg.shape
    yy, xx = np.mgrid[0:H, 0:W].astype(np.float64)
    rng = np.random.default_rng(5)
    for b in range(nb):
        c0, cx, cy = rng.uniform(-20, 20), rng.uniform(-0.05, 0.05), rng.uniform(-0.05, 0.05)
        f.data_minus_bg[b] += (c0 + cx * (xx - W / 2) + cy * (yy - H / 2)).astype(np.float32)
    return f


def _bg_ok(g, o):
    d = np.abs(g["bg"] - o["bg"])
    return (d <= 1e-4 * np.abs(o["bg"])) | (d <= 0.01 * o["bg_err"])


@pytest.mark.parametrize("mode,kinds", [("reference", ("star",)),
                                        ("analytic", ("star", "mixed"))])
def test_joint_background_parity(planed, mode, kinds):
    plans, hosts, PAD, ds, ws, psfs = field_classes(planed, mode, kinds)
    g, _ = run_gpu(plans, hosts, PAD, ds, ws, psfs, mode, native=planed.native,
                   bg_mode="joint")
    o = run_oracle(plans, hosts, PAD, ds, ws, psfs, mode, native=planed.native,
                   bg_joint=True)
    for p, h, gg, oo in zip(plans, hosts, g, o):
        r = compare(gg, oo, h["mmask"])
        msg = f"{p.key}: {r['max_rel']:.2e} {r['max_dpos']:.2e}"
        assert r["same_nst"].all(), msg
        assert r["same_flags"].all(), msg
        assert r["flux_ok"].all(), msg
        assert r["pos_ok"].all(), msg
        assert _bg_ok(gg, oo).all(), f"{p.key}: bg {gg['bg'][:2]} vs {oo['bg'][:2]}"
        assert np.abs(gg["bg"]).max() > 0


def test_joint_background_mixed_form_vs_float64(planed):
    """Every island on the tensor cores (residual form with background rows)
    stays as close to float64 as the plain form."""
    plans, hosts, PAD, ds, ws, psfs = field_classes(planed, "analytic")
    gp, fld = run_gpu(plans, hosts, PAD, ds, ws, psfs, "analytic", native=planed.native,
                      bg_mode="joint")
    gm, _ = run_gpu(plans, hosts, PAD, ds, ws, psfs, "analytic", native=planed.native,
                    bg_mode="joint", precision="mixed", tc_min_rows=0, tc_cond_max=1e30,
                    field=fld)
    o64 = run_oracle(plans, hosts, PAD, ds, ws, psfs, "analytic", precision="f64",
                     native=planed.native, bg_joint=True, processes=8)
    fp, fm = [], []
    for p, h, a, m, o in zip(plans, hosts, gp, gm, o64):
        mm = np.broadcast_to(h["mmask"][:, None, :], a["fluxes"].shape)
        for g, acc in ((a, fp), (m, fm)):
            d = np.abs(g["fluxes"] - o["fluxes"])
            acc.append(((d <= 1e-4 * np.abs(o["fluxes"])) | (d <= 0.01 * o["ferr"]))[mm])
            acc.append(_bg_ok(g, o).ravel())
    fp, fm = np.concatenate(fp).mean(), np.concatenate(fm).mean()
    assert fm >= fp - 0.01 and fm >= 0.98, (fp, fm)


def test_frozen_background_reports_zero_plane(planed):
    plans, hosts, PAD, ds, ws, psfs = field_classes(planed, "analytic", ("star",))
    g, _ = run_gpu(plans[:1], hosts[:1], PAD, ds, ws, psfs, "analytic",
                   native=planed.native)
    assert np.all(g[0]["bg"] == 0)
