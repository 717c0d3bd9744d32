"""Mixed form (tensor-core Gram from BF16 hi/lo pairs, residual form) against
the all-float64 oracle, beside the plain FP32 form on the same inputs.

Bar: the same LM iteration counts and converged/stalled flags as the plain
form; against float64, fluxes within 1e-4 relative or 0.01 sigma and
positions within 1e-3 px for every member where the plain form meets that
bar, and at least the plain form's pass fraction overall.
"""
import numpy as np
import pytest

from _common import field_classes, run_gpu, run_oracle

pytestmark = pytest.mark.gpu

REL, SIG, POS = 1e-4, 0.01, 1e-3


def _flux_ok(g, o, mmask):
    m = np.broadcast_to(mmask[:, None, :], g["fluxes"].shape)
    d = np.abs(g["fluxes"] - o["fluxes"])
    ok = (d <= REL * np.abs(o["fluxes"])) | (d <= SIG * o["ferr"])
    return ok[m]


def _pos_ok(g, o, mmask):
    dp = np.abs(g["p"][..., :2] - o["p"][..., :2]).max(axis=-1)
    return (dp <= POS)[mmask]


def _check(plans, hosts, gp, gm, o64, label, same_path=True, margin=0.0):
    fp, fm, pp, pm = [], [], [], []
    for p, h, a, b, o in zip(plans, hosts, gp, gm, o64):
        msg = f"{label} {p.key}"
        if same_path:
            np.testing.assert_array_equal(b["nst"], a["nst"], err_msg=msg)
            np.testing.assert_array_equal(b["conv"], a["conv"], err_msg=msg)
            np.testing.assert_array_equal(b["stall"], a["stall"], err_msg=msg)
        assert np.isfinite(b["fluxes"]).all() and np.isfinite(b["p"]).all(), msg
        fp.append(_flux_ok(a, o, h["mmask"]))
        fm.append(_flux_ok(b, o, h["mmask"]))
        pp.append(_pos_ok(a, o, h["mmask"]))
        pm.append(_pos_ok(b, o, h["mmask"]))
    fp, fm = np.concatenate(fp), np.concatenate(fm)
    pp, pm = np.concatenate(pp), np.concatenate(pm)
    assert fm.mean() >= fp.mean() - margin, \
        f"{label}: flux pass {fm.mean():.4f} < plain {fp.mean():.4f}"
    assert pm.mean() >= pp.mean() - margin, \
        f"{label}: pos pass {pm.mean():.4f} < plain {pp.mean():.4f}"
    return fp.mean(), fm.mean()


@pytest.fixture(scope="module")
def small():
    from uniphot_b200.synth import make_small_field
    return make_small_field(0)


@pytest.mark.parametrize("mode,kinds", [("reference", ("star",)),
                                        ("analytic", ("star", "mixed"))])
def test_every_island_on_tensor_cores(small, mode, kinds):
    """tc_min_rows = 0 and no conditioning limit route every island (Gram
    rows 3..) through the tensor-core kernel."""
    plans, hosts, PAD, ds, ws, psfs = field_classes(small, mode, kinds)
    gp, fld = run_gpu(plans, hosts, PAD, ds, ws, psfs, mode, native=small.native)
    gm, _ = run_gpu(plans, hosts, PAD, ds, ws, psfs, mode, native=small.native,
                    precision="mixed", tc_min_rows=0, tc_cond_max=1e30, field=fld)
    o64 = run_oracle(plans, hosts, PAD, ds, ws, psfs, mode, precision="f64",
                     native=small.native, processes=8)
    fp, fm = _check(plans, hosts, gp, gm, o64, mode)
    assert fm >= 0.99, fm


def test_blends_default_threshold():
    """Reduced production field: the blended classes whose islands exceed
    the default 24 Gram rows (8 and 16 members, windows 32-128 px)."""
    from uniphot_b200.synth import make_production_field
    f = make_production_field(3, side=512, n_bands=3, n_src=300)
    plans, hosts, PAD, ds, ws, psfs = field_classes(f, "analytic")
    want = {(32, 8, "mixed", 31), (48, 8, "mixed", 31), (96, 16, "mixed", 127),
            (128, 16, "mixed", 127)}
    keep = [i for i, p in enumerate(plans) if p.key in want]
    assert len(keep) == len(want)
    plans = [plans[i] for i in keep]
    hosts = [hosts[i] for i in keep]
    gp, fld = run_gpu(plans, hosts, PAD, ds, ws, psfs, "analytic", native=f.native)
    gm, _ = run_gpu(plans, hosts, PAD, ds, ws, psfs, "analytic", native=f.native,
                    precision="mixed", field=fld)
    o64 = run_oracle(plans, hosts, PAD, ds, ws, psfs, "analytic", precision="f64",
                     native=f.native, processes=8)
    _check(plans, hosts, gp, gm, o64, "blends")


def test_mixed_deterministic(small):
    plans, hosts, PAD, ds, ws, psfs = field_classes(small, "analytic")
    a, fld = run_gpu(plans, hosts, PAD, ds, ws, psfs, "analytic", native=small.native,
                     precision="mixed", tc_min_rows=0)
    b, _ = run_gpu(plans, hosts, PAD, ds, ws, psfs, "analytic", native=small.native,
                   precision="mixed", tc_min_rows=0, field=fld)
    for x, y in zip(a, b):
        for k in ("p", "fluxes", "ferr", "chi2", "nst"):
            np.testing.assert_array_equal(x[k], y[k])


def test_precision_stress_blends():
    """Crowded blends (2-12 sources 0.3-1.5 FWHM apart, flux ratios up to
    1e4, a quarter of the bands at low SNR): the mixed form stays as close to
    float64 as the plain form (within 2 points of its pass fraction).  The
    two forms may take different LM paths on these ill-conditioned
    problems, so iteration counts are not compared."""
    from uniphot_b200.synth import make_blend_field
    f = make_blend_field(0, n_islands=30, n_bands=8)
    plans, hosts, PAD, ds, ws, psfs = field_classes(f, "analytic")
    gp, fld = run_gpu(plans, hosts, PAD, ds, ws, psfs, "analytic", native=f.native)
    gm, _ = run_gpu(plans, hosts, PAD, ds, ws, psfs, "analytic", native=f.native,
                    precision="mixed", field=fld)
    o64 = run_oracle(plans, hosts, PAD, ds, ws, psfs, "analytic", precision="f64",
                     native=f.native, processes=8)
    fp, fm = _check(plans, hosts, gp, gm, o64, "stress", same_path=False, margin=0.02)
    print(f"stress: flux pass plain {fp:.4f} mixed {fm:.4f}")
