"""Step variants on the GPU vs the oracle: stall_count_mode="changed"
(island_solver.py:1118-1208) keeps an in-loop tracker of the last rejected
proposal -- identical-proposal rejects escalate lambda without counting
toward the stall, and a run of 4 sets the sticky diverged flag;
convergence="dlnp" (:1210-1333); step_mode="trust_region" (:1004-1116).
"""
import numpy as np
import pytest

from _common import compare, field_classes, run_gpu, run_oracle

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def small():
    from uniphot_b200.synth import make_small_field
    return make_small_field(0)


@pytest.mark.parametrize("mode,kinds", [("reference", ("star",)),
                                        ("analytic", ("star", "mixed"))])
def test_changed_mode_parity(small, mode, kinds):
    plans, hosts, PAD, ds, ws, psfs = field_classes(small, mode, kinds)
    g, _ = run_gpu(plans, hosts, PAD, ds, ws, psfs, mode, native=small.native,
                   stall_count_mode="changed")
    o = run_oracle(plans, hosts, PAD, ds, ws, psfs, mode, native=small.native,
                   stall_count_mode="changed")
    for p, h, gg, oo in zip(plans, hosts, g, o):
        r = compare(gg, oo, h["mmask"])
        msg = f"{p.key}: {r['max_rel']:.2e} {r['max_dpos']:.2e}"
        assert r["same_nst"].all() and r["same_flags"].all(), msg
        assert r["flux_ok"].all() and r["pos_ok"].all(), msg
        np.testing.assert_array_equal(gg["diverged"], oo["diverged"])
        np.testing.assert_array_equal(gg["n_same"], oo["n_same"])


def test_changed_mode_zero_weight_island(small):
    """Identical proposals never count: the island runs to max_steps with
    the diverged flag set, as in the oracle."""
    plans, hosts, PAD, ds, ws, psfs = field_classes(small, "analytic", ("star",))
    p, h = plans[0], hosts[0]
    ws2 = ws.copy()
    oy, ox = int(h["oy"][0]), int(h["ox"][0])
    ws2[:, oy:oy + p.bbox_class, ox:ox + p.bbox_class] = 0.0
    g, _ = run_gpu([p], [h], PAD, ds, ws2, psfs, "analytic", native=small.native,
                   max_steps=12, stall_count_mode="changed")
    o = run_oracle([p], [h], PAD, ds, ws2, psfs, "analytic", native=small.native,
                   max_steps=12, stall_count_mode="changed")
    g, o = g[0], o[0]
    assert g["nst"][0] == 12 and not g["conv"][0] and g["diverged"][0]
    assert g["n_same"][0] == o["n_same"][0] == 12
    np.testing.assert_array_equal(g["nst"], o["nst"])
    np.testing.assert_array_equal(g["diverged"], o["diverged"])


def test_changed_mode_tracker_carries_across_requeue(small):
    """A re-queued chunk carrying the tracker state equals one pass."""
    from uniphot_b200 import solver
    plans, hosts, PAD, ds, ws, psfs = field_classes(small, "analytic", ("mixed",))
    p, h = plans[0], hosts[0]
    full, fld = run_gpu([p], [h], PAD, ds, ws, psfs, "analytic", native=small.native,
                        stall_count_mode="changed")
    a, _ = run_gpu([p], [h], PAD, ds, ws, psfs, "analytic", max_steps=2, field=fld,
                   native=small.native, stall_count_mode="changed")
    a = a[0]
    tree, nt = solver.build_psf_tree(psfs, p.tier)
    kern = solver.make_class_kernels(p, ds.shape[0], nt, render_backend="fft", reg=1e-9,
                                     pos_step_max_pix=0.5, chi2_ftol_rel=1e-4,
                                     step_tol_pix=0.1, un_freeze_steps=0,
                                     render_mode="analytic", native_stamp=small.native,
                                     stall_count_mode="changed")
    rows = np.nonzero(~a["conv"])[0]
    assert rows.size > 0
    init = {k: a[k][rows] for k in ("p", "lam", "chi2", "consec", "nrej", "nst",
                                    "n_same", "prej", "diverged")}
    b = solver.run_class_chunk(kern, tree, h, rows, rows.size, 28, fld, fld, PAD,
                               init_state=init)
    f = full[0]
    np.testing.assert_array_equal(b["nst"], f["nst"][rows])
    np.testing.assert_array_equal(b["p"], f["p"][rows])


@pytest.mark.parametrize("mode,kinds", [("reference", ("star",)),
                                        ("analytic", ("star", "mixed"))])
def test_dlnp_parity(small, mode, kinds):
    """convergence="dlnp" (island_solver.py:1210-1333) vs the oracle.

    dlnp accepts a step when the float64 chi2 decreases; once steps are
    tiny the two sides' per-band float64 sums (different summation orders,
    ~1e-16 relative) can disagree on such a near-tie, as the reference's own
    reductions can.  Fluxes and positions must meet the parity bar on every
    island; iteration counts and flags must agree on every island except
    such near-ties, each reported with its final chi2 difference in float32
    ulps and held to 1e-6 relative (on the B200: 1 island of 26)."""
    plans, hosts, PAD, ds, ws, psfs = field_classes(small, mode, kinds)
    g, _ = run_gpu(plans, hosts, PAD, ds, ws, psfs, mode, native=small.native,
                   convergence="dlnp")
    o = run_oracle(plans, hosts, PAD, ds, ws, psfs, mode, native=small.native,
                   convergence="dlnp")
    same = []
    for p, h, gg, oo in zip(plans, hosts, g, o):
        r = compare(gg, oo, h["mmask"])
        msg = f"{p.key}: {r['max_rel']:.2e} {r['max_dpos']:.2e}"
        assert r["flux_ok"].all() and r["pos_ok"].all(), msg
        ok = r["same_nst"] & r["same_flags"]
        for i in np.nonzero(~ok)[0]:
            c32, c64 = np.float32(gg["chi2"][i]), float(oo["chi2"][i])
            ulps = abs(float(c32) - c64) / float(np.spacing(c32))
            print(f"{p.key} island {i}: steps {gg['nst'][i]} vs {oo['nst'][i]}, final chi2 "
                  f"{float(c32):.9g} vs {c64:.9g} ({ulps:.1f} float32 ulps)")
            assert abs(float(c32) - c64) <= 1e-6 * abs(c64), msg
        same.append(ok)
    same = np.concatenate(same)
    assert same.mean() >= 0.9, same.mean()


def test_dlnp_zero_weight_island_is_certified(small):
    plans, hosts, PAD, ds, ws, psfs = field_classes(small, "analytic", ("star",))
    p, h = plans[0], hosts[0]
    ws2 = ws.copy()
    oy, ox = int(h["oy"][0]), int(h["ox"][0])
    ws2[:, oy:oy + p.bbox_class, ox:ox + p.bbox_class] = 0.0
    g, _ = run_gpu([p], [h], PAD, ds, ws2, psfs, "analytic", native=small.native,
                   convergence="dlnp")
    g = g[0]
    assert g["nst"][0] == 1 and g["conv"][0] and not g["stall"][0]
    assert g["stall_dchi2"][0] == 0.0


@pytest.mark.parametrize("mode,kinds", [("analytic", ("star", "mixed"))])
def test_trust_region_parity(small, mode, kinds):
    """step_mode="trust_region" (island_solver.py:1004-1116) on the mixed
    classes, clip on the star classes.  Iteration counts, flags and the
    bound-pinned flag agree on every island (they did on all 38 on the
    B200, although the radius update branches on the gain ratio of two
    float chi2 values), fluxes and positions meet the parity bar."""
    plans, hosts, PAD, ds, ws, psfs = field_classes(small, mode, kinds)
    g, _ = run_gpu(plans, hosts, PAD, ds, ws, psfs, mode, native=small.native,
                   step_mode="trust_region")
    o = run_oracle(plans, hosts, PAD, ds, ws, psfs, mode, native=small.native,
                   step_mode="trust_region")
    n_same = n_all = 0
    for p, h, gg, oo in zip(plans, hosts, g, o):
        r = compare(gg, oo, h["mmask"])
        msg = f"{p.key}: {r['max_rel']:.2e} {r['max_dpos']:.2e} " \
              f"gpu nst {gg['nst'].tolist()} oracle nst {oo['nst'].tolist()}"
        assert r["flux_ok"].all() and r["pos_ok"].all(), msg
        same = r["same_nst"] & r["same_flags"]
        n_same += int(same.sum())
        n_all += same.size
        np.testing.assert_array_equal(gg["railed"][same], oo["railed"][same])
        if p.kind == "star":
            assert not gg["railed"].any()
        else:
            assert np.all(gg["lam"][gg["nst"] > 0] > 0)   # a radius, never unset
    assert n_same == n_all, f"{n_same}/{n_all}"


def test_trust_region_radius_carries_across_requeue(small):
    """A re-queued chunk carrying the radius in lam equals one pass."""
    from uniphot_b200 import solver
    plans, hosts, PAD, ds, ws, psfs = field_classes(small, "analytic", ("mixed",))
    p, h = plans[0], hosts[0]
    full, fld = run_gpu([p], [h], PAD, ds, ws, psfs, "analytic", native=small.native,
                        step_mode="trust_region")
    a, _ = run_gpu([p], [h], PAD, ds, ws, psfs, "analytic", max_steps=2, field=fld,
                   native=small.native, step_mode="trust_region")
    a = a[0]
    tree, nt = solver.build_psf_tree(psfs, p.tier)
    kern = solver.make_class_kernels(p, ds.shape[0], nt, render_backend="fft", reg=1e-9,
                                     pos_step_max_pix=0.5, chi2_ftol_rel=1e-4,
                                     step_tol_pix=0.1, un_freeze_steps=0,
                                     render_mode="analytic", native_stamp=small.native,
                                     step_mode="trust_region")
    rows = np.nonzero(~a["conv"])[0]
    assert rows.size > 0
    init = {k: a[k][rows] for k in ("p", "lam", "chi2", "consec", "nrej", "nst")}
    b = solver.run_class_chunk(kern, tree, h, rows, rows.size, 28, fld, fld, PAD,
                               init_state=init)
    f = full[0]
    np.testing.assert_array_equal(b["nst"], f["nst"][rows])
    np.testing.assert_array_equal(b["p"], f["p"][rows])
    np.testing.assert_array_equal(b["lam"], f["lam"][rows])


def test_trust_region_production_field_parity():
    """Reduced production field (512^2, 3 bands, 300 sources), classes of at
    most 2 members: galaxies with bounded log-radius and free Sersic n
    exercise the bound-pinned disclosure.  Iteration counts and flags agree
    on every island (28 of 28 on the B200)."""
    from uniphot_b200.synth import make_production_field
    f = make_production_field(3, side=512, n_bands=3, n_src=300)
    plans, hosts, PAD, ds, ws, psfs = field_classes(f, "analytic", ("mixed",))
    keep = [i for i, p in enumerate(plans) if p.nsrc_class <= 2]
    plans = [plans[i] for i in keep]
    hosts = [hosts[i] for i in keep]
    g, _ = run_gpu(plans, hosts, PAD, ds, ws, psfs, "analytic", native=f.native,
                   step_mode="trust_region")
    o = run_oracle(plans, hosts, PAD, ds, ws, psfs, "analytic", native=f.native,
                   processes=8, step_mode="trust_region")
    n_same = n_all = n_railed = 0
    for p, h, gg, oo in zip(plans, hosts, g, o):
        r = compare(gg, oo, h["mmask"])
        assert r["flux_ok"].all() and r["pos_ok"].all(), \
            f"{p.key}: {r['max_rel']:.2e} {r['max_dpos']:.2e}"
        same = r["same_nst"] & r["same_flags"]
        n_same += int(same.sum())
        n_all += same.size
        np.testing.assert_array_equal(gg["railed"][same], oo["railed"][same])
        n_railed += int(oo["railed"].sum())
    assert n_same == n_all, f"{n_same}/{n_all}"
    assert n_railed > 0
