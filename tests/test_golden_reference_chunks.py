"""The oracle against the reference's chunk runner for the options
``island_fit`` does not expose.

``tests/golden/solver_chunk_*.npz`` hold the output dicts of the reference's
``make_class_kernels`` / ``run_class_chunk`` (island_solver.py:1874-1922,
2793-3131) on every class of the small field (the galaxy field for the second
trust-region case), made by
``tests/golden/make_golden_solver.py`` with its float64 numpy stand-in for
JAX: the trust-region step (``:1004-1116``), the marginal flux errors and
the band-coadded residual (``:1549-1637``), scene subtraction with the
member add-back (``:1795-1818``, ``:2781-2790``) and the cross-band GLS
(``:607-723``, ``:867-919``).  The oracle's float64 reference-render solve
of the same classes must give identical iteration counts and flags and the
same parameters, fluxes and pass outputs.
"""

from pathlib import Path

import numpy as np
import pytest

from _common import TABLE

GOLDEN = Path(__file__).parent / "golden"

CROSSBAND = {"rank": 2,
             "u": np.array([[0.6, 0.64, 0.48], [0.0, 0.6, -0.8]], np.float32),
             "lam": np.array([400.0, 60.0], np.float32)}

# case -> (oracle options, class_host_arrays extras, compared pass outputs
#          [, field name: the small field unless given])
CASES = {
    "chunk_trust_region": (dict(step_mode="trust_region"), lambda f: {}, ("railed",)),
    "chunk_flux_marg_residual": (dict(flux_marg=True, residual=True), lambda f: {},
                                 ("femarg", "resid", "resid_w")),
    "chunk_scene_subtract": (dict(scene_subtract=True), lambda f: {}, ()),
    "chunk_crossband": (dict(crossband=CROSSBAND),
                        lambda f: dict(cb_scale=np.linspace(0.5, 1.5, f.pos_x.size)), ()),
    "chunk_trust_region_galaxies": (dict(step_mode="trust_region"), lambda f: {},
                                    ("railed",), "galaxies"),
}


# The trust region on the galaxy field leaves two 4-member islands and a
# railed singleton on shapes where chi2 is flat (one ee2 runs to -12, where
# the axis ratio hits its cap of 1000): there the dogleg steps follow the
# generator's finite-difference derivatives and the shapes move by up to 1.0
# while chi2 agrees to 4e-6, positions to 3.4e-3 px and fluxes to 6e-3
# sigma.  That case compares the objective's determined quantities only.
LOOSE = {"chunk_trust_region_galaxies": dict(pos=5e-3, flux_sigma=1e-2, ferr=1e-2,
                                             chi2=1e-5, shapes=False)}


def _classes(f, host_extra):
    from uniphot_b200.plan import class_host_arrays, free_n_gate, plan_island_classes
    plans, _ = plan_island_classes(f.island_set, f.buckets, f.source_type, f.logre,
                                   f.sersic_n, f.native, tier_ladder=(111, 221))
    PAD = max(p.bbox_class for p in plans) + 8
    nb, H, W = f.data_minus_bg.shape
    ds = np.zeros((nb, H + 2 * PAD, W + 2 * PAD), np.float32)
    ws = np.zeros_like(ds)
    ds[:, PAD:PAD + H, PAD:PAD + W] = f.data_minus_bg
    ws[:, PAD:PAD + H, PAD:PAD + W] = f.invvar
    fn = free_n_gate(f.source_type, f.s1_flux, f.s1_flux_var, True, 30.0)
    hosts = [class_host_arrays(p, pos_x=f.pos_x, pos_y=f.pos_y, source_type=f.source_type,
                               logre=f.logre, ee1=f.ee1, ee2=f.ee2, sersic_n=f.sersic_n,
                               free_n_all=fn, pos_max_shift_pix=5.0, pad=PAD,
                               s1_flux=f.s1_flux, **host_extra)
             for p in plans]
    return plans, hosts, PAD, ds, ws


def _close(name, a, b, atol, rtol=0.0):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    assert a.shape == b.shape, f"{name}: shape {a.shape} vs {b.shape}"
    np.testing.assert_array_equal(np.isnan(a), np.isnan(b), err_msg=f"{name}: NaN pattern")
    ok = ~np.isnan(a)
    np.testing.assert_allclose(a[ok], b[ok], atol=atol, rtol=rtol, err_msg=name)


@pytest.mark.parametrize("case", sorted(CASES))
def test_oracle_matches_reference_chunk_runner(case):
    from oracle.driver import solve_chunk
    from test_golden_reference_solver import _digest, _field
    path = GOLDEN / f"solver_{case}.npz"
    if not path.exists():
        pytest.skip(f"fixture {path.name} not generated")
    ref = dict(np.load(path))
    f = _field(CASES[case][3] if len(CASES[case]) > 3 else "small")
    assert str(ref.pop("digest")) == _digest(f), "synthetic field changed since the fixture"
    opts, host_extra, cols = CASES[case][:3]
    plans, hosts, PAD, ds, ws = _classes(f, host_extra(f))
    by_key = {}
    for k, v in ref.items():
        ci, name = k.split("/", 1)
        by_key.setdefault(ci, {})[name] = v
    ref_classes = {tuple(int(x) for x in d["class"]): d for d in by_key.values()}
    assert len(ref_classes) == len(plans)
    for p, h in zip(plans, hosts):
        r = ref_classes[(p.bbox_class, p.nsrc_class, p.tier, int(p.kind == "star"))]
        np.testing.assert_array_equal(r["isl_ids"], p.isl_ids)
        o_opts = dict(opts)
        if p.kind == "star" and o_opts.get("step_mode") == "trust_region":
            o_opts["step_mode"] = "clip"     # star classes keep the clip step
        o = solve_chunk(h, np.arange(p.n_islands), B=p.bbox_class, T=p.tier, dstack=ds,
                        wstack=ws, psfs=f.poly_psfs, mode="reference", table_path=TABLE,
                        precision="f64", max_steps=30, native=f.native, **o_opts)
        tag = f"{case} class {p.bbox_class}/{p.nsrc_class}/{p.tier}/{p.kind}"
        for k in ("nst", "conv", "stall", "diverged"):
            np.testing.assert_array_equal(o[k], r[k], err_msg=f"{tag}: {k}")
        tol = dict(pos=1e-4, flux_sigma=1e-3, ferr=1e-4, chi2=1e-6, shapes=True)
        tol.update(LOOSE.get(case, {}))
        m = np.asarray(h["mmask"])
        pm = np.broadcast_to(m[:, :, None], o["p"].shape)
        op, rp = np.where(pm, o["p"], 0.0), np.where(pm, r["p"], 0.0)
        _close(f"{tag}: positions", op[..., :2], rp[..., :2], tol["pos"])
        if tol["shapes"]:
            _close(f"{tag}: shapes", op[..., 2:], rp[..., 2:], 1e-4)
        fm = np.broadcast_to(m[:, None, :], o["fluxes"].shape)
        df = np.abs(o["fluxes"] - r["fluxes"])
        bound = np.maximum(1e-5 * np.abs(r["fluxes"]), tol["flux_sigma"] * r["ferr"])
        assert np.all((df <= bound) | ~fm), f"{tag}: fluxes"
        _close(f"{tag}: ferr", np.where(fm, o["ferr"], 0.0), np.where(fm, r["ferr"], 0.0),
               0.0, tol["ferr"])
        _close(f"{tag}: chi2", o["chi2"], r["chi2"], 1e-3, tol["chi2"])
        # the plateau certificate, to 1e-3 absolute (the flat-shape case: to
        # the chi2 tolerance times the island's chi2)
        s_atol = 1e-3 if tol["chi2"] <= 1e-6 else tol["chi2"] * float(np.max(np.abs(r["chi2"])))
        _close(f"{tag}: stall_dchi2", o["stall_dchi2"], r["stall_dchi2"], s_atol, 1e-4)
        for k in cols:
            a, b = np.asarray(o[k], np.float64), np.asarray(r[k], np.float64)
            if k == "femarg":
                a, b = np.where(fm, a, 0.0), np.where(fm, b, 0.0)
            scale = max(float(np.nanmax(np.abs(b))), 1e-30) if b.size else 1.0
            _close(f"{tag}: {k}", a, b, 1e-6 * scale, 1e-4)
