"""Generate the golden fixtures that pin the host logic and the oracle.

Runs the REFERENCE's own numpy modules (imported standalone from a reference
checkout, bypassing the package ``__init__`` which needs matplotlib):

* ``tract7dt/fit/grid_gpu/islands.py`` -- flux-aware radii, membership,
  bboxes, bucketing;
* ``tract7dt/fit/grid_gpu/island_plan.py`` -- class planning, host arrays,
  free-n gate;
* ``tract7dt/fit/grid_gpu/psf_polynomial.py`` -- numpy PSF stamp evaluation;
* ``tract7dt/fit/grid_gpu/sersic_mog.py`` -- the table loader;
* ``tract7dt/fit/grid_gpu/bg_polynomial.py`` -- the grid background basis.

Inputs are the seeded synthetic catalogs of ``uniphot_b200.synth``.  Output:
``tests/golden/*.npz``.  Usage (optionally naming the fixtures to write:
plan, psf, table, bg_basis)::

    python tests/golden/make_golden.py /root/reference [fixture ...]
"""

from __future__ import annotations

import importlib
import sys
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))


def load_reference(ref_root: str):
    root = Path(ref_root) / "tract7dt"
    for name, path in (("tract7dt", root), ("tract7dt.fit", root / "fit"),
                       ("tract7dt.fit.grid_gpu", root / "fit" / "grid_gpu")):
        mod = types.ModuleType(name)
        mod.__path__ = [str(path)]
        sys.modules[name] = mod
    mods = {}
    for m in ("islands", "island_plan", "psf_polynomial", "bg_polynomial",
              "sersic_mog"):
        mods[m] = importlib.import_module(f"tract7dt.fit.grid_gpu.{m}")
    return mods


def catalog_small(seed):
    from uniphot_b200.synth import make_small_field
    f = make_small_field(seed)
    return f


def catalog_field(seed):
    from uniphot_b200.synth import make_production_field
    return make_production_field(seed, side=512, n_bands=3, n_src=300)


def planning_fixture(ref, f, native, radius_mode, tier_ladder):
    isl_mod, plan_mod = ref["islands"], ref["island_plan"]
    n = f.pos_x.size
    r_psf = native / 2.0
    out = {}
    if radius_mode == "fof":
        radius = np.full(n, 4.0)
    else:
        sig = float(np.median([np.median(1.0 / np.sqrt(iv[::16, ::16][iv[::16, ::16] > 0]))
                               for iv in f.invvar]))
        stamp = f.poly_psfs[0].stamp_at(f.data_minus_bg.shape[2] / 2,
                                        f.data_minus_bg.shape[1] / 2)
        pr, pp = isl_mod.psf_radial_profile(stamp)
        radius = isl_mod.flux_aware_radii(
            f.source_type, f.logre, f.sersic_n, np.median(f.s1_flux, axis=1),
            sig, 0.5, pr, pp, r_psf)
        out.update(sigma_sky=sig, psf_r=pr, psf_p=pp, psf_stamp=stamp)
    iset = isl_mod.build_islands(f.pos_x, f.pos_y, f.source_type, f.logre,
                                 f.sersic_n, r_psf, radius=radius)
    bk = isl_mod.bucket_islands(iset, (32, 48, 64, 96, 128, 192, 256, 384),
                                (1, 2, 4, 8, 16, 32, 64))
    out.update(pos_x=f.pos_x, pos_y=f.pos_y, source_type=f.source_type,
               logre=f.logre, ee1=f.ee1, ee2=f.ee2, sersic_n=f.sersic_n,
               s1_flux=f.s1_flux, s1_flux_var=f.s1_flux_var, native=native,
               radius=iset.radius, labels=iset.labels, bbox=iset.bbox,
               n_src=iset.n_src, giant_ids=bk.giant_ids)
    free_n = plan_mod.free_n_gate(f.source_type, f.s1_flux, f.s1_flux_var,
                                  True, 30.0)
    out["free_n"] = free_n
    plans, capped = plan_mod.plan_island_classes(
        iset, bk, f.source_type, f.logre, f.sersic_n, native, joint_nsrc_cap=32)
    out["capped"] = np.asarray(capped, np.int64)
    keys = []
    for ci, p in enumerate(plans):
        keys.append([p.bbox_class, p.nsrc_class, 0 if p.kind == "star" else 1,
                     p.tier, p.n_gal_class])
        host = plan_mod.class_host_arrays(
            p, pos_x=f.pos_x, pos_y=f.pos_y, source_type=f.source_type,
            logre=f.logre, ee1=f.ee1, ee2=f.ee2, sersic_n=f.sersic_n,
            free_n_all=free_n, pos_max_shift_pix=5.0, pad=400)
        out[f"c{ci}_isl_ids"] = p.isl_ids
        for k in ("ox", "oy", "x0b", "y0b", "keep", "p0", "lower", "upper",
                  "prior_inv_sigma", "fn_flag", "mmask", "gsel", "gvalid"):
            out[f"c{ci}_{k}"] = host[k]
    out["class_keys"] = np.asarray(keys, np.int64).reshape(-1, 5)
    return out


def psf_fixture(ref):
    pp = ref["psf_polynomial"]
    rng = np.random.default_rng(11)
    out = {}
    for nt in (1, 3, 6, 10, 15):
        coefs = rng.normal(0, 1, (13, 11, nt)).astype(np.float32)
        psf = pp.PsfPolynomial(coefs, 1000.0, 900.0, 700.0, 650.0, 13, 11)
        xs = rng.uniform(0, 2000, 4)
        ys = rng.uniform(0, 1400, 4)
        out[f"nt{nt}_coefs"] = coefs
        out[f"nt{nt}_xy"] = np.stack([xs, ys], 1)
        out[f"nt{nt}_stamps"] = np.stack(
            [pp.evaluate_psf_at_np(psf, x, y) for x, y in zip(xs, ys)])
    return out


def table_fixture(ref):
    """Sampled rows plus SHA-256 digests of the reference table arrays."""
    import hashlib
    t = ref["sersic_mog"].load_table_np()
    rows = np.array([0, 43, 148, 348, 600, 748, 1148, 1208])
    out = {"rows": rows}
    for k in ("n_knots", "amps", "log_vars", "core_amp"):
        a = np.ascontiguousarray(np.asarray(t[k], np.float64))
        out[f"{k}_sha256"] = np.array(hashlib.sha256(a.tobytes()).hexdigest())
        out[f"{k}_rows"] = a[rows]
    out["n_min"] = np.asarray(t["n_min"])
    out["n_max"] = np.asarray(t["n_max"])
    return out


def bg_basis_fixture(ref):
    """The grid background basis at orders 0-2 on a few grid geometries."""
    bp = ref["bg_polynomial"]
    out = {}
    cases = [(37, 53, 0, 0, 1024.0, 1024.0, 1024.0, 1024.0),
             (41, 29, 300, 1700, 1000.5, 950.0, 1020.25, 990.0),
             (64, 64, 2048, 512, 2047.5, 2048.0, 2047.5, 2048.0)]
    for ci, (h, w, x0, y0, xo, xs, yo, ys) in enumerate(cases):
        out[f"case{ci}_geom"] = np.array([h, w, x0, y0, xo, xs, yo, ys], np.float64)
        for order in (0, 1, 2):
            out[f"case{ci}_o{order}"] = bp.make_bg_basis(h, w, x0, y0, xo, xs, yo, ys,
                                                         order=order)
    return out


def main(ref_root, which=None):
    ref = load_reference(ref_root)
    want = set(which or ("plan", "psf", "table", "bg_basis"))
    if "plan" in want:
        for seed in (0, 1):
            f = catalog_small(seed)
            np.savez_compressed(HERE / f"plan_small_s{seed}.npz",
                                **planning_fixture(ref, f, 55, "fof", (111, 221)))
        f = catalog_field(3)
        np.savez_compressed(HERE / "plan_field_s3.npz",
                            **planning_fixture(ref, f, 31, "flux", (111, 221)))
    if "psf" in want:
        np.savez_compressed(HERE / "psf_poly_eval.npz", **psf_fixture(ref))
    if "table" in want:
        np.savez_compressed(HERE / "sersic_table_ref.npz", **table_fixture(ref))
    if "bg_basis" in want:
        np.savez_compressed(HERE / "bg_basis_ref.npz", **bg_basis_fixture(ref))
    print("golden fixtures written to", HERE)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference", sys.argv[2:] or None)
