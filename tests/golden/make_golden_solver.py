"""Golden vectors of the reference's own island solver.

Runs ``island_fit`` of ``tract7dt/fit/grid_gpu/island_solver.py`` from a
reference checkout on seeded synthetic fields of ``uniphot_b200.synth``,
with JAX replaced by the numpy stand-in of ``jax_stand_in.py`` (float64
arithmetic, central-difference linearisation; this container has no JAX).
Each case writes ``tests/golden/solver_<case>.npz``: every per-source array
of the returned ``IslandFitResult`` plus ``digest``, a hash of the field the
case ran on (the test checks it before comparing).  The ``chunk_*`` cases
call ``make_class_kernels`` / ``run_class_chunk`` (island_solver.py:1874-1922,
2793-3131) on every class of the small field for the options ``island_fit``
does not expose (trust-region step, marginal flux errors, residual export,
scene subtraction, cross-band GLS) and store each class's output dict under
``<class index>/<key>``.

Usage::

    python tests/golden/make_golden_solver.py /root/reference [case ...]

Cases run in separate processes when several are named.
"""

from __future__ import annotations

import hashlib
import importlib
import sys
import time
import types
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE))


def _small():
    from uniphot_b200.synth import make_small_field
    return make_small_field(0)


def _galaxies():
    from uniphot_b200.synth import make_production_field
    return make_production_field(4, side=320, n_bands=3, n_src=40, margin=40)


def _giants():
    from uniphot_b200.synth import make_production_field
    return make_production_field(1, side=320, n_bands=3, n_src=40, margin=40)


def _large():
    from uniphot_b200.synth import make_production_field
    return make_production_field(3, side=256, n_bands=3, n_src=30, margin=40)


def _blends():
    from uniphot_b200.synth import make_blend_field
    return make_blend_field(0, n_islands=6, n_bands=3)


def _priors(f):
    n = f.pos_x.size
    return dict(pos_err=np.full(n, 0.3), re_prior_sig=0.5 * np.exp(f.logre),
                ell_prior_sig=np.full(n, 0.2), theta_prior_sig=np.full(n, 20.0),
                sersic_n_prior_sig=np.full(n, 1.0))


_POST = dict(compute_param_errors=True, compute_source_metrics=True)

# case -> (field builder, extra island_fit arguments (a callable of the field))
CASES = {
    "small": (_small, lambda f: dict(_POST, compute_re_profile=True)),
    "small_priors": (_small, lambda f: dict(_priors(f), compute_param_errors=True)),
    "small_changed": (_small, lambda f: dict(stall_count_mode="changed")),
    "small_dlnp": (_small, lambda f: dict(convergence="dlnp")),
    # EXP galaxies on the legacy "direct" render backend
    "small_direct": (_small, lambda f: dict(render_backend="direct")),
    "galaxies": (_galaxies, lambda f: dict(_POST)),
    "galaxies_changed": (_galaxies, lambda f: dict(stall_count_mode="changed")),
    "galaxies_dlnp": (_galaxies, lambda f: dict(convergence="dlnp")),
    # the Sersic index of every SERSIC source fitted (free_n_override), with
    # and without the u_n annealing budget (n live only in the first 3 steps)
    "galaxies_free_n": (_galaxies, lambda f: dict(free_n_override=(f.source_type == 3))),
    "galaxies_free_n_unfreeze": (_galaxies, lambda f: dict(
        free_n_override=(f.source_type == 3), un_freeze_steps=3)),
    "blends": (_blends, lambda f: dict(_POST)),
    # a 34-member island above the joint cap of 32 takes the giant path
    "giants": (_giants, lambda f: dict(_POST)),
    # a 14-member mixed island (class of 16, tier 111) and an 8-member one
    "large": (_large, lambda f: dict(_POST)),
}


# Chunk-level cases: the reference's make_class_kernels / run_class_chunk on
# every class of a field (the small one unless named), for options island_fit
# does not expose.
# case -> (make_class_kernels arguments, run_class_chunk arguments,
#          class_host_arrays extras (a callable of the field)[, field builder])
CROSSBAND = {"rank": 2,
             "u": np.array([[0.6, 0.64, 0.48], [0.0, 0.6, -0.8]], np.float32),
             "lam": np.array([400.0, 60.0], np.float32)}
CHUNK_CASES = {
    "chunk_trust_region": (dict(step_mode="trust_region"), {}, lambda f: {}),
    "chunk_flux_marg_residual": ({}, dict(compute_flux_marg=True, want_residual=True),
                                 lambda f: {}),
    "chunk_scene_subtract": (dict(scene_subtract=True), {},
                             lambda f: dict(s1_flux=f.s1_flux)),
    "chunk_crossband": (dict(crossband=CROSSBAND), {},
                        lambda f: dict(cb_scale=np.linspace(0.5, 1.5, f.pos_x.size))),
    # the trust region on the galaxy field (stalls, long trajectories)
    "chunk_trust_region_galaxies": (dict(step_mode="trust_region"), {}, lambda f: {},
                                    _galaxies),
}


def field_digest(f) -> str:
    h = hashlib.sha256()
    for a in (f.data_minus_bg, f.invvar, f.pos_x, f.pos_y, f.source_type, f.logre, f.ee1,
              f.ee2, f.sersic_n, f.s1_flux, f.s1_flux_var):
        h.update(np.ascontiguousarray(a).tobytes())
    for p in f.poly_psfs:
        h.update(np.ascontiguousarray(p.coefs, np.float32).tobytes())
    return h.hexdigest()


def load_reference_solver(ref_root: str):
    import jax_stand_in
    jax_stand_in.install()
    root = Path(ref_root) / "tract7dt"
    for name, path in (("tract7dt", root), ("tract7dt.fit", root / "fit"),
                       ("tract7dt.fit.grid_gpu", root / "fit" / "grid_gpu"),
                       ("tract7dt.fit.optimize", root / "fit" / "optimize"),
                       ("tract7dt.fit.optimize.gpu", root / "fit" / "optimize" / "gpu"),
                       ("tract7dt.fit.optimize.gpu.kernels",
                        root / "fit" / "optimize" / "gpu" / "kernels")):
        mod = types.ModuleType(name)
        mod.__path__ = [str(path)]
        sys.modules[name] = mod
    solver = importlib.import_module("tract7dt.fit.grid_gpu.island_solver")
    psfmod = importlib.import_module("tract7dt.fit.grid_gpu.psf_polynomial")
    return solver, psfmod


def run_case(ref_root: str, case: str) -> None:
    solver, psfmod = load_reference_solver(ref_root)
    build, extra = CASES[case]
    f = build()
    psfs = [psfmod.PsfPolynomial(coefs=np.asarray(p.coefs, np.float32),
                                 x_origin=p.x_origin, x_scale=p.x_scale,
                                 y_origin=p.y_origin, y_scale=p.y_scale,
                                 H_psf=p.coefs.shape[0], W_psf=p.coefs.shape[1])
            for p in f.poly_psfs]
    kw = f.fit_kwargs("reference")
    for k in ("render_mode", "tier_ladder", "native_stamp"):
        kw.pop(k)
    kw["psfs"] = psfs
    t0 = time.time()
    res = solver.island_fit(**kw, **extra(f))
    arrays = {k: np.asarray(v) for k, v in vars(res).items() if isinstance(v, np.ndarray)}
    np.savez_compressed(HERE / f"solver_{case}.npz", digest=np.array(field_digest(f)),
                        **arrays)
    print(f"{case}: {len(arrays)} arrays, {time.time() - t0:.0f} s", flush=True)


def run_chunk_case(ref_root: str, case: str) -> None:
    solver, psfmod = load_reference_solver(ref_root)
    plan_mod = importlib.import_module("tract7dt.fit.grid_gpu.island_plan")
    kern_kw, run_kw, host_kw = CHUNK_CASES[case][:3]
    f = (CHUNK_CASES[case][3] if len(CHUNK_CASES[case]) > 3 else _small)()
    psfs = [psfmod.PsfPolynomial(coefs=np.asarray(p.coefs, np.float32),
                                 x_origin=p.x_origin, x_scale=p.x_scale,
                                 y_origin=p.y_origin, y_scale=p.y_scale,
                                 H_psf=p.coefs.shape[0], W_psf=p.coefs.shape[1])
            for p in f.poly_psfs]
    native = int(psfs[0].H_psf)
    plans, _ = plan_mod.plan_island_classes(f.island_set, f.buckets, f.source_type,
                                            f.logre, f.sersic_n, native)
    free_n = plan_mod.free_n_gate(f.source_type, f.s1_flux, f.s1_flux_var, True, 30.0)
    PAD = max(p.bbox_class for p in plans) + 8
    nb, H, W = f.data_minus_bg.shape
    ds = np.zeros((nb, H + 2 * PAD, W + 2 * PAD), np.float32)
    ws = np.zeros_like(ds)
    ds[:, PAD:PAD + H, PAD:PAD + W] = f.data_minus_bg
    ws[:, PAD:PAD + H, PAD:PAD + W] = f.invvar
    import jax.numpy as jnp
    out = {}
    t0 = time.time()
    for ci, plan in enumerate(plans):
        host = plan_mod.class_host_arrays(
            plan, pos_x=f.pos_x, pos_y=f.pos_y, source_type=f.source_type, logre=f.logre,
            ee1=f.ee1, ee2=f.ee2, sersic_n=f.sersic_n, free_n_all=free_n,
            pos_max_shift_pix=5.0, pad=PAD, **host_kw(f))
        tree, nt = solver.build_psf_tree(psfs, int(plan.tier))
        kern = solver.make_class_kernels(
            plan, nb, nt, render_backend="fft", reg=1e-9, pos_step_max_pix=0.5,
            chi2_ftol_rel=1e-4, step_tol_pix=0.1, un_freeze_steps=0,
            has_priors=bool(host["has_priors"]), **kern_kw)
        rows = np.arange(plan.n_islands)
        res = solver.run_class_chunk(kern, tree, host, rows, rows.size, 30, jnp.asarray(ds),
                                     jnp.asarray(ws), PAD, **run_kw)
        out[f"{ci}/class"] = np.array([plan.bbox_class, plan.nsrc_class, plan.tier,
                                       int(plan.kind == "star")])
        out[f"{ci}/isl_ids"] = np.asarray(plan.isl_ids)
        for k, v in res.items():
            if v is not None and not isinstance(v, (float, int, str)):
                v = np.asarray(v)
                # stored as float32, the precision of the reference's outputs
                out[f"{ci}/{k}"] = v.astype(np.float32) if v.dtype == np.float64 else v
    np.savez_compressed(HERE / f"solver_{case}.npz", digest=np.array(field_digest(f)),
                        **out)
    print(f"{case}: {len(plans)} classes, {time.time() - t0:.0f} s", flush=True)


def main(argv):
    ref_root = argv[1]
    cases = argv[2:] or list(CASES) + list(CHUNK_CASES)
    if len(cases) == 1:
        (run_chunk_case if cases[0] in CHUNK_CASES else run_case)(ref_root, cases[0])
        return
    import subprocess
    procs = [subprocess.Popen([sys.executable, __file__, ref_root, c]) for c in cases]
    rc = [p.wait() for p in procs]
    if any(rc):
        raise SystemExit(f"failed cases: {[c for c, r in zip(cases, rc) if r]}")


if __name__ == "__main__":
    main(sys.argv)
