"""Shared helpers: build solver classes for a synthetic field and run the
CUDA path and the oracle on the same inputs."""
from __future__ import annotations

from pathlib import Path

import numpy as np

from uniphot_b200.plan import class_host_arrays, free_n_gate, plan_island_classes

ROOT = Path(__file__).resolve().parents[1]
TABLE = ROOT / "uniphot_b200" / "data" / "sersic_mog_table.npz"


def field_classes(f, mode: str, kinds=("star", "mixed"), priors: bool = False,
                  tier_ladder=None, free_n=None):
    """(plans, hosts, PAD, dstack, wstack, psfs) for a synthetic field;
    ``priors`` adds Gaussian priors on every member's position (0.3 px) and
    on galaxies' radius (50%), ellipticity (0.2), angle (20 deg) and Sersic
    index (1.0), centred on the seeds."""
    plans, _ = plan_island_classes(f.island_set, f.buckets, f.source_type, f.logre,
                                   f.sersic_n, f.native,
                                   tier_ladder=f.tier_ladder if tier_ladder is None else tier_ladder)
    plans = [p for p in plans if p.kind in kinds]
    PAD = max(p.bbox_class for p in plans) + 8
    nb, H, W = f.data_minus_bg.shape
    ds = np.zeros((nb, H + 2 * PAD, W + 2 * PAD), np.float32)
    ws = np.zeros_like(ds)
    ds[:, PAD:PAD + H, PAD:PAD + W] = f.data_minus_bg
    ws[:, PAD:PAD + H, PAD:PAD + W] = f.invvar
    fn = (free_n_gate(f.source_type, f.s1_flux, f.s1_flux_var, True, 30.0)
          if free_n is None else np.asarray(free_n, bool))
    pri = {}
    if priors:
        n = f.pos_x.size
        pri = dict(pos_err=np.full(n, 0.3), re_prior_sig=0.5 * np.exp(f.logre),
                   ell_prior_sig=np.full(n, 0.2), theta_prior_sig=np.full(n, 20.0),
                   sersic_n_prior_sig=np.full(n, 1.0))
    hosts = [class_host_arrays(p, pos_x=f.pos_x, pos_y=f.pos_y,
                               source_type=f.source_type, logre=f.logre, ee1=f.ee1,
                               ee2=f.ee2, sersic_n=f.sersic_n, free_n_all=fn,
                               pos_max_shift_pix=5.0, pad=PAD, s1_flux=f.s1_flux, **pri)
             for p in plans]
    psfs = f.mog_psfs if mode == "analytic" else f.poly_psfs
    return plans, hosts, PAD, ds, ws, psfs


def run_gpu(plans, hosts, PAD, ds, ws, psfs, mode, max_steps=30, field=None,
            native=0, precision="plain", tc_min_rows=-1, tc_cond_max=-1.0,
            bg_mode="frozen", stall_count_mode="proposals", convergence="legacy",
            step_mode="clip", param_errors=False, scene_subtract=False):
    from uniphot_b200 import solver
    if field is None:
        field = solver.DeviceField(ds, ws, PAD)
    outs = []
    for plan, host in zip(plans, hosts):
        tree, nt = solver.build_psf_tree(psfs, plan.tier)
        kern = solver.make_class_kernels(
            plan, ds.shape[0], nt, render_backend="fft", reg=1e-9,
            pos_step_max_pix=0.5, chi2_ftol_rel=1e-4, step_tol_pix=0.1,
            un_freeze_steps=0, has_priors=bool(host["has_priors"]), render_mode=mode,
            native_stamp=native, precision=precision, tc_min_rows=tc_min_rows,
            tc_cond_max=tc_cond_max, bg_mode=bg_mode, stall_count_mode=stall_count_mode,
            convergence=convergence, step_mode=step_mode, scene_subtract=scene_subtract)
        rows = np.arange(plan.n_islands)
        outs.append(solver.run_class_chunk(kern, tree, host, rows, rows.size,
                                           max_steps, field, field, PAD,
                                           compute_param_errors=param_errors))
    return outs, field


def run_oracle(plans, hosts, PAD, ds, ws, psfs, mode, precision="ref",
               max_steps=30, processes=1, native=0, bg_joint=False,
               stall_count_mode="proposals", convergence="legacy", step_mode="clip",
               param_errors=False, scene_subtract=False):
    """The oracle over every class (star classes keep the clip step, as the
    reference exempts them from the trust region)."""
    from oracle.driver import solve_chunk
    return [solve_chunk(h, np.arange(p.n_islands), B=p.bbox_class, T=p.tier,
                        dstack=ds, wstack=ws, psfs=psfs, mode=mode, table_path=TABLE,
                        precision=precision, max_steps=max_steps, processes=processes,
                        native=native, bg_joint=bg_joint,
                        stall_count_mode=stall_count_mode, convergence=convergence,
                        step_mode=step_mode if p.kind != "star" else "clip",
                        param_errors=param_errors, scene_subtract=scene_subtract)
            for p, h in zip(plans, hosts)]


def compare(g, o, mmask):
    """Per-island parity report between a GPU and an oracle result dict."""
    same_nst = g["nst"] == o["nst"]
    same_flags = (g["conv"] == o["conv"]) & (g["stall"] == o["stall"])
    fg, fo = g["fluxes"], o["fluxes"]
    sig = np.maximum(o["ferr"], 1e-30)
    m = np.broadcast_to(mmask[:, None, :], fg.shape)
    rel = np.abs(fg - fo) / np.maximum(np.abs(fo), 1e-30)
    flux_ok = (rel <= 1e-4) | (np.abs(fg - fo) <= 0.01 * sig)
    dp = np.abs(g["p"][..., :2] - o["p"][..., :2])
    pos_ok = dp <= 1e-3
    pm = np.broadcast_to(mmask[:, :, None], dp.shape)
    return dict(
        same_nst=same_nst, same_flags=same_flags,
        flux_ok=np.all(flux_ok | ~m, axis=(1, 2)),
        pos_ok=np.all(pos_ok | ~pm, axis=(1, 2)),
        max_rel=float(np.max(np.where(m, rel, 0))),
        max_dpos=float(np.max(np.where(pm, dp, 0))))
