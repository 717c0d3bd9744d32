"""Run the oracle over a solver class (test infrastructure only).

``solve_chunk`` mirrors ``run_class_chunk``'s result dict for a set of
class rows, island by island, optionally in a spawn-started process pool.
"""

from __future__ import annotations

import numpy as np

from .island_oracle import (IslandSolver, MogPsfBand, PolyPsfBand, SersicTable,
                            SolverConfig, island_inputs_from_host, solve_island)


def psf_bands(psfs, tier: int, mode: str):
    """Per-band oracle PSF objects (polynomial PSFs zero-padded to tier)."""
    out = []
    for p in psfs:
        if mode == "analytic":
            out.append(MogPsfBand(np.asarray(p.sigma, np.float64),
                                  np.asarray(p.e1, np.float64),
                                  np.asarray(p.e2, np.float64),
                                  np.asarray(p.weight, np.float64),
                                  float(p.x_origin), float(p.x_scale),
                                  float(p.y_origin), float(p.y_scale)))
        else:
            c = np.asarray(p.coefs, np.float32)
            H, W = c.shape[:2]
            if tier > H:
                z = np.zeros((tier, tier) + c.shape[2:], np.float32)
                y0, x0 = (tier - H) // 2, (tier - W) // 2
                z[y0:y0 + H, x0:x0 + W] = c
                c = z
            out.append(PolyPsfBand(c, float(p.x_origin), float(p.x_scale),
                                   float(p.y_origin), float(p.y_scale)))
    return out


def _one(args):
    (host, row, B, T, dstack, wstack, psf, table, mode, cfg, max_steps, native, bg, pe, fm, sm,
     rp, rs, ss, cb, rb) = args
    isl = island_inputs_from_host(host, row, B=B, T=T, dstack=dstack,
                                  wstack=wstack, psf=psf, table=table, mode=mode,
                                  native=native, bg_joint=bg)
    if rb is not None:
        isl.render_backend, isl.exp_mog = rb
    if cb is not None:
        isl.crossband = cb
        isl.cb_scale = float(np.asarray(host["cb_scale"])[row])
    if ss:
        add_back_members(isl, cfg, np.asarray(host["member_s1_flux"])[row])
    return solve_island(isl, cfg, max_steps, param_errors=pe, flux_marg=fm,
                        source_metrics=sm, re_profile=rp, residual=rs)


def add_back_members(isl, cfg, msf):
    """Scene subtract (island_solver.py:1795-1818, 2781-2790): the window
    data gain sum_k msf[k, b] m_k at the seed parameters, float32."""
    s = IslandSolver(isl, cfg)
    N = isl.stype.shape[0]
    data = isl.data.copy()
    for b in range(data.shape[0]):
        M, _ = s.models_band(b, isl.p0.astype(s.dt), False)
        add = np.tensordot(np.asarray(msf[:, b], np.float32), M[:N].astype(np.float32), 1)
        data[b] = (data[b] + add.astype(np.float32)).astype(np.float32)
    isl.data = data


def solve_chunk(host, rows, *, B, T, dstack, wstack, psfs, mode, table_path=None,
                precision="ref", max_steps=30, reg=1e-9, pos_step_max=0.5,
                ftol_rel=1e-4, step_tol=0.1, processes: int = 1, un_freeze_steps: int = 0,
                native: int = 0, bg_joint: bool = False,
                stall_count_mode: str = "proposals", convergence: str = "legacy",
                plateau_dlnp_tol: float = 0.5, step_mode: str = "clip",
                param_errors: bool = False, flux_marg: bool = False,
                source_metrics: bool = False, re_profile=None,
                residual: bool = False, scene_subtract: bool = False,
                crossband: dict | None = None, render_backend: str = "fft",
                exp_mog=None) -> dict:
    """``re_profile``: the log-radius offsets of the Re profile, or None;
    ``crossband``: the cross-band GLS channels ({"rank", "u", "lam"}, with
    the per-island scale from ``host["cb_scale"]``), or None;
    ``render_backend``: "fft" or the legacy "direct" (EXP galaxies from the
    exponential mixture ``exp_mog`` = (amp, var))."""
    table = SersicTable.load(table_path) if table_path is not None else None
    psf = psf_bands(psfs, T, mode)
    cfg = SolverConfig(reg=reg, pos_step_max=pos_step_max, ftol_rel=ftol_rel,
                       step_tol=step_tol, precision=precision,
                       un_freeze_steps=un_freeze_steps,
                       stall_count_mode=stall_count_mode, convergence=convergence,
                       plateau_dlnp_tol=plateau_dlnp_tol, step_mode=step_mode)
    jobs = [(host, int(r), B, T, dstack, wstack, psf, table, mode, cfg, max_steps,
             native, bg_joint, param_errors, flux_marg, source_metrics, re_profile, residual,
             scene_subtract, crossband,
             (render_backend, exp_mog) if render_backend != "fft" else None) for r in rows]
    if processes > 1 and len(jobs) > 1:
        import multiprocessing as mp
        with mp.get_context("spawn").Pool(processes) as pool:
            res = pool.map(_one, jobs, chunksize=max(1, len(jobs) // (4 * processes)))
    else:
        res = [_one(j) for j in jobs]
    out = {}
    for k in ("p", "fluxes", "ferr", "bg", "bg_err", "chi2", "conv", "stall", "diverged",
              "stall_dchi2", "nst", "lam", "consec", "nrej", "n_good", "n_same", "prej",
              "railed"):
        out[k] = np.stack([np.asarray(r[k]) for r in res])
    out["perr"] = np.stack([r["perr"] for r in res]) if param_errors else None
    out["femarg"] = np.stack([r["femarg"] for r in res]) if flux_marg else None
    out["smetrics"] = np.stack([r["smetrics"] for r in res]) if source_metrics else None
    out["swin"] = np.stack([r["swin"] for r in res]) if source_metrics else None
    out["reprof"] = np.stack([r["reprof"] for r in res]) if re_profile is not None else None
    out["resid"] = np.stack([r["resid"] for r in res]) if residual else None
    out["resid_w"] = np.stack([r["resid_w"] for r in res]) if residual else None
    out["steps_run"] = int(max(r["steps"] for r in res))
    return out


def solve_one_input(isl, cfg, max_steps: int = 30):
    """Pool entry: solve one prepared IslandInput."""
    return solve_island(isl, cfg, max_steps)


def solve_one_input_timed(isl, cfg, max_steps: int = 30):
    """Pool entry for timing the CPU path: (result, seconds spent solving
    inside the worker, excluding process start-up and transfers)."""
    import time
    t0 = time.perf_counter()
    res = solve_island(isl, cfg, max_steps)
    return res, time.perf_counter() - t0
