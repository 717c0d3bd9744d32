"""Benchmark: islands/s of the per-island VarPro-LM forced-photometry solve.

Workload (one "step"): every fitted island of the synthetic production field
(2048x2048, 20 bands, 5000 sources: 60% STAR / 20% EXP / 12% DEV / 8% SERSIC,
4-component elliptical Gaussian-mixture PSF varying as an order-2 polynomial,
analytic render mode) solved to convergence (max 30 LM iterations) on one GPU.

* ``value``: islands/s at the metric's tolerance: the solve's islands/s with
  the field and every chunk's inputs already resident in HBM
  (``IslandFitJob.solve``; CUDA events on the library stream, synchronize +
  barrier on both sides, max over ranks) times the fraction of islands whose
  every flux is within 1e-4 relative or 0.01 sigma of the float64 oracle,
  estimated on a class-stratified sample (every class in it, >= 100
  islands).  ``forms.*.value_all_islands`` counts every island.  The field
  stacks (671 MB) exceed L2, so no explicit flush is needed between steps.
  The LM-loop engine of each form is picked by ``IslandFitJob.autotune``
  before the warm-up (``autotune`` in the line).
* ``e2e``: the same metric through the public API ``island_fit(...)`` from
  host arrays: planning, field + inputs host->device, solve, results
  device->host, unpack.
* ``roofline``: the dominant kernel of an instrumented solve against its
  binding peak, and the t_lb model over every kernel kind (bytes / HBM,
  flops / pipe, exp2 / SFU; HBM and BF16 from MEASURED_PEAKS.json, FP32,
  FP64 and exp2f measured in the run).
* ``cpu_baseline``: the CPU restatement of the reference algorithm (the
  oracle, reference precision) on a seeded 1% sample of the same islands,
  every sampled island solved and timed inside its worker, over all host
  cores: islands x cores / core-seconds.

``--impl reference`` prints the reference arm: the same CPU measurement,
since the reference's own JAX solver is installed neither here nor on the
GPU box.  ``--batched``, ``--precision-stress``, ``--reference-render`` and
``--serve-only`` print the other configurations' lines.

Multi-GPU (torchrun): weak scaling, every rank solves its own seeded field
(islands are independent: no collective on the data path); time = max over
ranks.  ``--split-field``: strong scaling, the ranks split one field's
islands by longest processing time (``shard.shard_plan``).
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))
# chunks run on up to 32 streams: give them as many hardware queues (read at
# CUDA context creation, so before torch touches the device)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

METRIC = ("islands/s at <=1e-4 rel flux err vs FP64 (plain vs batched+mixed); "
          "p50/p99 serve latency")
WORKLOAD = ("production field 2048x2048, 20 bands, 5000 sources "
            "(60/20/12/8% STAR/EXP/DEV/SERSIC), 4-Gaussian order-2 PSF, "
            "analytic render, max 30 LM steps")


def _peaks():
    """(HBM GB/s, bf16 TFLOP/s burst, bf16 TFLOP/s sustained, source)."""
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return (float(d["hbm_gbs"]), float(d["bf16_tflops"]),
                float(d.get("bf16_tflops_sustained", d["bf16_tflops"])), "measured")
    return 6650.0, 1590.0, 1400.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    def __init__(self, index: int = 0):
        self.index = index
        self.rows = []
        self.proc = None

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                 "-i", str(self.index), "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4)
                          if len(r) > 5 + i and r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def _config(n_isl: int, world: int) -> dict:
    """The workload's config keys, shared by both arms."""
    return {"workload": WORKLOAD, "n_islands": n_isl,
            "l2": "inputs (671 MB field) larger than L2",
            "parallelism": f"dp{world} (island partition by field)"}


def make_field(seed: int, device: str):
    from uniphot_b200.synth import make_production_field
    return make_production_field(seed, device=device)


def _sample_rows(classes, frac: float, seed: int, min_n: int = 8):
    """Seeded sample of (class index, row) over all fitted islands."""
    allr = [(ci, r) for ci, c in enumerate(classes) for r in range(c[0].n_islands)]
    rng = np.random.default_rng(seed)
    n = max(min_n, int(round(frac * len(allr))))
    pick = rng.choice(len(allr), size=min(n, len(allr)), replace=False)
    return [allr[i] for i in sorted(pick)]


def _stratified_rows(classes, target: int, seed: int):
    """Class-stratified seeded sample: at least one island of every class
    (so every 8-, 16- and 32-member class is in it), the rest in proportion
    to the classes' sizes."""
    total = sum(c[0].n_islands for c in classes)
    rng = np.random.default_rng(seed)
    out = []
    for ci, c in enumerate(classes):
        n = c[0].n_islands
        k = min(n, max(1, int(round(target * n / total))))
        out += [(ci, int(r)) for r in np.sort(rng.choice(n, size=k, replace=False))]
    return out


def _island_cost(classes, ci):
    p = classes[ci][0]
    return p.nsrc_class * p.bbox_class ** 2 * max(p.tier, 31)


def cpu_oracle_time(classes, PAD, field, sample, precision="ref", processes=None):
    """Solve every sampled island with the oracle over all host cores
    (spawn pool, heaviest islands first).  Each island is timed inside its
    worker, so pool start-up and transfers are excluded.  Returns
    ([((ci, row), result)], per-island seconds, processes, wall seconds)."""
    from oracle.driver import psf_bands
    from oracle.island_oracle import (SersicTable, SolverConfig,
                                      island_inputs_from_host)
    import multiprocessing as mp
    from oracle import driver
    procs = processes or len(os.sched_getaffinity(0))
    nb, H, W = field.data_minus_bg.shape
    ds = np.zeros((nb, H + 2 * PAD, W + 2 * PAD), np.float32)
    ws = np.zeros_like(ds)
    ds[:, PAD:PAD + H, PAD:PAD + W] = field.data_minus_bg
    ws[:, PAD:PAD + H, PAD:PAD + W] = field.invvar
    table = SersicTable.load(ROOT / "uniphot_b200" / "data" / "sersic_mog_table.npz")
    cfg = SolverConfig(precision=precision)
    order = sorted(range(len(sample)), key=lambda i: -_island_cost(classes, sample[i][0]))
    jobs = []
    for i in order:
        ci, r = sample[i]
        plan, host = classes[ci][0], classes[ci][1]
        psf = psf_bands(field.mog_psfs, plan.tier, "analytic")
        isl = island_inputs_from_host(host, r, B=plan.bbox_class, T=plan.tier,
                                      dstack=ds, wstack=ws, psf=psf, table=table,
                                      mode="analytic", native=field.native)
        jobs.append((isl, cfg))
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(procs) as pool:
        res = pool.starmap(driver.solve_one_input_timed, jobs, chunksize=1)
    wall = time.perf_counter() - t0
    done = [None] * len(sample)
    secs = [0.0] * len(sample)
    for i, (r, dt) in zip(order, res):
        done[i] = (sample[i], r)
        secs[i] = dt
    return done, secs, procs, wall


def _cpu_baseline(classes, PAD, field, seed=1):
    """The CPU restatement at reference precision on a seeded 1% island
    sample: every sampled island solved, islands/s = islands x cores /
    (sum of the islands' solve times), i.e. the throughput of that many
    cores solving independent islands."""
    sample = _sample_rows(classes, 0.01, seed)
    done, secs, procs, wall = cpu_oracle_time(classes, PAD, field, sample)
    v = len(done) * procs / float(np.sum(secs))
    return {"value": v, "unit": "islands/s", "cores": procs, "kind": "port",
            "sample": f"seeded 1% island sample (seed {seed}): all {len(done)} islands solved "
                      f"by the oracle at reference precision (float32 render and Gram, "
                      f"float64 solves), {np.sum(secs):.1f} core-s inside {procs} workers "
                      f"({wall:.1f} s wall); value = islands x cores / core-s"}


def _flux_quality(get, classes, ref64, weights=None):
    """Per-flux error against the float64 oracle on the sampled islands;
    ``weights`` maps a class index to its islands per sampled island (the
    stratified estimator of the field-wide fraction of islands whose every
    flux passes)."""
    rel, ok, isl_ok, isl_w, by_n = [], [], [], [], {}
    for (ci, r), o in ref64:
        mm = classes[ci][1]["mmask"][r]
        fg = get(ci)["fluxes"][r][:, mm]
        fo = o["fluxes"][:, mm]
        so = o["ferr"][:, mm]
        d = np.abs(fg - fo)
        good = (d <= 1e-4 * np.abs(fo)) | (d <= 0.01 * so)
        rel.append((d / np.maximum(np.abs(fo), 1e-30)).ravel())
        ok.append(good.ravel())
        isl_ok.append(bool(good.all()))
        isl_w.append(1.0 if weights is None else weights[ci])
        n = classes[ci][0].nsrc_class
        if n >= 8:
            by_n.setdefault(n, []).append(float(good.mean()))
    if not rel:
        return None
    e = np.concatenate(rel)
    w = np.asarray(isl_w)
    return {"frac_within_1e-4_rel_or_0.01sigma": float(np.mean(np.concatenate(ok))),
            "islands_all_fluxes_pass_weighted": float(np.sum(w * np.asarray(isl_ok)) / w.sum()),
            "islands_all_fluxes_pass_sample": float(np.mean(isl_ok)),
            "frac_by_class_nsrc": {str(k): float(np.mean(v)) for k, v in sorted(by_n.items())},
            "rel_median": float(np.median(e)), "rel_p99": float(np.quantile(e, 0.99)),
            "n_fluxes": int(e.size)}


def _roofline_model(ktab, wall_ms, peaks):
    """The t_lb model: per kernel kind the time its algorithmic work needs at
    the binding peak -- max(bytes / HBM, flops / pipe peak, exp2 / SFU) --
    and the whole solve's achieved fraction sum(t_lb) / wall.  Pipe peaks:
    the tensor-core Gram at a third of the dense BF16 rate (three BF16
    products per FP32 product: hi*hi, hi*lo, lo*hi), the FP32 Gram and the
    render at the FP32 multiply-add rate, the float64 step and assembly at
    the FP64 rate."""
    pipe = {"gram_tc": (peaks["bf16_tflops"] / 3.0, "tensor"),
            "gram": (peaks["fp32_tflops"], "fp32"), "render": (peaks["fp32_tflops"], "fp32"),
            "step": (peaks["fp64_tflops"], "fp64"), "assemble": (peaks["fp64_tflops"], "fp64")}
    kinds, tsum = {}, 0.0
    for k, d in ktab.items():
        terms = {"hbm": d["alg_bytes"] / (peaks["hbm_gbs"] * 1e9)}
        if d["alg_flops"] > 0 and k in pipe:
            terms[pipe[k][1]] = d["alg_flops"] / (pipe[k][0] * 1e12)
        if d.get("alg_exps", 0) > 0:
            terms["sfu"] = d["alg_exps"] / (peaks["exp2_tera_per_s"] * 1e12)
        bound = max(terms, key=terms.get)
        t_lb = terms[bound] * 1e3
        tsum += t_lb
        kinds[k] = {"t_lb_ms": t_lb, "bound": bound, "ms_serialised": d["ms"],
                    "frac_of_serialised": t_lb / d["ms"] if d["ms"] > 0 else None}
    return {"sum_t_lb_ms": tsum, "wall_ms": wall_ms, "frac": tsum / wall_ms,
            "kinds": kinds}


def run_reference_arm(args, rank, world):
    if rank != 0:
        print(json.dumps({"impl": "reference", "rank": rank, "skipped": True}),
              file=sys.stderr)
        return
    import torch  # noqa: F401  -- generation uses torch on whatever is present
    dev = "cuda" if torch.cuda.is_available() else "cpu"
    field = make_field(args.seed, dev)
    from uniphot_b200.solver import plan_field
    # host-side class planning only; the oracle does all the arithmetic
    fp = plan_field(**field.fit_kwargs("analytic"))
    n_isl = sum(p.n_islands for p, _ in fp.classes)
    base = _cpu_baseline(fp.classes, fp.PAD, field)
    v = base["value"]
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "islands/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 render and Gram, f64 inner solves (reference precision)",
        "data": "synthetic (seeded production field)",
        "config": _config(n_isl, 1),
        "cpu_baseline": base,
        "note": "the reference's JAX solver is not installed here or on the GPU box "
                "(no jax module), so this arm times the CPU restatement of its "
                "algorithm; the sampled islands are solved once (the same sample and "
                "method as the GPU arm's cpu_baseline)",
        "e2e": {"value": v, "unit": "islands/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0}}))


def _reference_render_measure(args, local):
    """islands/s of the production field in the reference render mode:
    the same catalog with the band PSFs as pixelised polynomials."""
    import torch
    from uniphot_b200.solver import IslandFitJob
    from uniphot_b200.synth import make_production_field
    field = make_production_field(args.seed, device="cuda", side=args.side, n_src=args.n_src)
    kw = field.fit_kwargs("reference")
    kw["precision"] = args.precision
    job = IslandFitJob(**kw, device=local)
    stream = torch.cuda.ExternalStream(job.field.ctx.stream_ptr())
    for _ in range(args.warmup):
        job.solve()
    ms, launches = _timed_solves(job, args.steps, stream, torch.cuda.synchronize, None)
    n_gal = int(np.sum(np.asarray(field.source_type) != 0))
    out = {"value": job.n_islands * args.steps / (ms / 1e3), "unit": "islands/s",
           "ms_per_step": ms / args.steps, "n_islands": job.n_islands,
           "galaxies": n_gal, "precision": args.precision, "gpu_launches": int(launches),
           "workload": WORKLOAD.replace("analytic render", "reference render (pixelised "
                                        "polynomial PSF; galaxies by Fourier-domain "
                                        "convolution)")}
    job.close()
    return out


def _timed_solves(job, steps, stream, barrier, dist):
    """Device time (ms) of `steps` solves, max over ranks, and launches."""
    import torch
    launches = 0
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    barrier()
    e0.record(stream)
    for _ in range(steps):
        job.solve()
        launches += job.field.ctx.last_launch_count()
    e1.record(stream)
    barrier()
    ms = e0.elapsed_time(e1)
    if dist is not None:
        t = torch.tensor([ms], device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
    return ms, launches


class _ClassRun:
    """One class (its first n islands) of a planned field as its own job."""

    def __init__(self, job, field, kw, args):
        import inspect
        from uniphot_b200 import _lib
        from uniphot_b200.solver import (IslandFitJob, _slice_host, build_psf_tree,
                                         make_class_kernels)
        b, n, kind, t = args.only_class.split(",")
        key = (int(b), int(n), kind, int(t))
        plan, host = next((p, h) for p, h, _ in job.classes if p.key == key)
        d = {k: v.default for k, v in inspect.signature(IslandFitJob).parameters.items()}
        tree, nt = build_psf_tree(kw["psfs"], plan.tier)
        nb = len(kw["bandnames"])
        kern = make_class_kernels(
            plan, nb, nt, render_backend=d["render_backend"], reg=d["reg"],
            pos_step_max_pix=d["pos_step_max_pix"], chi2_ftol_rel=d["chi2_ftol_rel"],
            step_tol_pix=d["step_tol_pix"], un_freeze_steps=d["un_freeze_steps"],
            has_priors=bool(host["has_priors"]), render_mode="analytic",
            native_stamp=field.native, precision=args.precision)
        rows = np.arange(min(args.class_islands, plan.n_islands))
        self.job = _lib.Job(job.field.ctx)
        self.job.add_chunk(kern.desc, _slice_host(host, rows), nb)
        self.n_islands = int(rows.size)
        self.max_steps = int(d["max_steps"])

    def solve(self):
        self.job.solve(self.max_steps)


def _class_job(job, field, kw, args):
    return _ClassRun(job, field, kw, args)


def _stress_measure(args, device):
    """Crowded blends vs the float64 oracle, plain and mixed forms: per-flux
    relative error, pass fraction at 1e-4 relative or 0.01 sigma, position
    error, and islands/s of each form on the whole field."""
    import torch
    from uniphot_b200.solver import IslandFitJob
    from uniphot_b200.synth import make_blend_field
    field = make_blend_field(args.seed, n_islands=args.stress_islands, n_bands=40,
                             device="cuda")
    kw = field.fit_kwargs("analytic")
    out = {"workload": f"{args.stress_islands} blends of 2-12 point sources 0.3-1.5 "
                       f"FWHM apart, flux ratios log-U up to 1e4, 40 bands (a quarter "
                       f"at SNR 3-10 for faint members), production PSF",
           "refinement_iterations_per_linearisation": {"plain": 0, "mixed": 1}}
    jobs = {}
    for prec in ("plain", "mixed"):
        job = IslandFitJob(**dict(kw, precision=prec), device=device)
        for _ in range(2):
            job.solve()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        job.solve()
        torch.cuda.synchronize()
        out.setdefault("islands_per_s", {})[prec] = job.n_islands / (time.perf_counter() - t0)
        jobs[prec] = job
    out["n_islands"] = jobs["plain"].n_islands
    sample = _sample_rows(jobs["plain"].classes, 0.0, 3, min_n=args.stress_sample)
    nb, H, W = field.data_minus_bg.shape
    ref64, _, _, _ = cpu_oracle_time(jobs["plain"].classes, jobs["plain"].PAD, field,
                                     sample, precision="f64")
    out["fp64_sample_islands"] = len(ref64)
    for prec, job in jobs.items():
        get = _class_results(job)
        q = _flux_quality(get, job.classes, ref64)
        dpos = []
        for (ci, r), o in ref64:
            mm = job.classes[ci][1]["mmask"][r]
            dpos.append(np.abs(get(ci)["p"][r][mm, :2] - o["p"][mm, :2]).max(axis=1))
        dp = np.concatenate(dpos) if dpos else np.zeros(0)
        q["pos_err_px_median"] = float(np.median(dp)) if dp.size else None
        q["pos_err_px_max"] = float(dp.max()) if dp.size else None
        q["frac_pos_within_1e-3_px"] = float(np.mean(dp <= 1e-3)) if dp.size else None
        nst = np.concatenate([get(ci)["nst"] for ci in range(len(job.classes))])
        q["lm_iterations"] = {"median": float(np.median(nst)), "p90": float(np.percentile(nst, 90)),
                              "max": int(nst.max())}
        if prec == "mixed":
            # the conditioning indicator of every island (worst band) at the
            # final parameters, over the whole field, and the sampled fluxes'
            # pass fraction by its range
            ac = np.concatenate([np.nanmax(get(ci)["acond"], axis=1)
                                 for ci in range(len(job.classes))])
            edges = (1.0, 10.0, 1e3, 1e6, np.inf)
            q["conditioning"] = {
                "what": "pivot spread of the f64 elimination of each band's diagonally "
                        "scaled member normal matrix (worst band), final parameters",
                "p50": float(np.percentile(ac, 50)), "p90": float(np.percentile(ac, 90)),
                "p99": float(np.percentile(ac, 99)), "max": float(ac.max()),
                "frac_above_tc_cond_max_10": float(np.mean(ac > 10.0)),
                "islands_by_range": {f"{lo:g}-{hi:g}": int(np.sum((ac >= lo) & (ac < hi)))
                                     for lo, hi in zip(edges[:-1], edges[1:])}}
            passed = {}
            for (ci, r), o in ref64:
                a = float(np.nanmax(get(ci)["acond"][r]))
                mm = job.classes[ci][1]["mmask"][r]
                f, f64 = get(ci)["fluxes"][r][:, mm], o["fluxes"][:, mm]
                d = np.abs(f - f64)
                ok = (d <= 1e-4 * np.abs(f64)) | (d <= 0.01 * o["ferr"][:, mm])
                key = next(f"{lo:g}-{hi:g}" for lo, hi in zip(edges[:-1], edges[1:]) if a < hi)
                n_ok, n_all = passed.get(key, (0, 0))
                passed[key] = (n_ok + int(ok.sum()), n_all + int(ok.size))
            q["conditioning"]["sample_flux_pass_by_range"] = {
                k: {"fluxes": n, "frac_within": ok / n} for k, (ok, n) in sorted(passed.items())}
        out[prec] = q
        job.close()
    return out


def _batched_measure(args, device):
    """The batched configuration: ``args.batched_tiles`` distinct 2048^2
    production-style tiles (the production field's generator at its source
    density, 60/20/12/8% STAR/EXP/DEV/SERSIC, clustered islands of 1-64
    members) for each band count 5, 20 and 40.  A band count's tiles are
    packed into one job (every tile's chunks bound to its own field and PSF;
    tiles beyond the device budget go to the next job), the LM-loop engine
    picked by the autotuner on the first job (per-chunk engine or work queue
    with 16 lanes).  The ``args.batched_islands`` island stream is that job
    solved repeatedly: islands/s per band count and form is the job's
    islands over its device time per solve, and the whole configuration's
    islands/s weights the three band counts equally (a third of the stream
    each).  Per member-count class on the first 20-band tile.  Islands above
    32 members keep their seeds (giant rows, the reference's joint cap) and
    are counted apart.  Host memory holds one band count's tiles at a
    time."""
    import dataclasses
    import gc
    import torch
    from uniphot_b200 import _lib
    from uniphot_b200.solver import DeviceField, IslandFitJob, estimate_device_bytes, plan_field
    from uniphot_b200.synth import make_production_field

    def timed(job, steps):
        stream = torch.cuda.ExternalStream(job.field.ctx.stream_ptr())
        job.solve()
        ms, _ = _timed_solves(job, steps, stream, torch.cuda.synchronize, None)
        return ms / steps

    def solve_packed(tiles, prec, tune_first, tuning):
        """Device ms of one pass over the tiles, packed into jobs under the
        device budget; the engine picked on the first job."""
        budget, total, njobs, groups, cur, used = 120e9, 0.0, 0, [], [], 0.0
        for kw, fp in tiles:
            nb, H, W = np.shape(kw["data_minus_bg"])
            need = estimate_device_bytes(fp, nb, H, W, precision=prec)
            if cur and used + need > budget:
                groups.append(cur)
                cur, used = [], 0.0
            cur.append((kw, fp))
            used += need
        groups.append(cur)
        for grp in groups:
            ctx = _lib.Context(device)
            job = _lib.Job(ctx)
            fits = []
            for kw, fp in grp:
                fld = DeviceField.from_unpadded(kw["data_minus_bg"], kw["invvar"], fp.PAD,
                                                device=device, context=ctx)
                fits.append(IslandFitJob(**dict(kw, precision=prec), device=device,
                                         field=fld, plan=fp, job=job))
            if tune_first and tuning is None:
                tuning = fits[-1].autotune(candidates=(("chunks", 0), ("queue", 16)),
                                           repeats=1)
            elif tuning is not None:
                eng, lanes = tuning["picked"].split("/")
                job.set_engine(eng, int(lanes))
            total += timed(fits[-1], args.batched_steps)
            njobs += 1
            job.close()
            ctx.close()
        return total, tuning, njobs

    def solve_alone(kw, fp, prec):
        job = IslandFitJob(**dict(kw, precision=prec), device=device, plan=fp)
        ms = timed(job, args.batched_steps)
        job.close()
        job.field.ctx.close()
        return ms

    out = {"target_islands": args.batched_islands, "tiles_per_band_count": args.batched_tiles,
           "band_counts": [5, 20, 40], "fields": []}
    tuning = {"plain": None, "mixed": None}
    for k, nb in enumerate((5, 20, 40)):
        t0 = time.perf_counter()
        tiles = []
        for t in range(args.batched_tiles):
            f = make_production_field(args.seed + 101 * k + 7 * t, side=2048, n_bands=nb,
                                      n_src=5000, device="cuda")
            kw = f.fit_kwargs("analytic")
            tiles.append((kw, plan_field(**kw)))
            del f
        row = {"n_bands": nb, "tiles": len(tiles), "side": 2048, "n_src_per_tile": 5000,
               "generation_s": time.perf_counter() - t0,
               "n_islands": sum(sum(p.n_islands for p, _ in fp.classes) for _, fp in tiles),
               "giant_islands": sum(int(len(fp.capped)) for _, fp in tiles)}
        for prec in ("plain", "mixed"):
            ms, tuning[prec], njobs = solve_packed(tiles, prec, True, tuning[prec])
            row[prec] = {"islands_per_s": row["n_islands"] / (ms / 1e3), "ms_per_solve": ms,
                         "jobs": njobs, "autotune": tuning[prec]}
            if nb == 20:
                kw, fp = tiles[0]
                groups = {}
                for p, h in fp.classes:
                    groups.setdefault(int(p.nsrc_class), []).append((p, h))
                per_class = {}
                for nsrc, cl in sorted(groups.items()):
                    sub = dataclasses.replace(fp, classes=cl, capped=[])
                    m = sum(p.n_islands for p, _ in cl)
                    msc = solve_alone(kw, sub, prec)
                    per_class[str(nsrc)] = {"islands": m, "islands_per_s": m / (msc / 1e3),
                                            "ms_per_solve": msc}
                row[prec]["by_member_class_first_tile"] = per_class
        out["fields"].append(row)
        del tiles
        gc.collect()
        torch.cuda.empty_cache()
    for prec in ("plain", "mixed"):
        # a third of the island stream per band count: harmonic weighting
        per_isl_s = sum(1.0 / r[prec]["islands_per_s"] for r in out["fields"]) / 3.0
        out[prec + "_islands_per_s"] = 1.0 / per_isl_s
        out[prec + "_stream_seconds"] = args.batched_islands * per_isl_s
    out["n_islands_distinct"] = sum(r["n_islands"] for r in out["fields"])
    return out


def _serve_measure(args, rates, device):
    """Serving: the same seeded request pool streamed with Poisson arrivals
    through the packing server (admitted requests solved as one job, mixed
    precision; its LM loop on the per-chunk engine, and on the work-queue
    engine), through the batched+mixed server (worker contexts overlapping
    on the device) and through one plain FP32 worker (one request at a
    time)."""
    from uniphot_b200.serve import PackedServer, Server, latency_summary, poisson_stream
    from uniphot_b200.synth import make_serving_request
    pool = [make_serving_request(i, device="cuda").fit_kwargs("analytic")
            for i in range(args.serve_requests)]
    out = {"requests": len(pool), "workers": args.serve_workers,
           "hbm_budget_bytes": 160e9,
           "request_shapes": "cutout side log-normal 64-1024 px, bands U{1..40}, "
                             "sources 5-2000 at the production density, PSF "
                             "polynomial coefficients drawn per request",
           "rates": []}
    def packed(engine):
        return lambda prec: PackedServer(device=device, planners=4, engines=4,
                                         hbm_budget_bytes=160e9, precision=prec,
                                         engine=engine)

    def workers(n):
        return lambda prec: Server(device=device, workers=n, hbm_budget_bytes=160e9,
                                   precision=prec)

    forms = (("packed_mixed", "mixed", packed("chunks"), 4),
             ("packed_mixed_queue", "mixed", packed("queue"), 4),
             ("batched_mixed", "mixed", workers(args.serve_workers), args.serve_workers),
             ("one_at_a_time_plain", "plain", workers(1), 1))
    for name, prec, make, warm in forms:
        with make(prec) as srv:
            # warm-up: every request of the pool once (so that every kernel
            # the stream uses is loaded, whichever form runs first), then one
            # per worker or engine
            for f in [srv.submit(dict(kw, precision=prec)) for kw in pool]:
                f.result()
            for f in [srv.submit(dict(pool[i % len(pool)], precision=prec))
                      for i in range(warm)]:
                f.result()
        for rate in rates:
            with make(prec) as srv:
                futs = poisson_stream(srv, [dict(kw, precision=prec) for kw in pool],
                                      rate, seed=7)
                for f in futs:
                    f.result()
            summ = latency_summary(srv.stats)
            summ["peak_admitted_bytes"] = srv.peak_in_use
            if hasattr(srv, "packs"):
                summ["packs"] = len(srv.packs)
                summ["mean_pack_size"] = float(np.mean(srv.packs))
            row = next((r for r in out["rates"] if r["rate_hz"] == rate), None)
            if row is None:
                row = {"rate_hz": rate}
                out["rates"].append(row)
            row[name] = summ
    return out


def _kernel_table(job):
    """Instrumented solve: per kind device ms, launches and algorithmic work."""
    job.job.set_profile(True)
    job.solve()
    kt = job.job.kernel_times()
    kw = job.job.kernel_work()
    job.job.set_profile(False)
    out = {}
    for k, (ms, n) in kt.items():
        if n == 0:
            continue
        by, fl, ex = kw[k]
        out[k] = {"ms": ms, "launches": n, "alg_bytes": by, "alg_flops": fl,
                  "alg_exps": ex,
                  "gbs": by / (ms * 1e6) if ms > 0 else None,
                  "tflops": fl / (ms * 1e9) if ms > 0 and fl > 0 else None,
                  "exp_tera_per_s": ex / (ms * 1e9) if ms > 0 and ex > 0 else None}
    return out


# DRAM traffic of the render from the committed ncu capture of the
# quarter-size field (profiles/render_quarter_field_traffic.md: dram__bytes
# read + write per launch, and the stamp bytes the same launches wrote);
# traffic grows with the stamp area rendered, so a full-size launch's
# traffic is this ratio times its algorithmic bytes.
RENDER_TRAFFIC_CAPTURE = {"dram_bytes_per_launch": 3074364.0,
                          "alg_bytes_per_launch": 7062344.0}


def _class_results(job):
    cache = {}

    def get(ci):
        if ci not in cache:
            plan, host, ids = job.classes[ci]
            parts = [job.job.read(i) for i in ids]
            cache[ci] = {k: np.concatenate([q[k] for q in parts], axis=0)
                         for k in ("fluxes", "p", "nst", "acond")}
        return cache[ci]
    return get


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--quality-islands", type=int, default=100,
                    help="target size of the class-stratified float64 sample that "
                         "qualifies the metric")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--precision", default="mixed", choices=["plain", "mixed"],
                    help="Gram form of the headline number (the other form is "
                         "timed too and reported beside it)")
    ap.add_argument("--profile-run", action="store_true",
                    help="one instrumented solve and exit (for ncu)")
    ap.add_argument("--side", type=int, default=2048,
                    help="field side (the workload is 2048; smaller sides "
                         "are for profiler captures)")
    ap.add_argument("--n-src", type=int, default=5000)
    ap.add_argument("--serve-rate", type=float, default=20.0,
                    help="Poisson arrival rate (requests/s) of the serving run")
    ap.add_argument("--serve-requests", type=int, default=40)
    ap.add_argument("--serve-workers", type=int, default=4)
    ap.add_argument("--no-serve", action="store_true")
    ap.add_argument("--serve-only", action="store_true",
                    help="run only the serving measurement (rates from "
                         "--serve-rates) and print its JSON line")
    ap.add_argument("--serve-rates", default="10,50,200,2000")
    ap.add_argument("--reference-render", action="store_true",
                    help="time the solve of the production field in the reference "
                         "render mode (pixelised polynomial PSF; galaxies by the "
                         "Fourier-domain convolution) and print its JSON line")
    ap.add_argument("--precision-stress", action="store_true",
                    help="run only the precision-stress measurement (crowded "
                         "blends, 40 bands) and print its JSON line")
    ap.add_argument("--split-field", action="store_true",
                    help="multi-GPU strong scaling: every rank takes its share of one "
                         "field's islands (default: weak scaling, a field per rank)")
    ap.add_argument("--batched", action="store_true",
                    help="run only the batched configuration (--batched-tiles 2048^2 tiles "
                         "per band count 5, 20 and 40, packed into one job per band count) "
                         "and print its JSON line")
    ap.add_argument("--batched-islands", type=int, default=100000)
    ap.add_argument("--batched-tiles", type=int, default=3,
                    help="distinct 2048^2 tiles per band count in the batched configuration")
    ap.add_argument("--batched-steps", type=int, default=2)
    ap.add_argument("--stress-islands", type=int, default=2000)
    ap.add_argument("--stress-sample", type=int, default=120)
    ap.add_argument("--only-class", default=None,
                    help="with --profile-run: solve only the class 'B,N,kind,T' "
                         "(e.g. 96,32,mixed,127), for kernel captures")
    ap.add_argument("--class-islands", type=int, default=3,
                    help="with --only-class: its first n islands")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference_arm(args, rank, world)
    import torch
    torch.cuda.set_device(local)
    if args.precision_stress:
        if rank == 0:
            print(json.dumps({"precision_stress": _stress_measure(args, local)}),
                  flush=True)
        return
    if args.batched:
        if rank == 0:
            print(json.dumps({"batched": _batched_measure(args, local)}), flush=True)
        return
    if args.reference_render:
        if rank == 0:
            print(json.dumps({"reference_render": _reference_render_measure(args, local)}),
                  flush=True)
        return
    if args.serve_only:
        if rank == 0:
            rates = [float(r) for r in args.serve_rates.split(",")]
            print(json.dumps({"serve": _serve_measure(args, rates, local)}), flush=True)
        return
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    from uniphot_b200.solver import IslandFitJob, island_fit
    from uniphot_b200.synth import make_production_field
    # weak scaling: every rank its own seeded field; --split-field (strong
    # scaling): every rank the same field, its islands partitioned over the
    # ranks by longest processing time (shard.shard_plan), no collective on
    # the data path
    field = make_production_field(args.seed + (0 if args.split_field else 7919 * rank),
                                  device="cuda", side=args.side, n_src=args.n_src)
    kw = field.fit_kwargs("analytic")
    kw["precision"] = args.precision
    plan_kw = {}
    if args.split_field:
        from uniphot_b200.shard import shard_plan
        from uniphot_b200.solver import plan_field
        fp_all = plan_field(**kw)
        plan_kw = {"plan": shard_plan(fp_all, world, rank)}
    job = IslandFitJob(**kw, **plan_kw, device=local)
    n_isl = job.n_islands
    tot_isl = (sum(p.n_islands for p, _ in fp_all.classes) if args.split_field
               else world * n_isl)
    stream = torch.cuda.ExternalStream(job.field.ctx.stream_ptr())
    if args.profile_run:
        if args.only_class:
            run = _class_job(job, field, kw, args)
        else:
            run = job
        kt = _kernel_table(run)
        torch.cuda.synchronize()
        print(json.dumps({"profile_run": True, "n_islands": run.n_islands,
                          "only_class": args.only_class, "precision": args.precision,
                          "kernels": kt}), flush=True)
        job.close()
        return

    def barrier():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()

    # the LM-loop engine of each form is picked by timing its candidates on
    # this job (bitwise the same results), before the warm-up
    tuning = {args.precision: job.autotune()}
    for _ in range(args.warmup):
        job.solve()
    with ClockSampler(local) as clk:
        ms, launches = _timed_solves(job, args.steps, stream, barrier, dist)
    value = tot_isl * args.steps / (ms / 1e3)
    # the other Gram form on the same resident field
    other = "plain" if args.precision == "mixed" else "mixed"
    job_o = IslandFitJob(**dict(kw, precision=other), **plan_kw, device=local,
                         field=job.field)
    tuning[other] = job_o.autotune()
    for _ in range(args.warmup):
        job_o.solve()
    ms_o, _ = _timed_solves(job_o, args.steps, stream, barrier, dist)
    value_o = tot_isl * args.steps / (ms_o / 1e3)
    # the production post-convergence set (parameter covariance and source
    # metrics) on top of the same solve
    job_p = IslandFitJob(**kw, **plan_kw, device=local, field=job.field,
                         compute_param_errors=True, compute_source_metrics=True)
    for _ in range(args.warmup):
        job_p.solve()
    ms_p, _ = _timed_solves(job_p, args.steps, stream, barrier, dist)
    job_p.close()
    ktab = _kernel_table(job)
    ktab_o = _kernel_table(job_o)
    res = job.result()
    # e2e through the public API (host arrays in, results out)
    e2e_t = []
    for _ in range(args.e2e_steps):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        if args.split_field:
            # the rank's share through the job API (planning, upload, solve,
            # read-back, unpack), from the field's host arrays
            part = IslandFitJob(**kw, **plan_kw, device=local)
            part.solve()
            part.result()
            part.close()
        else:
            island_fit(**kw, device=local)
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        e2e_t.append(time.perf_counter() - t0)
    e2e_v = tot_isl / float(np.median(e2e_t))
    nb, H, W = field.data_minus_bg.shape
    PAD = job.PAD
    h2d = 2 * 4 * nb * (H + 2 * PAD) * (W + 2 * PAD)
    for plan, host, _ in job.classes:
        h2d += sum(np.asarray(host[k]).nbytes for k in (
            "ox", "oy", "x0b", "y0b", "st", "sn", "fn_flag", "mmask", "keep", "p0",
            "lower", "upper", "prior_mean", "prior_inv_sigma"))
    d2h = sum(p.n_islands * (6 * p.nsrc_class * 4 + 2 * nb * p.nsrc_class * 4 + 40)
              for p, _, _ in job.classes)
    # compute-pipe peaks of this device (FP32, FP64, exp2f), beside the
    # measured HBM and BF16 figures
    hbm, bf16, bf16_sus, src = _peaks()
    pk = job.field.ctx.measure_peaks()
    peaks = dict(pk, hbm_gbs=hbm, bf16_tflops=bf16_sus)
    model = _roofline_model(ktab, ms / args.steps, peaks)
    # the dominant kernel (largest device time) against its binding roof
    dom = max(ktab, key=lambda k: ktab[k]["ms"])
    d = ktab[dom]
    bound = model["kinds"][dom]["bound"]
    if bound == "sfu":
        roof = {"achieved": d["exp_tera_per_s"], "peak": pk["exp2_tera_per_s"],
                "unit": "10^12 exp2/s"}
    elif bound in ("fp32", "fp64", "tensor"):
        pkv = {"fp32": pk["fp32_tflops"], "fp64": pk["fp64_tflops"],
               "tensor": bf16_sus / 3.0}[bound]
        roof = {"achieved": d["tflops"], "peak": pkv, "unit": "TFLOP/s"}
    else:
        roof = {"achieved": d["gbs"], "peak": hbm, "unit": "GB/s"}
    roof = {"kernel": dom, "bound": bound, **roof, "frac": roof["achieved"] / roof["peak"]}
    per_launch = d["alg_bytes"] / d["launches"]
    roof["traffic"] = (RENDER_TRAFFIC_CAPTURE["dram_bytes_per_launch"] * per_launch /
                       RENDER_TRAFFIC_CAPTURE["alg_bytes_per_launch"]) if dom == "render" else None
    roof["alg_bytes_per_launch"] = per_launch
    roof["hbm_frac"] = d["gbs"] / hbm
    roof["peaks"] = (f"HBM and BF16 {src} (MEASURED_PEAKS.json; BF16 sustained); FP32, "
                     f"FP64 and exp2f measured in this run (uph_measure_peaks)")
    roof["model"] = model
    # results of both forms, kept for the float64 comparison below
    res_forms = {args.precision: _class_results(job), other: _class_results(job_o)}
    for get in res_forms.values():
        for ci in range(len(job.classes)):
            get(ci)
    forms = {
        "mixed": "batched+mixed: LM loop as CUDA graphs on up to 32 streams; tcgen05 "
                 "BF16 hi/lo Gram (residual form) for islands with > 24 Gram rows",
        "plain": "plain: same engine, FP32 Gram on CUDA cores for every island"}
    dtypes = {"mixed": "mixed: bf16x3 tensor-core Gram (fp32 accumulate) for islands with "
                       "> 24 Gram rows, fp32 render and Gram otherwise, f64 solves",
              "plain": "f32 render and Gram, f64 inner solves"}
    out = {
        "metric": METRIC, "value": value, "unit": "islands/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "strong" if args.split_field else "weak", "vs_baseline": None,
        "dtype": dtypes[args.precision],
        "data": "synthetic (seeded production field; per-rank seed)",
        "config": dict(_config(tot_isl if args.split_field else n_isl, world),
                       parallelism=(f"dp{world} (one field's islands split over the ranks "
                                    f"by longest processing time)" if args.split_field
                                    else f"dp{world} (island partition by field)")),
        "form": forms[args.precision],
        "forms": {args.precision: {"value_all_islands": value,
                                   "ms_per_step": ms / args.steps, "kernels": ktab},
                  other: {"value_all_islands": value_o, "ms_per_step": ms_o / args.steps,
                          "kernels": ktab_o, "form": forms[other], "dtype": dtypes[other]}},
        "post_convergence": {
            "options": ["compute_param_errors", "compute_source_metrics"],
            "value": tot_isl * args.steps / (ms_p / 1e3), "unit": "islands/s",
            "ms_per_step": ms_p / args.steps},
        "e2e": {"value": e2e_v, "unit": "islands/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h)},
        "gpu_launches": int(launches),
        "autotune": tuning,
        "clocks": clk.summary(),
        "roofline": roof,
        "device_peaks": pk,
        "quality": {"converged_frac": float(np.mean(res.converged)),
                    "mean_steps": float(np.mean(res.n_steps))},
    }
    classes = job.classes
    job_o.close()
    job.close()
    if rank == 0 and world == 1 and not args.no_serve:
        sv = _serve_measure(args, [args.serve_rate], local)
        r = sv["rates"][0]
        out["serve"] = sv
        out["serve_latency_ms"] = {form: {k: r[form][k] for k in ("p50_ms", "p95_ms", "p99_ms")}
                                   for form in ("packed_mixed", "batched_mixed")}
    # CPU legs after every GPU measurement: the CPU baseline and the float64
    # comparison that qualifies the metric
    if not args.no_cpu and rank == 0:
        out["cpu_baseline"] = _cpu_baseline(classes, PAD, field)
        sample = _stratified_rows(classes, args.quality_islands, 2)
        ref64, secs, procs, wall = cpu_oracle_time(classes, PAD, field, sample,
                                                   precision="f64")
        sampled = {}
        for ci, _ in sample:
            sampled[ci] = sampled.get(ci, 0) + 1
        weights = {ci: classes[ci][0].n_islands / k for ci, k in sampled.items()}
        q = {f: _flux_quality(get, classes, ref64, weights) for f, get in res_forms.items()}
        q["sample"] = (f"{len(ref64)} islands, class-stratified (every class, at least one "
                       f"island each, the rest in proportion), float64 oracle, "
                       f"{wall:.0f} s on {procs} cores; 'weighted' = the field-wide "
                       f"fraction estimated with class weights")
        out["quality"]["flux_vs_fp64"] = q
        # the metric counts the islands solved at the tolerance: islands/s
        # times the estimated fraction of islands whose every flux is within
        # 1e-4 relative or 0.01 sigma of float64
        for f in (args.precision, other):
            frac = q[f]["islands_all_fluxes_pass_weighted"]
            out["forms"][f]["islands_at_tolerance_frac"] = frac
            out["forms"][f]["value"] = out["forms"][f]["value_all_islands"] * frac
        frac = out["forms"][args.precision]["islands_at_tolerance_frac"]
        out["value"] = value * frac
        out["e2e"]["value"] = e2e_v * frac
        out["e2e"]["value_all_islands"] = e2e_v
        out["value_counts"] = ("islands whose every flux is within 1e-4 relative or 0.01 "
                               "sigma of the float64 oracle (islands/s x the class-weighted "
                               "pass fraction of the stratified sample); value_all_islands "
                               "counts every island")
    else:
        out["value_counts"] = "every island (no float64 comparison in this run)"
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
