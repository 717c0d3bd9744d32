"""Drop-in replacement of the reference's island solver entry points.

Mirrors ``tract7dt/fit/grid_gpu/island_solver.py``:

* ``build_psf_tree(psfs, tier)``           (:1851-1871)
* ``make_class_kernels(plan, n_bands, n_terms, ...)``  (:1874-1922)
* ``run_class_chunk(kernels, psf_tree, host, rows, width, max_steps,
  dstack_dev, wstack_dev, pad, init_state=None, ...)``  (:2793-3131)
* ``run_class_chunk_resilient`` (:3165-3230) -- width halving on
  ``RESOURCE_EXHAUSTED``
* ``island_fit(**kw)``                    (:3233-3595)

with the same argument meaning, array layouts, result dict keys, flags and
``ValueError`` on invalid option values.  All arithmetic runs in the CUDA
library behind ``include/uniphot_b200.h``; there is no CPU path.

Differences, by design:

* the LM loop runs on the device for the whole step budget: the reference's
  main pass (``max_steps_main`` steps) plus hard re-queue carrying the exact
  LM state is the same per-island trajectory, so one pass of ``max_steps``
  is run (``bucket_stats`` still reports the counts);
* ``dstack_dev`` is a :class:`DeviceField` (the field stacks resident in
  HBM inside the library context); ``wstack_dev`` is accepted and ignored;
* options whose kernels are not built (crossband GLS) raise ``ValueError``;
  ``scene_subtract`` adds each island's members back at their seeds on the
  device; the post-convergence passes (``compute_param_errors``,
  ``compute_flux_marg``, ``compute_source_metrics``, ``compute_re_profile``,
  ``want_residual`` / ``return_island_residual``) run on the device;
  the step variants (``step_mode="trust_region"``, ``stall_count_mode=
  "changed"``, ``convergence="dlnp"``) run on the device.
"""

from __future__ import annotations

import hashlib

import time
from dataclasses import dataclass
from typing import Callable, Optional

import numpy as np

from . import _lib
from .plan import (DEFAULT_CHI2_FTOL_REL, DEFAULT_MAX_STEPS, REPROF_DELTAS_LN,
                   DEFAULT_MAX_STEPS_MAIN, DEFAULT_POS_STEP_MAX,
                   DEFAULT_STEP_TOL_PIX, DEFAULT_UN_FREEZE_STEPS,
                   IslandFitResult, class_host_arrays, free_n_gate,
                   giant_seed_rows, plan_island_classes, unpack_class_results)
from .psf import MogPsf
from .sersic import load_table

SOURCE_STAR = 0
DEVICE_MAX_NSRC = 32
_CARRY_KEYS = ("p", "lam", "chi2", "consec", "nrej", "nst", "diverged",
               "n_same", "prej")


def _is_mog(psf) -> bool:
    return isinstance(psf, MogPsf) or hasattr(psf, "sigma") and hasattr(psf, "weight")


def _pad_coefs(psf, tier: int) -> np.ndarray:
    """Zero-pad a pixelised PSF to (tier, tier), centre pixel kept at H//2
    (island_solver.py:193-206)."""
    coefs = np.asarray(psf.coefs, np.float32)
    H, W = coefs.shape[:2]
    if tier <= H and tier <= W:
        return coefs
    out = np.zeros((tier, tier) + coefs.shape[2:], np.float32)
    y0, x0 = (tier - H) // 2, (tier - W) // 2
    out[y0:y0 + H, x0:x0 + W] = coefs
    return out


@dataclass
class PsfTree:
    """Per-band PSF stack for one tier, ready for upload."""
    mode: str                  # "reference" | "analytic"
    tier: int
    params: np.ndarray         # (nb, T, T, nt) or (nb, K, 4, nt)
    origin_scale: np.ndarray   # (nb, 4)

    @property
    def n_terms(self) -> int:
        return int(self.params.shape[-1])


def build_psf_tree(psfs: list, tier: int):
    """Stack the per-band PSFs (zero-padded to ``tier``) -> (tree, n_terms)."""
    os_ = np.array([[p.x_origin, p.x_scale, p.y_origin, p.y_scale] for p in psfs],
                   np.float32)
    if _is_mog(psfs[0]):
        K = max(int(np.asarray(p.sigma).shape[0]) for p in psfs)
        nt = int(np.asarray(psfs[0].sigma).shape[1])
        par = np.zeros((len(psfs), K, 4, nt), np.float32)
        for b, p in enumerate(psfs):
            k = np.asarray(p.sigma).shape[0]
            par[b, :k, 0] = p.sigma
            par[b, :k, 1] = p.e1
            par[b, :k, 2] = p.e2
            par[b, :k, 3] = p.weight
            if k < K:       # unused components: unit sigma, zero weight
                par[b, k:, 0, 0] = 1.0
        tree = PsfTree("analytic", int(tier), par, os_)
    else:
        par = np.stack([_pad_coefs(p, int(tier)) for p in psfs]).astype(np.float32)
        tree = PsfTree("reference", int(tier), par, os_)
    return tree, tree.n_terms


def _fingerprint(*arrays) -> str:
    h = hashlib.sha1()
    for a in arrays:
        a = np.ascontiguousarray(a)
        h.update(str((a.dtype.str, a.shape)).encode())
        h.update(a.tobytes())
    return h.hexdigest()


class DeviceField:
    """The padded field stacks resident on one device (a library context).

    Plays the role of the reference's ``dstack_dev``/``wstack_dev``.  A
    context holds one field at a time for new chunks: uploading another field
    to the same context supersedes this one (:meth:`check_current` raises),
    while the chunks already added from it keep reading it."""

    def __init__(self, data_pad: np.ndarray, invvar_pad: np.ndarray, pad: int,
                 device: int = 0, context: Optional[_lib.Context] = None):
        self.ctx = context if context is not None else _lib.Context(device)
        self.ctx.upload_field(data_pad, invvar_pad, pad)
        self.gen = self.ctx.field_gen
        self.pad = int(pad)
        self.n_bands = int(data_pad.shape[0])
        self.shape = tuple(data_pad.shape)
        self._psf_key = {}
        self._mog_key = None
        self._table = False

    @classmethod
    def from_unpadded(cls, data_minus_bg: np.ndarray, invvar: np.ndarray, pad: int,
                      device: int = 0, context: Optional[_lib.Context] = None):
        """Upload the unpadded (n_bands, H, W) field; the zero-padded stacks
        are built on the device."""
        self = cls.__new__(cls)
        self.ctx = context if context is not None else _lib.Context(device)
        self.ctx.upload_field_unpadded(data_minus_bg, invvar, pad)
        self.gen = self.ctx.field_gen
        nb, H, W = np.shape(data_minus_bg)
        self.pad = int(pad)
        self.n_bands = int(nb)
        self.shape = (int(nb), int(H) + 2 * int(pad), int(W) + 2 * int(pad))
        self._psf_key = {}
        self._mog_key = None
        self._table = False
        return self

    @classmethod
    def from_tiles(cls, data: np.ndarray, invvar: np.ndarray, pad: int, tiles, coefs,
                   order: int, norm, device: int = 0,
                   context: Optional[_lib.Context] = None):
        """The island stage's padded stacks built on the device from the raw
        (n_bands, H, W) band data: a border of ``pad`` zeros and each pass-1
        tile's frozen planar background subtracted over its core
        (island_stage.py:1728-1751; ``tiles`` (n, 4) = (x0, y0, x1, y1),
        ``coefs`` (n, n_bands, M), ``norm`` = (x_origin, x_scale, y_origin,
        y_scale), M = 1, 3, 6 for ``order`` 0, 1, 2)."""
        self = cls.from_unpadded(data, invvar, pad, device=device, context=context)
        self.ctx.subtract_tile_backgrounds(tiles, coefs, order, norm)
        return self

    def subtract_star_scene(self, psfs: list, x, y, flux, native: int | None = None):
        """Field-wide scene subtraction of the star models on the device
        (island_stage.py:2024-2118): every source's pass-1 flux (n,
        n_bands) times its stamp (the band's polynomial PSF at its position,
        Lanczos-shifted, on the ``native`` stamp) removed from the data
        stack, in source order per pixel.  Pass the stars to subtract (the
        reference subtracts the fit set's STAR members and keeps extended
        sources)."""
        self.check_current()
        T = int(native if native is not None else psfs[0].H_psf)
        tree, _ = build_psf_tree(psfs, T)
        if tree.mode != "reference":
            raise ValueError("the scene subtraction takes pixelised polynomial PSFs")
        self.ctx.scene_subtract_stars(x, y, flux, tree.params, tree.origin_scale)

    def download(self) -> tuple:
        """The padded (data, invvar) stacks on the host."""
        self.check_current()
        return self.ctx.download_field(self.shape)

    def check_current(self):
        """Raise unless this is still the field its context holds."""
        if self.ctx.field_gen != self.gen:
            raise ValueError("the DeviceField was superseded by a later field upload "
                             "to its context; upload it again")

    def ensure_psf(self, tree: PsfTree):
        # keyed by content: object ids can be reused once a tree is freed
        key = _fingerprint(tree.params, tree.origin_scale)
        if tree.mode == "reference":
            if self._psf_key.get(tree.tier) != key:
                self.ctx.upload_psf_poly(tree.tier, tree.params, tree.origin_scale)
                self._psf_key[tree.tier] = key
        else:
            if self._mog_key != key:
                self.ctx.upload_psf_mog(tree.params, tree.origin_scale)
                self._mog_key = key

    def ensure_exp_mog(self):
        if not getattr(self, "_exp_mog", False):
            from .sparse import exp_mixture
            amp, var = exp_mixture()
            self.ctx.upload_exp_mog(amp, var)
            self._exp_mog = True

    def ensure_table(self):
        if not self._table:
            self.ctx.upload_sersic_table(load_table())
            self._table = True


@dataclass
class ClassKernels:
    """Opaque per-class handle (the reference returns a 16-tuple of jitted
    programs; here it is the class descriptor of the CUDA solver)."""
    desc: _lib.ClassDesc
    render_mode: str
    n_bands: int
    kind: str
    step_protocol: str = "proposals"
    step_mode: str = "clip"


def make_class_kernels(plan, n_bands: int, n_terms: int, *, render_backend: str,
                       reg: float, pos_step_max_pix: float, chi2_ftol_rel: float,
                       step_tol_pix: float, un_freeze_steps: int,
                       star_render_split: bool = True, has_priors: bool = False,
                       stall_count_mode: str = "proposals", step_mode: str = "clip",
                       scene_subtract: bool = False, crossband: dict | None = None,
                       convergence: str = "legacy", plateau_dlnp_tol: float = 0.5,
                       render_mode: str = "reference",
                       native_stamp: int = 0, precision: str = "plain",
                       tc_min_rows: int = -1, tc_cond_max: float = -1.0,
                       bg_mode: str = "frozen") -> ClassKernels:
    if stall_count_mode not in ("proposals", "changed"):
        raise ValueError(f"stall_count_mode must be 'proposals' or 'changed', "
                         f"got {stall_count_mode!r}")
    if step_mode not in ("clip", "trust_region"):
        raise ValueError(f"step_mode must be 'clip' or 'trust_region', got {step_mode!r}")
    if convergence not in ("legacy", "dlnp"):
        raise ValueError(f"convergence must be 'legacy' or 'dlnp', got {convergence!r}")
    if convergence == "dlnp" and step_mode != "clip":
        raise ValueError("convergence='dlnp' requires step_mode='clip' "
                         "(trust-region support pending)")
    if step_mode == "trust_region" and stall_count_mode == "changed":
        # the reference dispatches the trust-region step but runs the
        # "changed" tracker loop, whose arity it does not match
        raise ValueError("step_mode='trust_region' runs with "
                         "stall_count_mode='proposals' only")
    if convergence == "dlnp" and stall_count_mode == "changed":
        raise ValueError("convergence='dlnp' subsumes stall_count_mode='changed' "
                         "(distinct-proposal counting is the dlnp behavior); "
                         "leave stall_count_mode at 'proposals'")
    if render_backend not in ("fft", "direct", "auto"):
        raise ValueError(f"unknown render_backend: {render_backend!r}")
    if render_mode not in ("reference", "analytic"):
        raise ValueError(f"render_mode must be 'reference' or 'analytic', "
                         f"got {render_mode!r}")
    if precision not in _lib.PRECISIONS:
        raise ValueError(f"precision must be 'plain' or 'mixed', got {precision!r}")
    if bg_mode not in ("frozen", "joint"):
        raise ValueError(f"bg_mode must be 'frozen' or 'joint', got {bg_mode!r}")
    unsupported = []
    # star-only classes keep the clip step (island_solver.py:1910-1912)
    step_eff = str(step_mode) if str(plan.kind) != "star" else "clip"
    if crossband is not None:
        unsupported.append("crossband")
    if unsupported:
        raise ValueError("not supported by the B200 island solver: "
                         + ", ".join(unsupported))
    if int(plan.nsrc_class) > DEVICE_MAX_NSRC:
        raise ValueError(f"nsrc class {plan.nsrc_class} exceeds the device limit "
                         f"{DEVICE_MAX_NSRC}; lower joint_nsrc_cap")
    desc = _lib.ClassDesc(
        bbox=int(plan.bbox_class), nsrc=int(plan.nsrc_class), tier=int(plan.tier),
        render_mode=_lib.RENDER_MODES[render_mode], reg=float(reg),
        pos_step_max=float(pos_step_max_pix), chi2_ftol_rel=float(chi2_ftol_rel),
        step_tol_pix=float(step_tol_pix), un_freeze_steps=int(un_freeze_steps),
        has_priors=int(bool(has_priors)), native_stamp=int(native_stamp),
        precision=_lib.PRECISIONS[precision], tc_min_rows=int(tc_min_rows),
        stall_changed=int(stall_count_mode == "changed"),
        convergence_dlnp=int(convergence == "dlnp"),
        plateau_dlnp_tol=float(plateau_dlnp_tol),
        bg_joint=int(bg_mode == "joint"), tc_cond_max=float(tc_cond_max),
        scene_subtract=int(bool(scene_subtract)),
        step_tr=int(step_eff == "trust_region"),
        # the legacy EXP-only direct-convolution backend (source_model.py:
        # 218-256, 298-303); STAR renders the same in both backends
        render_direct=int(render_mode == "reference" and render_backend == "direct"))
    return ClassKernels(desc, render_mode, int(n_bands), str(plan.kind),
                        step_protocol="dlnp" if convergence == "dlnp"
                        else str(stall_count_mode), step_mode=step_eff)


def _slice_host(host: dict, rows: np.ndarray, scene_subtract: bool = False) -> dict:
    keys = ("ox", "oy", "x0b", "y0b", "st", "sn", "fn_flag", "mmask", "keep",
            "p0", "lower", "upper", "prior_mean", "prior_inv_sigma")
    out = {k: np.asarray(host[k])[rows] for k in keys}
    if scene_subtract:
        if host.get("member_s1_flux") is None:
            raise ValueError("scene_subtract needs the class host arrays' member_s1_flux "
                             "(class_host_arrays with s1_flux)")
        out["member_s1_flux"] = np.asarray(host["member_s1_flux"])[rows]
    return out


def run_class_chunk(kernels: ClassKernels, psf_tree: PsfTree, host: dict,
                    rows: np.ndarray, width: int, max_steps: int, dstack_dev,
                    wstack_dev, pad: int, init_state: dict | None = None,
                    compute_param_errors: bool = False, want_residual: bool = False,
                    compute_source_metrics: bool = False,
                    compute_flux_marg: bool = False,
                    compute_re_profile: bool = False) -> dict:
    """Fit one chunk of a class; returns the reference's result dict."""
    t0 = time.perf_counter()
    rows = np.asarray(rows, np.int64)
    n_c = int(rows.size)
    if int(width) < n_c:
        raise ValueError(f"chunk width {width} < rows {n_c}")
    if not isinstance(dstack_dev, DeviceField):
        raise ValueError("dstack_dev must be a uniphot_b200.solver.DeviceField")
    if int(pad) != dstack_dev.pad:
        raise ValueError(f"pad {pad} != the uploaded field's pad {dstack_dev.pad}")
    dstack_dev.ensure_psf(psf_tree)
    if np.any(np.asarray(host["st"])[rows] != SOURCE_STAR):
        dstack_dev.ensure_table()
        if kernels.desc.render_direct:
            dstack_dev.ensure_exp_mog()
    N = int(host["mmask"].shape[1])
    arrays = _slice_host(host, rows, bool(kernels.desc.scene_subtract))
    init = None
    if init_state is not None:
        init = {k: np.asarray(init_state[k]) for k in ("p", "lam", "chi2", "consec",
                                                       "nrej", "nst")}
        for k in ("n_same", "prej", "diverged"):   # "changed"-mode tracker carry
            if init_state.get(k) is not None:
                init[k] = np.asarray(init_state[k])
    desc = kernels.desc
    if (compute_param_errors or compute_flux_marg or compute_source_metrics
            or compute_re_profile or want_residual):
        # the post-convergence passes are per-call options in the reference
        desc = _lib.ClassDesc.from_buffer_copy(desc)
        desc.param_errors = int(bool(compute_param_errors))
        desc.flux_marg = int(bool(compute_flux_marg))
        desc.source_metrics = int(bool(compute_source_metrics))
        desc.re_profile = int(bool(compute_re_profile))
        desc.residual = int(bool(want_residual))
    out = dstack_dev.ctx.run_chunk(desc, arrays, int(max_steps), kernels.n_bands, init)
    if not compute_param_errors:
        out["perr"] = None
    if not compute_flux_marg:
        out["femarg"] = None
    if not compute_source_metrics:
        out["smetrics"] = out["swin"] = None
    if not compute_re_profile:
        out["reprof"] = None
    if not want_residual:
        out["resid"] = out["resid_w"] = None
    out["wall_s"] = time.perf_counter() - t0
    return out


def run_class_chunk_resilient(kernels, psf_tree, host, rows, width, max_steps,
                              dstack_dev, wstack_dev, pad, *, init_state=None,
                              log_fn=None, **kw) -> dict:
    """run_class_chunk, halving the chunk on a device-memory failure."""
    try:
        out = run_class_chunk(kernels, psf_tree, host, rows, width, max_steps,
                              dstack_dev, wstack_dev, pad, init_state=init_state, **kw)
        out["widths_ran"] = [int(width)]
        out["halved"] = False
        return out
    except _lib.UphError as exc:
        n_c = int(np.asarray(rows).size)
        if "RESOURCE_EXHAUSTED" not in str(exc) or n_c <= 1:
            raise
        half = max(1, int(width) // 2)
        msg = (f"island chunk of {n_c} at width {width} hit {exc!s:.80} -- "
               f"retrying as chunk(s) of width {half}")
        (log_fn or (lambda m: print("island: " + m, flush=True)))(msg)
        parts = []
        for lo in range(0, n_c, half):
            sl = slice(lo, min(lo + half, n_c))
            sub = None if init_state is None else {k: v[sl] for k, v in init_state.items()}
            parts.append(run_class_chunk_resilient(
                kernels, psf_tree, host, np.asarray(rows)[sl], half, max_steps,
                dstack_dev, wstack_dev, pad, init_state=sub, log_fn=log_fn, **kw))
        merged = dict(parts[0])
        for k, v0 in parts[0].items():
            if k in ("wall_s", "steps_run", "widths_ran", "halved"):
                continue
            if isinstance(v0, np.ndarray):
                merged[k] = np.concatenate([p[k] for p in parts], axis=0)
        merged["wall_s"] = float(sum(p["wall_s"] for p in parts))
        merged["steps_run"] = int(max(p["steps_run"] for p in parts))
        merged["widths_ran"] = sorted({w for p in parts for w in p["widths_ran"]})
        merged["halved"] = True
        return merged


def _chunk_size(plan, n_bands: int, budget_bytes: float,
                fft_galaxies: bool = False) -> int:
    """Islands per chunk under a device scratch budget (stamps, Gram, GN
    blocks dominate; reference-mode galaxies add their unshifted Fourier
    rows, 7 T x T per member and band)."""
    N, B, T = int(plan.nsrc_class), int(plan.bbox_class), int(plan.tier)
    Sz = min(T, B)
    R = 7 if plan.kind == "mixed" else 3
    nL = N * (6 if plan.kind == "mixed" else 2)
    K = nL + N + 1
    per = 4.0 * n_bands * (N * R * Sz * Sz + K * K + nL * nL + nL) + 8.0 * nL * nL
    if fft_galaxies and plan.kind == "mixed":
        per += 4.0 * n_bands * N * 7 * T * T
    return int(max(1, min(plan.n_islands, budget_bytes // max(per, 1.0))))


def estimate_device_bytes(fp: "FieldPlan", n_bands: int, H: int, W: int,
                          chunk_budget_bytes: float = 16e9,
                          precision: str = "plain") -> int:
    """Device memory a solve of the planned field holds: the padded field
    stacks plus every class's chunk buffers (stamps, Grams, GN blocks, with
    the same per-island estimate that sizes the chunks; the mixed form adds
    up to 16 partial Grams per island-band)."""
    PAD = int(fp.PAD)
    total = 8.0 * n_bands * (H + 2 * PAD) * (W + 2 * PAD)
    for plan, _ in fp.classes:
        n = int(plan.n_islands)
        per_chunk = _chunk_size(plan, n_bands, chunk_budget_bytes)
        N, B, T = int(plan.nsrc_class), int(plan.bbox_class), int(plan.tier)
        Sz = min(T, B)
        R = 7 if plan.kind == "mixed" else 3
        nL = N * (6 if plan.kind == "mixed" else 2)
        K = nL + N + 1
        per = 4.0 * n_bands * (N * R * Sz * Sz + K * K + nL * nL + nL) + 8.0 * nL * nL
        # partial FP32 Grams of large windows (the library's pixel split)
        if K > 32 and B * B >= 4096:
            per += min(8, B * B // 2048) * 4.0 * n_bands * K * K
        if precision == "mixed":
            per += 16 * 4.0 * n_bands * K * K
        total += per * n + 64 * 1024 * -(-n // max(per_chunk, 1))
    return int(total)


def pad_stacks(data_minus_bg, invvar, PAD: int):
    """Zero-padded (n_bands, H + 2 PAD, W + 2 PAD) float32 field stacks
    (island_solver.py:3334-3344)."""
    nb, H, W = data_minus_bg.shape
    dstack = np.zeros((nb, H + 2 * PAD, W + 2 * PAD), np.float32)
    wstack = np.zeros_like(dstack)
    dstack[:, PAD:PAD + H, PAD:PAD + W] = data_minus_bg
    wstack[:, PAD:PAD + H, PAD:PAD + W] = invvar
    return dstack, wstack


@dataclass
class FieldPlan:
    """Host-side plan of a field: classes with their host arrays."""
    classes: list          # [(IslandClassPlan, host dict)]
    capped: list
    PAD: int
    native: int
    render_mode: str


def plan_field(*, psfs, island_set, buckets, pos_x, pos_y, source_type, logre, ee1,
               ee2, sersic_n, s1_flux, s1_flux_var, pos_err=None, re_prior_sig=None,
               ell_prior_sig=None, theta_prior_sig=None, sersic_n_prior_sig=None,
               fit_sersic_n=True, n_fit_min_snr=30.0, pos_max_shift_pix=5.0,
               nsrc_max=None, joint_nsrc_cap=32, free_n_override=None, log_fn=None,
               render_mode=None, tier_ladder=(111, 221), native_stamp=None,
               **_ignored) -> FieldPlan:
    """Class planning and per-class host arrays (no device work)."""
    if render_mode is None:
        render_mode = "analytic" if _is_mog(psfs[0]) else "reference"
    if native_stamp is not None:
        native = int(native_stamp)
    elif render_mode == "reference":
        native = int(psfs[0].H_psf)
    else:
        native = _native_for_mog(psfs)
    if free_n_override is not None:
        free_n_all = np.asarray(free_n_override, bool)
    else:
        free_n_all = free_n_gate(source_type, s1_flux, s1_flux_var, fit_sersic_n,
                                 n_fit_min_snr)
    plans, capped = plan_island_classes(
        island_set, buckets, source_type, logre, sersic_n, native,
        joint_nsrc_cap=joint_nsrc_cap, nsrc_max=nsrc_max, log_fn=log_fn,
        tier_ladder=tier_ladder)
    PAD = int(max((p.bbox_class for p in plans), default=32)) + 8
    kw = dict(pos_x=pos_x, pos_y=pos_y, source_type=source_type, logre=logre,
              ee1=ee1, ee2=ee2, sersic_n=sersic_n, free_n_all=free_n_all,
              pos_max_shift_pix=float(pos_max_shift_pix), pad=PAD, pos_err=pos_err,
              re_prior_sig=re_prior_sig, ell_prior_sig=ell_prior_sig,
              theta_prior_sig=theta_prior_sig, sersic_n_prior_sig=sersic_n_prior_sig)
    classes = [(p, class_host_arrays(p, **kw)) for p in plans]
    return FieldPlan(classes, capped, PAD, native, render_mode)


class IslandFitJob:
    """``island_fit`` split into its three phases: construction plans the
    classes and uploads the field and every chunk's inputs to the device,
    :meth:`solve` runs all chunks (device-resident, concurrent), and
    :meth:`result` reads them back and unpacks the per-source rows.
    ``engine`` picks the LM loop's scheduling: "queue" (every chunk's
    iteration as one persistent work-queue kernel per kernel kind, islands
    retired on the device) or "chunks" (each chunk's iterations as its own
    graph on a stream pool); the results are the same bit for bit.
    ``job``: add the chunks to this (shared) library job instead of a job of
    their own -- the packed server puts several requests' fields into one
    job this way; the job's owner solves and closes it."""

    def __init__(self, *, bandnames: list, data_minus_bg: np.ndarray,
                 invvar: np.ndarray, psfs: list, island_set, buckets, pos_x, pos_y,
                 source_type, logre, ee1, ee2, sersic_n, s1_flux, s1_flux_var,
                 pos_err=None, re_prior_sig=None, ell_prior_sig=None,
                 theta_prior_sig=None, sersic_n_prior_sig=None,
                 render_backend: str = "fft", fit_sersic_n: bool = True,
                 n_fit_min_snr: float = 30.0, pos_max_shift_pix: float = 5.0,
                 pos_step_max_pix: float = DEFAULT_POS_STEP_MAX,
                 max_steps: int = DEFAULT_MAX_STEPS,
                 max_steps_main: int | None = DEFAULT_MAX_STEPS_MAIN,
                 chi2_ftol_rel: float = DEFAULT_CHI2_FTOL_REL,
                 step_tol_pix: float = DEFAULT_STEP_TOL_PIX,
                 un_freeze_steps: int = DEFAULT_UN_FREEZE_STEPS, reg: float = 1e-9,
                 nsrc_max: int | None = None, joint_nsrc_cap: int = 32,
                 star_render_split: bool = True,
                 stall_count_mode: str = "proposals", convergence: str = "legacy",
                 plateau_dlnp_tol: float = 0.5, step_mode: str = "clip",
                 include_giants: bool = True,
                 compute_param_errors: bool = False,
                 compute_flux_marg: bool = False,
                 compute_source_metrics: bool = False,
                 compute_re_profile: bool = False,
                 return_island_residual: bool = False, free_n_override=None,
                 log_fn: Optional[Callable[[str], None]] = None,
                 render_mode: str | None = None, tier_ladder=(111, 221),
                 native_stamp: int | None = None, device: int = 0,
                 field: DeviceField | None = None,
                 chunk_budget_bytes: float = 16e9, precision: str = "plain",
                 plan: "FieldPlan | None" = None, bg_mode: str = "frozen",
                 engine: str = "chunks", lanes: int = 0,
                 job: "_lib.Job | None" = None):
        self.log_fn = log_fn
        if render_mode is None:
            render_mode = "analytic" if _is_mog(psfs[0]) else "reference"
        self.render_mode = render_mode
        n_bands = len(bandnames)
        self.bandnames, self.n_bands = list(bandnames), n_bands
        fp = plan if plan is not None else plan_field(
            psfs=psfs, island_set=island_set, buckets=buckets, pos_x=pos_x,
            pos_y=pos_y, source_type=source_type, logre=logre, ee1=ee1, ee2=ee2,
            sersic_n=sersic_n, s1_flux=s1_flux, s1_flux_var=s1_flux_var,
            pos_err=pos_err, re_prior_sig=re_prior_sig, ell_prior_sig=ell_prior_sig,
            theta_prior_sig=theta_prior_sig, sersic_n_prior_sig=sersic_n_prior_sig,
            fit_sersic_n=fit_sersic_n, n_fit_min_snr=n_fit_min_snr,
            pos_max_shift_pix=pos_max_shift_pix, nsrc_max=nsrc_max,
            joint_nsrc_cap=joint_nsrc_cap, free_n_override=free_n_override,
            log_fn=log_fn, render_mode=render_mode, tier_ladder=tier_ladder,
            native_stamp=native_stamp)
        PAD = fp.PAD
        H, W = data_minus_bg.shape[1], data_minus_bg.shape[2]
        if field is None or field.pad != PAD or field.shape != (
                n_bands, H + 2 * PAD, W + 2 * PAD):
            field = DeviceField.from_unpadded(
                data_minus_bg, invvar, PAD, device=device,
                context=field.ctx if field is not None else None)
        field.check_current()
        self.field, self.PAD = field, PAD
        plans = [p for p, _ in fp.classes]
        capped = fp.capped
        if job is not None:
            # chunks added to a job shared with other fields (packed
            # serving): its owner solves and closes it
            if job.ctx is not field.ctx:
                raise ValueError("a shared job must belong to the field's context")
            self.job, self._own_job = job, False
        else:
            self.job, self._own_job = _lib.Job(field.ctx), True
            self.job.set_engine(engine, lanes)
        self.tuning = None
        self.classes = []
        trees = {}
        for plan, host in fp.classes:
            T = int(plan.tier)
            if T not in trees:
                trees[T] = build_psf_tree(psfs, T)
            tree, n_terms = trees[T]
            field.ensure_psf(tree)
            if np.any(np.asarray(host["st"]) != SOURCE_STAR):
                field.ensure_table()
                if render_backend == "direct" and render_mode == "reference":
                    field.ensure_exp_mog()
            kern = make_class_kernels(
                plan, n_bands, n_terms, render_backend=render_backend, reg=reg,
                pos_step_max_pix=pos_step_max_pix, chi2_ftol_rel=chi2_ftol_rel,
                step_tol_pix=step_tol_pix, un_freeze_steps=un_freeze_steps,
                star_render_split=star_render_split,
                has_priors=bool(host["has_priors"]),
                stall_count_mode=stall_count_mode, convergence=convergence,
                plateau_dlnp_tol=plateau_dlnp_tol, step_mode=step_mode,
                render_mode=render_mode,
                native_stamp=fp.native, precision=precision, bg_mode=bg_mode)
            kern.desc.param_errors = int(bool(compute_param_errors))
            kern.desc.flux_marg = int(bool(compute_flux_marg))
            kern.desc.source_metrics = int(bool(compute_source_metrics))
            kern.desc.re_profile = int(bool(compute_re_profile))
            kern.desc.residual = int(bool(return_island_residual))
            chunk = _chunk_size(plan, n_bands, chunk_budget_bytes,
                                fft_galaxies=render_mode == "reference")
            ids = []
            for lo in range(0, plan.n_islands, chunk):
                rows = np.arange(lo, min(lo + chunk, plan.n_islands))
                ids.append(self.job.add_chunk(kern.desc, _slice_host(host, rows),
                                              n_bands))
            self.classes.append((plan, host, ids))
        self.max_steps = int(max_steps)
        self.max_steps_main = max_steps_main
        self.island_set, self.buckets, self.capped = island_set, buckets, capped
        self.include_giants = include_giants
        self.compute_param_errors = bool(compute_param_errors)
        self.compute_flux_marg = bool(compute_flux_marg)
        self.compute_source_metrics = bool(compute_source_metrics)
        self.compute_re_profile = bool(compute_re_profile)
        self.return_island_residual = bool(return_island_residual)
        self.island_residuals = {}
        self.src = dict(pos_x=pos_x, pos_y=pos_y, logre=logre, ee1=ee1, ee2=ee2,
                        sersic_n=sersic_n)
        self.n_islands = sum(p.n_islands for p, _, _ in self.classes)

    def solve(self):
        t0 = time.perf_counter()
        self.job.solve(self.max_steps)
        self.solve_wall_s = time.perf_counter() - t0

    # LM-loop engine configurations the autotuner times: (engine, lanes)
    AUTOTUNE_CANDIDATES = (("chunks", 0), ("queue", 8), ("queue", 16), ("queue", 32),
                           ("queue_per_cta", 16))

    def autotune(self, candidates=AUTOTUNE_CANDIDATES, repeats: int = 2) -> dict:
        """Time this job's solve under each LM-loop engine configuration and
        keep the fastest.  Every configuration computes bitwise the same
        results (the queue kernels run the per-chunk kernels' work for each
        unit), so the choice changes only the speed.  Each candidate runs one
        untimed solve (graph capture, allocations) and ``repeats`` timed ones
        (device time of the whole solve from the library's events, best of
        the repeats).  The choice and the times are kept in ``self.tuning``
        and returned."""
        times = {}
        for engine, lanes in candidates:
            self.job.set_engine(engine, lanes)
            self.solve()
            best = float("inf")
            for _ in range(max(1, repeats)):
                self.solve()
                best = min(best, self.field.ctx.last_timing()[1])
            times[f"{engine}/{lanes}"] = best
        pick = min(times, key=times.get)
        engine, lanes = pick.split("/")
        self.job.set_engine(engine, int(lanes))
        self.tuning = {"ms_per_solve": times, "picked": pick,
                       "what": "LM-loop engine and lanes, by device time of a full solve"}
        return self.tuning

    def result(self) -> IslandFitResult:
        out_rows, bucket_stats = [], []
        n_bands = self.n_bands
        for plan, host, ids in self.classes:
            parts = [self.job.read(i) for i in ids]
            res = {k: np.concatenate([p[k] for p in parts], axis=0)
                   for k in parts[0] if isinstance(parts[0][k], np.ndarray)}
            nst = res["nst"]
            bucket_stats.append(dict(
                bbox_class=int(plan.bbox_class), nsrc_class=int(plan.nsrc_class),
                tier=int(plan.tier), kind=plan.kind, n_islands=int(plan.n_islands),
                n_chunks=len(ids), mean_steps=float(nst.mean()),
                max_steps_used=int(nst.max()),
                n_unconverged=int((~res["conv"]).sum()),
                n_stalled=int(res["stall"].sum()),
                n_requeued=int((nst > (self.max_steps_main or self.max_steps)).sum())))
            if self.log_fn is not None:
                self.log_fn(f"bucket bbox={plan.bbox_class} nsrc={plan.nsrc_class} "
                            f"kind={plan.kind} tier={plan.tier}: {plan.n_islands} "
                            f"islands, mean_steps={nst.mean():.1f}")
            out_rows.append(unpack_class_results(
                plan, host, self.island_set, res["p"], res["fluxes"], res["ferr"],
                res["chi2"], res["conv"], res["stall"], res["nst"],
                res_pdchi2=res["stall_dchi2"], res_div=res["diverged"],
                res_ngood=res["n_good"], n_bands=n_bands,
                res_bg=res.get("bg"), res_bg_err=res.get("bg_err"),
                res_railed=res.get("railed"),
                res_perr=res["perr"] if self.compute_param_errors else None,
                res_femarg=res["femarg"] if self.compute_flux_marg else None,
                res_smetrics=res["smetrics"] if self.compute_source_metrics else None,
                res_swin=res["swin"] if self.compute_source_metrics else None,
                res_reprof=res["reprof"] if self.compute_re_profile else None,
                reprof_deltas=REPROF_DELTAS_LN if self.compute_re_profile else None))
            if self.return_island_residual:
                # per-island coadded residual at the converged parameters,
                # keyed by global island id with the window origin
                for r in range(plan.n_islands):
                    self.island_residuals[int(plan.isl_ids[r])] = dict(
                        resid=res["resid"][r], resid_w=res["resid_w"][r],
                        x0b=float(host["x0b"][r]), y0b=float(host["y0b"][r]),
                        B=int(plan.bbox_class))
        giant_ids = np.concatenate([np.asarray(self.buckets.giant_ids, np.int64).ravel(),
                                    np.asarray(self.capped, np.int64)])
        if self.include_giants and giant_ids.size:
            out_rows.extend(giant_seed_rows(giant_ids, self.island_set,
                                            n_bands=n_bands, **self.src))
        return _assemble_result(self.bandnames, out_rows, bucket_stats)

    def close(self):
        if self._own_job:
            self.job.close()


def _assemble_result(bandnames, out_rows, bucket_stats) -> IslandFitResult:
    """IslandFitResult from per-class (and giant) row dicts."""
    cat = {k: np.concatenate([r[k] for r in out_rows], axis=0) for k in out_rows[0]}
    return IslandFitResult(
        bandnames=list(bandnames), source_idx=cat["src"].astype(np.int64),
        pos_x=cat["pos_x"], pos_y=cat["pos_y"], logre=cat["logre"],
        ee1=cat["ee1"], ee2=cat["ee2"], sersic_n=cat["sersic_n"],
        fluxes=cat["fluxes"], flux_err=cat["flux_err"], chi2=cat["chi2"],
        chi2_nu=cat["chi2_nu"], n_steps=cat["n_steps"],
        converged=cat["converged"], stalled=cat["stalled"],
        diverged=cat["diverged"], stall_dchi2=cat["stall_dchi2"],
        free_n=cat["free_n"], railed=cat["railed"], island_id=cat["island_id"],
        island_nsrc=cat["island_nsrc"], island_giant=cat["island_giant"],
        re_upper_pix=cat["re_upper_pix"], pos_x_err=cat["pos_x_err"],
        pos_y_err=cat["pos_y_err"], re_err=cat["re_err"], ell_err=cat["ell_err"],
        re_prof_lo=cat["re_prof_lo"], re_prof_hi=cat["re_prof_hi"],
        theta_err=cat["theta_err"], sersic_n_err=cat["sersic_n_err"],
        pos_x_prior_frac=cat["pos_x_prior_frac"],
        pos_y_prior_frac=cat["pos_y_prior_frac"],
        re_prior_frac=cat["re_prior_frac"], ell_prior_frac=cat["ell_prior_frac"],
        theta_prior_frac=cat["theta_prior_frac"],
        sersic_n_prior_frac=cat["sersic_n_prior_frac"], rchisq=cat["rchisq"],
        fracflux=cat["fracflux"], fracin=cat["fracin"],
        fracmasked=cat["fracmasked"], flux_win=cat["flux_win"],
        flux_marg_var=cat["flux_marg_var"], bg_plane=cat["bg_plane"],
        bg_plane_err=cat["bg_plane_err"], bucket_stats=bucket_stats)


def giant_only_result(*, bandnames, island_set, buckets, pos_x, pos_y, logre, ee1,
                      ee2, sersic_n, joint_nsrc_cap=32, **_ignored) -> IslandFitResult:
    """Result of a field whose islands all take the giant path (no bucket
    left to fit): every member keeps its seed, flagged as a giant -- the rows
    ``island_fit`` appends for giants."""
    ids = [np.asarray(buckets.giant_ids, np.int64).ravel()]
    for (bc, nc), b in buckets.buckets.items():
        if joint_nsrc_cap is None or nc > int(joint_nsrc_cap):
            ids.append(np.asarray(b.island_ids, np.int64))
    giant_ids = np.concatenate(ids)
    rows = giant_seed_rows(giant_ids, island_set, n_bands=len(bandnames), pos_x=pos_x,
                           pos_y=pos_y, logre=logre, ee1=ee1, ee2=ee2, sersic_n=sersic_n)
    return _assemble_result(bandnames, rows, [])


def island_fit(**kwargs) -> IslandFitResult:
    """Fit all bucketed islands (+ giants) on the GPU; same keywords and
    result as the reference's ``island_fit`` (plus ``render_mode``,
    ``tier_ladder``, ``native_stamp``, ``device``, ``field``)."""
    job = IslandFitJob(**kwargs)
    try:
        job.solve()
        res = job.result()
        if job.return_island_residual:
            return res, job.island_residuals
        return res
    finally:
        job.close()


def _native_for_mog(psfs) -> int:
    """Native stamp for an analytic PSF: the odd side covering +-4 sigma of
    the widest component anywhere near the field centre (>= 31)."""
    s = max(float(np.max(np.abs(np.asarray(p.sigma)[:, 0]))) for p in psfs)
    side = int(2 * np.ceil(4.0 * s) + 1)
    return max(31, side | 1)


def island_fit_singletons(**kwargs):
    """Fit only the nsrc_class == 1 buckets."""
    return island_fit(nsrc_max=1, include_giants=False, **kwargs)
