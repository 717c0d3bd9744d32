"""Class planning, per-class host arrays and result unpacking (host numpy).

Same contract as the reference's ``fit/grid_gpu/island_plan.py``:

* ``plan_island_classes`` (:356) -- bucket -> (B, N, kind, tier T) classes;
  islands with any extended member are "mixed" and take the smallest tier of
  ``(native, 111, 221)`` covering ``2 * nre(n) * Re`` of their largest
  extended member; buckets with ``nsrc > joint_nsrc_cap`` go to the giant
  path.
* ``class_host_arrays`` (:493) -- window origins, seeds, keep masks, box
  bounds, priors.
* ``unpack_class_results`` (:702) / ``giant_seed_rows`` (:1019) -- island
  rows -> per-source rows.
* ``free_n_gate`` (:199), ``ladder_width`` (:96), ``IslandFitResult`` (:221).
"""

from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

SOURCE_STAR = 0
SOURCE_SERSIC = 3
SERSIC_N_MIN = 0.29
SERSIC_N_MAX = 6.3
# log-radius offsets of the Re profile scan (island_plan.py:58-60)
REPROF_DELTAS_LN = np.array([-2.5, -1.5, -0.9, -0.5, -0.25, -0.1,
                             0.1, 0.25, 0.5, 0.9, 1.5, 2.5], np.float32)

DEFAULT_MAX_STEPS = 30
DEFAULT_MAX_STEPS_MAIN = 8
DEFAULT_CHI2_FTOL_REL = 1e-4
DEFAULT_STEP_TOL_PIX = 0.1
DEFAULT_POS_STEP_MAX = 0.5
DEFAULT_UN_FREEZE_STEPS = 0
HARD_CHUNK_DIV = 4


def ladder_width(n_rows: int, cap: int) -> int:
    """Smallest power of two >= n_rows, capped at ``cap``."""
    n = max(1, int(n_rows))
    return int(min(1 << (n - 1).bit_length(), max(1, int(cap))))


def sersic_n_to_u_np(n):
    t = (np.clip(n, SERSIC_N_MIN + 1e-4, SERSIC_N_MAX - 1e-4) - SERSIC_N_MIN) \
        / (SERSIC_N_MAX - SERSIC_N_MIN)
    return np.log(t / (1.0 - t))


def free_n_gate(source_type, s1_flux, s1_flux_var, fit_sersic_n, n_fit_min_snr):
    """Free Sersic n for SERSIC rows whose median-band S1 S/N passes."""
    st = np.asarray(source_type)
    out = np.zeros(st.shape[0], dtype=bool)
    if fit_sersic_n and bool(np.any(st == SOURCE_SERSIC)):
        with np.errstate(divide="ignore", invalid="ignore"):
            snr_b = np.abs(s1_flux) / np.sqrt(np.maximum(s1_flux_var, 1e-30))
        snr = np.nanmedian(snr_b, axis=1)
        out = (st == SOURCE_SERSIC) & np.isfinite(snr) & (snr >= float(n_fit_min_snr))
    return out


def _propagate_shape_sigmas(ee1, ee2, re, ell_err, theta_err, re_err):
    """Catalog-frame (Re, ELL, THETA) prior sigmas -> internal
    (logre, ee1, ee2) sigmas through the soft-ellipse Jacobian
    (island_plan.py:103-192).  NaN where absent/invalid."""
    ee1 = np.asarray(ee1, np.float64)
    ee2 = np.asarray(ee2, np.float64)
    re = np.asarray(re, np.float64)
    ell_err = np.asarray(ell_err, np.float64)
    theta_err = np.asarray(theta_err, np.float64)
    re_err = np.asarray(re_err, np.float64)
    re_ok = np.isfinite(re_err) & (re_err > 0) & (re > 0)
    sig_lr = np.where(re_ok, re_err / np.where(re > 0, re, 1.0), np.nan)
    mag = np.hypot(ee1, ee2)
    e_s = 1.0 - np.exp(-mag)
    ab = (1.0 - e_s) / np.maximum(1.0 + e_s, 1e-12)
    phi = -np.degrees(np.arctan2(ee2, ee1) / 2.0)
    ell = np.clip(1.0 - ab, 0.0, 0.999)
    ang = np.radians(-2.0 * phi)
    ba = 1.0 - ell
    e = (1.0 - ba) / (1.0 + ba)
    ee = -np.log(np.maximum(1.0 - e, 1e-15))
    ca, sa = np.cos(ang), np.sin(ang)
    dee = 1.0 / np.maximum((2.0 - ell) * (1.0 - ell), 1e-15)
    k = 2.0 * np.pi / 180.0
    ok = (np.isfinite(ell_err) & (ell_err > 0) & np.isfinite(theta_err)
          & (theta_err > 0))
    le = np.where(ok, ell_err, 0.0)
    te = np.where(ok, theta_err, 0.0)
    v1 = (dee * ca * le) ** 2 + (k * ee * sa * te) ** 2
    v2 = (dee * sa * le) ** 2 + (k * ee * ca * te) ** 2
    s1 = np.where(ok & (v1 > 0), np.sqrt(np.where(v1 > 0, v1, 1.0)), np.nan)
    s2 = np.where(ok & (v2 > 0), np.sqrt(np.where(v2 > 0, v2, 1.0)), np.nan)
    return sig_lr, s1, s2


@dataclass
class IslandClassPlan:
    class_idx: int
    bbox_class: int
    nsrc_class: int
    kind: str
    tier: int
    isl_ids: np.ndarray = field(repr=False)
    midx: np.ndarray = field(repr=False)
    mmask: np.ndarray = field(repr=False)
    bbox: np.ndarray = field(repr=False)
    n_src_of: np.ndarray = field(repr=False)
    n_gal_class: int = 0
    tangent_chunk: int = 6
    chunk_main: int = 1
    chunk_hard: int = 1

    @property
    def n_islands(self) -> int:
        return int(self.isl_ids.shape[0])

    @property
    def key(self):
        return (self.bbox_class, self.nsrc_class, self.kind, self.tier)


def plan_island_classes(island_set, buckets, source_type, logre, sersic_n,
                        native, *, joint_nsrc_cap=32, nsrc_max=None,
                        log_fn=None, crossband_rank=0, tier_ladder=(111, 221)):
    """Occupied buckets -> solver classes and the capped giant ids.

    ``tier_ladder`` are the stamp tiers above the native one (the reference
    hard-codes 111 and 221)."""
    todo = {k: b for k, b in buckets.buckets.items()
            if nsrc_max is None or k[1] <= int(nsrc_max)}
    capped = []
    if joint_nsrc_cap is not None:
        for k in [k for k in list(todo) if k[1] > int(joint_nsrc_cap)]:
            capped.extend(todo.pop(k).island_ids.tolist())
        if capped and log_fn is not None:
            log_fn(f"joint_nsrc_cap={joint_nsrc_cap}: {len(capped)} island(s) "
                   f"-> giant path")
    if not todo:
        raise ValueError("no buckets selected")
    st = np.asarray(source_type)
    lr = np.asarray(logre)
    sn = np.asarray(sersic_n)
    plans = []
    for (bc, nc) in sorted(todo):
        b = todo[(bc, nc)]
        ids = b.island_ids
        midx = np.maximum(b.member_idx.astype(np.int64), 0)
        mm = b.member_mask.astype(bool)
        is_gal = (st[midx] != SOURCE_STAR) & mm
        has_ext = is_gal.any(axis=1)
        ngal = is_gal.sum(axis=1)
        nre = np.where(sn[midx] < 1.5, 4.0, np.where(sn[midx] < 3.0, 6.0, 8.0))
        half = np.where(is_gal, nre * np.exp(lr[midx].astype(float)), 0.0).max(axis=1)
        ladder = [t for t in (native, *tier_ladder) if t >= native]
        tier = np.full(ids.size, ladder[-1], np.int64)
        for t in reversed(ladder):
            tier = np.where(2 * half <= t, t, tier)
        groups = [("star", native, np.nonzero(~has_ext)[0])]
        for t in ladder:
            groups.append(("mixed", int(t), np.nonzero(has_ext & (tier == t))[0]))
        for kind, T, sel in groups:
            if sel.size == 0:
                continue
            plans.append(IslandClassPlan(
                class_idx=len(plans), bbox_class=int(bc), nsrc_class=int(nc),
                kind=kind, tier=int(T), isl_ids=ids[sel].astype(np.int64),
                midx=midx[sel], mmask=mm[sel], bbox=island_set.bbox[ids[sel]],
                n_src_of=island_set.n_src[ids[sel]].astype(np.int32),
                n_gal_class=int(ngal[sel].max()) if kind == "mixed" else 0))
    return plans, capped


def class_host_arrays(plan, *, pos_x, pos_y, source_type, logre, ee1, ee2,
                      sersic_n, free_n_all, pos_max_shift_pix, pad,
                      pos_err=None, re_prior_sig=None, ell_prior_sig=None,
                      theta_prior_sig=None, sersic_n_prior_sig=None,
                      s1_flux=None, cb_scale=None) -> dict:
    """Per-class seeds, bounds, keep masks, window origins and priors."""
    B, N, T = int(plan.bbox_class), int(plan.nsrc_class), int(plan.tier)
    midx, mmask = plan.midx, plan.mmask
    n_isl = plan.n_islands
    bbox = plan.bbox
    ox = bbox[:, 0] - (B - (bbox[:, 2] - bbox[:, 0])) // 2 + pad
    oy = bbox[:, 1] - (B - (bbox[:, 3] - bbox[:, 1])) // 2 + pad
    x0b = (ox - pad).astype(np.float32)
    y0b = (oy - pad).astype(np.float32)
    sx = np.asarray(pos_x)[midx].astype(np.float32)
    sy = np.asarray(pos_y)[midx].astype(np.float32)
    st = np.asarray(source_type)[midx].astype(np.int32)
    lr = np.asarray(logre)[midx].astype(np.float32)
    e1 = np.asarray(ee1)[midx].astype(np.float32)
    e2 = np.asarray(ee2)[midx].astype(np.float32)
    sn = np.asarray(sersic_n)[midx].astype(np.float32)
    u0 = sersic_n_to_u_np(sn).astype(np.float32)
    is_ext = st != SOURCE_STAR
    G = int(plan.n_gal_class)
    is_gal = is_ext & mmask
    if G > 0:
        order = np.argsort(~is_gal, axis=1, kind="stable")
        gsel = order[:, :G].astype(np.int32)
        gvalid = np.take_along_axis(is_gal, order, axis=1)[:, :G]
    else:
        gsel = np.zeros((n_isl, 0), np.int32)
        gvalid = np.zeros((n_isl, 0), bool)

    def gat(a):
        if a is None:
            return np.full((n_isl, N), np.nan)
        return np.asarray(a, np.float64)[midx]
    pe, rps, eps, tps, nps = (gat(pos_err), gat(re_prior_sig), gat(ell_prior_sig),
                              gat(theta_prior_sig), gat(sersic_n_prior_sig))
    has_n_prior = (st == SOURCE_SERSIC) & np.isfinite(nps) & (nps > 0) & mmask
    fn_flag = (np.asarray(free_n_all)[midx] | has_n_prior) & mmask
    keep = np.zeros((n_isl, N, 6), bool)
    keep[:, :, 0:2] = mmask[:, :, None]
    keep[:, :, 2:5] = (is_ext & mmask)[:, :, None]
    keep[:, :, 5] = fn_flag
    p0 = np.stack([sx, sy, lr, e1, e2, u0], axis=2).astype(np.float32)
    one = np.ones((n_isl, N), np.float32)
    lower = np.stack([sx - pos_max_shift_pix, sy - pos_max_shift_pix,
                      np.full((n_isl, N), np.log(0.1), np.float32),
                      -100 * one, -100 * one, -12 * one], axis=2).astype(np.float32)
    upper = np.stack([sx + pos_max_shift_pix, sy + pos_max_shift_pix,
                      np.full((n_isl, N), np.log(0.75 * T), np.float32),
                      100 * one, 100 * one, 12 * one], axis=2).astype(np.float32)
    inv = np.zeros((n_isl, N, 6))
    pos_ok = np.isfinite(pe) & (pe > 0) & mmask
    pinv = np.where(pos_ok, 1.0 / np.where(pos_ok, pe, 1.0), 0.0)
    inv[:, :, 0] = pinv
    inv[:, :, 1] = pinv
    ext_ok = is_ext & mmask
    s_lr, s_e1, s_e2 = _propagate_shape_sigmas(e1, e2, np.exp(lr.astype(np.float64)),
                                               eps, tps, rps)
    ok = ext_ok & np.isfinite(s_lr) & (s_lr > 0)
    inv[:, :, 2] = np.where(ok, 1.0 / np.where(ok, s_lr, 1.0), 0.0)
    ok = ext_ok & np.isfinite(s_e1) & (s_e1 > 0) & np.isfinite(s_e2) & (s_e2 > 0)
    inv[:, :, 3] = np.where(ok, 1.0 / np.where(ok, s_e1, 1.0), 0.0)
    inv[:, :, 4] = np.where(ok, 1.0 / np.where(ok, s_e2, 1.0), 0.0)
    sn64 = sn.astype(np.float64)
    dndu = (sn64 - SERSIC_N_MIN) * (SERSIC_N_MAX - sn64) / (SERSIC_N_MAX - SERSIC_N_MIN)
    inv[:, :, 5] = np.where(has_n_prior, dndu / np.where(has_n_prior, nps, 1.0), 0.0)
    pinv32 = inv.astype(np.float32)
    msf = None
    if s1_flux is not None:
        msf = (np.asarray(s1_flux, np.float32)[midx]
               * (mmask & ~is_ext)[:, :, None]).astype(np.float32)
    out = dict(ox=ox, oy=oy, x0b=x0b, y0b=y0b, st=st, lr=lr, e1=e1, e2=e2,
               sn=sn, fn_flag=fn_flag, is_ext=is_ext, mmask=mmask, keep=keep,
               gsel=gsel, gvalid=gvalid, p0=p0, lower=lower, upper=upper,
               prior_mean=p0.copy(), prior_inv_sigma=pinv32,
               has_priors=bool(np.any(pinv32 != 0)), member_s1_flux=msf)
    if cb_scale is not None:
        cs = np.asarray(cb_scale, np.float64)[midx]
        out["cb_scale"] = (np.where(mmask, cs, 0.0).sum(axis=1)
                           / np.maximum(mmask.sum(axis=1), 1)).astype(np.float32)
    return out


@dataclass
class IslandFitResult:
    """Per-source rows for every fitted or giant island member."""
    bandnames: list
    source_idx: np.ndarray
    pos_x: np.ndarray
    pos_y: np.ndarray
    logre: np.ndarray
    ee1: np.ndarray
    ee2: np.ndarray
    sersic_n: np.ndarray
    fluxes: np.ndarray
    flux_err: np.ndarray
    chi2: np.ndarray
    n_steps: np.ndarray
    converged: np.ndarray
    free_n: np.ndarray
    stalled: np.ndarray = None
    diverged: np.ndarray = None
    stall_dchi2: np.ndarray = None
    railed: np.ndarray = None
    chi2_nu: np.ndarray = None
    island_id: np.ndarray = None
    island_nsrc: np.ndarray = None
    island_giant: np.ndarray = None
    re_upper_pix: np.ndarray = None
    pos_x_err: np.ndarray = None
    pos_y_err: np.ndarray = None
    re_err: np.ndarray = None
    re_prof_lo: np.ndarray = None
    re_prof_hi: np.ndarray = None
    ell_err: np.ndarray = None
    theta_err: np.ndarray = None
    sersic_n_err: np.ndarray = None
    pos_x_prior_frac: np.ndarray = None
    pos_y_prior_frac: np.ndarray = None
    re_prior_frac: np.ndarray = None
    ell_prior_frac: np.ndarray = None
    theta_prior_frac: np.ndarray = None
    sersic_n_prior_frac: np.ndarray = None
    rchisq: np.ndarray = None
    fracflux: np.ndarray = None
    fracin: np.ndarray = None
    fracmasked: np.ndarray = None
    flux_win: np.ndarray = None
    flux_marg_var: np.ndarray = None
    # planar background of the member's island per band (c0 + c1 X + c2 Y
    # over the island window, X, Y = (pixel - (B - 1) / 2) / (B / 2)) and
    # its error, when the fit solved it jointly (bg_mode="joint"); else 0
    bg_plane: np.ndarray = None
    bg_plane_err: np.ndarray = None
    bucket_stats: list = field(default_factory=list)

    @property
    def requeue_idx(self):
        return self.source_idx[~self.converged]


def _nan(n):
    return np.full(n, np.nan, np.float32)


def re_profile_interval(res_p, res_reprof, deltas, ii, kk, is_ext):
    """Re interval where the chi2 profile along log Re stays below 1
    (island_plan.py:913-952): walking outward from the fit on each side,
    the first offset whose profile reaches 1 is linearly interpolated with
    the previous point (the fit itself at 0); a side that never reaches 1
    ends at its outermost offset.  NaN for point sources."""
    d = np.asarray(deltas, np.float64)
    order = np.argsort(d)
    d = d[order]
    prof = res_reprof[ii, kk, :].astype(np.float64)[:, order]
    prof = np.where(np.isfinite(prof), prof, np.inf)

    def crossing(pr, dd):
        P = np.concatenate([np.zeros((pr.shape[0], 1)), pr], axis=1)
        D = np.concatenate([[0.0], dd])
        hit = P >= 1.0
        any_hit = hit.any(axis=1)
        j = np.maximum(np.argmax(hit, axis=1), 1)
        p0 = P[np.arange(P.shape[0]), j - 1]
        p1 = P[np.arange(P.shape[0]), j]
        t = np.where(p1 > p0, (1.0 - p0) / np.maximum(p1 - p0, 1e-30), 1.0)
        return np.where(any_hit, D[j - 1] + np.clip(t, 0.0, 1.0) * (D[j] - D[j - 1]), dd[-1])
    neg, pos = d < 0, d > 0
    lo = crossing(prof[:, neg][:, ::-1], d[neg][::-1])
    hi = crossing(prof[:, pos], d[pos])
    re = np.exp(res_p[ii, kk, 2].astype(np.float64))
    ext = is_ext[ii, kk]
    return (np.where(ext, re * np.exp(lo), np.nan).astype(np.float32),
            np.where(ext, re * np.exp(hi), np.nan).astype(np.float32))


def catalog_errors(res_p, res_perr, host, ii, kk, n_final) -> dict:
    """Catalog-frame 1-sigma errors and prior fractions of the members
    (ii, kk) from the per-member covariance rows of ``res_perr`` (n_isl, N,
    13): var(x, y, logre, ee1, ee2, u), cov(ee1, ee2), six prior fractions
    (island_plan.py:796-885).

    Non-kept slots and degenerate variances (non-finite or <= 0) give NaN.
    Re = exp(logre) scales its error by Re; ELL = 2e/(1+e) with e = 1 -
    exp(-|ee|) and THETA = -atan2(ee2, ee1)/2 in degrees take the exact
    2x2 quadratic forms of their gradients in (ee1, ee2) with the ee1-ee2
    covariance (undefined at |ee| = 0: NaN); Sersic n = n(u) scales by
    dn/du = (n - n_min)(n_max - n)/(n_max - n_min) on free-n members.  The
    ELL / THETA prior fractions weight the ee1 / ee2 fractions radially
    (ee1^2, ee2^2) and tangentially (ee2^2, ee1^2) over |ee|^2; a fraction
    is NaN where its parameter carries no prior or is not fitted."""
    keep = host["keep"][ii, kk, :]
    var = res_perr[ii, kk, :6].astype(np.float64)
    cov = res_perr[ii, kk, 6].astype(np.float64)
    ok = keep & np.isfinite(var) & (var > 0)
    sig = np.sqrt(np.where(ok, var, 1.0))
    sig = np.where(ok, sig, np.nan)
    e1 = res_p[ii, kk, 3].astype(np.float64)
    e2 = res_p[ii, kk, 4].astype(np.float64)
    r2 = e1 * e1 + e2 * e2
    r = np.sqrt(r2)
    rs = np.where(r > 0, r, 1.0)
    radial = (e1 * e1 * var[:, 3] + 2.0 * e1 * e2 * cov + e2 * e2 * var[:, 4]) / (rs * rs)
    tangential = (e2 * e2 * var[:, 3] - 2.0 * e1 * e2 * cov + e1 * e1 * var[:, 4]) / rs ** 4
    q = np.exp(-r)
    dell = 2.0 * q / (2.0 - q) ** 2
    shape_ok = ok[:, 3] & ok[:, 4] & np.isfinite(cov) & (r > 0)

    def root(v):
        good = shape_ok & np.isfinite(v) & (v > 0)
        return np.where(good, np.sqrt(np.where(good, v, 1.0)), np.nan)
    nm = n_final[ii, kk].astype(np.float64)
    dndu = (nm - SERSIC_N_MIN) * (SERSIC_N_MAX - nm) / (SERSIC_N_MAX - SERSIC_N_MIN)
    fn = host["fn_flag"][ii, kk]
    out = dict(
        pos_x_err=sig[:, 0], pos_y_err=sig[:, 1],
        re_err=np.exp(res_p[ii, kk, 2].astype(np.float64)) * sig[:, 2],
        ell_err=root(dell * dell * radial),
        theta_err=root((90.0 / np.pi) ** 2 * tangential),
        sersic_n_err=np.where(fn, sig[:, 5] * np.abs(dndu), np.nan))
    pf = res_perr[ii, kk, 7:13].astype(np.float64)
    has = host["prior_inv_sigma"][ii, kk, :] > 0

    def frac(j):
        return np.where(keep[:, j] & has[:, j], pf[:, j], np.nan)
    both = keep[:, 3] & keep[:, 4] & has[:, 3] & has[:, 4] & (r2 > 0)
    r2s = np.where(r2 > 0, r2, 1.0)
    out.update(
        pos_x_prior_frac=frac(0), pos_y_prior_frac=frac(1), re_prior_frac=frac(2),
        ell_prior_frac=np.where(both, (e1 * e1 * pf[:, 3] + e2 * e2 * pf[:, 4]) / r2s,
                                np.nan),
        theta_prior_frac=np.where(both, (e2 * e2 * pf[:, 3] + e1 * e1 * pf[:, 4]) / r2s,
                                  np.nan),
        sersic_n_prior_frac=np.where(fn & has[:, 5], pf[:, 5], np.nan))
    return {k: np.asarray(v, np.float32) for k, v in out.items()}


def unpack_class_results(plan, host, island_set, res_p, res_f, res_fe,
                         res_chi2, res_conv, res_stall, res_nst,
                         res_perr=None, res_pdchi2=None, res_div=None,
                         res_ngood=None, n_bands=0, res_bg=None, res_bg_err=None,
                         res_railed=None, res_femarg=None, res_smetrics=None,
                         res_swin=None, res_reprof=None, reprof_deltas=None,
                         **_unused) -> dict:
    """Island rows -> source rows for the valid member slots.

    Parameter errors and prior fractions come from ``res_perr`` (the
    device covariance pass, ``compute_param_errors``; NaN without it);
    ``flux_marg_var`` from ``res_femarg`` (the shape-marginalised flux
    variance increment, ``compute_flux_marg``), the source metrics and
    window fluxes from ``res_smetrics`` / ``res_swin``
    (``compute_source_metrics``), the Re interval from ``res_reprof``
    (``compute_re_profile``); NaN without them."""
    midx, mmask, is_ext = plan.midx, host["mmask"], host["is_ext"]
    fn = host["fn_flag"]
    ii, kk = np.nonzero(mmask)
    u = res_p[:, :, 5]
    nfree = SERSIC_N_MIN + (SERSIC_N_MAX - SERSIC_N_MIN) / (1.0 + np.exp(-u))
    nfin = np.where(fn, nfree, host["sn"]).astype(np.float32)
    n = ii.size
    if res_ngood is not None and int(n_bands) > 0:
        keep_isl = (host["keep"] & mmask[:, :, None]).reshape(mmask.shape[0], -1).sum(axis=1)
        nfree_isl = keep_isl + float(n_bands) * mmask.sum(axis=1)
        dof = res_ngood.astype(np.float64) - nfree_isl
        with np.errstate(invalid="ignore", divide="ignore"):
            cn = np.where((dof > 0) & np.isfinite(res_chi2),
                          res_chi2 / np.maximum(dof, 1.0), np.nan)
        chi2_nu = cn[ii].astype(np.float32)
    else:
        chi2_nu = _nan(n)
    nb = max(int(n_bands), 0)
    if res_reprof is not None and reprof_deltas is not None:
        rlo, rhi = re_profile_interval(res_p, res_reprof, reprof_deltas, ii, kk, is_ext)
    else:
        rlo, rhi = _nan(n), _nan(n)
    if res_smetrics is not None:
        mets = dict(rchisq=res_smetrics[ii, kk, 0], fracflux=res_smetrics[ii, kk, 1],
                    fracin=res_smetrics[ii, kk, 2], fracmasked=res_smetrics[ii, kk, 3],
                    flux_win=res_swin[ii, :, kk])
    else:
        mets = dict(rchisq=_nan(n), fracflux=_nan(n), fracin=_nan(n), fracmasked=_nan(n),
                    flux_win=np.full((n, nb), np.nan, np.float32))
    if res_perr is not None:
        errs = catalog_errors(res_p, res_perr, host, ii, kk, nfin)
    else:
        errs = {k: _nan(n) for k in (
            "pos_x_err", "pos_y_err", "re_err", "ell_err", "theta_err", "sersic_n_err",
            "pos_x_prior_frac", "pos_y_prior_frac", "re_prior_frac", "ell_prior_frac",
            "theta_prior_frac", "sersic_n_prior_frac")}
    return dict(
        src=midx[ii, kk],
        pos_x=res_p[ii, kk, 0], pos_y=res_p[ii, kk, 1],
        logre=np.where(is_ext[ii, kk], res_p[ii, kk, 2], host["lr"][ii, kk]),
        ee1=np.where(is_ext[ii, kk], res_p[ii, kk, 3], host["e1"][ii, kk]),
        ee2=np.where(is_ext[ii, kk], res_p[ii, kk, 4], host["e2"][ii, kk]),
        sersic_n=nfin[ii, kk], fluxes=res_f[ii, :, kk], flux_err=res_fe[ii, :, kk],
        chi2=res_chi2[ii], chi2_nu=chi2_nu, n_steps=res_nst[ii],
        converged=res_conv[ii], stalled=res_stall[ii],
        diverged=(res_div[ii] if res_div is not None else np.zeros(n, bool)),
        stall_dchi2=(res_pdchi2[ii].astype(np.float32) if res_pdchi2 is not None
                     else _nan(n)),
        railed=(res_railed[ii] if res_railed is not None else np.zeros(n, bool)),
        free_n=fn[ii, kk],
        island_id=plan.isl_ids[ii].astype(np.int32),
        island_nsrc=island_set.n_src[plan.isl_ids][ii].astype(np.int32),
        island_giant=np.zeros(n, bool),
        re_upper_pix=np.exp(host["upper"][ii, kk, 2].astype(np.float64)).astype(np.float32),
        re_prof_lo=rlo, re_prof_hi=rhi, **errs, **mets,
        flux_marg_var=(res_femarg[ii, :, kk].astype(np.float32) if res_femarg is not None
                       else np.full((n, nb), np.nan, np.float32)),
        bg_plane=(res_bg[ii].astype(np.float32) if res_bg is not None
                  else np.zeros((n, nb, 3), np.float32)),
        bg_plane_err=(res_bg_err[ii].astype(np.float32) if res_bg_err is not None
                      else np.zeros((n, nb, 3), np.float32)))


def giant_seed_rows(giant_ids, island_set, *, pos_x, pos_y, logre, ee1, ee2,
                    sersic_n, n_bands) -> list:
    """Giant islands keep the seed geometry; nothing is solved."""
    rows = []
    nb = max(int(n_bands), 0)
    for g in sorted(int(i) for i in np.asarray(giant_ids).ravel()):
        src = np.asarray(island_set.members[g], np.int64)
        n = src.size
        nn = lambda: _nan(n)  # noqa: E731
        rows.append(dict(
            src=src,
            pos_x=np.asarray(pos_x)[src].astype(np.float32),
            pos_y=np.asarray(pos_y)[src].astype(np.float32),
            logre=np.asarray(logre)[src].astype(np.float32),
            ee1=np.asarray(ee1)[src].astype(np.float32),
            ee2=np.asarray(ee2)[src].astype(np.float32),
            sersic_n=np.asarray(sersic_n)[src].astype(np.float32),
            fluxes=np.full((n, nb), np.nan, np.float32),
            flux_err=np.full((n, nb), np.nan, np.float32),
            chi2=nn(), chi2_nu=nn(), n_steps=np.zeros(n, np.int32),
            converged=np.ones(n, bool), stalled=np.zeros(n, bool),
            diverged=np.zeros(n, bool), stall_dchi2=nn(),
            railed=np.zeros(n, bool), free_n=np.zeros(n, bool),
            island_id=np.full(n, g, np.int32), island_nsrc=np.full(n, n, np.int32),
            island_giant=np.ones(n, bool), re_upper_pix=nn(),
            pos_x_err=nn(), pos_y_err=nn(), re_err=nn(), ell_err=nn(),
            re_prof_lo=nn(), re_prof_hi=nn(), theta_err=nn(), sersic_n_err=nn(),
            pos_x_prior_frac=nn(), pos_y_prior_frac=nn(), re_prior_frac=nn(),
            ell_prior_frac=nn(), theta_prior_frac=nn(), sersic_n_prior_frac=nn(),
            rchisq=nn(), fracflux=nn(), fracin=nn(), fracmasked=nn(),
            flux_win=np.full((n, nb), np.nan, np.float32),
            flux_marg_var=np.full((n, nb), np.nan, np.float32),
            bg_plane=np.zeros((n, nb, 3), np.float32),
            bg_plane_err=np.zeros((n, nb, 3), np.float32)))
    return rows
