"""Seeded synthetic forced-photometry fields for the benchmark configurations.

The truth image is rendered independently of the solver's forward model:
every source is an analytic mixture of Gaussians (galaxy MoG from the Sersic
table, convolved analytically with the band's Gaussian-mixture PSF) sampled
at pixel centres around its exact sub-pixel position -- no Lanczos shift, no
pixelised PSF -- so the fit carries a realistic small model mismatch.

* ``make_small_field`` -- the small plain-method field: 256x256, 3 bands,
  constant 3-component circular PSF (sigma 1.2/2.0/3.5 px, weights
  0.7/0.25/0.05), 30 STAR + 10 EXP, log-uniform fluxes 1e2-1e5 per band,
  planar background 100 +- 0.01 px^-1 gradients (one tile per band),
  Poisson(model + bg) + N(0, 5^2) noise, exact inverse-variance weights,
  positions jittered N(0, 0.3 px), friends-of-friends islands at 8 px.
* ``make_production_field`` -- the production field: 2048x2048, 20 bands,
  4-component elliptical Gaussian-mixture PSF whose sigma, e1, e2 and weights
  are order-2 polynomials in position (FWHM 2.5-4.5 px), 5000 sources
  (60% STAR, 20% EXP, 12% DEV, 8% SERSIC with n ~ U(0.5, 6)), r_e log-uniform
  0.5-15 px, fluxes log-uniform 1e1-1e6, Poisson-clustered positions, planar
  background per 256x256 tile.  ``scale`` shrinks side/bands/sources for CPU
  tests.

Public datasets are not used: these seeded inputs stand in for them.
"""

from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

from . import islands as _isl
from .psf import MogPsf, PsfPolynomial, mog_to_poly_psf, rasterize_mog_psf
from .sersic import load_table, mog_params_np

SOURCE_STAR, SOURCE_EXP, SOURCE_DEV, SOURCE_SERSIC = 0, 1, 2, 3


@dataclass
class Field:
    """A synthetic field plus everything ``island_fit`` takes."""
    data_minus_bg: np.ndarray      # (n_b, H, W) f32
    invvar: np.ndarray             # (n_b, H, W) f32
    mog_psfs: list                 # per band MogPsf (analytic render)
    poly_psfs: list                # per band PsfPolynomial (reference render)
    pos_x: np.ndarray
    pos_y: np.ndarray
    source_type: np.ndarray
    logre: np.ndarray
    ee1: np.ndarray
    ee2: np.ndarray
    sersic_n: np.ndarray
    s1_flux: np.ndarray            # (n_src, n_b)
    s1_flux_var: np.ndarray
    true_x: np.ndarray
    true_y: np.ndarray
    true_flux: np.ndarray          # (n_src, n_b)
    island_set: object
    buckets: object
    native: int
    tier_ladder: tuple

    @property
    def bandnames(self):
        return [f"b{i}" for i in range(self.data_minus_bg.shape[0])]

    def fit_kwargs(self, render_mode: str) -> dict:
        """Keyword arguments of ``island_fit`` for this field."""
        return dict(
            bandnames=self.bandnames, data_minus_bg=self.data_minus_bg,
            invvar=self.invvar,
            psfs=self.mog_psfs if render_mode == "analytic" else self.poly_psfs,
            island_set=self.island_set, buckets=self.buckets,
            pos_x=self.pos_x, pos_y=self.pos_y, source_type=self.source_type,
            logre=self.logre, ee1=self.ee1, ee2=self.ee2,
            sersic_n=self.sersic_n, s1_flux=self.s1_flux,
            s1_flux_var=self.s1_flux_var, render_mode=render_mode,
            tier_ladder=self.tier_ladder, native_stamp=self.native)


def ellipse_soft(re_pix, ab, phi_deg):
    """(re, b/a, phi) -> (logre, ee1, ee2) soft-ellipse parameters
    (source_model.py:104-121)."""
    re = np.clip(np.asarray(re_pix, np.float64), 0.1, 1000.0)
    ba = np.clip(np.asarray(ab, np.float64), 0.1, 1.0)
    e = np.clip((1.0 / ba - 1.0) / (1.0 / ba + 1.0), 0.0, 0.999999)
    ee = -np.log(np.maximum(1.0 - e, 1e-12))
    ang = np.deg2rad(-2.0 * np.asarray(phi_deg, np.float64))
    return (np.log(re).astype(np.float32), (ee * np.cos(ang)).astype(np.float32),
            (ee * np.sin(ang)).astype(np.float32))


def _cov_unit(logre, ee1, ee2):
    """Vectorised unit-variance galaxy covariance (cxx, cyy, cxy)."""
    re = np.clip(np.exp(logre.astype(np.float64)), 0.1, 1000.0)
    e1 = np.where((ee1 == 0) & (ee2 == 0), 1e-4, ee1).astype(np.float64)
    e2 = ee2.astype(np.float64)
    ee = np.hypot(e1, e2)
    e = 1.0 - np.exp(-ee)
    ib = np.minimum((1 + e) / np.maximum(1 - e, 1e-4), 1000.0)
    th = 0.5 * np.arctan2(e2, e1)
    ct, st = np.cos(th), np.sin(th)
    s2 = 1.0 / (ib * ib)
    return (re * re * (ct * ct * s2 + st * st), re * re * (st * st * s2 + ct * ct),
            re * re * ct * st * (1 - s2))


def render_truth(shape, psfs: list, x, y, stype, logre, ee1, ee2, sersic_n,
                 flux, half, device="cpu"):
    """Sum of flux * analytic unit models, sampled at pixel centres.

    ``half[i]`` is the render half-size of source i (pixels).  Batched over
    sources with torch (any device)."""
    import torch
    nb, H, W = shape
    table = load_table()
    n = x.shape[0]
    cxx, cyy, cxy = _cov_unit(logre, ee1, ee2)
    kg = table["amps"].shape[1] + 1
    gal_a = np.zeros((n, kg))
    gal_v = np.zeros((n, kg))
    for i in range(n):
        if stype[i] == SOURCE_STAR:
            gal_a[i, 0] = 1.0
        else:
            nn = 1.0 if stype[i] == SOURCE_EXP else float(sersic_n[i])
            a, v, core = mog_params_np(table, nn)
            gal_a[i, :a.size] = a
            gal_v[i, :a.size] = v
            gal_a[i, a.size] = core
    out = torch.zeros((nb, H, W), dtype=torch.float64, device=device)
    flat = out.view(nb, -1)
    for hs in np.unique(half):
        sel = np.nonzero(half == hs)[0]
        R = int(hs)
        S = 2 * R + 1
        off = torch.arange(-R, R + 1, dtype=torch.float64, device=device)
        for b in range(nb):
            wq_all, cq_all = psfs[b].components_at(x[sel], y[sel])
            K = wq_all.shape[1]
            chunk = max(1, int(4e7 // (K * kg * S * S)))
            for c0 in range(0, sel.size, chunk):
                ids = sel[c0:c0 + chunk]
                m = ids.size
                ix = np.rint(x[ids]).astype(np.int64)
                iy = np.rint(y[ids]).astype(np.int64)
                t = lambda a: torch.as_tensor(a, dtype=torch.float64, device=device)  # noqa: E731
                fx, fy = t(x[ids] - ix), t(y[ids] - iy)
                xx = (off[None, :] - fx[:, None])[:, None, None, :]      # (m,1,1,S)
                yy = (off[None, :] - fy[:, None])[:, None, :, None]      # (m,1,S,1)
                wq = t(wq_all[c0:c0 + m])                                # (m,K)
                cq = t(cq_all[c0:c0 + m])                                # (m,K,3)
                ga, gv = t(gal_a[ids]), t(gal_v[ids])                    # (m,kg)
                A = gv[:, None, :] * t(cxx[ids])[:, None, None] + cq[:, :, None, 0]
                C = gv[:, None, :] * t(cyy[ids])[:, None, None] + cq[:, :, None, 1]
                Bc = gv[:, None, :] * t(cxy[ids])[:, None, None] + cq[:, :, None, 2]
                det = A * C - Bc * Bc                                     # (m,K,kg)
                amp = (wq[:, :, None] * ga[:, None, :]
                       / (2 * math.pi * torch.sqrt(det))) * t(flux[ids, b])[:, None, None]
                A, C, Bc, det, amp = (v.reshape(m, K * kg, 1, 1)
                                      for v in (A, C, Bc, det, amp))
                Q = (C * xx * xx - 2 * Bc * xx * yy + A * yy * yy) / det
                img = (amp * torch.exp(-0.5 * Q)).sum(dim=1)              # (m,S,S)
                gy = torch.as_tensor(iy, device=device)[:, None, None] + off.long()[None, :, None]
                gx = torch.as_tensor(ix, device=device)[:, None, None] + off.long()[None, None, :]
                ok = (gy >= 0) & (gy < H) & (gx >= 0) & (gx < W)
                idx = (gy * W + gx).expand(m, S, S)[ok]
                flat[b].index_add_(0, idx, img[ok])
    return out.cpu().numpy()


def _noise(model, bg, rng):
    lam = np.clip(model + bg, 0.0, None)
    data = rng.poisson(lam).astype(np.float64) + rng.normal(0.0, 5.0, lam.shape)
    invvar = 1.0 / (lam + 25.0)
    return (data - bg).astype(np.float32), invvar.astype(np.float32)


def _islands(x, y, stype, logre, sersic_n, native, radius=None, s1_flux=None,
             invvar=None, psf_stamp=None, kappa=0.5):
    r_psf = native / 2.0
    if radius is None:
        sig = float(np.median([np.median(1.0 / np.sqrt(iv[::16, ::16][iv[::16, ::16] > 0]))
                               for iv in invvar]))
        pr, pp = _isl.psf_radial_profile(psf_stamp)
        radius = _isl.flux_aware_radii(stype, logre, sersic_n,
                                       np.median(s1_flux, axis=1), sig, kappa,
                                       pr, pp, r_psf)
    iset = _isl.build_islands(x, y, stype, logre, sersic_n, r_psf, radius=radius)
    return iset, _isl.bucket_islands(iset)


def make_small_field(seed: int = 0, n_star: int = 30, n_exp: int = 10,
                     side: int = 256, n_bands: int = 3, device="cpu") -> Field:
    """Small plain-method field (see module docstring)."""
    rng = np.random.default_rng(seed)
    nb, H, W = n_bands, side, side
    n = n_star + n_exp
    sig = np.array([1.2, 2.0, 3.5])
    wts = np.array([0.7, 0.25, 0.05])
    mogs = [MogPsf.constant(sig, np.zeros(3), np.zeros(3), wts,
                            x_origin=W / 2, x_scale=W / 2, y_origin=H / 2,
                            y_scale=H / 2) for _ in range(nb)]
    native = 55
    polys = [rasterize_mog_psf(m, native, W / 2, H / 2) for m in mogs]
    tx = rng.uniform(4, W - 4, n)
    ty = rng.uniform(4, H - 4, n)
    st = np.array([SOURCE_STAR] * n_star + [SOURCE_EXP] * n_exp, np.int32)
    re = np.where(st == SOURCE_EXP, rng.uniform(1, 4, n), 1.0)
    q = rng.uniform(0.4, 1.0, n)
    pa = rng.uniform(0, 180.0, n)
    lr, e1, e2 = ellipse_soft(re, q, pa)
    lr = np.where(st == SOURCE_STAR, 0.0, lr).astype(np.float32)
    e1 = np.where(st == SOURCE_STAR, 0.0, e1).astype(np.float32)
    e2 = np.where(st == SOURCE_STAR, 0.0, e2).astype(np.float32)
    sn = np.ones(n, np.float32)
    flux = np.exp(rng.uniform(np.log(1e2), np.log(1e5), (n, nb)))
    half = np.full(n, native // 2)
    model = render_truth((nb, H, W), mogs, tx, ty, st, lr, e1, e2, sn, flux,
                         half, device)
    yy, xx = np.mgrid[0:H, 0:W].astype(np.float64)
    bg = np.stack([100.0 + rng.uniform(-0.01, 0.01) * (xx - W / 2)
                   + rng.uniform(-0.01, 0.01) * (yy - H / 2) for _ in range(nb)])
    dmb, iv = _noise(model, bg, rng)
    px = (tx + rng.normal(0, 0.3, n)).astype(np.float32)
    py = (ty + rng.normal(0, 0.3, n)).astype(np.float32)
    s1 = (flux * (1 + 0.05 * rng.normal(size=flux.shape))).astype(np.float32)
    s1v = ((0.05 * flux) ** 2 + 25.0).astype(np.float32)
    iset, bk = _islands(px, py, st, lr, sn, native, radius=np.full(n, 4.0))
    return Field(dmb, iv, mogs, polys, px, py, st, lr, e1, e2, sn, s1, s1v,
                 tx, ty, flux, iset, bk, native, (111, 221))


def make_production_field(seed: int = 0, side: int = 2048, n_bands: int = 20,
                          n_src: int = 5000, device="cpu",
                          tier_ladder=(63, 127), margin: float = 40.0) -> Field:
    """Production field (see module docstring); cluster centres keep
    ``margin`` px from the edges."""
    rng = np.random.default_rng(seed)
    nb, H, W = n_bands, side, side
    native = 31
    mogs = []
    for b in range(nb):
        fwhm = rng.uniform(2.5, 4.5)
        s0 = fwhm / 2.355
        base_s = np.array([0.75, 1.1, 1.8, 3.2]) * s0
        base_w = np.array([0.45, 0.35, 0.15, 0.05])
        sig = np.zeros((4, 6))
        e1 = np.zeros((4, 6))
        e2 = np.zeros((4, 6))
        wt = np.zeros((4, 6))
        sig[:, 0] = base_s
        sig[:, 1:3] = base_s[:, None] * rng.uniform(-0.08, 0.08, (4, 2))
        sig[:, 3:6] = base_s[:, None] * rng.uniform(-0.04, 0.04, (4, 3))
        e1[:, 0] = rng.uniform(-0.06, 0.06, 4)
        e2[:, 0] = rng.uniform(-0.06, 0.06, 4)
        e1[:, 1:6] = rng.uniform(-0.02, 0.02, (4, 5))
        e2[:, 1:6] = rng.uniform(-0.02, 0.02, (4, 5))
        wt[:, 0] = base_w
        wt[:, 1:6] = base_w[:, None] * rng.uniform(-0.05, 0.05, (4, 5))
        mogs.append(MogPsf(sig, e1, e2, wt, W / 2, W / 2, H / 2, H / 2))
    polys = [mog_to_poly_psf(m, native, W, H) for m in mogs]
    # Poisson-clustered positions: power-law cluster sizes 1..64.
    xs, ys = [], []
    while sum(len(a) for a in xs) < n_src:
        size = int(min(64, max(1, np.floor(rng.pareto(1.2) + 1))))
        cx, cy = rng.uniform(margin, W - margin), rng.uniform(margin, H - margin)
        spread = 3.0 + 1.5 * math.sqrt(size)
        xs.append(np.clip(cx + rng.normal(0, spread, size), 8, W - 8))
        ys.append(np.clip(cy + rng.normal(0, spread, size), 8, H - 8))
    tx = np.concatenate(xs)[:n_src]
    ty = np.concatenate(ys)[:n_src]
    n = tx.size
    u = rng.uniform(size=n)
    st = np.where(u < 0.6, SOURCE_STAR, np.where(u < 0.8, SOURCE_EXP,
                  np.where(u < 0.92, SOURCE_DEV, SOURCE_SERSIC))).astype(np.int32)
    re = np.exp(rng.uniform(np.log(0.5), np.log(15.0), n))
    q = rng.uniform(0.4, 1.0, n)
    pa = rng.uniform(0, 180.0, n)
    lr, e1s, e2s = ellipse_soft(re, q, pa)
    is_star = st == SOURCE_STAR
    lr = np.where(is_star, 0.0, lr).astype(np.float32)
    e1s = np.where(is_star, 0.0, e1s).astype(np.float32)
    e2s = np.where(is_star, 0.0, e2s).astype(np.float32)
    sn = np.where(st == SOURCE_DEV, 4.0, np.where(st == SOURCE_SERSIC,
                  rng.uniform(0.5, 6.0, n), 1.0)).astype(np.float32)
    flux = np.exp(rng.uniform(np.log(1e1), np.log(1e6), (n, 1)))
    flux = flux * np.exp(rng.normal(0, 0.3, (n, nb)))
    nre = np.where(sn < 1.5, 4.0, np.where(sn < 3.0, 6.0, 8.0))
    half = np.where(is_star, native // 2,
                    np.minimum(tier_ladder[-1] // 2,
                               np.ceil(nre * np.exp(lr) + native // 2))).astype(np.int64)
    model = render_truth((nb, H, W), mogs, tx, ty, st, lr, e1s, e2s, sn, flux,
                         half, device)
    bg = np.zeros((nb, H, W))
    yy, xx = np.mgrid[0:H, 0:W].astype(np.float64)
    for b in range(nb):
        for ty0 in range(0, H, 256):
            for tx0 in range(0, W, 256):
                gx, gy = rng.uniform(-0.01, 0.01, 2)
                sl = (slice(ty0, ty0 + 256), slice(tx0, tx0 + 256))
                bg[b][sl] = 100.0 + gx * (xx[sl] - tx0 - 128) + gy * (yy[sl] - ty0 - 128)
    dmb, iv = _noise(model, bg, rng)
    px = (tx + rng.normal(0, 0.3, n)).astype(np.float32)
    py = (ty + rng.normal(0, 0.3, n)).astype(np.float32)
    s1 = (flux * (1 + 0.05 * rng.normal(size=flux.shape))).astype(np.float32)
    s1v = ((0.05 * flux) ** 2 + 25.0).astype(np.float32)
    stamp = polys[0].stamp_at(W / 2, H / 2)
    iset, bk = _islands(px, py, st, lr, sn, native, s1_flux=s1, invvar=iv,
                        psf_stamp=stamp)
    return Field(dmb, iv, mogs, polys, px, py, st, lr, e1s, e2s, sn, s1, s1v,
                 tx, ty, flux, iset, bk, native, tuple(tier_ladder))


def serving_request_shape(rng) -> tuple:
    """(side, n_bands, n_sources) of one serving request: cutout side
    log-normal clipped to 64-1024 px, bands uniform in 1..40, sources at the
    production field's density (x U(0.5, 2)) clipped to 5-2000."""
    side = int(np.clip(np.exp(rng.normal(np.log(256.0), 0.6)), 64, 1024))
    n_bands = int(rng.integers(1, 41))
    dens = 5000.0 / 2048.0 ** 2
    n_src = int(np.clip(round(dens * side * side * rng.uniform(0.5, 2.0)), 5, 2000))
    return side, n_bands, n_src


def make_serving_request(seed: int, device="cpu") -> Field:
    """One serving request: a field cutout drawn like the production field
    (its own PSF polynomial coefficients, sources, noise) with the shape of
    ``serving_request_shape``."""
    rng = np.random.default_rng(10_000 + seed)
    side, nb, n_src = serving_request_shape(rng)
    return make_production_field(seed, side=side, n_bands=nb, n_src=n_src,
                                 device=device, margin=min(40.0, side / 4.0))


def make_blend_field(seed: int = 0, n_islands: int = 400, n_bands: int = 40,
                     device="cpu", spacing: int = 64) -> Field:
    """Precision-stress field: ``n_islands`` crowded blends of 2-12 point
    sources on a grid ``spacing`` px apart.  Within a blend each new source
    sits U(0.3, 1.5) FWHM from a random earlier member; the brightest has a
    flux log-U(1e3, 1e6) and the others fainter by a ratio log-U(1, 1e4).  A
    quarter of the bands scale every flux down to SNR ~3-10 for the faint
    members.  PSF as in the production field (4-Gaussian, order-2
    polynomial); islands by the production field's flux-aware radii."""
    rng = np.random.default_rng(20_000 + seed)
    g = int(math.ceil(math.sqrt(n_islands)))
    side = g * spacing + spacing
    nb, H, W = n_bands, side, side
    native = 31
    base = make_production_field(seed, side=64, n_bands=nb, n_src=5, margin=16)
    mogs = [type(m)(m.sigma, m.e1, m.e2, m.weight, W / 2, W / 2, H / 2, H / 2)
            for m in base.mog_psfs]
    fwhm = 2.355 * float(np.mean([m.sigma[1, 0] for m in mogs]))
    xs, ys, fl = [], [], []
    for i in range(n_islands):
        cx = spacing + (i % g) * spacing + rng.uniform(-2, 2)
        cy = spacing + (i // g) * spacing + rng.uniform(-2, 2)
        k = int(rng.integers(2, 13))
        px, py = [cx], [cy]
        for _ in range(k - 1):
            j = int(rng.integers(0, len(px)))
            r = rng.uniform(0.3, 1.5) * fwhm
            a = rng.uniform(0, 2 * math.pi)
            px.append(px[j] + r * math.cos(a))
            py.append(py[j] + r * math.sin(a))
        f0 = math.exp(rng.uniform(math.log(1e3), math.log(1e6)))
        ratios = np.exp(rng.uniform(0, math.log(1e4), k))
        ratios[0] = 1.0
        xs.extend(px)
        ys.extend(py)
        fl.extend(f0 / ratios)
    tx, ty = np.asarray(xs), np.asarray(ys)
    n = tx.size
    flux = np.asarray(fl)[:, None] * np.exp(rng.normal(0, 0.3, (n, nb)))
    faint = rng.uniform(size=nb) < 0.25
    flux[:, faint] *= np.exp(rng.uniform(np.log(1e-3), np.log(1e-2), faint.sum()))
    st = np.full(n, SOURCE_STAR, np.int32)
    zero = np.zeros(n, np.float32)
    sn = np.ones(n, np.float32)
    half = np.full(n, native // 2)
    model = render_truth((nb, H, W), mogs, tx, ty, st, zero, zero, zero, sn, flux,
                         half, device)
    bg = np.full((nb, H, W), 100.0)
    dmb, iv = _noise(model, bg, rng)
    px = (tx + rng.normal(0, 0.3, n)).astype(np.float32)
    py = (ty + rng.normal(0, 0.3, n)).astype(np.float32)
    s1 = (flux * (1 + 0.05 * rng.normal(size=flux.shape))).astype(np.float32)
    s1v = ((0.05 * flux) ** 2 + 25.0).astype(np.float32)
    polys = [mog_to_poly_psf(m, native, W, H) for m in mogs]
    stamp = polys[0].stamp_at(W / 2, H / 2)
    iset, bk = _islands(px, py, st, zero, sn, native, s1_flux=s1, invvar=iv,
                        psf_stamp=stamp)
    return Field(dmb, iv, mogs, polys, px, py, st, zero, zero.copy(), zero.copy(),
                 sn, s1, s1v, tx, ty, flux, iset, bk, native, (63, 127))
