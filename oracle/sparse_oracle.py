"""CPU restatement of the reference's per-grid sparse forced photometry
(test infrastructure only: the checker of
``uph_sparse_band_solve``; nothing in ``uniphot_b200`` imports it).

Follows ``tract7dt/fit/grid_gpu/forced_phot_sparse.py``:

* stamps: the polynomial PSF at each source's full-image position
  (``psf_polynomial.py:134-197``) -- for extended sources the "fft"
  backend's galaxy stamp (``source_model.py:304-318``,
  ``sersic_mog.py:153-194``), or the "direct" backend's EXP stamp
  (``source_model.py:218-256, 298-303``) -- renormalised to unit sum on the
  all-star path (``:126-170``), Lanczos-3
  shifted by the fractional grid-local position (``:126-170``,
  ``lanczos.py:50-181``), placed at ``stamp_top_left`` (``:255-269``);
* ``solver_inner`` (``:498-555``): per-source diagonal, data and background
  couplings under the stamp (``per_source_self_blocks``, ``:355-376``),
  stamp-overlap pairs from the neighbour list (``per_pair_overlap``,
  ``:378-405``), the background Gram over the whole grid (``:417-441``);
* ``assemble_and_solve`` (``:443-496``): scatter-add of the pairs, element-
  wise ridge ``reg |diag|``, float64 solve and the diagonal of the inverse.

Arithmetic: float32 stamps and products with float64 sums rounded to
float32 (the reference sums float32 on the device), float64 solve.
"""

from __future__ import annotations

import numpy as np

from .island_oracle import (correlate_x, correlate_y, cov_terms, fft_pad_for,
                            lanczos3_taps, poly_basis)

_TERMS = {0: ((0, 0),), 1: ((0, 0), (1, 0), (0, 1)),
          2: ((0, 0), (1, 0), (0, 1), (2, 0), (1, 1), (0, 2))}


def galaxy_fft(psf_img, amps, vars_, core, cg):
    """The "fft" backend's galaxy stamp (sersic_mog.py:153-194): the
    mixture's transform times rfft2 of the zero-padded PSF, cropped, plus
    core times the PSF."""
    H, W = psf_img.shape
    pad = fft_pad_for(max(H, W))
    z = np.zeros((pad, pad))
    z[:H, :W] = psf_img
    P = np.fft.rfft2(z)
    v = np.fft.rfftfreq(pad)[None, :]
    w = np.fft.fftfreq(pad)[:, None]
    expo = -2.0 * np.pi ** 2 * (cg[0] * v * v + cg[1] * w * w + 2.0 * cg[2] * v * w)
    F = sum(a * np.exp(vv * expo) for a, vv in zip(amps, vars_))
    return np.fft.irfft2(P * F, s=(pad, pad))[:H, :W] + core * psf_img


def exp_profile_direct(H, W, logre, ee1, ee2, amp, var):
    """The "direct" backend's intrinsic exponential profile
    (source_model.py:218-256): the six-Gaussian mixture ``amp``/``var``
    sampled at pixel centres on a grid centred at (W//2, H//2), the
    quadratic form clipped at 200, normalised to unit sum."""
    y, x = np.meshgrid(np.arange(H) - H // 2, np.arange(W) - W // 2, indexing="ij")
    re = float(np.clip(np.exp(logre), 0.1, 1000.0))
    ee = float(np.hypot(ee1, ee2))
    e = 1.0 - np.exp(-ee)
    inv_ba = min((1.0 + e) / max(1.0 - e, 1e-4), 1000.0)
    th = 0.5 * np.arctan2(ee2, ee1)
    # rows of the shape matrix: (a, b) and (c, d)
    a, b = re * np.cos(th) / inv_ba, re * np.sin(th)
    c, d = -re * np.sin(th) / inv_ba, re * np.cos(th)
    prof = np.zeros((H, W))
    for am, v in zip(np.asarray(amp, np.float64), np.asarray(var, np.float64)):
        sxx, sxy, syy = v * (a * a + b * b), v * (a * c + b * d), v * (c * c + d * d)
        det = max(sxx * syy - sxy * sxy, 1e-12)
        q = (syy * x * x - 2.0 * sxy * x * y + sxx * y * y) / det
        prof += am / (2.0 * np.pi * np.sqrt(det)) * np.exp(-0.5 * np.minimum(q, 200.0))
    tot = prof.sum()
    return prof / tot if tot > 0 else prof


def convolve_same(img, ker):
    """Linear 2-D convolution cropped to ``img``'s shape, centred as
    scipy's / JAX's ``mode="same"``: the full result's rows and columns from
    (K - 1) // 2 on, K the kernel side."""
    H, W = img.shape
    kh, kw = ker.shape
    full = np.zeros((H + kh - 1, W + kw - 1))
    for i in range(kh):
        for j in range(kw):
            full[i:i + H, j:j + W] += ker[i, j] * img
    oy, ox = (kh - 1) // 2, (kw - 1) // 2
    return full[oy:oy + H, ox:ox + W]


def exp_stamp_direct(psf_img, logre, ee1, ee2, amp, var):
    """The "direct" backend's EXP stamp (source_model.py:298-303): the
    profile convolved with the PSF stamp ("same") and renormalised to unit
    box sum."""
    H, W = psf_img.shape
    s = convolve_same(exp_profile_direct(H, W, logre, ee1, ee2, amp, var), psf_img)
    tot = s.sum()
    return s / tot if tot > 0 else s


def stamps(psf, pos_x, pos_y, grid_x0, grid_y0, renorm=True, gal=None, table=None,
           backend="fft", exp_mog=None):
    """(n, H, W) float32 Lanczos-shifted PSF stamps (unit sum when
    ``renorm``); ``gal`` = (source_type, logre, ee1, ee2, sersic_n) renders
    the extended sources with the "fft" backend from ``table``, or, with
    ``backend="direct"``, the EXP sources from ``exp_mog`` = (amp, var)."""
    f32 = np.float32
    coefs = np.asarray(psf.coefs, np.float32)
    nt = coefs.shape[-1]
    out = []
    for s_i, (x, y) in enumerate(zip(np.asarray(pos_x, np.float32),
                                     np.asarray(pos_y, np.float32))):
        X = float(f32((f32(x) - f32(psf.x_origin)) / f32(psf.x_scale)))
        Y = float(f32((f32(y) - f32(psf.y_origin)) / f32(psf.y_scale)))
        b, _, _ = poly_basis(X, Y, nt)
        raw = (coefs.astype(np.float64) @ b).astype(np.float32)
        if gal is not None and int(gal[0][s_i]) != 0 and backend == "direct":
            if int(gal[0][s_i]) != 1:
                raise ValueError("the direct backend renders STAR and EXP sources only")
            raw = exp_stamp_direct(raw.astype(np.float64), float(gal[1][s_i]),
                                   float(gal[2][s_i]), float(gal[3][s_i]),
                                   *exp_mog).astype(np.float32)
        elif gal is not None and int(gal[0][s_i]) != 0:
            amps, vars_, core = table.lookup(float(gal[4][s_i]))[:3]
            cg, _ = cov_terms(float(gal[1][s_i]), float(gal[2][s_i]), float(gal[3][s_i]))
            raw = galaxy_fft(raw.astype(np.float64), amps, vars_, core, cg).astype(np.float32)
        if renorm:
            raw = (raw / np.float32(max(float(raw.astype(np.float64).sum()), 1e-12))
                   ).astype(np.float32)
        xg = f32(f32(x) - f32(grid_x0))
        yg = f32(f32(y) - f32(grid_y0))
        dx = float(f32(xg - np.rint(xg)))
        dy = float(f32(yg - np.rint(yg)))
        Lx = lanczos3_taps(dx)[0].astype(np.float32)
        Ly = lanczos3_taps(dy)[0].astype(np.float32)
        out.append(correlate_y(correlate_x(raw, Lx), Ly).astype(np.float32))
    return np.stack(out)


def bg_basis(h, w, x0, y0, xo, xs, yo, ys, order):
    X = (np.arange(w, dtype=np.float64) + x0 - xo) / xs
    Y = (np.arange(h, dtype=np.float64) + y0 - yo) / ys
    return np.stack([(X[None, :] ** m * Y[:, None] ** n) for m, n in _TERMS[order]],
                    axis=-1).astype(np.float32)        # (h, w, M)


def solve_band(data, invvar, pix_good, pos_x, pos_y, psf, grid_x0, grid_y0,
               bg_norm, order, nbr_idx, nbr_mask, reg=1e-9, renorm=True, gal=None,
               table=None, backend="fft", exp_mog=None):
    """(fluxes, bg_coefs, flux_var, bg_var) of one band, float32.  With
    extended sources in ``gal`` no stamp is renormalised (the "direct"
    backend's EXP stamps carry their own unit-sum normalisation)."""
    h, w = data.shape
    mixed = gal is not None and bool(np.any(np.asarray(gal[0]) != 0))
    S = stamps(psf, pos_x, pos_y, grid_x0, grid_y0, renorm and not mixed,
               gal if mixed else None, table, backend, exp_mog)
    n, H, W = S.shape
    x = np.asarray(pos_x, np.float32) - np.float32(grid_x0)
    y = np.asarray(pos_y, np.float32) - np.float32(grid_y0)
    ixt = np.rint(x).astype(np.int64) - W // 2
    iyt = np.rint(y).astype(np.int64) - H // 2
    wg = np.where(pix_good, invvar, 0.0).astype(np.float32)
    Bg = bg_basis(h, w, grid_x0, grid_y0, *bg_norm, order)
    M = Bg.shape[-1]
    # values under each stamp (zero outside the grid)
    ky = np.arange(H)[:, None]
    kx = np.arange(W)[None, :]
    Wu = np.zeros((n, H, W), np.float32)
    Du = np.zeros((n, H, W), np.float32)
    Bu = np.zeros((n, H, W, M), np.float32)
    Se = np.zeros_like(S)
    for s in range(n):
        ys_, xs_ = iyt[s] + ky, ixt[s] + kx
        inb = (ys_ >= 0) & (ys_ < h) & (xs_ >= 0) & (xs_ < w)
        yc, xc = np.clip(ys_, 0, h - 1), np.clip(xs_, 0, w - 1)
        Wu[s] = np.where(inb, wg[yc, xc], 0.0)
        Du[s] = data[yc, xc]
        Bu[s] = Bg[yc, xc]
        Se[s] = np.where(inb, S[s], 0.0)
    ws = (Wu * Se).astype(np.float32)
    f64 = np.float64
    diag = (ws.astype(f64) * Se).sum(axis=(1, 2)).astype(np.float32)
    tWd = (ws.astype(f64) * Du).sum(axis=(1, 2)).astype(np.float32)
    tWB = (ws[..., None].astype(f64) * Bu).sum(axis=(1, 2)).astype(np.float32)
    k_max = nbr_idx.shape[1]
    off = np.zeros((n, k_max), np.float32)
    for s in range(n):
        for k in range(k_max):
            if not nbr_mask[s, k]:
                continue
            t = int(nbr_idx[s, k])
            di, dj = iyt[s] - iyt[t], ixt[s] - ixt[t]
            tky, tkx = ky + di, kx + dj
            inn = (tky >= 0) & (tky < H) & (tkx >= 0) & (tkx < W)
            st = np.where(inn, Se[t][np.clip(tky, 0, H - 1), np.clip(tkx, 0, W - 1)], 0.0)
            off[s, k] = f64((Wu[s].astype(f64) * Se[s] * st).sum())
    bw = (Bg.reshape(-1, M) * wg.reshape(-1, 1)).astype(np.float32)
    BtWB = (bw.T.astype(f64) @ Bg.reshape(-1, M)).astype(np.float32)
    BtWd = (bw.T.astype(f64) @ data.reshape(-1).astype(f64)).astype(np.float32)
    A = np.zeros((n + M, n + M), np.float32)
    A[np.arange(n), np.arange(n)] = diag
    for s in range(n):
        for k in range(k_max):
            if nbr_mask[s, k]:
                A[s, int(nbr_idx[s, k])] += off[s, k]
    A[:n, n:] = tWB
    A[n:, :n] = tWB.T
    A[n:, n:] = BtWB
    b = np.concatenate([tWd, BtWd])
    d = np.diag(A).copy()
    A = A + np.diag((np.float32(reg) * np.maximum(np.abs(d), np.float32(1e-30))).astype(np.float32))
    A64 = A.astype(f64)
    xs = np.linalg.solve(A64, b.astype(f64)).astype(np.float32)
    var = np.diag(np.linalg.inv(A64)).astype(np.float32)
    return xs[:n], xs[n:], var[:n], var[n:]
