"""CPU restatement of the island stage's field-stack build (test
infrastructure: the checker of the device kernel, never the product path).

The padded stacks are the band data and inverse variances placed inside a
border of ``pad`` zeros, with each pass-1 tile's frozen planar background
subtracted from the data over the tile's core rectangle
(island_stage.py:1728-1751): ``stack[b, pad + y0:pad + y1, pad + x0:pad +
x1] -= (basis @ coefs[t, b]).reshape(h, w)`` with ``basis`` the tile's
make_bg_basis (bg_polynomial.py:125-178, float32 terms X^m Y^n computed in
float64), tiles in order.  Pinned to the reference's own make_bg_basis by
``tests/golden/stacks_small.npz`` (``tests/golden/make_golden_stacks.py``).
"""

from __future__ import annotations

import numpy as np

from .sparse_oracle import bg_basis


def field_stacks(data, invvar, pad, tiles, coefs, order, norm):
    """(data stack, invvar stack), each (n_bands, H + 2 pad, W + 2 pad)
    float32.  ``tiles`` (n, 4) = (x0, y0, x1, y1) cores, ``coefs`` (n,
    n_bands, M) float32, ``norm`` = (x_origin, x_scale, y_origin, y_scale)."""
    data = np.asarray(data, np.float32)
    invvar = np.asarray(invvar, np.float32)
    nb, H, W = data.shape
    dmb = np.zeros((nb, H + 2 * pad, W + 2 * pad), np.float32)
    iv = np.zeros_like(dmb)
    dmb[:, pad:pad + H, pad:pad + W] = data
    iv[:, pad:pad + H, pad:pad + W] = invvar
    xo, xs, yo, ys = (float(v) for v in norm)
    for t, (x0, y0, x1, y1) in enumerate(np.asarray(tiles, np.int64)):
        h, w = int(y1 - y0), int(x1 - x0)
        basis = bg_basis(h, w, int(x0), int(y0), xo, xs, yo, ys, order).reshape(h * w, -1)
        for b in range(nb):
            dmb[b, pad + y0:pad + y1, pad + x0:pad + x1] -= (
                basis @ np.asarray(coefs[t][b], np.float32)).reshape(h, w)
    return dmb, iv


def scene_subtract_stars(dmb, x, y, flux, psfs, native, pad):
    """The field-wide star scene subtraction (island_stage.py:2024-2118) on a
    padded data stack (modified in place and returned): per band, per source
    in index order with a nonzero flux, ``dmb[b, iy:iy + T, ix:ix + T] -=
    flux * stamp`` over the part inside the stack, with the stamp the band's
    polynomial PSF at the float32 position, Lanczos-shifted, not
    renormalised (``_star_stamps_jit``, island_stage.py:99-130; the
    stamps of ``sparse_oracle.stamps``, pinned to the reference through the
    per-grid solve's golden fixtures) and the corner ``round(x) - T // 2 +
    pad`` of the float64 position.  ``psfs``: per-band polynomial PSFs of
    stamp side ``native``."""
    from .sparse_oracle import stamps
    x = np.asarray(x, np.float64)
    y = np.asarray(y, np.float64)
    flux = np.asarray(flux, np.float32)
    T = int(native)
    nb, Hp, Wp = dmb.shape
    ixt = np.round(x).astype(np.int64) - T // 2 + pad
    iyt = np.round(y).astype(np.int64) - T // 2 + pad
    for b in range(nb):
        st = stamps(psfs[b], x.astype(np.float32), y.astype(np.float32), 0, 0, renorm=False)
        for k in range(x.size):
            f = np.float32(flux[k, b])
            if f == 0.0:
                continue
            ix, iy = int(ixt[k]), int(iyt[k])
            y0c, x0c = max(0, -iy), max(0, -ix)
            ye, xe = min(T, Hp - iy), min(T, Wp - ix)
            if ye <= y0c or xe <= x0c:
                continue
            dmb[b, iy + y0c:iy + ye, ix + x0c:ix + xe] -= f * st[k, y0c:ye, x0c:xe]
    return dmb
