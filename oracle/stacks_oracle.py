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
