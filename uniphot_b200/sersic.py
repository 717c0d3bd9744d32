"""Sersic mixture-of-Gaussians table (data shared with the reference).

The table (``data/sersic_mog_table.npz``) holds, on a knot grid in n, the
amplitudes and log-variances of up to 15 Gaussian components plus a delta
core amplitude.  Lookup is linear interpolation in n inside one knot segment
(``searchsorted(..., 'right') - 1``), clamped to [n_min, n_max], as in the
reference's ``fit/grid_gpu/sersic_mog.py:81-100``.  The device copy of the
table is uploaded by the C-ABI (``uph_upload_sersic_table``).
"""

from __future__ import annotations

from functools import lru_cache
from pathlib import Path

import numpy as np

K_MAX = 15
_PATH = Path(__file__).resolve().parent / "data" / "sersic_mog_table.npz"


@lru_cache(maxsize=1)
def load_table() -> dict:
    z = np.load(_PATH)
    return {k: np.asarray(z[k]) for k in z.files}


def mog_params_np(table: dict, n: float):
    """(amps[15], vars[15], core) at Sersic index n."""
    kn = table["n_knots"]
    n = float(np.clip(n, float(table["n_min"]), float(table["n_max"])))
    i = int(np.clip(np.searchsorted(kn, n, side="right") - 1, 0, kn.size - 2))
    n0, n1 = kn[i], kn[i + 1]
    t = (n - n0) / (n1 - n0) if n1 > n0 else 0.0
    a = (1 - t) * table["amps"][i] + t * table["amps"][i + 1]
    lv = (1 - t) * table["log_vars"][i] + t * table["log_vars"][i + 1]
    core = (1 - t) * table["core_amp"][i] + t * table["core_amp"][i + 1]
    return a, np.exp(lv), float(core)
