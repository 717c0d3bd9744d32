"""Golden vectors of the island stage's field-stack build: the seeded field
and tiles of ``tests/test_stacks_cpu.py`` through the reference's own
``make_bg_basis`` (bg_polynomial.py:125-178) and the subtraction loop of
island_stage.py:1728-1751 (restated here around the reference's basis, as
the loop itself sits inside ``run_island_prestage``).  Writes
``tests/golden/stacks_small.npz``: the padded data stack per background
order and ``digest``, a hash of the inputs.

Usage::

    python tests/golden/make_golden_stacks.py /root/reference
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE))


def main(ref_root: str) -> None:
    import importlib
    from make_golden_solver import load_reference_solver
    from test_stacks_cpu import PAD, digest, small_case
    load_reference_solver(ref_root)
    bgp = importlib.import_module("tract7dt.fit.grid_gpu.bg_polynomial")
    out = {}
    for order in (0, 1, 2):
        data, invvar, tiles, coefs, norm = small_case(order)
        nb, H, W = data.shape
        dmb = np.zeros((nb, H + 2 * PAD, W + 2 * PAD), np.float32)
        dmb[:, PAD:PAD + H, PAD:PAD + W] = data
        for t, (x0, y0, x1, y1) in enumerate(tiles):
            h, w = y1 - y0, x1 - x0
            basis = bgp.make_bg_basis(h, w, x0, y0, *norm, order=order)
            for b in range(nb):
                dmb[b, PAD + y0:PAD + y1, PAD + x0:PAD + x1] -= (
                    basis @ np.asarray(coefs[t][b], np.float32)).reshape(h, w)
        out[f"dmb_order{order}"] = dmb
        out[f"digest_order{order}"] = np.array(digest(order))
    np.savez_compressed(HERE / "stacks_small.npz", **out)
    print("wrote", HERE / "stacks_small.npz")


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "")
