"""Write ``sersic_mog_table.npz``: the Sersic mixture-of-Gaussians table.

The galaxy profiles must use the same mixture table as the reference
(``tract7dt/data/sersic_mog_table.npz``, read by
``tract7dt/fit/grid_gpu/sersic_mog.py:48-56``) for the rendered models to
agree; the table is data, so this script copies its numeric arrays (knots,
amplitudes, log-variances, delta-core amplitude, bounds) into the package.
Run once with the path of a reference checkout:

    python tests/golden/make_sersic_table.py <reference checkout>
"""
import sys
from pathlib import Path

import numpy as np


def main(ref_root: str) -> None:
    src = Path(ref_root) / "tract7dt" / "data" / "sersic_mog_table.npz"
    z = np.load(src)
    out = Path(__file__).resolve().parents[2] / "uniphot_b200" / "data" / "sersic_mog_table.npz"
    np.savez_compressed(
        out, n_knots=z["n_knots"], amps=z["amps"], log_vars=z["log_vars"],
        core_amp=z["core_amp"], n_min=z["n_min"], n_max=z["n_max"])
    print(f"wrote {out}")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <reference checkout>")
    main(sys.argv[1])
