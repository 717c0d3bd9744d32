"""Write ``exp_mog.npz``: the exponential profile's mixture of Gaussians.

The "direct" render backend of the per-grid solve draws EXP galaxies from
the six-component mixture the reference keeps in
``tract7dt/fit/grid_gpu/source_model.py:56-75`` (Tractor's published
exponential-profile fit, amplitudes normalised to unit sum, float32); the
rendered stamps must use the same numbers to agree, so this script copies
the two arrays out of that module.  Run once with the path of a reference
checkout:

    python tests/golden/make_exp_mog.py <reference checkout>
"""
import ast
import sys
from pathlib import Path

import numpy as np


def _literal(tree, name):
    """The list literal inside the first ``name = np.array([...], ...)``."""
    for node in tree.body:
        if (isinstance(node, ast.Assign) and isinstance(node.targets[0], ast.Name)
                and node.targets[0].id == name and isinstance(node.value, ast.Call)):
            return ast.literal_eval(node.value.args[0])
    raise KeyError(name)


def main(ref_root: str) -> None:
    src = Path(ref_root) / "tract7dt" / "fit" / "grid_gpu" / "source_model.py"
    tree = ast.parse(src.read_text())
    amp = np.asarray(_literal(tree, "EXP_AMP"), np.float32)
    amp = (amp / np.sum(amp)).astype(np.float32)
    var = np.asarray(_literal(tree, "EXP_VAR"), np.float32)
    out = Path(__file__).resolve().parents[2] / "uniphot_b200" / "data" / "exp_mog.npz"
    np.savez_compressed(out, amp=amp, var=var)
    print(f"wrote {out}: {amp.size} components")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit(f"usage: python {sys.argv[0]} <reference checkout>")
    main(sys.argv[1])
