"""Oracle results for the heavy blend classes of the reduced production field.

The GPU test ``tests/test_gpu_blend_classes.py`` holds the plain CUDA form to
the parity bar on every class of 8, 16 and 32 members of
``make_production_field(3, side=512, n_bands=3, n_src=300)`` (analytic render
mode).  The oracle needs minutes of CPU per 32-member island, so its results
are computed once here and committed as ``oracle_blends.npz``:

* ``<class>/ref/<key>``: the oracle at reference precision (float32 render,
  residual and Gram, float64 inner solves), which the plain form must match
  (iteration counts, flags, fluxes, positions);
* ``<class>/f64/<key>``: the all-float64 oracle, against which the mixed
  form's fluxes are reported;
* ``digest``: a hash of the field (the test regenerates the field on the CPU
  and checks it before comparing), ``classes``: the class keys.

Usage::

    python tests/golden/make_oracle_blends.py [processes]
"""

from __future__ import annotations

import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE.parents[0]))
sys.path.insert(0, str(HERE))

KEYS = ("p", "fluxes", "ferr", "chi2", "conv", "stall", "diverged", "nst", "n_good")


def blend_field():
    from uniphot_b200.synth import make_production_field
    return make_production_field(3, side=512, n_bands=3, n_src=300)


def blend_classes(f):
    """The field's analytic-mode classes with at least 8 member slots."""
    from _common import field_classes
    plans, hosts, PAD, ds, ws, psfs = field_classes(f, "analytic")
    keep = [i for i, p in enumerate(plans) if p.nsrc_class >= 8]
    return ([plans[i] for i in keep], [hosts[i] for i in keep], PAD, ds, ws, psfs)


def _solve_class(args):
    from _common import run_oracle
    plan, host, PAD, ds, ws, psfs, prec, native = args
    return run_oracle([plan], [host], PAD, ds, ws, psfs, "analytic", precision=prec,
                      native=native)[0]


def main(argv):
    import multiprocessing as mp
    from make_golden_solver import field_digest
    procs = int(argv[0]) if argv else 8
    f = blend_field()
    plans, hosts, PAD, ds, ws, psfs = blend_classes(f)
    out = {"digest": np.array(field_digest(f)),
           "classes": np.array([",".join(map(str, p.key)) for p in plans])}
    # heaviest classes first, so the pool's tail is short
    jobs = sorted(((ci, prec) for prec in ("ref", "f64") for ci in range(len(plans))),
                  key=lambda j: -plans[j[0]].nsrc_class * plans[j[0]].bbox_class ** 2)
    t0 = time.perf_counter()
    with mp.get_context("spawn").Pool(procs) as pool:
        res = pool.map(_solve_class, [(plans[ci], hosts[ci], PAD, ds, ws, psfs, prec,
                                       f.native) for ci, prec in jobs], chunksize=1)
    print(f"oracle: {time.perf_counter() - t0:.1f} s", flush=True)
    for (ci, prec), r in zip(jobs, res):
        for k in KEYS:
            out[f"{ci}/{prec}/{k}"] = np.asarray(r[k])
    np.savez_compressed(HERE / "oracle_blends.npz", **out)


if __name__ == "__main__":
    main(sys.argv[1:])
