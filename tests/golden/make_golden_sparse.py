"""Golden vectors of the reference's per-grid sparse forced photometry.

Runs ``solve_band_sparse`` of ``tract7dt/fit/grid_gpu/forced_phot_sparse.py``
(``:683-718``, through ``launch_band_sparse`` / ``solver_inner`` /
``assemble_and_solve``) from a reference checkout, with JAX replaced by the
float64 numpy stand-in of ``jax_stand_in.py``, on the seeded grids of
``tests/test_sparse_cpu.py``.  Writes ``tests/golden/sparse_<case>.npz``:
fluxes, background coefficients and their variances, the neighbour list the
case used, and ``digest``, a hash of the inputs.

Usage::

    python tests/golden/make_golden_sparse.py /root/reference
"""

from __future__ import annotations

import hashlib
import importlib
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE.parent))
sys.path.insert(0, str(HERE))


def _galaxy_params(n, seed):
    rng = np.random.default_rng(seed)
    st = np.array([0, 1, 2, 3] * ((n + 3) // 4), np.int32)[:n]
    lr = rng.uniform(0.0, 1.2, n).astype(np.float32)
    e1 = rng.uniform(-0.3, 0.3, n).astype(np.float32)
    e2 = rng.uniform(-0.3, 0.3, n).astype(np.float32)
    sn = np.where(st == 1, 1.0, np.where(st == 2, 4.0, rng.uniform(0.7, 5.0, n)))
    return st, lr, e1, e2, sn.astype(np.float32)


def _exp_params(n, seed):
    rng = np.random.default_rng(seed)
    st = np.where(np.arange(n) % 2 == 0, 0, 1).astype(np.int32)
    lr = rng.uniform(0.0, 1.0, n).astype(np.float32)
    e1 = rng.uniform(-0.3, 0.3, n).astype(np.float32)
    e2 = rng.uniform(-0.3, 0.3, n).astype(np.float32)
    return st, lr, e1, e2, np.ones(n, np.float32)


# case -> (grid arguments, bg order, k_max, source parameters (or None), backend)
CASES = {
    "order0": (dict(seed=1, n=12, order=0, noise=5.0), 0, 32, None, "direct"),
    "order1": (dict(seed=2, n=12, order=1, noise=5.0), 1, 32, None, "direct"),
    "order2": (dict(seed=3, n=12, order=2, noise=5.0), 2, 32, None, "direct"),
    "crowded": (dict(seed=4, n=40, order=1, noise=5.0), 1, 4, None, "direct"),
    "galaxies_fft": (dict(seed=7, n=16, order=1, noise=5.0), 1, 32,
                     lambda n: _galaxy_params(n, 7), "fft"),
    "exp_direct": (dict(seed=8, n=12, order=1, noise=5.0), 1, 32,
                   lambda n: _exp_params(n, 8), "direct"),
    # denser grids: many overlapping stamp pairs and stamps clipped at the edge
    "field_stars": (dict(seed=11, n=150, order=2, h=200, w=220, noise=5.0), 2, 32, None,
                    "direct"),
    "field_mixed": (dict(seed=12, n=80, order=1, h=160, w=150, noise=5.0), 1, 32,
                    lambda n: _galaxy_params(n, 12), "fft"),
}


def case_inputs(case):
    """(grid dict, neighbour idx, mask, bg order, source parameters, backend)."""
    from test_sparse_cpu import _grid
    from uniphot_b200.sparse import build_neighbor_list
    gk, order, kmax, srcs, backend = CASES[case]
    g = _grid(**gk)
    idx, mask = build_neighbor_list(g["px"], g["py"], 15, 15, k_max=kmax)
    gal = srcs(g["px"].size) if srcs is not None else None
    return g, idx, mask, order, gal, backend


def digest(g, idx, mask, gal) -> str:
    h = hashlib.sha256()
    for a in (g["data"], g["invvar"], g["good"], g["px"], g["py"], g["psf"].coefs, idx, mask):
        h.update(np.ascontiguousarray(a).tobytes())
    if gal is not None:
        for a in gal:
            h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


def main(argv):
    ref_root = argv[1]
    from make_golden_solver import load_reference_solver
    _, psfmod = load_reference_solver(ref_root)
    fps = importlib.import_module("tract7dt.fit.grid_gpu.forced_phot_sparse")
    for case in argv[2:] or list(CASES):
        g, idx, mask, order, gal, backend = case_inputs(case)
        p = g["psf"]
        psf = psfmod.PsfPolynomial(coefs=np.asarray(p.coefs, np.float32),
                                   x_origin=p.x_origin, x_scale=p.x_scale,
                                   y_origin=p.y_origin, y_scale=p.y_scale,
                                   H_psf=p.coefs.shape[0], W_psf=p.coefs.shape[1])
        h, w = g["data"].shape
        kw = {}
        if gal is not None:
            kw = dict(source_type=gal[0], logre=gal[1], ee1=gal[2], ee2=gal[3],
                      sersic_n=gal[4])
        inp = fps.GridBandInputs(
            data=g["data"], invvar=g["invvar"], pix_good=g["good"], pos_x=g["px"],
            pos_y=g["py"], psf_jax=psf.to_jax(), band_h=h, band_w=w, grid_x0=g["gx0"],
            grid_y0=g["gy0"], bg_x_origin=g["bn"][0], bg_x_scale=g["bn"][1],
            bg_y_origin=g["bn"][2], bg_y_scale=g["bn"][3], render_backend=backend, **kw)
        r = fps.solve_band_sparse(inp, idx, mask, reg=1e-9, bg_poly_order=order)
        np.savez_compressed(HERE / f"sparse_{case}.npz",
                            digest=np.array(digest(g, idx, mask, gal)),
                            fluxes=np.asarray(r.fluxes), bg_coefs=np.asarray(r.bg_coefs),
                            flux_var=np.asarray(r.flux_var), bg_var=np.asarray(r.bg_var))
        print(case, "done", flush=True)


if __name__ == "__main__":
    main(sys.argv)
