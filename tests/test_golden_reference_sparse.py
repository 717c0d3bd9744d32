"""The sparse oracle against the reference's own per-grid solve.

``tests/golden/sparse_<case>.npz`` hold the results of the reference's
``solve_band_sparse`` (forced_phot_sparse.py:683-718) on the seeded grids of
``test_sparse_cpu.py``, made by ``tests/golden/make_golden_sparse.py`` with
the float64 numpy stand-in for JAX: background orders 0-2, a crowded grid
with a neighbour list truncated at 4, stars with EXP/DEV/SERSIC galaxies on
the "fft" backend, and stars with EXP galaxies on the "direct" backend
(source_model.py:218-256, 298-303).  The oracle must give the same fluxes
(1e-5 relative or 1e-3 sigma), background coefficients (1e-3 sigma) and
variances (1e-5 relative).
"""

import sys
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).parent / "golden"
sys.path.insert(0, str(GOLDEN))

from make_golden_sparse import CASES, case_inputs, digest  # noqa: E402


@pytest.mark.parametrize("case", sorted(CASES))
def test_sparse_oracle_matches_reference(case):
    from _common import TABLE
    from oracle import sparse_oracle as SO
    from oracle.island_oracle import SersicTable
    path = GOLDEN / f"sparse_{case}.npz"
    if not path.exists():
        pytest.skip(f"fixture {path.name} not generated")
    r = np.load(path)
    g, idx, mask, order, gal, backend = case_inputs(case)
    assert str(r["digest"]) == digest(g, idx, mask, gal), "inputs changed since the fixture"
    z = np.load(Path(__file__).parents[1] / "uniphot_b200" / "data" / "exp_mog.npz")
    f, b, fv, bv = SO.solve_band(
        g["data"], g["invvar"], g["good"], g["px"], g["py"], g["psf"], g["gx0"], g["gy0"],
        g["bn"], order, idx, mask, reg=1e-9, gal=gal,
        table=SersicTable.load(TABLE) if gal is not None else None, backend=backend,
        exp_mog=(z["amp"], z["var"]))
    df = np.abs(f - r["fluxes"])
    assert np.all(df <= np.maximum(1e-5 * np.abs(r["fluxes"]), 1e-3 * np.sqrt(r["flux_var"])))
    assert np.all(np.abs(b - r["bg_coefs"]) <= 1e-3 * np.sqrt(r["bg_var"]))
    np.testing.assert_allclose(fv, r["flux_var"], rtol=1e-5)
    np.testing.assert_allclose(bv, r["bg_var"], rtol=1e-5)


def test_direct_backend_rejects_dev_and_sersic():
    from oracle import sparse_oracle as SO
    g, idx, mask, order, gal, _ = case_inputs("exp_direct")
    st = gal[0].copy()
    st[1] = 2
    z = np.load(Path(__file__).parents[1] / "uniphot_b200" / "data" / "exp_mog.npz")
    with pytest.raises(ValueError):
        SO.solve_band(g["data"], g["invvar"], g["good"], g["px"], g["py"], g["psf"],
                      g["gx0"], g["gy0"], g["bn"], order, idx, mask,
                      gal=(st,) + tuple(gal[1:]), backend="direct",
                      exp_mog=(z["amp"], z["var"]))


def test_exp_profile_direct_known_answers():
    """Unit sum, centred peak, and a round profile's symmetry."""
    from oracle import sparse_oracle as SO
    z = np.load(Path(__file__).parents[1] / "uniphot_b200" / "data" / "exp_mog.npz")
    assert z["amp"].size == 6 and abs(float(z["amp"].sum()) - 1.0) < 1e-6
    p = SO.exp_profile_direct(15, 15, np.log(2.0), 0.0, 0.0, z["amp"], z["var"])
    assert abs(p.sum() - 1.0) < 1e-12
    assert np.unravel_index(np.argmax(p), p.shape) == (7, 7)
    np.testing.assert_allclose(p, p.T, atol=1e-15)
    np.testing.assert_allclose(p, p[::-1, ::-1], atol=1e-15)
    k = np.zeros((5, 5))
    k[2, 2] = 1.0
    np.testing.assert_allclose(SO.convolve_same(p, k), p, atol=1e-15)
