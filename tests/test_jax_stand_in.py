"""The numpy stand-in for JAX that the reference-solver fixtures are made
with (``tests/golden/jax_stand_in.py``): the JAX semantics the reference's
code relies on, checked against plain numpy.  The module is only imported
here, never installed as ``jax``, so no other test sees it."""

import sys
from pathlib import Path

import numpy as np
import pytest

sys.path.insert(0, str(Path(__file__).parent / "golden"))
import jax_stand_in as J  # noqa: E402

jnp, lax = J.jnp, J.lax


def test_float32_is_widened_and_at_updates_are_functional():
    a = jnp.zeros(4, dtype=jnp.float32)
    assert a.dtype == np.float64 and jnp.float32(1.5).dtype == np.float64
    b = a.at[1].set(2.0).at[jnp.asarray([1, 3])].add(1.0)
    np.testing.assert_array_equal(a, 0.0)                 # a unchanged
    np.testing.assert_array_equal(b, [0.0, 3.0, 0.0, 1.0])
    c = b.at[jnp.asarray([1, 1])].add(1.0)                # repeated indices accumulate
    assert c[1] == 5.0
    assert jnp.asarray(np.ones(2, np.float32)).dtype == np.float64
    assert jnp.fft.rfft2(np.ones((4, 4), np.float32)).dtype == np.complex128


def test_vmap_with_pytree_axes_and_outputs():
    def f(x, d, s):
        return {"sum": x + d["a"] * s, "prod": x * d["b"]}, x.sum()
    x = np.arange(6.0).reshape(3, 2)
    d = {"a": np.array([1.0, 2.0, 3.0]), "b": np.array([5.0, 7.0])}
    out, tot = J.vmap(f, in_axes=(0, {"a": 0, "b": None}, None))(x, d, 10.0)
    np.testing.assert_allclose(out["sum"], x + 10.0 * d["a"][:, None])
    np.testing.assert_allclose(out["prod"], x * d["b"][None])
    np.testing.assert_allclose(tot, x.sum(axis=1))


def test_scan_map_and_loops():
    carry, ys = lax.scan(lambda c, x: (c + x, c * x), 0.0, np.arange(1.0, 5.0))
    assert carry == 10.0
    np.testing.assert_allclose(ys, [0.0, 2.0, 9.0, 24.0])
    c2, none = lax.scan(lambda c, _: (c * 2, None), 1.0, None, length=5)
    assert c2 == 32.0 and none is None
    np.testing.assert_allclose(lax.map(lambda v: v ** 2, np.arange(3.0)), [0.0, 1.0, 4.0])
    assert lax.fori_loop(0, 4, lambda i, v: v + i, 0) == 6
    assert lax.while_loop(lambda v: v < 10, lambda v: v * 3, 1) == 27


def test_batched_solve_and_dynamic_slice_clamping():
    rng = np.random.default_rng(0)
    A = rng.normal(size=(5, 3, 3)) + 3 * np.eye(3)
    b = rng.normal(size=(5, 3))
    x = jnp.linalg.solve(A, b)                # (..., n) right-hand side: vectors
    np.testing.assert_allclose(np.einsum("kij,kj->ki", A, x), b, atol=1e-12)
    img = np.arange(25.0).reshape(5, 5)
    # start indices are clamped so that the slice stays inside the array
    np.testing.assert_array_equal(lax.dynamic_slice(img, (4, -2), (2, 3)), img[3:5, 0:3])


@pytest.mark.parametrize("scale", [1.0, 300.0])
def test_linearize_matches_the_analytic_derivative(scale):
    # samples around the centre; at scale 300 the step is relative to 300
    xs = scale + np.arange(7.0) - 3.0

    def f(p):
        return jnp.exp(-0.5 * ((xs - p[0]) / p[1]) ** 2)
    p0 = np.array([scale + 0.3, 1.7])
    y0, lin = J.linearize(f, p0)
    t = np.array([0.4, -1.1])
    g = np.exp(-0.5 * ((xs - p0[0]) / p0[1]) ** 2)
    dg = g * ((xs - p0[0]) / p0[1] ** 2 * t[0] + (xs - p0[0]) ** 2 / p0[1] ** 3 * t[1])
    np.testing.assert_allclose(y0, g)
    assert np.abs(dg).max() > 0.1
    np.testing.assert_allclose(lin(t), dg, atol=1e-6 * np.abs(dg).max())
