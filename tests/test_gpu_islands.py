"""Island decomposition on the GPU (uph_island_roots) against the host
port, which the golden fixtures pin to the reference's build_islands
(islands.py:361-560): identical labels, members and boxes."""
import numpy as np
import pytest

from uniphot_b200.islands import build_islands

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ctx():
    from uniphot_b200 import _lib
    return _lib.Context(0)


def _same(a, b):
    assert a.n_islands == b.n_islands
    np.testing.assert_array_equal(a.labels, b.labels)
    np.testing.assert_array_equal(a.bbox, b.bbox)
    np.testing.assert_array_equal(a.n_src, b.n_src)
    for m1, m2 in zip(a.members, b.members):
        np.testing.assert_array_equal(m1, m2)


@pytest.mark.parametrize("seed,n", [(0, 300), (1, 5000), (2, 100_000)])
def test_device_islands_match_the_host(ctx, seed, n):
    rng = np.random.default_rng(seed)
    side = 2048.0 * np.sqrt(n / 5000.0)
    # clustered positions and a spread of radii (stars and galaxies)
    cen = rng.uniform(0, side, (max(n // 20, 1), 2))
    pick = rng.integers(0, cen.shape[0], n)
    xy = cen[pick] + rng.normal(0, 25.0, (n, 2))
    r = np.where(rng.uniform(size=n) < 0.8, rng.uniform(4, 15, n), rng.uniform(10, 60, n))
    fs = rng.uniform(size=n) < 0.01
    host = build_islands(xy[:, 0], xy[:, 1], None, None, None, 15.0, radius=r,
                         forced_singleton=fs)
    dev = build_islands(xy[:, 0], xy[:, 1], None, None, None, 15.0, radius=r,
                        forced_singleton=fs, context=ctx)
    _same(host, dev)
    assert host.n_islands < n        # some coupling happened


def test_device_islands_on_the_synthetic_fields(ctx):
    from uniphot_b200.synth import make_production_field, make_small_field
    for f in (make_small_field(0), make_production_field(3, side=512, n_bands=3, n_src=300)):
        s = f.island_set
        dev = build_islands(f.pos_x, f.pos_y, f.source_type, f.logre, f.sersic_n, s.r_psf,
                            radius=s.radius, context=ctx)
        _same(s, dev)


def test_union_find_gives_up_with_a_timeout_status_and_the_context_recovers(ctx):
    """With the retry limit at 0 every coupled pair that is not yet linked
    runs out at once: the call reports UPH_ERR_TIMEOUT (no device fault,
    no hang); after the default limit is restored the same context labels
    the field correctly."""
    from uniphot_b200 import _lib
    rng = np.random.default_rng(5)
    n = 2000
    xy = rng.uniform(0, 400.0, (n, 2))
    r = np.full(n, 6.0)
    host = build_islands(xy[:, 0], xy[:, 1], None, None, None, 15.0, radius=r)
    assert host.n_islands < n
    ctx.set_island_retry_limit(0)
    try:
        with pytest.raises(_lib.UphError, match="status 4.*retries exhausted"):
            ctx.island_roots(xy[:, 0], xy[:, 1], r)
    finally:
        ctx.set_island_retry_limit(_lib.ISLAND_TRIES_DEFAULT)
    dev = build_islands(xy[:, 0], xy[:, 1], None, None, None, 15.0, radius=r, context=ctx)
    _same(host, dev)
