"""The field-stack build (island_stage.py:1728-1751) on the host: the
oracle's restatement against the reference's own make_bg_basis and
subtraction (golden ``stacks_small.npz``), bit for bit."""
import hashlib
from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).parent / "golden"
PAD = 7


def small_case(order: int):
    """A seeded 3-band 70 x 90 field, four tile cores (two of them sharing
    an edge region, one touching the border), per-tile per-band planar
    coefficients of the given order, normalisation about the field centre."""
    rng = np.random.default_rng(40 + order)
    nb, H, W = 3, 70, 90
    data = rng.normal(100.0, 10.0, (nb, H, W)).astype(np.float32)
    invvar = rng.uniform(0.5, 2.0, (nb, H, W)).astype(np.float32)
    tiles = np.array([[0, 0, 45, 35], [45, 0, 90, 35], [0, 35, 60, 70], [50, 30, 90, 70]],
                     np.int32)
    M = (1, 3, 6)[order]
    coefs = rng.normal(0.0, 5.0, (len(tiles), nb, M)).astype(np.float32)
    coefs[:, :, 0] += 100.0
    norm = (45.0, 45.0, 35.0, 35.0)
    return data, invvar, tiles, coefs, norm


def digest(order: int) -> str:
    h = hashlib.sha256()
    for a in small_case(order)[:4]:
        h.update(np.ascontiguousarray(a).tobytes())
    return h.hexdigest()


@pytest.mark.parametrize("order", [0, 1, 2])
def test_oracle_stack_build_matches_the_reference(order):
    from oracle.stacks_oracle import field_stacks
    z = np.load(GOLDEN / "stacks_small.npz")
    assert str(z[f"digest_order{order}"]) == digest(order)
    data, invvar, tiles, coefs, norm = small_case(order)
    dmb, iv = field_stacks(data, invvar, PAD, tiles, coefs, order, norm)
    np.testing.assert_array_equal(dmb, z[f"dmb_order{order}"])
    assert np.all(iv[:, :PAD] == 0) and np.all(iv[:, PAD:PAD + 70, PAD:PAD + 90] == invvar)


def test_scene_subtraction_waves_keep_source_order_per_pixel():
    """The star scene subtraction's schedule (host code of the library, no
    device): every wave's stamps are pairwise disjoint, and of two
    overlapping stamps the earlier source is in an earlier wave -- against
    an all-pairs restatement on clustered positions, stamps off the field's
    edges and coincident sources."""
    from uniphot_b200 import _lib
    rng = np.random.default_rng(3)
    T = 31
    cx, cy = rng.uniform(0, 400, 30), rng.uniform(0, 400, 30)
    x = np.concatenate([cx[k] + rng.normal(0, 12, 8) for k in range(30)] + [[-40.2, -40.2]])
    y = np.concatenate([cy[k] + rng.normal(0, 12, 8) for k in range(30)] + [[5.5, 5.5]])
    wave = _lib.scene_waves(x, y, T)
    ix = np.round(x).astype(int) - T // 2
    iy = np.round(y).astype(int) - T // 2
    ref = np.zeros(x.size, int)
    for i in range(x.size):
        for j in range(i):
            if abs(ix[i] - ix[j]) < T and abs(iy[i] - iy[j]) < T:
                ref[i] = max(ref[i], ref[j] + 1)
    np.testing.assert_array_equal(wave, ref)
    assert wave.max() >= 3 and wave[-1] == wave[-2] + 1
    with pytest.raises(ValueError):
        _lib.scene_waves([np.nan], [0.0], T)
