"""The field-stack build on the device (``uph_subtract_tile_backgrounds``,
``DeviceField.from_tiles``) against the reference's own subtraction (golden
``stacks_small.npz``, made with the reference's make_bg_basis): the border
and inverse variances exact, the data within two float32 ulps of the
background plane (the host sums the terms through a BLAS matrix-vector
product, the device in term order); and an island solve on the device-built
stacks against one on host-built stacks."""
from pathlib import Path

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).parent / "golden"


@pytest.mark.parametrize("order", [0, 1, 2])
def test_device_stack_build_matches_the_reference(order):
    from test_stacks_cpu import PAD, digest, small_case
    from uniphot_b200.solver import DeviceField
    z = np.load(GOLDEN / "stacks_small.npz")
    assert str(z[f"digest_order{order}"]) == digest(order)
    data, invvar, tiles, coefs, norm = small_case(order)
    fld = DeviceField.from_tiles(data, invvar, PAD, tiles, coefs, order, norm)
    d, w = fld.download()
    ref = z[f"dmb_order{order}"]
    nb, H, W = data.shape
    inner = np.zeros(ref.shape, bool)
    inner[:, PAD:PAD + H, PAD:PAD + W] = True
    assert np.all(d[~inner] == 0) and np.all(w[~inner] == 0)
    np.testing.assert_array_equal(w[:, PAD:PAD + H, PAD:PAD + W], invvar)
    bg = np.abs(data - ref[:, PAD:PAD + H, PAD:PAD + W])
    tol = 2 * np.spacing(np.maximum(bg, np.abs(data)).astype(np.float32))
    err = np.abs(d - ref)[:, PAD:PAD + H, PAD:PAD + W]
    assert np.all(err <= tol), f"max error {err.max():.3g}"
    print(f"order {order}: {np.mean(err == 0):.4f} of pixels bit-identical")


def test_device_stack_build_rejects_bad_tiles_and_bound_fields():
    from test_stacks_cpu import PAD, small_case
    from uniphot_b200 import _lib
    from uniphot_b200.solver import DeviceField
    data, invvar, tiles, coefs, norm = small_case(1)
    fld = DeviceField.from_unpadded(data, invvar, PAD)
    bad = tiles.copy()
    bad[0, 2] = 1000
    with pytest.raises(ValueError, match="outside"):
        fld.ctx.subtract_tile_backgrounds(bad, coefs, 1, norm)
    with pytest.raises(ValueError, match="scale"):
        fld.ctx.subtract_tile_backgrounds(tiles, coefs, 1, (0.0, 0.0, 0.0, 1.0))
    # a field held by a live job's chunks is not modified in place
    from uniphot_b200.synth import make_small_field
    f = make_small_field(0)
    kw = f.fit_kwargs("analytic")
    from uniphot_b200.solver import IslandFitJob, plan_field
    fp = plan_field(**kw)
    fld2 = DeviceField.from_unpadded(kw["data_minus_bg"], kw["invvar"], fp.PAD)
    job = IslandFitJob(**kw, field=fld2, plan=fp)
    nb = kw["data_minus_bg"].shape[0]
    with pytest.raises(_lib.UphError, match="live job"):
        fld2.ctx.subtract_tile_backgrounds(np.array([[0, 0, 4, 4]], np.int32),
                                           np.zeros((1, nb, 1), np.float32), 0,
                                           (0.0, 1.0, 0.0, 1.0))
    job.close()


def test_island_solve_on_device_built_stacks():
    """The small field's data as raw bands plus per-tile planes: the island
    solve on stacks built on the device equals the one on the host-built
    stacks (the oracle's restatement of the reference loop) where the two
    stacks agree bit for bit, and stays within the parity bar elsewhere."""
    from oracle.stacks_oracle import field_stacks
    from uniphot_b200.solver import DeviceField, island_fit, plan_field
    from uniphot_b200.synth import make_small_field
    f = make_small_field(0)
    kw = f.fit_kwargs("analytic")
    data_mb = np.asarray(kw["data_minus_bg"], np.float32)
    nb, H, W = data_mb.shape
    rng = np.random.default_rng(5)
    tiles = np.array([[0, 0, W // 2, H // 2], [W // 2, 0, W, H // 2],
                      [0, H // 2, W // 2, H], [W // 2, H // 2, W, H]], np.int32)
    coefs = rng.normal(0.0, 2.0, (4, nb, 3)).astype(np.float32)
    coefs[:, :, 0] += 50.0
    norm = (W / 2.0, W / 2.0, H / 2.0, H / 2.0)
    fp = plan_field(**kw)
    # raw = data_minus_bg + plane, rounded as the host would hold it
    dmb0, _ = field_stacks(np.zeros_like(data_mb), kw["invvar"], fp.PAD, tiles, coefs, 1, norm)
    plane = -dmb0[:, fp.PAD:fp.PAD + H, fp.PAD:fp.PAD + W]
    raw = (data_mb + plane).astype(np.float32)
    host_dmb, _ = field_stacks(raw, kw["invvar"], fp.PAD, tiles, coefs, 1, norm)
    host = island_fit(**dict(kw, data_minus_bg=host_dmb[:, fp.PAD:fp.PAD + H, fp.PAD:fp.PAD + W]))
    fld = DeviceField.from_tiles(raw, kw["invvar"], fp.PAD, tiles, coefs, 1, norm)
    d, _ = fld.download()
    dev = island_fit(**kw, field=fld, plan=fp)
    same = np.array_equal(d, host_dmb)
    o1, o2 = np.argsort(host.source_idx), np.argsort(dev.source_idx)
    if same:
        for k in ("fluxes", "pos_x", "pos_y", "n_steps", "converged", "stalled"):
            np.testing.assert_array_equal(getattr(host, k)[o1], getattr(dev, k)[o2], err_msg=k)
    else:
        np.testing.assert_array_equal(host.n_steps[o1], dev.n_steps[o2])
        np.testing.assert_allclose(dev.pos_x[o2], host.pos_x[o1], atol=1e-3)
        df = np.abs(dev.fluxes[o2].astype(np.float64) - host.fluxes[o1])
        assert np.all((df <= 1e-4 * np.abs(host.fluxes[o1])) | (df <= 0.01 * host.flux_err[o1]))


def test_star_scene_subtraction_matches_the_oracle():
    """The field-wide star scene subtraction on the device against the
    oracle's restatement of the reference loop (island_stage.py:2024-2118)
    on a field with an order-2 polynomial PSF, clustered (overlapping)
    stamps and stamps cut by the stack's border: within 1e-5 of the
    subtracted light (the stamps' float32 evaluation orders differ) plus
    four ulps, bitwise the same on a second run, and the border and the
    inverse variances untouched."""
    from oracle.stacks_oracle import scene_subtract_stars
    from uniphot_b200.solver import DeviceField
    from uniphot_b200.synth import make_production_field
    f = make_production_field(6, side=256, n_bands=3, n_src=60, margin=40)
    data = np.asarray(f.data_minus_bg, np.float32)
    invvar = np.asarray(f.invvar, np.float32)
    nb, H, W = data.shape
    PAD = 8
    star = np.asarray(f.source_type) == 0
    x = np.concatenate([np.asarray(f.pos_x, np.float64)[star], [-3.7, W + 2.2, 100.5]])
    y = np.concatenate([np.asarray(f.pos_y, np.float64)[star], [50.25, H - 1.4, 100.5]])
    flux = np.concatenate([np.asarray(f.s1_flux, np.float32)[star],
                           np.full((3, nb), 500.0, np.float32)])
    flux[1, 0] = 0.0                      # a source skipped in one band
    psfs = f.poly_psfs
    T = int(psfs[0].coefs.shape[0])
    ref = np.zeros((nb, H + 2 * PAD, W + 2 * PAD), np.float32)
    ref[:, PAD:PAD + H, PAD:PAD + W] = data
    before = ref.copy()
    scene_subtract_stars(ref, x, y, flux, psfs, T, PAD)
    outs = []
    for _ in range(2):
        fld = DeviceField.from_unpadded(data, invvar, PAD)
        fld.subtract_star_scene(psfs, x, y, flux, native=T)
        outs.append(fld.download())
    d, w = outs[0]
    np.testing.assert_array_equal(d, outs[1][0])
    np.testing.assert_array_equal(w[:, PAD:PAD + H, PAD:PAD + W], invvar)
    sub = np.abs(before - ref)
    assert sub.max() > 0
    tol = 1e-5 * sub + 4 * np.spacing(np.maximum(np.abs(ref), np.abs(before)))
    err = np.abs(d - ref)
    assert np.all(err <= tol), f"max error {err.max():.3g} where {sub[err > tol].max():.3g} was removed"
