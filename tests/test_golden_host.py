"""Host logic pinned against fixtures produced by the reference's own numpy
modules (tests/golden/make_golden.py): island membership, bboxes, buckets,
class planning and per-class host arrays must be identical."""
from pathlib import Path

import numpy as np
import pytest

from uniphot_b200 import islands as I
from uniphot_b200 import plan as P

GOLD = Path(__file__).resolve().parent / "golden"
FIXTURES = ["plan_small_s0.npz", "plan_small_s1.npz", "plan_field_s3.npz"]


def _load(name):
    return dict(np.load(GOLD / name, allow_pickle=False))


def _islands(z):
    native = int(z["native"])
    if "psf_stamp" in z:
        pr, pp = I.psf_radial_profile(z["psf_stamp"])
        np.testing.assert_allclose(pr, z["psf_r"])
        np.testing.assert_allclose(pp, z["psf_p"])
        radius = I.flux_aware_radii(z["source_type"], z["logre"], z["sersic_n"],
                                    np.median(z["s1_flux"], axis=1),
                                    float(z["sigma_sky"]), 0.5, pr, pp, native / 2.0)
        np.testing.assert_allclose(radius, z["radius"], rtol=0, atol=0)
    else:
        radius = np.full(z["pos_x"].size, 4.0)
    iset = I.build_islands(z["pos_x"], z["pos_y"], z["source_type"], z["logre"],
                           z["sersic_n"], native / 2.0, radius=radius)
    bk = I.bucket_islands(iset)
    return iset, bk


@pytest.mark.parametrize("name", FIXTURES)
def test_membership_identical(name):
    z = _load(name)
    iset, bk = _islands(z)
    np.testing.assert_array_equal(iset.labels, z["labels"])
    np.testing.assert_array_equal(iset.bbox, z["bbox"])
    np.testing.assert_array_equal(iset.n_src, z["n_src"])
    np.testing.assert_array_equal(bk.giant_ids, z["giant_ids"])


@pytest.mark.parametrize("name", FIXTURES)
def test_class_plan_and_host_arrays_identical(name):
    z = _load(name)
    iset, bk = _islands(z)
    native = int(z["native"])
    free_n = P.free_n_gate(z["source_type"], z["s1_flux"], z["s1_flux_var"], True, 30.0)
    np.testing.assert_array_equal(free_n, z["free_n"])
    plans, capped = P.plan_island_classes(iset, bk, z["source_type"], z["logre"],
                                          z["sersic_n"], native, joint_nsrc_cap=32)
    np.testing.assert_array_equal(np.asarray(capped, np.int64), z["capped"])
    keys = np.asarray([[p.bbox_class, p.nsrc_class, 0 if p.kind == "star" else 1,
                        p.tier, p.n_gal_class] for p in plans], np.int64).reshape(-1, 5)
    np.testing.assert_array_equal(keys, z["class_keys"])
    for ci, p in enumerate(plans):
        host = P.class_host_arrays(
            p, pos_x=z["pos_x"], pos_y=z["pos_y"], source_type=z["source_type"],
            logre=z["logre"], ee1=z["ee1"], ee2=z["ee2"], sersic_n=z["sersic_n"],
            free_n_all=free_n, pos_max_shift_pix=5.0, pad=400)
        np.testing.assert_array_equal(p.isl_ids, z[f"c{ci}_isl_ids"])
        for k in ("ox", "oy", "x0b", "y0b", "keep", "p0", "lower", "upper",
                  "prior_inv_sigma", "fn_flag", "mmask", "gsel", "gvalid"):
            np.testing.assert_array_equal(host[k], z[f"c{ci}_{k}"], err_msg=f"{ci} {k}")


def test_bucket_giants_and_empty():
    iset = I.build_islands(np.zeros(0), np.zeros(0), None, None, None, 10.0)
    assert iset.n_islands == 0
    # one island far larger than the largest class becomes a giant
    x = np.arange(20) * 20.0
    iset = I.build_islands(x, np.zeros(20), None, None, None, 12.0)
    assert iset.n_islands == 1
    bk = I.bucket_islands(iset)
    assert list(bk.giant_ids) == [0] and not bk.buckets


def test_build_islands_rejects_nonfinite():
    with pytest.raises(ValueError):
        I.build_islands(np.array([0.0, np.nan]), np.zeros(2), None, None, None, 5.0)


def test_ladder_width():
    assert P.ladder_width(5, 4096) == 8
    assert P.ladder_width(1, 4096) == 1
    assert P.ladder_width(3000, 1024) == 1024


def test_giant_rows_keep_seed_geometry():
    iset = I.build_islands(np.array([0.0, 3.0, 100.0]), np.zeros(3), None, None,
                           None, 5.0)
    rows = P.giant_seed_rows([0], iset, pos_x=np.array([0.0, 3.0, 100.0]),
                             pos_y=np.zeros(3), logre=np.zeros(3), ee1=np.zeros(3),
                             ee2=np.zeros(3), sersic_n=np.ones(3), n_bands=2)
    r = rows[0]
    assert list(r["src"]) == [0, 1]
    assert r["island_giant"].all() and r["converged"].all()
    assert np.isnan(r["fluxes"]).all() and r["fluxes"].shape == (2, 2)
    np.testing.assert_array_equal(r["pos_x"], [0.0, 3.0])
