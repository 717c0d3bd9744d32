"""Heavy blends of the headline workload on the GPU against the oracle.

Every class of 8, 16 and 32 members of the reduced production field
(512^2, 3 bands, 300 sources, analytic render: 4-Gaussian order-2 PSF,
EXP/DEV/SERSIC members, tiers 31/63/127) solved by the plain CUDA form and
compared with the oracle at reference precision, committed by
``tests/golden/make_oracle_blends.py``.  Bar on every island: identical LM
iteration counts, converged / stalled flags and good-pixel counts, chi2
within 1e-5 relative.  On islands that converge, also fluxes within 1e-4
relative or 0.01 sigma and positions within 1e-3 px -- unless the float32
oracle itself misses that flux bar against the float64 oracle on the
island (its solution is not determined to the bar in float32): there the
GPU's fluxes must be no further from the float32 oracle than the float32
oracle is from float64, and positions within 1e-2 px.  Stalled islands
(four rejected steps in a row: the LM ends on a chi2 plateau) are held to
the chi2 alone: along the plateau the faint members' fluxes and positions
are not determined to float32 rounding.  Measured on the B200: every island
has the oracle's iteration count and flags and chi2 within 2e-6; the
converged islands are within 7e-4 sigma and 1.2e-4 px, except the 32-member
island where the float32 oracle is 0.059 sigma from float64 (GPU: 0.016
sigma, 6.3e-3 px); stalled islands end up to 0.08 sigma and 2.3e-3 px away.

The mixed form (tensor-core Gram for every island: ``tc_min_rows=0`` and no
conditioning routing) is held to the all-float64 oracle: its fraction of
fluxes within 1e-4 relative or 0.01 sigma of float64 must reach the plain
form's on the same islands.
"""
from pathlib import Path

import numpy as np
import pytest

from _common import compare, run_gpu

pytestmark = pytest.mark.gpu

GOLD = Path(__file__).resolve().parent / "golden" / "oracle_blends.npz"


@pytest.fixture(scope="module")
def blends():
    import sys
    sys.path.insert(0, str(GOLD.parent))
    from make_golden_solver import field_digest
    from make_oracle_blends import blend_classes, blend_field
    g = np.load(GOLD)
    f = blend_field()
    assert str(g["digest"]) == field_digest(f), "field generator drifted"
    plans, hosts, PAD, ds, ws, psfs = blend_classes(f)
    assert [",".join(map(str, p.key)) for p in plans] == g["classes"].tolist()
    ref = [{k.split("/")[2]: g[k] for k in g.files if k.startswith(f"{ci}/ref/")}
           for ci in range(len(plans))]
    f64 = [{k.split("/")[2]: g[k] for k in g.files if k.startswith(f"{ci}/f64/")}
           for ci in range(len(plans))]
    return f, plans, hosts, PAD, ds, ws, psfs, ref, f64


def test_blend_classes_cover_8_16_32(blends):
    plans = blends[1]
    assert {8, 16, 32} <= {p.nsrc_class for p in plans}


def test_plain_form_matches_oracle_on_heavy_blends(blends):
    f, plans, hosts, PAD, ds, ws, psfs, ref, f64 = blends
    g, _ = run_gpu(plans, hosts, PAD, ds, ws, psfs, "analytic", native=f.native)
    bad = []
    for p, h, gg, oo, o64 in zip(plans, hosts, g, ref, f64):
        r = compare(gg, oo, h["mmask"])
        gap = np.abs(oo["p"][..., :2] - o64["p"][..., :2]).max()
        dchi = np.abs(gg["chi2"] / oo["chi2"] - 1).max()
        msg = (f"{p.key}: max rel flux {r['max_rel']:.2e}, max dpos {r['max_dpos']:.2e} "
               f"(float32-float64 oracle gap {gap:.2e}), chi2 rel {dchi:.2e}, "
               f"gpu nst {gg['nst'].tolist()} oracle nst {oo['nst'].tolist()}, "
               f"stalled {oo['stall'].tolist()}")
        print(msg)
        for i in range(len(oo["nst"])):
            m = h["mmask"][i]
            df = np.abs(gg["fluxes"][i][:, m] - oo["fluxes"][i][:, m])
            sig = np.maximum(oo["ferr"][i][:, m], 1e-30)
            gap_f = np.abs(oo["fluxes"][i][:, m] - o64["fluxes"][i][:, m]) / sig
            print(f"   island {i}: nst {oo['nst'][i]} stalled {oo['stall'][i]} "
                  f"flux dev max {np.max(df / sig):.3g} sigma (float32-float64 oracle "
                  f"{np.max(gap_f):.3g} sigma), dpos "
                  f"{np.abs(gg['p'][i][m, :2] - oo['p'][i][m, :2]).max():.2e}")
        ok = (r["same_nst"].all() and r["same_flags"].all() and dchi <= 1e-5
              and np.array_equal(gg["n_good"], oo["n_good"]))
        for i in np.nonzero(~oo["stall"])[0]:
            m = h["mmask"][i]
            fo, fg, f6 = oo["fluxes"][i][:, m], gg["fluxes"][i][:, m], o64["fluxes"][i][:, m]
            sig = np.maximum(oo["ferr"][i][:, m], 1e-30)
            d32, d64 = np.abs(fg - fo), np.abs(fo - f6)
            oracle_ok = np.all((d64 <= 1e-4 * np.abs(f6)) | (d64 <= 0.01 * sig))
            dpos = np.abs(gg["p"][i][m, :2] - oo["p"][i][m, :2]).max()
            if oracle_ok:
                ok = ok and bool(r["flux_ok"][i]) and bool(r["pos_ok"][i])
            else:
                ok = ok and np.max(d32 / sig) <= np.max(d64 / sig) and dpos <= 1e-2
        if not ok:
            bad.append(msg)
    assert not bad, "\n".join(bad)


def _pass_frac(res, f64, hosts):
    ok = []
    for r, o, h in zip(res, f64, hosts):
        m = np.broadcast_to(h["mmask"][:, None, :], r["fluxes"].shape)
        d = np.abs(r["fluxes"] - o["fluxes"])
        good = (d <= 1e-4 * np.abs(o["fluxes"])) | (d <= 0.01 * o["ferr"])
        ok.append(good[m])
    return float(np.mean(np.concatenate(ok)))


def test_mixed_form_vs_float64_on_heavy_blends(blends):
    f, plans, hosts, PAD, ds, ws, psfs, _, f64 = blends
    plain, fld = run_gpu(plans, hosts, PAD, ds, ws, psfs, "analytic", native=f.native)
    mixed, _ = run_gpu(plans, hosts, PAD, ds, ws, psfs, "analytic", native=f.native,
                       field=fld, precision="mixed", tc_min_rows=0, tc_cond_max=1e30)
    fp, fm = _pass_frac(plain, f64, hosts), _pass_frac(mixed, f64, hosts)
    print(f"fluxes within 1e-4 rel or 0.01 sigma of float64: plain {fp:.4f} mixed {fm:.4f}")
    assert fm >= fp - 1e-12, (fp, fm)
