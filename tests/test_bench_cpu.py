"""The bench's measurement helpers on the host: the class-stratified sample
behind the metric's tolerance, the tolerance estimator (per-flux pass
fraction and the class-weighted fraction of islands whose every flux
passes), and the t_lb roofline model."""
import numpy as np
import pytest

import bench


class _Plan:
    def __init__(self, n, nsrc):
        self.n_islands = n
        self.nsrc_class = nsrc


def _classes(sizes):
    return [(_Plan(n, 1 << (i % 6)), {"mmask": np.ones((n, 2), bool)})
            for i, n in enumerate(sizes)]


def test_stratified_sample_covers_every_class_and_is_seeded():
    sizes = [500, 120, 40, 3, 1, 1, 60]
    classes = _classes(sizes)
    a = bench._stratified_rows(classes, 100, 2)
    b = bench._stratified_rows(classes, 100, 2)
    assert a == b
    assert {ci for ci, _ in a} == set(range(len(sizes)))
    assert 95 <= len(a) <= 110
    for ci, r in a:
        assert 0 <= r < sizes[ci]
    assert len(set(a)) == len(a)
    # proportional where a class is large enough
    n0 = sum(1 for ci, _ in a if ci == 0)
    assert abs(n0 - 100 * 500 / sum(sizes)) <= 1


def test_flux_quality_counts_passes_and_weights_islands_by_class():
    classes = _classes([4, 2])
    fl = {0: np.ones((4, 3, 2)), 1: np.ones((2, 3, 2))}

    def get(ci):
        return {"fluxes": fl[ci]}
    ref = []
    # class 0: island 0 exact, island 1 one flux off by 1e-3 relative
    for r in range(2):
        f = np.ones((3, 2))
        if r == 1:
            f[0, 0] = 1.0 / (1 + 1e-3)
        ref.append(((0, r), {"fluxes": f, "ferr": np.full((3, 2), 1e-6)}))
    # class 1: island 0 one flux 3e-4 relative (0.003 sigma) off: it fails
    # the relative prong and passes through the sigma prong
    f = np.ones((3, 2))
    f[1, 1] = 1.0 - 3e-4
    ref.append(((1, 0), {"fluxes": f, "ferr": np.full((3, 2), 0.1)}))
    q = bench._flux_quality(get, classes, ref, weights={0: 2.0, 1: 2.0})
    assert q["n_fluxes"] == 18
    assert q["frac_within_1e-4_rel_or_0.01sigma"] == pytest.approx(17 / 18)
    assert q["islands_all_fluxes_pass_sample"] == pytest.approx(2 / 3)
    assert q["islands_all_fluxes_pass_weighted"] == pytest.approx(2 / 3)
    q2 = bench._flux_quality(get, classes, ref, weights={0: 1.0, 1: 8.0})
    # the passing class-1 island now stands for more of the field
    assert q2["islands_all_fluxes_pass_weighted"] == pytest.approx((1 + 8) / (1 + 1 + 8))


def test_roofline_model_takes_the_binding_peak_per_kind():
    peaks = {"hbm_gbs": 1000.0, "bf16_tflops": 300.0, "fp32_tflops": 10.0,
             "fp64_tflops": 5.0, "exp2_tera_per_s": 2.0}
    ktab = {
        "render": {"alg_bytes": 1e9, "alg_flops": 1e11, "alg_exps": 1e10, "ms": 50.0},
        "gram_tc": {"alg_bytes": 4e9, "alg_flops": 1e12, "alg_exps": 0, "ms": 20.0},
        "trial_chi2": {"alg_bytes": 2e9, "alg_flops": 0.0, "ms": 10.0},
    }
    m = bench._roofline_model(ktab, 100.0, peaks)
    k = m["kinds"]
    # render: hbm 1 ms, fp32 10 ms, sfu 5 ms -> fp32
    assert k["render"]["bound"] == "fp32" and k["render"]["t_lb_ms"] == pytest.approx(10.0)
    # tensor-core Gram at a third of BF16: 1e12 / 1e14 = 10 ms vs hbm 4 ms
    assert k["gram_tc"]["bound"] == "tensor" and k["gram_tc"]["t_lb_ms"] == pytest.approx(10.0)
    assert k["trial_chi2"]["bound"] == "hbm" and k["trial_chi2"]["t_lb_ms"] == pytest.approx(2.0)
    assert m["sum_t_lb_ms"] == pytest.approx(22.0)
    assert m["frac"] == pytest.approx(0.22)
    assert k["render"]["frac_of_serialised"] == pytest.approx(0.2)
