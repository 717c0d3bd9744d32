"""Serving on the GPU: requests solved concurrently through the server give
the same results as each request solved alone (bitwise: every request owns
its buffers and the kernels are deterministic)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

FIELDS = ("pos_x", "pos_y", "logre", "ee1", "ee2", "sersic_n", "fluxes", "flux_err",
          "chi2", "n_steps", "converged", "stalled", "diverged", "source_idx")


def _requests():
    from uniphot_b200.synth import make_production_field
    shapes = [(96, 3, 20), (160, 5, 60), (128, 2, 40), (200, 4, 90), (112, 6, 30),
              (144, 3, 50)]
    out = []
    for i, (side, nb, ns) in enumerate(shapes):
        f = make_production_field(100 + i, side=side, n_bands=nb, n_src=ns,
                                  margin=side / 4)
        out.append(f.fit_kwargs("analytic"))
    return out


@pytest.mark.parametrize("precision", ["mixed", "plain"])
def test_results_alone_equal_results_in_the_mix(precision):
    from uniphot_b200.serve import Server, latency_summary
    from uniphot_b200.solver import island_fit
    reqs = [dict(kw, precision=precision) for kw in _requests()]
    alone = [island_fit(**kw) for kw in reqs]
    with Server(workers=3, hbm_budget_bytes=160e9, precision=precision) as srv:
        futs = [srv.submit(kw) for kw in reqs]
        mixed = [f.result(timeout=600) for f in futs]
    for a, m in zip(alone, mixed):
        for k in FIELDS:
            np.testing.assert_array_equal(getattr(a, k), getattr(m, k), err_msg=k)
    s = latency_summary(srv.stats)
    assert s["requests"] == len(reqs) and s["p99_ms"] > 0
    assert max(st.worker for st in srv.stats) >= 1   # more than one slot was used
