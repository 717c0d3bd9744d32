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


@pytest.mark.parametrize("precision,engine", [("mixed", "queue"), ("plain", "queue"),
                                              ("mixed", "chunks")])
def test_packed_results_equal_results_alone(precision, engine):
    """Requests packed into one job (every request's chunks bound to its own
    field and PSF, solved together) give each request's result alone."""
    from uniphot_b200.serve import PackedServer
    from uniphot_b200.solver import island_fit
    reqs = [dict(kw, precision=precision) for kw in _requests()]
    alone = [island_fit(**kw) for kw in reqs]
    with PackedServer(planners=2, engines=1, hbm_budget_bytes=160e9, precision=precision,
                      engine=engine) as srv:
        # submitted at once: the first pack starts with the first planned
        # requests and the rest are admitted while it is on the device
        futs = [srv.submit(kw) for kw in reqs]
        packed = [f.result(timeout=600) for f in futs]
    for a, m in zip(alone, packed):
        for k in FIELDS:
            np.testing.assert_array_equal(getattr(a, k), getattr(m, k), err_msg=k)
    assert sum(srv.packs) == len(reqs)
    assert max(srv.packs) > 1


def test_one_job_holds_chunks_of_two_fields():
    """Two fields uploaded one after the other to one context, their chunks
    in one job: each field's result equals its own job's, and the first
    DeviceField is reported as superseded for new chunks."""
    from uniphot_b200 import _lib
    from uniphot_b200.solver import DeviceField, IslandFitJob, plan_field
    from uniphot_b200.synth import make_production_field
    kws = []
    for i, (side, nb, ns) in enumerate([(128, 3, 40), (160, 3, 60)]):
        f = make_production_field(200 + i, side=side, n_bands=nb, n_src=ns,
                                  margin=side / 4)
        kws.append(dict(f.fit_kwargs("analytic"), precision="mixed"))
    alone = []
    for kw in kws:
        j = IslandFitJob(**kw)
        j.solve()
        alone.append(j.result())
        j.close()
    ctx = _lib.Context(0)
    job = _lib.Job(ctx)
    fits, fields = [], []
    for kw in kws:
        fp = plan_field(**kw)
        fld = DeviceField.from_unpadded(kw["data_minus_bg"], kw["invvar"], fp.PAD, context=ctx)
        fields.append(fld)
        fits.append(IslandFitJob(**kw, field=fld, plan=fp, job=job))
    job.solve(fits[0].max_steps)
    for a, fj in zip(alone, fits):
        m = fj.result()
        for k in FIELDS:
            np.testing.assert_array_equal(getattr(a, k), getattr(m, k), err_msg=k)
    with pytest.raises(ValueError, match="superseded"):
        fields[0].check_current()
    job.close()
    ctx.close()
