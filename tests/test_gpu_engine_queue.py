"""The job-wide work-queue engine against the per-chunk engine.

The engines run the same per-island computations (the queue kernels call
the per-chunk kernels' bodies for each unit of work; only the CTA that
processes a unit, and when, differs), so every output of a solve must be
bitwise identical: parameters, fluxes, errors, chi2, iteration counts and
flags, on every island of every class, for the plain and mixed forms, the
two render modes, the background and step variants, with the post-loop
passes, and for a job of many chunks of different classes solved at once.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KEYS = ("p", "fluxes", "ferr", "chi2", "nst", "conv", "stall", "diverged", "n_good", "lam")


def _same(a, b, label):
    for k in KEYS:
        np.testing.assert_array_equal(a[k], b[k], err_msg=f"{label}: {k}")


def _job(f, mode, engine, **kw):
    from uniphot_b200.solver import IslandFitJob
    args = dict(f.fit_kwargs(mode), **kw)
    job = IslandFitJob(**args, engine=engine)
    job.solve()
    out = []
    for plan, host, ids in job.classes:
        for i in ids:
            out.append(job.job.read(i))
    launches = job.field.ctx.last_launch_count()
    job.close()
    return out, launches


@pytest.mark.parametrize("mode,kw", [
    ("analytic", dict(precision="plain")),
    ("analytic", dict(precision="mixed")),
    ("reference", dict(precision="plain")),
    ("analytic", dict(precision="plain", step_mode="trust_region")),
    ("analytic", dict(precision="plain", convergence="dlnp")),
    ("analytic", dict(precision="mixed", bg_mode="joint")),
    ("analytic", dict(precision="plain", compute_param_errors=True,
                      compute_source_metrics=True)),
])
def test_queue_engine_equals_chunk_engine_small_field(mode, kw):
    from uniphot_b200.synth import make_small_field
    f = make_small_field(0)
    a, la = _job(f, mode, "chunks", **kw)
    for engine in ("queue", "queue_per_cta"):
        b, lb = _job(f, mode, engine, **kw)
        assert len(a) == len(b) > 1
        for i, (x, y) in enumerate(zip(a, b)):
            _same(x, y, f"{engine} {mode} {kw} chunk {i}")


@pytest.mark.parametrize("precision", ["plain", "mixed"])
def test_queue_engine_equals_chunk_engine_production_field(precision):
    """Every class of the reduced production field (300 sources, tiers
    31/63/127, blends up to 32 members) solved as one job."""
    from uniphot_b200.synth import make_production_field
    f = make_production_field(3, side=512, n_bands=3, n_src=300)
    a, la = _job(f, "analytic", "chunks", precision=precision)
    for engine in ("queue", "queue_per_cta"):
        b, lb = _job(f, "analytic", engine, precision=precision)
        assert len(a) == len(b) > 10
        for i, (x, y) in enumerate(zip(a, b)):
            _same(x, y, f"{engine} {precision} chunk {i}")
        print(f"launches: chunks engine {la}, {engine} engine {lb}")
        assert lb < la
