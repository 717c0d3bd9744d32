"""Width halving of run_class_chunk_resilient on device-memory failures
(the reference's run_class_chunk_resilient, island_solver.py:3134-3230).

A stand-in for run_class_chunk raises the library's out-of-memory error
(``RESOURCE_EXHAUSTED: ...``, the text _lib gives UPH_ERR_OOM) whenever a
chunk holds more than ``cap`` islands and otherwise returns per-row arrays
derived from the row indices, so the test sees exactly how the chunk was
split, what carry state each part received and how the parts were merged.
No GPU is touched.
"""
import numpy as np
import pytest

from uniphot_b200 import _lib, solver


def _stand_in(cap, calls, fail_text="RESOURCE_EXHAUSTED: cudaMalloc of chunk buffers"):
    def run(kernels, psf_tree, host, rows, width, max_steps, dstack_dev, wstack_dev,
            pad, init_state=None, **kw):
        rows = np.asarray(rows)
        calls.append((rows.copy(), int(width),
                      None if init_state is None else {k: v.copy() for k, v in
                                                       init_state.items()}))
        if rows.size > cap:
            raise _lib.UphError(fail_text)
        lam0 = (np.zeros(rows.size, np.float32) if init_state is None
                else init_state["lam"].astype(np.float32))
        return dict(p=np.stack([rows, rows + 0.5], axis=1).astype(np.float32)[:, None, :],
                    fluxes=(rows[:, None, None] * 10.0 + np.arange(3)[None, :, None]
                            ).astype(np.float32),
                    lam=lam0 + rows.astype(np.float32),
                    nst=(rows % 7).astype(np.int32),
                    conv=(rows % 2 == 0),
                    wall_s=0.25, steps_run=int(rows.size))
    return run


def test_halves_until_it_fits_and_merges_in_row_order(monkeypatch):
    calls = []
    monkeypatch.setattr(solver, "run_class_chunk", _stand_in(3, calls))
    rows = np.arange(100, 110)
    init = {"lam": np.linspace(1.0, 2.0, rows.size).astype(np.float32)}
    logs = []
    out = solver.run_class_chunk_resilient(None, None, None, rows, 10, 30, None, None, 8,
                                           init_state=init, log_fn=logs.append)
    # 10 -> halves of 5 (still too big) -> parts of 2 (5 // 2) -> fits
    assert out["halved"] is True
    assert out["widths_ran"] == [2]
    ran = [c for c in calls if c[0].size <= 3]
    np.testing.assert_array_equal(np.concatenate([c[0] for c in ran]), rows)
    # every part got the slice of the carry state matching its rows
    np.testing.assert_array_equal(np.concatenate([c[2]["lam"] for c in ran]), init["lam"])
    np.testing.assert_array_equal(out["p"][:, 0, 0], rows.astype(np.float32))
    np.testing.assert_array_equal(out["lam"], init["lam"] + rows.astype(np.float32))
    np.testing.assert_array_equal(out["nst"], rows % 7)
    np.testing.assert_array_equal(out["conv"], rows % 2 == 0)
    assert out["fluxes"].shape == (rows.size, 3, 1)
    assert out["wall_s"] == pytest.approx(0.25 * len(ran))
    assert out["steps_run"] == max(c[0].size for c in ran)
    assert logs and all("retrying" in m for m in logs)


def test_no_halving_when_it_fits(monkeypatch):
    calls = []
    monkeypatch.setattr(solver, "run_class_chunk", _stand_in(64, calls))
    rows = np.arange(5)
    out = solver.run_class_chunk_resilient(None, None, None, rows, 8, 30, None, None, 8)
    assert out["halved"] is False and out["widths_ran"] == [8]
    assert len(calls) == 1


def test_other_errors_and_single_islands_are_not_retried(monkeypatch):
    calls = []
    monkeypatch.setattr(solver, "run_class_chunk",
                        _stand_in(0, calls, fail_text="uph_run_chunk: status 1: bad tier"))
    with pytest.raises(_lib.UphError, match="bad tier"):
        solver.run_class_chunk_resilient(None, None, None, np.arange(4), 4, 30, None, None, 8)
    assert len(calls) == 1
    calls.clear()
    monkeypatch.setattr(solver, "run_class_chunk", _stand_in(0, calls))
    with pytest.raises(_lib.UphError, match="RESOURCE_EXHAUSTED"):
        solver.run_class_chunk_resilient(None, None, None, np.arange(1), 1, 30, None, None, 8,
                                         log_fn=lambda m: None)
    assert len(calls) == 1
