"""The allocation-free final-flux entry point against the allocating one.

Callers that cannot allocate device memory (a host inside a framework that
owns the device pool, or a serving process with a fixed budget) own every
buffer and call uph_fluxes_noalloc; its intermediates live in a fixed device
array inside the library.  Its results must reproduce uph_run_chunk
(max_steps=0) -- the fluxes, sqrt(diag inv A64) and chi2 at fixed
parameters -- within 1e-6 relative: on two calls in a row on two island
classes, on a call issued on a non-default stream, on a later call with
fewer islands than the one before (the array keeps the earlier call's
contents), and with device free memory unchanged across a warm call.
Islands that fail the entry point's checks (a galaxy member, a window
outside the field) come back NaN and leave the other islands' results
unchanged.  This file is collected last so that a failure here never hides
another test.
"""
import numpy as np
import pytest

from _common import field_classes

pytestmark = pytest.mark.gpu


def _setup():
    import torch
    from uniphot_b200 import solver
    from uniphot_b200.synth import make_small_field
    f = make_small_field(0)
    plans, hosts, PAD, ds, ws, psfs = field_classes(f, "reference", ("star",))
    assert len(plans) >= 2
    field = solver.DeviceField(ds, ws, PAD)
    cuda = torch.device("cuda", 0)
    d_data = torch.as_tensor(ds, device=cuda)
    d_w = torch.as_tensor(ws, device=cuda)
    return f, plans, hosts, PAD, ds, psfs, field, d_data, d_w


def _reference(f, plan, host, psfs, nb, field, PAD):
    from uniphot_b200 import solver
    tree, nt = solver.build_psf_tree(psfs, plan.tier)
    kern = solver.make_class_kernels(
        plan, nb, nt, render_backend="fft", reg=1e-9, pos_step_max_pix=0.5,
        chi2_ftol_rel=1e-4, step_tol_pix=0.1, un_freeze_steps=0,
        render_mode="reference", native_stamp=f.native)
    rows = np.arange(plan.n_islands)
    return solver.run_class_chunk(kern, tree, host, rows, rows.size, 0, field, field, PAD), \
        tree, nt


def _buffers(host, tree, d_data, d_w, rows=None, stype=None, ox=None):
    import torch
    cuda = d_data.device
    nb = d_data.shape[0]
    sel = np.arange(host["mmask"].shape[0]) if rows is None else np.asarray(rows)

    def dev(a, dt):
        return torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=cuda)

    n, N = sel.size, host["mmask"].shape[1]
    return dict(
        data=d_data, invvar=d_w, psf_coefs=dev(tree.params, torch.float32),
        psf_origin_scale=dev(tree.origin_scale, torch.float32),
        ox=dev(host["ox"][sel] if ox is None else ox, torch.int32),
        oy=dev(host["oy"][sel], torch.int32),
        x0b=dev(host["x0b"][sel], torch.float32), y0b=dev(host["y0b"][sel], torch.float32),
        stype=dev(host["st"][sel] if stype is None else stype, torch.int32),
        mmask=dev(host["mmask"][sel], torch.uint8),
        p=dev(host["p0"][sel].reshape(n, 6 * N), torch.float32),
        fluxes=torch.full((n, nb, N), np.nan, dtype=torch.float32, device=cuda),
        ferr=torch.full((n, nb, N), np.nan, dtype=torch.float32, device=cuda),
        chi2=torch.full((n,), np.nan, dtype=torch.float32, device=cuda))


def _call(bufs, plan, f, nt, Hp, Wp, stream):
    from uniphot_b200 import _lib
    n, nb, N = bufs["fluxes"].shape
    _lib.fluxes_noalloc({k: v.data_ptr() for k, v in bufs.items()},
                        n_islands=n, nsrc=N, bbox=plan.bbox_class, tier=plan.tier,
                        native_stamp=f.native, n_bands=nb, Hp=Hp, Wp=Wp, nt=nt,
                        stream=stream)


def _check(bufs, ref, mmask, rows, what):
    got = {k: bufs[k].cpu().numpy() for k in ("fluxes", "ferr", "chi2")}
    m = np.broadcast_to(mmask[rows][:, None, :], got["fluxes"].shape)
    for k in ("fluxes", "ferr"):
        np.testing.assert_allclose(got[k][m], ref[k][rows][m], rtol=1e-6, atol=0,
                                   err_msg=f"{what} {k}")
    np.testing.assert_allclose(got["chi2"], ref["chi2"][rows], rtol=1e-6,
                               err_msg=f"{what} chi2")


def test_noalloc_matches_allocating_entry_point_on_two_calls():
    import torch
    f, plans, hosts, PAD, ds, psfs, field, d_data, d_w = _setup()
    nb, Hp, Wp = ds.shape
    for call, ci in enumerate([0, 1]):
        p, h = plans[ci], hosts[ci]
        ref, tree, nt = _reference(f, p, h, psfs, nb, field, PAD)
        bufs = _buffers(h, tree, d_data, d_w)
        _call(bufs, p, f, nt, Hp, Wp, torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        _check(bufs, ref, h["mmask"], np.arange(p.n_islands), f"call {call}")


def test_noalloc_on_a_side_stream_then_fewer_islands_without_allocating():
    import torch
    f, plans, hosts, PAD, ds, psfs, field, d_data, d_w = _setup()
    nb, Hp, Wp = ds.shape
    ci = int(np.argmax([p.n_islands for p in plans]))
    p, h = plans[ci], hosts[ci]
    assert p.n_islands >= 3
    ref, tree, nt = _reference(f, p, h, psfs, nb, field, PAD)
    full = _buffers(h, tree, d_data, d_w)
    sub_rows = np.arange(1, p.n_islands, 2)
    sub = _buffers(h, tree, d_data, d_w, rows=sub_rows)
    torch.cuda.synchronize()
    side = torch.cuda.Stream()
    # every buffer exists before the first call; the warm call below must
    # leave the device's free memory unchanged
    _call(full, p, f, nt, Hp, Wp, side.cuda_stream)
    side.synchronize()
    _check(full, ref, h["mmask"], np.arange(p.n_islands), "side stream, all islands")
    free0 = torch.cuda.mem_get_info()[0]
    _call(sub, p, f, nt, Hp, Wp, side.cuda_stream)
    side.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert free1 == free0, f"device free memory moved by {free0 - free1} bytes"
    _check(sub, ref, h["mmask"], sub_rows, "side stream, fewer islands")
    # the earlier call's outputs are the caller's and stay as they were
    _check(full, ref, h["mmask"], np.arange(p.n_islands), "earlier outputs")


def test_noalloc_marks_invalid_islands_nan_and_keeps_the_rest():
    import torch
    f, plans, hosts, PAD, ds, psfs, field, d_data, d_w = _setup()
    nb, Hp, Wp = ds.shape
    ci = int(np.argmax([p.n_islands for p in plans]))
    p, h = plans[ci], hosts[ci]
    assert p.n_islands >= 3
    ref, tree, nt = _reference(f, p, h, psfs, nb, field, PAD)
    stype = h["st"].copy()
    stype[0, 0] = 1                      # an EXP member: not a point source
    ox = h["ox"].copy()
    ox[1] = Wp - p.bbox_class + 1        # window past the field's right edge
    bufs = _buffers(h, tree, d_data, d_w, stype=stype, ox=ox)
    _call(bufs, p, f, nt, Hp, Wp, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    fl = bufs["fluxes"].cpu().numpy()
    fe = bufs["ferr"].cpu().numpy()
    c2 = bufs["chi2"].cpu().numpy()
    for i in (0, 1):
        assert np.isnan(c2[i]) and np.isnan(fl[i]).all() and np.isnan(fe[i]).all()
    rest = np.arange(2, p.n_islands)
    m = np.broadcast_to(h["mmask"][rest][:, None, :], fl[rest].shape)
    np.testing.assert_allclose(fl[rest][m], ref["fluxes"][rest][m], rtol=1e-6, atol=0)
    np.testing.assert_allclose(fe[rest][m], ref["ferr"][rest][m], rtol=1e-6, atol=0)
    np.testing.assert_allclose(c2[rest], ref["chi2"][rest], rtol=1e-6)


def test_noalloc_rejects_work_beyond_the_fixed_array():
    from uniphot_b200 import _lib
    with pytest.raises(ValueError, match="scratch"):
        _lib.fluxes_noalloc({k: 1 << 20 for k in (
            "data", "invvar", "psf_coefs", "psf_origin_scale", "ox", "oy", "x0b",
            "y0b", "stype", "mmask", "p", "fluxes", "ferr", "chi2")},
            n_islands=100000, nsrc=32, bbox=128, tier=127, native_stamp=31,
            n_bands=20, Hp=4096, Wp=4096, nt=6)
