"""The allocation-free final-flux entry point against the allocating one.

Callers that cannot allocate device memory (a host inside a framework that
owns the device pool, or a serving process with a fixed budget) own every
buffer and call uph_fluxes_noalloc; its intermediates live in a fixed device
array inside the library.  Two calls in a row, on two different island
classes, must reproduce uph_run_chunk(max_steps=0) -- the fluxes,
sqrt(diag inv A64) and chi2 at fixed parameters -- within 1e-6 relative.
This file is collected last so that a failure here never hides another test.
"""
import numpy as np
import pytest

from _common import field_classes

pytestmark = pytest.mark.gpu


def test_noalloc_matches_allocating_entry_point_on_two_calls():
    import torch
    from uniphot_b200 import _lib, solver
    from uniphot_b200.synth import make_small_field
    f = make_small_field(0)
    plans, hosts, PAD, ds, ws, psfs = field_classes(f, "reference", ("star",))
    assert len(plans) >= 2
    field = solver.DeviceField(ds, ws, PAD)
    nb, Hp, Wp = ds.shape
    cuda = torch.device("cuda", 0)

    def dev(a, dt):
        return torch.as_tensor(np.ascontiguousarray(a), dtype=dt, device=cuda)

    d_data, d_w = dev(ds, torch.float32), dev(ws, torch.float32)
    for call, ci in enumerate([0, 1]):
        p, h = plans[ci], hosts[ci]
        tree, nt = solver.build_psf_tree(psfs, p.tier)
        kern = solver.make_class_kernels(
            p, nb, nt, render_backend="fft", reg=1e-9, pos_step_max_pix=0.5,
            chi2_ftol_rel=1e-4, step_tol_pix=0.1, un_freeze_steps=0,
            render_mode="reference", native_stamp=f.native)
        rows = np.arange(p.n_islands)
        ref = solver.run_class_chunk(kern, tree, h, rows, rows.size, 0, field, field, PAD)
        n, N = h["mmask"].shape
        bufs = dict(
            data=d_data, invvar=d_w, psf_coefs=dev(tree.params, torch.float32),
            psf_origin_scale=dev(tree.origin_scale, torch.float32),
            ox=dev(h["ox"], torch.int32), oy=dev(h["oy"], torch.int32),
            x0b=dev(h["x0b"], torch.float32), y0b=dev(h["y0b"], torch.float32),
            stype=dev(h["st"], torch.int32), mmask=dev(h["mmask"], torch.uint8),
            p=dev(h["p0"].reshape(n, 6 * N), torch.float32),
            fluxes=torch.full((n, nb, N), np.nan, dtype=torch.float32, device=cuda),
            ferr=torch.full((n, nb, N), np.nan, dtype=torch.float32, device=cuda),
            chi2=torch.full((n,), np.nan, dtype=torch.float32, device=cuda))
        _lib.fluxes_noalloc({k: v.data_ptr() for k, v in bufs.items()},
                            n_islands=n, nsrc=N, bbox=p.bbox_class, tier=p.tier,
                            native_stamp=f.native, n_bands=nb, Hp=Hp, Wp=Wp, nt=nt,
                            stream=torch.cuda.current_stream().cuda_stream)
        torch.cuda.synchronize()
        got = {k: bufs[k].cpu().numpy() for k in ("fluxes", "ferr", "chi2")}
        m = np.broadcast_to(h["mmask"][:, None, :], got["fluxes"].shape)
        for k in ("fluxes", "ferr"):
            np.testing.assert_allclose(got[k][m], ref[k][m], rtol=1e-6, atol=0,
                                       err_msg=f"call {call} {k}")
        np.testing.assert_allclose(got["chi2"], ref["chi2"], rtol=1e-6,
                                   err_msg=f"call {call} chi2")


def test_noalloc_rejects_work_beyond_the_fixed_array():
    from uniphot_b200 import _lib
    with pytest.raises(ValueError, match="scratch"):
        _lib.fluxes_noalloc({k: 1 << 20 for k in (
            "data", "invvar", "psf_coefs", "psf_origin_scale", "ox", "oy", "x0b",
            "y0b", "stype", "mmask", "p", "fluxes", "ferr", "chi2")},
            n_islands=100000, nsrc=32, bbox=128, tier=127, native_stamp=31,
            n_bands=20, Hp=4096, Wp=4096, nt=6)
