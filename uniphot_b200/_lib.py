"""ctypes binding of the C ABI in ``include/uniphot_b200.h``.

The shared library is built in-tree (``uniphot_b200/libuniphot_b200.so``);
there is no fallback: if it is missing or fails to load, every entry point
raises.
"""

from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "libuniphot_b200.so"

UPH_OK, UPH_ERR_INVALID, UPH_ERR_OOM, UPH_ERR_CUDA, UPH_ERR_TIMEOUT, \
    UPH_ERR_STATE = range(6)
ISLAND_TRIES_DEFAULT = 1 << 20      # UPH_ISLAND_TRIES_DEFAULT
RENDER_MODES = {"reference": 0, "analytic": 1}
PRECISIONS = {"plain": 0, "mixed": 1}
ENGINES = {"chunks": 0, "queue": 1, "queue_per_cta": 2}   # UPH_ENGINE_*

EXPORTED = ("uph_create", "uph_destroy", "uph_last_error", "uph_set_stream",
            "uph_get_stream", "uph_upload_field", "uph_upload_field_device", "uph_upload_field_unpadded",
            "uph_upload_psf_poly", "uph_upload_psf_mog",
            "uph_upload_sersic_table", "uph_run_chunk", "uph_last_timing",
            "uph_last_launch_count", "uph_job_create", "uph_job_destroy",
            "uph_job_add_chunk", "uph_job_solve", "uph_job_read",
            "uph_job_set_profile", "uph_job_kernel_time", "uph_job_kernel_work",
            "uph_job_chunk_time", "uph_sparse_band_solve", "uph_island_roots",
            "uph_set_island_retry_limit", "uph_job_kernel_exps", "uph_measure_peaks",
            "uph_job_set_engine", "uph_upload_exp_mog", "uph_subtract_tile_backgrounds",
            "uph_download_field", "uph_scene_subtract_stars", "uph_scene_waves")
KERNEL_KINDS = ("render", "gram", "assemble", "step", "trial_chi2", "accept",
                "gram_tc")

_P = C.c_void_p


class ClassDesc(C.Structure):
    _fields_ = [("bbox", C.c_int32), ("nsrc", C.c_int32), ("tier", C.c_int32),
                ("render_mode", C.c_int32), ("reg", C.c_float),
                ("pos_step_max", C.c_float), ("chi2_ftol_rel", C.c_float),
                ("step_tol_pix", C.c_float), ("un_freeze_steps", C.c_int32),
                ("has_priors", C.c_int32), ("native_stamp", C.c_int32),
                ("precision", C.c_int32), ("tc_min_rows", C.c_int32),
                ("stall_changed", C.c_int32), ("convergence_dlnp", C.c_int32),
                ("plateau_dlnp_tol", C.c_float), ("bg_joint", C.c_int32),
                ("tc_cond_max", C.c_float), ("step_tr", C.c_int32),
                ("param_errors", C.c_int32), ("flux_marg", C.c_int32),
                ("source_metrics", C.c_int32), ("re_profile", C.c_int32),
                ("residual", C.c_int32), ("scene_subtract", C.c_int32),
                ("render_direct", C.c_int32)]


class ChunkIn(C.Structure):
    _fields_ = [("n_islands", C.c_int32)] + [(n, _P) for n in (
        "ox", "oy", "x0b", "y0b", "stype", "n_frozen", "free_n", "mmask",
        "keep", "p0", "lower", "upper", "prior_mean", "prior_inv_sigma",
        "init_lam", "init_chi2", "init_consec", "init_nrej", "init_nst",
        "init_n_same", "init_prej", "init_diverged", "member_s1_flux", "seed_p")]


class ChunkOut(C.Structure):
    _fields_ = [(n, _P) for n in (
        "p", "fluxes", "ferr", "chi2", "conv", "stall", "diverged",
        "stall_dchi2", "nst", "lam", "consec", "nrej", "n_good")] + \
        [("steps_run", C.c_int32), ("bg", _P), ("bg_err", _P), ("n_same", _P),
         ("prej", _P), ("railed", _P), ("perr", _P), ("femarg", _P),
         ("smetrics", _P), ("swin", _P), ("reprof", _P), ("resid", _P),
         ("resid_w", _P), ("acond", _P)]


class SparseBand(C.Structure):
    _fields_ = [("band_h", C.c_int32), ("band_w", C.c_int32), ("data", _P),
                ("invvar", _P), ("pix_good", _P), ("n_sources", C.c_int32),
                ("pos_x", _P), ("pos_y", _P), ("grid_x0", C.c_int32),
                ("grid_y0", C.c_int32), ("psf_coefs", _P), ("psf_h", C.c_int32),
                ("psf_w", C.c_int32), ("psf_nterms", C.c_int32),
                ("psf_x_origin", C.c_float), ("psf_x_scale", C.c_float),
                ("psf_y_origin", C.c_float), ("psf_y_scale", C.c_float),
                ("renorm", C.c_int32), ("bg_x_origin", C.c_double),
                ("bg_x_scale", C.c_double), ("bg_y_origin", C.c_double),
                ("bg_y_scale", C.c_double), ("bg_order", C.c_int32),
                ("k_max", C.c_int32), ("neighbor_idx", _P), ("neighbor_mask", _P),
                ("reg", C.c_float), ("source_type", _P), ("logre", _P), ("ee1", _P),
                ("ee2", _P), ("sersic_n", _P), ("render_direct", C.c_int32),
                ("exp_k", C.c_int32), ("exp_amp", _P), ("exp_var", _P)]


class SparseOut(C.Structure):
    _fields_ = [("fluxes", _P), ("bg_coefs", _P), ("flux_var", _P), ("bg_var", _P),
                ("converged", C.c_int32)]


class UphError(RuntimeError):
    pass


_lib = None


def lib():
    """Load (once) the in-tree CUDA library; raises if absent."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise UphError(f"CUDA library not built: {LIB_PATH} (run "
                           f"__graft_entry__.build() or "
                           f"python -m uniphot_b200.csrc.build)")
        L = C.CDLL(str(LIB_PATH))
        L.uph_create.argtypes = [C.c_int, C.POINTER(_P)]
        L.uph_destroy.argtypes = [_P]
        L.uph_last_error.argtypes = [_P]
        L.uph_last_error.restype = C.c_char_p
        L.uph_set_stream.argtypes = [_P, _P]
        L.uph_get_stream.argtypes = [_P]
        L.uph_get_stream.restype = _P
        L.uph_upload_field.argtypes = [_P, _P, _P, C.c_int32, C.c_int32, C.c_int32, C.c_int32]
        L.uph_upload_field_device.argtypes = L.uph_upload_field.argtypes
        L.uph_upload_field_unpadded.argtypes = L.uph_upload_field.argtypes
        L.uph_upload_psf_poly.argtypes = [_P, C.c_int32, _P, _P, C.c_int32, C.c_int32]
        L.uph_upload_psf_mog.argtypes = [_P, _P, _P, C.c_int32, C.c_int32, C.c_int32]
        L.uph_upload_sersic_table.argtypes = [_P, _P, _P, _P, _P, C.c_int32, C.c_int32,
                                              C.c_double, C.c_double]
        L.uph_run_chunk.argtypes = [_P, C.POINTER(ClassDesc), C.POINTER(ChunkIn),
                                    C.c_int32, C.POINTER(ChunkOut)]
        L.uph_last_timing.argtypes = [_P, C.POINTER(C.c_float)]
        L.uph_last_launch_count.argtypes = [_P]
        L.uph_last_launch_count.restype = C.c_int64
        L.uph_job_create.argtypes = [_P, C.POINTER(_P)]
        L.uph_job_destroy.argtypes = [_P]
        L.uph_job_add_chunk.argtypes = [_P, C.POINTER(ClassDesc), C.POINTER(ChunkIn),
                                        C.POINTER(C.c_int32)]
        L.uph_job_solve.argtypes = [_P, C.c_int32]
        L.uph_job_read.argtypes = [_P, C.c_int32, C.POINTER(ChunkOut)]
        L.uph_job_set_profile.argtypes = [_P, C.c_int32]
        L.uph_job_kernel_time.argtypes = [_P, C.c_int32, C.POINTER(C.c_float),
                                          C.POINTER(C.c_int64)]
        L.uph_job_kernel_work.argtypes = [_P, C.c_int32, C.POINTER(C.c_double),
                                          C.POINTER(C.c_double)]
        L.uph_job_chunk_time.argtypes = [_P, C.c_int32, C.POINTER(C.c_float)]
        L.uph_sparse_band_solve.argtypes = [_P, C.POINTER(SparseBand), C.POINTER(SparseOut)]
        L.uph_island_roots.argtypes = [_P, _P, _P, _P, _P, C.c_int32, _P]
        L.uph_set_island_retry_limit.argtypes = [_P, C.c_int32]
        L.uph_job_kernel_exps.argtypes = [_P, C.c_int32, C.POINTER(C.c_double)]
        L.uph_job_set_engine.argtypes = [_P, C.c_int32, C.c_int32]
        L.uph_measure_peaks.argtypes = [_P, C.POINTER(C.c_double)]
        L.uph_upload_exp_mog.argtypes = [_P, _P, _P, C.c_int32]
        L.uph_subtract_tile_backgrounds.argtypes = [_P, C.c_int32, _P, _P, C.c_int32, _P]
        L.uph_download_field.argtypes = [_P, _P, _P]
        L.uph_scene_subtract_stars.argtypes = [_P, C.c_int32, _P, _P, _P, C.c_int32,
                                               C.c_int32, _P, _P]
        L.uph_scene_waves.argtypes = [C.c_int32, _P, _P, C.c_int32, _P]
        _lib = L
    return _lib


def ptr(a):
    return None if a is None else a.ctypes.data_as(_P)


def scene_waves(x, y, T: int) -> np.ndarray:
    """The wave of each source in the ordered star scene subtraction
    (uph_scene_waves; host only)."""
    xs = np.ascontiguousarray(x, np.float64)
    ys = np.ascontiguousarray(y, np.float64)
    w = np.zeros(xs.size, np.int32)
    if lib().uph_scene_waves(int(xs.size), ptr(xs), ptr(ys), int(T), ptr(w)) < 0:
        raise ValueError("scene_waves: bad positions or stamp side")
    return w


class Context:
    """One uph_ctx (one CUDA device)."""

    def __init__(self, device: int = 0):
        L = lib()
        h = _P()
        rc = L.uph_create(int(device), C.byref(h))
        if rc != UPH_OK:
            raise UphError(f"uph_create(device={device}) failed with status {rc}")
        self._h = h
        self.device = int(device)
        self._keep = []
        # bumped by every field upload: a DeviceField records the value it
        # was uploaded under, so a superseded one is detected
        self.field_gen = 0

    def close(self):
        if getattr(self, "_h", None):
            lib().uph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:   # noqa: BLE001 -- interpreter shutdown
            pass

    @property
    def handle(self):
        return self._h

    def check(self, rc: int, what: str):
        if rc == UPH_OK:
            return
        msg = lib().uph_last_error(self._h).decode(errors="replace")
        if rc == UPH_ERR_OOM and "RESOURCE_EXHAUSTED" not in msg:
            msg = "RESOURCE_EXHAUSTED: " + msg
        if rc == UPH_ERR_INVALID:
            raise ValueError(f"{what}: {msg}")
        raise UphError(f"{what}: status {rc}: {msg}")

    def set_stream(self, stream_ptr: int):
        self.check(lib().uph_set_stream(self._h, _P(stream_ptr) if stream_ptr else None),
                   "uph_set_stream")

    def stream_ptr(self) -> int:
        return int(lib().uph_get_stream(self._h) or 0)

    def upload_field(self, data: np.ndarray, invvar: np.ndarray, pad: int):
        d = np.ascontiguousarray(data, np.float32)
        w = np.ascontiguousarray(invvar, np.float32)
        nb, Hp, Wp = d.shape
        self.check(lib().uph_upload_field(self._h, ptr(d), ptr(w), nb, Hp, Wp, int(pad)),
                   "uph_upload_field")
        self.field_gen += 1

    def island_roots(self, x, y, radius, forced_singleton=None) -> np.ndarray:
        """Minimum member index of every source's island (uph_island_roots)."""
        xs = np.ascontiguousarray(x, np.float64)
        ys = np.ascontiguousarray(y, np.float64)
        rs = np.ascontiguousarray(radius, np.float64)
        fs = (None if forced_singleton is None
              else np.ascontiguousarray(np.asarray(forced_singleton).astype(np.uint8)))
        out = np.zeros(xs.size, np.int32)
        self.check(lib().uph_island_roots(self._h, ptr(xs), ptr(ys), ptr(rs), ptr(fs),
                                          int(xs.size), ptr(out)), "uph_island_roots")
        return out

    def measure_peaks(self) -> dict:
        """FP32 / FP64 multiply-add and exp2f rates of this device
        (uph_measure_peaks)."""
        out = (C.c_double * 3)()
        self.check(lib().uph_measure_peaks(self._h, out), "uph_measure_peaks")
        return {"fp32_tflops": out[0], "exp2_tera_per_s": out[1], "fp64_tflops": out[2]}

    def set_island_retry_limit(self, tries: int):
        """Unite attempts per coupled pair in island_roots before it gives up
        with UphError (status UPH_ERR_TIMEOUT); see uph_set_island_retry_limit."""
        self.check(lib().uph_set_island_retry_limit(self._h, int(tries)),
                   "uph_set_island_retry_limit")

    def sparse_band_solve(self, inputs, nbr_idx, nbr_mask, reg: float, order: int, M: int):
        """One band of one grid through uph_sparse_band_solve; returns a
        ``uniphot_b200.sparse.SparseForcedPhotResult``."""
        from .sparse import SparseForcedPhotResult
        h, w = int(inputs.band_h), int(inputs.band_w)
        d = np.ascontiguousarray(np.asarray(inputs.data, np.float32).reshape(h, w))
        iv = np.ascontiguousarray(np.asarray(inputs.invvar, np.float32).reshape(h, w))
        gd = np.ascontiguousarray(np.asarray(inputs.pix_good).astype(np.uint8).reshape(h, w))
        px = np.ascontiguousarray(inputs.pos_x, np.float32)
        py = np.ascontiguousarray(inputs.pos_y, np.float32)
        n = int(px.size)
        psf = inputs.psf
        cf = np.ascontiguousarray(psf.coefs, np.float32)
        H, W, nterms = cf.shape
        kmax = int(nbr_idx.shape[1]) if nbr_idx.ndim == 2 else 0
        ni = np.ascontiguousarray(nbr_idx, np.int32)
        nm = np.ascontiguousarray(nbr_mask).astype(np.uint8)
        ib = SparseBand(band_h=h, band_w=w, data=ptr(d), invvar=ptr(iv), pix_good=ptr(gd),
                        n_sources=n, pos_x=ptr(px), pos_y=ptr(py),
                        grid_x0=int(inputs.grid_x0), grid_y0=int(inputs.grid_y0),
                        psf_coefs=ptr(cf), psf_h=H, psf_w=W, psf_nterms=nterms,
                        psf_x_origin=float(psf.x_origin), psf_x_scale=float(psf.x_scale),
                        psf_y_origin=float(psf.y_origin), psf_y_scale=float(psf.y_scale),
                        renorm=int(bool(getattr(inputs, "renorm", True))),
                        bg_x_origin=float(inputs.bg_x_origin),
                        bg_x_scale=float(inputs.bg_x_scale),
                        bg_y_origin=float(inputs.bg_y_origin),
                        bg_y_scale=float(inputs.bg_y_scale), bg_order=int(order),
                        k_max=kmax, neighbor_idx=ptr(ni), neighbor_mask=ptr(nm),
                        reg=float(reg))
        keep = []
        st = getattr(inputs, "source_type", None)
        if st is not None and np.any(np.asarray(st) != 0):
            if getattr(inputs, "render_backend", "fft") == "direct":
                from .sparse import exp_mixture
                amp, var = exp_mixture()
                keep.extend((amp, var))
                ib.render_direct, ib.exp_k = 1, int(amp.size)
                ib.exp_amp, ib.exp_var = ptr(amp), ptr(var)
            elif not getattr(self, "_table", False):
                from .sersic import load_table
                self.upload_sersic_table(load_table())
                self._table = True
            zeros = np.zeros(n, np.float32)

            def f32(a, fill):
                return np.ascontiguousarray(fill if a is None else a, np.float32)
            arrs = (np.ascontiguousarray(st, np.int32),
                    f32(getattr(inputs, "logre", None), zeros),
                    f32(getattr(inputs, "ee1", None), zeros),
                    f32(getattr(inputs, "ee2", None), zeros),
                    f32(getattr(inputs, "sersic_n", None), np.ones(n, np.float32)))
            keep.extend(arrs)
            ib.source_type, ib.logre, ib.ee1, ib.ee2, ib.sersic_n = (ptr(a) for a in arrs)
        fl = np.zeros(n, np.float32)
        fv = np.zeros(n, np.float32)
        bg = np.zeros(M, np.float32)
        bv = np.zeros(M, np.float32)
        ob = SparseOut(fluxes=ptr(fl), bg_coefs=ptr(bg), flux_var=ptr(fv), bg_var=ptr(bv))
        self.check(lib().uph_sparse_band_solve(self._h, C.byref(ib), C.byref(ob)),
                   "uph_sparse_band_solve")
        return SparseForcedPhotResult(fluxes=fl, bg_coefs=bg, flux_var=fv, bg_var=bv,
                                      converged=bool(ob.converged))

    def upload_field_unpadded(self, data: np.ndarray, invvar: np.ndarray, pad: int):
        d = np.ascontiguousarray(data, np.float32)
        w = np.ascontiguousarray(invvar, np.float32)
        nb, H, W = d.shape
        self.check(lib().uph_upload_field_unpadded(self._h, ptr(d), ptr(w), nb, H, W,
                                                   int(pad)), "uph_upload_field_unpadded")
        self.field_gen += 1

    def upload_field_device(self, d_ptr: int, w_ptr: int, nb, Hp, Wp, pad):
        self.check(lib().uph_upload_field_device(self._h, _P(d_ptr), _P(w_ptr), nb, Hp,
                                                 Wp, int(pad)), "uph_upload_field_device")
        self.field_gen += 1

    def upload_psf_poly(self, tier: int, coefs: np.ndarray, origin_scale: np.ndarray):
        cf = np.ascontiguousarray(coefs, np.float32)
        os_ = np.ascontiguousarray(origin_scale, np.float32)
        self.check(lib().uph_upload_psf_poly(self._h, int(tier), ptr(cf), ptr(os_),
                                             cf.shape[0], cf.shape[-1]),
                   "uph_upload_psf_poly")

    def subtract_tile_backgrounds(self, tiles, coefs, order: int, norm):
        """Subtract each tile's planar background from the uploaded data
        stack (uph_subtract_tile_backgrounds): tiles (n, 4) = (x0, y0, x1,
        y1) cores, coefs (n, n_bands, M), norm = (x_origin, x_scale,
        y_origin, y_scale)."""
        t = np.ascontiguousarray(np.asarray(tiles, np.int32).reshape(-1, 4))
        c = np.ascontiguousarray(coefs, np.float32)
        nm = np.ascontiguousarray(np.asarray(norm, np.float64).reshape(4))
        if c.shape[0] != t.shape[0]:
            raise ValueError(f"{t.shape[0]} tiles but coefficients for {c.shape[0]}")
        self.check(lib().uph_subtract_tile_backgrounds(self._h, int(t.shape[0]), ptr(t), ptr(c),
                                                       int(order), ptr(nm)),
                   "uph_subtract_tile_backgrounds")

    def scene_subtract_stars(self, x, y, flux, coefs, origin_scale):
        """Subtract flux x the star stamps from the uploaded data stack
        (uph_scene_subtract_stars): x, y (n,), flux (n, n_bands), coefs
        (n_bands, T, T, nt), origin_scale (n_bands, 4)."""
        xs = np.ascontiguousarray(x, np.float64)
        ys = np.ascontiguousarray(y, np.float64)
        fl = np.ascontiguousarray(flux, np.float32)
        cf = np.ascontiguousarray(coefs, np.float32)
        os_ = np.ascontiguousarray(origin_scale, np.float32)
        nb, T, T2, nt = cf.shape
        if T != T2 or fl.shape != (xs.size, nb) or ys.size != xs.size:
            raise ValueError("scene_subtract_stars: inconsistent shapes")
        self.check(lib().uph_scene_subtract_stars(self._h, int(xs.size), ptr(xs), ptr(ys),
                                                  ptr(fl), int(T), int(nt), ptr(cf),
                                                  ptr(os_)), "uph_scene_subtract_stars")

    def download_field(self, shape) -> tuple:
        """The padded (data, invvar) stacks of the given (n_bands, Hp, Wp)
        shape, copied to the host."""
        d = np.empty(shape, np.float32)
        w = np.empty(shape, np.float32)
        self.check(lib().uph_download_field(self._h, ptr(d), ptr(w)), "uph_download_field")
        return d, w

    def upload_exp_mog(self, amp: np.ndarray, var: np.ndarray):
        """The "direct" backend's exponential mixture (uph_upload_exp_mog)."""
        a = np.ascontiguousarray(amp, np.float32)
        v = np.ascontiguousarray(var, np.float32)
        self.check(lib().uph_upload_exp_mog(self._h, ptr(a), ptr(v), int(a.size)),
                   "uph_upload_exp_mog")

    def upload_psf_mog(self, params: np.ndarray, origin_scale: np.ndarray):
        pr = np.ascontiguousarray(params, np.float32)
        os_ = np.ascontiguousarray(origin_scale, np.float32)
        nb, K, _, nt = pr.shape
        self.check(lib().uph_upload_psf_mog(self._h, ptr(pr), ptr(os_), nb, K, nt),
                   "uph_upload_psf_mog")

    def upload_sersic_table(self, table: dict):
        kn = np.ascontiguousarray(table["n_knots"], np.float64)
        am = np.ascontiguousarray(table["amps"], np.float64)
        lv = np.ascontiguousarray(table["log_vars"], np.float64)
        co = np.ascontiguousarray(table["core_amp"], np.float64)
        self.check(lib().uph_upload_sersic_table(
            self._h, ptr(kn), ptr(am), ptr(lv), ptr(co), kn.size, am.shape[1],
            float(table["n_min"]), float(table["n_max"])), "uph_upload_sersic_table")

    def run_chunk(self, desc: ClassDesc, arrays: dict, max_steps: int,
                  nb: int, init_state: dict | None = None) -> dict:
        """One chunk through uph_run_chunk (upload, solve, read)."""
        cin, keep_alive = chunk_in(arrays, init_state)
        n, N = arrays["mmask"].shape
        out, cout = chunk_out(n, N, nb, int(desc.bbox) if desc.residual else 0)
        rc = lib().uph_run_chunk(self._h, C.byref(desc), C.byref(cin), int(max_steps),
                                 C.byref(cout))
        self.check(rc, "uph_run_chunk")
        return finish_out(out, cout)

    def last_timing(self):
        buf = (C.c_float * 4)()
        lib().uph_last_timing(self._h, buf)
        return [float(x) for x in buf]

    def last_launch_count(self) -> int:
        return int(lib().uph_last_launch_count(self._h))


def chunk_in(arrays: dict, init_state: dict | None = None):
    """ChunkIn over contiguous copies of class host arrays (kept alive by the
    returned dict)."""
    n, N = arrays["mmask"].shape
    nP = 6 * N

    def f32(a, shape):
        return np.ascontiguousarray(np.asarray(a, np.float32).reshape(shape))

    def i32(a, shape):
        return np.ascontiguousarray(np.asarray(a, np.int32).reshape(shape))

    def u8(a, shape):
        return np.ascontiguousarray(np.asarray(a).astype(np.uint8).reshape(shape))
    keep = dict(
        ox=i32(arrays["ox"], n), oy=i32(arrays["oy"], n),
        x0b=f32(arrays["x0b"], n), y0b=f32(arrays["y0b"], n),
        stype=i32(arrays["st"], (n, N)), n_frozen=f32(arrays["sn"], (n, N)),
        free_n=u8(arrays["fn_flag"], (n, N)), mmask=u8(arrays["mmask"], (n, N)),
        keep=u8(arrays["keep"], (n, nP)), p0=f32(arrays["p0"], (n, nP)),
        lower=f32(arrays["lower"], (n, nP)), upper=f32(arrays["upper"], (n, nP)),
        prior_mean=f32(arrays["prior_mean"], (n, nP)),
        prior_inv_sigma=f32(arrays["prior_inv_sigma"], (n, nP)))
    if arrays.get("member_s1_flux") is not None:
        # scene subtract: S1 fluxes and the seeds of the add-back
        keep["member_s1_flux"] = f32(arrays["member_s1_flux"], (n, N, -1))
        keep["seed_p"] = f32(arrays["p0"], (n, nP))
    if init_state is not None:
        keep["p0"] = f32(init_state["p"], (n, nP))
        for k, conv in (("lam", f32), ("chi2", f32), ("consec", i32), ("nrej", i32),
                        ("nst", i32)):
            keep["init_" + k] = conv(init_state[k], n)
        # "changed"-mode tracker carry (the reference's _CARRY_KEYS)
        if init_state.get("n_same") is not None:
            keep["init_n_same"] = i32(init_state["n_same"], n)
        if init_state.get("prej") is not None:
            keep["init_prej"] = f32(init_state["prej"], (n, nP))
        if init_state.get("diverged") is not None:
            keep["init_diverged"] = u8(init_state["diverged"], n)
    cin = ChunkIn(n_islands=n)
    for k, v in keep.items():
        setattr(cin, k, ptr(v))
    return cin, keep


def chunk_out(n: int, N: int, nb: int, B: int = 0):
    """Output arrays of one chunk (the residual images only when B > 0)."""
    out = dict(p=np.zeros((n, N, 6), np.float32),
               fluxes=np.zeros((n, nb, N), np.float32),
               ferr=np.zeros((n, nb, N), np.float32),
               chi2=np.zeros(n, np.float32), conv=np.zeros(n, np.uint8),
               stall=np.zeros(n, np.uint8), diverged=np.zeros(n, np.uint8),
               stall_dchi2=np.zeros(n, np.float32), nst=np.zeros(n, np.int32),
               lam=np.zeros(n, np.float32), consec=np.zeros(n, np.int32),
               nrej=np.zeros(n, np.int32), n_good=np.zeros(n, np.int64),
               bg=np.zeros((n, nb, 3), np.float32), bg_err=np.zeros((n, nb, 3), np.float32),
               n_same=np.zeros(n, np.int32), prej=np.zeros((n, 6 * N), np.float32),
               railed=np.zeros(n, np.uint8), perr=np.zeros((n, N, 13), np.float32),
               femarg=np.zeros((n, nb, N), np.float32),
               smetrics=np.zeros((n, N, 4), np.float32), swin=np.zeros((n, nb, N), np.float32),
               reprof=np.zeros((n, N, 12), np.float32),
               acond=np.zeros((n, nb), np.float32))
    if B > 0:
        out["resid"] = np.zeros((n, B, B), np.float32)
        out["resid_w"] = np.zeros((n, B, B), np.float32)
    cout = ChunkOut()
    for k, v in out.items():
        setattr(cout, k, ptr(v))
    return out, cout


def finish_out(out: dict, cout: ChunkOut) -> dict:
    for k in ("conv", "stall", "diverged", "railed"):
        out[k] = out[k].astype(bool)
    out["steps_run"] = int(cout.steps_run)
    return out


class Job:
    """Many chunks resident on the device, solved concurrently."""

    def __init__(self, ctx: Context):
        self.ctx = ctx
        h = _P()
        ctx.check(lib().uph_job_create(ctx.handle, C.byref(h)), "uph_job_create")
        self._h = h
        self.shapes = []

    def add_chunk(self, desc: ClassDesc, arrays: dict, nb: int,
                  init_state: dict | None = None) -> int:
        cin, _keep = chunk_in(arrays, init_state)
        cid = C.c_int32(-1)
        self.ctx.check(lib().uph_job_add_chunk(self._h, C.byref(desc), C.byref(cin),
                                               C.byref(cid)), "uph_job_add_chunk")
        n, N = arrays["mmask"].shape
        self.shapes.append((n, N, nb, int(desc.bbox) if desc.residual else 0))
        return int(cid.value)

    def set_engine(self, engine: str, lanes: int = 0):
        """LM loop engine: "queue" (persistent work-queue kernels, one per
        kernel kind, for all chunks of a lane; ``lanes`` lanes overlap, 0
        for the default), "queue_per_cta" (the same queue, one unit per
        CTA) or "chunks" (each chunk's iterations as its own graph on a
        stream pool); see uph_job_set_engine."""
        self.ctx.check(lib().uph_job_set_engine(self._h, ENGINES[engine], int(lanes)),
                       "uph_job_set_engine")

    def solve(self, max_steps: int):
        self.ctx.check(lib().uph_job_solve(self._h, int(max_steps)), "uph_job_solve")

    def read(self, cid: int) -> dict:
        n, N, nb, B = self.shapes[cid]
        out, cout = chunk_out(n, N, nb, B)
        self.ctx.check(lib().uph_job_read(self._h, int(cid), C.byref(cout)),
                       "uph_job_read")
        return finish_out(out, cout)

    def set_profile(self, on: bool):
        self.ctx.check(lib().uph_job_set_profile(self._h, int(bool(on))),
                       "uph_job_set_profile")

    def kernel_times(self) -> dict:
        res = {}
        for i, name in enumerate(KERNEL_KINDS):
            ms = C.c_float(0)
            cnt = C.c_int64(0)
            lib().uph_job_kernel_time(self._h, i, C.byref(ms), C.byref(cnt))
            res[name] = (float(ms.value), int(cnt.value))
        return res

    def chunk_time(self, chunk_id: int) -> float:
        """ms from the start of the last solve to the end of one chunk."""
        ms = C.c_float(0)
        self.ctx.check(lib().uph_job_chunk_time(self._h, int(chunk_id), C.byref(ms)),
                       "uph_job_chunk_time")
        return float(ms.value)

    def kernel_work(self) -> dict:
        """Algorithmic (bytes, flops, exponentials) per kernel kind of the
        last instrumented solve."""
        res = {}
        for i, name in enumerate(KERNEL_KINDS):
            by = C.c_double(0)
            fl = C.c_double(0)
            ex = C.c_double(0)
            lib().uph_job_kernel_work(self._h, i, C.byref(by), C.byref(fl))
            lib().uph_job_kernel_exps(self._h, i, C.byref(ex))
            res[name] = (float(by.value), float(fl.value), float(ex.value))
        return res

    def close(self):
        if getattr(self, "_h", None):
            lib().uph_job_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # noqa: BLE001
            pass


# ---------------------------------------------------------------------------
# Allocation-free final-flux pass (uph_fluxes_noalloc): for callers that own
# all device memory and cannot allocate (see include/uniphot_b200.h).
# ---------------------------------------------------------------------------

class NoallocArgs(C.Structure):
    _fields_ = [(n, _P) for n in (
        "data", "invvar", "psf_coefs", "psf_origin_scale", "ox", "oy", "x0b",
        "y0b", "stype", "mmask", "p", "fluxes", "ferr", "chi2")] + \
        [(n, C.c_int32) for n in ("n_islands", "nsrc", "bbox", "tier",
                                  "native_stamp", "n_bands", "Hp", "Wp", "nt")] + \
        [("reg", C.c_float), ("stream", _P), ("err_buf", C.c_char_p),
         ("err_len", C.c_int32)]


NOALLOC_SCRATCH_BYTES = 32 << 20


def fluxes_noalloc(ptrs: dict, *, n_islands: int, nsrc: int, bbox: int, tier: int,
                   native_stamp: int, n_bands: int, Hp: int, Wp: int, nt: int,
                   reg: float = 1e-9, stream: int = 0) -> None:
    """Call uph_fluxes_noalloc with caller-owned device pointers
    (``ptrs[name]`` = integer device address for every pointer field)."""
    L = lib()
    fn = L.uph_fluxes_noalloc
    fn.argtypes = [C.POINTER(NoallocArgs)]
    fn.restype = C.c_int
    err = C.create_string_buffer(256)
    a = NoallocArgs()
    for name, _t in NoallocArgs._fields_[:14]:
        setattr(a, name, _P(int(ptrs[name])))
    a.n_islands, a.nsrc, a.bbox, a.tier = int(n_islands), int(nsrc), int(bbox), int(tier)
    a.native_stamp, a.n_bands, a.Hp, a.Wp, a.nt = (int(native_stamp), int(n_bands),
                                                   int(Hp), int(Wp), int(nt))
    a.reg = float(reg)
    a.stream = _P(int(stream)) if stream else None
    a.err_buf = C.cast(err, C.c_char_p)
    a.err_len = 256
    rc = fn(C.byref(a))
    if rc != UPH_OK:
        msg = err.value.decode(errors="replace")
        if rc == UPH_ERR_INVALID:
            raise ValueError(msg)
        raise UphError(f"uph_fluxes_noalloc: status {rc}: {msg}")
