"""Python binding of the B200 SC-PHD calibration filter (ctypes over the C ABI).

`SCPHDCameraCalibration` mirrors the step API of the reference class of the same
name (src/scphdcameracalibration.cuh:29-44): predict(dt), update(u, v,
fixed_camera) -- with an optional disparity vector d for (u,v,d) measurements --
resample(), checkStuff() and the particle/mixture dumps of writeMat().  Errors
raise ScphdError with the library's message; there is no CPU fallback: if the
CUDA library cannot be loaded, constructing a filter fails.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional, Sequence

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "csrc", "libscphd_b200.so")

SCPHD_FP32 = 0
SCPHD_FP64 = 1
SCPHD_MIX_FITTED = 0
SCPHD_MIX_MERGED = 1

# names of the 16 counters of scphd_get_counters, in the order include/scphd.h gives them
COUNTER_NAMES = (
    "map_truncations", "scratch_overflows", "frames_updated", "resamplings",
    "units_last_update", "survivors_last_update", "units_total", "survivors_total",
    "clouds_read", "clouds_written", "gaussians_fitted", "merged_rows",
    "mahalanobis_evaluations", "max_survivors_per_parent", "unit_weight_fits", "reserved",
)

_STATUS = {0: "OK", 1: "INVALID", 2: "CUDA", 3: "CAPACITY", 4: "NAN", 5: "NO_DEVICE"}


class ScphdError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"scphd {_STATUS.get(status, status)}: {message}")
        self.status = status


class ScphdConfig(ctypes.Structure):
    """Mirror of `scphd_config` in include/scphd.h (field order and types)."""

    _fields_ = [
        ("n_parents", ctypes.c_int32),
        ("particles_per_feature", ctypes.c_int32),
        ("max_gaussians", ctypes.c_int32),
        ("max_measurements", ctypes.c_int32),
        ("meas_dim", ctypes.c_int32),
        ("precision", ctypes.c_int32),
        ("max_survivors", ctypes.c_int32),
        ("device", ctypes.c_int32),
        ("seed", ctypes.c_uint64),
        ("prior_a", ctypes.c_double * 12),
        ("prior_b", ctypes.c_double * 12),
        ("cam_std", ctypes.c_double * 6),
        ("feat_std", ctypes.c_double * 3),
        ("fx", ctypes.c_double),
        ("fy", ctypes.c_double),
        ("u0", ctypes.c_double),
        ("v0", ctypes.c_double),
        ("std_u", ctypes.c_double),
        ("std_v", ctypes.c_double),
        ("std_d", ctypes.c_double),
        ("pd", ctypes.c_double),
        ("kappa", ctypes.c_double),
        ("baseline", ctypes.c_double),
        ("ps", ctypes.c_double),
        ("min_weight", ctypes.c_double),
        ("min_separation", ctypes.c_double),
        ("min_neff", ctypes.c_double),
        ("w0", ctypes.c_double),
        ("d0", ctypes.c_double),
        ("vu0", ctypes.c_double),
        ("vv0", ctypes.c_double),
        ("vd0", ctypes.c_double),
        ("var_d0", ctypes.c_double),
        ("var_vu0", ctypes.c_double),
        ("var_vv0", ctypes.c_double),
        ("var_vd0", ctypes.c_double),
    ]

    def copy(self) -> "ScphdConfig":
        c = ScphdConfig()
        ctypes.pointer(c)[0] = self
        return c

    def as_dict(self) -> dict:
        out = {}
        for name, _ in self._fields_:
            v = getattr(self, name)
            out[name] = list(v) if isinstance(v, ctypes.Array) else v
        return out


class ScphdRunOptions(ctypes.Structure):
    """scphd_run_options: driver settings read from a configuration file."""
    _fields_ = [("max_steps", ctypes.c_int32), ("slam", ctypes.c_int32), ("save_all_maps", ctypes.c_int32),
                ("verbosity", ctypes.c_int32)]


class ScphdFrame(ctypes.Structure):
    """scphd_frame: one filter's measurements for a batched step."""
    _fields_ = [("u", ctypes.c_void_p), ("v", ctypes.c_void_p), ("d", ctypes.c_void_p),
                ("n", ctypes.c_int32), ("fixed_camera", ctypes.c_int32)]


def reference_defaults() -> ScphdConfig:
    """The values of the reference's config/calibration.cfg, read the way its code
    reads them (the shipped {mean,std} prior becomes the box mean +- max(std, 0)),
    meas_dim 2, baseline 1, kappa = lambda / (2 v0)^2 with lambda = 10.0001
    (src/disparitymeasurementmodel.cu:157-162)."""
    c = ScphdConfig()
    c.n_parents = 100
    c.particles_per_feature = 100
    c.max_gaussians = 256
    c.max_measurements = 64
    c.meas_dim = 2
    c.precision = SCPHD_FP64
    c.max_survivors = 0
    c.device = 0
    c.seed = 0x5C9D0000
    mean = [0.0, -50.0, -3.0, 0.0, 0.0, 0.0, 0.3927, 0.1, 0.0, 0.0, 0.0, 0.0]
    std = [0.0, 0.0, 3.0, 0.0, 0.0, 0.0, 0.0, 0.1, 0.0, 0.0, 0.0, 0.0]
    for i in range(12):
        c.prior_a[i] = mean[i] - std[i]
        c.prior_b[i] = mean[i] + std[i]
    for i, v in enumerate([0.0, 0.0, 0.15, 0.0, 0.001, 0.0]):
        c.cam_std[i] = v
    for i, v in enumerate([0.05, 0.05, 0.1]):
        c.feat_std[i] = v
    c.fx, c.fy, c.u0, c.v0 = -895.6561, -891.2656, 400.0, 300.0
    c.std_u = c.std_v = 5.0
    c.std_d = 1.0
    c.pd = 0.95
    c.kappa = 10.0001 / (2 * 300.0) ** 2
    c.baseline = 1.0
    c.ps = 0.9
    c.min_weight = 0.0001
    c.min_separation = 6.0
    c.min_neff = 0.75
    c.w0, c.d0, c.vu0, c.vv0, c.vd0 = 0.000001, 8.0, 0.0, 0.0, 0.0
    c.var_d0, c.var_vu0, c.var_vv0, c.var_vd0 = 2.0, 6.0, 6.0, 0.05
    return c


_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Load the CUDA library.  Raises if it is missing: there is no fallback."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise ScphdError(5, f"CUDA library not built: {path} (run __graft_entry__.build())")
    lib = ctypes.CDLL(path)
    P = ctypes.POINTER
    d, i32, i64, u8 = ctypes.c_double, ctypes.c_int32, ctypes.c_int64, ctypes.c_uint8
    vp = ctypes.c_void_p
    sigs = {
        "scphd_config_defaults": (None, [P(ScphdConfig)]),
        "scphd_create": (i32, [P(ScphdConfig), P(vp)]),
        "scphd_destroy": (i32, [vp]),
        "scphd_predict": (i32, [vp, d]),
        "scphd_update": (i32, [vp, P(d), P(d), P(d), i32, i32]),
        "scphd_update_device": (i32, [vp, vp, vp, vp, i32, i32]),
        "scphd_resample": (i32, [vp, P(i32)]),
        "scphd_step": (i32, [vp, d, P(d), P(d), P(d), i32, i32]),
        "scphd_step_device": (i32, [vp, d, vp, vp, vp, i32, i32]),
        "scphd_check": (i32, [vp]),
        "scphd_synchronize": (i32, [vp]),
        "scphd_get_particles": (i32, [vp, P(d), P(d)]),
        "scphd_get_map_sizes": (i32, [vp, P(i32)]),
        "scphd_get_map_weights": (i32, [vp, i32, P(d)]),
        "scphd_get_map_clouds": (i32, [vp, i32, P(d), P(d)]),
        "scphd_get_mixture": (i32, [vp, i32, i32, P(d), P(i32)]),
        "scphd_get_normalizers": (i32, [vp, P(d), P(d)]),
        "scphd_get_resample_indices": (i32, [vp, P(i32)]),
        "scphd_set_state": (i32, [vp, P(d), P(d), P(i32), P(d), P(d), P(d)]),
        "scphd_get_counters": (i32, [vp, P(i64)]),
        "scphd_merge_components": (i32, [P(d), P(u8), i32, d, i32, P(d), P(i32), P(i32)]),
        "scphd_systematic_resample": (i32, [P(d), i32, d, P(i32)]),
        "scphd_stream": (vp, [vp]),
        "scphd_set_profiling": (i32, [vp, i32]),
        "scphd_get_stage_times": (i32, [vp, P(d), P(i64)]),
        "scphd_device_bytes": (i32, [P(ScphdConfig), P(i64)]),
        "scphd_batch_create": (i32, [P(vp), i32, i32, P(vp)]),
        "scphd_batch_destroy": (i32, [vp]),
        "scphd_batch_step": (i32, [vp, d, P(ScphdFrame)]),
        "scphd_batch_step_device": (i32, [vp, d, P(ScphdFrame)]),
        "scphd_batch_stream": (vp, [vp]),
        "scphd_server_create": (i32, [i32, i32, i32, i64, i32, P(vp)]),
        "scphd_server_destroy": (i32, [vp]),
        "scphd_server_submit": (i32, [vp, P(ScphdConfig), i32, P(i32), P(d), P(d), P(d), P(i32), d, P(i64)]),
        "scphd_server_step": (i32, [vp, P(i32)]),
        "scphd_server_drain": (i32, [vp]),
        "scphd_server_job_status": (i32, [vp, i64, P(i32), P(i32)]),
        "scphd_server_job_result": (i32, [vp, i64, P(d), P(d)]),
        "scphd_server_stats": (i32, [vp, P(i64)]),
        "scphd_server_step_times": (i32, [vp, i64, i32, P(d), P(i32), P(i32)]),
        "scphd_get_config": (i32, [vp, P(ScphdConfig)]),
        "scphd_set_autotune": (i32, [vp, i32]),
        "scphd_get_launch_shapes": (i32, [vp, P(i32), P(i32), P(i32)]),
        "scphd_set_fused": (i32, [vp, i32]),
        "scphd_get_fused": (i32, [vp, P(i32)]),
        "scphd_batch_set_fused": (i32, [vp, i32]),
        "scphd_batch_get_fused": (i32, [vp, P(i32)]),
        "scphd_get_particles_async": (i32, [vp, vp, vp]),
        "scphd_set_fit_split": (i32, [vp, i32]),
        "scphd_get_fit_split": (i32, [vp, P(i32), P(i32)]),
        "scphd_batch_set_fit_split": (i32, [vp, i32]),
        "scphd_batch_get_fit_split": (i32, [vp, P(i32), P(i32)]),
        "scphd_config_from_file": (i32, [ctypes.c_char_p, P(ScphdConfig), P(ScphdRunOptions)]),
        "scphd_read_mat_frames": (i32, [ctypes.c_char_p, ctypes.c_char_p, P(i32), P(i32), P(i32), P(d), i64]),
        "scphd_write_mat": (i32, [vp, ctypes.c_char_p, i32]),
        "scphd_write_mat_arrays": (i32, [ctypes.c_char_p, i32, P(ctypes.c_char_p), P(i32), P(i32),
                                         P(P(d))]),
        "scphd_last_error": (ctypes.c_char_p, []),
        "scphd_kernel_launches": (i64, []),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def _check(status: int) -> None:
    if status != 0:
        msg = _lib.scphd_last_error() if _lib is not None else b""
        raise ScphdError(status, (msg or b"").decode(errors="replace"))


def _dptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def _iptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_int32))


def _f64(x) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(x, dtype=np.float64))


def device_bytes(config: ScphdConfig) -> int:
    """Device memory a filter with this configuration allocates (no device needed)."""
    lib = load_library()
    out = ctypes.c_int64(0)
    _check(lib.scphd_device_bytes(ctypes.byref(config), ctypes.byref(out)))
    return int(out.value)


def config_from_file(path: str, base: Optional[ScphdConfig] = None):
    """Read a configuration file in the reference's libconfig syntax; returns the
    filter configuration (starting from `base` or the library defaults) and the
    driver options {max_steps, slam, save_all_maps, verbosity}."""
    lib = load_library()
    cfg = base.copy() if base is not None else ScphdConfig()
    if base is None:
        lib.scphd_config_defaults(ctypes.byref(cfg))
    opts = ScphdRunOptions(1 << 30, 0, 0, 0)
    _check(lib.scphd_config_from_file(os.fsencode(path), ctypes.byref(cfg), ctypes.byref(opts)))
    return cfg, {"max_steps": int(opts.max_steps), "slam": bool(opts.slam),
                 "save_all_maps": bool(opts.save_all_maps), "verbosity": int(opts.verbosity)}


def read_mat_frames(path: str, var: str):
    """Frames of a MAT cell array of 2 x n or 3 x n matrices, as a list of (rows, n)
    arrays (the reference's readMatfile)."""
    lib = load_library()
    n, rows = ctypes.c_int32(0), ctypes.c_int32(0)
    _check(lib.scphd_read_mat_frames(os.fsencode(path), var.encode(), ctypes.byref(n), ctypes.byref(rows),
                                     None, None, 0))
    cap = 1 << 16
    while True:
        sizes = np.zeros(n.value, np.int32)
        data = np.zeros(cap, np.float64)
        st = lib.scphd_read_mat_frames(os.fsencode(path), var.encode(), ctypes.byref(n), ctypes.byref(rows),
                                       _iptr(sizes), _dptr(data), cap)
        if st == 3:   # capacity
            cap *= 4
            continue
        _check(st)
        break
    out, at, r = [], 0, rows.value
    for k in range(n.value):
        out.append(data[at:at + r * sizes[k]].reshape(r, sizes[k]).copy())
        at += r * sizes[k]
    return out


def write_mat_arrays(path: str, arrays: dict) -> None:
    """Write named real matrices to a MAT file."""
    lib = load_library()
    items = [(k, np.asfortranarray(np.atleast_2d(np.asarray(v, np.float64)))) for k, v in arrays.items()]
    n = len(items)
    names = (ctypes.c_char_p * n)(*[k.encode() for k, _ in items])
    rows = (ctypes.c_int32 * n)(*[a.shape[0] for _, a in items])
    cols = (ctypes.c_int32 * n)(*[a.shape[1] for _, a in items])
    ptrs = (ctypes.POINTER(ctypes.c_double) * n)(*[a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))
                                                   for _, a in items])
    _check(lib.scphd_write_mat_arrays(os.fsencode(path), n, names, rows, cols, ptrs))


def kernel_launches() -> int:
    return int(load_library().scphd_kernel_launches())


class SCPHDCameraCalibration:
    """One SC-PHD calibration filter on one GPU (the reference's class, re-hosted)."""

    def __init__(self, config: ScphdConfig):
        self._lib = load_library()
        self.config = config.copy()
        h = ctypes.c_void_p()
        _check(self._lib.scphd_create(ctypes.byref(self.config), ctypes.byref(h)))
        self._h = h

    # -- lifecycle
    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            _check(self._lib.scphd_destroy(self._h))
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def n_parents(self) -> int:
        return int(self.config.n_parents)

    # -- the reference's step API
    def predict(self, dt: float) -> None:
        _check(self._lib.scphd_predict(self._h, float(dt)))

    def update(self, u: Sequence[float], v: Sequence[float], fixed_camera: bool = False,
               d: Optional[Sequence[float]] = None) -> None:
        u, v = _f64(u), _f64(v)
        dd = _f64(d) if d is not None else None
        if u.shape != v.shape or (dd is not None and dd.shape != u.shape):
            raise ScphdError(1, "u, v (and d) must have the same length")
        _check(self._lib.scphd_update(self._h, _dptr(u), _dptr(v), _dptr(dd), int(u.size),
                                      int(bool(fixed_camera))))

    def update_device(self, u_ptr: int, v_ptr: int, d_ptr: Optional[int], n: int,
                      fixed_camera: bool = False) -> None:
        """update() with measurement vectors already resident in device memory
        (FP64 device pointers, e.g. torch tensors' data_ptr())."""
        _check(self._lib.scphd_update_device(self._h, ctypes.c_void_p(u_ptr), ctypes.c_void_p(v_ptr),
                                             ctypes.c_void_p(d_ptr) if d_ptr else None, int(n),
                                             int(bool(fixed_camera))))

    def resample(self) -> bool:
        r = ctypes.c_int32(0)
        _check(self._lib.scphd_resample(self._h, ctypes.byref(r)))
        return bool(r.value)

    def step(self, dt: float, u, v, fixed_camera: bool = False, d=None) -> None:
        u, v = _f64(u), _f64(v)
        dd = _f64(d) if d is not None else None
        _check(self._lib.scphd_step(self._h, float(dt), _dptr(u), _dptr(v), _dptr(dd),
                                    int(u.size), int(bool(fixed_camera))))

    def step_device(self, dt: float, u_ptr: int, v_ptr: int, d_ptr: Optional[int], n: int,
                    fixed_camera: bool = False) -> None:
        """predict + update + resample with device-resident FP64 measurement vectors;
        no host synchronisation."""
        _check(self._lib.scphd_step_device(self._h, float(dt), ctypes.c_void_p(u_ptr), ctypes.c_void_p(v_ptr),
                                           ctypes.c_void_p(d_ptr) if d_ptr else None, int(n),
                                           int(bool(fixed_camera))))

    def set_autotune(self, enable: bool) -> None:
        """Tune the launch shapes on the first updates (default) or keep the default."""
        _check(self._lib.scphd_set_autotune(self._h, int(bool(enable))))

    def launch_shapes(self) -> dict:
        mt, lf, tuned = ctypes.c_int32(0), ctypes.c_int32(0), ctypes.c_int32(0)
        _check(self._lib.scphd_get_launch_shapes(self._h, ctypes.byref(mt), ctypes.byref(lf), ctypes.byref(tuned)))
        fz = ctypes.c_int32(0)
        _check(self._lib.scphd_get_fused(self._h, ctypes.byref(fz)))
        sp, st = ctypes.c_int32(0), ctypes.c_int32(0)
        _check(self._lib.scphd_get_fit_split(self._h, ctypes.byref(sp), ctypes.byref(st)))
        return {"merge_threads": mt.value, "likelihood_full": bool(lf.value), "tuned": bool(tuned.value),
                "fused": bool(fz.value), "fit_blocks_per_parent": sp.value, "fit_tuned": bool(st.value)}

    def set_fit_split(self, blocks_per_parent: int) -> None:
        """Cloud-fit blocks per parent (1, 2 or 4); fixes it instead of tuning it."""
        _check(self._lib.scphd_set_fit_split(self._h, int(blocks_per_parent)))

    def set_fused(self, mode: int) -> None:
        """Update path: 0 one kernel per stage (default), 1 the fused kernel."""
        _check(self._lib.scphd_set_fused(self._h, int(mode)))

    def writeMat(self, path: str, save_all_maps: bool = False) -> None:
        """The reference's writeMat: particles, weights and the MAP parent's map (and
        with save_all_maps the per-parent mixtures) to a MAT file."""
        _check(self._lib.scphd_write_mat(self._h, os.fsencode(path), int(bool(save_all_maps))))

    write_mat = writeMat

    def checkStuff(self) -> None:
        _check(self._lib.scphd_check(self._h))

    check_stuff = checkStuff

    def synchronize(self) -> None:
        _check(self._lib.scphd_synchronize(self._h))

    # -- state dumps (writeMat's particle / mixture content)
    def particles(self):
        n = self.n_parents
        st = np.zeros((n, 12), np.float64)
        lw = np.zeros(n, np.float64)
        _check(self._lib.scphd_get_particles(self._h, _dptr(st), _dptr(lw)))
        return st, lw

    def particles_async(self, states_ptr: int, log_weights_ptr: int) -> None:
        """Queue the copy of the parent states (n x 12 FP64) and log-weights (n FP64) into
        caller buffers (page-locked for an asynchronous copy) on the filter's stream; they
        hold the result once work recorded after this call on stream_handle is done."""
        _check(self._lib.scphd_get_particles_async(self._h, ctypes.c_void_p(states_ptr),
                                                   ctypes.c_void_p(log_weights_ptr)))

    def map_sizes(self) -> np.ndarray:
        s = np.zeros(self.n_parents, np.int32)
        _check(self._lib.scphd_get_map_sizes(self._h, _iptr(s)))
        return s

    def map_weights(self, p: int) -> np.ndarray:
        n = int(self.map_sizes()[p])
        w = np.zeros(n, np.float64)
        _check(self._lib.scphd_get_map_weights(self._h, int(p), _dptr(w)))
        return w

    def map_clouds(self, p: int):
        n = int(self.map_sizes()[p])
        P = int(self.config.particles_per_feature)
        x = np.zeros((n, 6, P), np.float64)
        om = np.zeros((n, P), np.float64)
        _check(self._lib.scphd_get_map_clouds(self._h, int(p), _dptr(x), _dptr(om)))
        return x, om

    def mixture(self, which: int, p: int) -> np.ndarray:
        cnt = ctypes.c_int32(0)
        _check(self._lib.scphd_get_mixture(self._h, int(which), int(p), None, ctypes.byref(cnt)))
        width = 29 if which == SCPHD_MIX_FITTED else 28
        out = np.zeros((cnt.value, width), np.float64)
        _check(self._lib.scphd_get_mixture(self._h, int(which), int(p), _dptr(out), ctypes.byref(cnt)))
        return out

    def normalizers(self, n_meas: int):
        ell = np.zeros((self.n_parents, n_meas), np.float64)
        ll = np.zeros(self.n_parents, np.float64)
        _check(self._lib.scphd_get_normalizers(self._h, _dptr(ell), _dptr(ll)))
        return ell, ll

    def resample_indices(self) -> np.ndarray:
        idx = np.zeros(self.n_parents, np.int32)
        _check(self._lib.scphd_get_resample_indices(self._h, _iptr(idx)))
        return idx

    def counters(self) -> np.ndarray:
        c = np.zeros(16, np.int64)
        _check(self._lib.scphd_get_counters(self._h, c.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
        return c

    def counters_by_name(self) -> dict:
        """scphd_get_counters as {name: value} (names: COUNTER_NAMES)."""
        return dict(zip(COUNTER_NAMES, (int(v) for v in self.counters())))

    @property
    def stream_handle(self) -> int:
        """cudaStream_t of the handle (an integer), e.g. for torch.cuda.ExternalStream."""
        return int(self._lib.scphd_stream(self._h) or 0)

    def set_profiling(self, enable: bool) -> None:
        _check(self._lib.scphd_set_profiling(self._h, int(bool(enable))))

    STAGES = ("predict_parents", "cloud_fit", "likelihood", "merge", "weights", "resample", "kalman_terms")

    def stage_times(self):
        """{stage: (total ms, launches)} since the last call (profiling mode)."""
        ms = np.zeros(8, np.float64)
        n = np.zeros(8, np.int64)
        _check(self._lib.scphd_get_stage_times(self._h, _dptr(ms), n.ctypes.data_as(ctypes.POINTER(ctypes.c_int64))))
        return {name: (float(ms[i]), int(n[i])) for i, name in enumerate(self.STAGES)}

    def set_state(self, states, log_weights, sizes, weights, clouds, omega) -> None:
        states, log_weights = _f64(states), _f64(log_weights)
        sizes = np.ascontiguousarray(np.asarray(sizes, np.int32))
        weights, clouds, omega = _f64(weights), _f64(clouds), _f64(omega)
        _check(self._lib.scphd_set_state(self._h, _dptr(states), _dptr(log_weights), _iptr(sizes),
                                         _dptr(weights), _dptr(clouds), _dptr(omega)))


class SCPHDBatch:
    """Several filters stepped together: one launch per stage for all of them
    (scphd_batch_* in include/scphd.h).  Each member gets the result it would get
    stepped alone.  The batch keeps its filters alive and returns them to their own
    streams on close()."""

    def __init__(self, filters: Sequence[SCPHDCameraCalibration], use_graph: bool = False):
        self._lib = load_library()
        self.filters = list(filters)
        arr = (ctypes.c_void_p * len(self.filters))(*[f._h.value for f in self.filters])
        h = ctypes.c_void_p()
        _check(self._lib.scphd_batch_create(arr, len(self.filters), int(bool(use_graph)), ctypes.byref(h)))
        self._h = h
        self._frames = (ScphdFrame * len(self.filters))()
        self._keep = []

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            _check(self._lib.scphd_batch_destroy(self._h))
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def step(self, dt: float, frames) -> None:
        """frames: per filter (u, v, d or None, fixed_camera) host arrays."""
        if len(frames) != len(self.filters):
            raise ScphdError(1, "one frame per filter")
        keep = []
        for i, (u, v, d, fixed) in enumerate(frames):
            u, v = _f64(u), _f64(v)
            dd = _f64(d) if d is not None else None
            if u.shape != v.shape or (dd is not None and dd.shape != u.shape):
                raise ScphdError(1, "u, v (and d) must have the same length")
            keep += [u, v, dd]
            fr = self._frames[i]
            fr.u, fr.v = u.ctypes.data, v.ctypes.data
            fr.d = dd.ctypes.data if dd is not None else None
            fr.n, fr.fixed_camera = int(u.size), int(bool(fixed))
        _check(self._lib.scphd_batch_step(self._h, float(dt), self._frames))

    def step_device(self, dt: float, frames) -> None:
        """frames: per filter (u_ptr, v_ptr, d_ptr or None, n, fixed_camera) with FP64
        device pointers that stay valid until the step has run on stream_handle()."""
        if len(frames) != len(self.filters):
            raise ScphdError(1, "one frame per filter")
        for i, (u, v, d, n, fixed) in enumerate(frames):
            fr = self._frames[i]
            fr.u, fr.v, fr.d = int(u), int(v), (int(d) if d else None)
            fr.n, fr.fixed_camera = int(n), int(bool(fixed))
        _check(self._lib.scphd_batch_step_device(self._h, float(dt), self._frames))

    def stream_handle(self) -> int:
        return int(self._lib.scphd_batch_stream(self._h) or 0)

    def set_fused(self, mode: int) -> None:
        """Update path before the first graph capture: 0 stage kernels (default), 1 fused."""
        _check(self._lib.scphd_batch_set_fused(self._h, int(mode)))

    def fused(self) -> bool:
        fz = ctypes.c_int32(0)
        _check(self._lib.scphd_batch_get_fused(self._h, ctypes.byref(fz)))
        return bool(fz.value)

    def set_fit_split(self, blocks_per_parent: int) -> None:
        """Cloud-fit blocks per parent (1, 2 or 4) before the first graph capture."""
        _check(self._lib.scphd_batch_set_fit_split(self._h, int(blocks_per_parent)))

    def fit_split(self) -> dict:
        sp, st = ctypes.c_int32(0), ctypes.c_int32(0)
        _check(self._lib.scphd_batch_get_fit_split(self._h, ctypes.byref(sp), ctypes.byref(st)))
        return {"fit_blocks_per_parent": sp.value, "fit_tuned": bool(st.value)}

    def synchronize(self) -> None:
        for f in self.filters:
            f.synchronize()


JOB_QUEUED, JOB_RUNNING, JOB_DONE = 0, 1, 2


class SCPHDServer:
    """Resident serving loop (scphd_server_* in include/scphd.h): jobs are admitted
    first come, first served under a device-memory budget and advanced together, one
    batched frame per step()."""

    def __init__(self, budget_bytes: int, precision: int = 0, meas_dim: int = 3, device: int = 0,
                 use_graph: bool = True):
        self._lib = load_library()
        self.precision, self.meas_dim, self.device = precision, meas_dim, device
        h = ctypes.c_void_p()
        _check(self._lib.scphd_server_create(int(device), int(precision), int(meas_dim), int(budget_bytes),
                                             int(bool(use_graph)), ctypes.byref(h)))
        self._h = h
        self._parents = {}

    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            _check(self._lib.scphd_server_destroy(self._h))
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, config: ScphdConfig, frames, fixed, dt: float) -> int:
        """frames: list of (n, meas_dim) arrays (u, v[, d]); fixed: per-frame flags."""
        sizes = np.array([len(z) for z in frames], np.int32)
        parts = [np.asarray(z, np.float64).reshape(len(z), -1)[:, :self.meas_dim] for z in frames if len(z)]
        cat = np.concatenate(parts, axis=0) if parts else np.zeros((0, self.meas_dim))
        u, v = _f64(cat[:, 0]), _f64(cat[:, 1])
        d = _f64(cat[:, 2]) if self.meas_dim == 3 else None
        fx = np.asarray(fixed, np.int32)
        jid = ctypes.c_int64(0)
        cfg = config.copy()
        _check(self._lib.scphd_server_submit(self._h, ctypes.byref(cfg), int(len(frames)), _iptr(sizes), _dptr(u),
                                             _dptr(v), _dptr(d), _iptr(fx), float(dt), ctypes.byref(jid)))
        self._parents[jid.value] = int(cfg.n_parents)
        return int(jid.value)

    def step(self) -> int:
        n = ctypes.c_int32(0)
        _check(self._lib.scphd_server_step(self._h, ctypes.byref(n)))
        return int(n.value)

    def drain(self) -> None:
        _check(self._lib.scphd_server_drain(self._h))

    def status(self, job: int):
        st, fd = ctypes.c_int32(0), ctypes.c_int32(0)
        _check(self._lib.scphd_server_job_status(self._h, int(job), ctypes.byref(st), ctypes.byref(fd)))
        return int(st.value), int(fd.value)

    def result(self, job: int):
        n = self._parents[job]
        st = np.zeros((n, 12), np.float64)
        lw = np.zeros(n, np.float64)
        _check(self._lib.scphd_server_job_result(self._h, int(job), _dptr(st), _dptr(lw)))
        return st, lw

    def stats(self) -> dict:
        out = (ctypes.c_int64 * 8)()
        _check(self._lib.scphd_server_stats(self._h, out))
        keys = ("queued", "running", "done", "bytes_in_use", "steps", "job_frames", "units", "rebuilds")
        return dict(zip(keys, [int(x) for x in out]))

    def step_times(self, first: int = 0, max_n: int = 1 << 20):
        ms = np.zeros(max_n, np.float64)
        jobs = np.zeros(max_n, np.int32)
        n = ctypes.c_int32(0)
        _check(self._lib.scphd_server_step_times(self._h, int(first), int(max_n), _dptr(ms), _iptr(jobs),
                                                 ctypes.byref(n)))
        return ms[:n.value], jobs[:n.value]


def merge_components(comps: np.ndarray, flags: np.ndarray, min_separation: float,
                     precision: int = SCPHD_FP64):
    """Device greedy merge of one component list (rows of 28); see include/scphd.h."""
    lib = load_library()
    comps = _f64(comps).reshape(-1, 28)
    n = comps.shape[0]
    fl = np.ascontiguousarray(np.asarray(flags, np.uint8))
    out = np.zeros((max(n, 1), 28), np.float64)
    n_out = ctypes.c_int32(0)
    mem = np.zeros(max(n, 1), np.int32)
    _check(lib.scphd_merge_components(_dptr(comps), fl.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), n,
                                      float(min_separation), int(precision), _dptr(out),
                                      ctypes.byref(n_out), _iptr(mem)))
    return out[: n_out.value], mem[:n]


def systematic_resample(weights: np.ndarray, u01: float) -> np.ndarray:
    lib = load_library()
    w = _f64(weights)
    idx = np.zeros(w.size, np.int32)
    _check(lib.scphd_systematic_resample(_dptr(w), int(w.size), float(u01), _iptr(idx)))
    return idx
