"""ctypes wrapper of the FP64 oracle (oracle/liboracle.so) -- TEST INFRASTRUCTURE.

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs use this
module, as the checker.  `RefLib` wraps oracle/_ref/libscphd_ref.so, the
reference's own sources compiled for the host (built where the reference tree is
present; tests that need it skip when it is absent).
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "liboracle.so")
REF_SO = os.path.join(HERE, "_ref", "libscphd_ref.so")

P = ctypes.POINTER
D, I32, U32, U64, U8 = ctypes.c_double, ctypes.c_int32, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint8
VP = ctypes.c_void_p

STAGE_PRIOR, STAGE_CAM, STAGE_FEAT, STAGE_SAMPLE, STAGE_RESAMPLE = 1, 2, 3, 4, 5


def build(ref_dir: str | None = None) -> None:
    """Build liboracle.so, and _ref/libscphd_ref.so when a reference tree is given
    (argument, or the REF_DIR environment variable) and holds the sources."""
    subprocess.run(["make", "-s", "liboracle.so"], cwd=HERE, check=True)
    ref_dir = ref_dir or os.environ.get("REF_DIR")
    if ref_dir and os.path.isdir(os.path.join(ref_dir, "src")):
        subprocess.run(["make", "-s", "ref", f"REF_DIR={ref_dir}"], cwd=HERE, check=True)


def _d(a):
    return None if a is None else a.ctypes.data_as(P(D))


def _i(a):
    return None if a is None else a.ctypes.data_as(P(I32))


def _f64(a):
    return np.ascontiguousarray(np.asarray(a, np.float64))


_olib = None


def lib():
    global _olib
    if _olib is None:
        if not os.path.exists(ORACLE_SO):
            build()
        L = ctypes.CDLL(ORACLE_SO)
        sigs = {
            "orc_create": (VP, [VP]),
            "orc_destroy": (None, [VP]),
            "orc_set_weight_mode": (None, [VP, I32]),
            "orc_set_threads": (I32, [I32]),
            "orc_predict": (None, [VP, D]),
            "orc_update": (None, [VP, P(D), P(D), P(D), I32, I32]),
            "orc_resample": (I32, [VP]),
            "orc_frame": (I32, [VP]),
            "orc_set_frame": (None, [VP, I32]),
            "orc_get_particles": (None, [VP, P(D), P(D)]),
            "orc_map_size": (I32, [VP, I32]),
            "orc_get_map": (None, [VP, I32, P(D), P(D), P(D)]),
            "orc_set_state": (None, [VP, P(D), P(D), P(I32), P(D), P(D), P(D)]),
            "orc_fitted_count": (I32, [VP, I32]),
            "orc_get_fitted": (None, [VP, I32, P(D)]),
            "orc_merged_count": (I32, [VP, I32]),
            "orc_get_merged": (None, [VP, I32, P(D)]),
            "orc_get_normalizers": (None, [VP, P(D), P(D)]),
            "orc_get_survivors": (None, [VP, P(I32)]),
            "orc_get_resample_indices": (None, [VP, P(I32)]),
            "orc_philox": (None, [P(U32), P(U32), P(U32)]),
            "orc_philox_rounds": (None, [P(U32), P(U32), I32, P(U32)]),
            "orc_normals4": (None, [U64, U32, U32, U32, U32, P(D)]),
            "orc_ctr_word3": (U32, [I32, I32, I32]),
            "orc_merge": (None, [P(D), P(U8), I32, D, P(D), P(I32), P(I32)]),
            "orc_systematic": (None, [P(D), I32, D, P(I32)]),
            "orc_mahal6": (D, [P(D), P(D)]),
            "orc_is_pos_def": (I32, [P(D)]),
            "orc_wrap_angle": (D, [D]),
            "orc_tie_key": (U32, [U32]),
            "orc_measure": (None, [VP, P(D), P(D), P(D)]),
            "orc_invert": (None, [VP, P(D), P(D), P(D)]),
            "orc_detect": (None, [VP, P(D), P(D), P(D)]),
            "orc_cap_keep": (None, [P(D), I32, I32, P(U8)]),
            "orc_truncations": (ctypes.c_int64, [VP]),
            "orc_precut_weights": (I32, [VP, I32, P(D)]),
            "orc_unit_weight_fits": (ctypes.c_int64, [VP]),
        }
        for name, (res, args) in sigs.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _olib = L
    return _olib


def set_threads(n: int = 0) -> int:
    return int(lib().orc_set_threads(int(n)))


class Oracle:
    """FP64 CPU restatement of the filter, same config struct as the device library."""

    def __init__(self, cfg, weight_mode: int = 0):
        self.cfg = cfg
        self.N = int(cfg.n_parents)
        self.P = int(cfg.particles_per_feature)
        self._h = lib().orc_create(ctypes.byref(cfg))
        if weight_mode:
            lib().orc_set_weight_mode(self._h, int(weight_mode))

    def __del__(self):
        if getattr(self, "_h", None):
            lib().orc_destroy(self._h)
            self._h = None

    def predict(self, dt):
        lib().orc_predict(self._h, float(dt))

    def update(self, u, v, fixed_camera=False, d=None):
        u, v = _f64(u), _f64(v)
        dd = _f64(d) if d is not None else None
        lib().orc_update(self._h, _d(u), _d(v), _d(dd), int(u.size), int(bool(fixed_camera)))

    def resample(self) -> bool:
        return bool(lib().orc_resample(self._h))

    @property
    def frame(self) -> int:
        return int(lib().orc_frame(self._h))

    def set_frame(self, frame: int) -> None:
        lib().orc_set_frame(self._h, int(frame))

    def state(self):
        """The whole state as set_state takes it (with the frame counter)."""
        st, lw = self.particles()
        sizes = self.map_sizes()
        parts = [self.map(p) for p in range(self.N)]
        cat = lambda i, shp: np.concatenate([q[i] for q in parts]) if sizes.sum() else np.zeros(shp)
        return (st, lw, sizes, cat(0, (0,)), cat(1, (0, 6, self.P)), cat(2, (0, self.P))), self.frame

    def load(self, state_and_frame) -> None:
        state, frame = state_and_frame
        self.set_state(*state)
        self.set_frame(frame)

    def particles(self):
        st = np.zeros((self.N, 12))
        lw = np.zeros(self.N)
        lib().orc_get_particles(self._h, _d(st), _d(lw))
        return st, lw

    def map_sizes(self):
        return np.array([lib().orc_map_size(self._h, p) for p in range(self.N)], np.int32)

    def map(self, p):
        n = lib().orc_map_size(self._h, p)
        W = np.zeros(n)
        x = np.zeros((n, 6, self.P))
        om = np.zeros((n, self.P))
        if n:
            lib().orc_get_map(self._h, p, _d(W), _d(x), _d(om))
        return W, x, om

    def set_state(self, states, logw, sizes, W, clouds, omega):
        states, logw, W, clouds, omega = map(_f64, (states, logw, W, clouds, omega))
        sizes = np.ascontiguousarray(np.asarray(sizes, np.int32))
        lib().orc_set_state(self._h, _d(states), _d(logw), _i(sizes), _d(W), _d(clouds), _d(omega))

    def fitted(self, p):
        n = lib().orc_fitted_count(self._h, p)
        out = np.zeros((n, 29))
        if n:
            lib().orc_get_fitted(self._h, p, _d(out))
        return out

    def merged(self, p):
        n = lib().orc_merged_count(self._h, p)
        out = np.zeros((n, 28))
        if n:
            lib().orc_get_merged(self._h, p, _d(out))
        return out

    def normalizers(self, M):
        ell = np.zeros((self.N, M))
        ll = np.zeros(self.N)
        lib().orc_get_normalizers(self._h, _d(ell), _d(ll))
        return ell, ll

    def survivors(self):
        s = np.zeros(self.N, np.int32)
        lib().orc_get_survivors(self._h, _i(s))
        return s

    def precut_weights(self, p):
        """Entry weights of parent p's new map before the capacity cut (last update)."""
        n = lib().orc_precut_weights(self._h, p, None)
        w = np.zeros(n)
        if n:
            lib().orc_precut_weights(self._h, p, _d(w))
        return w

    def unit_weight_fits(self) -> int:
        """In-view clouds fitted with unit weights (all their weights were 0) since create."""
        return int(lib().orc_unit_weight_fits(self._h))

    def truncations(self) -> int:
        """Maps cut at max_gaussians since create."""
        return int(lib().orc_truncations(self._h))

    def resample_indices(self):
        idx = np.zeros(self.N, np.int32)
        lib().orc_get_resample_indices(self._h, _i(idx))
        return idx

    def measure(self, X, e12):
        y = np.zeros(6)
        lib().orc_measure(self._h, _d(_f64(X)), _d(_f64(e12)), _d(y))
        return y

    def invert(self, y, e12):
        X = np.zeros(6)
        lib().orc_invert(self._h, _d(_f64(y)), _d(_f64(e12)), _d(X))
        return X

    def detect(self, g29, z):
        out = np.zeros(28)
        z3 = np.zeros(3)
        z3[: len(z)] = z
        lib().orc_detect(self._h, _d(_f64(g29)), _d(z3), _d(out))
        return out


def philox(ctr, key):
    """The generator of the random streams (Philox4x32, 7 rounds)."""
    c = (U32 * 4)(*ctr)
    k = (U32 * 2)(*key)
    o = (U32 * 4)()
    lib().orc_philox(c, k, o)
    return list(o)


def philox_rounds(ctr, key, rounds):
    c = (U32 * 4)(*ctr)
    k = (U32 * 2)(*key)
    o = (U32 * 4)()
    lib().orc_philox_rounds(c, k, int(rounds), o)
    return list(o)


def normals4(seed, s, j, p, c3):
    z = np.zeros(4)
    lib().orc_normals4(int(seed), s, j, p, c3, _d(z))
    return z


def ctr_word3(frame, stage, block):
    return int(lib().orc_ctr_word3(frame, stage, block))


def merge(comps, flags, min_sep):
    comps = _f64(comps).reshape(-1, 28)
    n = comps.shape[0]
    fl = np.ascontiguousarray(np.asarray(flags, np.uint8))
    out = np.zeros((max(n, 1), 28))
    nout = I32(0)
    mem = np.zeros(max(n, 1), np.int32)
    lib().orc_merge(_d(comps), fl.ctypes.data_as(P(U8)), n, float(min_sep), _d(out), ctypes.byref(nout), _i(mem))
    return out[: nout.value], mem[:n]


def cap_keep(w, cap):
    """Entries kept when a map with entry weights w is cut to cap entries."""
    w = _f64(w)
    keep = np.zeros(w.size, np.uint8)
    lib().orc_cap_keep(_d(w), int(w.size), int(cap), keep.ctypes.data_as(P(U8)))
    return keep.astype(bool)


def systematic(w, u01):
    w = _f64(w)
    idx = np.zeros(w.size, np.int32)
    lib().orc_systematic(_d(w), int(w.size), float(u01), _i(idx))
    return idx


def mahal6(a28, b28):
    return float(lib().orc_mahal6(_d(_f64(a28)), _d(_f64(b28))))


def is_pos_def(cov36):
    return bool(lib().orc_is_pos_def(_d(_f64(cov36).reshape(36))))


def wrap_angle(a):
    return float(lib().orc_wrap_angle(float(a)))


def tie_key(r):
    return int(lib().orc_tie_key(int(r)))


class RefLib:
    """The reference's own kernels/math compiled for the host (oracle/_ref)."""

    def __init__(self, path: str = REF_SO):
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = ctypes.CDLL(path)
        sigs = {
            "ref_safe_log": (D, [D]),
            "ref_wrap_angle": (D, [D]),
            "ref_cholesky": (None, [P(D), P(D), I32]),
            "ref_is_pos_def": (I32, [P(D)]),
            "ref_mahal": (D, [P(D), P(D)]),
            "ref_measure": (None, [P(D), P(D), P(D), P(D)]),
            "ref_invert": (None, [P(D), P(D), P(D), P(D)]),
            "ref_noisy_motion": (None, [P(D), D, P(D)]),
            "ref_world_to_disparity": (None, [P(D), P(D), I32, P(D), P(I32), P(D), P(D)]),
            "ref_detections": (None, [P(D), P(D), I32, P(D), P(D), I32, P(D)]),
            "ref_update": (None, [P(D), I32, P(D), P(D), I32, D, P(D), P(U8)]),
        }
        for name, (res, args) in sigs.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        self.L = L

    @staticmethod
    def model8(cfg):
        lam = cfg.kappa * (2 * cfg.v0) ** 2
        return np.array([cfg.fx, cfg.fy, cfg.u0, cfg.v0, cfg.std_u, cfg.std_v, cfg.pd, lam])

    def measure(self, m8, X, e12):
        y = np.zeros(6)
        self.L.ref_measure(_d(_f64(m8)), _d(_f64(X)), _d(_f64(e12)), _d(y))
        return y

    def invert(self, m8, y, e12):
        X = np.zeros(6)
        self.L.ref_invert(_d(_f64(m8)), _d(_f64(y)), _d(_f64(e12)), _d(X))
        return X

    def noisy_motion(self, e12, dt, a6):
        e = _f64(e12).copy()
        self.L.ref_noisy_motion(_d(e), float(dt), _d(_f64(a6)))
        return e

    def world_to_disparity(self, m8, X6xn, ex12, indices):
        X6xn = _f64(X6xn)
        n = X6xn.shape[1]
        y = np.zeros((6, n))
        pd = np.zeros(n)
        idx = np.ascontiguousarray(np.asarray(indices, np.int32))
        self.L.ref_world_to_disparity(_d(_f64(m8)), _d(X6xn), n, _d(_f64(ex12)), _i(idx), _d(y), _d(pd))
        return y, pd

    def detections(self, m8, fit29, u, v):
        fit29 = _f64(fit29).reshape(-1, 29)
        G = fit29.shape[0]
        u, v = _f64(u), _f64(v)
        out = np.zeros((G * u.size, 43))
        self.L.ref_detections(_d(_f64(m8)), _d(fit29), G, _d(u), _d(v), int(u.size), _d(out))
        return out

    def update(self, det43, G, birth43, norms, min_weight):
        det43, birth43, norms = _f64(det43), _f64(birth43), _f64(norms)
        M = norms.size
        out = np.zeros(((G + 1) * M, 43))
        flags = np.zeros((G + 1) * M, np.uint8)
        self.L.ref_update(_d(det43), int(G), _d(birth43), _d(norms), M, float(min_weight), _d(out),
                          flags.ctypes.data_as(P(U8)))
        return out, flags

    def cholesky(self, A, n):
        L = np.zeros(n * n)
        self.L.ref_cholesky(_d(_f64(A).reshape(-1)), _d(L), n)
        return L

    def is_pos_def(self, cov36):
        return bool(self.L.ref_is_pos_def(_d(_f64(cov36).reshape(36))))

    def mahal(self, a28, b28):
        return float(self.L.ref_mahal(_d(_f64(a28)), _d(_f64(b28))))

    def wrap_angle(self, a):
        return float(self.L.ref_wrap_angle(float(a)))
