"""Seeded synthetic calibration scenes and the filter configurations used on them.

A scene follows the workload shapes the filter is benchmarked on: a rig with
focal 500 px (fx = fy = -500 in the reference's sign convention, where
u = u0 - fx x / z), principal point (320, 240), a 640x480 image, stereo baseline
0.2 m; static landmarks uniform in a 10x10x10 m box 2..12 m ahead of camera 1;
camera 1 fixed at the world origin, camera 2 (the one being calibrated) on a
smooth seeded trajectory about its calibration pose; measurements (u, v, d) with
detection probability pD, Gaussian noise (sigma 1 px, 1 px, 0.5 px) and Poisson
clutter uniform over image x disparity [1, 64].  Frames alternate between the
fixed camera (even k) and camera 2 (odd k), as the reference's driver does
(src/main.cpp:78-91), with dt = 0.5 (src/main.cpp:81).

The world->camera transform is the reference's Euler convention
(src/disparitymeasurementmodel.cu:3-80), restated in numpy.
"""
from __future__ import annotations

from dataclasses import dataclass, field
from typing import List, Optional

import numpy as np

FOCAL = 500.0
U0, V0 = 320.0, 240.0
IMG_W, IMG_H = 640.0, 480.0
BASELINE_M = 0.2
SIGMA_UV, SIGMA_D = 1.0, 0.5
D_MIN, D_MAX = 1.0, 64.0
DT = 0.5
SCENE_SEED_BASE = 0x5C9D0000


def rotation_terms(ang):
    """Rows of the world->camera rotation for Euler angles (theta, phi, psi)."""
    th, ph, ps = ang
    ct, st, cf, sf, cp, sp = np.cos(th), np.sin(th), np.cos(ph), np.sin(ph), np.cos(ps), np.sin(ps)
    return np.array([
        [cf * cp, ct * sp + st * sf * cp, st * sp - ct * sf * cp],
        [-cf * sp, ct * cp - st * sf * sp, st * cp + ct * sf * sp],
        [sf, -st * cf, ct * cf],
    ])


def project(points: np.ndarray, ext12: np.ndarray, fx=-FOCAL, fy=-FOCAL, u0=U0, v0=V0, B=BASELINE_M):
    """(n,3) world points -> (n,3) (u, v, d) and an in-image mask (reference in-FOV test)."""
    R = rotation_terms(ext12[6:9])
    pc = (points - ext12[None, 0:3]) @ R.T
    x, y, z = pc[:, 0], pc[:, 1], pc[:, 2]
    with np.errstate(divide="ignore", invalid="ignore"):
        u = u0 - fx / z * x
        v = v0 - fy / z * y
        d = -fx * B / z
    ok = (u >= 0) & (u <= 2 * u0) & (v >= 0) & (v <= 2 * v0) & (d >= 0) & np.isfinite(d)
    return np.stack([u, v, d], axis=1), ok


@dataclass
class Scene:
    seed: int
    landmarks: np.ndarray            # (L, 3)
    cam2: np.ndarray                 # (frames, 12) camera-2 extrinsics per frame
    calib: np.ndarray                # (12,) calibration pose (frame-0 camera 2 state)
    frames: List[np.ndarray] = field(default_factory=list)   # per frame (n, 3) u, v, d
    fixed: List[bool] = field(default_factory=list)          # frame from the fixed camera
    clutter_rate: float = 10.0
    pd: float = 0.95

    @property
    def n_frames(self) -> int:
        return len(self.frames)


def make_scene(n_landmarks: int, n_frames: int, clutter_rate: float, seed: int, pd: float = 0.95,
               slam: bool = False, rng_box=(10.0, 10.0, 10.0), z_near: float = 2.0) -> Scene:
    """Seeded stereo calibration scene.  slam=True gives camera-2 frames only."""
    rng = np.random.default_rng(seed)
    bx, by, bz = rng_box
    lm = np.stack([rng.uniform(-bx / 2, bx / 2, n_landmarks),
                   rng.uniform(-by / 2, by / 2, n_landmarks),
                   rng.uniform(z_near, z_near + bz, n_landmarks)], axis=1)
    # calibration pose of camera 2: baseline offset along x plus small rotations
    calib = np.zeros(12)
    calib[0:3] = [BASELINE_M, 0.0, 0.0] + rng.normal(0, 0.02, 3)
    calib[6:9] = rng.normal(0, 0.02, 3)
    # smooth trajectory: sinusoidal drift of position and angles, with consistent velocities
    amp_p, amp_a = rng.uniform(0.05, 0.2, 3), rng.uniform(0.005, 0.02, 3)
    w_p, w_a = rng.uniform(0.02, 0.08, 3), rng.uniform(0.02, 0.08, 3)
    ph_p, ph_a = rng.uniform(0, 2 * np.pi, 3), rng.uniform(0, 2 * np.pi, 3)
    t = np.arange(n_frames) * DT
    cam2 = np.zeros((n_frames, 12))
    cam2[:, 0:3] = calib[0:3] + amp_p * (np.sin(w_p * t[:, None] + ph_p) - np.sin(ph_p))
    cam2[:, 3:6] = amp_p * w_p * np.cos(w_p * t[:, None] + ph_p)
    cam2[:, 6:9] = calib[6:9] + amp_a * (np.sin(w_a * t[:, None] + ph_a) - np.sin(ph_a))
    cam2[:, 9:12] = amp_a * w_a * np.cos(w_a * t[:, None] + ph_a)
    sc = Scene(seed=seed, landmarks=lm, cam2=cam2, calib=cam2[0].copy(),
               clutter_rate=clutter_rate, pd=pd)
    zero = np.zeros(12)
    for k in range(n_frames):
        fixed = (not slam) and (k % 2 == 0)
        e = zero if fixed else cam2[k]
        z, ok = project(lm, e)
        det = ok & (rng.uniform(size=n_landmarks) < pd)
        zt = z[det]
        zt = zt + rng.normal(0, 1, zt.shape) * np.array([SIGMA_UV, SIGMA_UV, SIGMA_D])
        nc = rng.poisson(clutter_rate)
        zc = np.stack([rng.uniform(0, IMG_W, nc), rng.uniform(0, IMG_H, nc),
                       rng.uniform(D_MIN, D_MAX, nc)], axis=1)
        zk = np.concatenate([zt, zc], axis=0)
        zk = zk[rng.permutation(zk.shape[0])]
        sc.frames.append(np.ascontiguousarray(zk))
        sc.fixed.append(fixed)
    return sc


def scene_seed(config_index: int, filter_index: int = 0) -> int:
    return SCENE_SEED_BASE + 1000 * config_index + filter_index


# ------------------------------------------------------------------ configurations
WORKLOADS = {
    # name: (parents, landmarks, clutter rate, max Gaussians/parent, frames, max measurements)
    "plain_c0": dict(n_parents=256, n_landmarks=50, clutter=10.0, max_gaussians=64, frames=100, max_meas=128,
                     max_survivors=384),
    "plain_c1": dict(n_parents=4096, n_landmarks=200, clutter=50.0, max_gaussians=256, frames=500, max_meas=384,
                     max_survivors=512),
    "precision_c3": dict(n_parents=16384, n_landmarks=400, clutter=100.0, max_gaussians=512, frames=300,
                         max_meas=768, max_survivors=1536),
}


def filter_config(n_parents: int, max_gaussians: int, max_meas: int, clutter_rate: float,
                  precision: int = 0, calib: Optional[np.ndarray] = None, seed: int = 1,
                  particles_per_feature: int = 100, meas_dim: int = 3):
    """scphd_config for a synthetic scene.  The model parameters are the rig's; the
    filter parameters (birth weight, thresholds, prior box) are this
    implementation's choices for these scenes: w0 = kappa / 10 so that a birth
    keeps a weight of order 1/(M/10+1) only for unexplained measurements, and
    min_weight = 1e-3."""
    from .scphd import ScphdConfig
    c = ScphdConfig()
    c.n_parents = n_parents
    c.particles_per_feature = particles_per_feature
    c.max_gaussians = max_gaussians
    c.max_measurements = max_meas
    c.meas_dim = meas_dim
    c.precision = precision
    c.max_survivors = 0
    c.device = 0
    c.seed = seed
    calib = np.zeros(12) if calib is None else calib
    half = np.array([0.3, 0.3, 0.3, 0.05, 0.05, 0.05, 0.05, 0.05, 0.05, 0.01, 0.01, 0.01])
    for i in range(12):
        c.prior_a[i] = calib[i] - half[i]
        c.prior_b[i] = calib[i] + half[i]
    for i, v in enumerate([0.05, 0.05, 0.05, 0.005, 0.005, 0.005]):
        c.cam_std[i] = v
    for i, v in enumerate([0.01, 0.01, 0.01]):
        c.feat_std[i] = v
    c.fx = c.fy = -FOCAL
    c.u0, c.v0 = U0, V0
    c.std_u = c.std_v = SIGMA_UV
    c.std_d = SIGMA_D
    c.pd = 0.95
    c.kappa = clutter_rate / (IMG_W * IMG_H * (D_MAX - D_MIN))
    c.baseline = BASELINE_M
    c.ps = 0.9
    c.min_weight = 1e-3
    c.min_separation = 6.0
    c.min_neff = 0.75
    c.w0 = c.kappa / 10.0
    c.d0 = 20.0
    c.vu0 = c.vv0 = c.vd0 = 0.0
    c.var_d0 = 100.0
    c.var_vu0 = c.var_vv0 = 6.0
    c.var_vd0 = 0.05
    return c


def workload(name: str, precision: int = 0, filter_index: int = 0, n_frames: Optional[int] = None):
    """(scene, config) for a named workload of WORKLOADS."""
    w = WORKLOADS[name]
    idx = {"plain_c0": 0, "plain_c1": 1, "precision_c3": 3}[name]
    sd = scene_seed(idx, filter_index)
    sc = make_scene(w["n_landmarks"], n_frames or w["frames"], w["clutter"], sd)
    cfg = filter_config(w["n_parents"], w["max_gaussians"], w["max_meas"], w["clutter"], precision,
                        calib=sc.calib, seed=sd)
    cfg.max_survivors = w["max_survivors"]
    return sc, cfg


# ------------------------------------------------------------------ many filters
def batched_specs(n_filters: int = 64, seed: int = SCENE_SEED_BASE + 2000):
    """Filters of the many-filter workload: parent counts log-uniform in [512, 8192],
    landmark counts uniform in [20, 400], clutter rates uniform in [5, 80], each with
    its own seeded scene and trajectory."""
    rng = np.random.default_rng(seed)
    specs = []
    for i in range(n_filters):
        n = int(round(float(np.exp(rng.uniform(np.log(512.0), np.log(8192.0))))))
        specs.append(dict(index=i, n_parents=n, n_landmarks=int(rng.integers(20, 401)),
                          clutter=float(rng.uniform(5.0, 80.0))))
    return specs


def spec_filter(spec: dict, n_frames: int, precision: int = 0, max_gaussians: int = 256, config_index: int = 2,
                survivors_per_gaussian: int = 3):
    """(scene, config) of one filter of a many-filter workload.  The measurement
    capacity is the scene's largest frame rounded up to 32."""
    sd = scene_seed(config_index, spec["index"])
    sc = make_scene(spec["n_landmarks"], n_frames, spec["clutter"], sd)
    mmax = max(int(z.shape[0]) for z in sc.frames) if sc.frames else 0
    mcap = max(32, (mmax + 8 + 31) // 32 * 32)
    cfg = filter_config(spec["n_parents"], max_gaussians, mcap, spec["clutter"], precision, calib=sc.calib, seed=sd)
    cfg.max_survivors = survivors_per_gaussian * max_gaussians
    return sc, cfg


def plan_waves(sizes, budget: int):
    """Greedy grouping of filters (in order) into device-resident waves whose summed
    device bytes stay within budget; a filter larger than the budget is refused."""
    waves, cur, used = [], [], 0
    for i, b in enumerate(sizes):
        if b > budget:
            raise ValueError(f"filter {i} needs {b} bytes, more than the budget {budget}")
        if used + b > budget and cur:
            waves.append(cur)
            cur, used = [], 0
        cur.append(i)
        used += b
    if cur:
        waves.append(cur)
    return waves


def serving_arrivals(rate: float = 20.0, seconds: float = 60.0, seed: int = SCENE_SEED_BASE + 4000):
    """Poisson arrivals of calibration jobs: (time, spec) with 100-1000 frames
    (uniform), 512-8192 parents (log-uniform), 20-400 landmarks, clutter 5-80."""
    rng = np.random.default_rng(seed)
    t, out, i = 0.0, [], 0
    while True:
        t += float(rng.exponential(1.0 / rate))
        if t >= seconds:
            return out
        out.append((t, dict(index=i, n_parents=int(round(float(np.exp(rng.uniform(np.log(512.0), np.log(8192.0)))))),
                            n_landmarks=int(rng.integers(20, 401)), clutter=float(rng.uniform(5.0, 80.0)),
                            n_frames=int(rng.integers(100, 1001)))))
        i += 1
