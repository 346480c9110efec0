"""Filter evaluation: calibration error and OSPA of the MAP map.

Restates the reference's offline scoring (load_disparity_results.m,
compute_disparity_error.m; its MATLAB helpers `ospa_dist` and `weightedcov` are not
in the reference tree, so OSPA follows its published definition, Schuhmacher, Vo
and Vo, "A consistent metric for performance evaluation of multi-object filters",
IEEE TSP 2008):

* expected pose = weighted mean of the parent states (load_disparity_results.m:24-26),
  the three angles as circular means (atan2 of the weighted sine and cosine sums, so
  that parents either side of +-pi average to +-pi, not to 0); calibration error =
  expected pose - true pose on the position (x,y,z) and angle (theta, phi, psi)
  components (:66), each angle difference wrapped into [-pi, pi] as the reference's
  wrapAngle does (src/device_math.cu:308-318);
* the map of the MAP parent keeps the features of weight >= 0.33 (:31), cardinality =
  sum of weights (:32); each feature's sample cloud is projected into camera 1 and
  summarised by its mean (u, v, d) (:36-52);
* OSPA between those means and the true landmarks in camera 1's view, cut-off c = 10,
  order p = 1, Euclidean on (u, v, d) (compute_disparity_error.m:89-97).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Optional

import numpy as np

from .scene import project


def ospa(X: np.ndarray, Y: np.ndarray, c: float = 10.0, p: float = 1.0):
    """OSPA distance between point sets X (m, d) and Y (n, d); returns
    (distance, localisation part, cardinality part)."""
    from scipy.optimize import linear_sum_assignment
    X = np.asarray(X, float).reshape(-1, X.shape[-1] if np.ndim(X) > 1 else 1) if len(X) else np.zeros((0, 3))
    Y = np.asarray(Y, float).reshape(-1, Y.shape[-1] if np.ndim(Y) > 1 else 1) if len(Y) else np.zeros((0, 3))
    m, n = len(X), len(Y)
    if m == 0 and n == 0:
        return 0.0, 0.0, 0.0
    if m == 0 or n == 0:
        return float(c), 0.0, float(c)
    if m > n:
        X, Y, m, n = Y, X, n, m
    D = np.linalg.norm(X[:, None, :] - Y[None, :, :], axis=2)
    D = np.minimum(D, c) ** p
    r, col = linear_sum_assignment(D)
    loc = D[r, col].sum()
    card = (c ** p) * (n - m)
    dist = ((loc + card) / n) ** (1.0 / p)
    return float(dist), float((loc / n) ** (1.0 / p)), float((card / n) ** (1.0 / p))


ANGLES = slice(6, 9)   # theta, phi, psi of a 12-D parent state


def wrap_angle(a):
    """Angle(s) into [-pi, pi], as wrapAngle (src/device_math.cu:308-318): the
    remainder of a / 2pi (sign of a), moved by 2pi when beyond pi."""
    r = np.fmod(np.asarray(a, float), 2 * np.pi)
    r = np.where(r > np.pi, r - 2 * np.pi, r)
    return np.where(r < -np.pi, r + 2 * np.pi, r)


def expected_pose(states: np.ndarray, log_weights: np.ndarray) -> np.ndarray:
    """Weighted mean of the parent states; the angles as weighted circular means."""
    w = np.exp(log_weights - np.max(log_weights))
    w /= w.sum()
    mean = (w[:, None] * states).sum(axis=0)
    ang = states[:, ANGLES]
    mean[ANGLES] = np.arctan2((w[:, None] * np.sin(ang)).sum(axis=0), (w[:, None] * np.cos(ang)).sum(axis=0))
    return mean


def calibration_error(states: np.ndarray, log_weights: np.ndarray, truth12: np.ndarray):
    e = expected_pose(states, log_weights) - truth12
    e[ANGLES] = wrap_angle(e[ANGLES])
    return {"position_m": float(np.linalg.norm(e[0:3])), "angle_rad": float(np.linalg.norm(e[ANGLES])),
            "components": e[[0, 1, 2, 6, 7, 8]].tolist()}


@dataclass
class MapEstimate:
    positions: np.ndarray      # (n, 3) world means of the kept features
    disparity: np.ndarray      # (n, 3) mean (u, v, d) in camera 1
    cardinality: float         # sum of all feature weights


def map_estimate(weights: np.ndarray, clouds: np.ndarray, min_weight: float = 0.33,
                 cam1: Optional[np.ndarray] = None) -> MapEstimate:
    """weights (G,), clouds (G, 6, P) world samples of one parent's map."""
    cam1 = np.zeros(12) if cam1 is None else cam1
    keep = weights >= min_weight
    pos = clouds[keep, 0:3, :].mean(axis=2) if keep.any() else np.zeros((0, 3))
    disp = []
    for g in np.where(keep)[0]:
        z, _ = project(clouds[g, 0:3, :].T, cam1)
        disp.append(z.mean(axis=0))
    return MapEstimate(pos, np.array(disp).reshape(-1, 3), float(weights.sum()))


def truth_disparity(landmarks: np.ndarray, cam1: Optional[np.ndarray] = None) -> np.ndarray:
    z, ok = project(landmarks, np.zeros(12) if cam1 is None else cam1)
    return z[ok]


def frame_metrics(states, log_weights, map_weights_of, map_clouds_of, scene, k: int):
    """Metrics of frame k for a filter exposing its MAP parent's map through the two
    callables (parent -> weights, parent -> clouds)."""
    pmap = int(np.argmax(log_weights))
    est = map_estimate(map_weights_of(pmap), map_clouds_of(pmap))
    d, loc, card = ospa(est.disparity, truth_disparity(scene.landmarks))
    cal = calibration_error(states, log_weights, scene.cam2[k])
    return {"ospa": d, "ospa_loc": loc, "ospa_card": card, "n_features": int(len(est.disparity)),
            "cardinality": est.cardinality, "calib_position_m": cal["position_m"],
            "calib_angle_rad": cal["angle_rad"], "map_parent": pmap}
