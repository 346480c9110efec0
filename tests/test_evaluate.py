"""Evaluation metrics (OSPA, calibration error, MAP map) and their use on the oracle."""
import numpy as np
import pytest


def test_ospa_properties(pkg):
    ospa = pkg.evaluate.ospa
    X = np.array([[0.0, 0, 0], [10, 0, 0]])
    assert ospa(X, X)[0] == 0.0
    # one missing object: cardinality penalty c per unmatched point, p = 1
    d, loc, card = ospa(X[:1], X, c=10.0, p=1.0)
    assert d == pytest.approx(5.0) and loc == 0.0 and card == pytest.approx(5.0)
    # localisation error below the cut-off
    d, loc, card = ospa(X + [1.0, 0, 0], X, c=10.0)
    assert d == pytest.approx(1.0) and card == 0.0
    # symmetric, cut off at c, empty sets
    Y = np.array([[100.0, 0, 0]])
    assert ospa(X, Y)[0] == pytest.approx(ospa(Y, X)[0])
    assert ospa(Y, X[:1])[0] == pytest.approx(10.0)
    assert ospa(np.zeros((0, 3)), np.zeros((0, 3)))[0] == 0.0
    assert ospa(np.zeros((0, 3)), X)[0] == 10.0


def test_calibration_error_of_weighted_mean(pkg):
    st = np.zeros((4, 12))
    st[:, 0] = [1, 2, 3, 4]
    lw = np.log(np.array([0.1, 0.2, 0.3, 0.4]))
    e = pkg.evaluate.calibration_error(st, lw, np.zeros(12))
    assert e["position_m"] == pytest.approx(3.0)


def test_calibration_angle_error_wraps(pkg, orc):
    """Angles either side of +-pi: the truth at 3.1 rad and an estimate at -3.1 rad are
    0.083 rad apart, not 6.2; the circular mean of parents at +3.13 and -3.13 is pi."""
    ev = pkg.evaluate
    st = np.zeros((1, 12))
    st[0, 6:9] = [-3.1, 0.2, -3.1]
    truth = np.zeros(12)
    truth[6:9] = [3.1, 0.2, 3.1]
    e = ev.calibration_error(st, np.zeros(1), truth)
    gap = 2 * np.pi - 6.2
    assert e["angle_rad"] == pytest.approx(np.sqrt(2) * gap, rel=1e-12)
    assert e["components"][3] == pytest.approx(gap, rel=1e-12)
    st = np.zeros((2, 12))
    st[:, 6] = [3.13, -3.13]
    pose = ev.expected_pose(st, np.log([0.5, 0.5]))
    assert abs(ev.wrap_angle(pose[6] - np.pi)) < 1e-12
    # the wrap agrees with the oracle's restatement of wrapAngle
    for a in np.linspace(-20, 20, 101):
        assert ev.wrap_angle(a) == pytest.approx(orc.wrap_angle(a), abs=1e-15)


def test_metrics_on_an_oracle_run(pkg, orc):
    """A few dozen frames of a small scene through the oracle: the MAP map is populated,
    OSPA lies in [0, c] and the calibration error is finite.  (How well the filter as
    written calibrates on a given scene is not asserted.)"""
    sc = pkg.scene.make_scene(n_landmarks=15, n_frames=24, clutter_rate=2.0, seed=pkg.scene.scene_seed(0, 3))
    cfg = pkg.scene.filter_config(64, 128, 64, 2.0, precision=1, calib=sc.calib, seed=3, particles_per_feature=32)
    o = orc.Oracle(cfg)
    for k in range(sc.n_frames):
        z = sc.frames[k]
        o.predict(pkg.scene.DT)
        o.update(z[:, 0], z[:, 1], sc.fixed[k], d=z[:, 2])
        o.resample()
    st, lw = o.particles()
    m = pkg.evaluate.frame_metrics(st, lw, lambda p: o.map(p)[0], lambda p: o.map(p)[1], sc, sc.n_frames - 1)
    assert m["n_features"] > 5
    assert 0 <= m["ospa"] <= 10.0 and m["ospa"] == pytest.approx(m["ospa_loc"] + m["ospa_card"], abs=1e-9)
    assert np.isfinite(m["calib_position_m"]) and np.isfinite(m["calib_angle_rad"])
