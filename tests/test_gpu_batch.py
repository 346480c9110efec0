"""Batched steps (scphd_batch_*) against the same filters stepped one at a time.

A batched step runs predict + update + resample for every member with one launch
per stage; each member must end in exactly the state it reaches alone (same
kernels' arithmetic, same random streams), so the comparison is bit-exact.
"""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu


def _need_gpu():
    if not gpu_available():
        pytest.skip("no CUDA device")


def _members(pkg, precision, meas_dim=3):
    """Three filters of different sizes on different scenes."""
    out = []
    for i, (n, g, m) in enumerate([(48, 96, 64), (130, 160, 96), (7, 64, 48)]):
        sc = pkg.scene.make_scene(n_landmarks=12 + 4 * i, n_frames=6, clutter_rate=3.0,
                                  seed=pkg.scene.scene_seed(5, i))
        cfg = pkg.scene.filter_config(n_parents=n, max_gaussians=g, max_meas=m, clutter_rate=3.0,
                                      precision=precision, calib=sc.calib, seed=100 + i,
                                      particles_per_feature=40 + 10 * i, meas_dim=meas_dim)
        out.append((sc, cfg))
    return out


def _frame(sc, k, i, meas_dim):
    z = sc.frames[k]
    if i == 2 and k == 3:   # one member sees an empty frame
        z = z[:0]
    return z[:, 0], z[:, 1], (z[:, 2] if meas_dim == 3 else None), sc.fixed[k]


def _state(f):
    st, lw = f.particles()
    sizes = f.map_sizes()
    mix = [f.mixture(1, p) for p in range(0, f.n_parents, 5)]
    return st, lw, sizes, mix, f.resample_indices()


def _assert_same(a, b, what):
    for x, y, name in zip(a[:3], b[:3], ("states", "log-weights", "map sizes")):
        assert np.array_equal(x, y), f"{what}: {name} differ"
    for j, (x, y) in enumerate(zip(a[3], b[3])):
        assert x.shape == y.shape and np.array_equal(x, y), f"{what}: merged mixture {j} differs"
    assert np.array_equal(a[4], b[4]), f"{what}: resampling indices differ"


DIAG = 7 + np.array([0, 2, 5, 9, 14, 20])   # packed diagonal of a merged row's covariance


def _assert_close(a, b, what):
    """FP32 rounding: map sizes and resampling indices exact; values to 1e-4 in their own
    scale (the tolerance tier of the FP32 tests): weights relative, means per standard
    deviation, covariance entries per sqrt(S_aa S_bb), so that an off-diagonal entry small
    beside its variances is not held to a relative bound."""
    assert np.array_equal(a[2], b[2]), f"{what}: map sizes differ"
    np.testing.assert_allclose(a[0], b[0], rtol=1e-9, atol=1e-9, err_msg=f"{what}: states")
    np.testing.assert_allclose(a[1], b[1], rtol=1e-4, atol=1e-4, err_msg=f"{what}: log-weights")
    for j, (x, y) in enumerate(zip(a[3], b[3])):
        assert x.shape == y.shape, f"{what}: merged mixture {j} count"
        # weights equal to FP32 rounding may list two components in the other order
        x, y = x[np.argsort(x[:, 1], kind="stable")], y[np.argsort(y[:, 1], kind="stable")]
        np.testing.assert_allclose(x[:, 0], y[:, 0], rtol=1e-4, atol=1e-9, err_msg=f"{what}: merged weights {j}")
        sd = np.sqrt(np.maximum(y[:, DIAG], 1e-30))
        m_err = np.abs(x[:, 1:7] - y[:, 1:7]) / np.maximum(sd, 1e-12)
        assert (m_err <= 1e-4).all(), f"{what}: merged means {j}, {m_err.max():.2e} SD"
        for aa in range(6):
            for bb in range(aa + 1):
                e = 7 + aa * (aa + 1) // 2 + bb
                c_err = np.abs(x[:, e] - y[:, e]) / np.maximum(sd[:, aa] * sd[:, bb], 1e-30)
                assert (c_err <= 1e-4).all(), f"{what}: merged covariance ({aa},{bb}) {j}, {c_err.max():.2e}"
    assert np.array_equal(a[4], b[4]), f"{what}: resampling indices differ"


@pytest.mark.parametrize("fused", [0, 1])
@pytest.mark.parametrize("use_graph", [False, True])
@pytest.mark.parametrize("precision", [1, 0])
def test_batch_matches_filters_alone(pkg, use_graph, precision, fused):
    """fused: the batch's update path (0 stage kernels, 1 fused kernel); the filters
    alone run the stage kernels.  The FP32 fused batch equals them to FP32 rounding only
    (its build may contract multiply-adds differently, and later frames then part at
    thresholds): it is compared on its first three frames, map sizes exactly and values
    to 1e-4; every other case bit for bit over all frames."""
    _need_gpu()
    approx = bool(fused) and precision == 0
    meas_dim = 3
    members = _members(pkg, precision, meas_dim)
    alone = [pkg.SCPHDCameraCalibration(cfg) for _, cfg in members]
    for f in alone:
        f.set_fused(0)
    batched = [pkg.SCPHDCameraCalibration(cfg) for _, cfg in members]
    batch = pkg.SCPHDBatch(batched, use_graph=use_graph)
    batch.set_fused(fused)
    assert batch.fused() == bool(fused)
    for k in range(3 if approx else 5):
        frames = [_frame(sc, k, i, meas_dim) for i, (sc, _) in enumerate(members)]
        for f, (u, v, d, fixed) in zip(alone, frames):
            f.predict(0.5)
            f.update(u, v, fixed_camera=fixed, d=d)
            f.resample()
        batch.step(0.5, frames)
        for i, (fa, fb) in enumerate(zip(alone, batched)):
            (_assert_close if approx else _assert_same)(_state(fa), _state(fb), f"frame {k} member {i}")
    batch.close()
    if approx:
        return
    # members keep working on their own after the batch is gone
    for f, (sc, _) in zip(alone + batched, members + members):
        z = sc.frames[5]
        f.step(0.5, z[:, 0], z[:, 1], fixed_camera=sc.fixed[5], d=z[:, 2])
    for i in range(3):
        _assert_same(_state(alone[i]), _state(batched[i]), f"after batch member {i}")


@pytest.mark.parametrize("use_graph", [False, True])
def test_batch_steps_back_to_back(pkg, use_graph):
    """Host-frame batch steps queued without waiting in between: a step refills the
    page-locked frame buffers once the previous step's copies are done, while its kernels
    may still run, so every member must still end where it gets alone."""
    _need_gpu()
    members = _members(pkg, 1)
    alone = [pkg.SCPHDCameraCalibration(cfg) for _, cfg in members]
    batched = [pkg.SCPHDCameraCalibration(cfg) for _, cfg in members]
    batch = pkg.SCPHDBatch(batched, use_graph=use_graph)
    for k in range(6):
        frames = [_frame(sc, k, i, 3) for i, (sc, _) in enumerate(members)]
        for f, (u, v, d, fixed) in zip(alone, frames):
            f.step(0.5, u, v, fixed_camera=fixed, d=d)
        batch.step(0.5, [(np.ascontiguousarray(u), np.ascontiguousarray(v), np.ascontiguousarray(d), fixed)
                         for u, v, d, fixed in frames])
    batch.synchronize()
    for i in range(3):
        _assert_same(_state(alone[i]), _state(batched[i]), f"member {i}")
    batch.close()


def test_batch_two_dim_and_device_frames(pkg):
    _need_gpu()
    import torch
    meas_dim = 2
    members = _members(pkg, 1, meas_dim)
    alone = [pkg.SCPHDCameraCalibration(cfg) for _, cfg in members]
    batched = [pkg.SCPHDCameraCalibration(cfg) for _, cfg in members]
    batch = pkg.SCPHDBatch(batched, use_graph=True)
    for k in range(4):
        frames = [_frame(sc, k, i, meas_dim) for i, (sc, _) in enumerate(members)]
        dev = []
        for f, (u, v, d, fixed) in zip(alone, frames):
            f.step(0.5, u, v, fixed_camera=fixed)
            tu = torch.tensor(np.asarray(u, np.float64), device="cuda")
            tv = torch.tensor(np.asarray(v, np.float64), device="cuda")
            dev.append((tu, tv, fixed))
        torch.cuda.synchronize()
        batch.step_device(0.5, [(tu.data_ptr(), tv.data_ptr(), None, tu.numel(), fixed) for tu, tv, fixed in dev])
        batch.synchronize()
        for i, (fa, fb) in enumerate(zip(alone, batched)):
            _assert_same(_state(fa), _state(fb), f"frame {k} member {i}")
    batch.close()


def test_batch_predict_outside_the_batch(pkg):
    """A predict() issued on a member between batched steps is applied before the
    next batched step, as predict(); predict() would be alone."""
    _need_gpu()
    members = _members(pkg, 1)
    alone = [pkg.SCPHDCameraCalibration(cfg) for _, cfg in members]
    batched = [pkg.SCPHDCameraCalibration(cfg) for _, cfg in members]
    batch = pkg.SCPHDBatch(batched)
    frames0 = [_frame(sc, 0, i, 3) for i, (sc, _) in enumerate(members)]
    frames1 = [_frame(sc, 1, i, 3) for i, (sc, _) in enumerate(members)]
    for f, (u, v, d, fixed) in zip(alone, frames0):
        f.step(0.5, u, v, fixed_camera=fixed, d=d)
    batch.step(0.5, frames0)
    alone[1].predict(0.25)
    batched[1].predict(0.25)
    for f, (u, v, d, fixed) in zip(alone, frames1):
        f.step(0.5, u, v, fixed_camera=fixed, d=d)
    batch.step(0.5, frames1)
    for i in range(3):
        _assert_same(_state(alone[i]), _state(batched[i]), f"member {i}")
    batch.close()


def test_batch_argument_errors(pkg):
    _need_gpu()
    members = _members(pkg, 1)
    fs = [pkg.SCPHDCameraCalibration(cfg) for _, cfg in members]
    with pytest.raises(pkg.ScphdError):
        pkg.SCPHDBatch([fs[0], fs[0]])              # listed twice
    other = members[0][1].copy()
    other.precision = 0
    with pytest.raises(pkg.ScphdError):
        pkg.SCPHDBatch([fs[0], pkg.SCPHDCameraCalibration(other)])   # mixed precision
    b = pkg.SCPHDBatch(fs)
    with pytest.raises(pkg.ScphdError):
        pkg.SCPHDBatch([fs[1]])                     # already in a batch
    sc = members[0][0]
    big = np.zeros(1000)
    frames = [_frame(sc, 0, 0, 3)] * 2 + [(big, big, big, False)]
    with pytest.raises(pkg.ScphdError):
        b.step(0.5, frames)                         # over max_measurements
    with pytest.raises(pkg.ScphdError):
        fs[0].close()                               # destroy while batched is refused
    b.close()


def test_filters_of_different_sizes_in_one_process(pkg):
    """A filter created after a larger one must not lower the larger one's merge
    launch limits (the dynamic shared-memory limit is per kernel, not per filter)."""
    _need_gpu()
    members = _members(pkg, 0)
    big = pkg.SCPHDCameraCalibration(members[1][1])
    small = pkg.SCPHDCameraCalibration(members[2][1])
    for k in range(2):
        for f, (sc, _) in ((big, members[1]), (small, members[2])):
            z = sc.frames[k]
            f.step(0.5, z[:, 0], z[:, 1], fixed_camera=sc.fixed[k], d=z[:, 2])
    big.checkStuff()
    small.checkStuff()
