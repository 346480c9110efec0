"""scphd_get_particles_async: parent states and log-weights copied on the filter's stream
into page-locked buffers, read one step later while the next step runs, equal what the
synchronous scphd_get_particles returns for a twin filter stepped the same way."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, 1])
def test_async_particles_equal_synchronous(pkg, precision):
    if not gpu_available():
        pytest.skip("no CUDA device")
    import torch
    sc = pkg.scene.make_scene(n_landmarks=20, n_frames=8, clutter_rate=5.0, seed=pkg.scene.scene_seed(9, 1))
    cfg = pkg.scene.filter_config(n_parents=64, max_gaussians=96, max_meas=96, clutter_rate=5.0,
                                  precision=precision, calib=sc.calib, seed=91, particles_per_feature=100)
    f, twin = pkg.SCPHDCameraCalibration(cfg), pkg.SCPHDCameraCalibration(cfg)
    stream = torch.cuda.ExternalStream(f.stream_handle)
    n = cfg.n_parents
    bufs = [(torch.full((n, 12), np.nan, dtype=torch.float64, pin_memory=True),
             torch.full((n,), np.nan, dtype=torch.float64, pin_memory=True)) for _ in range(2)]
    evs = [torch.cuda.Event(), torch.cuda.Event()]
    expect = []
    for k, z in enumerate(sc.frames):
        for g in (f, twin):
            g.step(pkg.scene.DT, z[:, 0], z[:, 1], fixed_camera=sc.fixed[k], d=z[:, 2])
        st, lw = bufs[k % 2]
        f.particles_async(st.data_ptr(), lw.data_ptr())
        evs[k % 2].record(stream)
        expect.append(twin.particles())
        if k > 0:   # the previous step's buffers, read while this step may still run
            evs[(k - 1) % 2].synchronize()
            st_p, lw_p = bufs[(k - 1) % 2]
            assert np.array_equal(st_p.numpy(), expect[k - 1][0]), f"step {k - 1} states"
            assert np.array_equal(lw_p.numpy(), expect[k - 1][1]), f"step {k - 1} log-weights"
    last = len(sc.frames) - 1
    evs[last % 2].synchronize()
    assert np.array_equal(bufs[last % 2][0].numpy(), expect[last][0])
    assert np.array_equal(bufs[last % 2][1].numpy(), expect[last][1])
    f.close()
    twin.close()
