"""Launch-shape tuning (scphd_set_autotune / scphd_get_launch_shapes): a filter that
tunes its merge and likelihood launch shapes on its first updates must end in exactly
the state of the same filter run with the default shape."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision", [0, 1])
def test_tuned_shapes_leave_results_unchanged(pkg, precision):
    if not gpu_available():
        pytest.skip("no CUDA device")
    sc = pkg.scene.make_scene(n_landmarks=30, n_frames=12, clutter_rate=8.0, seed=pkg.scene.scene_seed(6, 0))
    cfg = pkg.scene.filter_config(n_parents=96, max_gaussians=128, max_meas=96, clutter_rate=8.0,
                                  precision=precision, calib=sc.calib, seed=61, particles_per_feature=40)
    tuned, plain = pkg.SCPHDCameraCalibration(cfg), pkg.SCPHDCameraCalibration(cfg)
    plain.set_autotune(False)
    assert plain.launch_shapes() == {"merge_threads": 256, "likelihood_full": True, "tuned": True}
    assert not tuned.launch_shapes()["tuned"]
    for k, z in enumerate(sc.frames):
        for f in (tuned, plain):
            f.step(pkg.scene.DT, z[:, 0], z[:, 1], fixed_camera=sc.fixed[k], d=z[:, 2])
        st_a, lw_a = tuned.particles()
        st_b, lw_b = plain.particles()
        assert np.array_equal(st_a, st_b) and np.array_equal(lw_a, lw_b), f"frame {k}"
        assert np.array_equal(tuned.map_sizes(), plain.map_sizes()), f"frame {k} map sizes"
        for p in range(0, cfg.n_parents, 7):
            assert np.array_equal(tuned.mixture(1, p), plain.mixture(1, p)), f"frame {k} parent {p}"
    s = tuned.launch_shapes()
    assert s["tuned"] and s["merge_threads"] in (128, 256)
