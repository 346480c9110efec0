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
    assert plain.launch_shapes() == {"merge_threads": 256, "likelihood_full": True, "tuned": True, "fused": False,
                                     "fit_blocks_per_parent": 1, "fit_tuned": True}
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
    # the cloud-fit split is tuned on the updates after the first 16: not yet here
    assert not s["fit_tuned"] and s["fit_blocks_per_parent"] == 1
    for k in range(12):   # updates 17-22 tune it (collected at the next update), results unchanged
        z = sc.frames[k % sc.n_frames]
        for f in (tuned, plain):
            f.step(pkg.scene.DT, z[:, 0], z[:, 1], fixed_camera=sc.fixed[k % sc.n_frames], d=z[:, 2])
        st_a, lw_a = tuned.particles()
        st_b, lw_b = plain.particles()
        assert np.array_equal(st_a, st_b) and np.array_equal(lw_a, lw_b), f"extra frame {k}"
        for p in range(0, cfg.n_parents, 7):
            assert np.array_equal(tuned.mixture(0, p), plain.mixture(0, p)), f"extra frame {k} parent {p}"
    s = tuned.launch_shapes()
    assert s["fit_tuned"] and s["fit_blocks_per_parent"] in (1, 2, 4)


@pytest.mark.parametrize("precision", [0, 1])
def test_fit_split_leaves_results_unchanged(pkg, precision):
    """The cloud fit with 1, 2 and 4 blocks per parent (the parent's Gaussians dealt out
    over 8, 16 or 32 warps) gives identical states, maps and mixtures: at 100 samples per
    feature (the specialised kernel, tail pass of 4 samples x 8 Gaussians), 72 (tail of
    8 samples x 4 Gaussians) and 50 (no tail pass)."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    for P in (100, 72, 50):
        sc = pkg.scene.make_scene(n_landmarks=40, n_frames=6, clutter_rate=10.0, seed=pkg.scene.scene_seed(6, P))
        cfg = pkg.scene.filter_config(n_parents=48, max_gaussians=96, max_meas=128, clutter_rate=10.0,
                                      precision=precision, calib=sc.calib, seed=P, particles_per_feature=P)
        fs = [pkg.SCPHDCameraCalibration(cfg) for _ in range(3)]
        for f, split in zip(fs, (1, 2, 4)):
            f.set_fit_split(split)
            assert f.launch_shapes()["fit_blocks_per_parent"] == split
        for k, z in enumerate(sc.frames):
            for f in fs:
                f.predict(pkg.scene.DT)
                f.update(z[:, 0], z[:, 1], fixed_camera=sc.fixed[k], d=z[:, 2])
            ref = fs[0]
            st0, lw0 = ref.particles()
            for f in fs[1:]:
                st, lw = f.particles()
                assert np.array_equal(st, st0) and np.array_equal(lw, lw0), f"P {P} frame {k}"
                assert np.array_equal(f.map_sizes(), ref.map_sizes()), f"P {P} frame {k} map sizes"
                assert np.array_equal(f.counters(), ref.counters()), f"P {P} frame {k} counters"
                for p in range(cfg.n_parents):
                    assert np.array_equal(f.mixture(0, p), ref.mixture(0, p)), f"P {P} frame {k} parent {p} fitted"
                    assert np.array_equal(f.mixture(1, p), ref.mixture(1, p)), f"P {P} frame {k} parent {p} merged"
                    assert np.array_equal(f.map_weights(p), ref.map_weights(p)), f"P {P} frame {k} parent {p} map"
            for f in fs:
                f.resample()
        for f in fs:
            f.close()


@pytest.mark.parametrize("precision", [0, 1])
def test_fused_update_equals_stage_kernels(pkg, precision):
    """The fused update (one launch: cloud fit, Kalman terms, likelihood and merge of
    every parent) and the stage kernels give the same states, maps and mixtures -- in
    FP64 bit for bit; in FP32 to FP32 rounding on the first frames (the two builds may
    contract multiply-adds differently, and later frames then part at thresholds) --
    on a scene whose maps reach the capacity and with more measurements than a fused
    block has threads (two likelihood passes per parent)."""
    if not gpu_available():
        pytest.skip("no CUDA device")
    sc = pkg.scene.make_scene(n_landmarks=420, n_frames=8, clutter_rate=90.0, seed=pkg.scene.scene_seed(6, 1))
    cfg = pkg.scene.filter_config(n_parents=72, max_gaussians=96, max_meas=384, clutter_rate=90.0,
                                  precision=precision, calib=sc.calib, seed=62, particles_per_feature=50)
    fused, staged = pkg.SCPHDCameraCalibration(cfg), pkg.SCPHDCameraCalibration(cfg)
    fused.set_fused(1)
    staged.set_fused(0)
    assert fused.launch_shapes()["fused"] and not staged.launch_shapes()["fused"]
    exact = precision == 1
    same = (lambda a, b: np.array_equal(a, b)) if exact else \
        (lambda a, b: a.shape == b.shape and np.allclose(a, b, rtol=1e-4, atol=1e-6))
    big = False
    n_frames = len(sc.frames) if exact else 3
    for k, z in enumerate(sc.frames[:n_frames]):
        big |= z.shape[0] > 256
        for f in (fused, staged):
            f.step(pkg.scene.DT, z[:, 0], z[:, 1], fixed_camera=sc.fixed[k], d=z[:, 2])
        st_a, lw_a = fused.particles()
        st_b, lw_b = staged.particles()
        assert same(st_a, st_b) and same(lw_a, lw_b), f"frame {k}"
        assert np.array_equal(fused.map_sizes(), staged.map_sizes()), f"frame {k} map sizes"
        for p in range(0, cfg.n_parents, 5):
            assert same(fused.mixture(1, p), staged.mixture(1, p)), f"frame {k} parent {p} merged"
            assert same(fused.mixture(0, p), staged.mixture(0, p)), f"frame {k} parent {p} fitted"
            assert same(fused.map_weights(p), staged.map_weights(p)), f"frame {k} parent {p} map"
        e_a, l_a = fused.normalizers(z.shape[0])
        e_b, l_b = staged.normalizers(z.shape[0])
        assert same(e_a, e_b) and same(l_a, l_b), f"frame {k} normalisers"
    assert big, "no frame had more measurements than a fused block's threads"
    if exact:
        assert np.array_equal(fused.counters()[[0, 2, 3, 4, 5, 6, 7, 11]],
                              staged.counters()[[0, 2, 3, 4, 5, 6, 7, 11]])
        assert fused.counters()[0] > 0, "the map capacity never bound"
