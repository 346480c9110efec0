"""The command-line driver and the result writer on the GPU: scphd_calibrate runs the
reference driver's loop on the reference fixture's first frames, and every file it
writes (prior.mat, k.mat) must hold exactly the state of the same filter stepped
through the library from Python with the same configuration and frames."""
import os
import subprocess

import numpy as np
import pytest
import scipy.io as sio

from conftest import gpu_available
from test_io import CLI, REFERENCE_STYLE, _cells, _fixture_frames

pytestmark = pytest.mark.gpu

SMALL = (REFERENCE_STYLE.replace("n_particles = 100 ; particles_per_feature = 100",
                                 "n_particles = 24 ; particles_per_feature = 32")
         .replace("max_steps = 100", "max_steps = 5")
         .replace("save_all_maps = false", "save_all_maps = true")
         + "\nmax_gaussians = 64\nmax_measurements = 64\nseed = 4242\nprecision = \"fp64\"\n")


def _need_gpu():
    if not gpu_available():
        pytest.skip("no CUDA device")


def _check_file(m, f, k_label):
    st, lw = f.particles()
    assert np.array_equal(m["particles"], st.T), f"{k_label}: particles"
    assert np.array_equal(m["log_weights"][:, 0], lw), f"{k_label}: log-weights"
    w = np.exp(lw - lw.max())
    np.testing.assert_allclose(m["weights"][:, 0], w / w.sum(), rtol=1e-15, atol=0, err_msg=k_label)
    pmap = int(np.argmax(lw))
    feat = m["features"][0, 0]
    mw = f.map_weights(pmap)
    if len(mw):
        assert np.array_equal(feat["weights"][:, 0], mw), f"{k_label}: MAP map weights"
        xyz, _ = f.map_clouds(pmap)
        P = xyz.shape[2]
        parts = feat["particles"]
        assert parts.shape == (6, len(mw) * P)
        assert np.array_equal(parts.reshape(6, len(mw), P).transpose(1, 0, 2), xyz), f"{k_label}: MAP clouds"
    else:
        assert feat["weights"].size == 0


def test_driver_files_equal_the_library_state(pkg, tmp_path):
    _need_gpu()
    z1, z2 = _fixture_frames()
    data = str(tmp_path / "sim.mat")
    sio.savemat(data, {"Z1": _cells(z1), "Z2": _cells(z2)}, do_compression=True)
    cfg_path = tmp_path / "small.cfg"
    cfg_path.write_text(SMALL)
    out = tmp_path / "out"
    out.mkdir()
    run = subprocess.run([CLI, str(cfg_path), data, "--out", str(out), "--quiet"], capture_output=True, text=True,
                         timeout=600)
    assert run.returncode == 0, run.stderr
    cfg, opts = pkg.config_from_file(str(cfg_path))
    assert opts["max_steps"] == 5 and opts["save_all_maps"]
    f = pkg.SCPHDCameraCalibration(cfg)
    _check_file(sio.loadmat(str(out / "prior.mat")), f, "prior")
    for k in range(5):
        f.predict(0.5)
        z, fixed = (z1[k], True) if k % 2 == 0 else (z2[k], False)
        f.update(z[0], z[1], fixed_camera=fixed)
        m = sio.loadmat(str(out / f"{k}.mat"))
        _check_file(m, f, f"frame {k}")
        for p in range(0, cfg.n_parents, 5):
            for key, which, off in (("features_predicted", pkg.SCPHD_MIX_FITTED, 2),
                                    ("features_merged", pkg.SCPHD_MIX_MERGED, 1)):
                rows = f.mixture(which, p)
                e = m[key][p, 0]
                n = len(rows)
                assert e["weights"].shape == (1, n) and np.array_equal(e["weights"][0], rows[:, 0])
                if n:
                    assert np.array_equal(e["means"], rows[:, off:off + 6].T)
                    full = e["covs"].reshape(6, 6, n)
                    tri = [(a, c) for a in range(6) for c in range(a + 1)]
                    for q, (a, c) in enumerate(tri):
                        assert np.array_equal(full[a, c], rows[:, off + 6 + q])
                        assert np.array_equal(full[c, a], rows[:, off + 6 + q])
        assert m["features_updated"].size == 0
        f.checkStuff()
        f.resample()
    f.close()
