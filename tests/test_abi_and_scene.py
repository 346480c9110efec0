"""C-ABI surface (no device calls), config layout, scene generator, and the
host-side replica plan used for multi-GPU runs (gloo, world size 2)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol(pkg):
    hdr = open(os.path.join(ROOT, "include", "scphd.h")).read()
    names = sorted(set(re.findall(r"\b(scphd_[a-z_0-9]+)\s*\(", hdr)))
    assert len(names) >= 20
    lib = pkg.load_library()
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_config_layout_matches_header_defaults(pkg):
    lib = pkg.load_library()
    c = pkg.ScphdConfig()
    lib.scphd_config_defaults(ctypes.byref(c))
    r = pkg.reference_defaults()
    for name, _ in pkg.ScphdConfig._fields_:
        a, b = getattr(c, name), getattr(r, name)
        if isinstance(a, ctypes.Array):
            assert list(a) == pytest.approx(list(b)), name
        elif name not in ("max_measurements",):
            assert a == pytest.approx(b), name


def test_create_without_device_fails_loudly(pkg):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("device present")
    except Exception:
        pass
    with pytest.raises(pkg.ScphdError) as e:
        pkg.SCPHDCameraCalibration(pkg.reference_defaults())
    assert e.value.status in (2, 5)


def test_scene_is_seeded_and_shaped(pkg):
    a = pkg.scene.make_scene(50, 10, 10.0, seed=pkg.scene.scene_seed(0))
    b = pkg.scene.make_scene(50, 10, 10.0, seed=pkg.scene.scene_seed(0))
    assert all(np.array_equal(x, y) for x, y in zip(a.frames, b.frames))
    assert a.landmarks.shape == (50, 3)
    assert a.fixed == [k % 2 == 0 for k in range(10)]
    for z in a.frames:
        assert z.shape[1] == 3
        assert np.all((z[:, 0] >= -10) & (z[:, 0] <= 650))
    # every detected landmark projects into the image and disparity is positive
    z, ok = pkg.scene.project(a.landmarks, np.zeros(12))
    assert np.all(z[ok, 2] > 0)


def test_workload_configs(pkg):
    sc, cfg = pkg.scene.workload("plain_c0", n_frames=3)
    assert cfg.n_parents == 256 and cfg.max_gaussians == 64 and cfg.meas_dim == 3
    sc, cfg = pkg.scene.workload("plain_c1", n_frames=2)
    assert cfg.n_parents == 4096 and cfg.max_gaussians == 256
    assert cfg.kappa == pytest.approx(50.0 / (640 * 480 * 63))
