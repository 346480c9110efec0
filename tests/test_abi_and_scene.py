"""C-ABI surface (no device calls), config layout, scene generator, and the
host-side replica plan used for multi-GPU runs (gloo, world size 2)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_library_exports_every_declared_symbol(pkg):
    hdr = "".join(open(os.path.join(ROOT, "include", h)).read() for h in ("scphd.h", "scphd_io.h"))
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


def test_server_without_device_fails_loudly(pkg):
    try:
        import torch
        if torch.cuda.is_available():
            pytest.skip("device present")
    except Exception:
        pass
    with pytest.raises(pkg.ScphdError) as e:
        pkg.SCPHDServer(1 << 30)
    assert e.value.status in (2, 5)


def test_device_bytes_and_wave_plan(pkg):
    """Device footprint is pure arithmetic (no device) and grows with every capacity;
    the wave planner keeps each wave within the budget and the filters in order."""
    base = pkg.scene.filter_config(n_parents=100, max_gaussians=64, max_meas=64, clutter_rate=5.0)
    b0 = pkg.device_bytes(base)
    for field, val in (("n_parents", 200), ("max_gaussians", 128), ("max_measurements", 256),
                       ("particles_per_feature", 200), ("precision", 1)):
        c = base.copy()
        setattr(c, field, val)
        assert pkg.device_bytes(c) > b0, field
    bad = base.copy()
    bad.meas_dim = 4
    with pytest.raises(pkg.ScphdError):
        pkg.device_bytes(bad)
    sizes = [5, 3, 4, 9, 1, 1, 8]
    waves = pkg.scene.plan_waves(sizes, 10)
    assert [i for w in waves for i in w] == list(range(len(sizes)))
    assert all(sum(sizes[i] for i in w) <= 10 for w in waves)
    with pytest.raises(ValueError):
        pkg.scene.plan_waves([11], 10)


def test_counter_names_follow_the_header(pkg):
    """COUNTER_NAMES lists scphd_get_counters' entries in the order the header documents."""
    with open(os.path.join(ROOT, "include", "scphd.h")) as fh:
        text = " ".join(fh.read().split())
    doc = text[text.index("Counters since create:"):text.index("scphd_status scphd_get_counters")]
    parts = re.split(r"\[(\d+)\]", doc)
    entries = {int(parts[i]): parts[i + 1] for i in range(1, len(parts) - 1, 2)}
    assert sorted(entries) == list(range(16))
    keyword = {"map_truncations": "truncation", "scratch_overflows": "overflow", "frames_updated": "frames updated",
               "resamplings": "resampling", "units_last_update": "units of the last",
               "survivors_last_update": "survivors of the last", "units_total": "units since",
               "survivors_total": "survivors since", "clouds_read": "read", "clouds_written": "written",
               "gaussians_fitted": "fitted", "merged_rows": "merged", "mahalanobis_evaluations": "Mahalanobis",
               "max_survivors_per_parent": "largest survivor", "unit_weight_fits": "unit sample",
               "reserved": "reserved"}
    assert len(pkg.COUNTER_NAMES) == 16 and set(pkg.COUNTER_NAMES) == set(keyword)
    for k, name in enumerate(pkg.COUNTER_NAMES):
        assert keyword[name] in entries[k], (k, name, entries[k])
