"""Configuration files, MAT measurement files and MAT result files (include/scphd_io.h),
on the host: the reader of the reference's libconfig keys, the level-5 MAT reader of
Z1/Z2 cell arrays (compressed, with other variables beside them), the MAT writer, and
the command-line driver's --dry-run (no GPU)."""
import json
import os
import subprocess

import numpy as np
import pytest
import scipy.io as sio

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CLI = os.path.join(ROOT, "scphd-camera-calibration_b200", "csrc", "scphd_calibrate")

# the reference's settings in its own key layout (prior given as {mean, std}, the way
# the shipped configuration file gives it), with comments in all three styles
REFERENCE_STYLE = """
verbosity = 0      # chatter
save_all_maps = false
max_steps = 100
n_particles = 100 ; particles_per_feature = 100
min_weight = 0.0001
min_separation = 6.0
max_velocity = 5.0 ;   // read by the reference, unused on this path
min_range = 0.5 ;
min_neff = 0.75 ;
ps = 0.9
prior : {
  cartesian : { x : {mean = 0.0 ; std = 0.0}; y : {mean = -50.0 ; std = 0.0};
                z : {mean = -3.0 ; std = 3.0}; vx : {mean = 0.0 ; std = 0.0};
                vy : {mean = 0.0 ; std = 0.0}; vz : {mean = 0.0 ; std = 0.0}; }
  angular : { x : {mean = 0.3927 ; std = 0.00}; y : {mean = 0.1 ; std = 0.1};
              z : {mean = 0.0 ; std = 0.0}; vx : {mean = 0.0 ; std = 0.00};
              vy : {mean = 0.0 ; std = 0.00}; vz : {mean = 0.0 ; std = 0.00}; }
}
/* camera motion:
   accelerations */
camera_motion_model : {
  cartesian : { ax = 0.0 ay = 0.00 az = 0.15 }
  angular : { ax = 0.0000 ay = 0.001 az = 0.000 }
}
feature_motion_model : { ax = 0.05 ay = 0.05 az = 0.1 }
measurement_model : { fx = -895.6561 fy = -891.2656 u0 = 400.0 v0 = 300.0
                      std_u = 5.0 std_v = 5.0 lambda = 10.0001 pd = 0.95 }
birth : { w0 = 0.000001 ; d0 = 8.0 vu0 = 0.0 vv0 = 0.0 vd0 = 0.0 var_d0 = 2.0
          var_vu0 = 6.0 var_vv0 = 6.0 var_vd0 = 0.05 }
"""

FIELDS = ["n_parents", "particles_per_feature", "min_weight", "min_separation", "min_neff", "ps", "fx", "fy",
          "u0", "v0", "std_u", "std_v", "pd", "kappa", "w0", "d0", "vu0", "vv0", "vd0", "var_d0", "var_vu0",
          "var_vv0", "var_vd0"]


def _write(tmp_path, name, text):
    p = tmp_path / name
    p.write_text(text)
    return str(p)


def test_config_in_the_references_layout_gives_its_values(pkg, tmp_path):
    cfg, opts = pkg.config_from_file(_write(tmp_path, "ref.cfg", REFERENCE_STYLE))
    ref = pkg.reference_defaults()
    for f in FIELDS:
        assert getattr(cfg, f) == pytest.approx(getattr(ref, f), rel=1e-15), f
    for i in range(12):
        assert cfg.prior_a[i] == ref.prior_a[i] and cfg.prior_b[i] == ref.prior_b[i], i
    for i in range(6):
        assert cfg.cam_std[i] == ref.cam_std[i]
    for i in range(3):
        assert cfg.feat_std[i] == ref.feat_std[i]
    assert opts == {"max_steps": 100, "slam": False, "save_all_maps": False, "verbosity": 0}


def test_config_code_keys_and_extensions(pkg, tmp_path):
    text = """
    n_particles = 512, slam = true, save_all_maps = TRUE
    prior : { cartesian : { z : { a = -6.0; b = 0.5 } } }   # the keys the reference's code reads
    measurement_model : { v0 = 240.0; lambda = 9.0; std_d = 0.5 }
    precision = "fp32"; meas_dim = 3; max_gaussians = 128; max_measurements = 96; seed = 0x1234
    baseline = 0.2
    """
    cfg, opts = pkg.config_from_file(_write(tmp_path, "x.cfg", text))
    assert cfg.n_parents == 512 and opts["slam"] and opts["save_all_maps"]
    assert cfg.prior_a[2] == -6.0 and cfg.prior_b[2] == 0.5
    assert cfg.kappa == pytest.approx(9.0 / 480.0 ** 2)
    assert cfg.precision == pkg.SCPHD_FP32 and cfg.meas_dim == 3
    assert cfg.max_gaussians == 128 and cfg.max_measurements == 96 and cfg.seed == 0x1234
    assert cfg.std_d == 0.5 and cfg.baseline == 0.2


@pytest.mark.parametrize("text,needle", [
    ("n_particles = 100\nps 0.9\n", ":2"),                     # missing '='
    ("prior : { cartesian : { x : { a = 1.0 } }\n", "}"),        # unclosed group
    ("n_particles = \"many\"\n", "n_particles"),                 # not a number
    ("ps = 0.9x\n", ":1"),                                       # bad value
    ("prior : { cartesian : { x : { a = 1.0 } } }\n", "a and b"),
])
def test_config_errors_name_the_line_or_key(pkg, tmp_path, text, needle):
    with pytest.raises(pkg.ScphdError) as e:
        pkg.config_from_file(_write(tmp_path, "bad.cfg", text))
    assert needle in str(e.value)
    with pytest.raises(pkg.ScphdError):
        pkg.config_from_file(str(tmp_path / "missing.cfg"))


def _cells(frames):
    c = np.empty((1, len(frames)), dtype=object)
    for k, z in enumerate(frames):
        c[0, k] = np.asarray(z, np.float64)
    return c


def _fixture_frames():
    g = np.load(os.path.join(HERE, "golden", "disparity_sim_frames.npz"))
    return [g["Z1_%d" % k] for k in range(12)], [g["Z2_%d" % k] for k in range(12)]


def test_mat_frames_from_the_reference_fixture(pkg, tmp_path):
    """Z1/Z2 of the reference's disparity_sim.mat (first 12 frames, committed as a
    fixture), written back as a compressed level-5 file beside other variables."""
    z1, z2 = _fixture_frames()
    path = str(tmp_path / "sim.mat")
    sio.savemat(path, {"campose_2": np.arange(6.0), "Z1": _cells(z1), "Z2": _cells(z2),
                       "meta": {"name": "x", "k": np.eye(2)}}, do_compression=True)
    r1, r2 = pkg.read_mat_frames(path, "Z1"), pkg.read_mat_frames(path, "Z2")
    assert len(r1) == 12 and len(r2) == 12
    for a, b in zip(r1 + r2, z1 + z2):
        assert a.shape == b.shape and np.array_equal(a, b)


def test_mat_frames_three_rows_empty_frames_and_storage_types(pkg, tmp_path):
    rng = np.random.default_rng(3)
    frames = [rng.uniform(0, 100, (3, n)) for n in (5, 0, 7)]
    frames.append(np.array([[1, 2, 3], [4, 5, 6], [7, 8, 9]], np.uint8))   # integer storage
    path = str(tmp_path / "uvd.mat")
    sio.savemat(path, {"Z2": _cells(frames)}, do_compression=False)
    r = pkg.read_mat_frames(path, "Z2")
    assert [x.shape for x in r] == [(3, 5), (3, 0), (3, 7), (3, 3)]
    for a, b in zip(r, frames):
        assert np.array_equal(a, np.asarray(b, np.float64))
    with pytest.raises(pkg.ScphdError):
        pkg.read_mat_frames(path, "Z1")                      # absent
    sio.savemat(path, {"Z1": np.eye(3)})
    with pytest.raises(pkg.ScphdError):
        pkg.read_mat_frames(path, "Z1")                      # not a cell array


def test_mat_writer_round_trip(pkg, tmp_path):
    rng = np.random.default_rng(4)
    arrays = {"a": rng.normal(size=(12, 5)), "b": rng.normal(size=(7, 1)), "empty": np.zeros((0, 0))}
    path = str(tmp_path / "w.mat")
    pkg.write_mat_arrays(path, arrays)
    m = sio.loadmat(path)
    for k, v in arrays.items():
        assert m[k].shape == v.shape and np.array_equal(m[k], v), k


def test_driver_dry_run(pkg, tmp_path):
    z1, z2 = _fixture_frames()
    data = str(tmp_path / "sim.mat")
    sio.savemat(data, {"Z1": _cells(z1), "Z2": _cells(z2)}, do_compression=True)
    cfg = _write(tmp_path, "ref.cfg", REFERENCE_STYLE.replace("max_steps = 100", "max_steps = 7"))
    assert os.path.exists(CLI), "driver not built"
    out = subprocess.run([CLI, cfg, data, "--dry-run"], capture_output=True, text=True, timeout=60)
    assert out.returncode == 0, out.stderr
    s = json.loads(out.stdout)
    assert s["frames"] == 12 and s["steps"] == 7 and s["rows"] == 2
    assert s["z1_measurements"] == sum(z.shape[1] for z in z1)
    assert s["z1_sum"] == pytest.approx(sum(float(z.sum()) for z in z1), rel=1e-12)
    assert s["z2_sum"] == pytest.approx(sum(float(z.sum()) for z in z2), rel=1e-12)
    assert s["n_parents"] == 100 and s["meas_dim"] == 2
    assert s["max_measurements"] % 32 == 0 and s["max_measurements"] >= max(z.shape[1] for z in z1 + z2)
    bad = subprocess.run([CLI, cfg], capture_output=True, text=True, timeout=60)
    assert bad.returncode != 0
