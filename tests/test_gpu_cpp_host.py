"""The C++ host class (include/scphd.hpp) in a reference-shaped driver, on the
reference's own measurement frames, against the oracle."""
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, gpu_available

pytestmark = pytest.mark.gpu


def test_cpp_driver_matches_oracle(tmp_path, pkg, orc):
    if not gpu_available():
        pytest.skip("no CUDA device")
    exe = tmp_path / "host_driver"
    libdir = os.path.join(ROOT, "scphd-camera-calibration_b200", "csrc")
    cxx = "/usr/bin/g++" if os.path.exists("/usr/bin/g++") else "g++"
    subprocess.run([cxx, "-std=c++17", "-O2", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "host_driver.cpp"), "-o", str(exe),
                    "-L", libdir, "-lscphd_b200", f"-Wl,-rpath,{libdir}"], check=True)
    g = np.load(os.path.join(ROOT, "tests", "golden", "disparity_sim_frames.npz"))
    frames = []
    for k in range(6):
        Z = g["Z1_%d" % k] if k % 2 == 0 else g["Z2_%d" % k]
        frames.append((Z, k % 2 == 0))
    fb = tmp_path / "frames.bin"
    with open(fb, "wb") as fh:
        fh.write(np.int32(len(frames)).tobytes())
        for Z, fixed in frames:
            fh.write(np.int32(Z.shape[1]).tobytes() + np.int32(int(fixed)).tobytes())
            fh.write(np.ascontiguousarray(Z[0], np.float64).tobytes())
            fh.write(np.ascontiguousarray(Z[1], np.float64).tobytes())
    out = tmp_path / "out.bin"
    N, ppf = 24, 48
    subprocess.run([str(exe), str(fb), str(out), f"n_parents={N}", f"ppf={ppf}"], check=True)
    res = np.fromfile(out, np.float64)
    st, w = res[: N * 12].reshape(N, 12), res[N * 12:]
    cfg = pkg.reference_defaults()
    cfg.n_parents, cfg.particles_per_feature = N, ppf
    o = orc.Oracle(cfg)
    for Z, fixed in frames:
        o.predict(0.5)
        o.update(Z[0], Z[1], fixed)
        o.resample()
    st_r, lw_r = o.particles()
    np.testing.assert_allclose(st, st_r, rtol=1e-9, atol=1e-9)
    np.testing.assert_allclose(w, np.exp(lw_r), rtol=1e-6, atol=1e-9)
