"""Device path vs the FP64 oracle, frame by frame, through the C ABI.

FP64 device mode: parent states, log-weights, map sizes, fitted and merged
mixtures, normalisers and resampling indices against the oracle on the same
seeded scenes and random streams.  Counts and resampling indices must match
exactly; floating point within the tolerances stated below.
"""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu

# FP64 device arithmetic differs from the oracle only in operation order and in
# CUDA's vs glibc's log/sin/cos (<= 2 ulp): relative tolerances for FP64 mode
RT_STATE = 1e-9      # parent states (FP64 path in both modes)
RT_LW = 1e-7         # parent log-weights (sum of ~M log-normalisers)
RT_MIX = 1e-6        # means/covariances of fitted and merged mixtures
AT_MIX = 1e-7
# A sample cloud with fewer in-view samples than dimensions refits to a singular
# covariance, and so does its Kalman posterior; the reference's PD test on it (Cholesky
# without NaN) is decided by rounding.  Device and oracle both class such a posterior
# as not PD (every pivot must exceed 1e-10 of its diagonal), so every value is held to
# the FP64 tolerance.


def _two_tier(a, b, rtol, atol, frac, what):
    """Every value within atol + rtol |b| (frac is kept for the callers' signatures)."""
    err = np.abs(a - b)
    bad = err > atol + rtol * np.abs(b)
    assert not bad.any(), f"{what}: {int(bad.sum())} values off, max error {err.max():.3e}"


def _need_gpu():
    if not gpu_available():
        pytest.skip("no CUDA device")


def _pair(pkg, orc, cfg):
    return pkg.SCPHDCameraCalibration(cfg), orc.Oracle(cfg)


def _compare_frame(gpu, ref, M, k, strict=True):
    st_g, lw_g = gpu.particles()
    st_r, lw_r = ref.particles()
    np.testing.assert_allclose(st_g, st_r, rtol=RT_STATE, atol=1e-9, err_msg=f"frame {k} states")
    _two_tier(lw_g, lw_r, RT_LW, 1e-7, 0.95, f"frame {k} log-weights")
    ng, nr = gpu.map_sizes(), ref.map_sizes()
    assert np.array_equal(ng, nr), f"frame {k} map sizes {ng[:8]} vs {nr[:8]}"
    if M > 0:
        eg, llg = gpu.normalizers(M)
        er, llr = ref.normalizers(M)
        _two_tier(eg, er, 1e-9, 1e-9, 0.99, f"frame {k} normalisers")
        _two_tier(llg, llr, 1e-9, 1e-7, 0.95, f"frame {k} loglik")
    for p in range(0, gpu.n_parents, max(1, gpu.n_parents // 4)):
        fg, fr = gpu.mixture(0, p), ref.fitted(p)
        assert fg.shape == fr.shape, f"frame {k} parent {p} fitted count"
        live = fr[:, 1] > 0   # fits of all-out-of-view clouds are placeholders in both
        np.testing.assert_allclose(fg[live], fr[live], rtol=RT_MIX, atol=AT_MIX,
                                   err_msg=f"frame {k} parent {p} fitted")
        mg, mr = gpu.mixture(1, p), ref.merged(p)
        assert mg.shape == mr.shape, f"frame {k} parent {p} merged count {mg.shape} vs {mr.shape}"
        np.testing.assert_allclose(mg, mr, rtol=RT_MIX, atol=AT_MIX, err_msg=f"frame {k} parent {p} merged")


@pytest.mark.parametrize("meas_dim", [3, 2])
def test_fp64_frames_match_oracle(pkg, orc, meas_dim):
    _need_gpu()
    sc = pkg.scene.make_scene(n_landmarks=20, n_frames=8, clutter_rate=4.0, seed=pkg.scene.scene_seed(0, 11))
    cfg = pkg.scene.filter_config(n_parents=48, max_gaussians=160, max_meas=96, clutter_rate=4.0,
                                  precision=pkg.SCPHD_FP64, calib=sc.calib, seed=11, particles_per_feature=48,
                                  meas_dim=meas_dim)
    gpu, ref = _pair(pkg, orc, cfg)
    for k in range(sc.n_frames):
        z = sc.frames[k]
        for f in (gpu, ref):
            f.predict(pkg.scene.DT)
            f.update(z[:, 0], z[:, 1], fixed_camera=sc.fixed[k], d=z[:, 2] if meas_dim == 3 else None)
        _compare_frame(gpu, ref, z.shape[0], k)
        rg, rr = gpu.resample(), ref.resample()
        assert rg == rr, f"frame {k} resample decision"
        if rr:
            assert np.array_equal(gpu.resample_indices(), ref.resample_indices()), f"frame {k} resample idx"
    c = gpu.counters()
    assert c[0] == 0 and c[1] == 0, f"capacity hit in a parity scene: {c}"


@pytest.mark.parametrize("particles", [7, 33])
def test_fp64_frames_match_oracle_sample_counts(pkg, orc, particles):
    """Sample counts that leave a 16-sample pass of a half-warp partly filled (P = 7)
    or reach one sample into a third pass (P = 33), both padded to 4-sample rows."""
    _need_gpu()
    sc = pkg.scene.make_scene(n_landmarks=16, n_frames=6, clutter_rate=4.0, seed=pkg.scene.scene_seed(0, 12))
    cfg = pkg.scene.filter_config(n_parents=24, max_gaussians=160, max_meas=96, clutter_rate=4.0,
                                  precision=pkg.SCPHD_FP64, calib=sc.calib, seed=12,
                                  particles_per_feature=particles)
    gpu, ref = _pair(pkg, orc, cfg)
    for k in range(sc.n_frames):
        z = sc.frames[k]
        for f in (gpu, ref):
            f.predict(pkg.scene.DT)
            f.update(z[:, 0], z[:, 1], fixed_camera=sc.fixed[k], d=z[:, 2])
        _compare_frame(gpu, ref, z.shape[0], k)
        assert gpu.resample() == ref.resample(), f"frame {k} resample decision"


def test_fp64_largest_sample_count_matches_oracle(pkg, orc):
    """216 samples per Gaussian, the most whose FP64 sample rows fit one cloud-fit
    block's shared memory; 217 is refused at create, as is more than 256 in FP32."""
    _need_gpu()
    sc = pkg.scene.make_scene(n_landmarks=12, n_frames=4, clutter_rate=3.0, seed=pkg.scene.scene_seed(0, 14))
    cfg = pkg.scene.filter_config(n_parents=8, max_gaussians=64, max_meas=64, clutter_rate=3.0,
                                  precision=pkg.SCPHD_FP64, calib=sc.calib, seed=14, particles_per_feature=216)
    gpu, ref = _pair(pkg, orc, cfg)
    for k in range(sc.n_frames):
        z = sc.frames[k]
        for f in (gpu, ref):
            f.predict(pkg.scene.DT)
            f.update(z[:, 0], z[:, 1], fixed_camera=sc.fixed[k], d=z[:, 2])
        _compare_frame(gpu, ref, z.shape[0], k)
        assert gpu.resample() == ref.resample(), f"frame {k} resample decision"
    big = cfg.copy()
    big.particles_per_feature = 217
    with pytest.raises(pkg.ScphdError) as e:
        pkg.SCPHDCameraCalibration(big)
    assert e.value.status == 3
    fp32 = cfg.copy()
    fp32.precision = pkg.SCPHD_FP32
    fp32.particles_per_feature = 256
    f = pkg.SCPHDCameraCalibration(fp32)
    z = sc.frames[0]
    f.step(pkg.scene.DT, z[:, 0], z[:, 1], fixed_camera=sc.fixed[0], d=z[:, 2])
    f.checkStuff()
    fp32.particles_per_feature = 257
    with pytest.raises(pkg.ScphdError):
        pkg.SCPHDCameraCalibration(fp32)


def test_fp64_frames_match_oracle_certain_detection(pkg, orc):
    """pd = 1: a non-detection cloud's in-view samples carry weight 1 - pd = 0, so a
    cloud whose out-of-view samples stay out of view has all in-view weights 0 and is
    fitted with unit weights (the reference's fallback), from samples drawn again."""
    _need_gpu()
    # a scene (searched with the oracle) where such fits occur in frames 3, 5 and 7
    sc = pkg.scene.make_scene(n_landmarks=20, n_frames=8, clutter_rate=4.0, seed=pkg.scene.scene_seed(0, 27))
    cfg = pkg.scene.filter_config(n_parents=32, max_gaussians=160, max_meas=96, clutter_rate=4.0,
                                  precision=pkg.SCPHD_FP64, calib=sc.calib, seed=27, particles_per_feature=40)
    cfg.pd = 1.0
    gpu, ref = _pair(pkg, orc, cfg)
    for k in range(sc.n_frames):
        z = sc.frames[k]
        for f in (gpu, ref):
            f.predict(pkg.scene.DT)
            f.update(z[:, 0], z[:, 1], fixed_camera=sc.fixed[k], d=z[:, 2])
        _compare_frame(gpu, ref, z.shape[0], k)
        assert gpu.resample() == ref.resample(), f"frame {k} resample decision"
    assert gpu.counters()[14] > 0, "no Gaussian took the unit-weight fit"


def test_reference_fixture_frames(pkg, orc):
    """The reference's own measurement frames (data/disparity_sim.mat, committed as
    tests/golden/disparity_sim_frames.npz) with its shipped model parameters and
    particle counts (n_particles 100, particles_per_feature 100), for max_steps = 100
    frames of its driver loop (src/main.cpp:73-97: predict(0.5), Z1 with the fixed
    camera on even frames, Z2 on odd ones, resample).  The map capacity is set far
    above the largest map of this run (596), so the cap never binds and the filter
    is the reference's uncapped recurrence."""
    _need_gpu()
    import os
    g = np.load(os.path.join(os.path.dirname(__file__), "golden", "disparity_sim_frames.npz"))
    cfg = pkg.reference_defaults()
    assert cfg.n_parents == 100 and cfg.particles_per_feature == 100
    cfg.max_gaussians = 1024
    cfg.max_survivors = 640
    cfg.max_measurements = 64
    cfg.precision = pkg.SCPHD_FP64
    gpu, ref = _pair(pkg, orc, cfg)
    resampled = 0
    for k in range(100):
        Z = g["Z1_%d" % k] if k % 2 == 0 else g["Z2_%d" % k]
        for f in (gpu, ref):
            f.predict(0.5)
            f.update(Z[0], Z[1], fixed_camera=(k % 2 == 0))
        _compare_frame(gpu, ref, Z.shape[1], k)
        rg, rr = gpu.resample(), ref.resample()
        assert rg == rr, f"frame {k} resample decision"
        if rr:
            resampled += 1
            assert np.array_equal(gpu.resample_indices(), ref.resample_indices()), f"frame {k} resample idx"
    c = gpu.counters()
    assert c[0] == 0 and c[1] == 0 and ref.truncations() == 0, f"capacity hit: {c[:2]}"
    assert resampled > 0


def _run_lockstep(pkg, gpu, ref, sc, n_frames):
    """Step device and oracle together, comparing every frame; returns the number of
    frames that resampled."""
    resampled = 0
    for k in range(n_frames):
        z = sc.frames[k]
        for f in (gpu, ref):
            f.predict(pkg.scene.DT)
            f.update(z[:, 0], z[:, 1], fixed_camera=sc.fixed[k], d=z[:, 2])
        _compare_frame(gpu, ref, z.shape[0], k)
        rg, rr = gpu.resample(), ref.resample()
        assert rg == rr, f"frame {k} resample decision"
        if rr:
            resampled += 1
            assert np.array_equal(gpu.resample_indices(), ref.resample_indices()), f"frame {k} resample idx"
    return resampled


def test_fp64_capped_maps_match_oracle(pkg, orc):
    """The map capacity binds: the plain_c1 scene (200 landmarks, clutter 50/frame,
    (u,v,d), <= 256 Gaussians per parent, 100 samples per Gaussian) on 48 parents for
    14 frames.  The cap first binds at frame 5 and then cuts most parents' maps every
    frame; device and oracle must keep the same entries (map sizes exact, every
    value within the FP64 tolerances) and count the same truncations."""
    _need_gpu()
    sc, cfg = pkg.scene.workload("plain_c1", precision=pkg.SCPHD_FP64, n_frames=14)
    cfg.n_parents = 48
    gpu, ref = _pair(pkg, orc, cfg)
    _run_lockstep(pkg, gpu, ref, sc, sc.n_frames)
    c = gpu.counters()
    assert ref.truncations() > 100, ref.truncations()
    assert c[0] == ref.truncations(), (int(c[0]), ref.truncations())
    assert c[1] == 0, "survivor scratch overflow"


def test_fp64_config0_all_frames_match_oracle(pkg, orc):
    """BASELINE config 0 in full: 256 parents, 50 landmarks, clutter 10/frame,
    <= 64 Gaussians per parent, 100 samples per Gaussian, all 100 frames, FP64,
    compared with the oracle after every frame.  The cap binds on every parent from
    about frame 10 on."""
    _need_gpu()
    sc, cfg = pkg.scene.workload("plain_c0", precision=pkg.SCPHD_FP64)
    assert cfg.n_parents == 256 and cfg.max_gaussians == 64 and sc.n_frames == 100
    gpu, ref = _pair(pkg, orc, cfg)
    resampled = _run_lockstep(pkg, gpu, ref, sc, sc.n_frames)
    c = gpu.counters()
    assert c[0] == ref.truncations() and ref.truncations() > 0
    assert c[1] == 0
    assert resampled > 0


def test_merge_decisions_identical_inputs(pkg, orc):
    """Greedy merge on identical component lists: counts, membership exact."""
    _need_gpu()
    rng = np.random.default_rng(5)
    for trial in range(6):
        n = int(rng.integers(5, 300))
        comps = np.zeros((n, 28))
        centers = rng.uniform(0, 100, (max(1, n // 4), 6))
        for i in range(n):
            c = centers[rng.integers(len(centers))]
            A = rng.normal(0, 1, (6, 6)) * 0.5
            C = A @ A.T + np.diag(rng.uniform(0.5, 3, 6))
            comps[i, 0] = rng.choice([rng.uniform(1e-3, 1), 0.25])   # exact ties too
            comps[i, 1:7] = c + rng.normal(0, 1.0, 6)
            comps[i, 7:] = [C[a, b] for a in range(6) for b in range(a + 1)]
        flags = (rng.uniform(size=n) < 0.1).astype(np.uint8)
        mo, memo = orc.merge(comps, flags, 6.0)
        for prec in (pkg.SCPHD_FP64, pkg.SCPHD_FP32):
            if prec == pkg.SCPHD_FP32:
                comps32 = comps.astype(np.float32).astype(np.float64)
                mo, memo = orc.merge(comps32, flags, 6.0)
                mg, memg = pkg.merge_components(comps32, flags, 6.0, prec)
                tol = dict(rtol=2e-4, atol=2e-4)
            else:
                mg, memg = pkg.merge_components(comps, flags, 6.0, prec)
                tol = dict(rtol=1e-10, atol=1e-10)
            assert mg.shape == mo.shape, f"trial {trial} prec {prec} count"
            assert np.array_equal(memg, memo), f"trial {trial} prec {prec} membership"
            np.testing.assert_allclose(mg, mo, **tol)


def test_systematic_resample_identical_weights(pkg, orc):
    _need_gpu()
    rng = np.random.default_rng(9)
    for n in (1, 7, 256, 1000, 4096, 16384):
        w = rng.exponential(size=n) ** 3
        w /= w.sum()
        for u in (0.0001, 0.37, 0.9999):
            a = pkg.systematic_resample(w, u)
            b = orc.systematic(w, u)
            assert np.array_equal(a, b), f"n={n} u={u}"


def test_capacity_and_argument_errors(pkg):
    _need_gpu()
    cfg = pkg.reference_defaults()
    cfg.n_parents = 8
    cfg.max_measurements = 4
    f = pkg.SCPHDCameraCalibration(cfg)
    f.predict(0.5)
    with pytest.raises(pkg.ScphdError) as e:
        f.update(np.zeros(5), np.zeros(5))
    assert e.value.status == 3
    f.update(np.array([10.0]), np.array([20.0]))
    f.update(np.zeros(0), np.zeros(0))   # empty frame is legal
    bad = cfg.copy()
    bad.meas_dim = 4
    with pytest.raises(pkg.ScphdError):
        pkg.SCPHDCameraCalibration(bad)


def test_fp32_frames_track_oracle(pkg, orc):
    """FP32 device mode against the FP64 oracle on the same streams.  Parent states are
    FP64 in both and equal until weights (FP32 normalisers) steer a resampling
    differently; map sizes and normalisers agree to FP32 accuracy.  A survivor,
    sample or merge on a threshold can flip between FP32 and FP64, changing that
    parent's map, so log-weights are held per parent: 90 % within 0.05 and all
    within 1.0."""
    _need_gpu()
    sc = pkg.scene.make_scene(n_landmarks=25, n_frames=6, clutter_rate=5.0, seed=pkg.scene.scene_seed(0, 12))
    cfg = pkg.scene.filter_config(n_parents=64, max_gaussians=160, max_meas=96, clutter_rate=5.0,
                                  precision=pkg.SCPHD_FP32, calib=sc.calib, seed=12, particles_per_feature=100)
    gpu, ref = _pair(pkg, orc, cfg)
    for k in range(sc.n_frames):
        z = sc.frames[k]
        for f in (gpu, ref):
            f.predict(pkg.scene.DT)
            f.update(z[:, 0], z[:, 1], fixed_camera=sc.fixed[k], d=z[:, 2])
        ng, nr = gpu.map_sizes(), ref.map_sizes()
        assert np.abs(ng.astype(float) - nr).sum() <= 0.05 * nr.sum() + 2, f"frame {k} map sizes"
        eg, _ = gpu.normalizers(z.shape[0])
        er, _ = ref.normalizers(z.shape[0])
        rel = np.abs(eg - er) / np.maximum(1.0, np.abs(er))
        assert np.median(rel) < 1e-5 and np.quantile(rel, 0.99) < 1e-3, f"frame {k} normalisers"
        st_g, lw_g = gpu.particles()
        st_r, lw_r = ref.particles()
        err = np.abs(lw_g - lw_r)
        assert np.mean(err <= 0.05) >= 0.9 and err.max() <= 1.0, f"frame {k} log-weights {err.max():.3f}"
        rg, rr = gpu.resample(), ref.resample()
        assert rg == rr
        if rr and not np.array_equal(gpu.resample_indices(), ref.resample_indices()):
            break   # ancestries diverge from here on; the comparison ends


def _state(f):
    """A filter's whole state as set_state takes it."""
    st, lw = f.particles()
    sizes = f.map_sizes()
    ws, cl, om = [], [], []
    for p in range(f.n_parents):
        if sizes[p]:
            ws.append(f.map_weights(p))
            x, o = f.map_clouds(p)
            cl.append(x)
            om.append(o)
    P = int(f.config.particles_per_feature)
    cat = lambda xs, shp: np.concatenate(xs) if xs else np.zeros(shp)
    return st, lw, sizes, cat(ws, (0,)), cat(cl, (0, 6, P)), cat(om, (0, P))


@pytest.mark.parametrize("clutter", [5.0, 1e-30])
def test_fp32_one_step_normalisers(pkg, clutter):
    """One FP64 state loaded into a fresh FP64 and a fresh FP32 filter; the next
    predict + update's normalisers agree to FP32 accuracy.  With clutter 5 the FP32
    normaliser sums around the parent's largest log-constant; with clutter 1e-30 per
    frame log(M w0 + kappa) is about -85, more than 60 below the Gaussians'
    log-constants, and it takes its online log-sum-exp.  (Run on, the two modes part
    at a prune decision on a threshold there, so the comparison is one step.)"""
    _need_gpu()
    sc = pkg.scene.make_scene(n_landmarks=25, n_frames=5, clutter_rate=clutter, seed=pkg.scene.scene_seed(0, 12))
    cfg = pkg.scene.filter_config(n_parents=64, max_gaussians=160, max_meas=96, clutter_rate=clutter,
                                  precision=pkg.SCPHD_FP64, calib=sc.calib, seed=12, particles_per_feature=100)
    src = pkg.SCPHDCameraCalibration(cfg)
    for k in range(3):
        z = sc.frames[k]
        src.step(pkg.scene.DT, z[:, 0], z[:, 1], fixed_camera=sc.fixed[k], d=z[:, 2])
    state = _state(src)
    out = []
    for prec in (pkg.SCPHD_FP64, pkg.SCPHD_FP32):
        c = cfg.copy()
        c.precision = prec
        f = pkg.SCPHDCameraCalibration(c)
        f.set_state(*state)
        z = sc.frames[3]
        f.predict(pkg.scene.DT)
        f.update(z[:, 0], z[:, 1], fixed_camera=sc.fixed[3], d=z[:, 2])
        out.append(f.normalizers(z.shape[0])[0])
    e64, e32 = out
    rel = np.abs(e32 - e64) / np.maximum(1.0, np.abs(e64))
    assert np.median(rel) < 1e-5 and np.quantile(rel, 0.99) < 1e-3, (np.median(rel), np.quantile(rel, 0.99))


@pytest.mark.parametrize("prec", [1, 0])
def test_map_capacity_keeps_largest_weights(pkg, orc, prec):
    """max_gaussians binds: the new map holds the max_gaussians largest weights of
    (merged components, retained non-detection terms), ties in entry order, and
    keeps the entries' order."""
    _need_gpu()
    sc = pkg.scene.make_scene(n_landmarks=30, n_frames=5, clutter_rate=6.0, seed=pkg.scene.scene_seed(0, 21))
    cfg = pkg.scene.filter_config(n_parents=16, max_gaussians=12, max_meas=96, clutter_rate=6.0,
                                  precision=prec, calib=sc.calib, seed=21, particles_per_feature=32)
    gpu = pkg.SCPHDCameraCalibration(cfg)
    hit = False
    for k in range(sc.n_frames):
        z = sc.frames[k]
        gpu.predict(pkg.scene.DT)
        gpu.update(z[:, 0], z[:, 1], fixed_camera=sc.fixed[k], d=z[:, 2])
        sizes = gpu.map_sizes()
        assert np.all(sizes <= 12)
        for p in range(4):
            mg = gpu.mixture(1, p)
            fr = gpu.mixture(0, p)
            wnd = fr[:, 0] * (1 - fr[:, 1])
            cand = np.concatenate([mg[:, 0], np.where(wnd >= cfg.min_weight, wnd, -1.0)])
            valid = np.where(cand >= 0)[0]
            if valid.size > 12:
                hit = True
                order = sorted(valid, key=lambda e: (-cand[e], e))[:12]
                keep = np.sort(order)
            else:
                keep = valid
            np.testing.assert_allclose(gpu.map_weights(p), cand[keep], rtol=1e-6)
        gpu.resample()
    assert hit, "the capacity never bound in this scene"
    assert gpu.counters()[0] > 0
