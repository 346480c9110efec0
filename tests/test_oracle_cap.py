"""The oracle's map-capacity cut (max_gaussians).

The reference keeps every merged component and every retained non-detection cloud
(src/scphdcameracalibration.cu:1923-1942); this implementation bounds each parent's
map at max_gaussians entries, keeping the largest weights -- compared rounded to
single precision, equal keys in entry order -- and the kept entries in their order.
The device applies the same rule in its merge kernel; these CPU tests pin the
oracle's statement of it."""
import numpy as np


def test_cap_keep_rule(orc):
    w = np.array([0.5, 0.2, 0.5, 0.1, 0.2, 0.3])
    assert orc.cap_keep(w, 3).tolist() == [True, False, True, False, False, True]
    # the fourth largest is one of two equal weights: the earlier entry wins
    assert orc.cap_keep(w, 4).tolist() == [True, True, True, False, False, True]
    assert orc.cap_keep(w, 6).all() and orc.cap_keep(w, 10).all()
    assert not orc.cap_keep(w, 0).any()
    rng = np.random.default_rng(3)
    for _ in range(50):
        n = int(rng.integers(1, 400))
        w = rng.choice(np.r_[rng.uniform(1e-3, 1, 8), 0.25], size=n)
        cap = int(rng.integers(1, n + 1))
        keep = orc.cap_keep(w, cap)
        assert keep.sum() == min(cap, n)
        expect = sorted(range(n), key=lambda e: (-np.float32(w[e]), e))[:cap]
        assert np.array_equal(np.flatnonzero(keep), np.sort(expect))
    # weights equal to single precision are ties: entry order decides
    w = np.array([0.3, 0.3 * (1 + 1e-12), 0.2, 0.3 * (1 - 1e-12)])
    assert orc.cap_keep(w, 2).tolist() == [True, True, False, False]
    assert orc.cap_keep(w, 1).tolist() == [True, False, False, False]


def test_capped_map_is_the_cut_of_the_uncapped_map(pkg, orc):
    """A capped and an uncapped oracle run in lockstep on one scene: up to the first
    frame at which the cap binds their maps are identical, and at that frame the
    capped map's weights are exactly the cut of the uncapped map's weights."""
    sc = pkg.scene.make_scene(n_landmarks=30, n_frames=6, clutter_rate=6.0, seed=pkg.scene.scene_seed(0, 21))
    cap = 12
    cfg = pkg.scene.filter_config(n_parents=12, max_gaussians=cap, max_meas=96, clutter_rate=6.0,
                                  precision=pkg.SCPHD_FP64, calib=sc.calib, seed=21, particles_per_feature=24)
    free_cfg = cfg.copy()
    free_cfg.max_gaussians = 100000
    capped, free = orc.Oracle(cfg), orc.Oracle(free_cfg)
    checked = 0
    for k in range(sc.n_frames):
        z = sc.frames[k]
        for o in (capped, free):
            o.predict(pkg.scene.DT)
            o.update(z[:, 0], z[:, 1], sc.fixed[k], d=z[:, 2])
        sizes_free = free.map_sizes()
        assert np.all(capped.map_sizes() <= cap)
        if capped.truncations() == 0:
            assert np.array_equal(capped.map_sizes(), sizes_free)
            for p in range(cfg.n_parents):
                np.testing.assert_array_equal(capped.map(p)[0], free.map(p)[0])
            assert capped.resample() == free.resample()
            continue
        assert capped.truncations() == int(np.sum(sizes_free > cap))
        for p in range(cfg.n_parents):
            Wf, xf, _ = free.map(p)
            Wc, xc, _ = capped.map(p)
            keep = orc.cap_keep(Wf, cap)
            np.testing.assert_array_equal(Wc, Wf[keep])
            np.testing.assert_array_equal(xc, xf[keep])
            checked += int(sizes_free[p] > cap)
        break
    assert checked > 0, "the cap never bound in this scene"


def test_merge_orders_weights_equal_to_single_precision_by_index(orc):
    """The greedy merge's argmax compares weights rounded to single precision: two
    components whose FP64 weights differ only in their last bits are a tie, and the
    reference's index rule (tie key) orders them, whichever is heavier in FP64."""
    comps = np.zeros((2, 28))
    comps[0, 0], comps[1, 0] = 0.3, 0.3 * (1 + 1e-12)
    comps[0, 1:7], comps[1, 1:7] = 0.0, 100.0   # far apart: no merge
    diag = [0, 2, 5, 9, 14, 20]
    comps[:, 7 + np.array(diag)] = 1.0
    out, mem = orc.merge(comps, np.zeros(2, np.uint8), 6.0)
    assert len(out) == 2 and orc.tie_key(0) < orc.tie_key(1)
    assert mem.tolist() == [0, 1] and out[0, 0] == comps[0, 0]
    comps[1, 0] = 0.3 * (1 + 1e-6)   # distinct in single precision: the heavier first
    out, mem = orc.merge(comps, np.zeros(2, np.uint8), 6.0)
    assert mem.tolist() == [1, 0]
