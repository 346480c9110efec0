"""FP32 device mode against the FP64 oracle on identical inputs, one step at a time.

At checkpoint frames of an FP64 run, the whole filter state (parent states,
log-weights, every map as Euclidean sample clouds) is loaded into the oracle and
into a fresh FP32 filter; both run the next predict + update and every output is
compared.  FP32 mode computes the sample clouds, refits, Kalman algebra,
normalisers and merge in FP32 (parent states, log-weight accumulation and the
resampling prefix sum stay FP64), so values carry FP32 rounding and a decision that
sits on a threshold can flip: a sample on the image border (changing its Gaussian's
mean pD), a weight at min_weight, a posterior whose smallest Cholesky pivot lies
between the FP64 test (1e-10 of its diagonal) and the FP32 one (1e-5), a Mahalanobis
distance at min_separation.  The tolerances below are therefore stated in two tiers:
a bound that holds for almost every value (by quantile) and a count bound on the
values a flipped decision may move.

Stated tolerances (FP32 device vs FP64 oracle, identical inputs):
  fitted weights                relative error <= 1e-6, every row
  fitted mean pD                equal in >= 99.5 % of rows
  fitted means                  |error| <= 1e-4 SD + 1e-6 |mean| for >= 99 % of values,
                                <= 1e-2 SD + 1e-6 |mean| for every value
  fitted covariances            |error| <= 1e-4 sqrt(S_aa S_bb) for >= 99 %, <= 1e-2 all
                                (means and covariances: rows with equal mean pD whose
                                cloud has >= 7 in-view samples; fewer give a singular
                                sample covariance whose FP32 value is rounding residue)
  normalisers log l_{p,m}       |error| <= 1e-4 for >= 99 %, <= 1e-2 for >= 99.9 %
  parent log-likelihoods        relative error <= 1e-4 for >= 98 % of parents, <= 1e-3 all
  map sizes, merged counts      equal for >= 97 % of parents
  merged weights                relative error <= 1e-4 for >= 99 % of rows
  merged means, covariances     as fitted means and covariances, >= 99 % of values
                                (parents whose merged counts are equal; rows paired
                                by nearest mean, since weights equal in FP32 but not in
                                FP64 list the components in another order)
"""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu

DIAG = [0, 2, 5, 9, 14, 20]   # packed-lower positions of the 6 diagonal entries


def _state(f):
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


def _mean_cov_errors(a, b, moff, coff):
    """Errors of b's means and packed covariances against a's, in the units the
    tolerances use: means per SD of a's diagonal (with a 1e-6 |mean| floor added to
    the bound, returned separately), covariances per sqrt(S_aa S_bb)."""
    sd = np.sqrt(np.maximum(a[:, coff + np.array(DIAG)], 1e-300))
    em = np.abs(b[:, moff:moff + 6] - a[:, moff:moff + 6])
    floor = 1e-6 * np.abs(a[:, moff:moff + 6])
    ec = []
    for i in range(6):
        for j in range(i + 1):
            e = i * (i + 1) // 2 + j
            ec.append(np.abs(b[:, coff + e] - a[:, coff + e]) / (sd[:, i] * sd[:, j]))
    return (em - floor) / sd, np.stack(ec, axis=1) if ec else np.zeros((0, 21))


def _pair_rows(a, b):
    """Row of b paired with each row of a (merged mixtures): the greedy merge lists its
    components in the order of their centres' weights, and many weights near 1 are
    equal in FP32 but not in FP64, so the two lists come in different orders.  Rows are
    paired by an assignment minimising the largest mean difference in a's standard
    deviations."""
    from scipy.optimize import linear_sum_assignment
    sd = np.sqrt(np.maximum(a[:, 7 + np.array(DIAG)], 1e-300))
    cost = (np.abs(b[None, :, 1:7] - a[:, None, 1:7]) / sd[:, None, :]).max(axis=2)
    r, c = linear_sum_assignment(np.minimum(cost, 1e12))
    out = np.empty(len(a), int)
    out[r] = c
    return out


def _q(x, tol):
    """Fraction of values within tol."""
    x = np.asarray(x).ravel()
    return 1.0 if x.size == 0 else float(np.mean(x <= tol))


@pytest.mark.parametrize("workload,n_parents,checkpoints", [
    ("plain_c1", 64, (3, 7, 11)),     # 200 landmarks, clutter 50, cap 256 (binding from frame 5)
    ("plain_c0", 128, (2, 20, 60)),   # 50 landmarks, clutter 10, cap 64
])
def test_fp32_one_step_within_stated_tolerances(pkg, orc, workload, n_parents, checkpoints):
    if not gpu_available():
        pytest.skip("no CUDA device")
    n_frames = max(checkpoints) + 2
    sc, cfg = pkg.scene.workload(workload, precision=pkg.SCPHD_FP64, n_frames=n_frames)
    cfg.n_parents = n_parents
    cfg32 = cfg.copy()
    cfg32.precision = pkg.SCPHD_FP32
    P, pd = int(cfg.particles_per_feature), float(cfg.pd)
    src = pkg.SCPHDCameraCalibration(cfg)
    report = []
    for k in range(max(checkpoints) + 1):
        z = sc.frames[k]
        src.step(pkg.scene.DT, z[:, 0], z[:, 1], fixed_camera=sc.fixed[k], d=z[:, 2])
        if k not in checkpoints:
            continue
        state = _state(src)
        ref, f32 = orc.Oracle(cfg), pkg.SCPHDCameraCalibration(cfg32)
        zn, fixed = sc.frames[k + 1], sc.fixed[k + 1]
        for f in (ref, f32):
            f.set_state(*state)
            f.predict(pkg.scene.DT)
            f.update(zn[:, 0], zn[:, 1], fixed_camera=fixed, d=zn[:, 2])
        M = zn.shape[0]
        # fitted mixtures: rows correspond one to one
        fw, pd_eq, fm, fc = [], [], [], []
        mcount_eq, mw, mm, mc = [], [], [], []
        for p in range(n_parents):
            a, b = ref.fitted(p), f32.mixture(pkg.SCPHD_MIX_FITTED, p)
            assert a.shape == b.shape, f"frame {k + 1} parent {p}: fitted counts differ"
            if len(a):
                fw.append(np.abs(b[:, 0] - a[:, 0]) / a[:, 0])
                same = np.abs(b[:, 1] - a[:, 1]) <= 1e-6
                pd_eq.append(same)
                n_in = np.rint(a[:, 1] * P / pd) if pd > 0 else np.zeros(len(a))
                live = same & (n_in >= 7)
                if live.any():
                    em, ec = _mean_cov_errors(a[live], b[live], 2, 8)
                    fm.append(em)
                    fc.append(ec)
            a, b = ref.merged(p), f32.mixture(pkg.SCPHD_MIX_MERGED, p)
            mcount_eq.append(a.shape == b.shape)
            if a.shape == b.shape and len(a):
                b = b[_pair_rows(a, b)]
                mw.append(np.abs(b[:, 0] - a[:, 0]) / a[:, 0])
                em, ec = _mean_cov_errors(a, b, 1, 7)
                mm.append(em)
                mc.append(ec)
        cat = lambda xs: np.concatenate([np.ravel(x) for x in xs]) if xs else np.zeros(0)
        fw, pd_eq, fm, fc, mw, mm, mc = map(cat, (fw, pd_eq, fm, fc, mw, mm, mc))
        e64, l64 = ref.normalizers(M)
        e32, l32 = f32.normalizers(M)
        de = np.abs(e32 - e64)
        dl = np.abs(l32 - l64) / np.maximum(1.0, np.abs(l64))
        sizes_eq = np.mean(ref.map_sizes() == f32.map_sizes())
        row = dict(frame=k + 1, fitted_w_max=float(fw.max(initial=0)), pd_equal=float(pd_eq.mean()),
                   fitted_mean_sd_p99=float(np.quantile(fm, 0.99)) if fm.size else 0.0,
                   fitted_mean_sd_max=float(fm.max(initial=0)),
                   fitted_cov_p99=float(np.quantile(fc, 0.99)) if fc.size else 0.0,
                   fitted_cov_max=float(fc.max(initial=0)),
                   ell_p99=float(np.quantile(de, 0.99)), ell_max=float(de.max()),
                   loglik_rel_p99=float(np.quantile(dl, 0.99)), loglik_rel_max=float(dl.max()),
                   map_sizes_equal=float(sizes_eq), merged_counts_equal=float(np.mean(mcount_eq)),
                   merged_w_p99=float(np.quantile(mw, 0.99)) if mw.size else 0.0,
                   merged_mean_sd_p99=float(np.quantile(mm, 0.99)) if mm.size else 0.0,
                   merged_cov_p99=float(np.quantile(mc, 0.99)) if mc.size else 0.0)
        report.append(row)
        print(row)
        msg = f"{workload} frame {k + 1}: {row}"
        assert fw.max(initial=0) <= 1e-6, msg
        assert pd_eq.mean() >= 0.995, msg
        assert _q(fm, 1e-4) >= 0.99 and fm.max(initial=0) <= 1e-2, msg
        assert _q(fc, 1e-4) >= 0.99 and fc.max(initial=0) <= 1e-2, msg
        assert _q(de, 1e-4) >= 0.99 and _q(de, 1e-2) >= 0.999, msg
        assert _q(dl, 1e-4) >= 0.98 and dl.max() <= 1e-3, msg
        assert sizes_eq >= 0.97 and np.mean(mcount_eq) >= 0.97, msg
        assert _q(mw, 1e-4) >= 0.99, msg
        assert _q(mm, 1e-4) >= 0.99 and _q(mc, 1e-4) >= 0.99, msg
        f32.close()
    assert len(report) == len(checkpoints)
