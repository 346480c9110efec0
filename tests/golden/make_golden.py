"""Generate the committed golden fixtures (run where the reference tree is
available, with REF_DIR pointing at it; the GPU box only reads the .npz files).

    REF_DIR=<reference tree> python tests/golden/make_golden.py

disparity_sim_frames.npz  the first 100 measurement frames Z1/Z2 of the
                          reference's data/disparity_sim.mat (2 x n, u;v) --
                          max_steps of its shipped config/calibration.cfg --
                          and campose_2, read with scipy.
ref_kernels.npz           inputs and outputs of the reference's OWN code
                          compiled for the host (oracle/_ref/libscphd_ref.so):
                          computeMeasurement/invertMeasurement, worldToDisparity
                          Kernel (in-FOV pD), computeDetectionsKernel,
                          updateKernel, computeMahalDist<6,36>, isPosDef,
                          cholesky, wrapAngle and the oriented CV motion model.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
N_FRAMES = 100


def ref_dir() -> str:
    d = os.environ.get("REF_DIR")
    if not d or not os.path.isfile(os.path.join(d, "src", "kernels.cu")):
        sys.exit("make_golden.py needs REF_DIR=<reference tree holding src/kernels.cu and data/>")
    return d


def frames():
    import scipy.io as sio
    m = sio.loadmat(os.path.join(ref_dir(), "data", "disparity_sim.mat"))
    out = {"campose_2": m["campose_2"].ravel()}
    for k in range(N_FRAMES):
        out["Z1_%d" % k] = np.asarray(m["Z1"][0, k], np.float64)
        out["Z2_%d" % k] = np.asarray(m["Z2"][0, k], np.float64)
    np.savez_compressed(os.path.join(HERE, "disparity_sim_frames.npz"), **out)


def spd(rng, scale=1.0):
    A = rng.normal(0, 1, (6, 6))
    C = A @ A.T + np.diag(rng.uniform(0.2, 2.0, 6))
    C[:2, :2] *= 20 * scale
    return C


def packed(C):
    return np.array([C[a, b] for a in range(6) for b in range(a + 1)])


def ref_kernels():
    sys.path.insert(0, ROOT)
    from oracle import oracle as orc
    orc.build(ref_dir())
    ref = orc.RefLib()
    rng = np.random.default_rng(20240607)
    m8 = np.array([-895.6561, -891.2656, 400.0, 300.0, 5.0, 5.0, 0.95, 10.0001])
    out = {"model8": m8}
    # transforms
    n = 64
    X = np.stack([rng.normal(0, 3, n), rng.normal(0, 3, n), rng.uniform(2, 40, n),
                  rng.normal(0, 0.3, n), rng.normal(0, 0.3, n), rng.normal(0, 0.3, n)])
    ex = rng.normal(0, 0.2, (4, 12))
    ex[:, 1] -= 1.0
    idx = rng.integers(0, 4, n).astype(np.int32)
    y, pd = ref.world_to_disparity(m8, X, ex.ravel(), idx)
    Xb = np.stack([ref.invert(m8, y[:, i], ex[idx[i]]) for i in range(n)], axis=1)
    out.update(w2d_X=X, w2d_ext=ex, w2d_idx=idx, w2d_y=y, w2d_pd=pd, d2w_X=Xb)
    # detections + update for one map
    G, M = 7, 5
    fit = np.zeros((G, 29))
    for j in range(G):
        fit[j, 0] = rng.uniform(0.05, 1.0)
        fit[j, 1] = rng.choice([0.95, 0.475, 0.0])
        fit[j, 2:8] = [rng.uniform(100, 700), rng.uniform(100, 500), 8.0, 0.0, 0.0, 0.0]
        fit[j, 8:] = packed(spd(rng))
    u = rng.uniform(100, 700, M)
    v = rng.uniform(100, 500, M)
    u[:3] = fit[:3, 2] + rng.normal(0, 3, 3)
    v[:3] = fit[:3, 3] + rng.normal(0, 3, 3)
    det = ref.detections(m8, fit, u, v)
    out.update(det_fit=fit, det_u=u, det_v=v, det_out=det)
    births = np.zeros((M, 43))
    for m in range(M):
        C = np.diag([25.0, 25.0, 2.0, 6.0, 6.0, 0.05])
        births[m, 0] = np.log(1e-6)
        births[m, 1:7] = [u[m], v[m], 8.0, 0, 0, 0]
        births[m, 7:] = C.T.ravel()
    norms = np.array([np.logaddexp.reduce(np.append(det[m * G:(m + 1) * G, 0], np.log(M * 1e-6 + 10.0001 / 600 ** 2)))
                      for m in range(M)])
    upd, flags = ref.update(det, G, births, norms, 1e-4)
    out.update(upd_births=births, upd_norms=norms, upd_out=upd, upd_flags=flags)
    # Mahalanobis / PD / Cholesky / wrap / motion
    K = 40
    A = np.zeros((K, 28))
    B = np.zeros((K, 28))
    for i in range(K):
        A[i, 1:7] = rng.normal(0, 3, 6)
        B[i, 1:7] = A[i, 1:7] + rng.normal(0, 2, 6)
        A[i, 7:] = packed(spd(rng, 0.05))
        B[i, 7:] = packed(spd(rng, 0.05))
    out.update(mahal_a=A, mahal_b=B, mahal_d=np.array([ref.mahal(A[i], B[i]) for i in range(K)]))
    covs = []
    for i in range(K):
        C = spd(rng)
        if i % 3 == 0:
            C[5, 5] = -abs(C[5, 5])
        covs.append(C)
    covs = np.array(covs)
    out.update(pd_cov=covs, pd_out=np.array([ref.is_pos_def(c.T.ravel()) for c in covs]),
               chol_out=np.array([ref.cholesky(c.T.ravel(), 6) for c in covs]))
    ang = rng.uniform(-30, 30, 50)
    out.update(wrap_in=ang, wrap_out=np.array([ref.wrap_angle(a) for a in ang]))
    states = rng.normal(0, 1, (10, 12))
    acc = rng.normal(0, 1, (10, 6))
    out.update(motion_in=states, motion_acc=acc,
               motion_out=np.array([ref.noisy_motion(states[i], 0.5, acc[i]) for i in range(10)]))
    np.savez_compressed(os.path.join(HERE, "ref_kernels.npz"), **out)


if __name__ == "__main__":
    frames()
    ref_kernels()
    print("written", os.listdir(HERE))
