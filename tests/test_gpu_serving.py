"""Serving loop (scphd_server_*): jobs admitted by device-memory budget, advanced in
batched steps while others arrive and retire; each job's result must equal the same
filter stepped alone (bit-exact: the batched kernels run the same arithmetic on the
same random streams)."""
import numpy as np
import pytest

from conftest import gpu_available

pytestmark = pytest.mark.gpu


def _need_gpu():
    if not gpu_available():
        pytest.skip("no CUDA device")


def _jobs(pkg, precision, meas_dim=3):
    out = []
    for i, (n, lm, nf) in enumerate([(40, 10, 5), (96, 16, 8), (17, 8, 4), (64, 20, 7), (130, 12, 6)]):
        sc = pkg.scene.make_scene(n_landmarks=lm, n_frames=nf, clutter_rate=3.0, seed=pkg.scene.scene_seed(4, i))
        cfg = pkg.scene.filter_config(n_parents=n, max_gaussians=96, max_meas=64, clutter_rate=3.0,
                                      precision=precision, calib=sc.calib, seed=700 + i,
                                      particles_per_feature=32 + 8 * i, meas_dim=meas_dim)
        out.append((sc, cfg))
    return out


def _alone(pkg, sc, cfg, meas_dim):
    f = pkg.SCPHDCameraCalibration(cfg)
    for k, z in enumerate(sc.frames):
        f.step(pkg.scene.DT, z[:, 0], z[:, 1], fixed_camera=sc.fixed[k], d=z[:, 2] if meas_dim == 3 else None)
    r = f.particles()
    f.close()
    return r


@pytest.mark.parametrize("precision,meas_dim,graph", [(1, 3, True), (0, 3, False), (1, 2, True)])
def test_served_jobs_equal_jobs_alone(pkg, precision, meas_dim, graph):
    _need_gpu()
    jobs = _jobs(pkg, precision, meas_dim)
    sizes = [pkg.device_bytes(cfg) for _, cfg in jobs]
    # jobs 1 and 4 fit together, so job 4 (arriving at step 5) waits for retirements
    budget = int(sizes[1] + sizes[4] + 1_000_000)
    srv = pkg.SCPHDServer(budget, precision=precision, meas_dim=meas_dim, use_graph=graph)
    ids = {}
    arrivals = {0: [0, 1], 2: [2, 3], 5: [4]}   # step index -> jobs arriving then
    saw_queue = False
    for it in range(200):
        for i in arrivals.get(it, []):
            sc, cfg = jobs[i]
            ids[i] = srv.submit(cfg, [z[:, :meas_dim] for z in sc.frames], sc.fixed, pkg.scene.DT)
        st = srv.stats()
        saw_queue |= st["queued"] > 0 and st["running"] > 0
        n = srv.step()
        if n == 0 and it > max(arrivals) and srv.stats()["queued"] == 0:
            break
    srv.drain()
    st = srv.stats()
    assert st["done"] == len(jobs) and st["running"] == 0 and st["queued"] == 0
    assert saw_queue, "the budget never held a job back"
    assert st["rebuilds"] >= 3
    ms, nj = srv.step_times()
    assert len(ms) == st["steps"] and np.all(ms > 0) and nj.sum() == st["job_frames"]
    assert st["job_frames"] == sum(sc.n_frames for sc, _ in jobs)
    for i, (sc, cfg) in enumerate(jobs):
        assert srv.status(ids[i]) == (pkg.JOB_DONE, sc.n_frames)
        s_srv, lw_srv = srv.result(ids[i])
        s_one, lw_one = _alone(pkg, sc, cfg, meas_dim)
        assert np.array_equal(s_srv, s_one), f"job {i}: states differ from the job alone"
        assert np.array_equal(lw_srv, lw_one), f"job {i}: log-weights differ from the job alone"
    srv.close()


def test_server_refusals(pkg):
    _need_gpu()
    jobs = _jobs(pkg, 1)
    sc, cfg = jobs[1]
    frames = [z for z in sc.frames]
    small = pkg.SCPHDServer(pkg.device_bytes(cfg) // 2, precision=1)
    with pytest.raises(pkg.ScphdError):
        small.submit(cfg, frames, sc.fixed, pkg.scene.DT)       # larger than the whole budget
    small.close()
    srv = pkg.SCPHDServer(1 << 34, precision=0)
    with pytest.raises(pkg.ScphdError):
        srv.submit(cfg, frames, sc.fixed, pkg.scene.DT)         # precision differs
    c32 = cfg.copy()
    c32.precision = 0
    srv.submit(c32, frames, sc.fixed, pkg.scene.DT)
    with pytest.raises(pkg.ScphdError):
        srv.submit(c32, frames, sc.fixed, 0.25)                 # another dt
    big = [np.zeros((500, 3))] + frames[1:]
    with pytest.raises(pkg.ScphdError):
        srv.submit(c32, big, sc.fixed, pkg.scene.DT)            # frame over max_measurements
    while srv.step():
        pass
    srv.drain()
    assert srv.stats()["done"] == 1
    srv.close()
