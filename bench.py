#!/usr/bin/env python
"""Benchmark of the SC-PHD calibration filter step on B200.

One step = one filter frame (predict + update + resample) of the single-filter
workload `plain_c1` (4096 parent particles, 200 landmarks, clutter rate 50 per
frame, <= 256 Gaussians per parent, 100 samples per Gaussian, (u,v,d)
measurements, FP32 Kalman/merge, FP64 weights and resampling prefix).  Metric:
Gaussian-measurement updates/s, one unit = one (parent, prior Gaussian,
measurement) triple, counted on the device for each frame.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

N > 1 runs under torchrun, one independent filter replica per GPU (weak scaling;
the filters share nothing, so there is no data-path collective); value is the
sum of all ranks' units over the max of the ranks' device times.
"""
from __future__ import annotations

import argparse
import datetime
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "scphd-camera-calibration_b200")
METRIC = "Gaussian-measurement updates/s"
UNIT = "updates/s"


def load_package():
    if "scphd_b200" in sys.modules:
        return sys.modules["scphd_b200"]
    spec = importlib.util.spec_from_file_location(
        "scphd_b200", os.path.join(PKG_DIR, "__init__.py"), submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["scphd_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def read_peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as fh:
            pk = json.load(fh)
        return float(pk["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200",
                 "-i", str(self.gpu)], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        with open(self.path) as fh:
            for line in fh:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) < 9:
                    continue
                try:
                    sm.append(float(parts[1]))
                    smax.append(float(parts[2]))
                except ValueError:
                    continue
                for nm, val in zip(names, parts[5:9]):
                    if val.lower().startswith("active"):
                        reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def combine_ranks(ms_total: float, units: float, e2e_ms: float, e2e_units: float, dist=None, device=None):
    """Whole-job figures over the ranks of a replica run: device times take the MAX
    over ranks (the job ends with its slowest rank), units the SUM.  Works with any
    torch.distributed backend (NCCL on GPUs, gloo in the CPU tests)."""
    import torch
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return ms_total, units, e2e_ms, e2e_units
    t = torch.tensor([ms_total, units, e2e_ms, e2e_units], dtype=torch.float64, device=device)
    mx, sm = t.clone(), t.clone()
    dist.all_reduce(mx, op=dist.ReduceOp.MAX)
    dist.all_reduce(sm, op=dist.ReduceOp.SUM)
    return mx[0].item(), sm[1].item(), mx[2].item(), sm[3].item()


def replica_seed_index(rank: int) -> int:
    """Filter index of a rank's replica: each rank runs its own seeded scene."""
    return rank


CPU_SAMPLE_PARENTS = 32   # parents of the workload's scene in the timed CPU sample


def cpu_model() -> str:
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def _oracle_step(o, sc, k, DT):
    z = sc.frames[k]
    g = int(o.map_sizes().sum())
    t0 = time.perf_counter()
    o.predict(DT)
    o.update(z[:, 0], z[:, 1], sc.fixed[k], d=z[:, 2])
    o.resample()
    return g * z.shape[0], time.perf_counter() - t0


def cpu_sample(pkg, workload: str, sample_parents: int, prefill: int, frames: int, threads_list):
    """Units/s of the FP64 oracle (the CPU restatement of the reference's filter step,
    with the same map capacity as the device) on a bounded sample of the workload:
    the workload's scene and configuration with `sample_parents` parents.  `prefill`
    untimed frames (all threads) populate the maps; their end state is copied into a
    fresh oracle per thread count, and the same `frames` frames are timed from it, so
    every thread count does identical work.  Units/s is additive over parents."""
    sys.path.insert(0, ROOT)
    from oracle import oracle as orc
    orc.build()
    all_threads = os.cpu_count() or 1
    sc, cfg = pkg.scene.workload(workload, precision=pkg.SCPHD_FP64, n_frames=prefill + frames)
    cfg.n_parents = min(int(cfg.n_parents), sample_parents)
    orc.set_threads(all_threads)
    o = orc.Oracle(cfg)
    for k in range(prefill):
        _oracle_step(o, sc, k, pkg.scene.DT)
    snap = o.state()
    out = {}
    for th in threads_list:
        used = orc.set_threads(th)
        oc = orc.Oracle(cfg)
        oc.load(snap)
        units, secs = 0, []
        for k in range(prefill, prefill + frames):
            u, dt = _oracle_step(oc, sc, k, pkg.scene.DT)
            units += u
            secs.append(dt)
        out[th] = {"value": units / sum(secs), "threads": used, "units": units, "seconds": sum(secs),
                   "ms_per_frame": 1e3 * sum(secs) / len(secs), "truncations": oc.truncations()}
    orc.set_threads(all_threads)
    return out, int(cfg.n_parents)


def run_reference(args):
    """--impl reference: the reference's filter step on the host cores -- the oracle,
    the project's C++ restatement of it (the reference's own program cannot be built
    here: it needs libconfig, matio, the CUDA SDK helpers and compute_20) -- on the
    same bounded sample of the workload as the b200 arm's cpu_baseline leg, all host
    threads.  Config 0 (plain_c0) is host-sized and runs at full size from frame 0."""
    world, rank, _ = dist_env()
    if rank != 0:
        return
    pkg = load_package()
    threads = os.cpu_count() or 1
    full = args.workload == "plain_c0"
    prefill = (0 if full else args.cpu_prefill) + args.warmup   # warm-up frames are untimed
    sample = 1 << 30 if full else CPU_SAMPLE_PARENTS
    res, n_used = cpu_sample(pkg, args.workload, sample, prefill, args.steps, [threads])
    r = res[threads]
    n_full = int(pkg.scene.WORKLOADS[args.workload]["n_parents"])
    line = {
        "impl": "reference", "metric": METRIC, "value": r["value"], "unit": UNIT, "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_frame"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": args.workload, "n_parents": n_used, "n_parents_full": n_full,
                   "note": "parent sample of the workload; units/s is additive over parents"},
        "cpu_baseline": {"value": r["value"], "unit": UNIT, "cores": r["threads"], "kind": "port",
                         "cpu_model": cpu_model(), "nproc": threads,
                         "sample": f"{n_used} of {n_full} parents of {args.workload}, {prefill} untimed frames "
                                   f"(map population and warm-up), then {args.steps} timed frames "
                                   f"({r['seconds']:.1f} s)"},
        "e2e": {"value": r["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def measurements_note(pkg, workload):
    """Why a scene's measured count per frame is below landmarks x pD + clutter."""
    w = pkg.scene.WORKLOADS[workload]
    expect = w["n_landmarks"] * 0.95 + w["clutter"]
    return (f"the landmark box (10 x 10 x 10 m, 2-12 m ahead) extends beyond the 640x480 field of view, "
            f"so fewer landmarks are seen than the ~{expect:.0f} measurements per frame the config's "
            f"{w['n_landmarks']} landmarks (pD 0.95) and clutter {w['clutter']:g} would give; "
            f"units are G x M, so this understates throughput")


def run_b200(args):
    import torch
    world, rank, local = dist_env()
    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=180),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    pkg = load_package()
    prec = pkg.SCPHD_FP32 if args.precision == "fp32" else pkg.SCPHD_FP64
    K, W = args.steps, args.warmup
    n_frames = args.prefill + W + 4 * K + 1
    sc, cfg = pkg.scene.workload(args.workload, precision=prec, filter_index=replica_seed_index(rank),
                                 n_frames=n_frames)
    if args.parents:
        cfg.n_parents = args.parents   # smaller case for profiler captures; not a bench line
    cfg.device = local
    filt = pkg.SCPHDCameraCalibration(cfg)
    filt.set_fused({"staged": 0, "fused": 1}[args.update_path])
    dev = torch.device("cuda", local)
    dframes = []
    for z in sc.frames:
        zt = torch.tensor(np.ascontiguousarray(z.T), dtype=torch.float64, device=dev).contiguous()
        dframes.append(zt)
    torch.cuda.synchronize()
    k = 0

    def dstep():
        nonlocal k
        zt = dframes[k]
        filt.step_device(pkg.scene.DT, zt[0].data_ptr(), zt[1].data_ptr(), zt[2].data_ptr(), zt.shape[1],
                         sc.fixed[k])
        k += 1

    for _ in range(args.prefill + W):
        dstep()
    filt.synchronize()
    shapes = filt.launch_shapes()   # tuned on the untimed frames
    stream = torch.cuda.ExternalStream(filt.stream_handle)
    c0 = filt.counters()
    l0 = pkg.kernel_launches()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(K + 1)]
    timed_meas = [int(sc.frames[k + i].shape[0]) for i in range(K)]
    ev[0].record(stream)
    for i in range(K):
        dstep()
        ev[i + 1].record(stream)
    ev[K].synchronize()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clk = clocks.stop()
    ms_total = ev[0].elapsed_time(ev[K])
    frame_ms = [ev[i].elapsed_time(ev[i + 1]) for i in range(K)]
    c1 = filt.counters()
    launches = pkg.kernel_launches() - l0
    units = int(c1[6] - c0[6])
    # per-stage device times (events around each stage on the filter's stream)
    filt.set_profiling(True)   # profiling runs the stage kernels one by one, each timed
    c_p0 = filt.counters()
    prof_meas = 0
    for _ in range(K):
        prof_meas += int(sc.frames[k].shape[0])
        dstep()
    stages = filt.stage_times()
    filt.set_profiling(False)
    c_p1 = filt.counters()
    # the fused update's own time (when the tuner chose it): events around each update
    # (measurement conversion, the fused kernel, the parent-weight kernel)
    fused_ms = None
    if shapes.get("fused"):
        fused_ms = 0.0
        ea, eb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for _ in range(K):
            zt = dframes[k]
            filt.predict(pkg.scene.DT)
            ea.record(stream)
            filt.update_device(zt[0].data_ptr(), zt[1].data_ptr(), zt[2].data_ptr(), zt.shape[1], sc.fixed[k])
            eb.record(stream)
            filt.resample()
            eb.synchronize()
            fused_ms += ea.elapsed_time(eb)
            k += 1
    # end to end through the host-array C ABI: H2D of the frame, step, D2H of the result.
    # Each step's parent states and log-weights are copied into one of two page-locked
    # buffers on the filter's stream and read on the host one step later (while the next
    # step runs); the last step's result is read before the clock stops.
    h2d = d2h = 0
    ee0, ee1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ce0 = filt.counters()
    N = int(cfg.n_parents)
    res_bufs = [(torch.empty((N, 12), dtype=torch.float64, pin_memory=True),
                 torch.empty(N, dtype=torch.float64, pin_memory=True)) for _ in range(2)]
    res_ev = [torch.cuda.Event(), torch.cuda.Event()]
    checksum = 0.0
    torch.cuda.synchronize()
    ee0.record(stream)
    for i in range(K):
        z = sc.frames[k]
        filt.step(pkg.scene.DT, z[:, 0], z[:, 1], sc.fixed[k], d=z[:, 2])
        st, lw = res_bufs[i % 2]
        filt.particles_async(st.data_ptr(), lw.data_ptr())
        res_ev[i % 2].record(stream)
        h2d += 3 * 8 * z.shape[0]
        d2h += st.numel() * 8 + lw.numel() * 8
        if i > 0:   # the previous step's result, on the host
            res_ev[(i - 1) % 2].synchronize()
            checksum += float(res_bufs[(i - 1) % 2][1][0])
        k += 1
    res_ev[(K - 1) % 2].synchronize()
    checksum += float(res_bufs[(K - 1) % 2][1][0])
    ee1.record(stream)
    ee1.synchronize()
    if not np.isfinite(checksum):
        raise RuntimeError("non-finite log-weight read back in the end-to-end pass")
    ce1 = filt.counters()
    e2e_ms = ee0.elapsed_time(ee1)
    e2e_units = int(ce1[6] - ce0[6])

    ms_all, units_all, e2e_ms_all, e2e_units_all = combine_ranks(ms_total, float(units), e2e_ms,
                                                                 float(e2e_units), dist, dev)
    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return
    value = units_all / (ms_all / 1e3)
    e2e_value = e2e_units_all / (e2e_ms_all / 1e3)

    # rooflines.  Algorithmic bytes of each stage over the profiled frames, from the
    # device counters (Gaussians fitted, clouds read and written, survivors, merged
    # components): the compulsory reads and writes of the rows each stage consumes and
    # produces, s bytes per value (4 in FP32).
    peak, peak_kind = read_peaks()
    sz = 4 if prec == pkg.SCPHD_FP32 else 8
    P = int(cfg.particles_per_feature)
    N = int(cfg.n_parents)
    fitted = c_p1[10] - c_p0[10]
    rd, wr = c_p1[8] - c_p0[8], c_p1[9] - c_p0[9]
    surv = c_p1[7] - c_p0[7]
    merged = c_p1[11] - c_p0[11]
    ell_vals = N * prof_meas   # normalisers written by the likelihood, read by the merge
    stage_bytes = {
        # map entries (merged component: 28 values; carried cloud: weight) read, fitted
        # rows (29) written, carried clouds read and candidate clouds written (7 P each)
        "cloud_fit": fitted * (28 + 29) * sz + (rd + wr) * 7 * P * sz,
        # fitted rows (29) read, Kalman-term rows (48) and likelihood rows (12) written
        "kalman_terms": fitted * (29 + 48 + 12) * sz,
        # likelihood rows (12) read, normalisers written, survivors (rank + weight) written
        "likelihood": fitted * 12 * sz + ell_vals * sz + surv * (4 + sz),
        # survivors read with their Gaussians' gain, posterior covariance and fitted mean
        # (18 + 21 + 6); normalisers and fitted weight and pD read; merged rows (28) written
        # to the merge output and the new map; carried entries written (weight + reference)
        "merge": surv * (4 + sz + 45 * sz) + ell_vals * sz + fitted * 2 * sz + merged * 28 * sz * 2
                 + fitted * (sz + 4),
    }
    stage_roofline = {}
    for nm, by in stage_bytes.items():
        ms, nl = stages.get(nm, (0.0, 0))
        if nl and ms > 0:
            gbs = by / nl / (ms / nl / 1e3) / 1e9
            stage_roofline[nm] = {"bytes_per_launch": by / nl, "ms_per_launch": ms / nl, "achieved_gbs": gbs,
                                  "frac": gbs / peak}
    if fused_ms:
        # one launch per frame covers the four stages of every parent
        name, n_launch = "fused_update", K
        per_launch = sum(stage_bytes.values()) / K
        w_ms = stages.get("weights", (0.0, 1))
        avg_ms = fused_ms / K - w_ms[0] / max(1, w_ms[1])   # less the parent-weight kernel
    else:
        dom = max(((nm, v) for nm, v in stages.items() if nm in stage_bytes), key=lambda kv: kv[1][0])
        name, (stage_ms, n_launch) = dom
        per_launch = stage_bytes[name] / max(1, n_launch)
        avg_ms = stage_ms / max(1, n_launch)
    achieved = per_launch / (avg_ms / 1e3) / 1e9 if avg_ms > 0 else 0.0
    # compute side: algorithmic FP32 flops (about 250 per cloud sample: draw, two
    # camera transforms, prediction, moments) against the nominal FP32 CUDA-core peak
    # (148 SMs x 128 lanes x 2 flops x 1.965 GHz); the cloud fit is issue-bound, not HBM-bound
    fp32_peak_tflops = 148 * 128 * 2 * 1.965e9 / 1e12
    flops = fitted * P * 250.0 / max(1, K)
    compute = {"flops_per_launch": flops, "achieved_tflops": flops / (avg_ms / 1e3) / 1e12 if avg_ms > 0 else 0.0,
               "peak_tflops": fp32_peak_tflops, "peak_source": "nominal FP32 CUDA-core rate",
               "flops_counted": "250 per cloud sample (the cloud fit's sampling, transforms, prediction, moments)"}
    compute["frac"] = compute["achieved_tflops"] / fp32_peak_tflops
    traffic = None   # recorded for full-size plain_c1 launches only
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp) and args.workload == "plain_c1" and not args.parents:
        with open(tp) as fh:
            tj = json.load(fh)
        tr = tj.get(name)
        if tr:
            traffic = tr.get("bytes_per_launch_scaled")
        # issue side of the cloud fit: the warp instructions per fitted Gaussian of the
        # recorded capture x the Gaussians fitted per launch, over the launch's issue slots
        # (148 SMs x 4 schedulers x the median SM clock sampled in the timed region)
        ti = tj.get("cloud_fit_issue")
        if ti and name == "cloud_fit" and avg_ms > 0 and clk and clk.get("sm_mhz"):
            inst = ti["warp_instructions_per_gaussian"] * fitted / max(1, K)
            slots = 148 * 4 * clk["sm_mhz"] * 1e6 * avg_ms / 1e3
            compute["issue"] = {"warp_instructions_per_launch": inst, "issue_slots_per_launch": slots,
                                "frac": inst / slots,
                                "instructions_source": "profiles/k_cloud_fit_plain_c1_512parents.md"}

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        res, n_used = cpu_sample(pkg, args.workload, CPU_SAMPLE_PARENTS, args.cpu_prefill, args.cpu_frames,
                                 [threads, 1])
        ra, r1 = res[threads], res[1]
        cpu = {"value": ra["value"], "unit": UNIT, "cores": ra["threads"], "kind": "port",
               "threads_all": {"threads": ra["threads"], "value": ra["value"], "ms_per_frame": ra["ms_per_frame"]},
               "threads_1": {"threads": 1, "value": r1["value"], "ms_per_frame": r1["ms_per_frame"]},
               "cpu_model": cpu_model(), "nproc": threads,
               "sample": f"{n_used} of {cfg.n_parents} parents of {args.workload}, {args.cpu_prefill} untimed "
                         f"frames to populate the maps, then the same {args.cpu_frames} frames timed at "
                         f"{ra['threads']} threads ({ra['seconds']:.1f} s) and at 1 thread ({r1['seconds']:.1f} s)"}

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
        "ms_per_step": ms_all / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": args.precision, "data": "synthetic",
        "config": {"workload": args.workload, "n_parents": int(cfg.n_parents),
                   "landmarks": int(pkg.scene.WORKLOADS[args.workload]["n_landmarks"]),
                   "clutter_rate": float(pkg.scene.WORKLOADS[args.workload]["clutter"]),
                   "max_gaussians": int(cfg.max_gaussians),
                   "particles_per_feature": P, "meas_dim": int(cfg.meas_dim), "prefill_frames": args.prefill,
                   "mean_gaussians_per_parent": fitted / max(1, K) / cfg.n_parents,
                   "mean_measurements": float(np.mean(timed_meas)),
                   "measurements_note": measurements_note(pkg, args.workload),
                   "l2": "no flush: the resident map/cloud state is larger than L2",
                   "parallelism": f"replicas{world}", "launch_shapes": shapes},
        "frame_ms": {"p50": float(np.percentile(frame_ms, 50)), "p99": float(np.percentile(frame_ms, 99)),
                     "max": float(max(frame_ms))},
        "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d // K, "d2h_bytes_per_step": d2h // K},
        "gpu_launches": int(launches),
        "roofline": {"bound": "hbm", "kernel": name, "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": peak_kind,
                     "algorithmic_bytes_per_launch": per_launch, "avg_launch_ms": avg_ms,
                     "compute": compute},
        "stage_ms_per_frame": {k2: v[0] / max(1, v[1]) for k2, v in stages.items()},
        "stage_roofline": stage_roofline,
        "cpu_baseline": cpu,
        "clocks": clk,
        "counters": {"map_truncations": int(c1[0] - c0[0]), "scratch_overflows": int(c1[1]),
                     "max_survivors_per_parent": int(c1[13]), "max_survivors_capacity": int(cfg.max_survivors),
                     "clouds_read_per_parent_frame": float(c1[8] - c0[8]) / (K * cfg.n_parents),
                     "clouds_written_per_parent_frame": float(c1[9] - c0[9]) / (K * cfg.n_parents),
                     "fitted_per_parent_frame": float(c1[10] - c0[10]) / (K * cfg.n_parents),
                     "merged_per_parent_frame": float(c1[11] - c0[11]) / (K * cfg.n_parents)},
    }
    filt.close()
    if world == 1 and not args.no_extras:
        line.update(extra_workloads(args, pkg))
    print(json.dumps(line), flush=True)
    if dist:
        dist.destroy_process_group()


def extra_workloads(args, pkg):
    """Short runs of the many-filter and serving workloads, reported beside the
    single-filter line: 64 filters of the plain_c0 shape (256 parents, <= 64
    Gaussians, 50 landmarks, clutter 10) batched against the same filters stepped one
    at a time, and a serving window of Poisson arrivals with per-frame latencies."""
    import copy
    import torch
    out = {}
    a = copy.copy(args)
    a.workload, a.filters, a.steps, a.warmup, a.prefill = "batched_c0x64", 64, 10, 3, 20
    r = run_batched(a, pkg)
    out["batched_c0x64"] = {
        "value": r["batched"]["value"], "unit": UNIT, "plain_value": r["plain"]["value"],
        "batched_over_plain": r["batched_over_plain"], "filters": r["filters"], "parents": r["parents"],
        "waves": r["waves"], "frame_ms": r["wave_frame_ms"], "steps": r["batched"]["steps"],
        "e2e": r["e2e"]["value"], "gpu_launches": r["gpu_launches"],
        "note": "batched = one batch step per frame for all 64 filters (graph-replayed); plain = the same "
                "filters stepped one after another; frames alternate in pairs so both see maps of one size"}
    torch.cuda.empty_cache()
    a = copy.copy(args)
    a.serve_seconds = args.extra_serve_seconds
    sv = run_serving(a, pkg)
    out["serving_c4"] = {
        "value": sv["value"], "unit": UNIT, "window_s": sv["config"]["window_s"],
        "frame_latency_ms": sv["frame_latency_ms"], "admission_wait_s": sv["admission_wait_s"],
        "jobs_admitted": sv["config"]["admitted"], "jobs_completed": sv["config"]["completed"],
        "mean_jobs_per_step": sv["mean_jobs_per_step"], "device_busy_fraction": sv["device_busy_fraction"],
        "note": "Poisson arrivals at 20 jobs/s from an empty server; value = updates over the wall-clock "
                "window; latency = device time of the batched step that advanced a job's frame"}
    return out


def run_batched(args, pkg, quiet=False):
    """Many-filter workload: 64 filters of uneven size (batched_specs), grouped into
    device-resident waves under an 80% HBM budget.  Each wave is one SCPHDBatch
    stepped from a captured CUDA graph (seven kernels per frame for all its filters).
    Timed per wave: K pairs of batched frames alternating with K pairs of frames in
    which the same filters are stepped plain, one filter at a time (device events on
    the batch stream), then K batched frames end to end from host arrays with the
    parent states read back.  Rates are all waves' units over all waves' times."""
    import torch
    dev = torch.device("cuda", 0)
    prec = pkg.SCPHD_FP32 if args.precision == "fp32" else pkg.SCPHD_FP64
    K, W, PF = args.steps, args.warmup, args.prefill
    n_pairs = max(1, (K + 1) // 2)
    n_frames = PF + W + 4 * n_pairs + K
    if args.workload == "batched_c0x64":
        # the single-filter workload plain_c0 (256 parents, 50 landmarks, clutter 10,
        # <= 64 Gaussians), 64 filters on their own seeded scenes
        specs = [dict(index=i, n_parents=256, n_landmarks=50, clutter=10.0) for i in range(args.filters)]
        built = [pkg.scene.spec_filter(sp, n_frames, prec, max_gaussians=64, config_index=0,
                                       survivors_per_gaussian=6) for sp in specs]
    else:
        specs = pkg.scene.batched_specs(args.filters)
        built = [pkg.scene.spec_filter(sp, n_frames, prec) for sp in specs]
    sizes = [pkg.device_bytes(cfg) for _, cfg in built]
    free, total = torch.cuda.mem_get_info(dev)
    budget = int(0.8 * free)
    waves = pkg.scene.plan_waves(sizes, budget)
    DT = pkg.scene.DT
    res = {"units_b": 0, "ms_b": 0.0, "units_p": 0, "ms_p": 0.0, "units_e": 0, "ms_e": 0.0,
           "frame_ms": [], "launches": 0, "h2d": 0, "d2h": 0, "truncations": 0, "overflows": 0}
    clocks = ClockSampler(0)
    clocks.start()
    for wave in waves:
        scs = [built[i][0] for i in wave]
        fs = [pkg.SCPHDCameraCalibration(built[i][1]) for i in wave]
        dfr = [[torch.tensor(np.ascontiguousarray(z.T), dtype=torch.float64, device=dev) for z in sc.frames]
               for sc in scs]
        torch.cuda.synchronize()
        batch = pkg.SCPHDBatch(fs, use_graph=True)
        stream = torch.cuda.ExternalStream(batch.stream_handle())
        k = 0
        # each frame's device pointers, gathered once: the timed steps then hold no tensor
        # indexing on the host (both forms get the same argument lists)
        fargs = [[(z[kk][0].data_ptr(), z[kk][1].data_ptr(), z[kk][2].data_ptr(), z[kk].shape[1], sc.fixed[kk])
                  for z, sc in zip(dfr, scs)] for kk in range(n_frames)]

        def bstep():
            nonlocal k
            batch.step_device(DT, fargs[k])
            k += 1

        def pstep():
            # the same frame for every member, stepped plain: one filter at a time
            nonlocal k
            for f, (pu, pv, pd, n, fixed) in zip(fs, fargs[k]):
                f.step_device(DT, pu, pv, pd, n, fixed)
            k += 1

        for _ in range(PF + W):
            bstep()
        batch.synchronize()
        l0 = pkg.kernel_launches()
        lb = 0
        # batched and plain frames alternate in pairs (a fixed-camera and a moving-camera
        # frame each), so that both forms are timed on maps of the same size; members
        # stepped plain run on the batch's stream, one filter after another
        for i in range(n_pairs):
            for form in ("b", "p"):
                c0 = [f.counters() for f in fs]
                e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
                e[0].record(stream)
                for j in range(2):
                    (bstep if form == "b" else pstep)()
                    e[j + 1].record(stream)
                e[2].synchronize()
                c1 = [f.counters() for f in fs]
                res["ms_" + form] += e[0].elapsed_time(e[2])
                res["units_" + form] += sum(int(b[6] - a[6]) for a, b in zip(c0, c1))
                if form == "b":
                    res["frame_ms"] += [e[0].elapsed_time(e[1]), e[1].elapsed_time(e[2])]
                    res["truncations"] += sum(int(b[0] - a[0]) for a, b in zip(c0, c1))
                    lb += 14   # seven kernels per batched frame, two frames
        res["launches"] += lb
        res["overflows"] += sum(int(f.counters()[1]) for f in fs)
        # end to end: host frames in, parent states out, through the public API.  The
        # frames are host arrays (columns made contiguous before the clock starts, as a
        # caller holds them); each step's parent states and log-weights of every member
        # are copied into one of two page-locked buffer sets on the batch's stream and read
        # on the host one step later, while the next step runs.
        c1 = [f.counters() for f in fs]
        hframes = [[(np.ascontiguousarray(sc.frames[kk][:, 0]), np.ascontiguousarray(sc.frames[kk][:, 1]),
                     np.ascontiguousarray(sc.frames[kk][:, 2]), sc.fixed[kk]) for sc in scs]
                   for kk in range(k, k + K)]
        res_bufs = [[(torch.empty((f.n_parents, 12), dtype=torch.float64, pin_memory=True),
                      torch.empty(f.n_parents, dtype=torch.float64, pin_memory=True)) for f in fs] for _ in range(2)]
        res_ev = [torch.cuda.Event(), torch.cuda.Event()]
        checksum = 0.0
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        for i in range(K):
            batch.step(DT, hframes[i])
            res["h2d"] += sum(3 * 8 * fr[0].shape[0] for fr in hframes[i])
            for f, (st, lw) in zip(fs, res_bufs[i % 2]):
                f.particles_async(st.data_ptr(), lw.data_ptr())
                res["d2h"] += st.numel() * 8 + lw.numel() * 8
            res_ev[i % 2].record(stream)
            if i > 0:   # the previous step's results, on the host
                res_ev[(i - 1) % 2].synchronize()
                checksum += sum(float(lw[0]) for _, lw in res_bufs[(i - 1) % 2])
            k += 1
        res_ev[(K - 1) % 2].synchronize()
        checksum += sum(float(lw[0]) for _, lw in res_bufs[(K - 1) % 2])
        e1.record(stream)
        e1.synchronize()
        if not np.isfinite(checksum):
            raise RuntimeError("non-finite log-weight read back in the end-to-end pass")
        c2 = [f.counters() for f in fs]
        res["ms_e"] += e0.elapsed_time(e1)
        res["units_e"] += sum(int(b[6] - a[6]) for a, b in zip(c1, c2))
        batch.close()
        for f in fs:
            f.close()
        del dfr
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    clk = clocks.stop()
    fm = res["frame_ms"]
    out = {
        "workload": args.workload, "filters": len(specs), "parents": int(sum(sp["n_parents"] for sp in specs)),
        "waves": [len(w) for w in waves], "hbm_budget_gb": budget / 1e9,
        "device_gb": sum(sizes) / 1e9,
        "batched": {"value": res["units_b"] / (res["ms_b"] / 1e3), "ms_per_step": res["ms_b"] / (2 * n_pairs),
                    "steps": 2 * n_pairs},
        "plain": {"value": res["units_p"] / (res["ms_p"] / 1e3), "ms_per_step": res["ms_p"] / (2 * n_pairs)},
        "batched_over_plain": (res["units_b"] / res["ms_b"]) / (res["units_p"] / res["ms_p"]),
        "wave_frame_ms": {"p50": float(np.percentile(fm, 50)), "p99": float(np.percentile(fm, 99))},
        "e2e": {"value": res["units_e"] / (res["ms_e"] / 1e3), "unit": UNIT,
                "h2d_bytes_per_step": res["h2d"] // K, "d2h_bytes_per_step": res["d2h"] // K},
        "gpu_launches": int(res["launches"]), "clocks": clk,
        "counters": {"map_truncations": res["truncations"], "scratch_overflows": res["overflows"]},
    }
    return out


def run_serving(args, pkg):
    """Serving workload: Poisson arrivals (20 jobs/s for --serve-seconds) of
    calibration jobs of uneven size, admitted first come, first served by the
    server under an 80% HBM budget and advanced in batched steps.  Scenes are
    generated when a job is handed to the server (host memory stays bounded while
    the offered load exceeds what the device serves); a job's wait counts from its
    arrival time.  Reports updates/s over the serving window (wall clock), per
    job-frame latency (device time of the step that advanced it), admission waits."""
    import torch
    prec = pkg.SCPHD_FP32 if args.precision == "fp32" else pkg.SCPHD_FP64
    arrivals = pkg.scene.serving_arrivals(seconds=args.serve_seconds)
    free, total = torch.cuda.mem_get_info(torch.device("cuda", 0))
    budget = int(0.8 * free)
    srv = pkg.SCPHDServer(budget, precision=prec, meas_dim=3, use_graph=True)
    DT = pkg.scene.DT
    # the clients: a producer thread turns arrivals into job data, in arrival order
    import queue as _queue
    import threading
    ready = _queue.Queue(maxsize=4)
    stop = threading.Event()

    def produce():
        for ta, sp in arrivals:
            sc, cfg = pkg.scene.spec_filter(sp, sp["n_frames"], prec, config_index=4)
            while not stop.is_set():
                try:
                    ready.put((ta, sc, cfg), timeout=0.1)
                    break
                except _queue.Full:
                    pass
            if stop.is_set():
                return

    producer = threading.Thread(target=produce, daemon=True)
    producer.start()
    held = None
    submitted, admitted_at, arrival_of = [], {}, {}
    clocks = ClockSampler(0)
    clocks.start()
    t0 = time.perf_counter()
    while True:
        now = time.perf_counter() - t0
        if now >= args.serve_seconds:
            break
        # hand arrived jobs to the server while its own queue is short
        while len(submitted) - len(admitted_at) < 2:
            if held is None:
                try:
                    held = ready.get_nowait()
                except _queue.Empty:
                    break
            if held[0] > now:
                break
            ta, sc, cfg = held
            jid = srv.submit(cfg, sc.frames, sc.fixed, DT)
            submitted.append(jid)
            arrival_of[jid] = ta
            held = None
        for jid in submitted:
            if jid not in admitted_at and srv.status(jid)[0] != pkg.JOB_QUEUED:
                admitted_at[jid] = time.perf_counter() - t0
        if srv.step() == 0:
            time.sleep(0.001)
    stop.set()
    srv.drain()
    wall = time.perf_counter() - t0
    clk = clocks.stop()
    st = srv.stats()
    ms, nj = srv.step_times()
    lat = np.repeat(ms, nj) if len(ms) else np.zeros(1)
    waits = [admitted_at[j] - arrival_of[j] for j in admitted_at]
    srv.close()
    line = {
        "metric": METRIC, "value": st["units"] / wall, "unit": UNIT, "n_gpus": 1, "steps": int(st["steps"]),
        "warmup": 0, "ms_per_step": float(np.mean(ms)) if len(ms) else None, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
        "config": {"workload": "serving_c4", "arrival_rate_per_s": 20.0, "window_s": args.serve_seconds,
                   "arrived": sum(1 for t, _ in arrivals if t <= wall), "handed_to_server": len(submitted),
                   "admitted": len(admitted_at), "completed": st["done"], "hbm_budget_gb": budget / 1e9,
                   "note": "value = updates over the wall-clock serving window, starting from an empty server"},
        "frame_latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                             "max": float(lat.max())},
        "admission_wait_s": {"p50": float(np.percentile(waits, 50)) if waits else None,
                             "p99": float(np.percentile(waits, 99)) if waits else None},
        "device_busy_fraction": float(ms.sum() / 1e3 / wall) if len(ms) else 0.0,
        "job_frames": int(st["job_frames"]), "batch_rebuilds": int(st["rebuilds"]),
        "mean_jobs_per_step": float(nj.mean()) if len(nj) else 0.0, "clocks": clk,
    }
    return line


def _match_rows(A, B, mean_cols, var_cols):
    """Pair the rows of two mixtures (nearest mean in units of A's standard
    deviations); returns per-pair |dmean|/sd and relative variance errors."""
    if not len(A) or not len(B):
        return np.zeros(0), np.zeros(0)
    sd = np.sqrt(np.maximum(A[:, var_cols], 1e-30))
    d = np.abs(B[None, :, mean_cols] - A[:, None, mean_cols]) / sd[:, None, :]
    j = np.argmin(d.max(axis=2), axis=1)
    dm = d[np.arange(len(A)), j].ravel()
    dv = (np.abs(B[j][:, var_cols] - A[:, var_cols]) / np.maximum(np.abs(A[:, var_cols]), 1e-30)).ravel()
    return dm, dv


def _capture_state(f):
    """Whole filter state as set_state takes it (Euclidean clouds)."""
    st, lw = f.particles()
    sizes = f.map_sizes()
    ws, cl, om = [], [], []
    for p in range(f.n_parents):
        if sizes[p]:
            ws.append(f.map_weights(p))
            x, o = f.map_clouds(p)
            cl.append(x)
            om.append(o)
    cat = lambda xs, shp: np.concatenate(xs) if xs else np.zeros(shp)
    P = int(f.config.particles_per_feature)
    return st, lw, sizes, cat(ws, (0,)), cat(cl, (0, 6, P)), cat(om, (0, P))


def run_precision(args, pkg):
    """Precision study on precision_c3 (16384 parents, 400 landmarks, <= 512
    Gaussians, clutter 100, 300 frames).  FP32 mode computes the Kalman algebra,
    refits and merge in FP32; parent states, the log-weight accumulation and the
    resampling prefix sum stay FP64 in both modes.

    (1) One-step errors: a 256-parent FP64 filter on the same scene is run; at
    checkpoint frames its whole state is loaded (set_state) into a fresh FP64 and a
    fresh FP32 filter, both run the next predict + update, and every output is
    compared: parent log-likelihoods, per-measurement log normalisers, fitted
    mixtures (rows correspond one to one) and merged mixtures (rows paired by
    nearest mean).
    (2) Trajectories at full size: FP64 and FP32 runs on each of --precision-seeds
    filter seeds (the scene is the same); once resampling differs the runs are different Monte-Carlo
    realisations, so the FP32-FP64 differences of OSPA and calibration error are
    set against the FP64 seed-to-seed spread."""
    import torch
    dev = torch.device("cuda", 0)
    DT = pkg.scene.DT
    n_frames = args.precision_frames
    # ---- (1) one-step errors
    sc, cfg64 = pkg.scene.workload("precision_c3", precision=pkg.SCPHD_FP64, n_frames=n_frames)
    cfg64.n_parents = 256
    cfg32 = cfg64.copy()
    cfg32.precision = pkg.SCPHD_FP32
    src = pkg.SCPHDCameraCalibration(cfg64)
    A = pkg.SCPHDCameraCalibration(cfg64)
    B = pkg.SCPHDCameraCalibration(cfg32)
    checkpoints = [k for k in (1, 3, 10, 30, 100, 200, n_frames - 2) if k < n_frames - 1]
    local = []
    for k in range(n_frames - 1):
        z = sc.frames[k]
        src.step(DT, z[:, 0], z[:, 1], sc.fixed[k], d=z[:, 2])
        if k not in checkpoints:
            continue
        state = _capture_state(src)
        zn = sc.frames[k + 1]
        outs = []
        for f in (A, B):
            f.set_state(*state)
            f.predict(DT)
            f.update(zn[:, 0], zn[:, 1], sc.fixed[k + 1], d=zn[:, 2])
            ell, ll = f.normalizers(len(zn))
            outs.append((ell, ll, [f.mixture(pkg.SCPHD_MIX_FITTED, p) for p in range(f.n_parents)],
                         [f.mixture(pkg.SCPHD_MIX_MERGED, p) for p in range(f.n_parents)], f.map_sizes()))
        (e64, l64, F64, M64, n64), (e32, l32, F32, M32, n32) = outs
        fm, fv, fw, mm, mv, same = [], [], [], [], [], 0
        for a, b in zip(F64, F32):
            live = (a[:, 1] > 0) & (a[:, 0] > 0)
            if live.any() and a.shape == b.shape:
                sd = np.sqrt(np.maximum(a[live][:, [8, 10, 13, 17, 22, 28]], 1e-30))
                fm.append((np.abs(b[live][:, 2:8] - a[live][:, 2:8]) / sd).ravel())
                fv.append((np.abs(b[live][:, [8, 10, 13, 17, 22, 28]] - a[live][:, [8, 10, 13, 17, 22, 28]])
                           / np.maximum(np.abs(a[live][:, [8, 10, 13, 17, 22, 28]]), 1e-30)).ravel())
                fw.append(np.abs(b[live, 0] - a[live, 0]) / a[live, 0])
        for a, b in zip(M64, M32):
            same += a.shape == b.shape
            dm, dv = _match_rows(a, b, list(range(1, 7)), [7, 9, 12, 16, 21, 27])
            mm.append(dm)
            mv.append(dv)
        cat = lambda xs: np.concatenate(xs) if xs and sum(len(x) for x in xs) else np.zeros(1)
        q = lambda x: {"p50": float(np.percentile(x, 50)), "p99": float(np.percentile(x, 99)),
                       "max": float(np.max(x))}
        lrel = np.abs(l32 - l64) / np.maximum(1.0, np.abs(l64))
        local.append({"frame": k + 1, "loglik_rel": q(lrel), "log_normaliser_abs": q(np.abs(e32 - e64)),
                      "fitted_weight_rel": q(cat(fw)), "fitted_mean_sd": q(cat(fm)), "fitted_var_rel": q(cat(fv)),
                      "merged_mean_sd": q(cat(mm)), "merged_var_rel": q(cat(mv)),
                      "merged_count_equal_frac": same / len(M64),
                      "map_size_equal_frac": float(np.mean(n32 == n64))})
    for f in (src, A, B):
        f.close()
    # ---- (2) trajectories at full size
    traj = {}
    n_seeds = max(2, args.precision_seeds)
    runs = []
    for seed_off in range(n_seeds):
        runs += [("fp64_s%d" % seed_off, pkg.SCPHD_FP64, seed_off), ("fp32_s%d" % seed_off, pkg.SCPHD_FP32, seed_off)]
    for name, prec, seed_off in runs:
        sc, cfg = pkg.scene.workload("precision_c3", precision=prec, n_frames=n_frames)
        cfg.seed = int(cfg.seed) + 7919 * seed_off
        if args.parents:
            cfg.n_parents = args.parents
        f = pkg.SCPHDCameraCalibration(cfg)
        dz = [torch.tensor(np.ascontiguousarray(z.T), dtype=torch.float64, device=dev) for z in sc.frames]
        torch.cuda.synchronize()
        rows, idx, t_dev = [], [], 0.0
        for k in range(n_frames):
            z = dz[k]
            t0 = time.perf_counter()
            f.predict(DT)
            f.update_device(z[0].data_ptr(), z[1].data_ptr(), z[2].data_ptr(), z.shape[1], sc.fixed[k])
            f.synchronize()
            t_dev += time.perf_counter() - t0
            if k >= n_frames // 2 or k == n_frames - 1:   # the summaries use the second half
                st, lw = f.particles()
                m = pkg.evaluate.frame_metrics(st, lw, f.map_weights, lambda p: f.map_clouds(p)[0], sc, k)
                pose = pkg.evaluate.expected_pose(st, lw)
                rows.append([m["ospa"], m["calib_position_m"], m["calib_angle_rad"], m["n_features"],
                             m["cardinality"], *pose[[0, 1, 2, 6, 7, 8]]])
            else:
                rows.append([np.nan] * 11)
            t0 = time.perf_counter()
            f.resample()
            f.synchronize()
            t_dev += time.perf_counter() - t0
            if k < 16:
                idx.append(f.resample_indices().copy())
        traj[name] = {"rows": np.array(rows), "idx": idx, "seconds": t_dev}
        f.close()
        del dz
        torch.cuda.synchronize()
        torch.cuda.empty_cache()
    a, b = traj["fp64_s0"], traj["fp32_s0"]
    aligned = 0
    for k in range(min(len(a["idx"]), len(b["idx"]))):
        if not np.array_equal(a["idx"][k], b["idx"][k]):
            break
        aligned = k + 1
    tail = slice(n_frames // 2, None)
    mean = lambda r, j: float(r["rows"][tail, j].mean())
    summ = {"frames": n_frames, "seeds": n_seeds, "one_step": local, "resampling_identical_frames": aligned}
    for j, nm in ((0, "ospa"), (1, "calib_position_m"), (2, "calib_angle_rad"), (3, "n_features")):
        v64 = np.array([mean(traj["fp64_s%d" % i], j) for i in range(n_seeds)])
        v32 = np.array([mean(traj["fp32_s%d" % i], j) for i in range(n_seeds)])
        diff = float(v32.mean() - v64.mean())
        se = float(np.sqrt(v64.var(ddof=1) / n_seeds + v32.var(ddof=1) / n_seeds))
        summ[nm] = {"fp64": v64.tolist(), "fp32": v32.tolist(), "fp64_mean": float(v64.mean()),
                    "fp32_mean": float(v32.mean()), "fp32_minus_fp64": diff, "diff_standard_error": se,
                    "diff_rel": diff / float(v64.mean()), "diff_rel_95": (abs(diff) + 1.96 * se) / float(v64.mean()),
                    "seed_sd_fp64": float(v64.std(ddof=1))}
        summ[nm + "_final"] = {k2: float(v["rows"][-1, j]) for k2, v in traj.items()}
    summ["seconds"] = {k2: v["seconds"] for k2, v in traj.items()}
    summ["note"] = ("trajectory figures are means over the second half of the frames, per seed; "
                    "diff_rel_95 = (|mean FP32 - mean FP64| + 1.96 standard errors) / mean FP64")
    if args.precision_dump:
        np.savez_compressed(args.precision_dump, **{k2: v["rows"] for k2, v in traj.items()})
    return summ


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--workload", default="plain_c1")
    ap.add_argument("--precision", default="fp32", choices=["fp32", "fp64"])
    ap.add_argument("--prefill", type=int, default=30)
    ap.add_argument("--cpu-prefill", type=int, default=30)
    ap.add_argument("--cpu-frames", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-extras", action="store_true", help="skip the short batched and serving runs")
    ap.add_argument("--update-path", default="staged", choices=["staged", "fused"],
                    help="update path of the single filter: one kernel per stage (default) or the fused kernel")
    ap.add_argument("--extra-serve-seconds", type=float, default=20.0, help="serving window of the extra run")
    ap.add_argument("--parents", type=int, default=0, help="override the parent count (profiling only)")
    ap.add_argument("--filters", type=int, default=64, help="filters of the batched_c2 workload")
    ap.add_argument("--serve-seconds", type=float, default=60.0, help="serving window of serving_c4")
    ap.add_argument("--precision-frames", type=int, default=300, help="frames of the precision_c3 study")
    ap.add_argument("--precision-dump", default="", help="npz of the per-frame trajectories")
    ap.add_argument("--precision-seeds", type=int, default=3, help="filter seeds per precision in the trajectories")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "precision_c3":
        import torch
        torch.cuda.set_device(0)
        print(json.dumps({"workload": "precision_c3", "study": run_precision(args, load_package())}), flush=True)
    elif args.workload == "serving_c4":
        import torch
        torch.cuda.set_device(0)
        print(json.dumps(run_serving(args, load_package())), flush=True)
    elif args.workload in ("batched_c2", "batched_c0x64"):
        import torch
        torch.cuda.set_device(0)
        pkg = load_package()
        r = run_batched(args, pkg)
        K = args.steps
        line = {"metric": METRIC, "value": r["batched"]["value"], "unit": UNIT, "n_gpus": 1,
                "steps": r["batched"]["steps"],
                "warmup": args.warmup, "ms_per_step": r["batched"]["ms_per_step"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": args.precision, "data": "synthetic",
                "config": {"workload": args.workload, "filters": r["filters"], "parents": r["parents"],
                           "waves": r["waves"], "prefill_frames": args.prefill,
                           "l2": "no flush: the resident state is larger than L2"},
                "e2e": r["e2e"], "gpu_launches": r["gpu_launches"], "clocks": r["clocks"],
                "plain": r["plain"], "batched_over_plain": r["batched_over_plain"],
                "wave_frame_ms": r["wave_frame_ms"], "counters": r["counters"]}
        print(json.dumps(line), flush=True)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()
