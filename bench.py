"""Throughput benchmark of the wavefront path integrator (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config C]

Workload: configuration 1 by default (64 spheres + 2-triangle plane + 4 sphere emitters,
1024x1024, 64 spp per frame, depth 8, NEE+MIS). One step = one progressive frame of the
whole image. Metric: Mrays/s of canonical queries (camera + continuation closest hits +
contributing shadow rays); Mpaths/s is reported beside it.

  value   device time (CUDA events on the session's stream, summed over the K frames), the
          scene already resident in HBM, L2 flushed between steps; N > 1: N independent
          replicas (own seeds), max device time over ranks, rays summed over ranks.
  e2e     through the C ABI with host buffers: camera upload, render, wait, readback of the
          W x H x 3 FP32 radiance into pinned host memory (asynchronous: each step's image is
          copied out while the next step renders; the last one is waited for inside the timed
          region), wall clock over the K steps, frames replayed from their CUDA graph.
  roofline  the extend (closest-hit) stage, timed live with events around its launches.
  cpu_baseline  the oracle's restatement of the reference integrator (two traces per bounce,
          linear primitive scan) on the host cores, on a bounded pixel sample.
  guiding  time-to-relMSE on the slit room (1024x1024, depth 10): device time of the plain
          render at a fixed sample budget, and of the guided render (network trained online
          from scratch, training inside the timed frames) until its relMSE against a converged
          plain render reaches the plain render's (rank 0, N = 1; --no-guiding skips it).

--impl reference runs that CPU restatement as the reference arm (rank 0 only).
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "gpu-pathed_b200"))

WORKLOADS = {
    0: dict(name="cornell-box-36tri", res=(512, 512), spp=16, depth=5),
    1: dict(name="spheres-64+4-emitters-plane", res=(1024, 1024), spp=64, depth=8),
    2: dict(name="icosphere-1310720tri-env2048x1024", res=(1920, 1080), spp=32, depth=6),
    3: dict(name="slit-room-2002tri+icosphere-1310720tri", res=(1024, 1024), spp=16, depth=10),
    # 48 scenes drawn from 0-3 (seed 0x5EED + 4), one launch per stage for all of them,
    # about half with their own guide network
    4: dict(name="batch-48-scenes", res=(0, 0), spp=0, depth=0),
}


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", 6650.0)), "measured"
    return 6650.0, "fallback"


L2_BYTES = 126 * 1024 * 1024  # B200 L2
L1_RESIDENT_BYTES = 1 << 20   # nodes + leaf entries this small stay in the SMs' L1 caches
ISSUE_SLOTS_PER_CYCLE = 4 * 148  # one warp instruction per cycle per SM sub-partition, 148 SMs
L2_PROBE_BYTES = 32 << 20     # pt_measure_l2_read buffer: well inside either die's L2 half


def traversal_bound(counts, prof):
    """The resource that bounds closest-hit traversal on this scene (nodes + leaf entries
    footprint): 'issue' when it fits in L1, 'l2' when it fits in L2, else 'hbm'."""
    footprint = counts.bvh_nodes * prof["node_bytes"] + (counts.num_triangles + counts.num_spheres) * prof["prim_bytes"]
    if footprint <= L1_RESIDENT_BYTES:
        return "issue", footprint
    if footprint <= L2_BYTES:
        return "l2", footprint
    return "hbm", footprint


class ClockSampler:
    """nvidia-smi SM clock / throttle sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        cmd = ["nvidia-smi", "-i", str(self.index),
               "--query-gpu=timestamp,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
               "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
               "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "50"]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def wait_first(self, timeout=5.0):
        """Block until the sampler delivered its first sample (it takes a moment to start)."""
        t_end = time.time() + timeout
        while self.proc is not None and not self.lines and time.time() < t_end:
            time.sleep(0.02)

    def stop(self, t0=None, t1=None):
        """Median SM clock and the throttle reasons seen in the wall-clock window [t0, t1]
        (time.time()); by nvidia-smi's own sample timestamps. A window shorter than the
        sampling interval may hold no sample: then the samples nearest to it stand in."""
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.12)  # one more sample after the window
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                ts = datetime.datetime.strptime(parts[0], "%Y/%m/%d %H:%M:%S.%f").timestamp()
                rows.append((ts, float(parts[1]), float(parts[2]), parts[4:8]))
            except ValueError:
                continue
        inside = [r for r in rows if t0 is None or t0 <= r[0] <= t1]
        used, where = inside, "inside the timed region"
        if not inside and rows and t0 is not None:
            before = [r for r in rows if r[0] < t0][-1:]
            after = [r for r in rows if r[0] > t1][:1]
            used, where = before + after, "nearest before and after the timed region (shorter than the 50 ms interval)"
        sm = sorted(r[1] for r in used)
        reasons = {nm for r in used for nm, v in zip(names, r[3]) if v.lower() == "active"}
        return {"sm_mhz": sm[len(sm) // 2] if sm else None, "sm_max_mhz": used[-1][2] if used else None,
                "reasons": sorted(reasons), "samples": len(inside), "from": where}


def _dist_init():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def replica_seed(rank):
    """Seed of replica `rank`: every rank renders its own samples."""
    return 0x5EED + 7919 * rank


def reduce_over_ranks(t, counts, world, device="cuda"):
    """Replicas: the job's time is the slowest rank's, its work the sum over ranks. Returns
    (max over ranks of t, [sum over ranks of each count]); one rank returns its own values."""
    if world <= 1:
        return float(t), [float(c) for c in counts]
    import torch
    import torch.distributed as dist

    tt = torch.tensor([float(t)], dtype=torch.float64, device=device)
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    rr = torch.tensor([float(c) for c in counts], dtype=torch.float64, device=device)
    dist.all_reduce(rr, op=dist.ReduceOp.SUM)
    return float(tt.item()), [float(x) for x in rr.tolist()]


def cpu_reference_run(cfg, seconds_target, threads=0, seed=0x5EED):
    """Oracle restatement of the reference integrator (reference trace convention, linear scan)
    on a bounded pixel sample. Returns (Mrays/s, Mpaths/s, sample description, threads)."""
    import numpy as np

    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc  # CPU baseline leg only
    import pathed

    wl = WORKLOADS[cfg]
    w, h = wl["res"]
    s = pathed.Session(w, h)
    s.load_config(cfg)
    sc = s.export_scene()
    s.close()
    o = orc.Oracle()
    osc = o.scene(sc)
    nthreads = threads or os.cpu_count() or 1
    rng = np.random.default_rng(1)
    # calibrate on a small sample, then size the run to about `seconds_target`
    spp = wl["spp"]
    npx = 64
    t0 = time.perf_counter()
    pix = np.sort(rng.choice(w * h, npx, replace=False)).astype(np.int32)
    o.render(osc, sc["camera"], w, h, pix, spp, wl["depth"], nee=True, seed=seed, trace_once=False,
             threads=nthreads)
    dt = max(time.perf_counter() - t0, 1e-3)
    npx = int(min(w * h, max(64, npx * seconds_target / dt)))
    pix = np.sort(rng.choice(w * h, npx, replace=False)).astype(np.int32)
    t0 = time.perf_counter()
    _, _, counts = o.render(osc, sc["camera"], w, h, pix, spp, wl["depth"], nee=True, seed=seed, trace_once=False,
                            threads=nthreads)
    dt = time.perf_counter() - t0
    rays = float(counts[0] + counts[1])
    paths = float(npx * spp)
    sample = f"{npx} seeded pixels x {spp} spp of the {w}x{h} frame ({paths:.0f} paths, {rays:.0f} canonical rays)"
    return rays / dt / 1e6, paths / dt / 1e6, sample, nthreads, dt


def run_reference(args):
    world, rank, _ = _dist_init()
    if rank != 0:
        return 0
    wl = WORKLOADS[args.config]
    if args.config == 4:
        print(json.dumps({"impl": "reference", "unavailable": "the reference renders one scene per session: no "
                          "batched form of configuration 4 exists (per-scene reference arms: --config 0-3)"}))
        return 0
    vals = []
    for _ in range(args.warmup):
        cpu_reference_run(args.config, 1.0)
    per = []
    for _ in range(args.steps):
        mr, mp, sample, thr, dt = cpu_reference_run(args.config, 8.0)
        vals.append(mr)
        per.append((mp, dt))
    v = sum(vals) / len(vals)
    ref_cuda = _reference_cuda(args, rays_per_path=(v / per[0][0]) if per[0][0] > 0 else None)
    line = {
        "impl": "reference", "metric": "Mrays/s", "value": v, "unit": "Mrays/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * sum(p[1] for p in per) / len(per),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "mpaths_per_s": sum(p[0] for p in per) / len(per),
        "config": {"workload": wl["name"], "resolution": list(wl["res"]), "spp": wl["spp"], "max_depth": wl["depth"],
                   "nee": True, "parallelism": "cpu-threads"},
        "cpu_baseline": {"value": v, "unit": "Mrays/s", "cores": os.cpu_count(), "kind": "port",
                         "sample": sample},
        "e2e": {"value": v, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_cuda": ref_cuda,
    }
    print(json.dumps(line), flush=True)
    return 0


def _reference_cuda(args, rays_per_path):
    """The reference's own CUDA integrator (renderKernel from its sources, linear primitive
    scan, curand) timed on this GPU on the same workload; Mrays/s from the canonical rays per
    path of the CPU restatement (same estimator, same expected path lengths)."""
    try:
        import torch

        if not torch.cuda.is_available():
            return {"unavailable": "no CUDA device"}
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc
        import pathed

        if not os.path.exists(orc.REFBENCH_LIB):
            return {"unavailable": "reference GPU build (oracle/_ref/librefbench.so) not built"}
        wl = WORKLOADS[args.config]
        w, h = wl["res"]
        s = pathed.Session(w, h)
        s.load_config(args.config)
        sc = s.export_scene()
        s.close()
        rb = orc.RefBench()
        rb.load(sc, w, h)
        rb.render(1, wl["depth"], True)  # warm-up
        ms = [rb.render(wl["spp"], wl["depth"], True) for _ in range(max(1, min(args.steps, 3)))]
        rb.close()
        mean_ms = sum(ms) / len(ms)
        paths = w * h * wl["spp"]
        out = {"ms_per_frame": mean_ms, "mpaths_per_s": paths / (mean_ms / 1e3) / 1e6,
               "build": "reference sources (src/renderers/path_tracer.cu et al.), nvcc -O3 sm_100a, FMA on",
               "frames": len(ms)}
        if rays_per_path:
            out["value"] = paths * rays_per_path / (mean_ms / 1e3) / 1e6
            out["unit"] = "Mrays/s"
            out["rays_per_path"] = rays_per_path
        return out
    except Exception as e:  # report, do not fail the arm
        return {"unavailable": f"{type(e).__name__}: {e}"}


def _time_frames(s, spp, steps, flush):
    """Device time (CUDA events on the session's stream around each frame, summed) of `steps`
    frames on the product path (graph replay, the shadow stages overlapped, no per-launch
    events) with L2 flushed before each, and the canonical rays and paths they traced."""
    import torch

    s.set_profiling(stage_timing=False, work_counters=False)
    dev_ms = 0.0
    rays = paths = 0
    for _ in range(steps):
        flush.zero_()  # L2 flush between steps (outside the frame's events)
        torch.cuda.synchronize()
        dev_ms += s.render(spp)
        st = s.stats()
        rays += st["rays_extend"] + st["rays_shadow"]
        paths += st["rays_camera"]
    return dev_ms, rays, paths


def _stage_frames(s, spp, steps, flush):
    """Per-stage device time and launches of `steps` frames with an event after every launch,
    all stages on one stream (a kernel's launch time is then its own, not shared with the
    overlapped shadow stage), L2 flushed before each frame; the launch shape is restored."""
    import torch

    import pathed

    overlap = s.get_launch()["overlap_shadow"]
    s.set_launch(overlap_shadow=2)
    s.set_profiling(stage_timing=True, work_counters=False)
    s.render(spp)  # untimed: direct launches after the graph replays
    stage_ms = {k: 0.0 for k in pathed.STAGES}
    stage_launches = {k: 0 for k in pathed.STAGES}
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        s.render(spp)
        p = s.profile()
        for k in pathed.STAGES:
            stage_ms[k] += p["stage_ms"][k]
            stage_launches[k] += p["stage_launches"][k]
    s.set_profiling(stage_timing=False, work_counters=False)
    s.set_launch(overlap_shadow=overlap)
    return stage_ms, stage_launches


def _count_frame(s, spp):
    """One untimed frame with work counters: node visits and leaf entries of the closest-hit
    stage, for the algorithmic-bytes accounting."""
    s.set_profiling(stage_timing=True, work_counters=True)
    s.render(spp)
    prof, st = s.profile(), s.stats()
    s.set_profiling(stage_timing=True, work_counters=False)
    return prof, st


def _roofline(workload, counts, prof_count, st_count, stage_ms, stage_launches, steps, l2_gbs, sm_mhz, shape=None):
    """Roofline of the closest-hit stage (k_extend) on the bound its scene sets:
      issue  nodes + leaf entries fit in L1 (a few KB): warp instructions issued per second
             (ncu's instructions per query x queries per launch / live launch time) against
             4 x 148 issue slots per cycle at the SM clock seen in the timed region;
      l2     they fit in L2: algorithmic bytes per launch / live launch time against the L2
             read bandwidth measured in this run (pt_measure_l2_read);
      hbm    otherwise: the same bytes against the measured HBM copy bandwidth.
    Algorithmic bytes = nodes x node bytes + leaf entries x 48 B + 48 B queue I/O per query."""
    hbm, peak_kind = _peaks()
    bound, footprint = traversal_bound(counts, prof_count)
    ext_launches = max(1, prof_count["stage_launches"]["extend"])
    q_ext = st_count["rays_extend"]
    nodes, prims = prof_count["extend_nodes"], prof_count["extend_prims"]
    algo_bytes_frame = nodes * prof_count["node_bytes"] + prims * prof_count["prim_bytes"] + q_ext * 48
    per_launch_bytes = algo_bytes_frame / ext_launches
    queries_per_launch = q_ext / ext_launches
    ext_ms = stage_ms["extend"] / max(1, stage_launches["extend"])
    bytes_gbs = per_launch_bytes / (ext_ms / 1e3) / 1e9
    bpq = _ncu_bytes_per_query(workload)
    roof = {"kernel": "k_extend (closest-hit traversal)", "bound": bound, "footprint_bytes": footprint,
            "traffic": None if bpq is None else bpq * queries_per_launch,
            "traffic_source": "ncu dram bytes per query x queries per launch (profiles/k_extend_traffic.txt)",
            "algorithmic_bytes_per_launch": per_launch_bytes, "algorithmic_gbs": bytes_gbs,
            "avg_launch_ms": ext_ms, "queries_per_launch": queries_per_launch,
            "nodes_per_query": nodes / max(1, q_ext), "prims_per_query": prims / max(1, q_ext),
            "hbm_frac": bytes_gbs / hbm}
    # instruction counts are measured per BVH shape; a shape without a capture takes the
    # nearest captured one, named in inst_source
    ipq, ishape = _ncu_shape_per_query(workload, shape, "warp_inst_per_query")
    inst_src = (None if ipq is None else f"ncu smsp__inst_executed.sum per query at shape {ishape}"
                + ("" if ishape == shape else f" (nearest capture; this run's shape is {shape})")
                + " (profiles/k_extend_issue.txt)")
    clk = sm_mhz or 1965.0
    issue_peak = ISSUE_SLOTS_PER_CYCLE * clk * 1e6 / 1e9  # G warp instructions / s
    issue_achieved = None if ipq is None else ipq * queries_per_launch / (ext_ms / 1e3) / 1e9
    if bound == "issue":
        fpq, _ = _ncu_shape_per_query(workload, shape, "fp32_flop_per_query")
        roof.update({"achieved": issue_achieved, "peak": issue_peak, "unit": "G warp-inst/s",
                     "frac": None if issue_achieved is None else issue_achieved / issue_peak,
                     "peak_source": f"4 x 148 issue slots per cycle at {clk:.0f} MHz (median SM clock, timed region)",
                     "inst_source": inst_src or f"no capture for this workload (shape {shape})",
                     "inst_shape_exact": ishape == shape})
        if fpq is not None:
            tflops = fpq * queries_per_launch / (ext_ms / 1e3) / 1e12
            fp_peak = 148 * 128 * 2 * clk * 1e6 / 1e12
            roof["fp32"] = {"achieved_tflops": tflops, "peak_tflops": fp_peak, "frac": tflops / fp_peak,
                            "flop_per_query": fpq}
    elif bound == "l2":
        roof.update({"achieved": bytes_gbs, "peak": l2_gbs, "unit": "GB/s",
                     "frac": bytes_gbs / l2_gbs if l2_gbs else None,
                     "peak_source": f"measured L2 read bandwidth of a {L2_PROBE_BYTES >> 20} MiB buffer in this run"})
    else:
        roof.update({"achieved": bytes_gbs, "peak": hbm, "unit": "GB/s", "frac": bytes_gbs / hbm,
                     "peak_source": peak_kind + " hbm_gbs (burst copy)"})
    if bound != "issue" and issue_achieved is not None:
        # most node and leaf bytes of the mesh scenes hit L1: the issue rate beside the bytes
        roof["issue_slots"] = {"achieved": issue_achieved, "peak": issue_peak, "unit": "G warp-inst/s",
                               "frac": issue_achieved / issue_peak, "inst_source": inst_src,
                               "inst_shape_exact": ishape == shape}
    # the shade stage beside it, on HBM: the queue records it must move per frame (a lower bound
    # of its DRAM traffic: gathers at material-sorted slots fetch whole 32-byte sectors)
    items = st_count["rays_extend"]
    cont = max(0, items - st_count["rays_camera"])
    shade_bytes = items * (4 + 72) + cont * 72 + st_count["rays_shadow"] * 48
    shade_ms = stage_ms["shade"] / max(1, steps)
    if shade_ms > 0:
        gbs = shade_bytes / (shade_ms / 1e3) / 1e9
        roof["shade"] = {"kernel": "k_shade_all / k_shade_class (shade stage)", "bound": "hbm",
                         "algorithmic_bytes_per_frame": shade_bytes, "ms_per_frame": shade_ms,
                         "achieved": gbs, "peak": hbm, "unit": "GB/s", "frac": gbs / hbm,
                         "bytes": "per item 4 B sorted slot + 72 B queue record (origin, direction, "
                                  "throughput, hit, random state) read; per continuation 72 B and per "
                                  "shadow ray 48 B written"}
    roof["stage_timing"] = ("per-stage CUDA events of as many frames again, all stages on one stream, "
                            "right after the timed frames (which overlap the shadow stage with the next "
                            "depth's closest-hit stage on a second stream)")
    roof["stage_ms_per_step"] = {k: v / steps for k, v in stage_ms.items()}
    roof["stage_share"] = {k: v / max(1e-9, sum(stage_ms.values())) for k, v in stage_ms.items()}
    return roof


def _reference_cuda_config(cfg, rays_per_path):
    """The reference's own CUDA integrator on configuration `cfg`, on this GPU. Configurations
    0 and 1 at their full size and spp; configurations 2 and 3 (a linear scan of 1.31M
    triangles per query) on a reduced frame that still fills the GPU (one resident wave of the
    reference's 16x16 blocks), 1 spp, its per-path time extrapolated to the full frame."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    import pathed

    if not os.path.exists(orc.REFBENCH_LIB):
        return {"unavailable": "reference GPU build (oracle/_ref/librefbench.so) not built"}
    wl = WORKLOADS[cfg]
    fw, fh = wl["res"]
    w, h, spp = (fw, fh, wl["spp"]) if cfg in (0, 1) else ((384, 216) if cfg == 2 else (288, 288)) + (1,)
    s = pathed.Session(w, h)
    s.load_config(cfg)
    sc = s.export_scene()
    s.close()
    rb = orc.RefBench()
    rb.load(sc, w, h)
    if cfg in (0, 1):
        rb.render(1, wl["depth"], True)  # warm-up
        ms = [rb.render(spp, wl["depth"], True) for _ in range(2)]
    else:
        ms = [rb.render(spp, wl["depth"], True)]
    rb.close()
    mean_ms = sum(ms) / len(ms)
    paths = w * h * spp
    mpaths = paths / (mean_ms / 1e3) / 1e6
    out = {"mpaths_per_s": mpaths, "ms_measured": mean_ms, "measured": f"{w}x{h}, {spp} spp, {len(ms)} frame(s)",
           "ms_per_frame": mean_ms * (fw * fh * wl["spp"]) / paths,
           "extrapolated": cfg not in (0, 1),
           "build": "reference sources (src/renderers/path_tracer.cu et al.), nvcc -O3 sm_100a, FMA on"}
    if rays_per_path:
        out["value"] = mpaths * rays_per_path
        out["unit"] = "Mrays/s"
        out["rays_per_path"] = rays_per_path
        out["rays_per_path_source"] = "canonical rays per path of our frames (same estimator, same path lengths)"
    return out


def _per_config(cfg, steps, warmup, flush, l2_gbs, tune_cache, with_reference):
    """Configuration `cfg` at its full size on rank 0: our Mrays/s and Mpaths/s (autotuned,
    device time), the closest-hit roofline on its bound and the reference CUDA backend."""
    import pathed

    wl = WORKLOADS[cfg]
    w, h = wl["res"]
    s = pathed.Session(w, h)
    s.load_config(cfg)
    tuned = s.autotune(wl["spp"], tune_cache)
    counts = s.counts()
    prof_count, st_count = _count_frame(s, wl["spp"])
    s.set_profiling(stage_timing=False, work_counters=False)  # warm-up on the timed path
    for _ in range(warmup):
        s.render(wl["spp"])
    dev_ms, rays, paths = _time_frames(s, wl["spp"], steps, flush)
    stage_ms, stage_launches = _stage_frames(s, wl["spp"], steps, flush)
    shape = extend_shape_key(counts.bvh_width, counts.bvh_max_leaf, s.get_launch(), tuned["bvh_builder"])
    s.close()
    out = {"workload": wl["name"], "resolution": [w, h], "spp": wl["spp"], "max_depth": wl["depth"],
           "value": rays / (dev_ms / 1e3) / 1e6, "unit": "Mrays/s", "mpaths_per_s": paths / (dev_ms / 1e3) / 1e6,
           "ms_per_step": dev_ms / steps, "steps": steps, "warmup": warmup, "triangles": counts.num_triangles,
           "spheres": counts.num_spheres,
           "autotuned": {k: tuned[k] for k in ("bvh_width", "sort_materials", "sort_rays", "speculate",
                                                "blocks_per_sm", "block", "wave_paths", "split_shade", "max_leaf",
                                                "bvh_builder", "shadow_order", "fuse_camera")},
           "roofline": _roofline(wl["name"], counts, prof_count, st_count, stage_ms, stage_launches, steps, l2_gbs,
                                 None, shape)}
    if with_reference:
        try:
            ref = _reference_cuda_config(cfg, rays / max(1, paths))
        except Exception as e:  # report, do not fail the line
            ref = {"unavailable": f"{type(e).__name__}: {e}"}
        out["reference_cuda"] = ref
        if ref.get("mpaths_per_s"):
            out["speedup_vs_reference_cuda"] = out["mpaths_per_s"] / ref["mpaths_per_s"]
    return out


def run_ours(args):
    import torch

    import pathed

    world, rank, local = _dist_init()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    wl = WORKLOADS[args.config]
    w, h = wl["res"]
    spp = args.spp or wl["spp"]
    batch = args.config == 4
    if batch:
        w = h = 16
    # the L2 read bandwidth that bounds traversal on L2-resident scenes, measured on this GPU
    l2_gbs, l2_ms = pathed.measure_l2_read(local, L2_PROBE_BYTES, 64, 5)
    s = pathed.Session(w, h)
    s.set_device(local)  # the library's CUDA runtime keeps its own current device
    specs = None
    if batch:
        specs = pathed.batch_generate(0x5EED + 4, 48)
        s.load_batch(specs)
        s.set_guiding(True)
        spp = 0
    else:
        if args.gpu_bvh:  # BVH built on the device (LBVH or PLOC, collapsed to the wide format)
            s.set_bvh_builder(2 if args.gpu_bvh == "ploc" else 1)
        s.load_config(args.config)
        if args.guided:  # learned guiding on the main workload (trained online during warm-up)
            s.set_guiding(True)
            if args.guide_inference:
                s.set_guide_inference(args.guide_inference == "tc")
    s.set_seed(replica_seed(rank))
    if args.wave_paths:
        s.set_launch(wave_paths=args.wave_paths)
    if args.quantized_bvh:
        s.set_bvh_quantized(True)
    tuned = None
    if not args.no_autotune:  # untimed: frames of this workload under each candidate shape
        tuned = s.autotune(spp if spp else 1, args.tune_cache)
    if args.sort_rays:
        s.set_launch(sort_rays=1 if args.sort_rays == "on" else 2)
    counts = s.counts()

    # one untimed frame with work counters for the algorithmic-bytes accounting
    prof_count, st_count = _count_frame(s, spp)
    s.set_profiling(stage_timing=False, work_counters=False)  # warm-up on the timed path
    for _ in range(args.warmup):
        s.render(spp)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device="cuda")

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    clocks = ClockSampler(local)
    clocks.start()
    clocks.wait_first()
    barrier()
    t_clk0 = time.time()
    dev_ms, rays, paths = _time_frames(s, spp, args.steps, flush)
    barrier()
    clk = clocks.stop(t_clk0, time.time())
    # per-stage times (the roofline's launch times and the stage breakdown): as many frames
    # again with an event after every launch, on one stream
    stage_ms, stage_launches = _stage_frames(s, spp, args.steps, flush)
    t_max, (rays_all, paths_all) = reduce_over_ranks(dev_ms, [rays, paths], world)
    value = rays_all / (t_max / 1e3) / 1e6

    # ---- end to end through the C ABI with host buffers, on the default path (no per-launch
    # profiling events, so frames replay their CUDA graph); one untimed frame captures it
    s.set_profiling(stage_timing=False, work_counters=False)
    if batch:  # every scene's image read back each step
        hosts = [torch.empty((d["height"], d["width"], 3), dtype=torch.float32).pin_memory().numpy() for d in specs]
    else:
        cam = s.export_scene()["camera"]
        host = torch.empty((h, w, 3), dtype=torch.float32).pin_memory().numpy()
        cam_host = torch.from_numpy(cam.copy()).pin_memory().numpy()
    s.render(0 if batch else spp)
    if not batch:  # the side stream and staging buffer of the asynchronous readback
        s.readback_async(host)
        s.readback_wait()
    captures0 = s.profile()["graph_captures"]
    barrier()
    e2e_rays = 0
    t0 = time.perf_counter()
    for step in range(args.steps):
        if batch:
            s.render(0)
            for k, hb in enumerate(hosts):
                s._check(pathed.lib.pt_batch_readback(s._h, k, hb.ctypes.data, hb.size, 0))
        else:
            s.set_camera(cam_host[0:3], cam_host[3:6], cam_host[6:9], float(cam_host[9]), bool(cam_host[10]))
            s.render_async(spp)
            if step:
                s.readback_wait()  # the previous step's image, copied out while this frame renders
            s.wait()
            s.readback_async(host)
        st = s.stats()
        e2e_rays += st["rays_extend"] + st["rays_shadow"]
    if not batch:
        s.readback_wait()  # the last step's image
    barrier()
    e2e_s, (e2e_rays,) = reduce_over_ranks(time.perf_counter() - t0, [e2e_rays], world)
    e2e_value = e2e_rays / e2e_s / 1e6
    e2e_captures = s.profile()["graph_captures"] - captures0  # 0: every timed frame replayed its graph

    roof = None
    if rank == 0:
        roof = _roofline(wl["name"], counts, prof_count, st_count, stage_ms, stage_launches, args.steps, l2_gbs,
                         clk.get("sm_mhz"),
                         extend_shape_key(counts.bvh_width, counts.bvh_max_leaf, s.get_launch(),
                                          tuned["bvh_builder"] if tuned else {None: 0, "lbvh": 1, "ploc": 2}[args.gpu_bvh]))
        roof["l2_probe"] = {"gbs": l2_gbs, "ms": l2_ms, "bytes": L2_PROBE_BYTES}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and not batch:
        mr, mp, sample, thr, _ = cpu_reference_run(args.config, args.cpu_seconds)
        cpu = {"value": mr, "unit": "Mrays/s", "cores": thr, "kind": "port", "sample": sample,
               "mpaths_per_s": mp, "algorithm": "reference integrator restated (two traces per bounce, linear scan)"}

    per_config = None
    if rank == 0 and world == 1 and not args.no_per_config and not batch:
        per_config = {str(c): _per_config(c, 3, 3, flush, l2_gbs, args.tune_cache, not args.no_reference_cuda)
                      for c in (0, 1, 2, 3) if c != args.config}

    guiding = None
    if rank == 0 and world == 1 and not args.no_guiding and not batch:
        guiding = guided_time_to_relmse()

    gpu_launches = sum(stage_launches.values())
    if rank == 0:
        line = {
            "metric": "Mrays/s", "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "mpaths_per_s": paths_all / (t_max / 1e3) / 1e6,
            "config": ({"workload": wl["name"], "resolution": [w, h], "spp": spp, "max_depth": wl["depth"],
                        "nee": True, "triangles": counts.num_triangles, "spheres": counts.num_spheres,
                        "bvh_width": counts.bvh_width, "parallelism": f"replicas{world}",
                        "guided": bool(args.guided), "bvh_builder": f"gpu-{args.gpu_bvh}" if args.gpu_bvh else "host-sah",
                        "bvh_nodes": "quantized" if args.quantized_bvh else "float",
                        "sort_rays": s.get_launch()["sort_rays"] == 1,
                        "l2": "flushed between steps (256 MiB write)"} if not batch else
                       {"workload": wl["name"], "scenes": len(specs), "guided_scenes": sum(d["guided"] for d in specs),
                        "paths_per_frame": sum(d["width"] * d["height"] * d["spp"] for d in specs),
                        "pixels": sum(d["width"] * d["height"] for d in specs), "triangles": counts.num_triangles,
                        "spheres": counts.num_spheres, "bvh_width": counts.bvh_width, "nee": True,
                        "draw": "pathed.batch_generate(0x5EED + 4, 48)", "parallelism": f"replicas{world}",
                        "l2": "flushed between steps (256 MiB write)"}),
            "e2e": {"value": e2e_value, "unit": "Mrays/s", "h2d_bytes_per_step": 0 if batch else 44,
                    "d2h_bytes_per_step": (sum(d["width"] * d["height"] for d in specs) if batch else w * h) * 3 * 4,
                    "graph_captures": e2e_captures},
            "roofline": roof,
            "cpu_baseline": cpu,
            "per_config": per_config,
            "guiding": guiding,
            "clocks": clk,
            "gpu_launches": gpu_launches,
        }
        if tuned is not None:
            line["config"]["autotuned"] = {k: tuned[k] for k in ("bvh_width", "sort_materials", "sort_rays",
                                                               "speculate", "blocks_per_sm", "block", "wave_paths",
                                                               "split_shade", "max_leaf", "bvh_builder",
                                                               "shadow_order", "fuse_camera", "best_ms", "default_ms")}
            if tuned["bvh_builder"] == 2:
                line["config"]["bvh_builder"] = "gpu-ploc (autotuned)"
        print(json.dumps(line), flush=True)
    s.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def _slit_session(res):
    import pathed

    s = pathed.Session(res, res)
    s.load_config(3)
    s.set_consistent_mis(True)
    return s


def _relmse(s, ref, den):
    import numpy as np

    return float(np.mean((s.readback().astype(np.float64) - ref) ** 2 / den))


def slit_reference(ref_spp=2048, res=1024):
    """Plain render of the slit room at `ref_spp` (seed 12345), its 64-spp passes accumulated
    in FP64 on the host: the relMSE reference."""
    import numpy as np

    r = _slit_session(res)
    r.set_seed(12345)
    acc = np.zeros((res, res, 3), np.float64)
    frames = ref_spp // 64
    for _ in range(frames):
        r.render(64)
        acc += r.readback(pass_only=True)
    r.close()
    return acc / frames


def plain_to_budget(ref, budget_spp=256, res=1024):
    """Device ms of `budget_spp` 1-spp plain frames and the relMSE they reach."""
    den = ref ** 2 + 1e-2
    p = _slit_session(res)
    p.set_seed(77)
    p.render(1)
    p.reset()
    t_plain = sum(p.render(1) for _ in range(budget_spp))
    target = _relmse(p, ref, den)
    p.close()
    return t_plain, target


def guided_to_target(ref, t_plain, target, res=1024, fraction=None, steps=None, warmup=None, lr=None,
                     schedule=None, seed=77, batch=None):
    """Device ms for the guided render, trained online from scratch inside the timed 1-spp
    frames, to reach `target` relMSE (crossing interpolated in log relMSE between checks).
    `schedule(frame)`, when given, sets the Adam steps of each frame."""
    import numpy as np

    den = ref ** 2 + 1e-2
    g = _slit_session(res)
    g.set_seed(seed)
    g.set_guiding(True)
    if fraction is not None:
        g.set_guide_fraction(fraction)
    if steps is not None or warmup is not None or lr is not None or batch is not None:
        g.set_guide_options(steps_per_frame=-1 if steps is None else steps, lr=0.0 if lr is None else lr,
                            warmup_steps=-1 if warmup is None else warmup, batch=batch or 0)
    t_guided, spp, prev, crossed = 0.0, 0, None, None
    while t_guided < 3 * t_plain:
        if schedule is not None:
            st = schedule(spp)
            st, rate = st if isinstance(st, tuple) else (st, 0.0)
            g.set_guide_options(steps_per_frame=int(st), lr=float(rate))
        t_guided += g.render(1)
        spp += 1
        if spp >= 16 and spp % 4 == 0:
            e = _relmse(g, ref, den)
            if e <= target:
                if prev is not None:
                    (t0, e0) = prev
                    f = (np.log(e0) - np.log(target)) / max(1e-12, np.log(e0) - np.log(e))
                    crossed = t0 + f * (t_guided - t0)
                else:
                    crossed = t_guided
                break
            prev = (t_guided, e)
    info = g.guide_info()
    g.close()
    return crossed, (spp if crossed is not None else None), info["steps"]


def guided_time_to_relmse(budget_spp=256, ref_spp=2048, res=1024):
    """Plain vs guided on the slit room: device ms for the plain render to reach `budget_spp`
    and for the guided render (trained online from scratch) to reach the same relMSE,
    relMSE = mean((I - I_ref)^2 / (I_ref^2 + 1e-2)) against a `ref_spp` plain render."""
    ref = slit_reference(ref_spp, res)
    t_plain, target = plain_to_budget(ref, budget_spp, res)
    crossed, spp, steps = guided_to_target(ref, t_plain, target, res)
    # the configuration's hyperparameters as written: guide fraction 0.5, Adam lr 1e-3, 2^18
    # samples per Adam step; the steps per frame, which it leaves open, on the automatic schedule
    aw_crossed, aw_spp, aw_steps = guided_to_target(ref, t_plain, target, res, fraction=0.5, steps=0, lr=1e-3,
                                                    batch=1 << 18)
    as_written = {"fraction": 0.5, "lr": 1e-3, "samples_per_step": 1 << 18,
                  "steps_per_frame": "automatic: 16 for the first 512 steps, 4 up to 1024, then 2",
                  "guided_ms": aw_crossed, "guided_spp": aw_spp, "guide_steps": aw_steps,
                  "speedup": (t_plain / aw_crossed) if aw_crossed else None}
    return {"workload": f"slit-room {res}x{res} depth 10 (2002 + 1310720 triangles, env through a 0.05 slit)",
            "reference": f"plain render, {ref_spp} spp, consistent MIS, passes accumulated in FP64",
            "plain_spp": budget_spp,
            "plain_ms": t_plain, "target_relmse": target, "guided_ms": crossed,
            "guided_spp": spp, "speedup": (t_plain / crossed) if crossed else None, "guide_steps": steps,
            "training": "online from scratch inside the timed frames (automatic Adam schedule: fraction 0.7, "
                        "lr 3e-3, 16 steps of 2^16 samples per frame early, fewer later), tcgen05 training kernel",
            "as_written": as_written}


class BatchRelmse:
    """Configuration 4's time-to-relMSE pieces: the 48-scene draw, relMSE references for its
    guided scenes (a plain render of those scenes alone at `ref_frames` frames; a scene renders
    bit-identically inside or outside a batch), the plain budget and guided runs."""

    def __init__(self, ref_frames=128, draw=0x5EED + 4, n=48):
        import numpy as np

        import pathed

        self.draw, self.n = draw, n
        self.specs = pathed.batch_generate(draw, n)
        self.gids = [i for i, d in enumerate(self.specs) if d["guided"]]
        self.ref_frames = ref_frames
        r = pathed.Session(16, 16)
        r.load_batch([self.specs[i] for i in self.gids])
        r.set_consistent_mis(True)
        r.set_seed(12345)
        acc = [np.zeros((self.specs[i]["height"], self.specs[i]["width"], 3), np.float64) for i in self.gids]
        for _ in range(ref_frames):
            r.render(0)
            for k in range(len(self.gids)):
                acc[k] += r.batch_readback(k, pass_only=True)
        self.refs = [a / ref_frames for a in acc]
        r.close()
        self.dens = [x ** 2 + 1e-2 for x in self.refs]

    def errors(self, sess):
        import numpy as np

        return [float(np.mean((sess.batch_readback(i).astype(np.float64) - self.refs[k]) ** 2 / self.dens[k]))
                for k, i in enumerate(self.gids)]

    def plain(self, budget_frames=16):
        import pathed

        p = pathed.Session(16, 16)
        p.load_batch(self.specs)
        p.set_consistent_mis(True)
        p.set_seed(77)
        t = 0.0
        for _ in range(budget_frames):
            t += p.render(0)
        target = self.errors(p)
        p.close()
        self.budget_frames, self.t_plain, self.target = budget_frames, t, target
        return t, target

    def guided(self, steps=None, batch=None, fraction=None, per_frame=None):
        """Guided run (trained online from scratch inside the timed frames) until the mean
        relMSE over the guided scenes reaches the plain budget's; `per_frame(frame, session)`
        may change options before each frame."""
        import numpy as np

        import pathed

        g = pathed.Session(16, 16)
        g.load_batch(self.specs)
        g.set_seed(77)
        g.set_guiding(True)
        if steps is not None or batch is not None:
            g.set_guide_options(steps_per_frame=-1 if steps is None else steps, batch=batch or 0)
        if fraction is not None:
            g.set_guide_fraction(fraction)
        t, prev, crossed, frames = 0.0, None, None, 0
        per_scene = [None] * len(self.gids)
        mt = float(np.mean(self.target))
        while t < 3 * self.t_plain:
            if per_frame is not None:
                per_frame(frames, g)
            t += g.render(0)
            frames += 1
            e = self.errors(g)
            for k in range(len(self.gids)):
                if per_scene[k] is None and e[k] <= self.target[k]:
                    per_scene[k] = t
            m = float(np.mean(e))
            if crossed is None and m <= mt:
                if prev is not None:
                    t0, m0 = prev
                    f = (np.log(m0) - np.log(mt)) / max(1e-12, np.log(m0) - np.log(m))
                    crossed = t0 + f * (t - t0)
                else:
                    crossed = t
            prev = (t, m)
            if crossed is not None and all(x is not None for x in per_scene):
                break
        info = g.guide_info()
        g.close()
        ratios = [self.t_plain / x if x else None for x in per_scene]
        done = sorted(x for x in ratios if x is not None)
        return {"guided_ms": crossed, "guided_frames": frames,
                "speedup": (self.t_plain / crossed) if crossed else None,
                "per_scene_speedup_median": done[len(done) // 2] if done else None,
                "per_scene_speedup_min": done[0] if done else None,
                "per_scene_not_reached": sum(x is None for x in ratios),
                "per_scene": [{"config": self.specs[i]["config"], "level": self.specs[i]["level"],
                               "res": self.specs[i]["width"], "spp": self.specs[i]["spp"],
                               "depth": self.specs[i]["max_depth"], "speedup": ratios[k]}
                              for k, i in enumerate(self.gids)],
                "guide_steps": info["steps"]}


def batch_time_to_relmse(budget_frames=16, ref_frames=128, draw=0x5EED + 4, n=48):
    """Configuration 4: the 48-scene batch rendered plain for `budget_frames` frames, then
    guided (one network per guided scene, trained online from scratch inside the timed frames)
    until the mean relMSE over the guided scenes reaches plain's. Times are device ms of whole
    batch frames, every scene included."""
    import numpy as np

    b = BatchRelmse(ref_frames, draw, n)
    t_plain, target = b.plain(budget_frames)
    out = b.guided()
    return {"workload": f"batch of {n} scenes (pathed.batch_generate({draw:#x}, {n})), {len(b.gids)} guided",
            "reference": f"plain render of the guided scenes, {ref_frames} frames, consistent MIS",
            "plain_frames": budget_frames, "plain_ms": t_plain, "target_mean_relmse": float(np.mean(target)),
            **out}


def extend_shape_key(width, leaf, launch, builder=0):
    """The closest-hit stage's shape as the instruction counts are keyed: BVH width, largest
    leaf, whether its speculation is on (speculate codes 1 and 3), its grid (blocks per SM x
    threads per block), the wave size (log2 of the paths per wave) and, for a tree built on
    the GPU, its builder (suffix _lbvh or _ploc; none for the host's SAH tree). The lane-refill
    traversal's instructions per query depend on all of them: the grid and the wave set how
    full the warps' lanes stay."""
    sp = 1 if launch["speculate"] in (1, 3) else 0
    q = max(0, int(launch["wave_paths"]).bit_length() - 1)
    tag = {1: "_lbvh", 2: "_ploc"}.get(int(builder or 0), "")
    return f"w{width}_l{leaf}_s{sp}_b{launch['blocks_per_sm']}x{launch['block_extend']}_q{q}{tag}"


def _ncu_per_query(workload, field, fname="k_extend_traffic.txt"):
    """A per-closest-hit-query figure that ncu measured on this workload (profiles/<fname>,
    one `<workload> <field>: value` line each), or None."""
    p = os.path.join(ROOT, "profiles", fname)
    try:
        with open(p) as f:
            for line in f:
                parts = line.split()
                if len(parts) == 3 and parts[0] == workload and parts[1] == field + ":":
                    return float(parts[2])
    except OSError:
        pass
    return None


def _ncu_shape_per_query(workload, shape, field):
    """`field` of profiles/k_extend_issue.txt measured at `shape` on this workload, else at the
    nearest captured shape: the same tree builder first, then the same BVH width, the same
    speculation, the closest leaf size, the same grid and the closest wave size. Returns (value, captured shape) or
    (None, None)."""
    p = os.path.join(ROOT, "profiles", "k_extend_issue.txt")
    found = {}
    try:
        with open(p) as f:
            for line in f:
                parts = line.split()
                if len(parts) == 3 and parts[1] == field + ":" and parts[0].startswith(workload + "@"):
                    found[parts[0].split("@", 1)[1]] = float(parts[2])
    except OSError:
        return None, None
    if not found or not shape:
        return None, None
    if shape in found:
        return found[shape], shape

    def parse(k):
        f = k.split("_")
        grid = f[3] if len(f) > 3 else ""
        wave = int(f[4][1:]) if len(f) > 4 else 0
        tree = f[5] if len(f) > 5 else "sah"
        return int(f[0][1:]), int(f[1][1:]), int(f[2][1:]), grid, wave, tree

    tw, tl, ts, tg, tq, tt = parse(shape)

    def distance(k):
        w, l, sp, g, q, t = parse(k)
        return (t != tt, w != tw, sp != ts, abs(l - tl), g != tg, abs(q - tq), k)

    best = min(found, key=distance)
    return found[best], best


def _ncu_bytes_per_query(workload):
    return _ncu_per_query(workload, "dram_bytes_per_query")


def ncu_frames(args):
    """Frames for an ncu capture (ncu times every launch itself; nothing is timed here). Prints
    one JSON line per frame with its closest-hit and shadow query counts, so per-query figures
    can be formed from the captured launches."""
    import pathed

    wl = WORKLOADS[args.config]
    w, h = args.res or wl["res"]
    spp = args.spp or wl["spp"]
    s = pathed.Session(w, h)
    s.load_config(args.config)
    builder = {None: 0, "lbvh": 1, "ploc": 2}[args.gpu_bvh]
    if builder:
        s.set_bvh_builder(builder)
    if args.tune_cache:  # the shape a benchmark run chose (read from its cache, no measuring)
        builder = s.autotune(spp, args.tune_cache)["bvh_builder"]
    if args.bvh:
        s.set_bvh(args.bvh[0], args.bvh[1])
    if args.speculate:
        s.set_launch(speculate=args.speculate)
    if args.sort_rays:
        s.set_launch(sort_rays=1 if args.sort_rays == "on" else 2)
    s.set_profiling(stage_timing=True, work_counters=False)  # direct launches, counted per stage
    for _ in range(args.ncu_frames):
        s.render(spp)
        st = s.stats()
        lc = s.get_launch()
        print(json.dumps({"workload": wl["name"], "resolution": [w, h], "spp": spp,
                          "shape": extend_shape_key(s.counts().bvh_width, s.counts().bvh_max_leaf, lc, builder),
                          "rays_extend": st["rays_extend"], "rays_shadow": st["rays_shadow"],
                          "extend_launches": s.profile()["stage_launches"]["extend"]}), flush=True)
    s.close()
    return 0


def ncu_train(calls, n=1 << 16):
    """Guide-gradient calls (pt_guide_gradients) of n seeded samples on each training kernel,
    for an ncu capture of the training launches: `calls` on mma.sync, then `calls` on tcgen05."""
    import numpy as np

    import pathed

    rng = np.random.default_rng(10)
    s = pathed.Session(8, 8)
    p = (rng.normal(0, 1, pathed.GUIDE_PARAMS) * 0.1).astype(np.float32)
    s.set_guide_params(p)
    x = rng.uniform(-1, 1, (n, 80)).astype(np.float32)
    wi = rng.normal(0, 1, (n, 3)).astype(np.float32)
    wi /= np.linalg.norm(wi, axis=1, keepdims=True)
    w = rng.exponential(1.0, n).astype(np.float32)
    out = {}
    for tc in (False, True):
        s.set_guide_training(tc)
        t0 = time.perf_counter()
        for _ in range(calls):
            s.guide_gradients(x, wi, w)
        out["tcgen05" if tc else "mma.sync"] = (time.perf_counter() - t0) / calls * 1e3
    s.close()
    print(json.dumps({"guide_gradient_calls": calls, "samples": n, "wall_ms_per_call": out}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=1, choices=[0, 1, 2, 3, 4])
    ap.add_argument("--spp", type=int, default=0)
    ap.add_argument("--wave-paths", type=int, default=0)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-guiding", action="store_true")
    ap.add_argument("--no-per-config", action="store_true",
                    help="skip the per_config block (the other single-scene configurations at full size)")
    ap.add_argument("--no-reference-cuda", action="store_true",
                    help="per_config without the reference CUDA backend's timings")
    ap.add_argument("--guided", action="store_true", help="render the main workload with learned guiding")
    ap.add_argument("--guide-inference", choices=("mma", "tc"), default=None,
                    help="with --guided: guide inference on mma.sync or on tcgen05 (default: the library's)")
    ap.add_argument("--gpu-bvh", nargs="?", const="lbvh", default=None, choices=["lbvh", "ploc"],
                    help="build the BVH on the GPU instead of the host: a linear BVH (default) or PLOC")
    ap.add_argument("--quantized-bvh", action="store_true",
                    help="traverse quantized wide nodes (8-bit child planes) instead of float nodes")
    ap.add_argument("--no-autotune", action="store_true",
                    help="skip the autotuner (BVH width, sorting, blocks per SM, block size) that runs before timing")
    ap.add_argument("--sort-rays", choices=("on", "off"), default=None,
                    help="force ray sorting before the closest-hit stage on or off (applied after the autotuner)")
    ap.add_argument("--tune-cache", default=None,
                    help="JSON-lines autotuner cache: a run stores its choice, a later run of the same workload "
                         "applies it without measuring (a profiled run then times what the plain run chose)")
    ap.add_argument("--time-to-relmse", action="store_true",
                    help="with --config 4: print the batch's guided-vs-plain time-to-relMSE line and exit")
    ap.add_argument("--ncu-frames", type=int, default=0,
                    help="profiling aid: load the configuration (at --res if given), render this many frames "
                         "with the default launch shape, print their closest-hit query counts and exit")
    ap.add_argument("--res", type=int, nargs=2, default=None, help="with --ncu-frames: width height")
    ap.add_argument("--bvh", type=int, nargs=2, default=None, metavar=("WIDTH", "LEAF"),
                    help="with --ncu-frames: BVH width and primitives per leaf")
    ap.add_argument("--speculate", type=int, default=0,
                    help="with --ncu-frames: pt_launch_config.speculate (1 both, 2 off, 3 closest hit, 4 shadow)")
    ap.add_argument("--ncu-train", type=int, default=0,
                    help="profiling aid: this many guide-gradient calls of 2^16 seeded samples on the mma.sync "
                         "training kernel, then as many on the tcgen05 kernel; prints their wall ms and exits")
    args = ap.parse_args()
    if args.ncu_frames:
        return ncu_frames(args)
    if args.ncu_train:
        return ncu_train(args.ncu_train)
    if args.impl == "reference":
        return run_reference(args)
    if args.time_to_relmse:
        if args.config != 4:
            ap.error("--time-to-relmse takes --config 4 (configuration 3's figure is in every default line)")
        print(json.dumps({"metric": "time-to-relMSE speed-up, guided vs plain", **batch_time_to_relmse()}))
        return 0
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
