"""Series/min of the B200 alignment path on the realistic single-series workload.

Workload: 2048 x 2048 x 61-tilt series (+-60 deg in 2 deg steps, tilt axis 84.7,
shifts N(0, 8 px) + 0.3 px/tilt drift, Poisson + Gaussian noise at SNR 0.05), run as
`-g 0,0,0,0,300,1,0 -p 10`: pre-processing, coarse alignment (3 x stretch cross-
correlation + tilt-axis search, tilt-angle offset search), the full projection-
matching schedule, and the aligned output stack.  Seeded synthetic data stands in
for the reference's simulated phantoms.

  value   series/min of the batched mixed-precision form: one step aligns --batch
          series (default 8) with FP16 re-projection operands, projection matching
          in one lockstep group (mf_align_many_device), raw stacks already in HBM and
          aligned stacks written to HBM; summed over ranks (independent series)
  e2e     the same through the C ABI with host buffers: uploads of the raw stacks
          from pinned memory and downloads of the aligned stacks inside the timed
          region
  plain   one series at a time with FP32 operands (the reference's arithmetic)
  served  the serving loop (mf_server_*) on a Poisson stream of mixed-size requests
          at 80% of the measured batched capacity: series/min and p50/p99 latency

`--impl reference` times the reference algorithm on the host cores: the reference
program has no CPU implementation (every stage is CUDA), so the CPU restatement in
oracle/ stands in, timed on a bounded sample and scaled to one series.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
PRECISIONS = {"fp32": 0, "bf16": 1, "fp16": 2}


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


class ClockSampler:
    """SM clocks and throttle reasons sampled through NVML during the timed region
    (a thread that only reads; no process is spawned, so the launching thread is
    not disturbed)."""

    def __init__(self, gpu: int, period_s: float = 0.25):
        self.gpu = gpu
        self.period = period_s
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        try:
            import pynvml as N
            N.nvmlInit()
            h = N.nvmlDeviceGetHandleByIndex(self.gpu)
            mx = N.nvmlDeviceGetMaxClockInfo(h, N.NVML_CLOCK_SM)
        except Exception:
            return
        bits = {"hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20, "hw_thermal_slowdown": 0x40,
                "sw_power_cap": 0x4}
        while not self._stop.is_set():
            try:
                sm = N.nvmlDeviceGetClockInfo(h, N.NVML_CLOCK_SM)
                r = N.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.rows.append((sm, mx, [k for k, b in bits.items() if r & b]))
            except Exception:
                pass
            self._stop.wait(self.period)
        try:
            N.nvmlShutdown()
        except Exception:
            pass

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": statistics.median(r[0] for r in self.rows),
                "sm_max_mhz": max(r[1] for r in self.rows),
                "reasons": sorted({k for r in self.rows for k in r[2]}),
                "samples": len(self.rows), "source": "nvml"}


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(values, device, pg=None):
    """Element-wise maximum of per-rank timings over all ranks (the slowest rank
    sets the job's time); `pg` is torch.distributed when a process group is up."""
    import torch
    t = torch.tensor(values, dtype=torch.float64, device=device)
    if pg is not None:
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return [float(v) for v in t]


def make_workload(scale: float):
    from markerfree_b200 import synth
    return synth.config(2, scale=scale)


def workload_config(s, scale):
    nz, ny, nx = s.stack.shape
    return {"workload": f"{nx}x{ny}x{nz}-tilt series (+-60 deg, 2 deg), T=300, -p 10: "
                        "pre-processing, coarse alignment, projection matching, aligned stack",
            "nx": nx, "ny": ny, "tilts": nz, "thickness": s.thickness, "nproj": 10,
            "scale": scale, "l2": "inputs (1 GiB raw stack) larger than L2 (126 MB)",
            "parallelism": "independent series per GPU"}


# ---------------------------------------------------------------------------
def cpu_sample(s, passes=14, target_s=8.0):
    """Reference algorithm on the host cores (oracle), bounded sample, scaled to
    one series.  Sample: for one held-out tilt at full size, the re-projection of
    a block of the Yb rows (grown until it takes about `target_s`), one correction
    (resample + R-weight) and one cross-correlation measurement; per-pass cost =
    (Z-1) x that tilt cost + Z corrections; a series = `passes` passes (14 in the
    reference's own example run)."""
    from oracle import oracle as O
    nz, ny, nx = s.stack.shape
    ang = s.angles
    t0 = time.time()
    st = O.preprocess(s.stack, ang)
    t_pre = time.time() - t0
    zt = int(np.argmin(np.abs(ang)))
    ip = zt + 6
    skip = np.ones(nz, np.uint8)
    skip[zt - 5:zt + 6] = 0
    i0, i1 = O.find_proj_range(ang, skip, ip, 10)
    t0 = time.time()
    corr = np.stack([O.correct_proj(st[i], 0.0, 0.0, 84.7, rweight=True) for i in range(i0, i1 + 1)]
                    + [O.correct_proj(st[ip], 0.0, 0.0, 84.7, rweight=True)])
    t_corr = (time.time() - t0) / corr.shape[0]
    ncpu = os.cpu_count() or 1
    rows = min(ny, 2 * ncpu)
    while True:
        sub = np.ascontiguousarray(corr[:-1, ny // 2 - rows // 2: ny // 2 - rows // 2 + rows, :])
        full = np.zeros((nz, rows, sub.shape[2]), np.float32)
        full[i0:i1 + 1] = sub
        t0 = time.time()
        O.reproject(full, ang, ip, i0, i1, s.thickness)
        dt = time.time() - t0
        if dt > target_s / 4 or rows >= ny:
            break
        rows = min(ny, int(rows * max(2.0, target_s / max(dt, 1e-3) * 0.8)))
    t_rep = dt * (ny / rows)
    t0 = time.time()
    O.measure_shift(corr[-1], corr[-1])
    t_cc = time.time() - t0
    t_pass = (nz - 1) * (t_rep + t_cc + t_corr) + nz * t_corr
    series_s = t_pre + passes * t_pass
    return {"value": 60.0 / series_s, "unit": "series/min", "cores": os.cpu_count(),
            "kind": "port",
            "sample": (f"oracle/ (FP32 C++ restatement, OpenMP, all {os.cpu_count()} host threads): "
                       f"re-projection of {rows}/{ny} rows of one held-out tilt with "
                       f"{i1 - i0 + 1} neighbours ({t_rep:.1f} s scaled to all rows), one "
                       f"resample+R-weight ({t_corr:.2f} s), one 2-D cross-correlation "
                       f"({t_cc:.2f} s), pre-processing ({t_pre:.1f} s); series = {passes} passes x "
                       f"({nz - 1} held-out tilts + {nz} corrections), coarse stages and "
                       f"tilt-axis searches not counted"),
            "seconds_per_series": series_s}


def run_reference(args):
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    s = make_workload(args.scale)
    t0 = time.time()
    samples = [cpu_sample(s) for _ in range(max(1, args.steps))]
    wall = time.time() - t0
    v = statistics.median(x["value"] for x in samples)
    cb = dict(samples[0])
    cb["value"] = v
    line = {"metric": "series/min (2k^2, 61 tilts)", "value": v, "unit": "series/min",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 60000.0 / v, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded phantom series)",
            "config": workload_config(s, args.scale), "impl": "reference", "cpu_baseline": cb,
            "e2e": {"value": v, "unit": "series/min", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "wall_s": wall}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
def profiled_traffic(name):
    """DRAM bytes per launch of a kernel at the bench workload's size, from the ncu
    capture summarised in profiles/<name> (null when there is none)."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    with open(p) as f:
        return json.load(f).get("bytes_per_launch")


def _time_steps(stream, fn, steps):
    """CUDA-event time (ms) of `steps` calls of fn on the library's stream."""
    import torch
    evs = []
    for _ in range(steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        fn()
        b.record(stream)
        evs.append((a, b))
    torch.cuda.synchronize()
    return sum(a.elapsed_time(b) for a, b in evs)


def served_run(mf, s, dev, n_req, seed=5):
    """The serving loop (continuous batching) on the served-request workload: sizes
    50% 2048^2, 30% 1024^2, 20% 4096^2; the 1024^2 and 4096^2 series are derived from
    the 2048^2 one by 2 x 2 binning and 2 x pixel replication, so one phantom serves
    all sizes.  Requests come from pinned host memory and return their parameters.

    Capacity: all n_req requests arrive at once; series/min = n_req / makespan
    (also in 2048^2-equivalents, weighting each request by its pixel count).
    Latency: a Poisson stream of n_req requests at 80% of that capacity; p50/p99
    of arrival-to-result."""
    import torch
    nz = s.stack.shape[0]
    st2 = s.stack
    st1 = st2.reshape(nz, st2.shape[1] // 2, 2, st2.shape[2] // 2, 2).mean(axis=(2, 4))
    st4 = np.repeat(np.repeat(st2, 2, axis=1), 2, axis=2)
    pinned = {}
    for key, arr, az in (("2048", st2, s.thickness), ("1024", st1, max(8, s.thickness // 2)),
                         ("4096", st4, s.thickness)):
        t = torch.from_numpy(np.ascontiguousarray(arr, np.float32)).pin_memory()
        pinned[key] = (t, arr.shape, az)
    del st4
    weight = {"2048": 1.0, "1024": 0.25, "4096": 4.0}
    rng = np.random.default_rng(seed)
    n4 = max(1, round(0.2 * n_req))
    n1 = max(1, round(0.3 * n_req))
    kinds = ["4096"] * n4 + ["1024"] * n1 + ["2048"] * (n_req - n4 - n1)
    rng.shuffle(kinds)

    def submit(srv, k):
        t, shape, az = pinned[k]
        return srv.submit(None, s.angles, raw_ptr=t.data_ptr(), shape=shape, align_z=az,
                          nproj=10, precision=PRECISIONS["fp16"])

    # capacity: everything queued at once
    srv = mf.Server(gpu=dev, hbm_budget=0, max_group=8, workers=3, group_wait_ms=40.0)
    t0 = time.perf_counter()
    ids = [submit(srv, k) for k in kinds]
    for j in ids:
        srv.wait(j, timeout_s=1800.0)
    makespan = time.perf_counter() - t0
    st_cap = srv.stats()
    srv.close()
    cap_spm = 60.0 * n_req / makespan
    cap_eq = 60.0 * sum(weight[k] for k in kinds) / makespan
    # latency: Poisson arrivals at 80% of the capacity just measured
    rate_per_s = 0.8 * cap_spm / 60.0
    arrivals = np.cumsum(rng.exponential(1.0 / rate_per_s, n_req))
    srv = mf.Server(gpu=dev, hbm_budget=0, max_group=8, workers=3, group_wait_ms=40.0)
    ids = []
    t0 = time.perf_counter()
    for k, ta in zip(kinds, arrivals):
        wait = ta - (time.perf_counter() - t0)
        if wait > 0:
            time.sleep(wait)
        ids.append(submit(srv, k))
    lats = [srv.wait(j, timeout_s=1800.0)[2] for j in ids]
    st_lat = srv.stats()
    srv.close()
    return {"requests": n_req, "mix": {"2048": kinds.count("2048"), "1024": kinds.count("1024"),
                                       "4096": kinds.count("4096")},
            "series_per_min": cap_spm, "equiv_2048_series_per_min": cap_eq,
            "capacity_makespan_s": makespan, "capacity_mean_group_size": st_cap["mean_group"],
            "peak_admitted_gb": st_cap["peak_bytes"] / 1e9,
            "latency_arrival_rate_per_min": rate_per_s * 60.0,
            "p50_s": st_lat["p50_s"], "p99_s": st_lat["p99_s"],
            "mean_latency_s": float(np.mean(lats)), "latency_mean_group_size": st_lat["mean_group"],
            "precision": "fp16 operands, f32 accumulation",
            "returns": "per-tilt parameters (aligned stacks not copied back)"}


def run_ours(args):
    import torch
    import markerfree_b200 as mf

    rank, world, local = dist_env()
    dev = local
    torch.cuda.set_device(dev)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", dev))
        pg = dist
    s = make_workload(args.scale)
    nz, ny, nx = s.stack.shape
    xo, yo = mf.binned_size(nx, ny, 1)
    ctx = mf.Context(dev)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=f"cuda:{dev}")
    B = args.batch
    prec = PRECISIONS[args.precision]
    kw = dict(offset=0.0, pitch_angle=0.0, zshift=0.0, align_z=s.thickness, out_bin=1, nproj=10,
              precision=prec)
    d_raw = torch.from_numpy(s.stack).to(f"cuda:{dev}")
    d_outs = [torch.empty((nz, yo, xo), dtype=torch.float32, device=f"cuda:{dev}")
              for _ in range(B)]
    angs = [s.angles] * B

    def barrier():
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize()

    last = {}

    def step():
        ps, passes = mf.align_many_device(ctx, [d_raw] * B, nx, ny, nz, angs, d_outs, **kw)
        last["passes"] = int(passes[0])
        last["axis"] = float(ps[0].rotate[0])

    log = lambda m: print(f"[bench] {m}", file=sys.stderr, flush=True)
    log(f"workload ready {nx}x{ny}x{nz}, batch {B}")
    for _ in range(args.warmup):
        step()
    barrier()
    log("warm-up done")
    l0 = ctx.kernel_launches()
    with ClockSampler(dev) as clk:
        torch.cuda.nvtx.range_push("timed")  # profilers select this range (ncu --nvtx)
        ms = _time_steps(stream, step, args.steps)
        barrier()
        torch.cuda.nvtx.range_pop()
        launches = ctx.kernel_launches() - l0
        # one more step with per-stage CUDA events on the library's stream (passes then
        # launch kernels one by one instead of replaying the graph; same kernels)
        ctx.set_profiling(True)
        ctx.stage_times()
        ctx.stage_breakdown()
        p_ms = _time_steps(stream, step, 1)
        st = ctx.stage_times()
        stages = ctx.stage_breakdown()
        ctx.set_profiling(False)
    # e2e through the C ABI with host buffers: per step B uploads from pinned memory,
    # the group alignment, B downloads of the aligned stacks
    h_raw = torch.from_numpy(s.stack).pin_memory()
    h_out = torch.empty((nz, yo, xo), dtype=torch.float32).pin_memory()
    d_ins = [torch.empty_like(d_raw) for _ in range(B)]

    def step_e2e():
        with torch.cuda.stream(stream):
            for d in d_ins:
                d.copy_(h_raw, non_blocking=True)
        mf.align_many_device(ctx, d_ins, nx, ny, nz, angs, d_outs, **kw)
        with torch.cuda.stream(stream):
            for d in d_outs:
                h_out.copy_(d, non_blocking=True)

    log("batched timing done")
    step_e2e()
    barrier()
    e_ms = _time_steps(stream, step_e2e, args.steps)
    log("e2e timing done")
    h2d_bytes = int(s.stack.nbytes) * B
    d2h_bytes = int(h_out.numel() * 4 + 3 * nz * 4) * B
    # the pinned buffers recorded their copies on the library's stream: release them
    # while that stream exists
    del d_ins, h_raw, h_out, step_e2e
    torch.cuda.synchronize()
    # the plain path: one series at a time, FP32 (the reference's arithmetic)
    kw32 = dict(kw, precision=PRECISIONS["fp32"])
    d_one = d_outs[0]

    def step_plain():
        mf.align_device(ctx, d_raw, nx, ny, nz, s.angles, d_one, **kw32)

    for _ in range(2):
        step_plain()
    barrier()
    pl_ms = _time_steps(stream, step_plain, args.steps)
    log("plain timing done")
    ms, e_ms, pl_ms = max_over_ranks([ms, e_ms, pl_ms], f"cuda:{dev}", pg)
    ms_step = ms / args.steps
    value = 60000.0 * B / ms_step * world
    e2e_value = 60000.0 * B / (e_ms / args.steps) * world
    plain_value = 60000.0 / (pl_ms / args.steps) * world
    pk, src = peaks()
    # dominant kernel: the re-projection, one launch per step of a pass for the group
    launches_rep = max(st["reproj_launches"], 1)
    t_launch = st["reproj_ms"] / launches_rep / 1e3
    bytes_launch = st["reproj_bytes"] / launches_rep
    achieved = bytes_launch / t_launch / 1e9 if t_launch > 0 else 0.0
    tensor_tflops = 2.0 * st["reproj_fma"] / launches_rep / t_launch / 1e12 if t_launch else 0.0
    kname = ("k_op_apply (FP32 banded operator)" if prec == 0 else
             "k_reproject_tc (tcgen05, 16-bit operands, FP32 accumulation in TMEM)")
    roof_rep = {"kernel": kname + f", one launch per held-out tilt step for a group of {B}",
                "bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / pk["hbm_gbs"], "peak_source": src,
                "traffic": profiled_traffic("traffic_reproject.json"),
                "avg_launch_ms": t_launch * 1e3, "bytes_per_launch": bytes_launch,
                "tensor_tflops": tensor_tflops,
                "tensor_frac_of_bf16_peak": tensor_tflops / (pk.get("bf16_tflops", 1590.0)),
                "share_of_step": st["reproj_ms"] / max(p_ms, 1e-9),
                "rest_of_pass_share_of_step": st["xcorr_ms"] / max(p_ms, 1e-9),
                "profiled_ms_per_step": p_ms}
    # the tilt-axis Radon kernel, timed on its own in the profiled step: compulsory
    # bytes (each tilt image once, the lines once) over its time, and its gather rate
    n_rad = max(stages["radon_launches"], 1.0)
    t_rad = stages["radon_ms"] / n_rad / 1e3
    b_rad = stages["radon_bytes"] / n_rad
    a_rad = b_rad / t_rad / 1e9 if t_rad > 0 else 0.0
    roof_rad = {"kernel": "k_radon (common-line sums of 100 candidate axes x all tilts, one "
                          "launch per tilt-axis search of one series)",
                "bound": "hbm", "achieved": a_rad, "peak": pk["hbm_gbs"], "unit": "GB/s",
                "frac": a_rad / pk["hbm_gbs"], "peak_source": src,
                "traffic": profiled_traffic("traffic_radon.json"),
                "avg_launch_ms": t_rad * 1e3, "bytes_per_launch": b_rad,
                "samples_per_launch": stages["radon_samples"] / n_rad,
                "samples_per_s": stages["radon_samples"] / max(stages["radon_ms"] / 1e3, 1e-12),
                "share_of_step": stages["radon_ms"] / max(p_ms, 1e-9),
                "profiled_ms_per_step": p_ms,
                "note": "gather-bound: the tilt images are L2-resident while a launch "
                        "samples them; the HBM fraction counts compulsory bytes only"}
    # the dominant kernel of the step carries the roofline; the other is kept beside it
    if roof_rad["share_of_step"] >= roof_rep["share_of_step"]:
        roof, roof_other = roof_rad, roof_rep
    else:
        roof, roof_other = roof_rep, roof_rad
    cfg = workload_config(s, args.scale)
    cfg.update({"series_per_step": B, "grouping": f"{B} series per group (lockstep passes)"})
    line = {"metric": "series/min (2k^2, 61 tilts)", "value": value, "unit": "series/min",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if prec == 0 else f"{args.precision} operands, f32 accumulation",
            "data": "synthetic (seeded phantom series, BASELINE shapes)",
            "config": cfg,
            "e2e": {"value": e2e_value, "unit": "series/min",
                    "h2d_bytes_per_step": h2d_bytes, "d2h_bytes_per_step": d2h_bytes},
            "plain": {"value": plain_value, "unit": "series/min",
                      "what": "one series at a time, FP32 operands (mf_align_device)"},
            "batched_over_plain": value / plain_value,
            "gpu_launches": int(launches), "passes_per_series": last.get("passes"),
            "stage_ms_per_step": {k: round(v, 2) for k, v in stages.items()},
            "roofline": roof, "roofline_other": roof_other, "clocks": clk.summary()}
    if rank == 0 and world == 1 and not args.no_serve:
        log("serving run")
        line["served"] = served_run(mf, s, dev, args.serve_requests)
        log("serving run done")
        line["served_over_plain"] = line["served"]["equiv_2048_series_per_min"] / plain_value
    if rank == 0 and world == 1 and not args.no_cpu:
        line["cpu_baseline"] = cpu_sample(s, passes=max(last.get("passes", 1), 1))
    if rank == 0:
        print(json.dumps(line), flush=True)
    del d_outs, d_one, d_raw
    torch.cuda.synchronize()
    ctx.close()
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def run_kernel_case(args):
    """One stage of the workload on its own, for profilers (ncu -k ...): `reproject`
    re-projects one held-out tilt (full size, 10 neighbours) with the banded
    operator; `xcorr` measures one cross-correlation shift; `axis` runs one
    tilt-axis search (100 candidates over 20 degrees)."""
    import torch
    import markerfree_b200 as mf
    s = make_workload(args.scale)
    nz, ny, nx = s.stack.shape
    ctx = mf.Context(0)
    ang = s.angles
    zt = int(np.argmin(np.abs(ang)))
    ip = zt + 11
    skip = np.ones(nz, np.uint8)
    skip[zt - 10:zt + 11] = 0
    i0, i1 = mf.find_proj_range(ang, skip, ip, 10)
    g = torch.Generator(device="cuda").manual_seed(7)
    corr = torch.randn((nz, ny, nx), generator=g, device="cuda", dtype=torch.float32)
    out = torch.empty((ny, nx), device="cuda", dtype=torch.float32)
    if args.kernel_case == "axis":
        ser = mf.Series(ctx, s.stack, ang)
        p = ser.get_param()
        p.rotate[:] = s.axis  # candidates around the true axis, as in the refinements
        ser.set_param(p)
        for _ in range(args.steps):
            ser.tilt_axis(20.0)
        ctx.sync()
        print(json.dumps({"kernel_case": "axis", "tilts": nz}))
        return 0
    for _ in range(args.steps):
        if args.kernel_case == "reproject":
            mf.dev_reproject(ctx, corr, nx, ny, nz, ang, ip, i0, i1, s.thickness,
                             args.kernel_method, out)
        else:
            mf.dev_measure_shift(ctx, out, corr[ip], nx, ny)
    ctx.sync()
    print(json.dumps({"kernel_case": args.kernel_case, "range": [i0, i1], "ip": ip}))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--kernel-case", default=None, choices=["reproject", "xcorr", "axis"],
                    help="run one stage alone (profiling)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=float, default=1.0, help="shrink the workload (tests only)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--precision", default="fp16", choices=list(PRECISIONS),
                    help="re-projection operands of the batched path (fp32 = the reference's "
                         "arithmetic; the plain line is always fp32)")
    ap.add_argument("--batch", type=int, default=8, help="series per group (one step)")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-loop run")
    ap.add_argument("--serve-requests", type=int, default=20)
    ap.add_argument("--kernel-method", type=int, default=1,
                    help="re-projection method of --kernel-case reproject (1 FP32, 2 FP16, 3 BF16)")
    args = ap.parse_args()
    if args.kernel_case:
        return run_kernel_case(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
