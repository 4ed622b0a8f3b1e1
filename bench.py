"""Series/min of the B200 alignment path on the realistic single-series workload.

Workload: 2048 x 2048 x 61-tilt series (+-60 deg in 2 deg steps, tilt axis 84.7,
shifts N(0, 8 px) + 0.3 px/tilt drift, Poisson + Gaussian noise at SNR 0.05), run as
`-g 0,0,0,0,300,1,0 -p 10`: pre-processing, coarse alignment (3 x stretch cross-
correlation + tilt-axis search, tilt-angle offset search), the full projection-
matching schedule, and the aligned output stack.  Seeded synthetic data stands in
for the reference's simulated phantoms.

  value   series/min of the batched form: one step aligns --batch distinct series
          (default 8) in FP32 (--precision, the reference's arithmetic), projection
          matching in one lockstep group (mf_align_many_device), raw stacks already
          in HBM and aligned stacks written to HBM; summed over ranks (independent
          series).  FP16/BF16 operand forms are reported beside it.
  e2e     the same through the C ABI with host buffers: uploads of the raw stacks
          from pinned memory and downloads of the aligned stacks inside the timed
          region, overlapped with the neighbouring steps' alignment on a second
          stream (the serial form is reported beside it)
  plain   one series at a time in FP32 (mf_align_device)
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


SEED0 = 2000  # series j of a step uses seed SEED0 + j
# Projection-matching passes per series of this workload, the FP32 library path's
# mean over the seeds SEED0 .. SEED0 + 7 (bench runs report the live count as
# `passes_per_series`); the CPU restatement's series time is scaled with it.
PASSES_PER_SERIES = 6.5


def make_batch(n: int, device, scale: float = 1.0):
    """n distinct seeded series of the 2048^2 x 61-tilt workload (torch tensors)."""
    from markerfree_b200 import synth
    return [synth.config_fast(2, seed=SEED0 + j, device=device, scale=scale) for j in range(n)]


def workload_config(s, scale, batch):
    nz, ny, nx = s.stack.shape
    return {"workload": f"{nx}x{ny}x{nz}-tilt series (+-60 deg, 2 deg), T=300, -p 10: "
                        "pre-processing, coarse alignment, projection matching, aligned stack",
            "nx": nx, "ny": ny, "tilts": nz, "thickness": s.thickness, "nproj": 10,
            "scale": scale, "series_per_step": batch,
            "series": f"{batch} distinct seeded series per step (seeds {SEED0}..{SEED0 + batch - 1})",
            "grouping": f"{batch} series per group (lockstep passes)",
            "l2": "inputs (1 GiB raw stack per series) larger than L2 (126 MB)",
            "parallelism": "independent series per GPU"}


def cpu_sample(s, passes=PASSES_PER_SERIES, rows_target_s=0.8):
    """The reference algorithm on the host cores (the oracle's FP32 C++ restatement,
    OpenMP over all threads) on a bounded sample of one series of the workload,
    and the series time it implies.

    Sample (about 4 s): pre-processing of 4 tilts; one stretch cross-correlation
    pass (Transform::DoIt) over 3 tilts; a 180-degree and a 20-degree tilt-axis
    search (CalcTIltAxis) over 3 tilts; the offset search (FindOffset) over 3
    tilts; and for one held-out tilt of a projection-matching pass the re-
    projection of a block of rows (grown to about `rows_target_s`), one
    correction (resample + R-weight) and one cross-correlation measurement.
    Series time = pre-processing x Z/4 + 3 stretch passes x (Z-1)/2 + 3 180-degree
    and 4 20-degree searches x Z/3 + the offset search x (Z-1)/2 + `passes` x
    ((Z-1) x (re-projection of all rows + measurement + correction) + Z
    corrections): the reference's schedule (Process.cpp:238-319)."""
    from oracle import oracle as O
    raw = s.stack.cpu().numpy() if hasattr(s.stack, "cpu") else s.stack
    nz, ny, nx = raw.shape
    ang = s.angles
    zt = int(np.argmin(np.abs(ang)))
    t_all = time.time()
    t0 = time.time()
    O.preprocess(np.ascontiguousarray(raw[zt - 2:zt + 2]), ang[zt - 2:zt + 2])
    t_pre = (time.time() - t0) * nz / 4
    st = O.preprocess(raw, ang) if not hasattr(s, "_pre") else s._pre
    s._pre = st
    sub = np.ascontiguousarray(st[zt - 1:zt + 2])
    sa = np.ascontiguousarray(ang[zt - 1:zt + 2])
    p = O.Param(3)
    t0 = time.time()
    O.Transform(sub, sa, p).doit()
    t_tr = (time.time() - t0) * (nz - 1) / 2
    t0 = time.time()
    O.tilt_axis(sub, sa, p, 180.0)
    t_ax180 = (time.time() - t0) * nz / 3
    p.rotate[:] = float(s.axis)
    t0 = time.time()
    O.tilt_axis(sub, sa, p, 20.0)
    t_ax20 = (time.time() - t0) * nz / 3
    t0 = time.time()
    O.find_offset(sub, sa, p)
    t_off = (time.time() - t0) * (nz - 1) / 2
    ip = zt + 6
    skip = np.ones(nz, np.uint8)
    skip[zt - 5:zt + 6] = 0
    i0, i1 = O.find_proj_range(ang, skip, ip, 10)
    t0 = time.time()
    corr = np.stack([O.correct_proj(st[i], 0.0, 0.0, float(s.axis), rweight=True)
                     for i in (i0, ip)])
    t_corr = (time.time() - t0) / 2
    rows = 16
    while True:
        blk = np.zeros((nz, rows, nx), np.float32)
        for i in range(i0, i1 + 1):
            blk[i] = corr[0, ny // 2 - rows // 2: ny // 2 - rows // 2 + rows]
        t0 = time.time()
        O.reproject(blk, ang, ip, i0, i1, s.thickness)
        dt = time.time() - t0
        if dt > rows_target_s / 3 or rows >= ny:
            break
        rows = min(ny, int(rows * max(2.0, rows_target_s / max(dt, 1e-3) * 0.8)))
    t_rep = dt * ny / rows
    t0 = time.time()
    O.measure_shift(corr[1], corr[1])
    t_cc = time.time() - t0
    t_pass = (nz - 1) * (t_rep + t_cc + t_corr) + nz * t_corr
    series_s = t_pre + 3 * t_tr + 3 * t_ax180 + 4 * t_ax20 + t_off + passes * t_pass
    sample_s = time.time() - t_all
    ncpu = os.cpu_count() or 1
    return {"value": 60.0 / series_s, "unit": "series/min", "cores": ncpu, "kind": "port",
            "sample": (f"oracle/ FP32 C++ restatement, OpenMP over {ncpu} host threads, one "
                       f"{nx}x{ny}x{nz} series: pre-processing of 4 tilts, one stretch pass, "
                       f"a 180- and a 20-degree tilt-axis search and the offset search over 3 "
                       f"tilts, {rows}/{ny} re-projected rows of one held-out tilt with "
                       f"{i1 - i0 + 1} neighbours, one correction, one cross-correlation; "
                       f"scaled to the reference's schedule with {passes:g} projection-matching "
                       f"passes (mean of the library's FP32 runs on these seeds)"),
            "seconds_per_series": series_s, "sample_s": sample_s,
            "stage_s_per_series": {"pre": t_pre, "stretch_passes": 3 * t_tr,
                                   "axis_searches": 3 * t_ax180 + 4 * t_ax20, "offset": t_off,
                                   "projection_matching": passes * t_pass}}


def run_reference(args):
    """The reference's CPU implementation of the path, timed on the host cores.  The
    reference program runs every stage on the GPU and has no CPU implementation,
    so the oracle's FP32 restatement stands in.  A step is one bounded sample of
    the workload (cpu_sample); `ms_per_step` is its wall time and `value` the
    series/min that sample implies, so value = series_fraction_per_step x 60000 /
    ms_per_step."""
    rank, world, local = dist_env()
    if rank != 0:
        return 0
    s = make_batch(1, "cpu", args.scale)[0]
    for _ in range(args.warmup):
        cpu_sample(s)
    t0 = time.time()
    samples = [cpu_sample(s) for _ in range(max(1, args.steps))]
    wall = time.time() - t0
    v = statistics.median(x["value"] for x in samples)
    ms_step = 1000.0 * wall / len(samples)
    cb = dict(samples[len(samples) // 2])
    cb["value"] = v
    line = {"metric": "series/min (2k^2, 61 tilts)", "value": v, "unit": "series/min",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded phantom series)",
            "config": workload_config(s, args.scale, args.batch), "impl": "reference",
            "series_fraction_per_step": v * ms_step / 60000.0,
            "cpu_baseline": cb,
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


def device_memory(dev):
    """Device memory in GB: free, torch's cache, and the stream-ordered pool the
    library allocates from (reserved / in use; needs cuda-python)."""
    import torch
    free, total = torch.cuda.mem_get_info(dev)
    out = f"free {free / 1e9:.1f}/{total / 1e9:.1f} GB, torch {torch.cuda.memory_reserved(dev) / 1e9:.1f}"
    try:
        from cuda.bindings import runtime as rt
        _, pool = rt.cudaDeviceGetDefaultMemPool(dev)
        _, res = rt.cudaMemPoolGetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrReservedMemCurrent)
        _, used = rt.cudaMemPoolGetAttribute(pool, rt.cudaMemPoolAttr.cudaMemPoolAttrUsedMemCurrent)
        out += f", pool {int(res) / 1e9:.1f} reserved / {int(used) / 1e9:.1f} in use"
    except Exception:  # cuda-python absent
        pass
    return out


def served_pool(dev):
    """Distinct seeded series for the serving run, by size class (2048^2, 1024^2,
    4096^2), each drawn like the uneven batch (synth.uneven_params with the size
    fixed: 31/41/61 tilts, slab 150/200/300, axis, SNR); 4096^2 is auto-binned to
    2048^2 for matching, as the reference does.
    Returns {class: [(pinned host tensor, angles, thickness), ...]}."""
    import torch
    from markerfree_b200 import synth
    pool = {}
    for key, size, count, seed0 in (("2048", 2048, 4, 5000), ("1024", 1024, 3, 5100),
                                    ("4096", 4096, 2, 5200)):
        out = []
        for j in range(count):
            s = synth.uneven_series(j, f"cuda:{dev}", size=size, seed0=seed0)
            h = torch.empty(s.stack.shape, dtype=torch.float32).pin_memory()
            h.copy_(s.stack)
            out.append((h, s.angles, s.thickness))
            del s
        pool[key] = out
    torch.cuda.empty_cache()
    return pool


def served_run(mf, dev, n_req, precision, seed=5):
    """The serving loop (continuous batching) on the served-request mix: sizes 50%
    2048^2, 30% 1024^2, 20% 4096^2, each request one of a pool of distinct seeded
    series of its size class (tilt counts and slab thicknesses vary too), from
    pinned host memory; requests of any shape share groups; results are the
    per-tilt parameters.

    Capacity: all n_req requests arrive at once; series/min = n_req / makespan
    (also in 2048^2-equivalents, weighting each request by its pixel count).
    Latency: a Poisson stream of n_req requests at 80% of that capacity; p50/p99
    of arrival-to-result."""
    pool = served_pool(dev)
    weight = {"2048": 1.0, "1024": 0.25, "4096": 4.0}
    rng = np.random.default_rng(seed)
    n4 = max(1, round(0.2 * n_req))
    n1 = max(1, round(0.3 * n_req))
    kinds = ["4096"] * n4 + ["1024"] * n1 + ["2048"] * (n_req - n4 - n1)
    rng.shuffle(kinds)
    picks = [int(rng.integers(len(pool[k]))) for k in kinds]

    def submit(srv, k, j):
        t, ang, az = pool[k][j]
        return srv.submit(None, ang, raw_ptr=t.data_ptr(), shape=tuple(t.shape), align_z=az,
                          nproj=10, precision=precision)

    # capacity: everything queued at once
    srv = mf.Server(gpu=dev, hbm_budget=0, max_group=8, workers=3, group_wait_ms=40.0)
    try:
        t0 = time.perf_counter()
        ids = [submit(srv, k, j) for k, j in zip(kinds, picks)]
        for i in ids:
            srv.wait(i, timeout_s=1800.0)
        makespan = time.perf_counter() - t0
        st_cap = srv.stats()
    finally:
        srv.close()
        print(f"[bench] serving capacity run over | {device_memory(dev)}", file=sys.stderr,
              flush=True)
    cap_spm = 60.0 * n_req / makespan
    cap_eq = 60.0 * sum(weight[k] for k in kinds) / makespan
    # latency: Poisson arrivals at 80% of the capacity just measured
    rate_per_s = 0.8 * cap_spm / 60.0
    arrivals = np.cumsum(rng.exponential(1.0 / rate_per_s, n_req))
    srv = mf.Server(gpu=dev, hbm_budget=0, max_group=8, workers=3, group_wait_ms=40.0)
    try:
        ids = []
        t0 = time.perf_counter()
        for k, j, ta in zip(kinds, picks, arrivals):
            wait = ta - (time.perf_counter() - t0)
            if wait > 0:
                time.sleep(wait)
            ids.append(submit(srv, k, j))
        lats = [srv.wait(i, timeout_s=1800.0)[2] for i in ids]
        st_lat = srv.stats()
    finally:
        srv.close()
    return {"requests": n_req, "mix": {"2048": kinds.count("2048"), "1024": kinds.count("1024"),
                                       "4096": kinds.count("4096")},
            "distinct_series": {k: len(v) for k, v in pool.items()},
            "series_per_min": cap_spm, "equiv_2048_series_per_min": cap_eq,
            "capacity_makespan_s": makespan, "capacity_mean_group_size": st_cap["mean_group"],
            "peak_admitted_gb": st_cap["peak_bytes"] / 1e9,
            "budget_gb": st_cap["budget_bytes"] / 1e9,
            "learned_budget_gb": st_cap["learned_budget_bytes"] / 1e9,
            "memory_retries": st_cap["memory_retries"] + st_lat["memory_retries"],
            "latency_arrival_rate_per_min": rate_per_s * 60.0,
            "p50_s": st_lat["p50_s"], "p99_s": st_lat["p99_s"],
            "mean_latency_s": float(np.mean(lats)), "latency_mean_group_size": st_lat["mean_group"],
            "precision": {0: "f32", 1: "bf16 operands, f32 accumulation",
                          2: "fp16 operands, f32 accumulation"}[precision],
            "returns": "per-tilt parameters (aligned stacks not copied back)"}


def uneven_run(mf, ctx, stream, dev, precisions, n=32, per_call=16, steps=1):
    """The uneven batch: n distinct seeded series of sizes U{1024..4096}^2, 31/41/61
    tilts over +-45..60 degrees, slab 150/200/300, axis U(80, 95), SNR
    U(0.03, 0.2) (synth.uneven_params), raw stacks resident in HBM.  One step
    aligns all n through mf_align_batch_device, per_call series per call, each
    call one lockstep group whose every stage is one launch over series of
    different sizes; no output stacks.  Returns series/min per precision."""
    import torch
    from markerfree_b200 import synth
    series = [synth.uneven_series(j, f"cuda:{dev}") for j in range(n)]
    torch.cuda.synchronize()
    out = {"series": n, "per_call": per_call,
           "sizes": sorted({int(s.stack.shape[2]) for s in series}),
           "tilts": sorted({int(s.stack.shape[0]) for s in series}),
           "raw_gb": sum(s.stack.numel() * 4 for s in series) / 1e9}
    for prec in precisions:
        passes = []

        def step():
            passes.clear()
            for h in range(0, n, per_call):
                part = series[h:h + per_call]
                _, ps = mf.align_batch_device(ctx, [s.stack for s in part], [s.angles for s in part],
                                              [s.thickness for s in part], None, nproj=10,
                                              precision=PRECISIONS[prec])
                passes.extend(int(x) for x in ps)

        step()
        torch.cuda.synchronize()
        ms = _time_steps(stream, step, steps)
        out[prec] = {"value": 60000.0 * n / (ms / steps), "unit": "series/min", "steps": steps,
                     "mean_passes": float(np.mean(passes))}
    del series
    torch.cuda.empty_cache()
    return out


def _params_diff(pa, pb):
    """Largest tilt-axis (deg) and shift (px) difference between two Param lists."""
    ax = max(float(np.abs(a.rotate.astype(np.float64) - b.rotate).max()) for a, b in zip(pa, pb))
    sh = max(float(max(np.abs(a.shift_x - b.shift_x).max(), np.abs(a.shift_y - b.shift_y).max()))
             for a, b in zip(pa, pb))
    return ax, sh


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

    def log(m):
        print(f"[bench] {m} | {device_memory(dev)}", file=sys.stderr, flush=True)
    B = args.batch
    series = make_batch(B, f"cuda:{dev}", args.scale)
    s0 = series[0]
    nz, ny, nx = s0.stack.shape
    xo, yo = mf.binned_size(nx, ny, 1)
    d_raws = [s.stack for s in series]
    angs = [s.angles for s in series]
    ctx = mf.Context(dev)
    stream = torch.cuda.ExternalStream(ctx.stream_ptr(), device=f"cuda:{dev}")
    prec = PRECISIONS[args.precision]
    kw = dict(offset=0.0, pitch_angle=0.0, zshift=0.0, align_z=s0.thickness, out_bin=1, nproj=10,
              precision=prec)
    d_outs = [torch.empty((nz, yo, xo), dtype=torch.float32, device=f"cuda:{dev}")
              for _ in range(B)]
    torch.cuda.synchronize()
    log(f"workload ready: {B} distinct {nx}x{ny}x{nz} series")

    def barrier():
        if pg is not None:
            pg.barrier()
        torch.cuda.synchronize()

    last = {}

    def step():
        ps, passes = mf.align_many_device(ctx, d_raws, nx, ny, nz, angs, d_outs, **kw)
        last["params"] = ps
        last["passes"] = float(np.mean(passes))

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
        # one more step with per-stage CUDA events on the library's stream
        ctx.set_profiling(True)
        ctx.stage_times()
        ctx.stage_breakdown()
        p_ms = _time_steps(stream, step, 1)
        st = ctx.stage_times()
        stages = ctx.stage_breakdown()
        ctx.set_profiling(False)
    params_main = last["params"]
    passes_main = last["passes"]
    log("batched timing done")
    # e2e through the C ABI with host buffers: per step B uploads from pinned memory,
    # the group alignment, B downloads of the aligned stacks.  Two forms:
    #  * serial: upload, align, download one after another on the library's stream;
    #  * pipelined (the reported e2e): a second stream uploads step i+1's stacks and
    #    downloads step i-1's aligned stacks while step i aligns (inputs and outputs
    #    double-buffered, events order the three); the timed region starts before
    #    the first upload and ends after the last download.
    # (built without loop variables: a pinned buffer still referenced when the
    # context's stream is gone would record its release on a destroyed stream)
    h_raws = [torch.empty(d.shape, dtype=torch.float32).pin_memory() for d in d_raws]
    for i in range(B):
        h_raws[i].copy_(d_raws[i])
    h_out = torch.empty((nz, yo, xo), dtype=torch.float32).pin_memory()
    d_ins = [[torch.empty_like(d_raws[0]) for _ in range(B)] for _ in range(2)]
    d_outs2 = [d_outs, [torch.empty_like(d_outs[0]) for _ in range(B)]]
    copy_stream = torch.cuda.Stream(device=f"cuda:{dev}")

    def step_e2e():
        with torch.cuda.stream(stream):
            for d, h in zip(d_ins[0], h_raws):
                d.copy_(h, non_blocking=True)
        mf.align_many_device(ctx, d_ins[0], nx, ny, nz, angs, d_outs, **kw)
        with torch.cuda.stream(stream):
            for d in d_outs:
                h_out.copy_(d, non_blocking=True)

    def run_pipelined(steps):
        up = [torch.cuda.Event(), torch.cuda.Event()]
        done = [torch.cuda.Event(), torch.cuda.Event()]
        down = [torch.cuda.Event(), torch.cuda.Event()]
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        t0.record(stream)
        copy_stream.wait_event(t0)

        def upload(j):
            with torch.cuda.stream(copy_stream):
                for d, h in zip(d_ins[j % 2], h_raws):
                    d.copy_(h, non_blocking=True)
            up[j % 2].record(copy_stream)

        upload(0)
        for i in range(steps):
            k = i % 2
            if i + 1 < steps:
                if i >= 1:
                    copy_stream.wait_event(done[(i + 1) % 2])  # step i-1 read those inputs
                upload(i + 1)
            stream.wait_event(up[k])
            if i >= 2:
                stream.wait_event(down[k])  # step i-2's outputs have left the device
            mf.align_many_device(ctx, d_ins[k], nx, ny, nz, angs, d_outs2[k], **kw)
            done[k].record(stream)
            copy_stream.wait_event(done[k])
            with torch.cuda.stream(copy_stream):
                for d in d_outs2[k]:
                    h_out.copy_(d, non_blocking=True)
            down[k].record(copy_stream)
        stream.wait_event(down[(steps - 1) % 2])
        t1.record(stream)
        torch.cuda.synchronize()
        return t0.elapsed_time(t1)

    step_e2e()
    barrier()
    es_ms = _time_steps(stream, step_e2e, args.steps)
    run_pipelined(2)
    barrier()
    e_ms = run_pipelined(args.steps)
    log("e2e timing done")
    h2d_bytes = int(sum(h.numel() for h in h_raws) * 4)
    d2h_bytes = int(h_out.numel() * 4 + 3 * nz * 4) * B
    # the pinned buffers recorded their copies on the library's stream: release them
    # while that stream exists
    del d_ins, d_outs2, h_raws, h_out, step_e2e, run_pipelined
    torch.cuda.synchronize()
    k_extra = max(1, min(args.steps, 3))
    # the 16-bit operand forms of the same step, with their distance from the FP32 result
    mixed = {}
    for name in ("fp16", "bf16"):
        if args.no_mixed or PRECISIONS[name] == prec:
            continue
        kwm = dict(kw, precision=PRECISIONS[name])

        def step_m():
            ps, passes = mf.align_many_device(ctx, d_raws, nx, ny, nz, angs, d_outs, **kwm)
            last["m_params"], last["m_passes"] = ps, float(np.mean(passes))

        step_m()
        barrier()
        if name == "fp16":
            ctx.set_profiling(True)
            ctx.stage_times()
            ctx.stage_breakdown()
            pm_ms = _time_steps(stream, step_m, 1)
            st_m = ctx.stage_times()
            ctx.stage_breakdown()
            ctx.set_profiling(False)
        m_ms = _time_steps(stream, step_m, k_extra)
        dax, dsh = _params_diff(last["m_params"], params_main)
        mixed[name] = {"value": 60000.0 * B / (m_ms / k_extra) * world, "unit": "series/min",
                       "steps": k_extra, "passes_per_series": last["m_passes"],
                       "max_axis_diff_vs_f32_deg": dax, "max_shift_diff_vs_f32_px": dsh}
        if name == "fp16":
            mixed[name]["reproject_stage_times"] = st_m
            mixed[name]["profiled_ms_per_step"] = pm_ms
    log("mixed-precision timing done")
    # the plain path: one series at a time (mf_align_device), FP32, the same series
    kw32 = dict(kw, precision=PRECISIONS["fp32"])

    def step_plain():
        for d, a, o in zip(d_raws, angs, d_outs):
            mf.align_device(ctx, d, nx, ny, nz, a, o, **kw32)

    step_plain()
    barrier()
    pl_ms = _time_steps(stream, step_plain, k_extra)
    log("plain timing done")
    ms, e_ms, es_ms, pl_ms = max_over_ranks([ms, e_ms, es_ms, pl_ms], f"cuda:{dev}", pg)
    ms_step = ms / args.steps
    value = 60000.0 * B / ms_step * world
    e2e_value = 60000.0 * B / (e_ms / args.steps) * world
    e2e_serial = 60000.0 * B / (es_ms / args.steps) * world
    plain_value = 60000.0 * B / (pl_ms / k_extra) * world
    pk, src = peaks()

    def reproj_roof(stt, kname, prof_ms, traffic_file):
        launches_rep = max(stt["reproj_launches"], 1)
        t_launch = stt["reproj_ms"] / launches_rep / 1e3
        bytes_launch = stt["reproj_bytes"] / launches_rep
        achieved = bytes_launch / t_launch / 1e9 if t_launch > 0 else 0.0
        flops = 2.0 * stt["reproj_fma"] / launches_rep / t_launch / 1e12 if t_launch else 0.0
        return {"kernel": kname + f", one launch per held-out tilt step for a group of {B}",
                "bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / pk["hbm_gbs"], "peak_source": src,
                "traffic": profiled_traffic(traffic_file),
                "avg_launch_ms": t_launch * 1e3, "bytes_per_launch": bytes_launch,
                "tflops": flops, "share_of_step": stt["reproj_ms"] / max(prof_ms, 1e-9),
                "rest_of_pass_share_of_step": stt["xcorr_ms"] / max(prof_ms, 1e-9),
                "profiled_ms_per_step": prof_ms}

    roof_rep = reproj_roof(st, "k_op_apply (FP32 banded operator, SIMT FMA)" if prec == 0 else
                           "k_reproject_tc (tcgen05, 16-bit operands, FP32 accumulation in TMEM)",
                           p_ms, "traffic_op_apply.json" if prec == 0 else
                           "traffic_reproject.json")
    roof_rep["note"] = ("FP32 FMA-bound on the banded operator; the HBM fraction counts "
                        "compulsory bytes (neighbour rows, operator, output)") if prec == 0 else ""
    if prec == 0:
        # the bound that applies: the SIMT FP32 pipe (nominal: 148 SMs x 128 lanes x
        # 2 flops at the sampled SM clock)
        mhz = clk.summary().get("sm_mhz") or 1965.0
        fp32_peak = 148 * 128 * 2 * float(mhz) * 1e6 / 1e12
        roof_rep["fp32_peak_tflops"] = fp32_peak
        roof_rep["fp32_frac"] = roof_rep["tflops"] / fp32_peak
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
                "note": "instruction-issue-bound (every sample: six FP32 coordinate ops, "
                        "the integer byte offset, the gather, the in-order line add); the "
                        "tilt images are L2/L1-resident while a launch samples them, so the "
                        "HBM fraction counts compulsory bytes only"}
    # the dominant kernel of the step carries the roofline; the others are kept beside it
    if roof_rad["share_of_step"] >= roof_rep["share_of_step"]:
        roof, others = roof_rad, [roof_rep]
    else:
        roof, others = roof_rep, [roof_rad]
    if "fp16" in mixed:
        others.append(reproj_roof(mixed["fp16"].pop("reproject_stage_times"),
                                  "k_reproject_tc (tcgen05, FP16 operands, FP32 accumulation in "
                                  "TMEM; fp16 form of the step)",
                                  mixed["fp16"].pop("profiled_ms_per_step"),
                                  "traffic_reproject.json"))
    cfg = workload_config(s0, args.scale, B)
    line = {"metric": "series/min (2k^2, 61 tilts)", "value": value, "unit": "series/min",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if prec == 0 else f"{args.precision} operands, f32 accumulation",
            "data": "synthetic (seeded phantom series)",
            "config": cfg,
            "e2e": {"value": e2e_value, "unit": "series/min",
                    "h2d_bytes_per_step": h2d_bytes, "d2h_bytes_per_step": d2h_bytes,
                    "form": "pipelined: a second stream uploads the next step's stacks and "
                            "downloads the previous step's aligned stacks while a step "
                            "aligns (double-buffered); first upload to last download timed",
                    "serial_value": e2e_serial},
            "plain": {"value": plain_value, "unit": "series/min", "steps": k_extra,
                      "what": "the same series one at a time, FP32 (mf_align_device)"},
            "batched_over_plain": value / plain_value,
            "mixed_precision": mixed,
            "gpu_launches": int(launches), "passes_per_series": passes_main,
            "tc_tuning": ctx.tc_tuning(),
            "stage_ms_per_step": {k: round(v, 2) for k, v in stages.items()},
            # inside pass_ms: the re-projection of every held-out-tilt step, and its
            # measurement (normalise, FFTs, filter, peak) with the re-correction
            "pass_ms_split": {"reproject_ms": round(st["reproj_ms"], 2),
                              "measure_recorrect_ms": round(st["xcorr_ms"], 2)},
            "roofline": roof, "roofline_other": others, "clocks": clk.summary()}
    if rank == 0 and world == 1 and not args.no_uneven:
        log("uneven batch")
        del d_outs
        torch.cuda.empty_cache()
        d_outs = None
        try:
            line["uneven_batch"] = uneven_run(mf, ctx, stream, dev, [args.precision, "fp16"])
        except mf.MfError as e:  # recorded, the headline line still prints
            line["uneven_batch"] = {"error": str(e)}
        log("uneven batch done")
    # the serving run and the CPU sample need none of the above: release the
    # stacks and the context (with its cuFFT plans) first
    del d_raws, series, s0
    d_outs = None
    torch.cuda.synchronize()
    ctx.close()
    ctx = None
    torch.cuda.empty_cache()
    if rank == 0 and world == 1 and not args.no_serve:
        log("serving run")
        try:
            line["served"] = served_run(mf, dev, args.serve_requests, PRECISIONS["fp16"])
            line["served_over_plain"] = (line["served"]["equiv_2048_series_per_min"] /
                                         plain_value)
        except mf.MfError as e:  # recorded, the headline line still prints
            line["served"] = {"error": str(e)}
        log("serving run done")
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = make_batch(1, "cpu", args.scale)[0]
        cpu_sample(cpu)  # pre-processes the series once
        line["cpu_baseline"] = cpu_sample(cpu)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def run_kernel_case(args):
    """One stage of the workload on its own, for profilers (ncu -k ...): `reproject`
    re-projects one held-out tilt (full size, 10 neighbours) with the banded
    operator; `xcorr` measures one cross-correlation shift; `axis` runs one
    tilt-axis search (100 candidates over 20 degrees); `pass` runs projection-
    matching passes of a group of --batch series in --precision; `coarse`
    pre-processes and coarsely aligns one series per step."""
    import torch
    import markerfree_b200 as mf
    s = make_batch(1, "cuda:0", args.scale)[0]
    s.stack = s.stack.cpu().numpy()
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
    if args.kernel_case == "pass":
        # one projection-matching pass of a group of --batch series (every pass kernel)
        batch = make_batch(args.batch, "cuda:0", args.scale)
        sers = []
        for b in batch:
            ser = mf.Series(ctx, b.stack.cpu().numpy(), b.angles)
            ser.set_precision(PRECISIONS[args.precision])
            p = ser.get_param()
            p.rotate[:] = b.axis
            ser.set_param(p)
            sers.append(ser)
        grp = mf.Group(sers, 0.0, batch[0].thickness, 10)
        for _ in range(args.steps):
            grp.doit()
        ctx.sync()
        grp.close()
        print(json.dumps({"kernel_case": "pass", "series": len(sers), "tilts": nz}))
        return 0
    if args.kernel_case == "coarse":
        # pre-processing and coarse alignment of one series per step (stretch
        # cross-correlations, three tilt-axis searches, the offset search)
        for _ in range(args.steps):
            ser = mf.Series(ctx, s.stack, ang)
            ser.coarse_align(0.0, 0.0)
            ser.close()
        ctx.sync()
        print(json.dumps({"kernel_case": "coarse", "tilts": nz}))
        return 0
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
    ap.add_argument("--kernel-case", default=None, choices=["reproject", "xcorr", "axis", "pass", "coarse"],
                    help="run one stage alone (profiling)")
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=float, default=1.0, help="shrink the workload (tests only)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline sample")
    ap.add_argument("--precision", default="fp32", choices=list(PRECISIONS),
                    help="re-projection operands of the headline batched path (fp32 = the "
                         "reference's arithmetic; the plain line is always fp32)")
    ap.add_argument("--no-mixed", action="store_true",
                    help="skip the fp16/bf16 forms of the batched step")
    ap.add_argument("--batch", type=int, default=8, help="series per group (one step)")
    ap.add_argument("--no-serve", action="store_true", help="skip the serving-loop run")
    ap.add_argument("--no-uneven", action="store_true", help="skip the uneven-batch run")
    ap.add_argument("--serve-requests", type=int, default=100)
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
