#!/usr/bin/env python
"""Benchmark of the VPL gather hot path on the scaled scene.

Workload ("scaled gather"): the room filled with 2,000 seeded boxes and UV spheres
(~300k triangles, 60/25/15 % Lambertian/Phong/Ward), 512 x 512 pixel-centre primary hits
(262,144 shading points), 32,768 VPLs traced on the device from the ceiling light
(max bounce 3, the first 32,768 in push order), RADIANCE clamp at 0.1 x the mean
unclamped contribution over 65,536 seeded pairs.  One step = the full gather: every
shading point x every VPL, shadow ray through the LBVH, both BRDFs, clamp, summed per
pixel (8.59e9 evaluations).  Inputs are resident in HBM; the L2 is flushed between
steps by writing a 256 MiB buffer outside the timed region.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Prints one JSON line.  Under torchrun each rank runs an independent replica of the
workload (weak scaling, no data-path collective); the timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "VPL-gather evals/s (shading-point x VPL evaluations with shadow rays)"
N_VPL = 32768
WIDTH = HEIGHT = 512
VPL_SEED = 2015
VPL_PARTICLES = 24000
MAX_BOUNCE = 3
TAU_PAIRS = 65536
# DRAM bytes (read + write) of one full gather launch of this workload, from the one-pass
# capture `ncu --metrics dram__bytes_read.sum,dram__bytes_write.sum --clock-control none
# -k regex:gather_persistent -s 3 -c 1 python bench.py --steps 1 --warmup 3 --skip-cpu
# --serve-duration 0` (36.76 MB read, 55.23 MB written; the writes are the per-chunk partial
# sums), recorded in profiles/.
TRAFFIC_BYTES_PER_LAUNCH = (36.76 + 55.23) * 1e6
# Warp instructions of one full gather launch of this workload (smsp__inst_executed.sum from
# the same one-pass capture, recorded in profiles/): the gather is instruction-issue bound
# (HBM idle, its ~34 MB working set in L2), so the roofline compares the issue rate it
# reaches with the SMs' peak of one warp instruction per scheduler per cycle.
INST_PER_LAUNCH = 89574058624
# The same for the secondary workloads' dominant kernels (one full launch each, same capture
# recipe; see profiles/): LightSlice's and MRCS's tracing passes and the guided path kernel.
LS_VIS_INST = 8194992935
MRCS_VIS_INST = 1532559557
GUIDED_INST = 407466344613


def workload_config():
    return {"workload": "scaled_gather_room_objects_300k_tris_512x512_32768_vpls",
            "scene": "room + light + 2000 seeded boxes/UV spheres (~300k triangles)",
            "shading_points": WIDTH * HEIGHT, "vpls": N_VPL, "max_bounce": MAX_BOUNCE,
            "clamp": "RADIANCE, tau = 0.1 x mean contribution over 65,536 seeded pairs",
            "l2": "flushed between timed steps (256 MiB write)", "parallelism": "replicas"}


# ---------------------------------------------------------------------------------------
def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def init_ranks(backend: str = "nccl", timeout_s: int = 120):
    """One process per GPU under torchrun: the process group (None for a single process),
    rendezvous on 127.0.0.1, with a short timeout so that a rank that never arrives ends the
    others' collectives with an error."""
    ws, _, _ = _dist()
    if ws <= 1:
        return None
    import datetime
    import torch.distributed as dist
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def max_over_ranks(pg, x: float, device) -> float:
    """The largest x over all ranks (every rank gets it); x itself without a group."""
    if pg is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def job_rate(world_size: int, units_per_rank_step: float, steps: int, max_seconds: float) -> float:
    """Whole-job throughput of replicas: every rank processes units_per_rank_step per step,
    the job takes as long as its slowest rank."""
    return world_size * units_per_rank_step * steps / max_seconds


class ClockSampler:
    """nvidia-smi clock / throttle-reason samples while the timed region runs."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def graph_kernels(g) -> int:
    """Kernel nodes of a captured torch CUDA graph (made with keep_graph=True)."""
    from cuda.bindings import runtime as rt
    graph = g.raw_cuda_graph()
    err, _, n = rt.cudaGraphGetNodes(graph, 0)
    err, nodes, n = rt.cudaGraphGetNodes(graph, n)
    if err != rt.cudaError_t.cudaSuccess:
        raise RuntimeError(f"cudaGraphGetNodes: {err}")
    kernel = rt.cudaGraphNodeType.cudaGraphNodeTypeKernel
    return sum(1 for x in nodes[:n] if rt.cudaGraphNodeGetType(x)[1] == kernel)


def kernels_per_call(fn, capture: bool = True):
    """Kernels one call of `fn` launches.  capture=True: `fn` (already warmed up, so that
    it allocates nothing) is captured once into a CUDA graph on the current stream and the
    graph's kernel nodes are counted.  capture=False, for calls that synchronise mid-way
    and so cannot be captured: one call runs under the CUDA activity profiler and its
    device events other than copies and memsets are counted."""
    import torch
    torch.cuda.synchronize()
    if not capture:
        from torch.autograd import DeviceType
        from torch.profiler import ProfilerActivity, profile
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            fn()
            torch.cuda.synchronize()
        n = sum(1 for e in prof.events() if e.device_type == DeviceType.CUDA
                and not e.name.startswith(("Memcpy", "Memset")))
        # None: the activity profiler saw nothing (another profiler, e.g. ncu, holds it)
        return n if n > 0 else None
    g = torch.cuda.CUDAGraph(keep_graph=True)
    with torch.cuda.graph(g, capture_error_mode="thread_local"):
        fn()
    torch.cuda.synchronize()
    n = graph_kernels(g)
    del g
    return n


def issue_roofline(inst, step_s, sm_mhz, kernel, note):
    """Issue-rate roofline of an instruction-bound kernel: its warp instructions per launch
    (ncu smsp__inst_executed.sum, recorded in profiles/) over the live step time, against
    SMs x 4 schedulers x one warp instruction per cycle at the sampled SM clock."""
    import torch
    sms = torch.cuda.get_device_properties(torch.cuda.current_device()).multi_processor_count
    mhz = sm_mhz or 1965.0
    peak = sms * 4 * mhz * 1e6
    ach = inst / step_s if inst else None
    return {"bound": "issue", "unit": "Gwarp-inst/s", "kernel": kernel,
            "achieved": None if ach is None else ach / 1e9, "peak": peak / 1e9,
            "frac": None if ach is None else ach / peak, "inst_per_launch": inst,
            "peak_source": f"{sms} SMs x 4 schedulers x 1 warp instruction per cycle at {mhz:.0f} MHz (sampled)",
            "note": note}


def cpu_scene_inputs(sc):
    """Receivers, VPLs and tau computed on the host (reference arm / CPU baseline)."""
    from oracle import Oracle, RefHarness
    o = Oracle(sc)
    recv = o.primary(Oracle.camera(sc.camera), threads=os.cpu_count() or 1)
    vpls = o.vpl_generate(VPL_SEED, VPL_PARTICLES, MAX_BOUNCE)
    return o, recv, vpls


def select_vpls(vpls: np.ndarray):
    v = vpls[:N_VPL]
    num_emitted = int(v["path"][-1]) + 1
    return v, num_emitted


def cpu_timer_impl():
    """(name, gather function) of the CPU reference: the reference's own code compiled by
    oracle/Makefile when available, else the C restatement."""
    from oracle import RefHarness
    return "reference" if RefHarness.available() else "port"


def cpu_rate(sc, o, recv, vpls, tau, scale, budget_s: float, threads: int):
    """Evaluations/s of the CPU path on a bounded, evenly spaced receiver sample."""
    from oracle import RefHarness
    kind = cpu_timer_impl()
    if kind == "reference":
        ref = RefHarness(sc)
        run = lambda r: ref.gather_mt(r, vpls, 3, tau, scale, threads)
    else:
        run = lambda r: o.gather(r, vpls, 3, tau, scale, cull=False, threads=threads)[0]
    # seeded uniform sample of all shading points (misses included, as on the GPU);
    # calibrate on a small slice, then size the sample to the time budget
    order = np.random.default_rng(VPL_SEED + 1).permutation(recv.shape[0])
    cal = recv[np.sort(order[:64])].copy()
    t0 = time.perf_counter()
    run(cal)
    dt = max(time.perf_counter() - t0, 1e-3)
    per_recv = dt / cal.shape[0]
    n = int(max(threads, min(recv.shape[0], budget_s / per_recv)))
    sample = recv[np.sort(order[:n])].copy()
    return kind, sample, run


# ---------------------------------------------------------------------------------------
def run_reference(args):
    ws, rank, local = _dist()
    if rank != 0:
        return 0
    from renzoku_b200 import scenegen as sg
    sc = sg.room_objects(2000, WIDTH, HEIGHT)
    o, recv, vpls_all = cpu_scene_inputs(sc)
    vpls, num_emitted = select_vpls(vpls_all)
    hit_idx = np.nonzero(recv["mat"] >= 0)[0]
    rng = np.random.default_rng(VPL_SEED)
    from oracle import Oracle
    ri = np.array([Oracle.draw_u32(VPL_SEED, 3, k, 0) % recv.shape[0] for k in range(TAU_PAIRS)], np.int32)
    vi = np.array([Oracle.draw_u32(VPL_SEED, 3, k, 1) % vpls.shape[0] for k in range(TAU_PAIRS)], np.int32)
    tau = float(np.float32(0.1 * o.mean_contribution(recv, ri, vi, vpls)))
    threads = os.cpu_count() or 1
    kind, sample, run = cpu_rate(sc, o, recv, vpls, tau, 1.0 / num_emitted, 6.0, threads)
    for _ in range(args.warmup):
        run(sample)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        run(sample)
        times.append(time.perf_counter() - t0)
    evals = sample.shape[0] * vpls.shape[0]
    v = evals * len(times) / sum(times)
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "evals/s", "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": workload_config(),
            "cpu_baseline": {"value": v, "unit": "evals/s", "cores": threads, "kind": kind,
                             "sample": f"{sample.shape[0]} seeded uniformly sampled shading points x {vpls.shape[0]} VPLs per step"},
            "e2e": {"value": v, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


def run_ours(args):
    import torch
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    pg = init_ranks("nccl")
    from renzoku_b200 import build as rbuild
    if rank == 0 or not os.path.exists(rbuild.LIB):
        rbuild.build()
    if pg:
        pg.barrier()
    from renzoku_b200 import rzk, scenegen as sg

    ctx = rzk.Context(local)
    sc = sg.room_objects(2000, WIDTH, HEIGHT)
    t0 = time.perf_counter()
    agg = rzk.AggregateCuda(ctx, sc)
    build_s = time.perf_counter() - t0
    cam = rzk.Camera(sc.camera)
    recv_t = agg.primary(cam)
    n_recv = cam.n_pixels
    vt, n_made = rzk.VplGeneratorCuda(agg).spawn(VPL_SEED, VPL_PARTICLES, MAX_BOUNCE)
    assert n_made >= N_VPL, f"only {n_made} VPLs from {VPL_PARTICLES} particles"
    vpls_np = rzk.records_from_device(vt, sg.VPL_DTYPE)
    vpls_np, num_emitted = select_vpls(vpls_np)
    vpl_t = vt[: N_VPL * 96].contiguous()
    ev = rzk.VirtualPointLightCuda(agg, rzk.CLAMP_RADIANCE, 1.0)
    mean = ev.mean_contribution(recv_t, n_recv, vpl_t, N_VPL, seed=VPL_SEED, n_pairs=TAU_PAIRS)
    tau = float(np.float32(0.1 * mean))
    ev.clamp_threshold = tau
    scale = 1.0 / num_emitted
    out = torch.empty((n_recv, 3), dtype=torch.float32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    def step():
        ev.gather(recv_t, n_recv, vpl_t, N_VPL, scale=scale, out=out, image_width=WIDTH)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    ctx.check()
    ctx.rays(reset=True)   # the device's shadow-ray counter covers the timed steps only
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    times = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            flush.fill_(1)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step()
            b.record(stream)
            b.synchronize()
            times.append(a.elapsed_time(b) / 1e3)
        torch.cuda.synchronize()
    if pg:
        pg.barrier()
    total = max_over_ranks(pg, sum(times), "cuda")
    ctx.check()
    rays_timed = ctx.rays(reset=True)
    evals_step = n_recv * N_VPL
    value = job_rate(ws, evals_step, len(times), total)
    launches_step = kernels_per_call(step)

    # end to end through the public host-buffer call: receivers + VPLs from pinned host
    # memory in, the image out, every step
    recv_h = torch.empty(n_recv * 96, dtype=torch.uint8).pin_memory()
    recv_h.copy_(recv_t.cpu())
    vpl_h = torch.empty(N_VPL * 96, dtype=torch.uint8).pin_memory()
    vpl_h.copy_(vpl_t.cpu())
    img_h = torch.empty((n_recv, 3), dtype=torch.float32).pin_memory()
    import ctypes
    lib = rzk.load()
    sp = ctypes.c_void_p(stream.cuda_stream)

    def e2e_step():
        rzk.check(lib.rzk_gather_host(ctx.h, agg.h, ctypes.c_void_p(recv_h.data_ptr()), n_recv, WIDTH,
                                      ctypes.c_void_p(vpl_h.data_ptr()), N_VPL, rzk.CLAMP_RADIANCE,
                                      tau, scale, ctypes.c_void_p(img_h.data_ptr()), sp), "gather_host")

    e2e_step()
    e2e_steps = max(1, min(args.steps, 3))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        e2e_step()
    e2e_s = max_over_ranks(pg, (time.perf_counter() - t0) / e2e_steps, "cuda")
    img_ok = bool(torch.isfinite(img_h).all()) and float(img_h.sum()) > 0

    # the allocation-free entry point on the same workload (its 16 MiB static array holds a
    # chunk ring of ~1,000 tiles beside the ordered VPL copy; rzk_gather's ring has 8,192)
    out_na = torch.empty_like(out)

    def noalloc_step():
        rzk.check(lib.rzk_gather_noalloc(agg.h, ctypes.c_void_p(recv_t.data_ptr()), n_recv, WIDTH,
                                         ctypes.c_void_p(vpl_t.data_ptr()), N_VPL, rzk.CLAMP_RADIANCE, tau, scale,
                                         ctypes.c_void_p(out_na.data_ptr()), sp), "gather_noalloc")

    noalloc_step()
    na_times = []
    for _ in range(max(1, min(args.steps, 3))):
        flush.fill_(1)
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        noalloc_step()
        b.record(stream)
        b.synchronize()
        na_times.append(a.elapsed_time(b) / 1e3)
    ctx.check()
    na_s = sum(na_times) / len(na_times)
    noalloc = {"value": evals_step / na_s, "unit": "evals/s", "ms_per_step": 1e3 * na_s,
               "rel_l2_vs_default": float((out_na - out).norm() / out.norm()),
               "bit_equal_to_default": bool(torch.equal(out_na, out)),
               "note": "rzk_gather_noalloc on the same inputs; scratch in its fixed 16 MiB device array"}

    line = None
    if rank == 0:
        # Algorithmic bytes per evaluation from the oracle's traversal counters on a seeded
        # sample (same visit rule as the kernel: root record + one 64-byte child pair per
        # inner pop + one 48-byte triangle per leaf test, culled pairs trace nothing),
        # plus the operand stream of each CTA tile and the output.
        from oracle import Oracle
        o = Oracle(sc)
        recv_np = rzk.records_from_device(recv_t, sg.RECEIVER_DTYPE)
        rng = np.random.default_rng(VPL_SEED)
        pick = np.sort(rng.choice(n_recv, 512, replace=False))
        samp = recv_np[pick].copy()
        ref32, ref64, cnt = o.gather(samp, vpls_np, rzk.CLAMP_RADIANCE, tau, scale, cull=True, f64=True,
                                     threads=os.cpu_count() or 1)
        # the timed image against the oracle (float and double) on the same sampled pixels
        got = out.cpu().numpy()[pick]
        parity = {"rel_l2_vs_oracle_f32": float(np.linalg.norm(got - ref32) / np.linalg.norm(ref32)),
                  "rel_l2_vs_oracle_f64": float(np.linalg.norm(got - ref64) / np.linalg.norm(ref64)),
                  "bound": 1e-3, "sample": "512 seeded shading points x all VPLs of the timed step"}
        pairs = samp.shape[0] * N_VPL
        trav = (32 * cnt["root_tests"] + 64 * cnt["inner_pops"] + 48 * cnt["leaf_tests"]) / pairs
        operand = 96.0 / 128 + 12.0 / N_VPL     # VPL record per 128-thread CTA, output per pair
        bytes_per_eval = trav + operand
        ms = 1e3 * total / len(times)
        achieved = bytes_per_eval * evals_step / (total / len(times)) / 1e9
        dram_gbs = TRAFFIC_BYTES_PER_LAUNCH / (total / len(times)) / 1e9 if N_VPL == 32768 else None
        peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
        if os.path.exists(peaks_path):
            peak = float(json.load(open(peaks_path))["hbm_gbs"])
            peak_src = "measured"
        else:
            peak, peak_src = 6650.0, "fallback"
        # issue roofline: SMs x 4 schedulers x one warp instruction per cycle at the SM clock
        # sampled under load (the clock's maximum where no sample was taken)
        clk_sum = clk.summary()
        props = torch.cuda.get_device_properties(local)
        sm_mhz = clk_sum["sm_mhz"] or clk_sum["sm_max_mhz"] or 1965.0
        issue_peak = props.multi_processor_count * 4 * sm_mhz * 1e6
        inst = INST_PER_LAUNCH if N_VPL == 32768 else None
        issue_achieved = inst / (total / len(times)) if inst else None
        rays_per_eval_oracle = cnt["rays"] / pairs
        # CPU baseline: the reference's own gather on this box's host cores, bounded sample
        threads = os.cpu_count() or 1
        if args.skip_cpu:   # profiling runs: the GPU part only
            kind, cpu_v, sample = "skipped", None, np.zeros(0, sg.RECEIVER_DTYPE)
        else:
            kind, sample, run = cpu_rate(sc, o, recv_np, vpls_np, tau, scale, 10.0, threads)
            tc = time.perf_counter()
            run(sample)
            cpu_v = sample.shape[0] * N_VPL / (time.perf_counter() - tc)
        clocks = clk.summary()
        line = {
            "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": ws, "steps": len(times),
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic", "config": workload_config(),
            "rays_per_s": ws * rays_timed / total,
            "rays_note": ("shadow rays counted on the device by the gather kernels over the timed steps "
                          "(rzk_context_rays), over the timed region"),
            "shadow_rays_per_step": rays_timed / len(times),
            "shadow_rays_per_eval": rays_timed / len(times) / evals_step,
            "shadow_rays_per_eval_oracle_sample": rays_per_eval_oracle,
            "e2e": {"value": ws * evals_step / e2e_s, "unit": "evals/s",
                    "h2d_bytes_per_step": n_recv * 96 + N_VPL * 96,
                    "d2h_bytes_per_step": n_recv * 12, "image_finite": img_ok},
            "roofline": {
                "bound": "issue", "unit": "Gwarp-inst/s",
                "achieved": None if issue_achieved is None else issue_achieved / 1e9,
                "peak": issue_peak / 1e9,
                "frac": None if issue_achieved is None else issue_achieved / issue_peak,
                "traffic": TRAFFIC_BYTES_PER_LAUNCH if N_VPL == 32768 else None,
                "traffic_note": "ncu dram__bytes_read.sum + dram__bytes_write.sum, one full launch",
                "inst_per_launch": inst,
                "peak_source": (f"{props.multi_processor_count} SMs x 4 schedulers x 1 warp instruction per cycle "
                                f"at the {sm_mhz:.0f} MHz SM clock sampled during the timed steps"),
                "note": ("achieved = the gather launch's warp instructions (ncu smsp__inst_executed.sum, one full "
                         "launch, recorded in profiles/) over the live CUDA-event time of a whole step (the gather "
                         "is 99.7% of it); the kernel is issue-bound: HBM is idle and L1/L2 serve its ~34 MB "
                         "working set"),
                "hbm_reference_traversal": {
                    "bytes_per_eval": bytes_per_eval, "achieved_gbs": achieved, "peak_gbs": peak,
                    "frac": achieved / peak, "peak_source": peak_src + " (MEASURED_PEAKS.json hbm_gbs)",
                    "dram_gbs": dram_gbs, "dram_frac": None if dram_gbs is None else dram_gbs / peak,
                    "note": ("the reference traversal's node and triangle bytes per evaluation (reference tree, "
                             "reference visit order) over the step time: a diagnostic, not a bound - the kernel "
                             "visits fewer nodes (SAH any-hit tree, occluder caches, Hilbert-ordered VPL chunks) "
                             "and L1/L2 serve them, so it exceeds the HBM copy peak; dram_gbs is what the launch "
                             "drew from HBM")},
            },
            "noalloc": noalloc,
            "cpu_baseline": {"value": cpu_v, "unit": "evals/s", "cores": threads, "kind": kind,
                             "sample": f"{sample.shape[0]} seeded uniformly sampled shading points x {N_VPL} VPLs"},
            "clocks": clocks,
            "parity": parity,
            "gpu_launches": launches_step * len(times),
            "gpu_launches_note": f"{launches_step} kernels per step, counted as the kernel nodes of one captured step",
            "tau": tau, "num_emitted": num_emitted, "bvh_build_s": build_s,
            "scene": {"triangles": agg.n_tris, "nodes": agg.n_nodes, "levels": agg.n_levels,
                      "device_bytes": agg.device_bytes},
        }
    if line is not None and ws == 1 and args.serve_duration > 0 and not args.skip_cpu:
        # the metric's second half: serving latency and throughput, batched server beside the
        # one-request-at-a-time server, on the serving mix (its own device-resident worlds)
        del flush
        torch.cuda.empty_cache()
        t0 = time.perf_counter()
        worlds = serve_setup(ctx)
        setup_s = time.perf_counter() - t0
        rates = [float(x) for x in SERVE_RATES.split(",")]
        sweep = serve_sweep(worlds, rates, args.serve_duration, args.budget_gb)
        keys = ("completed", "rejected", "throughput_rps", "evals_per_s", "paths_per_s", "p50_ms", "p95_ms",
                "p99_ms", "mean_queue_ms", "mean_run_ms")
        line["serving"] = {
            "workload": "serving_mix_8_scenes_50k_1M_tris", "duration_s_per_rate": args.serve_duration,
            "hbm_budget_gb": args.budget_gb, "setup_s": setup_s,
            "scene_triangles": [w["agg"].n_tris for w in worlds],
            "rates": [{"rate_rps": x["rate_rps"], "requests": x["requests"],
                       "batched": {k: x["batched"][k] for k in keys}, "plain": {k: x["plain"][k] for k in keys},
                       "evals_per_s_ratio": x["evals_per_s_ratio"], "p99_ratio": x["p99_ratio"]} for x in sweep],
            "note": ("Poisson arrivals at each rate; latency = the server's submit-to-completion time; the "
                     "one-request-at-a-time server is the plain per-request path on the same resident scenes"),
        }
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    if line is not None:
        print(json.dumps(line))
    return 0


def run_batch(args):
    """Batched gather: 64 seeded instances of uneven size (10k-500k triangles, 128^2-1024^2
    images, 1k-64k VPLs, all log-uniform), gathered (a) as 64 plain rzk_gather calls and
    (b) as one autotuned rzk_batch_run captured in a CUDA graph and replayed.  Inputs
    resident in HBM, L2 flushed before every timed step.  Prints one JSON line."""
    import torch
    from renzoku_b200 import build as rbuild
    rbuild.build()
    from renzoku_b200 import instances as im, rzk
    ctx = rzk.Context(0)
    if args.small:   # many small instances, where per-launch ramp and tail matter most
        specs = im.batch_specs(args.instances, seed=2024, tris=(10_000, 50_000), side=(64, 256), vpls=(1_000, 4_000))
    else:
        specs = im.batch_specs(args.instances, seed=2024)
    t0 = time.perf_counter()
    insts = [im.make_instance(ctx, s) for s in specs]
    setup_s = time.perf_counter() - t0
    ctx.check()
    evals = sum(i.n_recv * i.n_vpl for i in insts)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    def timed(fn, steps, warmup):
        for _ in range(warmup):
            fn()
        torch.cuda.synchronize()
        ts = []
        for _ in range(steps):
            flush.fill_(1)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            fn()
            b.record(stream)
            b.synchronize()
            ts.append(a.elapsed_time(b) / 1e3)
        return ts

    def plain():
        for i in insts:
            i.gather()

    jobs = rzk.make_jobs(i.job() for i in insts)
    t0 = time.perf_counter()
    variant, chunk_len, probe_ms, probes = rzk.autotune_batch(ctx, jobs, max_probe_jobs=8, table=True)
    tune_s = time.perf_counter() - t0
    batch = rzk.GatherBatch(ctx, jobs, variant=variant, chunk_len=chunk_len)
    batch.run()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph(keep_graph=True)
    side = torch.cuda.Stream()
    with torch.cuda.stream(side):
        with torch.cuda.graph(g, stream=side):
            batch.run(stream=side)
    torch.cuda.synchronize()
    graph_launches = graph_kernels(g)
    with ClockSampler(0) as clk:
        t_plain = timed(plain, args.steps, args.warmup)
        t_graph = timed(g.replay, args.steps, args.warmup)
    ctx.check()
    # the batched images against the plain ones with the same chunking (bit-exact when the
    # autotuned chunk length equals the plain default; otherwise a relative check)
    ref = [i.gather(out=torch.empty_like(i.out)) for i in insts]
    g.replay()
    torch.cuda.synchronize()
    rel = max(float((i.out - r).norm() / max(float(r.norm()), 1e-30)) for i, r in zip(insts, ref))
    del g
    batch.close()
    mp = sum(t_plain) / len(t_plain)
    mg = sum(t_graph) / len(t_graph)
    line = {
        "metric": "batched VPL-gather evals/s (64 uneven instances, one graph-captured persistent launch)",
        "value": evals / mg, "unit": "evals/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * mg, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"batched_gather_{len(insts)}_{'small_' if args.small else ''}instances_seed2024",
                   "instances": len(insts), "evals_per_step": evals,
                   "triangles": [i.agg.n_tris for i in insts],
                   "image_sides": [i.spec.width for i in insts], "vpls": [i.n_vpl for i in insts],
                   "l2": "flushed between timed steps (256 MiB write)"},
        "plain_launches": {"value": evals / mp, "ms_per_step": 1e3 * mp, "launches_per_step": 3 * len(insts)},
        "speedup_vs_plain": mp / mg,
        "autotune": {"variant": variant, "shape": rzk.batch_variant_info(variant), "chunk_len": chunk_len,
                     "probe_ms": probe_ms, "tune_s": tune_s,
                     "search": [{"variant": v, "shape": rzk.batch_variant_info(v),
                                 "ms_by_chunk_len": dict(zip(["default", "512", "1024", "2048"],
                                                             [float(x) for x in probes[v]]))}
                                for v in range(probes.shape[0])]},
        "max_rel_diff_vs_plain": rel, "gpu_launches": graph_launches * args.steps,
        "gpu_launches_note": f"{graph_launches} kernel nodes in the replayed graph per step",
        "clocks": clk.summary(),
        "setup_s": setup_s,
    }
    print(json.dumps(line))
    return 0


def run_restart(args):
    """Warm restart of device scenes: the time to build a scene from its description
    (upload, LBVH, SAH any-hit tree, lights) against the time to restore it from a blob
    of its device arrays (rzk_scene_deserialize), for the scaled scene (~300k triangles)
    and the sphere scene (~960k triangles); each restored scene is checked against the
    built one (BVH bytes).  Prints one JSON line."""
    import torch
    from renzoku_b200 import build as rbuild
    rbuild.build()
    from renzoku_b200 import rzk, scenegen as sg
    ctx = rzk.Context(0)
    rows = []
    for name, sc in (("room_objects_300k", sg.room_objects(2000, WIDTH, HEIGHT)),
                     ("room_spheres_960k", sg.room_spheres(20000, 1024, 1024))):
        rzk.AggregateCuda(ctx, sc).close()   # first-use costs (module load, pools) outside the timing
        build, save, restore = [], [], []
        for _ in range(max(1, args.steps)):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            agg = rzk.AggregateCuda(ctx, sc)
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            blob = agg.serialize()
            t2 = time.perf_counter()
            back = rzk.AggregateCuda.restore(ctx, blob, sc)
            torch.cuda.synchronize()
            t3 = time.perf_counter()
            build.append(t1 - t0)
            save.append(t2 - t1)
            restore.append(t3 - t2)
            same = all(x.tobytes() == y.tobytes() for x, y in zip(agg.bvh_dump(), back.bvh_dump()))
            agg.close()
            back.close()
        rows.append({"scene": name, "triangles": back.n_tris, "blob_bytes": len(blob),
                     "build_ms": 1e3 * min(build), "serialize_ms": 1e3 * min(save),
                     "restore_ms": 1e3 * min(restore), "restore_speedup": min(build) / min(restore),
                     "bvh_identical": same})
    ctx.check()
    line = {
        "metric": "scene restore time (ms, 960k-triangle scene, from a host blob)",
        "value": rows[-1]["restore_ms"], "unit": "ms", "n_gpus": 1, "steps": max(1, args.steps), "warmup": 1,
        "ms_per_step": rows[-1]["restore_ms"], "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "scene_warm_restart_300k_960k_tris", "timing": "host wall clock, min over steps"},
        "scenes": rows,
    }
    print(json.dumps(line))
    return 0


def run_mrcs(args):
    """Matrix row-column sampling on the scaled scene: 512 x 512 shading points, the first
    32,768 VPLs resampled by power to 10,000 columns, 256 stratified rows (32 x 32 strata),
    327 clusters (1% of the VPLs).  Reports the set-up stages and the gather over the
    clusters' representatives (every pixel x every representative, one shadow ray each),
    timed on the device with the L2 flushed between steps.  Prints one JSON line."""
    import torch
    from renzoku_b200 import build as rbuild
    rbuild.build()
    from renzoku_b200 import rzk, scenegen as sg
    ctx = rzk.Context(0)
    sc = sg.room_objects(2000, WIDTH, HEIGHT)
    agg = rzk.AggregateCuda(ctx, sc)
    cam = rzk.Camera(sc.camera)
    recv = agg.primary(cam)
    vt, n_made = rzk.VplGeneratorCuda(agg).spawn(VPL_SEED, VPL_PARTICLES, MAX_BOUNCE)
    vt = vt[: N_VPL * 96].contiguous()
    vpls_np = rzk.records_from_device(vt, sg.VPL_DTYPE)
    _, num_emitted = select_vpls(vpls_np)
    ev = rzk.VirtualPointLightCuda(agg, rzk.CLAMP_RADIANCE, 1.0)
    tau = float(np.float32(0.1 * ev.mean_contribution(recv, cam.n_pixels, vt, N_VPL, seed=VPL_SEED,
                                                       n_pairs=TAU_PAIRS)))
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    m = rzk.MrcsCuda(agg, cam, vt, N_VPL, rzk.CLAMP_RADIANCE, tau, rzk.mrcs_params(seed=VPL_SEED))
    setup_s = time.perf_counter() - t0
    info = m.info()
    _, _, reps, _ = m.clusters()
    n_reps = int((reps >= 0).sum())
    out = torch.empty((cam.n_pixels, 3), dtype=torch.float32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    def step():
        m.gather(recv, cam.n_pixels, scale=1.0 / num_emitted, out=out, image_width=WIDTH)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    times = []
    with ClockSampler(0) as clk:
        for _ in range(args.steps):
            flush.fill_(1)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step()
            b.record(stream)
            b.synchronize()
            times.append(a.elapsed_time(b) / 1e3)
    ctx.check()
    launches_step = kernels_per_call(step)
    ms = 1e3 * sum(times) / len(times)
    evals = cam.n_pixels * n_reps
    clk_sum = clk.summary()
    roofline = issue_roofline(MRCS_VIS_INST, ms / 1e3, clk_sum["sm_mhz"], "mrcs_vis_kernel",
                              "the tracing pass's warp instructions over the whole clustered-gather step")
    # CPU baseline: the reference's own MatrixRowColumnSampling (initialize, then
    # gather_clusters per pixel) run twice on seeded pixel samples of two sizes; the
    # difference isolates gather_clusters' cost per pixel x representative (the reference
    # is single-threaded: one global random stream).  The reference gets the first 10,000
    # VPLs: with more it resamples 10,000 columns but then clusters all of them, reading
    # past the end of its matrix (cluster_builder.cc:189-199), which has no defined result.
    cpu = {"value": None, "unit": "evals/s", "cores": 1, "kind": "skipped", "sample": ""}
    if not args.skip_cpu:
        from oracle import RefHarness
        if RefHarness.available():
            ref = RefHarness(sc)
            recv_np = rzk.records_from_device(recv, sg.RECEIVER_DTYPE)
            order = np.random.default_rng(VPL_SEED + 4).permutation(cam.n_pixels)
            small = recv_np[np.sort(order[:64])].copy()
            t0 = time.perf_counter()
            ref_vpls = vpls_np[:10_000].copy()
            _, _, r_small, _ = ref.mrcs(ref_vpls, rzk.CLAMP_RADIANCE, tau, VPL_SEED, small)
            t_small = time.perf_counter() - t0
            k = int(min(cam.n_pixels, 32768))
            big = recv_np[np.sort(order[:k])].copy()
            t0 = time.perf_counter()
            _, _, r_big, _ = ref.mrcs(ref_vpls, rzk.CLAMP_RADIANCE, tau, VPL_SEED, big)
            t_big = time.perf_counter() - t0
            reps_ref = int((r_big >= 0).sum())
            if t_big > t_small:
                cpu = {"value": (k - 64) * reps_ref / (t_big - t_small), "unit": "evals/s", "cores": 1,
                       "kind": "reference",
                       "sample": f"gather_clusters of {k} vs 64 seeded pixels x {reps_ref} representatives of "
                                 f"the first 10,000 VPLs (initialize included in both runs and cancelled)"}
    line = {
        "metric": "MRCS clustered-gather evals/s (pixel x cluster representative, shadow ray each)",
        "value": evals / (ms / 1e3), "unit": "evals/s", "n_gpus": 1, "steps": len(times),
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "mrcs_room_objects_300k_tris_512x512_32768_vpls",
                   "rows": info["rows"], "columns": info["columns"], "num_clusters": info["num_clusters"],
                   "representatives": n_reps, "evals_per_step": evals, "block_size": 32,
                   "l2": "flushed between timed steps (256 MiB write)"},
        "setup_s": setup_s,
        "setup_stage_ms": dict(zip(["pixels_and_columns", "reduced_matrix", "clustering", "representatives"],
                                   info["stage_ms"])),
        "clocks": clk_sum, "roofline": roofline, "cpu_baseline": cpu,
        "gpu_launches": launches_step * len(times),
        "gpu_launches_note": f"{launches_step} kernels per step, counted as the kernel nodes of one captured step",
        "image_finite": bool(torch.isfinite(out).all()), "tau": tau,
    }
    print(json.dumps(line))
    return 0


def run_lightslice(args):
    """LightSlice on the scaled scene: 512 x 512 shading points, the first 32,768 VPLs (those
    of bounce <= 1 are clustered), slices of at most 1,024 points (~256), 1,000 global
    clusters refined to at most 2,000 per slice over 32 neighbouring slices.  Reports the
    build stages (device reduced matrix + clustering, host refinement) and the clustered
    gather (every pixel x its slice's clusters, one shadow ray each) timed on the device with
    the L2 flushed between steps.  Prints one JSON line."""
    import torch
    from renzoku_b200 import build as rbuild
    rbuild.build()
    from renzoku_b200 import rzk, scenegen as sg
    ctx = rzk.Context(0)
    sc = sg.room_objects(2000, WIDTH, HEIGHT)
    agg = rzk.AggregateCuda(ctx, sc)
    cam = rzk.Camera(sc.camera)
    recv = agg.primary(cam)
    vt, n_made = rzk.VplGeneratorCuda(agg).spawn(VPL_SEED, VPL_PARTICLES, MAX_BOUNCE)
    vt = vt[: N_VPL * 96].contiguous()
    vpls_np = rzk.records_from_device(vt, sg.VPL_DTYPE)
    _, num_emitted = select_vpls(vpls_np)
    ev = rzk.VirtualPointLightCuda(agg, rzk.CLAMP_RADIANCE, 1.0)
    tau = float(np.float32(0.1 * ev.mean_contribution(recv, cam.n_pixels, vt, N_VPL, seed=VPL_SEED,
                                                       n_pairs=TAU_PAIRS)))
    params = rzk.lightslice_params(num_clusters=1000, max_slice_size=1024, num_neighbor_slices=32,
                                   max_slice_clusters=2000, seed=VPL_SEED)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ls = rzk.LightSliceCuda.create(agg, recv, WIDTH, HEIGHT, vt, N_VPL, params)
    build_s = time.perf_counter() - t0
    info = ls.info()
    counts = ls.clusters()["count"]
    slice_of = ls.find_slice(recv, cam.n_pixels).cpu().numpy()
    evals = int(counts[slice_of[slice_of >= 0]].sum())
    out = torch.empty((cam.n_pixels, 3), dtype=torch.float32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()

    def step():
        ls.gather(recv, cam.n_pixels, rzk.CLAMP_RADIANCE, tau, scale=1.0 / num_emitted, out=out)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    times = []
    with ClockSampler(0) as clk:
        for _ in range(args.steps):
            flush.fill_(1)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step()
            b.record(stream)
            b.synchronize()
            times.append(a.elapsed_time(b) / 1e3)
    ctx.check()
    launches_step = kernels_per_call(step, capture=False)
    ms = 1e3 * sum(times) / len(times)
    stages = dict(zip(["points_and_filter", "slicing", "reduced_matrix", "global_clustering",
                       "refinement", "maps", "tables"], info["ms"][:7]))
    clk_sum = clk.summary()
    roofline = issue_roofline(LS_VIS_INST, ms / 1e3, clk_sum["sm_mhz"], "cluster_vis_kernel",
                              "the tracing pass's warp instructions over the whole clustered-gather step")
    # CPU baseline: the reference's own LightSlice::gather_clusters on all host cores, on a
    # seeded sample of pixels, from the reference's refinement of the device's reduced matrix
    # and global clusters (the stages pinned bit-exact by the parity tests)
    cpu = {"value": None, "unit": "evals/s", "cores": os.cpu_count() or 1, "kind": "skipped", "sample": ""}
    parity = None
    if not args.skip_cpu:
        from oracle import RefHarness, column_magnitudes
        if RefHarness.available():
            ref = RefHarness(sc)
            rls = ref.lightslice(1024, 32, VPL_SEED)
            rls.set_vpls(vpls_np)
            R, V, _ = ls.matrix()
            R, V = R.cpu().numpy(), V.cpu().numpy()
            g_rep, g_w, assign = ls.global_clusters()
            rls.refine(R, V, g_rep, g_w, assign, column_magnitudes(R), 2000, VPL_SEED)
            recv_np = rzk.records_from_device(recv, sg.RECEIVER_DTYPE)
            order = np.random.default_rng(VPL_SEED + 2).permutation(cam.n_pixels)
            threads = os.cpu_count() or 1
            cal = order[:256]
            t0 = time.perf_counter()
            rls.gather(recv_np[np.sort(cal)].copy(), rzk.CLAMP_RADIANCE, tau, threads=threads)
            per = max(time.perf_counter() - t0, 1e-3) / len(cal)
            pick = np.sort(order[:int(min(cam.n_pixels, max(threads, 10.0 / per)))])
            t0 = time.perf_counter()
            exp = rls.gather(recv_np[pick].copy(), rzk.CLAMP_RADIANCE, tau, threads=threads)
            dt = time.perf_counter() - t0
            s_evals = int(counts[slice_of[pick][slice_of[pick] >= 0]].sum())
            cpu = {"value": s_evals / dt, "unit": "evals/s", "cores": threads, "kind": "reference",
                   "sample": f"{len(pick)} seeded pixels x their slices' clusters ({s_evals} evaluations)"}
            got = out.cpu().numpy()[pick] * np.float32(num_emitted)
            parity = {"rel_l2_vs_reference": float(np.linalg.norm(got - exp) / max(np.linalg.norm(exp), 1e-30)),
                      "sample": f"{len(pick)} pixels of the timed image against the reference's gather_clusters"}
    line = {
        "metric": "LightSlice clustered-gather evals/s (pixel x slice-cluster representative, shadow ray each)",
        "value": evals / (ms / 1e3), "unit": "evals/s", "n_gpus": 1, "steps": len(times),
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": "lightslice_room_objects_300k_tris_512x512_32768_vpls",
                   "slices": info["slices"], "points": info["points"], "vpls_used": info["vpls_used"],
                   "global_clusters": info["global_clusters"], "slice_clusters": info["slice_clusters"],
                   "evals_per_step": evals, "max_slice_size": 1024, "num_clusters": 1000,
                   "max_slice_clusters": 2000, "neighbor_slices": 32,
                   "l2": "flushed between timed steps (256 MiB write)"},
        "build_s": build_s, "build_stage_ms": stages, "clocks": clk_sum, "roofline": roofline,
        "cpu_baseline": cpu, "parity": parity,
        "gpu_launches": None if launches_step is None else launches_step * len(times),
        "gpu_launches_note": (f"{launches_step} kernels per step, counted by the CUDA activity profiler over one step"
                              if launches_step else "not counted: the CUDA activity profiler recorded nothing"),
        "image_finite": bool(torch.isfinite(out).all()), "tau": tau,
    }
    print(json.dumps(line))
    return 0


def run_guided(args):
    """Clustered-VPL guided path tracing: room + light + 20,000 seeded UV spheres (~960k
    triangles), 1024 x 1024 pixel-centre paths, 16 samples per pixel, max bounce 8 with
    Russian roulette (p = 0.5) beyond depth 3; guiding from a LightSlice built on 100,000
    VPLs with 4,096 global clusters and 32 x 32 Jensen maps per slice.  One step = one full
    frame (all spp).  Prints one JSON line."""
    import torch
    from renzoku_b200 import build as rbuild
    rbuild.build()
    from renzoku_b200 import rzk, scenegen as sg
    ctx = rzk.Context(0)
    side = args.side
    sc = sg.room_spheres(20000, side, side)
    t0 = time.perf_counter()
    agg = rzk.AggregateCuda(ctx, sc)
    cam = rzk.Camera(sc.camera)
    recv = agg.primary(cam)
    n_vpl = 100_000
    particles = 80_000
    while True:
        vt, made = rzk.VplGeneratorCuda(agg).spawn(VPL_SEED, particles, MAX_BOUNCE)
        if made >= n_vpl:
            break
        particles *= 2
    vt = vt[: n_vpl * 96].contiguous()
    params = rzk.lightslice_params(num_clusters=4096, max_slice_size=args.slice_size, num_neighbor_slices=32,
                                   max_slice_clusters=args.max_slice_clusters, seed=VPL_SEED)
    ls = rzk.LightSliceCuda.create(agg, recv, side, side, vt, n_vpl, params)
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    info = ls.info()
    out = torch.empty((cam.n_pixels, 3), dtype=torch.float32, device="cuda")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.current_stream()
    spp = args.spp

    def step():
        ls.guided_render(cam, spp, 8, rr_depth=3, rr_prob=0.5, seed=VPL_SEED, out=out, sampler=args.sampler)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    times = []
    with ClockSampler(0) as clk:
        for _ in range(args.steps):
            flush.fill_(1)
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step()
            b.record(stream)
            b.synchronize()
            times.append(a.elapsed_time(b) / 1e3)
    ctx.check()
    launches_step = kernels_per_call(step)
    ms = 1e3 * sum(times) / len(times)
    paths = cam.n_pixels * spp
    clk_sum = clk.summary()
    roofline = issue_roofline(GUIDED_INST if (side, spp, args.sampler) == (1024, 16, "jensen") else None,
                              ms / 1e3, clk_sum["sm_mhz"], "guided_kernel",
                              "the path kernel's warp instructions over the whole frame (chains and per-pixel mean "
                              "included in the time)")
    # CPU baseline: the reference's own tracer (trace_wellington with the same LightSlice
    # state, rebuilt by the reference's refinement from the device's reduced matrix and
    # global clusters) on a seeded sample of pixels; one host thread, because the reference
    # draws every path from its one global random stream
    cpu = {"value": None, "unit": "paths/s", "cores": 1, "kind": "skipped", "sample": ""}
    parity = None
    if not args.skip_cpu:
        from oracle import RefHarness, column_magnitudes
        if RefHarness.available():
            ref = RefHarness(sc)
            rls = ref.lightslice(args.slice_size, 32, VPL_SEED)
            rls.set_vpls(rzk.records_from_device(vt, sg.VPL_DTYPE))
            R, V, _ = ls.matrix()
            R, V = R.cpu().numpy(), V.cpu().numpy()
            g_rep, g_w, assign = ls.global_clusters()
            rls.refine(R, V, g_rep, g_w, assign, column_magnitudes(R), args.max_slice_clusters, VPL_SEED)
            order = np.random.default_rng(VPL_SEED + 3).permutation(cam.n_pixels)
            t0 = time.perf_counter()
            rls.guided(np.sort(order[:16]).astype(np.int32), spp, 8, rr_depth=3, rr_prob=0.5, seed=VPL_SEED,
                       sampler=args.sampler)
            per = max(time.perf_counter() - t0, 1e-3) / 16
            pick = np.sort(order[:int(min(cam.n_pixels, max(16, 10.0 / per)))]).astype(np.int32)
            t0 = time.perf_counter()
            want = rls.guided(pick, spp, 8, rr_depth=3, rr_prob=0.5, seed=VPL_SEED, sampler=args.sampler)
            dt = time.perf_counter() - t0
            cpu = {"value": len(pick) * spp / dt, "unit": "paths/s", "cores": 1, "kind": "reference",
                   "sample": f"{len(pick)} seeded pixels x {spp} spp"}
            if args.sampler == "jensen":
                got = out.cpu().numpy()[pick]
                m = want.mean(axis=1)
                parity = {"rel_l2_vs_reference": float(np.linalg.norm(got - m) / max(np.linalg.norm(m), 1e-30)),
                          "sample": f"{len(pick)} pixels of the timed frame against the reference tracer"}
    line = {
        "metric": ("guided path-tracing paths/s (LightSlice " +
                   ("Jensen-map" if args.sampler == "jensen" else "Metropolis-chain") +
                   " guiding, MIS with BRDF sampling)"),
        "value": paths / (ms / 1e3), "unit": "paths/s", "n_gpus": 1, "steps": len(times),
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"guided_pt_room_spheres_{agg.n_tris}_tris_{side}x{side}_{spp}spp_depth8_rr3"
                               + ("" if args.sampler == "jensen" else "_metropolis"),
                   "sampler": args.sampler, "triangles": agg.n_tris, "spp": spp, "max_bounce": 8, "rr_depth": 3, "rr_prob": 0.5,
                   "vpls": n_vpl, "vpls_used": info["vpls_used"], "global_clusters": info["global_clusters"],
                   "slices": info["slices"], "slice_clusters": info["slice_clusters"], "map_resolution": 32,
                   "max_slice_size": args.slice_size,
                   "l2": "flushed between timed steps (256 MiB write)"},
        "setup_s": setup_s, "lightslice_stage_ms": info["ms"][:7], "clocks": clk_sum, "roofline": roofline,
        "cpu_baseline": cpu, "parity": parity,
        "gpu_launches": launches_step * len(times),
        "gpu_launches_note": f"{launches_step} kernels per step, counted as the kernel nodes of one captured step",
        "image_finite": bool(torch.isfinite(out).all()), "image_mean": float(out.mean()),
    }
    print(json.dumps(line))
    return 0


SERVE_RATES = "5,10,20,50,100,200"


def serve_setup(ctx):
    """The serving mix's device-resident worlds: 8 rooms filled to 50k-1M triangles
    (log-uniform, seed 7), each with 100,000 VPLs, its clamp threshold and a LightSlice."""
    import math
    import torch
    from renzoku_b200 import instances as im, rzk, scenegen as sg
    rng = np.random.default_rng(7)
    worlds = []
    for k in range(8):
        n_tris = int(round(math.exp(rng.uniform(math.log(50_000), math.log(1_000_000)))))
        sc = sg.room_filled(n_tris, 256, 256, 700 + k)
        agg = rzk.AggregateCuda(ctx, sc)
        cam = rzk.Camera(sc.camera)
        recv = agg.primary(cam)
        vt, emitted = im.spawn_vpls(agg, VPL_SEED + k, 100_000)
        ev = rzk.VirtualPointLightCuda(agg, rzk.CLAMP_RADIANCE, 1.0)
        tau = float(np.float32(0.1 * ev.mean_contribution(recv, cam.n_pixels, vt, 100_000, seed=VPL_SEED,
                                                           n_pairs=TAU_PAIRS)))
        ls = rzk.LightSliceCuda.create(agg, recv, 256, 256, vt, 100_000,
                                       rzk.lightslice_params(num_clusters=1000, max_slice_size=1024,
                                                             num_neighbor_slices=32, max_slice_clusters=1000,
                                                             seed=VPL_SEED))
        worlds.append({"sc": sc, "agg": agg, "vpls": vt, "emitted": emitted, "tau": tau, "ls": ls})
    torch.cuda.synchronize()
    ctx.check()
    return worlds


def serve_sweep(worlds, rates, duration, budget_gb):
    """Poisson arrivals (seed 8 + rate) at each rate for `duration` seconds; every request a
    gather or a guided render (50/50) with image side 64-1024, 1k-100k VPLs and 1-16 spp,
    log-uniform, against one of the worlds.  The same request stream runs through the
    batched server and through the one-request-at-a-time server.  Latency is the server's
    submit-to-completion time; throughput counts completed work over the wall time of
    arrivals plus drain."""
    import dataclasses
    import math
    import torch
    from renzoku_b200 import rzk
    logu = lambda g, lo, hi: math.exp(g.uniform(math.log(lo), math.log(hi)))

    def requests(rate):
        g = np.random.default_rng(8 + int(rate * 1000))
        t, out = 0.0, []
        while True:
            t += g.exponential(1.0 / rate)
            if t > duration:
                return out
            side = max(64, int(round(logu(g, 64, 1024) / 8.0)) * 8)
            out.append({"t": t, "guided": bool(g.random() < 0.5), "scene": int(g.integers(8)), "side": side,
                        "vpls": int(round(logu(g, 1000, 100_000))), "spp": int(round(logu(g, 1, 16)))})

    def make_req(d, out):
        w = worlds[d["scene"]]
        cam = rzk.Camera(dataclasses.replace(w["sc"].camera, width=d["side"], height=d["side"]))
        r = rzk.RequestC()
        r.kind = rzk.REQ_GUIDED if d["guided"] else rzk.REQ_GATHER
        r.scene = w["agg"].h.value
        r.lightslice = w["ls"].h.value
        r.camera = rzk.camera_c(cam)
        r.d_vpls = w["vpls"].data_ptr()
        r.n_vpl = d["vpls"]
        r.clamp_mode = rzk.CLAMP_RADIANCE
        r.tau = w["tau"]
        r.scale = 1.0 / w["emitted"]
        r.spp, r.max_bounce, r.rr_depth, r.rr_prob, r.seed = d["spp"], 8, 3, 0.5, VPL_SEED
        r.d_rgb = out.data_ptr()
        return r

    def pct(x, q):
        return float(np.percentile(x, q)) if len(x) else None

    def run(batching, reqs):
        srv = rzk.Server(0, batching=batching, hbm_budget_bytes=int(budget_gb * (1 << 30)))
        pending, done, rejected = {}, [], 0
        t_start = time.perf_counter()
        for d in reqs:
            while True:
                now = time.perf_counter() - t_start
                if now >= d["t"]:
                    break
                time.sleep(min(0.002, d["t"] - now))
            out = torch.empty((d["side"] * d["side"], 3), dtype=torch.float32, device="cuda")
            t = srv.submit(make_req(d, out))
            if t is None:
                rejected += 1
            else:
                pending[t] = (out, d)
            for tk in list(pending):
                st, l, _ = srv.poll(tk)
                if st >= 2:
                    done.append((l, pending[tk][1]))
                    del pending[tk]
        for tk in list(pending):
            _, l = srv.wait(tk)
            done.append((l, pending[tk][1]))
        wall = time.perf_counter() - t_start
        stats = srv.stats()
        kind, q_ms, r_ms = srv.timings()
        srv.close()
        lat = np.array([l for l, _ in done])
        lat_g = np.array([l for l, d in done if not d["guided"]])
        lat_p = np.array([l for l, d in done if d["guided"]])
        evals = sum(d["side"] * d["side"] * d["vpls"] for _, d in done if not d["guided"])
        paths = sum(d["side"] * d["side"] * d["spp"] for _, d in done if d["guided"])
        return {"completed": len(done), "rejected": rejected, "wall_s": wall,
                "throughput_rps": len(done) / wall, "evals_per_s": evals / wall, "paths_per_s": paths / wall,
                "p50_ms": pct(lat, 50), "p95_ms": pct(lat, 95), "p99_ms": pct(lat, 99),
                "gather_p99_ms": pct(lat_g, 99), "guided_p99_ms": pct(lat_p, 99),
                "mean_queue_ms": float(q_ms.mean()) if len(q_ms) else None,
                "mean_run_ms": float(r_ms.mean()) if len(r_ms) else None,
                "launches": stats["launches"]}

    sweep = []
    for rate in rates:
        reqs = requests(rate)
        b = run(True, reqs)
        p = run(False, reqs)
        sweep.append({"rate_rps": rate, "requests": len(reqs), "batched": b, "plain": p,
                      "evals_per_s_ratio": b["evals_per_s"] / p["evals_per_s"] if p["evals_per_s"] else None,
                      "p99_ratio": b["p99_ms"] / p["p99_ms"] if b["p99_ms"] and p["p99_ms"] else None})
    return sweep


def run_serve(args):
    """Serving mix (see serve_sweep) at the --rates for --duration seconds each, batched
    server beside the one-request-at-a-time server.  Prints one JSON line (value = p99
    latency of the batched server at the lowest rate)."""
    import torch
    from renzoku_b200 import build as rbuild
    rbuild.build()
    from renzoku_b200 import rzk
    ctx = rzk.Context(0)
    t0 = time.perf_counter()
    worlds = serve_setup(ctx)
    setup_s = time.perf_counter() - t0
    rates = [float(x) for x in args.rates.split(",")]
    sweep = serve_sweep(worlds, rates, args.duration, args.budget_gb)
    first = sweep[0]["batched"]
    line = {
        "metric": f"serving p99 latency (ms) at {rates[0]:g} req/s, batched server",
        "value": first["p99_ms"], "unit": "ms", "n_gpus": 1, "steps": len(rates), "warmup": 0,
        "ms_per_step": first["p50_ms"], "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic",
        "config": {"workload": "serving_mix_8_scenes_50k_1M_tris", "duration_s": args.duration,
                   "hbm_budget_gb": args.budget_gb, "rates_rps": rates,
                   "scene_triangles": [w["agg"].n_tris for w in worlds]},
        "sweep": sweep, "setup_s": setup_s,
    }
    print(json.dumps(line))
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="scaled",
                    choices=["scaled", "batch", "lightslice", "mrcs", "guided", "serve", "restart"],
                    help="scaled: the 512x512 x 32,768-VPL gather (default); batch: 64 uneven "
                         "instances, batched + graph vs plain launches (1 GPU); lightslice: "
                         "LightSlice build + clustered gather on the scaled scene (1 GPU); mrcs: matrix "
                         "row-column sampling set-up + clustered gather on the scaled scene (1 GPU); restart: "
                         "scene build vs restore from a blob (1 GPU); guided: "
                         "LightSlice-guided path tracing, 1024^2 x 16 spp (1 GPU)")
    ap.add_argument("--spp", type=int, default=16)
    ap.add_argument("--sampler", choices=["jensen", "metropolis"], default="jensen",
                    help="guided: LightSlice's direction sampler")
    ap.add_argument("--side", type=int, default=1024)
    ap.add_argument("--max-slice-clusters", type=int, default=4096)
    ap.add_argument("--slice-size", type=int, default=4096)
    ap.add_argument("--rates", default=SERVE_RATES, help="serve: arrival rates (req/s)")
    ap.add_argument("--duration", type=float, default=20.0, help="serve: seconds of arrivals per rate")
    ap.add_argument("--serve-duration", type=float, default=8.0,
                    help="default workload: seconds of arrivals per rate of the serving sweep in its line "
                         "(0 leaves the sweep out)")
    ap.add_argument("--budget-gb", type=float, default=4.0, help="serve: HBM admission budget")
    ap.add_argument("--instances", type=int, default=64)
    ap.add_argument("--small", action="store_true",
                    help="batch: small instances (10k-50k triangles, 64^2-256^2 images, 1k-4k VPLs)")
    ap.add_argument("--vpls", type=int, default=0,
                    help="scaled: VPL count (default 32,768; smaller for profiling captures)")
    ap.add_argument("--skip-cpu", action="store_true",
                    help="scaled: leave out the CPU-baseline leg (profiling runs)")
    args = ap.parse_args()
    if args.vpls > 0:
        global N_VPL
        N_VPL = args.vpls
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch":
        return run_batch(args)
    if args.workload == "lightslice":
        return run_lightslice(args)
    if args.workload == "mrcs":
        return run_mrcs(args)
    if args.workload == "restart":
        return run_restart(args)
    if args.workload == "guided":
        return run_guided(args)
    if args.workload == "serve":
        return run_serve(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
