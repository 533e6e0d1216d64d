"""Benchmark: Mrays/s of the Kerr-Newman null-geodesic trace on a 3840x2160 frame.

Workload (the headline frame of the precision study): Kerr-Newman M = 1, a = 0.9, Q = 0.3,
outgoing Kerr-Schild chart, static observer at r = 50 M, inclination 75 deg, pinhole 3840x2160,
30 deg vertical FOV, one ray per pixel centre; escape at r = 1000 M, capture at r_+ + 1e-3,
Keplerian bolometric surface from the prograde ISCO to 20 M. One step = one frame traced by the
persistent DP5(4) kernel in MIXED precision (binary32 stepping, binary64 state, shell steps,
events and renormalisation). Synthetic inputs: the frame is generated on the device from the camera.

`python bench.py [--gpus N --steps K --warmup W] [--impl reference]`
Prints one JSON line on rank 0. Under torchrun each rank traces its own frame (weak scaling; the
only collective is the max-reduction of the timings).
"""

from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WIDTH, HEIGHT = 3840, 2160
SPIN, CHARGE, INCL_DEG, R_OBS, FOV_DEG = 0.9, 0.3, 75.0, 50.0, 30.0
ESCAPE, HORIZON_OFFSET, SURFACE_OUTER = 1000.0, 1e-3, 20.0
METRIC = "Mrays/s at 3840x2160 a=0.9, mixed vs plain at equal FP64 error; adjoint Mrays/s"
L2_BYTES = 126 * 2 ** 20
# DRAM bytes (read + write) per ray of the frame's kernels from ncu captures of the same scene at
# 1280x720 (the bulk and tail kernels; the one-kernel FP32 and FP64), scaled by the ray count. MIXED is the
# bulk and tail kernels together: the 128-byte hand-off record written and read back, and the
# 200-byte results (part of each still in the 126 MB L2 when a 720p launch ends).
TRAFFIC_BYTES_PER_RAY = {"mixed": (0.093696e6 + 62.725632e6 + 120.360704e6 + 160.456704e6) / 921600,
                         "fp32": (3.284480e6 + 146.337792e6) / 921600,
                         "fp64": (8.472576e6 + 141.483776e6) / 921600}


def workload_config(precision: str, policy: dict | None = None) -> dict:
    cfg = {
        "workload": f"kerr-newman-frame-{WIDTH}x{HEIGHT}", "width": WIDTH, "height": HEIGHT, "spin": SPIN,
        "charge": CHARGE, "inclination_deg": INCL_DEG, "observer_radius_m": R_OBS, "vertical_fov_deg": FOV_DEG,
        "escape_radius_m": ESCAPE, "capture": "r_+ + 1e-3", "surface": "prograde ISCO .. 20 M", "chart": "outgoing",
        "precision": precision, "stepper": "DP5(4) adaptive",
        "l2": "L2 flushed between timed frames (256 MiB write); results 1.66 GB/frame exceed L2",
    }
    if policy:
        cfg["policy"] = policy
    return cfg


def compact_config(precision: str, policy: dict) -> dict:
    """The headline line's config: the workload and the policy fields that set its cost."""
    return {"workload": f"kerr-newman-frame-{WIDTH}x{HEIGHT}",
            "scene": f"a={SPIN} Q={CHARGE} i={INCL_DEG:g}deg r_obs={R_OBS:g}M fov={FOV_DEG:g}deg",
            "precision": precision, "rtol": policy.get("position_rtol"), "l2": "flushed between frames"}


def compact_roofline(r: dict) -> dict:
    """The headline line's roofline: the dominant kernel's algorithmic FP32 FMA rate against the
    nominal FP32 FMA peak, the DRAM traffic per launch and the HBM fraction of its result stores."""
    return {"bound": r["bound"], "achieved": r["achieved"], "peak": r["peak"], "unit": r["unit"], "frac": r["frac"],
            "traffic": r["traffic"], "peak_source": "nominal",
            "hbm_frac": r["hbm_view"]["frac"]}


def make_headline(value, world, steps, warmup, ms_per_step, precision, policy, launches, clk, e2e, roofline,
                  scaling: str = "weak") -> dict:
    """The last stdout line: the contract keys only, well under 1 KB (the studies go on earlier lines)."""
    return rounded({
        "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": world, "steps": steps, "warmup": warmup,
        "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": scaling, "vs_baseline": None,
        "dtype": {"fp32": "f32", "mixed": "f32+f64", "fp64": "f64"}[precision],
        "data": "synthetic", "config": compact_config(precision, policy),
        "gpu_launches": int(launches), "clocks": {k: clk.get(k) for k in ("sm_mhz", "sm_max_mhz", "reasons")},
        "e2e": e2e, "roofline": compact_roofline(roofline),
    })


def rounded(x, digits: int = 6):
    """x with every float rounded to `digits` significant digits (for the short headline line)."""
    if isinstance(x, float):
        return float(f"{x:.{digits}g}") if math.isfinite(x) else x
    if isinstance(x, dict):
        return {k: rounded(v, digits) for k, v in x.items()}
    if isinstance(x, (list, tuple)):
        return [rounded(v, digits) for v in x]
    return x


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self) -> dict:
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peaks() -> dict:
    p = ROOT / "MEASURED_PEAKS.json"
    return json.loads(p.read_text()) if p.exists() else {}


def fp32_fma_peak_tflops(sm_count: int, sm_mhz: float) -> float:
    # 128 FP32 lanes per SM, one FMA (2 flops) per lane per clock
    return sm_count * 128 * 2 * sm_mhz * 1e6 / 1e12


def make_observation(G, width=None, height=None):
    width = width or WIDTH
    height = height or HEIGHT
    isco = G.prograde_isco(SPIN, CHARGE)
    return G.Observation.from_oblate(R_OBS, math.radians(INCL_DEG), 0.0, spin=SPIN, charge=CHARGE,
                                     chart=G.KerrSchildChart.OUTGOING, width=width, height=height,
                                     vertical_fov=math.radians(FOV_DEG), escape_radius=ESCAPE,
                                     surface=G.EquatorialSurface(isco, SURFACE_OUTER), horizon_offset=HORIZON_OFFSET)


def sample_pixels(n: int, seed: int = 64):
    import numpy as np

    rng = np.random.default_rng(seed)
    idx = np.sort(rng.choice(WIDTH * HEIGHT, size=n, replace=False))
    return idx % WIDTH, idx // WIDTH, idx


def oracle_job():
    """The headline frame as the CPU oracle's scene and events, set up from the oracle alone (its
    own observer placement and ISCO), so that a process that only runs the oracle maps no product
    library. The observer position equals make_observation's to the last bit (a CPU test checks)."""
    import oracle as O

    txyz = [0.0, *O.oblate_to_cartesian(SPIN, 1, R_OBS, math.radians(INCL_DEG), 0.0)]
    osc = O.scene(mass=1.0, spin=SPIN, charge=CHARGE, chart=1, observer_txyz=txyz, width=WIDTH,
                  height=HEIGHT, vertical_fov=math.radians(FOV_DEG))
    ev = O.events(escape_radius=ESCAPE, surface=(O.prograde_isco(1.0, SPIN, CHARGE), SURFACE_OUTER),
                  horizon_offset=HORIZON_OFFSET)
    return osc, ev


def cpu_oracle_sample(n_rays: int, threads: int):
    """Binary64 oracle (rtol 1e-10, atol 1e-12) on a seeded pixel sample of the frame."""
    import oracle as O

    osc, ev = oracle_job()
    px, py, idx = sample_pixels(n_rays)
    t0 = time.perf_counter()
    ref, status = O.trace_pixels(osc, O.custom_policy(1e-10, 1e-12), ev, px, py, threads=threads)
    dt = time.perf_counter() - t0
    return ref, idx, dt


def reference_gpu_algorithm_report(ref, idx, threads: int) -> dict:
    """Errors of the reference's own GPU algorithm (binary32 fixed-policy RK4, restated on the CPU
    as the second comparator) on the same oracle sample, for comparison with the CUDA modes."""
    import numpy as np
    import oracle as O

    osc, ev = oracle_job()
    t0 = time.perf_counter()
    rows = O.rk4_pixels(osc, ev, idx % WIDTH, idx // WIDTH, threads=threads)
    cpu_s = time.perf_counter() - t0
    F, R = O.F, O.RK4
    rt = rows[:, R["termination"]].astype(int)
    ot = ref[:, F["termination"]].astype(int)
    same = rt == ot
    rep = {"algorithm": "binary32 RK4, h = clamp(0.1 r, 0.005, 8), at most 2048 steps (geodesic_integration.wgsl)",
           "rays": int(idx.size), "class_mismatch": int((~same).sum()),
           "uncertain": int((rt == O.UNCERTAIN).sum()), "step_exhaustion": int((rt == O.STEP_EXHAUSTION).sum()),
           "steps_mean": float(rows[:, R["steps"]].mean()),
           "cpu_mrays_per_s": idx.size / cpu_s / 1e6, "cores": threads}
    esc = same & (ot == O.ESCAPE)
    if esc.any():
        d = np.stack([ref[esc, F["escape_dx"]], ref[esc, F["escape_dy"]], ref[esc, F["escape_dz"]]], axis=1)
        v = rows[esc][:, [R["source0"], R["source1"], R["source2"]]]
        rep["escape_direction_rad"] = float(np.max(np.arccos(np.clip((d * v).sum(1), -1, 1))))
    srf = same & (ot == O.SURFACE)
    if srf.any():
        g0 = ref[srf, F["frequency_ratio"]]
        rep["g_rel"] = float(np.max(np.abs(rows[srf, R["source2"]] - g0) / g0))
        rep["hit_radius"] = float(np.max(np.abs(rows[srf, R["source0"]] - ref[srf, F["source_radius"]])))
    if same.any():
        rep["travel_time"] = float(np.max(np.abs(rows[same, R["travel_time"]] - ref[same, F["travel_time"]])))
    return rep


def run_reference(args) -> None:
    """The reference's CPU algorithm (binary64 oracle port) on the host cores, bounded samples."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle as O

    threads = O.hardware_threads()
    n = args.cpu_sample
    times = []
    for _ in range(args.warmup):
        cpu_oracle_sample(max(n // 8, 64), threads)
    for _ in range(args.steps):
        _, _, dt = cpu_oracle_sample(n, threads)
        times.append(dt)
    total = sum(times)
    value = n * len(times) / total / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mrays/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config("f64 (CPU oracle, rtol 1e-10)"),
        "cpu_baseline": {"value": value, "unit": "Mrays/s", "cores": threads, "kind": "port",
                         "sample": f"{n} seeded pixels of the {WIDTH}x{HEIGHT} frame per step"},
        "e2e": {"value": value, "unit": "Mrays/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def error_report(gpu: dict, ref, idx) -> dict:
    import numpy as np
    import oracle as O

    F = O.F
    sel = idx
    gt = gpu["termination"][sel]
    ot = ref[:, F["termination"]].astype(int)
    same = gt == ot
    rep = {"rays": int(sel.size), "class_mismatch": int((~same).sum())}
    esc = same & (ot == 2)
    if esc.any():
        d = np.stack([ref[esc, F["escape_dx"]], ref[esc, F["escape_dy"]], ref[esc, F["escape_dz"]]], axis=1)
        th, ph = gpu["escape_theta"][sel][esc], gpu["escape_phi"][sel][esc]
        v = np.stack([np.sin(th) * np.cos(ph), np.sin(th) * np.sin(ph), np.cos(th)], axis=1)
        rep["escape_direction_rad"] = float(np.max(np.arccos(np.clip((d * v).sum(1), -1, 1))))
    srf = same & (ot == 7)
    if srf.any():
        g0 = ref[srf, F["frequency_ratio"]]
        rep["g_rel"] = float(np.max(np.abs(gpu["frequency_ratio"][sel][srf] - g0) / g0))
        rep["hit_radius"] = float(np.max(np.abs(gpu["source_radius"][sel][srf] - ref[srf, F["source_radius"]])))
    if same.any():
        rep["travel_time"] = float(np.max(np.abs(gpu["travel_time"][sel][same] - ref[same, F["travel_time"]])))
        for k in ("max_null_residual", "max_lz_drift", "max_carter_drift"):
            rep[k] = float(np.max(np.abs(gpu[k][sel][same] - ref[same, F[k]])))
        rep["event_residual_max"] = float(np.nanmax(gpu["event_residual"][sel][same]))
    return rep


def run_gpu(args) -> None:
    import numpy as np
    import torch

    import gravlume_b200 as G
    from gravlume_b200 import _native as N

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    dev = torch.device("cuda", local)
    obs = make_observation(G)
    scene = obs.pack()
    # weak scaling: every rank traces a frame of its own; strong: the ranks split one frame into
    # bands of whole tile rows (tile regions on the camera, no collective on the data path)
    region = None
    if args.scaling == "strong":
        from gravlume_b200.shard import region_pixel_rows, shard_region

        region = shard_region(WIDTH, HEIGHT, world, rank)
    cam = G.image_camera(0, WIDTH, HEIGHT, region=region)
    pipe = G.TracePipeline(local)
    precision = {"fp32": G.Precision.FP32, "mixed": G.Precision.MIXED, "fp64": G.Precision.FP64}[args.precision]
    pipe.set_policy(G.ReferencePolicy.frame(precision, persistent=int(args.persistent)))
    results = G.TraceResults(WIDTH * HEIGHT, dev)
    stream = torch.cuda.current_stream()
    if args.autotune:
        small = make_observation(G, max(WIDTH // 4, 64), max(HEIGHT // 4, 64))
        pipe.autotune([small.pack()], [G.image_camera(0, small.width, small.height)], repeats=1)
    policy = pipe.policy.as_dict()
    flush = torch.empty(256 * 2 ** 20, dtype=torch.uint8, device=dev)
    for _ in range(args.warmup):
        pipe.trace([scene], [cam], results, stream=stream)
    torch.cuda.synchronize()
    launches0 = pipe.stats().kernel_launches
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(torch.cuda.current_device()) as clocks:
        for k in range(args.steps):
            flush.fill_(k & 0xFF)
            ev[k][0].record(stream)
            pipe.trace([scene], [cam], results, stream=stream)
            ev[k][1].record(stream)
        torch.cuda.synchronize()
    if dist:
        dist.barrier()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = sum(step_ms)
    launches = pipe.stats().kernel_launches - launches0
    if dist:
        from gravlume_b200.shard import max_over_ranks

        total_ms = max_over_ranks(total_ms)
    rays = WIDTH * HEIGHT
    frames = world if args.scaling == "weak" else 1
    value = frames * rays * args.steps / (total_ms / 1e3) / 1e6
    d = results.numpy()
    if region is not None:  # this rank's band of the frame
        band = region_pixel_rows(region, WIDTH, HEIGHT)
        d = {k: v[band.start * WIDTH:band.stop * WIDTH] for k, v in d.items()}

    # ---- end to end through the host-buffer call (H2D job table, trace, D2H of every field)
    e2e_ms = None
    host = G.TraceResults(WIDTH * HEIGHT, None, host=True)
    e2e_steps = max(1, min(args.steps, 2))
    pipe.trace_host([scene], [cam])  # warm the workspace
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        sa, ca = pipe._arrays([scene], [cam])
        rs = host.struct()
        N.check(N.lib().glc_trace_host(pipe._h, sa, 1, ca, 1, rs), "glc_trace_host")
    e2e_ms = 1e3 * (time.perf_counter() - t0) / e2e_steps
    if dist:
        from gravlume_b200.shard import max_over_ranks

        e2e_ms = max_over_ranks(e2e_ms)  # every rank traces its own frame; the slowest sets the pace
    e2e = {"value": frames * rays / (e2e_ms / 1e3) / 1e6, "unit": "Mrays/s",
           "h2d_bytes_per_step": int(world * ctypes_sizeof_job()),
           "d2h_bytes_per_step": int(frames * WIDTH * HEIGHT * sum(N.RESULT_BYTES.values()))}

    if rank != 0:
        if dist:
            dist.destroy_process_group()
        return

    # ---- roofline: algorithmic flops of the attempted steps / average launch duration
    flops = np.zeros(4)
    N.lib().glc_flop_model(flops.ctypes.data)
    attempts = float(d["accepted_steps"].sum() + d["rejected_steps"].sum())
    alg_flops = attempts * flops[2]
    launch_s = (total_ms / args.steps) / 1e3
    rays_here = rays if region is None else len(band) * WIDTH
    achieved_tflops = alg_flops / launch_s / 1e12
    clk = clocks.summary()
    sm_count = pipe.stats().sm_count
    peak_mhz = clk["sm_mhz"] or 1965.0
    peak = fp32_fma_peak_tflops(sm_count, peak_mhz)
    roofline = {"bound": "fp32_fma", "achieved": achieved_tflops, "peak": peak, "unit": "TFLOP/s",
                "frac": achieved_tflops / peak,
                "peak_source": f"nominal {sm_count} SMs x 128 FP32 lanes x 2 x median SM clock {peak_mhz:.0f} MHz "
                               "under load (MEASURED_PEAKS.json has no FP32 figure)",
                "alg_flops_per_launch": alg_flops, "attempted_steps": attempts,
                "flops_per_attempt": float(flops[2]),
                "traffic": args.traffic_bytes if args.traffic_bytes is not None else (
                    TRAFFIC_BYTES_PER_RAY[args.precision] * rays_here if args.precision in TRAFFIC_BYTES_PER_RAY else None),
                "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the frame's kernels at 1280x720, scaled by rays",
                "algorithmic_bytes_per_launch": float(sum(N.RESULT_BYTES.values())) * rays_here}
    # the same launch against HBM, to show how far from bandwidth-bound the path is
    hbm_peak, hbm_source = 6650.0, "fallback"
    try:
        hbm_peak, hbm_source = float(json.loads((ROOT / "MEASURED_PEAKS.json").read_text())["hbm_gbs"]), "measured"
    except (OSError, ValueError, KeyError):
        pass
    hbm_achieved = roofline["algorithmic_bytes_per_launch"] / launch_s / 1e9
    roofline["hbm_view"] = {"achieved": hbm_achieved, "peak": hbm_peak, "unit": "GB/s", "frac": hbm_achieved / hbm_peak,
                            "peak_source": f"{hbm_source} copy bandwidth"}

    headline = make_headline(value, world, args.steps, args.warmup, total_ms / args.steps, args.precision, policy,
                             launches, clk, e2e, roofline, scaling=args.scaling)
    studies = {"roofline_detail": roofline, "class_histogram": np.bincount(d["termination"], minlength=9).tolist(),
               "steps_per_ray": {"mean": float(d["accepted_steps"].mean()), "max": int(d["accepted_steps"].max()),
                                 "rejected_mean": float(d["rejected_steps"].mean())}}

    # ---- CPU baseline: the binary64 oracle on a bounded seeded sample of the same frame
    ref = idx = None
    if args.cpu_sample > 0:
        import oracle as O

        threads = O.hardware_threads()
        ref, idx, cpu_s = cpu_oracle_sample(args.cpu_sample, threads)
        headline["cpu_baseline"] = rounded({"value": args.cpu_sample / cpu_s / 1e6, "unit": "Mrays/s",
                                            "cores": threads, "kind": "port",
                                            "sample": f"{args.cpu_sample} seeded pixels, rtol 1e-10"})

    # ---- precision study on the same frame: plain FP32 and FP64 at the same job, errors vs the oracle
    if args.compare:
        comp = {}
        if ref is not None:
            comp[args.precision] = error_report(d, ref, idx)
            comp["reference_gpu_algorithm"] = reference_gpu_algorithm_report(ref, idx, threads)
        shape = {k: policy[k] for k in ("persistent", "block_threads", "tile_w", "tile_h", "refill_interval",
                                         "rays_per_grab")}
        frame_tol = {k: policy[k] for k in ("position_rtol", "position_atol", "momentum_rtol", "momentum_atol",
                                             "maximum_step")}
        runs = (("fp32", G.Precision.FP32, {}), ("mixed", G.Precision.MIXED, {}),
                ("fp64_frame_tolerance", G.Precision.FP64, frame_tol),
                ("fp64_oracle_policy", G.Precision.FP64, {}))
        for name, prec, extra in runs:
            if name == args.precision:
                continue
            pipe.set_policy(G.ReferencePolicy.frame(prec, **shape, **extra))
            pipe.trace([scene], [cam], results, stream=stream)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            pipe.trace([scene], [cam], results, stream=stream)
            b.record(stream)
            torch.cuda.synchronize()
            ms = a.elapsed_time(b)
            dd = results.numpy()
            entry = {"mrays_per_s": rays / (ms / 1e3) / 1e6, "ms": ms,
                     "attempts_per_ray": float((dd["accepted_steps"] + dd["rejected_steps"]).mean()),
                     "policy": {k: getattr(pipe.policy, k) for k in ("position_rtol", "maximum_step")}}
            if ref is not None:
                entry["error_vs_oracle"] = error_report(dd, ref, idx)
            comp[name] = entry
        # tolerance sweep: throughput against error for each mode, so that modes can be compared at
        # equal error (binary32 stepping stops improving at its rounding floor)
        if ref is not None and args.sweep:
            sweep = []
            for rtol in (1e-5, 1e-6, 1e-7, 1e-8):
                for name, prec, pair in (("fp32", G.Precision.FP32, 0), ("mixed", G.Precision.MIXED, 0),
                                         ("mixed_pair_state", G.Precision.MIXED, 1), ("fp64", G.Precision.FP64, 0)):
                    pipe.set_policy(G.ReferencePolicy.frame(prec, **shape, position_rtol=rtol, momentum_rtol=rtol,
                                                            position_atol=rtol * 1e-2, momentum_atol=rtol * 1e-2,
                                                            maximum_step=1000.0, mixed_pair_state=pair))
                    pipe.trace([scene], [cam], results, stream=stream)
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record(stream)
                    pipe.trace([scene], [cam], results, stream=stream)
                    b.record(stream)
                    torch.cuda.synchronize()
                    ms = a.elapsed_time(b)
                    dd = results.numpy()
                    sweep.append({"precision": name, "rtol": rtol, "mrays_per_s": rays / (ms / 1e3) / 1e6,
                                  "error_vs_oracle": error_report(dd, ref, idx)})
            comp["tolerance_sweep"] = sweep
        comp[args.precision] = {"mrays_per_s": value / world, "ms": total_ms / args.steps,
                                "attempts_per_ray": float((d["accepted_steps"] + d["rejected_steps"]).mean()),
                                "error_vs_oracle": comp.get(args.precision)}
        studies["precision_study"] = comp
    if args.adjoint:
        studies["adjoint"] = adjoint_study(G, args, local)
    if args.batch:
        studies["batch"] = batch_study(G, local)
        studies["sky"] = sky_study(G, local)
    if args.footprint:
        studies["footprint"] = footprint_study(G, local, args.cpu_sample > 0)
    if args.scenes:
        studies["config1"] = config1_study(G, local, args.cpu_sample > 0)
        studies["scenes"] = scenes_study(G, local, args.cpu_sample > 0)
    if args.stress:
        studies["stress"] = stress_study(G, local, args.cpu_sample > 0, args.stress_side)
    # the studies go on earlier lines (and to --studies-out); the last line is the short headline
    for name, study in studies.items():
        print(json.dumps({"study": name, "result": study}), flush=True)
    if args.studies_out:
        Path(args.studies_out).write_text(json.dumps({"headline": headline, "studies": studies}, indent=1))
    print(json.dumps(headline), flush=True)
    if dist:
        dist.destroy_process_group()


def batch_job(G, seed: int = 4):
    """The batching workload: 64 seeded scenes in one job (square views with sides uniform in
    {128, 192, ..., 1024}; a ~ U[0, 0.99]; Q uniform under a^2 + Q^2 <= 0.98; inclination
    ~ U[5, 89] deg; observer radius log-uniform in [20, 1000] M; 30 deg FOV, Keplerian surface from
    the prograde ISCO to 20 M, escape at max(1000, 2 r_obs); a draw whose observer frame the
    reference's construction rejects -- Gram residual above 1e-12, which some far observers hit --
    is drawn again), plus one 2048x1024 equirectangular
    escape map of all sky directions from r = 15 M (a = 0.9, Q = 0.3, i = 60 deg, no surface).
    Returns (scenes, cameras, result slots, per-scene parameters)."""
    import numpy as np

    rng = np.random.default_rng(seed)
    scenes, cams, meta = [], [], []
    off = 0
    while len(scenes) < 64:
        i = len(scenes)
        side = int(rng.choice(np.arange(128, 1025, 64)))
        a = float(rng.uniform(0.0, 0.99))
        q = float(rng.uniform(0.0, math.sqrt(max(0.98 - a * a, 0.0))))
        incl = math.radians(float(rng.uniform(5.0, 89.0)))
        r_obs = float(math.exp(rng.uniform(math.log(20.0), math.log(1000.0))))
        obs = G.Observation.from_oblate(r_obs, incl, 0.0, spin=a, charge=q, chart=G.KerrSchildChart.OUTGOING,
                                        width=side, height=side, vertical_fov=math.radians(FOV_DEG),
                                        escape_radius=max(ESCAPE, 2.0 * r_obs),
                                        surface=G.EquatorialSurface(G.prograde_isco(a, q), SURFACE_OUTER),
                                        horizon_offset=HORIZON_OFFSET)
        try:
            scenes.append(obs.pack())
        except G.GlcError:
            continue
        cams.append(G.image_camera(i, side, side, offset=off))
        meta.append({"side": side, "spin": a, "charge": q, "inclination": incl, "observer_radius": r_obs})
        off += side * side
    from gravlume_b200 import _native as N

    sky = G.Observation.from_oblate(15.0, math.radians(60.0), 0.0, spin=0.9, charge=0.3,
                                    chart=G.KerrSchildChart.OUTGOING, width=64, height=64,
                                    vertical_fov=math.radians(FOV_DEG), escape_radius=ESCAPE, surface=None,
                                    horizon_offset=HORIZON_OFFSET)
    scenes.append(sky.pack())
    cams.append(G.image_camera(64, 2048, 1024, offset=off, kind=N.CAMERA_EQUIRECT))
    meta.append({"side": None, "spin": 0.9, "charge": 0.3, "inclination": math.radians(60.0), "observer_radius": 15.0,
                 "equirect": [2048, 1024]})
    off += 2048 * 1024
    return scenes, cams, off, meta


def batch_study(G, device: int) -> dict:
    """The 64-scene batch plus the equirectangular escape map (batch_job) in MIXED: one persistent
    work-queue launch (lane refill), its CUDA-graph replay, the one-thread-per-ray kernel, the
    warp-grab work queue, and the launch shape the autotuner picks on a 4-scene sub-job; CUDA-event
    time per job, L2 flushed in between."""
    import torch

    scenes, cams, slots, _ = batch_job(G)
    pipe = G.TracePipeline(device)
    res = G.TraceResults(slots, f"cuda:{device}")
    flush = torch.empty(256 * 2 ** 20, dtype=torch.uint8, device=f"cuda:{device}")
    stream = torch.cuda.current_stream()

    def timed(run, reps=2):
        run()
        torch.cuda.synchronize()
        best = float("inf")
        for _ in range(reps):
            flush.fill_(3)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            run()
            b.record(stream)
            torch.cuda.synchronize()
            best = min(best, a.elapsed_time(b))
        return best

    out = {"workload": "kerr-newman-batch-64-scenes+equirect-2048x1024", "rays": slots, "precision": "mixed"}
    pipe.set_policy(G.ReferencePolicy.frame(G.Precision.MIXED, persistent=1))
    ms = timed(lambda: pipe.trace(scenes, cams, res, stream=stream))
    out["persistent"] = {"ms": ms, "mrays_per_s": slots / (ms / 1e3) / 1e6}
    gstream = torch.cuda.Stream()
    torch.cuda.synchronize()  # order the graph's stream after the result buffers' initialisation
    graph = pipe.capture_graph(scenes, cams, res, gstream)
    with torch.cuda.stream(gstream):
        gs = torch.cuda.current_stream()

        def replay():
            graph.launch(gs)

        graph.launch(gs)
        gstream.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(gs)
        replay()
        b.record(gs)
        gstream.synchronize()
        ms = a.elapsed_time(b)
    graph.close()
    out["graph"] = {"ms": ms, "mrays_per_s": slots / (ms / 1e3) / 1e6}
    pipe.set_policy(G.ReferencePolicy.frame(G.Precision.MIXED, persistent=0))
    ms = timed(lambda: pipe.trace(scenes, cams, res, stream=stream))
    out["simple"] = {"ms": ms, "mrays_per_s": slots / (ms / 1e3) / 1e6}
    for grab in (64, 256):
        pipe.set_policy(G.ReferencePolicy.frame(G.Precision.MIXED, persistent=2, rays_per_grab=grab))
        ms = timed(lambda: pipe.trace(scenes, cams, res, stream=stream))
        out[f"warp_queue_grab{grab}"] = {"ms": ms, "mrays_per_s": slots / (ms / 1e3) / 1e6}
    sub_s = scenes[:4]
    sub_c, off = [], 0
    for j in range(4):
        sub_c.append(G.image_camera(j, cams[j].width, cams[j].height, offset=off))
        off += cams[j].width * cams[j].height
    pipe.set_policy(G.ReferencePolicy.frame(G.Precision.MIXED, persistent=1))
    tuned = pipe.autotune(sub_s, sub_c, repeats=1)
    pipe.set_policy(tuned)
    ms = timed(lambda: pipe.trace(scenes, cams, res, stream=stream))
    out["autotuned"] = {"ms": ms, "mrays_per_s": slots / (ms / 1e3) / 1e6,
                        "policy": {k: getattr(tuned, k) for k in ("persistent", "block_threads", "tile_w", "tile_h",
                                                                  "rays_per_grab", "refill_interval",
                                                                  "refill_min_idle")}}
    pipe.close()
    return out


def sky_study(G, device: int) -> dict:
    """The accelerators on the batch's escape map (2048x1024 equirectangular, all sky directions
    from r = 15 M, a = 0.9, Q = 0.3, no surface) in MIXED: plain tracing, interval capture
    certificates, the escape-direction map, and both; CUDA-event time per frame, L2 flushed."""
    import torch
    from gravlume_b200 import _native as N

    w, h = 2048, 1024
    sky = G.Observation.from_oblate(15.0, math.radians(60.0), 0.0, spin=0.9, charge=0.3,
                                    chart=G.KerrSchildChart.OUTGOING, width=64, height=64,
                                    vertical_fov=math.radians(FOV_DEG), escape_radius=ESCAPE, surface=None,
                                    horizon_offset=HORIZON_OFFSET)
    scene = sky.pack()
    cam = G.image_camera(0, w, h, kind=N.CAMERA_EQUIRECT)
    pipe = G.TracePipeline(device)
    res = G.TraceResults(w * h, f"cuda:{device}")
    flush = torch.empty(256 * 2 ** 20, dtype=torch.uint8, device=f"cuda:{device}")
    stream = torch.cuda.current_stream()
    out = {"workload": "kerr-newman-escape-map-equirect-2048x1024", "precision": "mixed"}
    for name, cert, emap in (("plain", 0, 0), ("certificates", 1, 0), ("escape_map", 0, 1), ("both", 1, 1)):
        pipe.set_policy(G.ReferencePolicy.frame(G.Precision.MIXED, capture_certificates=cert, escape_map=emap))
        pipe.trace([scene], [cam], res, stream=stream)
        best = float("inf")
        for _ in range(2):
            flush.fill_(5)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(stream)
            pipe.trace([scene], [cam], res, stream=stream)
            b.record(stream)
            torch.cuda.synchronize()
            best = min(best, a.elapsed_time(b))
        d = res.numpy()
        out[name] = {"ms": best, "mrays_per_s": w * h / (best / 1e3) / 1e6,
                     "certified_fraction": float(((d["flags"] & 16) != 0).mean()),
                     "reconstructed_fraction": float(((d["flags"] & 32) != 0).mean())}
    # shadow-edge refinement of the headline view without its surface (the shadow's whole rim in
    # view): the primary trace, then glc_refine_shadow_edges, CUDA events around the refinement
    import numpy as np

    pipe.set_policy(G.ReferencePolicy.frame(G.Precision.MIXED))
    view = G.Observation.from_oblate(R_OBS, math.radians(INCL_DEG), 0.0, spin=SPIN, charge=CHARGE,
                                     chart=G.KerrSchildChart.OUTGOING, width=WIDTH, height=HEIGHT,
                                     vertical_fov=math.radians(FOV_DEG), escape_radius=ESCAPE, surface=None,
                                     horizon_offset=HORIZON_OFFSET)
    vs, vcam = view.pack(), [G.image_camera(0, WIDTH, HEIGHT)]
    primary = G.TraceResults(WIDTH * HEIGHT, f"cuda:{device}", ["code"])
    pipe.trace([vs], vcam, primary, stream=stream)
    pipe.refine_shadow_edges([vs], vcam, primary, stream=stream)
    best = float("inf")
    for _ in range(2):
        flush.fill_(5)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        cov = pipe.refine_shadow_edges([vs], vcam, primary, stream=stream)
        b.record(stream)
        torch.cuda.synchronize()
        best = min(best, a.elapsed_time(b))
    c = cov.cpu().numpy()
    edges = int(((c > 0) & (c < 1)).sum())
    out["shadow_edges"] = {"workload": f"kerr-newman-sky-{WIDTH}x{HEIGHT} (headline view, no surface)",
                           "precision": "mixed", "refine_ms": best, "fractional_coverage_pixels": edges,
                           "escape_pixels": int((c == 1).sum()), "capture_pixels": int((c == 0).sum())}
    pipe.close()
    return out


def footprint_study(G, device: int, cpu: bool) -> dict:
    """Surface footprints (glc_surface_footprint) of the headline frame's surface pixels after its
    primary trace, per precision and method: the reference's quarter-pixel estimate (four
    neighbour traces per surface pixel) and the forward-mode tangent (one re-trace with two tangent
    channels). CUDA-event time of the footprint call alone, L2 flushed; the oracle's quarter-pixel
    footprint of 64 seeded surface pixels on all host threads for scale."""
    import numpy as np
    import torch

    obs = make_observation(G)
    scene = obs.pack()
    cam = [G.image_camera(0, WIDTH, HEIGHT)]
    pipe = G.TracePipeline(device)
    primary = G.TraceResults(WIDTH * HEIGHT, f"cuda:{device}")
    flush = torch.empty(256 * 2 ** 20, dtype=torch.uint8, device=f"cuda:{device}")
    stream = torch.cuda.current_stream()
    out = {"workload": f"kerr-newman-frame-{WIDTH}x{HEIGHT} surface pixels"}
    fields = {}
    for pname, prec in (("fp32", G.Precision.FP32), ("mixed", G.Precision.MIXED), ("fp64", G.Precision.FP64)):
        pipe.set_policy(G.ReferencePolicy.frame(prec))
        pipe.trace([scene], cam, primary, stream=stream)
        for method in ("quarter_pixel", "tangent"):
            fp = pipe.surface_footprint([scene], cam, primary, method, stream=stream)
            best = float("inf")
            for _ in range(2):
                flush.fill_(5)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                fp = pipe.surface_footprint([scene], cam, primary, method, stream=stream)
                b.record(stream)
                torch.cuda.synchronize()
                best = min(best, a.elapsed_time(b))
            f = G.footprint_fields(fp)
            listed = int((f["status"] != G.FootprintStatus.NO_SURFACE).sum())
            fields[(pname, method)] = f
            out[f"{pname}_{method}"] = {"ms": best, "surface_pixels": listed,
                                        "mpix_per_s": listed / (best / 1e3) / 1e6,
                                        "resolved_fraction": float((f["status"] == 1).sum() / max(listed, 1)),
                                        "discontinuity_fraction": float((f["status"] == 2).sum() / max(listed, 1))}
    # agreement of the two methods in binary64 where both resolve (quarter-pixel truncation)
    q, t = fields[("fp64", "quarter_pixel")], fields[("fp64", "tangent")]
    both = (q["status"] == 1) & (t["status"] == 1)
    jq, jt = q["jacobian"].reshape(-1, 4)[both], t["jacobian"].reshape(-1, 4)[both]
    rel = np.max(np.abs(jq - jt), axis=1) / np.max(np.abs(jq), axis=1)
    out["fp64_quarter_vs_tangent"] = {"median": float(np.median(rel)), "p99": float(np.quantile(rel, 0.99))}
    pipe.close()
    if cpu:
        import oracle as O

        rng = np.random.default_rng(11)
        surf = np.flatnonzero(q["status"] == 1)
        idx = np.sort(rng.choice(surf, 64, replace=False))
        osc = O.scene(mass=obs.mass, spin=obs.spin, charge=obs.charge, chart=int(obs.chart),
                      observer_txyz=obs.observer_txyz, target=obs.target_txyz, up_hint=obs.up_hint_xyz,
                      width=WIDTH, height=HEIGHT, vertical_fov=obs.vertical_fov)
        ev = O.events(escape_radius=ESCAPE, surface=(obs.surface.inner_radius, obs.surface.outer_radius),
                      horizon_offset=HORIZON_OFFSET)
        threads = O.hardware_threads()
        t0 = time.perf_counter()
        O.surface_footprint(osc, O.custom_policy(1e-10, 1e-12), ev, idx % WIDTH, idx // WIDTH, threads=threads)
        cpu_s = time.perf_counter() - t0
        out["cpu_oracle_quarter_pixel"] = {"mpix_per_s": idx.size / cpu_s / 1e6, "cores": threads,
                                           "sample": "64 seeded surface pixels, binary64 rtol 1e-10 atol 1e-12"}
    return out


def timed_trace(pipe, scenes, cams, res, stream, flush, reps=2):
    """Best CUDA-event time (ms) of reps traces of the job, L2 flushed before each."""
    import torch

    best = float("inf")
    for _ in range(reps):
        flush.fill_(3)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        pipe.trace(scenes, cams, res, stream=stream)
        b.record(stream)
        torch.cuda.synchronize()
        best = min(best, a.elapsed_time(b))
    return best


def frame_tolerance(G) -> dict:
    """The binary32 frame policy's tolerances and step cap, for running FP64 at the same tolerance."""
    p = G.ReferencePolicy.frame(G.Precision.FP32)
    return {k: getattr(p, k) for k in ("position_rtol", "position_atol", "momentum_rtol", "momentum_atol",
                                       "maximum_step")}


SCENE_SET = [(0.0, 0.0), (0.5, 0.0), (0.9, 0.3), (0.998, 0.0), (0.6, 0.7)]
SCENE_INCLINATIONS = [17.0, 60.0, 85.0]


def scenes_study(G, device: int, cpu: bool) -> dict:
    """The full-frame precision set at 1920x1080: (a, Q) in {(0,0), (0.5,0), (0.9,0.3), (0.998,0),
    (0.6,0.7)} x inclinations {17, 60, 85} deg, observer at r = 50 M, 30 deg FOV, surface from the
    prograde ISCO to 20 M. Per scene and precision (each at its frame tolerance: FP32 rtol 1e-6, MIXED 7e-7,
    FP64 at rtol 1e-6):
    CUDA-event Mrays/s (L2
    flushed, best of two) and, with the CPU leg, the errors against the binary64 oracle (rtol 1e-10)
    on 64 seeded pixels of the scene."""
    import numpy as np
    import torch

    w, h = 1920, 1080
    pipe = G.TracePipeline(device)
    res = G.TraceResults(w * h, f"cuda:{device}")
    flush = torch.empty(256 * 2 ** 20, dtype=torch.uint8, device=f"cuda:{device}")
    stream = torch.cuda.current_stream()
    precisions = (("fp32", G.Precision.FP32), ("mixed", G.Precision.MIXED), ("fp64", G.Precision.FP64))
    rows = []
    for a, q in SCENE_SET:
        isco = G.prograde_isco(a, q)
        for incl in SCENE_INCLINATIONS:
            obs = G.Observation.from_oblate(R_OBS, math.radians(incl), 0.0, spin=a, charge=q,
                                            chart=G.KerrSchildChart.OUTGOING, width=w, height=h,
                                            vertical_fov=math.radians(FOV_DEG), escape_radius=ESCAPE,
                                            surface=G.EquatorialSurface(isco, SURFACE_OUTER),
                                            horizon_offset=HORIZON_OFFSET)
            sc = obs.pack()
            cam = [G.image_camera(0, w, h)]
            row = {"spin": a, "charge": q, "inclination_deg": incl}
            ref = idx = None
            if cpu:
                import oracle as O

                rng = np.random.default_rng(int(1000 * a + 100 * q + incl))
                idx = np.sort(rng.choice(w * h, 64, replace=False))
                osc = O.scene(mass=1.0, spin=a, charge=q, chart=1, observer_txyz=obs.observer_txyz, width=w,
                              height=h, vertical_fov=obs.vertical_fov)
                ev = O.events(escape_radius=ESCAPE, surface=(isco, SURFACE_OUTER), horizon_offset=HORIZON_OFFSET)
                ref, _ = O.trace_pixels(osc, O.custom_policy(1e-10, 1e-12), ev, idx % w, idx // w,
                                        threads=O.hardware_threads())
            for name, prec in precisions:
                pipe.set_policy(G.ReferencePolicy.frame(prec, **frame_tolerance(G)))
                pipe.trace([sc], cam, res, stream=stream)
                ms = timed_trace(pipe, [sc], cam, res, stream, flush)
                entry = {"mrays_per_s": w * h / (ms / 1e3) / 1e6}
                if ref is not None:
                    entry["error_vs_oracle"] = error_report(res.numpy(), ref, idx)
                row[name] = entry
            rows.append(row)
    pipe.close()
    out = {"workload": f"kerr-newman-frames-{w}x{h}-15-scenes", "policy": "frame (FP32 rtol 1e-6, MIXED 7e-7, FP64 1e-6)", "scenes": rows}
    for name, _ in precisions:
        out[f"{name}_mrays_per_s_range"] = [min(r[name]["mrays_per_s"] for r in rows),
                                            max(r[name]["mrays_per_s"] for r in rows)]
        if cpu:
            out[f"{name}_class_mismatches"] = sum(r[name]["error_vs_oracle"]["class_mismatch"] for r in rows)
    return out


def config1_study(G, device: int, cpu: bool) -> dict:
    """The reference's CPU-runnable case: 256x256 pinhole, a = 0.9, Q = 0.3, i = 75 deg, r = 50 M,
    30 deg FOV, escape 1000 M, capture at r_+ + 1e-3, surface from the prograde ISCO to 20 M. FP64 at
    the oracle's policy (rtol 1e-10, atol 1e-12) and the three precisions at the frame tolerance:
    CUDA-event Mrays/s (best of three) and, with the CPU leg, errors against the binary64 oracle
    over every pixel of the frame (65,536 rays, about 20 s of host time on 16 threads)."""
    import numpy as np
    import torch

    w = h = 256
    obs = make_observation(G, w, h)
    sc = obs.pack()
    cam = [G.image_camera(0, w, h)]
    pipe = G.TracePipeline(device)
    res = G.TraceResults(w * h, f"cuda:{device}")
    flush = torch.empty(256 * 2 ** 20, dtype=torch.uint8, device=f"cuda:{device}")
    stream = torch.cuda.current_stream()
    ref = idx = None
    out = {"workload": "kerr-newman-frame-256x256"}
    if cpu:
        import oracle as O

        idx = np.arange(w * h)
        osc = O.scene(mass=1.0, spin=SPIN, charge=CHARGE, chart=1, observer_txyz=obs.observer_txyz, width=w,
                      height=h, vertical_fov=obs.vertical_fov)
        ev = O.events(escape_radius=ESCAPE, surface=(obs.surface.inner_radius, SURFACE_OUTER),
                      horizon_offset=HORIZON_OFFSET)
        threads = O.hardware_threads()
        t0 = time.perf_counter()
        ref, _ = O.trace_pixels(osc, O.custom_policy(1e-10, 1e-12), ev, idx % w, idx // w, threads=threads)
        out["cpu_oracle"] = {"mrays_per_s": idx.size / (time.perf_counter() - t0) / 1e6, "cores": threads,
                             "sample": "every pixel of the 256x256 frame, binary64 rtol 1e-10 atol 1e-12"}
    tol = frame_tolerance(G)
    runs = (("fp64_oracle_policy", G.ReferencePolicy.frame(G.Precision.FP64)),
            ("fp32", G.ReferencePolicy.frame(G.Precision.FP32, **tol)),
            ("mixed", G.ReferencePolicy.frame(G.Precision.MIXED, **tol)),
            ("fp64", G.ReferencePolicy.frame(G.Precision.FP64, **tol)))
    for name, pol in runs:
        pipe.set_policy(pol)
        pipe.trace([sc], cam, res, stream=stream)
        ms = timed_trace(pipe, [sc], cam, res, stream, flush, reps=3)
        entry = {"ms": ms, "mrays_per_s": w * h / (ms / 1e3) / 1e6}
        if ref is not None:
            entry["error_vs_oracle"] = error_report(res.numpy(), ref, idx)
        out[name] = entry
    pipe.close()
    return out


def pinhole_rays(scene, sx, sy):
    """Initial states of pinhole rays through continuous image-plane points (sx, sy) (tangents along
    image-right and image-up): the trace kernels' ray set-up evaluated in numpy."""
    import numpy as np

    R, U, A = (np.array(v[:4]) for v in (scene.image_right, scene.image_up, scene.arrival))
    u = np.array(scene.four_velocity[:4])
    g = np.array(scene.metric_covariant[:16]).reshape(4, 4)
    nrm = 1.0 / np.hypot(1.0, np.hypot(sx, sy))
    sight = (np.outer(sx, R) + np.outer(sy, U) - A) * nrm[:, None]
    st = np.zeros((sx.size, 8))
    st[:, :4] = np.array(scene.observer_txyz[:4])
    st[:, 4:] = (scene.frequency * (u - sight)) @ g.T
    return st


def stress_study(G, device: int, cpu: bool, side: int = 4096) -> dict:
    """Near-critical stress: a = 0.998, Q = 0.05, i = 85 deg, observer on the escape sphere at
    r = 1000 M. The critical curve is located along 256 image directions by bisection of capture
    against escape with the binary64 kernel at the strict policy (no surface); side^2 rays are drawn
    with impact parameters uniform within +-0.05 M of it (seeded) and traced in each precision at the
    frame tolerance (CUDA events), once without the surface (capture/escape classes and equatorial
    crossings) and once with it (surface hits and g). With the CPU leg, 256 of them are traced by the
    binary64 oracle at rtol 1e-12: class and crossing mismatches and the g error, with the distance
    from the curve of every mismatch."""
    import numpy as np
    import torch

    a, q, incl, r_obs, band = 0.998, 0.05, math.radians(85.0), 1000.0, 0.05
    isco = G.prograde_isco(a, q)

    def observation(surface):
        return G.Observation.from_oblate(r_obs, incl, 0.0, spin=a, charge=q, chart=G.KerrSchildChart.OUTGOING,
                                         width=64, height=64, vertical_fov=math.radians(FOV_DEG),
                                         escape_radius=r_obs, surface=G.EquatorialSurface(isco, SURFACE_OUTER)
                                         if surface else None, horizon_offset=HORIZON_OFFSET)

    pipe = G.TracePipeline(device)
    sky = observation(False)
    sc = sky.pack()
    pipe.set_policy(G.ReferencePolicy.strict_v1())
    n_dirs = 256
    psi = np.linspace(0.0, 2 * np.pi, n_dirs, endpoint=False)
    lo, hi = np.zeros(n_dirs), np.full(n_dirs, 12.0 / r_obs)
    for _ in range(40):
        mid = 0.5 * (lo + hi)
        d = pipe.trace_states(sky, pinhole_rays(sc, mid * np.cos(psi), mid * np.sin(psi))).numpy()
        cap = d["termination"] == G.Termination.HORIZON_CROSSING
        lo, hi = np.where(cap, mid, lo), np.where(cap, hi, mid)
    rc = 0.5 * (lo + hi)
    n = side * side
    rng = np.random.default_rng(3)
    k = rng.integers(0, n_dirs, n)
    rho = rc[k] + rng.uniform(-1.0, 1.0, n) * band / r_obs
    dist = (rho - rc[k]) * r_obs
    out = {"workload": f"kerr-newman-near-critical-{side}x{side}", "spin": a, "charge": q, "inclination_deg": 85.0,
           "observer_radius_m": r_obs, "band_m": band,
           "policy": "frame (FP32 rtol 1e-6, MIXED 7e-7), FP64 at rtol 1e-6"}
    stream = torch.cuda.current_stream()
    sample = np.sort(rng.choice(n, 256, replace=False))
    tol = frame_tolerance(G)
    # the sky variant probes the capture/escape boundary and the windings; the disk variant the
    # surface hits (almost every ray of the band ends on the disk at this inclination)
    for variant, surface in (("sky", False), ("disk", True)):
        obs = observation(surface)
        states = pinhole_rays(obs.pack(), rho * np.cos(psi[k]), rho * np.sin(psi[k]))
        dev_states = torch.as_tensor(states).to(f"cuda:{device}")
        cam = [G.raylist_camera(0, dev_states.data_ptr(), n, -1.0)]
        res = G.TraceResults(n, f"cuda:{device}")
        ref = None
        vo = {}
        if cpu:
            import oracle as O

            ev = O.events(escape_radius=r_obs, surface=(isco, SURFACE_OUTER) if surface else None,
                          horizon_offset=HORIZON_OFFSET)
            t0 = time.perf_counter()
            ref = O.trace_states(1.0, a, q, 1, O.custom_policy(1e-12, 1e-14), ev, states[sample], -1.0,
                                 threads=O.hardware_threads())
            vo["cpu_oracle_s"] = time.perf_counter() - t0
        for name, prec in (("fp32", G.Precision.FP32), ("mixed", G.Precision.MIXED), ("fp64", G.Precision.FP64)):
            pipe.set_policy(G.ReferencePolicy.frame(prec, **tol))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            pipe.trace([obs.packed], cam, res, stream=stream)
            e1.record(stream)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1)
            d = res.numpy()
            entry = {"ms": ms, "mrays_per_s": n / (ms / 1e3) / 1e6,
                     "attempts_per_ray": float((d["accepted_steps"] + d["rejected_steps"]).mean()),
                     "class_histogram": np.bincount(d["termination"], minlength=9).tolist(),
                     "max_equatorial_crossings": int(d["equatorial_crossings"].max())}
            if ref is not None:
                import oracle as O

                F = O.F
                ot = ref[:, F["termination"]].astype(int)
                cls = d["termination"][sample] != ot
                wind = (~cls) & (d["equatorial_crossings"][sample] != ref[:, F["equatorial_crossings"]])
                g_rel = None
                srf = np.flatnonzero((~cls) & (ot == 7))
                if srf.size:
                    # the oracle's surface observable at its own hit state (surface.rs:12-146)
                    g_ref = np.array([O.surface_observable(1.0, a, q, 1, isco, SURFACE_OUTER,
                                                           ref[i, F["t"]:F["p_z"] + 1])[1][2] for i in srf])
                    ok = np.isfinite(g_ref) & np.isfinite(d["frequency_ratio"][sample][srf])
                    if ok.any():
                        g_rel = float(np.max(np.abs(d["frequency_ratio"][sample][srf][ok] - g_ref[ok]) / g_ref[ok]))
                entry["oracle_sample"] = {
                    "rays": int(sample.size), "class_mismatch": int(cls.sum()), "crossing_mismatch": int(wind.sum()),
                    "mismatch_distance_m": [float(x) for x in np.sort(np.abs(dist[sample][cls | wind]))],
                    "g_rel": g_rel}
            vo[name] = entry
        out[variant] = vo
        del res, dev_states
    pipe.close()
    return out


def adjoint_study(G, args, device: int) -> dict:
    """Discrete adjoint throughput on the differentiation workload: 1024x1024 rays, a = 0.9, Q = 0.3,
    i = 60 deg, r_obs = 50 M, MIXED forward. The loss is the sum of squared g and hit-radius residuals
    against a target frame traced at (a, Q, i) offset by seeded N(0, 0.01) draws; one step is
    glc_forward_ckpt_into + glc_backward on one reused tape (no allocation inside a step), timed
    with CUDA events, best of three steps, for each checkpoint interval K."""
    import numpy as np
    import torch

    n = args.adjoint_side
    a, q, incl, r_obs = 0.9, 0.3, math.radians(60.0), 50.0
    isco = G.prograde_isco(a, q)

    def obs_at(a_, q_, i_):
        return G.Observation.from_oblate(r_obs, i_, 0.0, spin=a_, charge=q_, chart=G.KerrSchildChart.OUTGOING,
                                         width=n, height=n, vertical_fov=math.radians(FOV_DEG),
                                         escape_radius=ESCAPE, surface=G.EquatorialSurface(isco, SURFACE_OUTER),
                                         horizon_offset=HORIZON_OFFSET)

    rng = np.random.default_rng(5)
    da, dq, di = rng.normal(0.0, 0.01, 3)
    pipe = G.TracePipeline(device, G.ReferencePolicy.frame(G.Precision.MIXED))
    target = pipe.trace_image(obs_at(a + da, q + dq, incl + di))
    torch.cuda.synchronize()
    tgt = target.numpy()
    obs = obs_at(a, q, incl)
    stream = torch.cuda.current_stream()
    out = {"workload": f"kerr-newman-adjoint-{n}x{n}", "spin": a, "charge": q, "inclination_deg": 60.0,
           "observer_radius_m": r_obs, "forward_precision": "mixed", "backward_precision": "f32 stage products, f64 stage points and sums",
           "target_offsets": [float(da), float(dq), float(di)], "by_K": {}}
    for K in args.adjoint_k:
        # one tape per K, reused by every step (glc_forward_ckpt_into): the steps allocate nothing
        res, tape = pipe.forward_ckpt(obs, r_obs, incl, K=K)
        dl_dev = torch.zeros((n * n, 4), dtype=torch.float64, device=f"cuda:{device}")
        tape.backward(dl_dev, per_ray_params=False)
        torch.cuda.synchronize()
        times = []
        for it in range(3):
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record(stream)
            tape.forward_again(results=res)
            e1.record(stream)
            d = res.numpy()
            both = (d["termination"] == 7) & (tgt["termination"] == 7)
            dl = np.zeros((n * n, 4))
            dl[both, 0] = 2.0 * (d["source_radius"][both] - tgt["source_radius"][both])
            dl[both, 1] = 2.0 * (d["frequency_ratio"][both] - tgt["frequency_ratio"][both])
            dl_dev.copy_(torch.as_tensor(dl))
            torch.cuda.synchronize()
            e1b = torch.cuda.Event(enable_timing=True)
            e1b.record(stream)
            g = tape.backward(dl_dev, per_ray_params=False)
            e2.record(stream)
            torch.cuda.synchronize()
            fwd, bwd = e0.elapsed_time(e1), e1b.elapsed_time(e2)
            times.append((fwd, bwd))
            info = tape.info()
            grad = g["params"].cpu().numpy().tolist()
        tape.close()
        fwd, bwd = min(t[0] for t in times), min(t[1] for t in times)
        loss = float(((d["source_radius"][both] - tgt["source_radius"][both]) ** 2).sum() +
                     ((d["frequency_ratio"][both] - tgt["frequency_ratio"][both]) ** 2).sum())
        out["by_K"][str(K)] = {"forward_ckpt_ms": fwd, "backward_ms": bwd,
                               "mrays_per_s": n * n / ((fwd + bwd) / 1e3) / 1e6,
                               "checkpoint_slots": info["checkpoint_slots"], "tape_bytes": info["bytes"],
                               "loss": loss, "dL_d(a,Q,i,r_obs)": grad}
    out["mrays_per_s"] = max(v["mrays_per_s"] for v in out["by_K"].values())
    pipe.close()
    return out


def ctypes_sizeof_job() -> int:
    from gravlume_b200 import _native as N
    import ctypes

    return ctypes.sizeof(N.Scene) + ctypes.sizeof(N.Camera) + 16


def main() -> None:
    global WIDTH, HEIGHT
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["fp32", "mixed", "fp64"], default="mixed")
    ap.add_argument("--no-compare", dest="compare", action="store_false")
    ap.add_argument("--autotune", action="store_true")
    ap.add_argument("--persistent", action="store_true",
                    help="trace the frame with the persistent work-queue kernel instead of one thread per ray")
    ap.add_argument("--no-adjoint", dest="adjoint", action="store_false",
                    help="skip the discrete-adjoint throughput study (1024x1024, K = 16, 64, 256)")
    ap.add_argument("--adjoint-side", type=int, default=1024)
    ap.add_argument("--no-sweep", dest="sweep", action="store_false",
                    help="skip the tolerance sweep of the precision study")
    ap.add_argument("--no-footprint", dest="footprint", action="store_false",
                    help="skip the surface-footprint study")
    ap.add_argument("--no-scenes", dest="scenes", action="store_false",
                    help="skip the 256x256 and the 15-scene full-frame precision studies")
    ap.add_argument("--no-stress", dest="stress", action="store_false",
                    help="skip the near-critical stress study")
    ap.add_argument("--stress-side", type=int, default=4096, help="the stress study traces side^2 rays")
    ap.add_argument("--no-batch", dest="batch", action="store_false",
                    help="skip the 64-scene batch study (persistent launch, graph, autotuner)")
    ap.add_argument("--adjoint-k", type=int, nargs="+", default=[16, 64, 256])
    ap.add_argument("--cpu-sample", type=int, default=2048,
                    help="pixels of the frame traced by the CPU oracle (baseline and error report)")
    ap.add_argument("--traffic-bytes", type=float, default=None,
                    help="DRAM bytes per launch from an ncu capture, reported as roofline.traffic")
    ap.add_argument("--scaling", choices=["weak", "strong"], default="weak",
                    help="weak: a frame per rank; strong: the ranks split one frame into tile-row bands")
    ap.add_argument("--studies-out", default=None,
                    help="also write the headline and every study to this JSON file")
    ap.add_argument("--width", type=int, default=WIDTH, help="frame width (smaller frames for profiling)")
    ap.add_argument("--height", type=int, default=HEIGHT, help="frame height")
    args = ap.parse_args()
    WIDTH, HEIGHT = args.width, args.height
    if args.impl == "reference":
        run_reference(args)
    else:
        run_gpu(args)


if __name__ == "__main__":
    main()
