"""Benchmark of the field-convolution hot path on B200.

Default workload (one "step"): the filter-bank pair of a CNN layer in cct-core
form, on one batch of synthetic fields --
  y  = blockReduceSum(projectFrame(x, f, BorderZero, batchSize=16), 32)
  dx = blockReduceSum(backProjectFrame(g, f, BorderZero, batchSize=16), 64)
x: 64x64 VectorField of 16*32 planes ~ N(0,1); f: 64 filters of 5x5x32,
He-normal (std sqrt(2/800)); g: 64x64 of 16*64 planes ~ N(0,1).
2 x 6.711 GFLOP per step (2*B*H*W*K*C*R*S each way).

Other workloads (--workload): plain (256x256 (*) 5x5, BorderZero, batched
over 4096 planes for the HBM roofline), separable.

Prints one JSON line (rank 0).  Multi-GPU: replicas only -- every rank runs
the same step on its own GPU; value = all ranks' work / max rank time.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "cct-core_b200"))

GFLOP_FRAME = 2 * 16 * 64 * 64 * 64 * 32 * 5 * 5 / 1e9  # 6.711 per direction


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["frame", "plain", "separable"], default="frame")
    ap.add_argument("--precision", choices=["auto", "fp32", "bf16x3"], default="auto")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    return ap.parse_args()


# ----------------------------------------------------------------------------- dist
def dist_setup(n):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local))
        pg = dist
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return rank, world, local, pg


def barrier(pg):
    import torch
    if pg is not None:
        pg.barrier()
    torch.cuda.synchronize()


def max_over_ranks(pg, value):
    import torch
    if pg is None:
        return value
    t = torch.tensor([value], device="cuda", dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


# ----------------------------------------------------------------------------- clocks
class ClockSampler:
    """nvidia-smi sampling of SM clock and throttle reasons during timing."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.dev = device_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        time.sleep(1.0)  # let nvidia-smi start sampling before the timed region
        return self

    def __exit__(self, *exc):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                self.out, _ = self.proc.communicate()

    def summary(self):
        rows = []
        for line in (self.out or "").strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                rows.append((float(parts[1]), float(parts[2]), parts[5:9]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for _, _, flags in rows for i, v in enumerate(flags)
                          if v.lower() == "active"})
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": rows[0][1],
                "reasons": reasons, "samples": len(rows)}


# ----------------------------------------------------------------------------- workloads
def frame_workload(precision):
    """Build the projectFrame/backProjectFrame pair; returns a dict of callables."""
    import torch
    import cctconv as C
    from cctconv import _lib

    B, Cin, K, H, W, R = 16, 32, 64, 64, 64, 5
    prec = {"fp32": _lib.PREC_FP32, "bf16x3": _lib.PREC_BF16X3}
    if precision == "auto":
        try:
            _lib.Plan(C.make_desc((H, W, B * Cin), (R, R, K * Cin), C.BorderZero,
                                  _lib.CROSS_CORRELATION, C.NoSamplingConvolution,
                                  _lib.PROJECT_FRAME_BLOCK_REDUCE_SUM, B, _lib.PREC_BF16X3)).close()
            precision = "bf16x3"
        except _lib.CctError:
            precision = "fp32"
    p = prec[precision]
    fwd = _lib.Plan(C.make_desc((H, W, B * Cin), (R, R, K * Cin), C.BorderZero,
                                _lib.CROSS_CORRELATION, C.NoSamplingConvolution,
                                _lib.PROJECT_FRAME_BLOCK_REDUCE_SUM, B, p))
    bwd = _lib.Plan(C.make_desc((H, W, B * K), (R, R, K * Cin), C.BorderZero,
                                _lib.CONVOLUTION, C.NoSamplingConvolution,
                                _lib.BACK_PROJECT_FRAME_BLOCK_REDUCE_SUM, B, p))
    gen = torch.Generator(device="cuda").manual_seed(2)
    sets = 6  # 6 x 48 MB of fields > 126 MB L2: no step finds its inputs in L2
    xs = [torch.randn((B * Cin, H, W), device="cuda", generator=gen) for _ in range(sets)]
    gs = [torch.randn((B * K, H, W), device="cuda", generator=gen) for _ in range(sets)]
    ys = [torch.empty((B * K, H, W), device="cuda") for _ in range(sets)]
    dxs = [torch.empty((B * Cin, H, W), device="cuda") for _ in range(sets)]
    f = torch.randn((K * Cin, R, R), device="cuda", generator=gen) * (2.0 / 800) ** 0.5
    stream = torch.cuda.current_stream().cuda_stream
    state = {"i": 0}

    def step():
        i = state["i"] % sets
        state["i"] += 1
        fwd.run(xs[i].data_ptr(), f.data_ptr(), ys[i].data_ptr(), stream)
        bwd.run(gs[i].data_ptr(), f.data_ptr(), dxs[i].data_ptr(), stream)

    # host-buffer end-to-end step through the C-ABI (pinned host memory)
    hx = xs[0].cpu().pin_memory()
    hg = gs[0].cpu().pin_memory()
    hf = f.cpu().pin_memory()
    hy = torch.empty((B * K, H, W)).pin_memory()
    hdx = torch.empty((B * Cin, H, W)).pin_memory()

    def e2e_step():
        fwd.run_host(hx.data_ptr(), hf.data_ptr(), hy.data_ptr(), stream)
        bwd.run_host(hg.data_ptr(), hf.data_ptr(), hdx.data_ptr(), stream)

    nbytes = lambda t: t.numel() * 4  # noqa: E731
    return {
        "step": step, "e2e_step": e2e_step,
        "launch_single": lambda: fwd.run(xs[0].data_ptr(), f.data_ptr(), ys[0].data_ptr(), stream),
        "gflop_per_step": 2 * GFLOP_FRAME, "gflop_per_launch": GFLOP_FRAME,
        "h2d": nbytes(hx) + nbytes(hg) + 2 * nbytes(hf), "d2h": nbytes(hy) + nbytes(hdx),
        "metric": "GFLOP/s", "unit": "GFLOP/s", "precision": precision, "plan_algo": fwd.algo,
        "config": {"workload": "projectFrame+backProjectFrame (BlockReduceSum fused), B=16 C=32 "
                               "K=64 64x64 5x5 BorderZero", "B": B, "C": Cin, "K": K, "H": H, "W": W,
                   "R": R, "border": "BorderZero", "l2": "6 rotating input/output sets (288 MB > 126 MB L2)"},
        "dtype": "f32" if precision == "fp32" else "bf16x3 split, f32 accumulate",
        "keep": (fwd, bwd, xs, gs, ys, dxs, f, hx, hg, hf, hy, hdx),
        "kernel": "frame_f32_kernel" if precision == "fp32" else "frame_tc_kernel",
        "bytes_per_launch": 4 * (B * Cin * H * W + K * Cin * R * R + B * K * H * W),
    }


def plain_workload():
    import torch
    import cctconv as C
    from cctconv import _lib

    P, H, W, R = 4096, 256, 256, 5
    plan = _lib.Plan(C.make_desc((H, W, P), (R, R, 0), C.BorderZero, _lib.CONVOLUTION,
                                 C.NoSamplingConvolution, _lib.PLANE_BY_PLANE))
    gen = torch.Generator(device="cuda").manual_seed(1)
    x = torch.empty((P, H, W), device="cuda").uniform_(-1, 1, generator=gen)
    y = torch.empty_like(x)
    f = torch.empty((R, R), device="cuda").uniform_(-1, 1, generator=gen)
    stream = torch.cuda.current_stream().cuda_stream

    def step():
        plan.run(x.data_ptr(), f.data_ptr(), y.data_ptr(), stream)

    hx = x[:64].cpu().pin_memory()  # e2e on a 64-plane slice through run_host
    hy = torch.empty_like(hx).pin_memory()
    hf = f.cpu().pin_memory()
    plan64 = _lib.Plan(C.make_desc((H, W, 64), (R, R, 0), C.BorderZero, _lib.CONVOLUTION,
                                   C.NoSamplingConvolution, _lib.PLANE_BY_PLANE))

    def e2e_step():
        plan64.run_host(hx.data_ptr(), hf.data_ptr(), hy.data_ptr(), stream)

    byts = 4 * (2 * P * H * W + R * R)
    return {
        "step": step, "e2e_step": e2e_step, "launch_single": step,
        "gflop_per_step": 2 * P * H * W * R * R / 1e9, "gflop_per_launch": 2 * P * H * W * R * R / 1e9,
        "bytes_per_step": byts, "e2e_gb_per_step": 4 * (2 * 64 * H * W + R * R) / 1e9,
        "h2d": 4 * (64 * H * W + R * R), "d2h": 4 * 64 * H * W,
        "metric": "GB/s", "unit": "GB/s", "precision": "fp32", "plan_algo": plan.algo,
        "config": {"workload": "plain convolve 256x256 (*) 5x5 BorderZero, 4096 planes per launch",
                   "planes": P, "H": H, "W": W, "R": R, "l2": "1 GiB input > 126 MB L2"},
        "dtype": "f32", "keep": (plan, plan64, x, y, f, hx, hy, hf),
        "kernel": "direct_tma_kernel", "bytes_per_launch": byts,
    }


# ----------------------------------------------------------------------------- timing
def time_steps(fn, steps, warmup, pg):
    """W untimed steps, then K steps between CUDA events, bracketed by a
    barrier + device synchronise.  Returns (seconds, native launches in K)."""
    import torch
    from cctconv import _lib
    for _ in range(warmup):
        fn()
    barrier(pg)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n0 = _lib.launch_count()
    start.record()
    for _ in range(steps):
        fn()
    end.record()
    barrier(pg)
    return start.elapsed_time(end) / 1e3, _lib.launch_count() - n0


def time_single_launch(fn, reps=20, rounds=5):
    """Average device time of one launch of the dominant kernel: `reps`
    launches back to back between two CUDA events on the launching stream
    (so host-side launch latency is not counted), median over rounds."""
    import torch
    for _ in range(3):
        fn()
    torch.cuda.synchronize()
    times = []
    for _ in range(rounds):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(reps):
            fn()
        b.record()
        b.synchronize()
        times.append(a.elapsed_time(b) / 1e3 / reps)
    return statistics.median(times)


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def load_traffic(kernel):
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        return json.loads(p.read_text()).get(kernel)
    return None


# ----------------------------------------------------------------------------- cpu arm
def cpu_frame_sample(seconds_budget=10.0):
    """Oracle (FP32 restatement of the reference kernel loop) on one image of
    the batch, forward + backward, all host threads.  Returns (GFLOP/s,
    threads, sample description)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import numpy as np
    import oracle as O
    rng = np.random.default_rng(2)
    Cin, K, H, W, R = 32, 64, 64, 64, 5
    x = rng.standard_normal((Cin, H, W)).astype(np.float32)
    g = rng.standard_normal((K, H, W)).astype(np.float32)
    f = (rng.standard_normal((K * Cin, R, R)) * np.sqrt(2 / 800)).astype(np.float32)
    fd = O.make_desc(H, W, R, R, planes=Cin, f_planes=K * Cin, batch=1, border=O.ZERO,
                     orient=O.XCORR, mode=O.PROJECT_REDUCE)
    bd = O.make_desc(H, W, R, R, planes=K, f_planes=K * Cin, batch=1, border=O.ZERO,
                     orient=O.CONV, mode=O.BACKPROJECT_REDUCE)
    threads = os.cpu_count() or 1
    O.conv(fd, x, f, threads=threads)  # warm
    gflop = 2 * GFLOP_FRAME / 16
    reps, t0 = 0, time.perf_counter()
    while True:
        O.conv(fd, x, f, threads=threads)
        O.conv(bd, g, f, threads=threads)
        reps += 1
        el = time.perf_counter() - t0
        if el > seconds_budget or reps >= 200:
            break
    return gflop * reps / el, threads, f"{reps} x (fwd+bwd of 1 of 16 images), {el:.1f} s"


def cpu_plain_sample(seconds_budget=10.0):
    sys.path.insert(0, str(ROOT / "oracle"))
    import numpy as np
    import oracle as O
    rng = np.random.default_rng(1)
    P, H, W, R = 64, 256, 256, 5
    x = rng.uniform(-1, 1, (P, H, W)).astype(np.float32)
    f = rng.uniform(-1, 1, (R, R)).astype(np.float32)
    d = O.make_desc(H, W, R, R, planes=P, border=O.ZERO, orient=O.CONV)
    threads = os.cpu_count() or 1
    reps, t0 = 0, time.perf_counter()
    while True:
        O.conv(d, x, f, threads=threads)
        reps += 1
        el = time.perf_counter() - t0
        if el > seconds_budget or reps >= 200:
            break
    gb = 4 * (2 * P * H * W + R * R) / 1e9
    return gb * reps / el, threads, f"{reps} x 64 planes of 256x256, {el:.1f} s"


# ----------------------------------------------------------------------------- main
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    fn = cpu_frame_sample if args.workload == "frame" else cpu_plain_sample
    per = []
    for _ in range(max(args.warmup, 0)):
        fn(seconds_budget=1.0)
    for _ in range(args.steps):
        v, threads, sample = fn(seconds_budget=2.0)
        per.append(v)
    value = statistics.median(per)
    unit = "GFLOP/s" if args.workload == "frame" else "GB/s"
    cfg = {"workload": "projectFrame+backProjectFrame (BlockReduceSum fused), B=16 C=32 K=64 64x64 "
                       "5x5 BorderZero" if args.workload == "frame" else
                       "plain convolve 256x256 (*) 5x5 BorderZero"}
    line = {"impl": "reference", "metric": unit, "value": round(value, 3), "unit": unit,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded)", "config": cfg,
            "cpu_baseline": {"value": round(value, 3), "unit": unit, "cores": threads, "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(value, 3), "unit": unit, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": "cct-core is Scala/OpenCL (no JVM or CPU OpenCL runtime here); its "
                    "ConvolveHyperKernel loop is timed as the C restatement in oracle/"}
    print(json.dumps(line), flush=True)
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import torch
    from cctconv import _lib

    rank, world, local, pg = dist_setup(args.gpus)
    wl = frame_workload(args.precision) if args.workload == "frame" else plain_workload()
    peaks, peak_kind = load_peaks()

    with ClockSampler(torch.cuda.current_device()) as clocks:
        elapsed, launches = time_steps(wl["step"], args.steps, args.warmup, pg)
    t_max = max_over_ranks(pg, elapsed)

    per_launch = time_single_launch(wl["launch_single"])
    e2e_t, _ = time_steps(wl["e2e_step"], max(args.steps // 20, 3), 2, pg)
    e2e_t = max_over_ranks(pg, e2e_t)
    e2e_steps = max(args.steps // 20, 3)

    if wl["unit"] == "GFLOP/s":
        value = world * wl["gflop_per_step"] * args.steps / t_max
        e2e_val = world * wl["gflop_per_step"] * e2e_steps / e2e_t
        achieved = wl["gflop_per_launch"] / per_launch / 1e3  # TFLOP/s
        if wl["precision"] == "bf16x3":
            bound, peak, unit = "tensor", peaks["bf16_tflops"], "TFLOP/s"
        else:
            # CUDA-core FP32: 148 SMs x 128 FMA/clk x 2 at the max SM clock
            bound, unit = "fp32_simt", "TFLOP/s"
            peak = 148 * 128 * 2 * peaks.get("sm_max_mhz", 1965.0) / 1e6
    else:
        value = world * wl["bytes_per_step"] * args.steps / t_max / 1e9
        e2e_val = world * wl["e2e_gb_per_step"] * e2e_steps / e2e_t
        achieved = wl["bytes_per_launch"] / per_launch / 1e9
        bound, peak, unit = "hbm", peaks["hbm_gbs"], "GB/s"

    if rank != 0:
        if pg is not None:
            pg.destroy_process_group()
        return 0
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        fn = cpu_frame_sample if wl["unit"] == "GFLOP/s" else cpu_plain_sample
        v, threads, sample = fn(seconds_budget=10.0)
        cpu = {"value": round(v, 3), "unit": wl["unit"], "cores": threads, "kind": "port",
               "sample": sample}
    traffic = load_traffic(wl["kernel"])
    line = {
        "metric": wl["metric"], "value": round(value, 3), "unit": wl["unit"], "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * t_max / args.steps, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": wl["dtype"],
        "data": "synthetic (seeded)", "config": dict(wl["config"], parallelism=f"replicas{world}"),
        "roofline": {"bound": bound, "achieved": round(achieved, 3), "peak": round(peak, 1),
                     "unit": unit, "frac": round(achieved / peak, 4), "traffic": traffic,
                     "peak_source": peak_kind if bound != "fp32_simt" else "nominal FP32 at sm_max_mhz",
                     "kernel": wl["kernel"], "launch_ms": round(per_launch * 1e3, 4)},
        "cpu_baseline": cpu,
        "e2e": {"value": round(e2e_val, 3), "unit": wl["unit"], "h2d_bytes_per_step": wl["h2d"],
                "d2h_bytes_per_step": wl["d2h"]},
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
        "plan_algo": wl["plan_algo"],
    }
    print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
