"""Benchmark of the field-convolution hot path on B200.

Default workload (one "step"): the filter-bank pair of a CNN layer in cct-core
form, on one batch of synthetic fields --
  y  = blockReduceSum(projectFrame(x, f, BorderZero, batchSize=16), 32)
  dx = blockReduceSum(backProjectFrame(g, f, BorderZero, batchSize=16), 64)
x: 64x64 VectorField of 16*32 planes ~ N(0,1); f: 64 filters of 5x5x32,
He-normal (std sqrt(2/800)); g: 64x64 of 16*64 planes ~ N(0,1).
2 x 6.711 GFLOP per step (2*B*H*W*K*C*R*S each way).

Other workloads (--workload): plain (256x256 (*) 5x5, BorderZero, batched
over 4096 planes for the HBM roofline); fft (2048x2048 uniform[0,1] (*) 63x63
normalised Gaussian, sigma 10, BorderCyclic, through the FFT path, with its
max/RMS error against an FP64 FFT and the direct kernel's time beside it);
graph (the eight-layer 3x3 stack on 224x224x3, widths 64..512, stepped as
one captured launch sequence; batch 64 headline, batches 1 and 8 and FP32
beside it); serve (10,000 seeded convolve/projectFrame requests of uneven
sizes with Poisson arrivals, served with continuous batching and with plain
per-call dispatch: throughput and p50/p99 latency, rate swept 1k-50k/s).

Beside the headline each line carries: max/RMS error against an FP64
reference (error_vs_fp64), and per workload the neighbouring operators --
frame: the same layer's weight gradient (FilterAdjointBlockReduceSum, FP32 and
split BF16); plain: one 256x256 plane alone, the separable form, a
ScalarField (*) MatrixField and a ColorField convolution; fft: the direct
kernel and a dynamic filter; graph: batches 1, 8 and 64 in both precisions.

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
    ap.add_argument("--workload", choices=["frame", "plain", "fft", "graph", "serve"], default="frame")
    ap.add_argument("--precision", choices=["auto", "fp32", "bf16x3", "bf16x6"], default="auto")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-suite", action="store_true",
                    help="headline workload only (no sub-results for the other workloads)")
    ap.add_argument("--serve-requests", type=int, default=10000)
    ap.add_argument("--serve-rate", type=float, default=2000.0)
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
    """The slowest rank's time: every rank takes the same all-reduce."""
    import torch
    if pg is None:
        return value
    dev = "cuda" if pg.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], device=dev, dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def replica_value(units_per_rank, world, t_max):
    """Whole-job rate of N identical replicas: all ranks' units over the
    slowest rank's time."""
    return world * units_per_rank / t_max


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


# ----------------------------------------------------------------------------- configs
# One config dict per workload, printed identically by the GPU arm and the
# reference (CPU) arm, so both lines name the same workload.
def frame_config():
    return {"workload": "projectFrame+backProjectFrame (BlockReduceSum fused), B=16 C=32 "
                        "K=64 64x64 5x5 BorderZero", "B": 16, "C": 32, "K": 64, "H": 64, "W": 64,
            "R": 5, "border": "BorderZero", "l2": "6 rotating input/output sets (288 MB > 126 MB L2)"}


def plain_config():
    return {"workload": "plain convolve 256x256 (*) 5x5 BorderZero, 4096 planes per launch",
            "planes": 4096, "H": 256, "W": 256, "R": 5, "l2": "1 GiB input > 126 MB L2"}


def fft_config():
    return {"workload": "FFT convolve 2048x2048 uniform[0,1] (*) 63x63 normalised Gaussian "
                        "(sigma 10), BorderCyclic, static filter",
            "H": 2048, "W": 2048, "R": 63, "border": "BorderCyclic",
            "flops": "direct-equivalent 2*H*W*R*S per convolution",
            "l2": "8 rotating image/output sets (268 MB > 126 MB L2)"}


def graph_config(batch=64):
    return {"workload": "eight-layer 3x3 stack on 224x224x3 (widths 64,64,128,128,256,256,512,512; "
                        "DownsampleOutput(2) after layers 2,4,6; ReLU between layers), "
                        f"batch {batch}, one CUDA-graph replay per step",
            "batch": batch, "layers": 8, "gflop_per_step": round(12.196 * batch, 2),
            "l2": "activations of batch 64 (1.2 GB per step) exceed the 126 MB L2"}


CONFIGS = {"frame": frame_config, "plain": plain_config, "fft": fft_config, "graph": graph_config}


# ----------------------------------------------------------------------------- workloads
def errors_vs(y, ref):
    """Normwise max and RMS relative error of y against an FP64 reference."""
    import numpy as np
    d = np.asarray(y, np.float64) - ref
    return {"max_rel": float(np.abs(d).max() / np.abs(ref).max()),
            "rms_rel": float(np.sqrt((d * d).mean() / (ref * ref).mean()))}


def np_conv_same(x, f, flip):
    """FP64 zero-border 'same' filter bank in numpy (the accuracy reference the
    bench reports against; the tests check against the oracle):
    y[k, i, j] = sum_{c, r, s} x[c, i + r - h, j + s - h] * f'[k, c, r, s],
    f' = f flipped in r and s when `flip`."""
    import numpy as np
    C, H, W = x.shape
    K, _, R, S = f.shape
    h = (R - 1) // 2
    xp = np.pad(x.astype(np.float64), ((0, 0), (h, h), (h, h)))
    f = f.astype(np.float64)
    if flip:
        f = f[:, :, ::-1, ::-1]
    y = np.zeros((K, H * W))
    for r in range(R):
        for s in range(S):
            y += f[:, :, r, s] @ xp[:, r:r + H, s:s + W].reshape(C, -1)
    return y.reshape(K, H, W)


def frame_workload(precision):
    """Build the projectFrame/backProjectFrame pair; returns a dict of callables."""
    import torch
    import cctconv as C
    from cctconv import _lib

    B, Cin, K, H, W, R = 16, 32, 64, 64, 64, 5
    prec = {"fp32": _lib.PREC_FP32, "bf16x3": _lib.PREC_BF16X3, "bf16x6": _lib.PREC_BF16X6}
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

    # End to end through the C-ABI with host buffers, two steps in flight:
    # step k copies its inputs in, runs forward and backward and copies both
    # results out on stream k % 2 with buffer set k % 2, so one step's copies
    # overlap the other's (the two copy directions run on separate engines).
    streams = [torch.cuda.current_stream(), torch.cuda.Stream()]
    dsets = [dict(x=torch.empty_like(xs[0]), g=torch.empty_like(gs[0]), f=torch.empty_like(f),
                  y=torch.empty_like(ys[0]), dx=torch.empty_like(dxs[0])) for _ in range(2)]
    houts = [(hy, hdx), (torch.empty_like(hy).pin_memory(), torch.empty_like(hdx).pin_memory())]
    e2e_state = {"k": 0}

    def h2d(dst, src, s):
        _lib.check(_lib.LIB.cct_memcpy_h2d(dst.data_ptr(), src.data_ptr(), src.numel() * 4, s.cuda_stream))

    def d2h(dst, src, s):
        _lib.check(_lib.LIB.cct_memcpy_d2h(dst.data_ptr(), src.data_ptr(), src.numel() * 4, s.cuda_stream))

    def e2e_step():
        k = e2e_state["k"] % 2
        e2e_state["k"] += 1
        s, d, (oy, odx) = streams[k], dsets[k], houts[k]
        h2d(d["x"], hx, s)
        h2d(d["f"], hf, s)
        h2d(d["g"], hg, s)
        fwd.run(d["x"].data_ptr(), d["f"].data_ptr(), d["y"].data_ptr(), s.cuda_stream)
        bwd.run(d["g"].data_ptr(), d["f"].data_ptr(), d["dx"].data_ptr(), s.cuda_stream)
        d2h(oy, d["y"], s)
        d2h(odx, d["dx"], s)

    def e2e_begin():  # the side stream starts after the timed region opens
        streams[1].wait_stream(streams[0])

    def e2e_finish():  # the timed region closes after both streams drain
        streams[0].wait_stream(streams[1])

    def weight_gradient():
        """FilterAdjointBlockReduceSum beside the step: the 5x5 filter gradient
        of the same layer (the image zero-padded to 68x68, the 64x64 output
        gradient as the 'filter'), FP32 and split BF16, with the BF16 error
        against the FP32 kernel's result in FP64."""
        out = {}
        xa = torch.randn((B * Cin, H + R - 1, W + R - 1), device="cuda", generator=gen)
        ga = torch.randn((B * K, H, W), device="cuda", generator=gen)
        ys_ = {}
        for name, pr in (("fp32", _lib.PREC_FP32), ("bf16x3", _lib.PREC_BF16X3)):
            pl = _lib.Plan(C.make_desc((H + R - 1, W + R - 1, B * Cin), (H, W, B * K), C.BorderValid,
                                       _lib.CROSS_CORRELATION, C.NoSamplingConvolution,
                                       _lib.FILTER_ADJOINT_BLOCK_REDUCE_SUM, B, pr))
            yo = torch.empty((K * Cin, R, R), device="cuda")
            t = time_single_launch(lambda: pl.run(xa.data_ptr(), ga.data_ptr(), yo.data_ptr(), stream), reps=10)
            out[name] = {"ms": round(t * 1e3, 4), "GFLOP/s": round(GFLOP_FRAME / t, 1), "plan_algo": pl.algo}
            ys_[name] = yo.double().cpu().numpy()
            pl.close()
        out["bf16x3_vs_fp32"] = errors_vs(ys_["bf16x3"], ys_["fp32"])
        return out

    def frame_errors():
        """Image 0 of one forward and one backward step against FP64 numpy."""
        step()
        torch.cuda.synchronize()
        fn = f.double().cpu().numpy().reshape(K, Cin, R, R)
        fwd_ref = np_conv_same(xs[0][:Cin].double().cpu().numpy(), fn, flip=False)
        bwd_ref = np_conv_same(gs[0][:K].double().cpu().numpy(), fn.transpose(1, 0, 2, 3), flip=True)
        return {"projectFrame": errors_vs(ys[0][:K].cpu().numpy(), fwd_ref),
                "backProjectFrame": errors_vs(dxs[0][:Cin].cpu().numpy(), bwd_ref),
                "sample": "image 0 of the batch"}

    nbytes = lambda t: t.numel() * 4  # noqa: E731
    return {
        "step": step, "e2e_step": e2e_step, "e2e_begin": e2e_begin, "e2e_finish": e2e_finish,
        # both launches of the step (forward 32 -> 64 planes, backward 64 -> 32:
        # the same filter-bank kernel, 6.711 GFLOP each), each with its filter pack
        "launch_single": lambda: (fwd.run(xs[0].data_ptr(), f.data_ptr(), ys[0].data_ptr(), stream),
                                  bwd.run(gs[0].data_ptr(), f.data_ptr(), dxs[0].data_ptr(), stream)),
        "launches_per_single": 2,
        "gflop_per_step": 2 * GFLOP_FRAME, "gflop_per_launch": GFLOP_FRAME,
        "h2d": nbytes(hx) + nbytes(hg) + nbytes(hf), "d2h": nbytes(hy) + nbytes(hdx),
        "metric": "GFLOP/s", "unit": "GFLOP/s", "precision": precision, "plan_algo": fwd.algo,
        "config": frame_config(),
        "dtype": {"fp32": "f32", "bf16x6": "bf16x6 (three-term bf16 split), f32 accumulate"}.get(
            precision, "bf16x3 split, f32 accumulate"),
        "keep": (fwd, bwd, xs, gs, ys, dxs, f, hx, hg, hf, hy, hdx),
        # evaluated after the timed region, so the step launches come first in a launch list
        "extra": lambda: {"error_vs_fp64": frame_errors(), "weight_gradient_5x5": weight_gradient()},
        # the step's kernel: forward and backward launches (the filter-bank kernel)
        "kernel": "frame_f32_kernel" if precision == "fp32" else "bank_tc_kernel",
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

    # beside it: the single 256x256 plane (L2-resident, launch-bound) and the
    # separable form on the same 4096 planes (both passes fused per tile: one
    # read of the field and one write of the result)
    import ctypes
    one = _lib.Plan(C.make_desc((H, W, 0), (R, R, 0), C.BorderZero, _lib.CONVOLUTION,
                                C.NoSamplingConvolution, _lib.PLANE_BY_PLANE))
    single_s = time_single_launch(lambda: one.run(x.data_ptr(), f.data_ptr(), y.data_ptr(), stream),
                                  reps=100)
    rf = torch.empty(R, device="cuda").uniform_(-1, 1, generator=gen)
    cf = torch.empty(R, device="cuda").uniform_(-1, 1, generator=gen)
    tmp = torch.empty_like(x)

    def separable():
        _lib.check(_lib.LIB.cct_conv_separable(H, W, P, x.data_ptr(), rf.data_ptr(), R, cf.data_ptr(), R,
                                               _lib.BORDER_ZERO, _lib.CONVOLUTION, tmp.data_ptr(),
                                               y.data_ptr(), ctypes.c_void_p(stream)))
    sep_s = time_single_launch(separable, reps=10)

    def other_ops():
        """The other convolution operators beside the batched convolve: a
        1024x1024 ScalarField cross-correlated with an 8x8 MatrixField of 7x7
        matrices (64 output planes), and a 2048x2048 ColorField (RGBA8)
        convolved with a 5x5 filter (unpack, three planes, pack)."""
        sm_x = torch.empty((1024, 1024), device="cuda").uniform_(-1, 1, generator=gen)
        sm_m = torch.empty((7, 7, 8, 8), device="cuda").uniform_(-1, 1, generator=gen)
        sm_y = torch.empty((64, 1024, 1024), device="cuda")

        def scalar_matrix():
            _lib.check(_lib.LIB.cct_conv_scalar_matrix(1024, 1024, sm_x.data_ptr(), sm_m.data_ptr(), 8, 8, 7,
                                                       _lib.BORDER_ZERO, _lib.CROSS_CORRELATION,
                                                       _lib.SAMPLE_NONE, 1, sm_y.data_ptr(),
                                                       ctypes.c_void_p(stream)))
        t_sm = time_single_launch(scalar_matrix, reps=10)
        img = torch.randint(0, 256, (2048, 2048, 4), dtype=torch.uint8, device="cuda", generator=gen)
        out = torch.empty_like(img)
        cplan = _lib.ColorPlan(C.make_desc((2048, 2048, 0), (5, 5, 0), C.BorderZero, _lib.CONVOLUTION,
                                           C.NoSamplingConvolution, _lib.PLANE_BY_PLANE))
        cf = torch.empty((5, 5), device="cuda").uniform_(0, 0.08, generator=gen)
        t_c = time_single_launch(lambda: cplan.run(img.data_ptr(), cf.data_ptr(), out.data_ptr(), stream), reps=10)
        cplan.close()
        return {"ms": round(t_sm * 1e3, 4), "GFLOP/s": round(2 * 1024 * 1024 * 64 * 49 / t_sm / 1e9, 1),
                "color": {"ms": round(t_c * 1e3, 4),
                          "pixels/s": round(2048 * 2048 / t_c, 1)}}
    def unfused_frame():
        """projectFrame without the block reduce (CogFunctionAPI.scala:1370-1377):
        B=4 images of C=32 planes, 64 filters of 5x5x32, every (image, filter
        plane) pair an output plane: 8192 planes of 64x64 from 128 input
        planes, on the FP32 frame kernel without its reduce; HBM-bound on the output."""
        Bu, Cu, Ku, Hu, Wu, Ru = 4, 32, 64, 64, 64, 5
        pl = _lib.Plan(C.make_desc((Hu, Wu, Bu * Cu), (Ru, Ru, Ku * Cu), C.BorderZero, _lib.CROSS_CORRELATION,
                                   C.NoSamplingConvolution, _lib.PROJECT_FRAME, Bu))
        xu = torch.empty((Bu * Cu, Hu, Wu), device="cuda").uniform_(-1, 1, generator=gen)
        fu = torch.empty((Ku * Cu, Ru, Ru), device="cuda").uniform_(-1, 1, generator=gen)
        yu = torch.empty((Bu * Ku * Cu, Hu, Wu), device="cuda")
        t = time_single_launch(lambda: pl.run(xu.data_ptr(), fu.data_ptr(), yu.data_ptr(), stream), reps=10)
        byts = 4 * (xu.numel() + fu.numel() + yu.numel())
        torch.cuda.synchronize()
        ref = np_conv_same(xu[:1].double().cpu().numpy(), fu[:1].double().cpu().numpy()[:, None], flip=False)
        err = errors_vs(yu[:1].cpu().numpy(), ref)
        algo = pl.algo
        pl.close()
        return {"ms": round(t * 1e3, 4), "GB/s": round(byts / t / 1e9, 1),
                "hbm_frac": round(byts / t / 1e9 / load_peaks()[0]["hbm_gbs"], 4), "plan_algo": algo,
                "error_vs_fp64": dict(err, sample="output plane 0")}
    sep_bytes = 2 * 4 * P * H * W
    step()
    torch.cuda.synchronize()
    ref = np_conv_same(x[:1].double().cpu().numpy(), f.double().cpu().numpy()[None, None], flip=True)
    extra = {"error_vs_fp64": dict(errors_vs(y[:1].cpu().numpy(), ref), sample="plane 0"),
             "single_plane_256x256_us": round(single_s * 1e6, 2),
             "separable_5+5_4096x256x256": {"ms": round(sep_s * 1e3, 4),
                                            "GB/s": round(sep_bytes / sep_s / 1e9, 1)},
             "scalar_matrix_1024x1024_8x8_of_7x7": other_ops(),
             "project_frame_unfused_4x32x64_64x64_5x5": unfused_frame()}
    extra["color_2048x2048_5x5"] = extra["scalar_matrix_1024x1024_8x8_of_7x7"].pop("color")

    byts = 4 * (2 * P * H * W + R * R)
    return {
        "step": step, "e2e_step": e2e_step, "launch_single": step, "extra": extra,
        "gflop_per_step": 2 * P * H * W * R * R / 1e9, "gflop_per_launch": 2 * P * H * W * R * R / 1e9,
        "bytes_per_step": byts, "e2e_gb_per_step": 4 * (2 * 64 * H * W + R * R) / 1e9,
        "h2d": 4 * (64 * H * W + R * R), "d2h": 4 * 64 * H * W,
        "metric": "GB/s", "unit": "GB/s", "precision": "fp32", "plan_algo": plan.algo,
        "config": plain_config(),
        "dtype": "f32", "keep": (plan, plan64, one, x, y, f, hx, hy, hf, rf, cf, tmp),
        "kernel": "direct_tma_kernel", "bytes_per_launch": byts,
    }


def gaussian_filter(k=63, sigma=10.0):
    import numpy as np
    r = np.arange(k) - k // 2
    g = np.exp(-(r[:, None] ** 2 + r[None, :] ** 2) / (2 * sigma * sigma))
    return (g / g.sum()).astype(np.float32)


def fft_workload():
    """2048x2048 uniform[0,1] ScalarField (*) 63x63 normalised Gaussian,
    BorderCyclic.  The Gaussian is a constant filter, so its spectrum is made
    once on the host in FP64 (static filter), as the reference does for
    constant filters; each step transforms one image and inverts."""
    import numpy as np
    import torch
    import cctconv as C
    from cctconv import _lib

    n, k = 2048, 63
    f_host = gaussian_filter(k)
    mk = lambda algo: _lib.Plan(C.make_desc((n, n, 0), (k, k, 0), C.BorderCyclic,  # noqa: E731
                                            _lib.CONVOLUTION, C.NoSamplingConvolution,
                                            _lib.PLANE_BY_PLANE, algo=algo))
    plan = mk(_lib.ALGO_FFT)
    plan.set_static_filter(f_host.ctypes.data)
    gen = torch.Generator(device="cuda").manual_seed(3)
    sets = 8  # 8 x 33.5 MB of images and outputs > 126 MB L2
    xs = [torch.empty((n, n), device="cuda").uniform_(0, 1, generator=gen) for _ in range(sets)]
    ys = [torch.empty((n, n), device="cuda") for _ in range(sets)]
    stream = torch.cuda.current_stream().cuda_stream
    state = {"i": 0}

    def step():
        i = state["i"] % sets
        state["i"] += 1
        plan.run(xs[i].data_ptr(), 0, ys[i].data_ptr(), stream)

    # error of the FFT path against an FP64 FFT of the same cyclic convolution
    step()
    torch.cuda.synchronize()
    x64 = xs[0].double().cpu().numpy()
    g = np.zeros((n, n))
    h = k // 2
    for r in range(k):
        for s in range(k):
            g[(r - h) % n, (s - h) % n] += f_host[r, s]
    ref = np.real(np.fft.ifft2(np.fft.fft2(x64) * np.fft.fft2(g)))
    d = ys[0].double().cpu().numpy() - ref
    err = {"max_rel": float(np.abs(d).max() / np.abs(ref).max()),
           "rms_rel": float(np.sqrt((d * d).mean() / (ref * ref).mean()))}

    # the direct kernel on the same convolution, beside it
    direct = mk(_lib.ALGO_DIRECT)
    fd = torch.from_numpy(f_host).cuda()
    yd = torch.empty((n, n), device="cuda")
    direct_s = time_single_launch(lambda: direct.run(xs[0].data_ptr(), fd.data_ptr(),
                                                     yd.data_ptr(), stream), reps=3, rounds=3)
    torch.cuda.synchronize()
    dd = yd.double().cpu().numpy() - ref
    err["direct_max_rel"] = float(np.abs(dd).max() / np.abs(ref).max())
    # dynamic filter: the filter spectrum is made on the device every run
    dyn = mk(_lib.ALGO_FFT)
    dyn_s = time_single_launch(lambda: dyn.run(xs[0].data_ptr(), fd.data_ptr(), yd.data_ptr(),
                                               stream))

    hx = xs[0].cpu().pin_memory()
    hy = torch.empty((n, n)).pin_memory()

    def e2e_step():
        plan.run_host(hx.data_ptr(), 0, hy.data_ptr(), stream)

    gflop = 2.0 * n * n * k * k / 1e9  # direct-equivalent work of one convolution
    return {
        "step": step, "e2e_step": e2e_step, "launch_single": step,
        "gflop_per_step": gflop, "gflop_per_launch": gflop,
        # HBM bytes a run must move: the image in, the filter spectrum in, the result out
        "bytes_per_step": 4 * n * n * 2 + 8 * n * (n // 2 + 1),
        "bytes_per_launch": 4 * n * n * 2 + 8 * n * (n // 2 + 1),
        "e2e_gb_per_step": None, "h2d": 4 * n * n, "d2h": 4 * n * n,
        "metric": "GFLOP/s", "unit": "GFLOP/s", "precision": "fp32", "plan_algo": plan.algo,
        "config": fft_config(),
        "dtype": "f32", "keep": (plan, direct, dyn, xs, ys, fd, yd, hx, hy),
        "kernel": "fft_rows_r2c+fft_cols+fft_rows_c2r", "fft_hbm_roofline": True,
        "extra": {"error_vs_fp64": err, "direct_ms": round(direct_s * 1e3, 4),
                  "dynamic_filter_ms": round(dyn_s * 1e3, 4)},
    }


def graph_workload(precision):
    """The eight-layer stack (224x224x3 input, 3x3 filters, widths 64, 64,
    128, 128, 256, 256, 512, 512, DownsampleOutput(2) on layers 2, 4 and 6,
    ReLU between layers) stepped as a ComputeGraph: each step one replay of
    the captured launches.  Inputs uniform[-1,1], He-normal filters."""
    import numpy as np
    import torch
    from cctconv import _lib
    from cctconv.graph import eight_layer_stack

    # The split-precision stack runs the three-term split (BF16X6): the
    # two-term split keeps each layer within 1e-5 of FP64 but compounds to
    # about 1.4e-5 over the eight layers.
    prec = {"fp32": _lib.PREC_FP32, "bf16x3": _lib.PREC_BF16X3}.get(precision, _lib.PREC_BF16X6)

    def build(batch, p):
        st = eight_layer_stack(batch, p)
        rng = np.random.default_rng(4)
        fs = []
        for i, (kc, r, s_) in enumerate(st.filter_shapes):
            c = kc // (st.field_shapes[i + 1][0] // batch)
            fs.append((rng.standard_normal((kc, r, s_)) * np.sqrt(2.0 / (c * r * s_))).astype(np.float32))
        st.set_filters(fs)
        st.input.uniform_(-1, 1)
        st.bench_filters = fs
        return st

    B = 64
    stack = build(B, prec)
    stream = torch.cuda.current_stream().cuda_stream

    def step():
        stack.step(1, stream)

    def side(batch, p, steps=20):
        st = stack if (batch == B and p == prec) else build(batch, p)
        st.step(3, stream)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        st.step(steps, stream)
        b.record()
        b.synchronize()
        ms = a.elapsed_time(b) / steps
        out = {"ms_per_step": round(ms, 4), "GFLOP/s": round(st.flops_per_step / ms / 1e6, 1)}
        if st is not stack:
            st.close()
        return out

    extra = {"by_batch": {}}
    for p_name, p in (("bf16x6", _lib.PREC_BF16X6), ("bf16x3", _lib.PREC_BF16X3), ("fp32", _lib.PREC_FP32)):
        for b in (1, 8, 64):
            extra["by_batch"][f"{p_name}_b{b}"] = side(b, p)

    def graph_errors():
        """Image 0 of a batch-64 step against FP64 numpy (same-size zero-border
        layers, then the step-2 subsample, ReLU between layers): through all
        eight layers from the input (errors compound), and per layer from the
        GPU's own input to that layer."""
        stack.step(1, stream)
        torch.cuda.synchronize()
        widths = [64, 64, 128, 128, 256, 256, 512, 512]

        def layer(i, a):
            a = np_conv_same(a, stack.bench_filters[i].reshape(widths[i], a.shape[0], 3, 3), flip=False)
            if i in (1, 3, 5):
                a = a[:, ::2, ::2]
            return np.maximum(a, 0.0) if i < 7 else a

        a = stack.input[:3].double().cpu().numpy()
        per_layer = []
        for i in range(8):
            gin = stack.field(i)[:a.shape[0] if i == 0 else widths[i - 1]].double().cpu().numpy()
            gout = stack.field(i + 1)[:widths[i]].cpu().numpy()
            per_layer.append(errors_vs(gout, layer(i, gin))["max_rel"])
            a = layer(i, a)
        out = stack.field(len(stack.descs))[:512].cpu().numpy()
        return dict(errors_vs(out, a), per_layer_max_rel=per_layer,
                    sample="image 0; all eight layers from the input, and each layer from its GPU input")

    extra["error_vs_fp64"] = graph_errors()
    hx = stack.input.cpu().pin_memory()
    hy = torch.empty(stack.field_shapes[-1]).pin_memory()

    def e2e_step():
        stack.step_host(hx, hy, stream)

    gflop = stack.flops_per_step / 1e9
    # the dominant kernel: layer 8 (28x28, 512 -> 512), timed alone on its plan
    last = _lib.Plan(stack.descs[-1])
    lin = stack.field(len(stack.descs) - 1)
    lf = torch.randn(stack.filter_shapes[-1], device="cuda") * 0.02
    ly = torch.empty(stack.field_shapes[-1], device="cuda")
    if last.algo == _lib.PLAN_FRAME_BF16X3:
        lf_host = lf.cpu().numpy()  # held while the library copies from it
        last.set_static_filter(lf_host.ctypes.data)
        lf_ptr = 0
    else:
        lf_ptr = lf.data_ptr()
    d = stack.descs[-1]
    last_gflop = 2.0 * B * 512 * 28 * 28 * 512 * 9 / 1e9
    return {
        "step": step, "e2e_step": e2e_step,
        "launch_single": lambda: last.run(lin.data_ptr(), lf_ptr, ly.data_ptr(), stream),
        "gflop_per_step": gflop, "gflop_per_launch": last_gflop,
        "h2d": hx.numel() * 4, "d2h": hy.numel() * 4,
        "metric": "GFLOP/s", "unit": "GFLOP/s",
        "precision": {_lib.PREC_FP32: "fp32", _lib.PREC_BF16X3: "bf16x3"}.get(prec, "bf16x6"),
        "plan_algo": last.algo,
        "config": graph_config(B),
        "dtype": {_lib.PREC_FP32: "f32", _lib.PREC_BF16X3: "bf16x3 split, f32 accumulate"}.get(
            prec, "bf16x6 (three-term bf16 split), f32 accumulate"),
        "keep": (stack, last, lin, lf, ly, hx, hy),
        "kernel": "bank_tc_kernel (layer 8)" if prec != _lib.PREC_FP32 else "frame_f32_kernel (layer 8)",
        "extra": extra,
    }


def circuit_bench(steps=200):
    """A ComputeGraph that is a DAG, not a chain: two residual blocks
    (conv+ReLU, conv, add the block's input, ReLU) at B=16, 64 planes, 64x64,
    3x3, split BF16, stepped as one kernel circuit (a CUDA-graph replay over
    shared buffers) and, beside it, node by node from the host (each
    convolution through cct_conv_run, the adds and ReLUs as torch ops)."""
    import numpy as np
    import torch
    from cctconv import _lib
    from cctconv import circuit as K

    B, C, H, W = 16, 64, 64, 64
    d1 = _lib.new_desc(image_rows=H, image_cols=W, image_planes=B * C, filter_rows=3, filter_cols=3,
                       filter_planes=C * C, batch_size=B, orientation=_lib.CROSS_CORRELATION,
                       vector_mode=_lib.PROJECT_FRAME_BLOCK_REDUCE_SUM, precision=_lib.PREC_BF16X3,
                       flags=_lib.FLAG_RELU)
    d2 = _lib.new_desc(image_rows=H, image_cols=W, image_planes=B * C, filter_rows=3, filter_cols=3,
                       filter_planes=C * C, batch_size=B, orientation=_lib.CROSS_CORRELATION,
                       vector_mode=_lib.PROJECT_FRAME_BLOCK_REDUCE_SUM, precision=_lib.PREC_BF16X3)
    nodes = [K.conv(0, d1), K.conv(1, d2), K.add(2, 0), K.relu(3),
             K.conv(4, d1), K.conv(5, d2), K.add(6, 4), K.relu(7)]
    circ = K.Circuit([(H, W, B * C)], nodes, outputs=[8])
    rng = np.random.default_rng(6)
    fs = {i: (rng.standard_normal((C * C, 3, 3)) * np.sqrt(2.0 / (C * 9))).astype(np.float32) for i in (0, 1, 4, 5)}
    for i, f in fs.items():
        circ.set_filter(i, f)
    circ.field(0).uniform_(-1, 1)
    stream = torch.cuda.current_stream().cuda_stream
    gflop = 4 * 2.0 * B * C * H * W * C * 9 / 1e9

    def timed(fn, n):
        for _ in range(5):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(n):
            fn()
        b.record()
        b.synchronize()
        return a.elapsed_time(b) / n

    ms_circuit = timed(lambda: circ.step(1, stream), steps)
    # node by node from the host: the same plans and the same arithmetic
    plans = {i: _lib.Plan(nodes[i].conv) for i in (0, 1, 4, 5)}
    for i, pl in plans.items():
        pl.set_static_filter(fs[i].ctypes.data)
    x = circ.field(0).reshape(B * C, H, W).clone()
    t = [torch.empty_like(x) for _ in range(3)]

    def host_step():
        plans[0].run(x.data_ptr(), 0, t[0].data_ptr(), stream)
        plans[1].run(t[0].data_ptr(), 0, t[1].data_ptr(), stream)
        torch.clamp_min(t[1].add_(x), 0.0, out=t[2])
        plans[4].run(t[2].data_ptr(), 0, t[0].data_ptr(), stream)
        plans[5].run(t[0].data_ptr(), 0, t[1].data_ptr(), stream)
        torch.clamp_min(t[1].add_(t[2]), 0.0, out=t[0])

    ms_host = timed(host_step, steps)
    circ.step(1, stream)
    host_step()
    torch.cuda.synchronize()
    same = bool(torch.equal(circ.field(8).reshape(B * C, H, W), t[0]))
    nb, nbytes = circ.buffers()
    out = {"config": {"workload": f"2 residual blocks, B={B}, {C} planes, {H}x{W}, 3x3, BF16X3, 8 nodes"},
           "circuit_ms_per_step": round(ms_circuit, 4), "GFLOP/s": round(gflop / ms_circuit * 1e3, 1),
           "host_dispatch_ms_per_step": round(ms_host, 4), "same_result_bits": same,
           "buffers": nb, "fields": 1 + len(nodes), "buffer_MB": round(nbytes / 1e6, 1)}
    for pl in plans.values():
        pl.close()
    circ.close()
    return out


def serve_requests(n, seed=5):
    """n seeded request specs: side log-uniform in [32, 1024], filter size
    from {3,5,7,9}, planes from {1,4,16,64}, filters from {1,16,64}."""
    import numpy as np
    rng = np.random.default_rng(seed)
    side = np.exp(rng.uniform(np.log(32), np.log(1024), n)).astype(int)
    R = rng.choice([3, 5, 7, 9], n)
    C = rng.choice([1, 4, 16, 64], n)
    K = rng.choice([1, 16, 64], n)
    return [(int(a), int(b), int(c), int(d)) for a, b, c, d in zip(side, R, C, K)]


class ServeBench:
    """Continuous batching vs plain per-call dispatch on one seeded request
    stream: a shared pinned input pool (requests read its start), a ring of
    pinned output space, resident filter banks per (R, C, K)."""

    def __init__(self, n_requests):
        import numpy as np
        import torch
        self.rng = np.random.default_rng(5)
        self.specs = serve_requests(n_requests)
        max_in = max(s * s * c for s, r, c, k in self.specs)
        max_out = max(s * s * (c if k == 1 else k) for s, r, c, k in self.specs)
        self.pool = torch.from_numpy(self.rng.uniform(-1, 1, max_in).astype(np.float32)).pin_memory()
        self.ring_elems = max(4 * max_out, 1 << 29)
        self.ring = torch.empty(self.ring_elems).pin_memory()

    def build(self, server):
        from cctconv import _lib
        from cctconv.serve import conv_request
        banks, reqs, flops, hbytes = {}, [], 0.0, 0
        pos = 0
        for side, R, C, K in self.specs:
            key = (R, C, K)
            if key not in banks:
                fp = 1 if K == 1 else K * C
                banks[key] = server.add_filter(self.rng.uniform(-1, 1, (fp, R, R)).astype("float32"))
            if K == 1:
                d = _lib.new_desc(image_rows=side, image_cols=side, image_planes=C if C > 1 else 0,
                                  filter_rows=R, filter_cols=R, filter_planes=0,
                                  orientation=_lib.CONVOLUTION, vector_mode=_lib.PLANE_BY_PLANE)
                planes = C
            else:
                d = _lib.new_desc(image_rows=side, image_cols=side, image_planes=C, filter_rows=R,
                                  filter_cols=R, filter_planes=K * C, orientation=_lib.CROSS_CORRELATION,
                                  vector_mode=_lib.PROJECT_FRAME_BLOCK_REDUCE_SUM)
                planes = K
            out = side * side * planes
            if pos + out > self.ring_elems:
                pos = 0
            reqs.append(conv_request(d, self.pool.data_ptr(), self.ring.data_ptr() + 4 * pos, None, banks[key]))
            pos += (out + 63) // 64 * 64
            flops += 2.0 * side * side * planes * R * R * (C if K > 1 else 1)
            hbytes += 4 * side * side * (C + planes)
        return reqs, flops, hbytes

    def run(self, per_call, rate, n):
        import numpy as np
        from cctconv.serve import Server
        server = Server(slots=4, max_batch=64, per_call=per_call)  # admission by free HBM
        reqs, flops, hbytes = self.build(server)
        reqs, k = reqs[:n], n / len(reqs)
        arrivals = np.cumsum(np.random.default_rng(int(rate)).exponential(1.0 / rate, n))
        t0 = time.perf_counter()
        lat = server.replay(reqs, arrivals)
        wall = time.perf_counter() - t0
        st = server.stats()
        server.close()
        return {"rate": rate, "requests": n, "served_per_s": round(n / wall, 1),
                "p50_ms": round(float(np.percentile(lat, 50)) / 1e3, 3),
                "p99_ms": round(float(np.percentile(lat, 99)) / 1e3, 3),
                "GFLOP/s": round(flops * k / wall / 1e9, 1), "host_GB/s": round(hbytes * k / wall / 1e9, 2),
                "batches": st["batches"], "solo": st["solo"]}


SERVE_CONFIG = ("Poisson arrivals, side log-uniform 32-1024, R {3,5,7,9}, planes {1,4,16,64}, "
                "filters {1,16,64}, FP32 host I/O, resident filter banks")


def serve_suite(args, rates=(1000.0, 5000.0), n=2000):
    """The serving loop beside the headline: batched and per-call dispatch at
    two arrival rates on the first n requests of the seeded stream, with the
    clocks sampled while they run."""
    import torch
    sb = ServeBench(n)
    out = {"config": {"workload": f"{n} requests per rate, " + SERVE_CONFIG}, "rates": []}
    with ClockSampler(torch.cuda.current_device()) as clocks:
        for rate in rates:
            out["rates"].append({"batched": sb.run(False, rate, n), "per_call": sb.run(True, rate, n)})
    out["clocks"] = clocks.summary()
    return out


def run_serve(args):
    """Continuous batching vs plain per-call dispatch on the same request
    stream (rank 0 only; every rank serves its own stream under torchrun)."""
    rank, world, local, pg = dist_setup(args.gpus)
    sb = ServeBench(args.serve_requests)
    head = sb.run(False, args.serve_rate, args.serve_requests)
    base = sb.run(True, args.serve_rate, min(args.serve_requests, 3000))
    sweep = []
    for rate in (1000.0, 2000.0, 5000.0, 10000.0, 20000.0, 50000.0):
        n = min(args.serve_requests, 1500)
        sweep.append({"batched": sb.run(False, rate, n), "per_call": sb.run(True, rate, n)})
    if rank != 0:
        if pg is not None:
            pg.destroy_process_group()
        return 0
    line = {
        "metric": "served requests/s", "value": round(head["served_per_s"] * world, 1), "unit": "req/s",
        "n_gpus": world, "steps": args.serve_requests, "warmup": 0,
        "ms_per_step": round(1e3 / head["served_per_s"], 4), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
        "config": {"workload": f"{args.serve_requests} requests at {args.serve_rate:g}/s, " + SERVE_CONFIG,
                   "parallelism": f"replicas{world}"},
        "latency": {"p50_ms": head["p50_ms"], "p99_ms": head["p99_ms"]},
        "per_call": base, "batched": head, "sweep": sweep,
        "e2e": {"value": round(head["served_per_s"] * world, 1), "unit": "req/s",
                "h2d_bytes_per_step": None, "d2h_bytes_per_step": None},
        "gpu_launches": int(head["batches"] + head["solo"]),
    }
    print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()
    return 0


# ----------------------------------------------------------------------------- timing
def time_steps(fn, steps, warmup, pg, begin=None, finish=None):
    """W untimed steps, then K steps between CUDA events, bracketed by a
    barrier + device synchronise.  begin/finish join any side stream the
    steps use to the timed region.  Returns (seconds, native launches in K)."""
    import torch
    from cctconv import _lib
    for _ in range(warmup):
        fn()
    barrier(pg)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n0 = _lib.launch_count()
    start.record()
    if begin:
        begin()
    for _ in range(steps):
        fn()
    if finish:
        finish()
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
def _timed_reps(run, seconds_budget, max_reps):
    """Run `run` until seconds_budget has passed (at least once); (reps, seconds)."""
    reps, t0 = 0, time.perf_counter()
    while True:
        run()
        reps += 1
        el = time.perf_counter() - t0
        if el > seconds_budget or reps >= max_reps:
            return reps, el


def _band(full, scale, least=1):
    return max(least, min(full, int(round(full * scale))))


def cpu_frame_sample(seconds_budget=10.0, scale=1.0):
    """Oracle (FP32 restatement of the reference kernel loop) on one image of
    the batch, forward + backward, all host threads; `scale` < 1 takes a band
    of the image's rows (the same work per output).  Returns (GFLOP/s,
    threads, sample description)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import numpy as np
    import oracle as O
    rng = np.random.default_rng(2)
    Cin, K, W, R = 32, 64, 64, 5
    H = _band(64, scale, 2)
    x = rng.standard_normal((Cin, H, W)).astype(np.float32)
    g = rng.standard_normal((K, H, W)).astype(np.float32)
    f = (rng.standard_normal((K * Cin, R, R)) * np.sqrt(2 / 800)).astype(np.float32)
    fd = O.make_desc(H, W, R, R, planes=Cin, f_planes=K * Cin, batch=1, border=O.ZERO,
                     orient=O.XCORR, mode=O.PROJECT_REDUCE)
    bd = O.make_desc(H, W, R, R, planes=K, f_planes=K * Cin, batch=1, border=O.ZERO,
                     orient=O.CONV, mode=O.BACKPROJECT_REDUCE)
    threads = os.cpu_count() or 1
    gflop = 2 * (2 * K * Cin * H * W * R * R) / 1e9

    def run():
        O.conv(fd, x, f, threads=threads)
        O.conv(bd, g, f, threads=threads)
    reps, el = _timed_reps(run, seconds_budget, 200)
    return gflop * reps / el, threads, f"{reps} x (fwd+bwd of {H} of 64 rows of 1 of 16 images), {el:.2f} s"


def cpu_plain_sample(seconds_budget=10.0, scale=1.0):
    sys.path.insert(0, str(ROOT / "oracle"))
    import numpy as np
    import oracle as O
    rng = np.random.default_rng(1)
    H, W, R = 256, 256, 5
    P = _band(64, scale)
    x = rng.uniform(-1, 1, (P, H, W)).astype(np.float32)
    f = rng.uniform(-1, 1, (R, R)).astype(np.float32)
    d = O.make_desc(H, W, R, R, planes=P, border=O.ZERO, orient=O.CONV)
    threads = os.cpu_count() or 1
    reps, el = _timed_reps(lambda: O.conv(d, x, f, threads=threads), seconds_budget, 200)
    gb = 4 * (2 * P * H * W + R * R) / 1e9
    return gb * reps / el, threads, f"{reps} x {P} planes of 256x256, {el:.2f} s"


def cpu_fft_sample(seconds_budget=10.0, scale=1.0):
    """Oracle direct convolution (the reference's loop order, FP32) of a
    band of output rows of the 2048x2048 (*) 63x63 cyclic case, all host
    threads.  GFLOP/s in the same direct-equivalent flops as the GPU line."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import numpy as np
    import oracle as O
    n, k = 2048, 63
    band = _band(64, scale)
    rng = np.random.default_rng(3)
    # every output point costs R*S multiply-adds whatever the border, so a
    # (band + 62) x 2048 cyclic field stands in for a band of the full field
    x = rng.uniform(0, 1, (band + k - 1, n)).astype(np.float32)
    f = gaussian_filter(k)
    d = O.make_desc(band + k - 1, n, k, k, border=O.CYCLIC, orient=O.CONV)
    threads = os.cpu_count() or 1
    reps, el = _timed_reps(lambda: O.conv(d, x, f, threads=threads), seconds_budget, 50)
    gflop = 2.0 * (band + k - 1) * n * k * k / 1e9
    return gflop * reps / el, threads, f"{reps} x ({band + k - 1}x{n} (*) {k}x{k} cyclic), {el:.2f} s"


def cpu_graph_sample(seconds_budget=10.0, scale=1.0):
    """Oracle FP32 projectFrameBlockReduceSum of layer 8 of the stack (28x28,
    512 -> 512 planes, 3x3) for one sample (or a band of its rows), all
    host threads."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import numpy as np
    import oracle as O
    rng = np.random.default_rng(5)
    C = K = 512
    W = 28
    H = _band(28, scale)
    x = rng.uniform(-1, 1, (C, H, W)).astype(np.float32)
    f = (rng.standard_normal((K * C, 3, 3)) * np.sqrt(2 / (C * 9))).astype(np.float32)
    d = O.make_desc(H, W, 3, 3, planes=C, f_planes=K * C, batch=1, border=O.ZERO, orient=O.XCORR,
                    mode=O.PROJECT_REDUCE)
    threads = os.cpu_count() or 1
    reps, el = _timed_reps(lambda: O.conv(d, x, f, threads=threads), seconds_budget, 100)
    gflop = 2.0 * K * C * H * W * 9 / 1e9
    return gflop * reps / el, threads, f"{reps} x layer 8 of one sample ({H} of 28 rows, 512->512, 3x3), {el:.2f} s"


# ----------------------------------------------------------------------------- main
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.workload == "serve":
        print(json.dumps({"impl": "reference", "unavailable": "cct-core has no request-serving path; "
                          "the serve line reports plain per-call dispatch beside batching"}), flush=True)
        return 0
    fn = {"frame": cpu_frame_sample, "plain": cpu_plain_sample, "fft": cpu_fft_sample,
          "graph": cpu_graph_sample}[args.workload]
    # The whole run stays within about two minutes: at most 40 timed samples
    # (the median is reported), each given an equal share of the budget; a
    # sample that would overrun its share shrinks to a band of the workload
    # (the same work per output).
    samples = max(1, min(args.steps, 40))
    step_budget = min(2.0, 100.0 / samples)
    t0 = time.perf_counter()
    fn(seconds_budget=0.0)
    unit = time.perf_counter() - t0
    scale = min(1.0, step_budget / max(unit, 1e-9))
    per = []
    for _ in range(min(max(args.warmup, 0), 3)):
        fn(seconds_budget=0.0, scale=scale)
    for _ in range(samples):
        v, threads, sample = fn(seconds_budget=step_budget, scale=scale)
        per.append(v)
    value = statistics.median(per)
    sample = f"median of {samples} samples, last: {sample}"
    unit = "GB/s" if args.workload == "plain" else "GFLOP/s"
    # the same config dict as the GPU arm's line for this workload
    cfg = dict(CONFIGS[args.workload](), parallelism=f"replicas{args.gpus}")
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


def measure(wl, steps, warmup, pg, world, peaks, peak_kind):
    """Device-timed value, dominant-kernel roofline, end-to-end rate and
    clocks of one workload: W untimed steps, K timed steps between CUDA
    events (max over ranks), the dominant kernel timed alone, then the same
    step through the C-ABI with host buffers (copies inside the timed
    region)."""
    import torch
    with ClockSampler(torch.cuda.current_device()) as clocks:
        elapsed, launches = time_steps(wl["step"], steps, warmup, pg)
    t_max = max_over_ranks(pg, elapsed)
    per_launch = time_single_launch(wl["launch_single"]) / wl.get("launches_per_single", 1)
    e2e_steps = max(steps // 20, 3)
    e2e_t, _ = time_steps(wl["e2e_step"], e2e_steps, 2, pg, wl.get("e2e_begin"), wl.get("e2e_finish"))
    e2e_t = max_over_ranks(pg, e2e_t)

    if wl.get("fft_hbm_roofline"):
        # FFT: reported in direct-equivalent GFLOP/s; its roofline is HBM
        value = replica_value(wl["gflop_per_step"] * steps, world, t_max)
        e2e_val = replica_value(wl["gflop_per_step"] * e2e_steps, world, e2e_t)
        achieved = wl["bytes_per_launch"] / per_launch / 1e9
        bound, peak, unit = "hbm", peaks["hbm_gbs"], "GB/s"
    elif wl["unit"] == "GFLOP/s":
        value = replica_value(wl["gflop_per_step"] * steps, world, t_max)
        e2e_val = replica_value(wl["gflop_per_step"] * e2e_steps, world, e2e_t)
        achieved = wl["gflop_per_launch"] / per_launch / 1e3  # TFLOP/s
        if wl["precision"] in ("bf16x3", "bf16x6"):
            bound, peak, unit = "tensor", peaks["bf16_tflops"], "TFLOP/s"
        else:
            # CUDA-core FP32: 148 SMs x 128 FMA/clk x 2 at the max SM clock
            bound, unit = "fp32_simt", "TFLOP/s"
            peak = 148 * 128 * 2 * peaks.get("sm_max_mhz", 1965.0) / 1e6
    else:
        value = replica_value(wl["bytes_per_step"] * steps, world, t_max) / 1e9
        e2e_val = replica_value(wl["e2e_gb_per_step"] * e2e_steps, world, e2e_t)
        achieved = wl["bytes_per_launch"] / per_launch / 1e9
        bound, peak, unit = "hbm", peaks["hbm_gbs"], "GB/s"
    return {
        "metric": wl["metric"], "value": round(value, 3), "unit": wl["unit"],
        "steps": steps, "warmup": warmup, "ms_per_step": round(1e3 * t_max / steps, 4),
        "dtype": wl["dtype"], "config": dict(wl["config"], parallelism=f"replicas{world}"),
        "roofline": {"bound": bound, "achieved": round(achieved, 3), "peak": round(peak, 1),
                     "unit": unit, "frac": round(achieved / peak, 4), "traffic": load_traffic(wl["kernel"]),
                     "peak_source": peak_kind if bound != "fp32_simt" else "nominal FP32 at sm_max_mhz",
                     "kernel": wl["kernel"], "launch_ms": round(per_launch * 1e3, 4)},
        "e2e": {"value": round(e2e_val, 3), "unit": wl["unit"], "h2d_bytes_per_step": wl["h2d"],
                "d2h_bytes_per_step": wl["d2h"]},
        "gpu_launches": int(launches),
        "clocks": clocks.summary(),
        "plan_algo": wl["plan_algo"],
    }


def sub_result(build, steps, warmup, pg, world, peaks, peak_kind):
    """One workload measured beside the headline, with its extras (errors
    against FP64, neighbouring operators); its device memory is released
    before the next one."""
    import gc
    import torch
    wl = build()
    out = measure(wl, steps, warmup, pg, world, peaks, peak_kind)
    extra = wl.get("extra", {})
    out.update(extra() if callable(extra) else extra)
    del wl
    gc.collect()
    torch.cuda.synchronize()
    torch.cuda.empty_cache()
    return out


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "serve":
        return run_serve(args)
    import torch

    rank, world, local, pg = dist_setup(args.gpus)
    wl = {"frame": lambda: frame_workload(args.precision), "plain": plain_workload,
          "fft": fft_workload, "graph": lambda: graph_workload(args.precision)}[args.workload]()
    peaks, peak_kind = load_peaks()
    head = measure(wl, args.steps, args.warmup, pg, world, peaks, peak_kind)

    extra = wl.get("extra", {})
    extra = extra() if callable(extra) else extra
    suite = {}
    if args.workload == "frame" and world == 1 and not args.no_suite:
        # Every other workload, driver-timed in the same run (one GPU): the
        # plain FP32 filter bank on the same step (the denominator of the
        # split-BF16 speed-up), the memory-bound plane convolution, the FFT
        # path, the eight-layer stack and the serving loop.
        del wl
        sub_steps, sub_warm = max(args.steps, 10), max(args.warmup, 3)
        fp32 = sub_result(lambda: frame_workload("fp32"), sub_steps, sub_warm, pg, world, peaks, peak_kind)
        fp32.pop("weight_gradient_5x5", None)
        suite["frame_fp32"] = fp32
        if head["dtype"] != fp32["dtype"]:
            suite["frame_fp32"]["split_bf16_speedup"] = round(head["value"] / fp32["value"], 3)
        suite["plain_convolve"] = sub_result(plain_workload, sub_steps, sub_warm, pg, world, peaks, peak_kind)
        suite["fft_convolve"] = sub_result(fft_workload, sub_steps, sub_warm, pg, world, peaks, peak_kind)
        suite["graph_stack"] = sub_result(lambda: graph_workload(args.precision), max(args.steps // 2, 5),
                                          sub_warm, pg, world, peaks, peak_kind)
        suite["circuit_residual"] = circuit_bench()
        suite["serving"] = serve_suite(args)

    if rank != 0:
        if pg is not None:
            pg.destroy_process_group()
        return 0
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        fn = {"frame": cpu_frame_sample, "plain": cpu_plain_sample,
              "fft": cpu_fft_sample, "graph": cpu_graph_sample}[args.workload]
        v, threads, sample = fn(seconds_budget=10.0)
        cpu = {"value": round(v, 3), "unit": head["unit"], "cores": threads, "kind": "port",
               "sample": sample}
    line = {
        "metric": head["metric"], "value": head["value"], "unit": head["unit"], "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": head["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": head["dtype"],
        "data": "synthetic (seeded)", "config": head["config"],
        "roofline": head["roofline"], "cpu_baseline": cpu, "e2e": head["e2e"],
        "gpu_launches": head["gpu_launches"], "clocks": head["clocks"], "plan_algo": head["plan_algo"],
    }
    line.update(extra)
    line.update(suite)
    print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
