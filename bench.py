#!/usr/bin/env python
"""bench.py -- SAR backprojection throughput on B200 (Gpixel*pulses/s).

Workload (default): plain_large -- one 2048 x 2048 image from 1999 pulses x
1024 samples (complex64), N_fft 4096, Taylor 30, seeded synthetic data with
the reference's shapes (see halide-sar-app_b200/sarbp_b200/synth.py).

A step is one backprojection call of the reference's `backprojection_cuda`
interface: range compression (window, filter, pad, shift, FFT, shift) and
per-pixel pulse accumulation into the complex128 image, all on the device.
  value  inputs resident in HBM (sarbp_backprojection_device), K steps timed
         with CUDA events on the launching stream; per-step inputs plus
         outputs are ~250 MB, larger than the 126 MB L2
  e2e    the host-buffer entry point (sarbp_backprojection) from pinned
         host memory: host->device copies of phs, k_r, pos, r and the
         device->host copy of the image inside the timed region

Multi-GPU (torchrun, N > 1): every rank forms its own image (replicas, weak
scaling); the time is the max over ranks.

Other configurations (own JSON line each): --config batch96 (the batched
form), --config serve (the serving sweep), --config cli_sandia (the sarbp
CLI end to end with the reference's one-node Sandia command line, beside the
stage times of that run's log), --config streamed (a 4096^2 x 4000 image
formed in pulse chunks under a device-memory cap), --config resize (the
data/resize.py resampling on the device beside its scipy restatement),
--config distributed (the row-block schedule with its NCCL gather), and any
synth configuration name.

--impl reference times the reference algorithm's CPU implementation (the
C restatement in oracle/, reference precision, all host threads) on a
bounded pixel sample of the same workload; only rank 0 runs it.
"""
import argparse
import json
import os
import math
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "halide-sar-app_b200"))

FP32_PER_UNIT = 18  # FP32-pipe instructions per pixel*pulse (algorithmic)
SFU_PER_UNIT = 3    # SFU operations per pixel*pulse (algorithmic)
U8_LAUNCHES = 50    # back-to-back calls the output stage is timed over
SERVE_RATES = (100.0, 200.0, 400.0)  # req/s of the serving block of the default run
SERVE_REQUESTS = 400                 # requests per rate there
# DRAM bytes (read + write) of one bp_tile_kernel launch, from an ncu capture
# (dram__bytes_read.sum + dram__bytes_write.sum) of the default plain_large step
NCU_BP_TRAFFIC = {"plain_large": 565.913856e6 + 83.077632e6}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="plain_large")
    ap.add_argument("--cap-gb", type=float, default=1.25, help="--config streamed: device-memory cap (GB)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="CPU work of the bounded CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-e2e", action="store_true", help="skip the host-buffer timing (profiling)")
    ap.add_argument("--no-extras", action="store_true",
                    help="plain_large: skip the batch96 and serving blocks (profiling)")
    ap.add_argument("--tile", default="", help="e.g. 32x32")
    ap.add_argument("--chunk", type=int, default=0)
    ap.add_argument("--stage-cap", type=int, default=0)
    ap.add_argument("--min-blocks", type=int, default=0)
    ap.add_argument("--njobs", type=int, default=96, help="batch96: number of jobs")
    ap.add_argument("--no-autotune", action="store_true",
                    help="batch96: use --tile/--chunk/--min-blocks/--stage-cap instead of the autotuner")
    ap.add_argument("--per-job", action="store_true",
                    help="batch96: time every job alone instead (per-job rates by tile regime)")
    ap.add_argument("--only-job", type=int, default=-1,
                    help="batch96: run job J alone --steps times and exit (profiling one job)")
    ap.add_argument("--set", action="append", default=[], metavar="KEY=VALUE",
                    help="override a field of the synthetic config (e.g. P=1024 n=2048; profiling "
                         "captures of a smaller case of the same kernels)")
    ap.add_argument("--serve-rates", default="20,50,100,200,400", help="serve: arrival rates (req/s)")
    ap.add_argument("--serve-requests", type=int, default=2000, help="serve: requests per rate")
    ap.add_argument("--serve-lanes", type=int, default=3, help="serve: concurrent batches")
    ap.add_argument("--serve-batch-work", type=float, default=0.0,
                    help="serve: pixel*pulses per batch (0: library default)")
    return ap.parse_args()


class Clocks:
    """Samples nvidia-smi clocks and throttle reasons while running."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu_id), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx.append(float(f[1]))
                power.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "samples": len(sm),
                "power_w_max": max(power) if power else None, "reasons": sorted(reasons)}


def gpu_uuid(torch, dev):
    try:
        return "GPU-" + str(torch.cuda.get_device_properties(dev).uuid)
    except Exception:
        return str(dev)


def cpu_baseline_sample(data, seconds, nthreads=0):
    """Times the reference-precision CPU oracle on a pixel sample of the
    workload; range compression (all pulses) is charged pro rata."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.lib()
    k32 = data["k_r"].astype(np.float32).astype(np.float64)
    pos32 = data["pos"].astype(np.float32).astype(np.float64)
    nu, nv, P = data["nu"], data["nv"], data["P"]
    t0 = time.perf_counter()
    Q = O.range_compress(data["phs"], k32, data["taylor"], data["N_fft"], O.MODE_REF, nthreads)
    t_rc = time.perf_counter() - t0
    rng = np.random.default_rng(0)
    # calibrate on 512 pixels, then size the sample for `seconds`
    idx = rng.choice(nu * nv, 512, replace=False)
    t0 = time.perf_counter()
    O.backproject(Q, data["S"], data["delta_r"], k32, pos32, data["r"], nu, nv, idx, O.MODE_REF, nthreads)
    t_cal = time.perf_counter() - t0
    n = int(min(nu * nv, max(512, 512 * seconds / max(t_cal, 1e-6))))
    idx = rng.choice(nu * nv, n, replace=False)
    t0 = time.perf_counter()
    O.backproject(Q, data["S"], data["delta_r"], k32, pos32, data["r"], nu, nv, idx, O.MODE_REF, nthreads)
    t_bp = time.perf_counter() - t0
    t = t_bp + t_rc * n / (nu * nv)
    return dict(value=n * P / t / 1e9, seconds=t_bp + t_rc, t_rc=t_rc, t_bp=t_bp, n_pix=n,
                cores=O.max_threads())


def host_info():
    """The host the CPU figures were taken on: nproc, OMP_NUM_THREADS, model."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for ln in f:
                if ln.startswith("model name"):
                    model = ln.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"nproc": os.cpu_count(), "omp_num_threads": os.environ.get("OMP_NUM_THREADS"), "cpu_model": model}


def oracle_workload(name, seed, with_r=True):
    """The named configuration's workload generated by the oracle alone (the
    same data as sarbp_b200.synth.make, without the product library)."""
    from sarbp_b200.synth import CONFIGS, scene  # parameters only: loads no native code
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    cfg = CONFIGS[name]
    d = O.make_workload(cfg, scene(cfg["nscat"], cfg["half"], cfg["clutter"], seed), seed, with_r=with_r)
    d["name"] = name
    return d


def cpu_whole_image(name="plain_small", seed=2):
    """One whole image of `name` on the CPU oracle (reference precision, all
    host threads): range compression of all pulses and every pixel."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    d = oracle_workload(name, seed)
    k32 = d["k_r"].astype(np.float32).astype(np.float64)
    pos32 = d["pos"].astype(np.float32).astype(np.float64)
    t0 = time.perf_counter()
    O.backprojection(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], pos32, d["r"], d["nu"], d["nv"],
                     mode=O.MODE_REF)
    t = time.perf_counter() - t0
    return {"workload": "%s: %dx%d image, %d pulses x %d samples, N_fft %d" % (
                name, d["nu"], d["nv"], d["P"], d["S"], d["N_fft"]),
            "seconds": t, "value": d["nu"] * d["nv"] * d["P"] / t / 1e9, "unit": "Gpixel*pulses/s",
            "cores": O.max_threads()}


def run_reference(args, rank, world):
    if rank != 0:
        return
    data = oracle_workload(args.config, 2)
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.lib()
    k32 = data["k_r"].astype(np.float32).astype(np.float64)
    pos32 = data["pos"].astype(np.float32).astype(np.float64)
    nu, nv, P = data["nu"], data["nv"], data["P"]
    rng = np.random.default_rng(0)
    # per step: range compression of all pulses + a pixel sample sized so a
    # step takes ~2 s; throughput charges range compression pro rata
    t0 = time.perf_counter()
    Q = O.range_compress(data["phs"], k32, data["taylor"], data["N_fft"], O.MODE_REF)
    t_rc0 = time.perf_counter() - t0
    idx = rng.choice(nu * nv, 256, replace=False)
    t0 = time.perf_counter()
    O.backproject(Q, data["S"], data["delta_r"], k32, pos32, data["r"], nu, nv, idx, O.MODE_REF)
    t_cal = time.perf_counter() - t0
    n = int(min(nu * nv, max(256, 256 * 2.0 / max(t_cal, 1e-6))))
    units = t_tot = 0.0
    for step in range(args.warmup + args.steps):
        idx = rng.choice(nu * nv, n, replace=False)
        t0 = time.perf_counter()
        Q = O.range_compress(data["phs"], k32, data["taylor"], data["N_fft"], O.MODE_REF)
        t1 = time.perf_counter()
        O.backproject(Q, data["S"], data["delta_r"], k32, pos32, data["r"], nu, nv, idx, O.MODE_REF)
        t2 = time.perf_counter()
        if step >= args.warmup:
            units += n * P
            t_tot += (t2 - t1) + (t1 - t0) * n / (nu * nv)
    value = units / t_tot / 1e9
    cores = O.max_threads()
    sample = ("%d random pixels x %d pulses per step, range compression of all %d pulses "
              "charged pro rata (%d of %d pixels)" % (n, P, P, n, nu * nv))
    out = {
        "impl": "reference",
        "metric": metric_name(nu, nv, P),
        "value": value, "unit": "Gpixel*pulses/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_tot / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded, plain_large shapes)",
        "config": config_block(data, world),
        "cpu_baseline": {"value": value, "unit": "Gpixel*pulses/s", "cores": cores, "kind": "port",
                         "sample": sample, "host": host_info(), "whole_image": cpu_whole_image()},
        "e2e": {"value": value, "unit": "Gpixel*pulses/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "note": "reference CPU schedule restated in C (oracle/sarbp_oracle.c), inputs from the oracle's "
                "own generator; the reference itself needs Halide/FFTW/cnpy, which are not installable here",
    }
    print(json.dumps(out), flush=True)


def config_block(data, world):
    return {"workload": "%s: %dx%d image, %d pulses x %d samples, N_fft %d, Taylor %d" % (
                data["name"], data["nu"], data["nv"], data["P"], data["S"], data["N_fft"],
                data["taylor"]),
            "image": [data["nu"], data["nv"]], "npulses": data["P"], "nsamples": data["S"],
            "n_fft": data["N_fft"], "taylor": data["taylor"], "precision": "compat",
            "parallelism": "replicas%d" % world,
            "l2": "inputs+outputs %.0f MB per step (> 126 MB L2), no flush" % (
                (8.0 * data["P"] * data["S"] + 40.0 * data["nu"] * data["nv"]) / 1e6)}


def run_ours(args, rank, world, local_rank):
    import torch
    import torch.distributed as dist
    import sarbp_b200 as sb
    from sarbp_b200 import synth

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    over = {}
    for kv in args.set:
        k, v = kv.split("=", 1)
        over[k] = float(v) if "." in v or "e" in v else int(v)
    data = synth.make(args.config, seed=2 + rank, overrides=over or None)
    nu, nv, P, S = data["nu"], data["nv"], data["P"], data["S"]
    units = float(nu) * nv * P

    ctx = sb.Context(local_rank)
    stream = torch.cuda.current_stream(dev)
    ctx.set_stream(stream.cuda_stream)
    ffma_s, mufu_s = ctx.measure_peaks()

    t_phs = torch.from_numpy(data["phs"].view(np.float32).copy()).to(dev)
    t_k = torch.from_numpy(data["k_r"].astype(np.float32)).to(dev)
    t_pos = torch.from_numpy(data["pos"].astype(np.float32)).to(dev)
    t_r = torch.from_numpy(data["r"]).to(dev)
    t_out = torch.empty((nv, nu, 2), dtype=torch.float64, device=dev)
    tune = {}
    if args.tile:
        tune["tile"] = tuple(int(x) for x in args.tile.split("x"))
    if args.chunk:
        tune["pulse_chunk"] = args.chunk
    if args.stage_cap:
        tune["stage_cap"] = args.stage_cap
    if args.min_blocks:
        tune["min_blocks"] = args.min_blocks
    default_launch = not tune
    job = sb.make_job(S, P, data["N_fft"], data["taylor"], nu, nv, data["delta_r"], t_phs.data_ptr(),
                      t_k.data_ptr(), t_pos.data_ptr(), t_out.data_ptr(), r=t_r.data_ptr())

    def barrier():
        if world > 1:
            dist.barrier(device_ids=[local_rank])

    ctx.set_timing(False)
    for _ in range(args.warmup):
        ctx.run_jobs([job], **tune)
    ctx.synchronize()

    clocks = Clocks(gpu_uuid(torch, local_rank))
    clocks.start()
    time.sleep(0.3)
    l0 = ctx.launch_count()
    stage = []
    barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        ctx.run_jobs([job], **tune)
    ev1.record(stream)
    torch.cuda.synchronize()
    barrier()
    launches = ctx.launch_count() - l0
    ms = ev0.elapsed_time(ev1)
    ctx.synchronize()  # raises on a kernel status error
    clk = clocks.stop()
    # per-stage breakdown from the library's own events, outside the timed loop
    ctx.set_timing(True)
    for _ in range(max(3, min(args.steps, 10))):
        ctx.run_jobs([job], **tune)
        stage.append(ctx.last_stage_ms())
    ms_max = ms
    if world > 1:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms_max = float(t.item())
    value = world * units * args.steps / (ms_max * 1e-3) / 1e9

    # output stage (max|z| + u8 of the complex image), outside the step: the
    # HBM-bound tail, timed over U8_LAUNCHES back-to-back calls that rotate
    # over four copies of the image (4 x 67 MB, more than the 126 MB L2)
    t_u8 = torch.empty((nv, nu), dtype=torch.uint8, device=dev)
    imgs = [t_out] + [t_out.clone() for _ in range(3)]
    turn = [0]

    def u8_call():
        img = imgs[turn[0] % len(imgs)]
        turn[0] += 1
        ctx.img_output_u8_from_img_device(img.data_ptr(), nu, nv, data["db"][0], data["db"][1], t_u8.data_ptr())

    for _ in range(4):
        u8_call()
    u8_ms = timed_ms(torch, stream, u8_call, U8_LAUNCHES) / U8_LAUNCHES
    ctx.synchronize()
    del imgs

    # ---- e2e through the host-buffer entry point, pinned host memory ----
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()
    h_phs, h_k = pin(data["phs"]), pin(data["k_r"].astype(np.float32))
    h_pos, h_r = pin(data["pos"].astype(np.float32)), pin(data["r"])
    h_u, h_v = data["u"], data["v"]
    out_pinned = torch.empty((nv, nu, 2), dtype=torch.float64).pin_memory().numpy()

    def e2e_call():
        # same operator as sarbp_b200.Context.backprojection_cuda, writing into pinned memory
        import ctypes
        from sarbp_b200 import _lib
        o = sb._opts(sb.PREC_COMPAT, **tune)
        p = lambda a: ctypes.c_void_p(a.ctypes.data)
        _lib.check(_lib.lib().sarbp_backprojection(
            ctx.handle, p(h_phs), S, P, p(h_k), data["taylor"], data["N_fft"], data["delta_r"], p(h_u),
            nu, p(h_v), nv, p(h_pos), p(h_r), p(out_pinned), ctypes.byref(o)))

    if args.no_e2e:
        args.e2e_steps = 0
    else:
        e2e_call()
    barrier()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.e2e_steps):
        e2e_call()
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max(e0.elapsed_time(e1), 1e-6)
    if world > 1:
        t = torch.tensor([e2e_ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = world * units * args.e2e_steps / (e2e_ms * 1e-3) / 1e9 if args.e2e_steps else None
    h2d = h_phs.nbytes + h_k.nbytes + h_pos.nbytes + h_r.nbytes
    d2h = out_pinned.nbytes

    # ---- roofline of the backprojection kernel (FP32 + SFU) ----
    st = np.array(stage)
    bp_ms = float(st[:, 3].mean())
    geom_ms = float(st[:, 2].mean())
    rc_ms = float(st[:, 1].mean())
    prep_ms = float(st[:, 0].mean())
    bp_units_s = units / (bp_ms * 1e-3)
    t_fp32 = FP32_PER_UNIT * units / ffma_s
    t_sfu = SFU_PER_UNIT * units / mufu_s
    bound = "sfu" if t_sfu >= t_fp32 else "fp32"
    if bound == "sfu":
        achieved, peak = SFU_PER_UNIT * bp_units_s / 1e12, mufu_s / 1e12
    else:
        achieved, peak = FP32_PER_UNIT * bp_units_s / 1e12, ffma_s / 1e12
    rc_bytes = P * S * 8 + P * data["N_fft"] * 8
    u8_bytes = nu * nv * (16 + 16 + 1)  # max|z| pass, then image in and u8 out
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    out = {
        "metric": metric_name(nu, nv, P),
        "value": value, "unit": "Gpixel*pulses/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (split-precision; f64 per-pulse set-up)",
        "data": "synthetic (seeded, plain_large shapes)",
        "config": config_block(data, world),
        "gpu_launches": int(launches),
        "stage_ms": {"setup": prep_ms, "range_compress": rc_ms, "tile_geometry": geom_ms, "backproject": bp_ms,
                     "db_u8": u8_ms},
        "roofline": {"bound": bound, "achieved": achieved, "peak": peak, "unit": "Tops/s",
                     "frac": achieved / peak,
                     "traffic": NCU_BP_TRAFFIC.get(args.config) if default_launch else None,
                     "kernel": "bp_tile_kernel",
                     "per_unit": "%d FP32 instr + %d SFU ops per pixel*pulse" % (FP32_PER_UNIT, SFU_PER_UNIT),
                     "peak_source": "measured in this run: FFMA / MUFU chain microkernels",
                     "fp32": {"achieved": FP32_PER_UNIT * bp_units_s / 1e12, "peak": ffma_s / 1e12,
                              "frac": FP32_PER_UNIT * bp_units_s / ffma_s},
                     "sfu": {"achieved": SFU_PER_UNIT * bp_units_s / 1e12, "peak": mufu_s / 1e12,
                             "frac": SFU_PER_UNIT * bp_units_s / mufu_s}},
        "roofline_hbm": {
            "range_compress": {"bound": "hbm", "achieved": rc_bytes / (rc_ms * 1e-3) / 1e9,
                               "peak": hbm_peak, "unit": "GB/s",
                               "frac": rc_bytes / (rc_ms * 1e-3) / 1e9 / hbm_peak,
                               "bytes": rc_bytes},
            "db_u8": {"bound": "hbm", "achieved": u8_bytes / (u8_ms * 1e-3) / 1e9,
                      "peak": hbm_peak, "unit": "GB/s",
                      "frac": u8_bytes / (u8_ms * 1e-3) / 1e9 / hbm_peak, "bytes": u8_bytes,
                      "how": "sarbp_img_output_u8_from_img_device (max|z| kernel + u8 kernel), "
                             "%d back-to-back calls over four copies of the image (268 MB > L2)"
                             % U8_LAUNCHES},
            "peak_source": "MEASURED_PEAKS.json hbm_gbs" if "hbm_gbs" in peaks else "fallback 6650 GB/s"},
        "e2e": {"value": e2e_value, "unit": "Gpixel*pulses/s", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_ms / max(args.e2e_steps, 1),
                "steps": args.e2e_steps},
        "clocks": clk,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline_sample(data, args.cpu_seconds)
        out["cpu_baseline"] = {"value": cb["value"], "unit": "Gpixel*pulses/s", "cores": cb["cores"],
                               "kind": "port",
                               "sample": "%d random pixels x %d pulses (reference-precision C oracle, "
                                         "%d threads, %.1f s; range compression of all pulses "
                                         "charged pro rata)" % (cb["n_pix"], P, cb["cores"],
                                                                cb["seconds"]),
                               "host": host_info(), "whole_image": cpu_whole_image()}
    if world == 1 and args.config == "plain_large" and not args.no_extras:
        # the rest of the headline metric: the batched form (ratio to the
        # plain single image above) and the serving loop (p50/p99 and the
        # FP64 rel-L2 of a 5 % request sample), bounded to about a minute
        b = batch_measure(torch, ctx, stream, dev, 96, 7, steps=5, warmup=3, e2e_steps=1, full=False)
        out["batch96"] = {
            "metric": "Gpixel*pulses/s (96 uneven jobs, one persistent launch, CUDA-graph replay)",
            "value": b["value"], "unit": "Gpixel*pulses/s", "ms_per_step": b["ms_per_step"],
            "steps": b["steps"], "workload": b["workload"], "gpu_launches": b["gpu_launches"],
            "ratio_to_plain_single_image": b["value"] / value,
            "ratio_to_loop_of_per_image_calls": b["compare"]["speedup_vs_loop"],
            "compare": b["compare"], "autotuned": b["autotuned"], "l2": b["l2"], "clocks": b["clocks"]}
        s = serve_measure(torch, ctx, dev, SERVE_RATES, SERVE_REQUESTS, 3, 0.0, 7)
        out["serve"] = {"metric": "serving latency p50/p99 (ms) and throughput under Poisson arrivals",
                        "sweep": s["sweep"], "fp64_sample": s["fp64_sample"], "residency": s["residency"],
                        "peak_device_bytes": s["peak_device_bytes"], "workload": s["workload"],
                        "latency": s["latency"], "clocks": s["clocks"]}
    ctx.close()
    if rank == 0:
        print(json.dumps(out), flush=True)


def timed_ms(torch, stream, fn, steps):
    """CUDA-event milliseconds of `steps` calls of fn on `stream`."""
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1)


def batch_measure(torch, ctx, stream, dev, njobs, seed, steps, warmup, e2e_steps, tune=None,
                  lanes=3, batch_work=0.0, gmax=lambda ms: ms, full=True):
    """The batched form: `njobs` uneven image-formation jobs (images
    256^2..2048^2, 128-2000 pulses, 256-1024 samples, Taylor 17-35 dB, 5-15 km,
    20-50 deg) formed together in one autotuned persistent launch sequence
    replayed as a CUDA graph.  Compared with the same jobs as one batched call
    without the graph and as a loop of per-image calls of the split-precision
    kernel; with `full`, also a loop of per-image calls of the plain FP32
    kernel (PREC_NAIVE) and the e2e figures from host memory."""
    import sarbp_b200 as sb
    from sarbp_b200 import synth
    from sarbp_b200.batch import DeviceJob, HostJob

    t0 = time.time()
    cfgs = synth.batch_jobs(njobs=njobs, seed=seed)
    jobs = [DeviceJob(c, torch, dev) for c in cfgs]
    synth_s = time.time() - t0
    units = float(sum(j.units for j in jobs))
    J = [j.job for j in jobs]
    sp = stream.cuda_stream
    t0 = time.time()
    if tune is not None:  # a fixed launch shape (profiling one shape)
        tune_ms = -1.0
    else:
        tune, tune_ms = ctx.autotune(J)
    tune_s = time.time() - t0
    plan = sb.Plan(ctx, J, **tune)
    for _ in range(warmup):
        plan.launch(sp)
    plan.wait()
    clocks = Clocks(gpu_uuid(torch, dev))
    clocks.start()
    n0 = ctx.launch_count()
    ms_graph = gmax(timed_ms(torch, stream, lambda: plan.launch(sp), steps))
    launches = ctx.launch_count() - n0
    plan.wait()
    clk = clocks.stop()
    k2 = max(1, steps // 2) if full else 1
    ms_batch = gmax(timed_ms(torch, stream, lambda: ctx.run_jobs(J, **tune), k2))
    ctx.synchronize()
    ms_loop = gmax(timed_ms(torch, stream, lambda: [ctx.run_jobs([j]) for j in J], k2))
    ctx.synchronize()
    g = lambda ms, k: units * k / (ms * 1e-3) / 1e9
    res = {
        "value": g(ms_graph, steps), "ms_per_step": ms_graph / steps, "steps": steps,
        "pixel_pulses_per_step": units, "gpu_launches": int(launches),
        "workload": "%d jobs, images %s, pulses %d-%d, samples %s, Taylor %d-%d dB "
                    "(float-quotient window above 30 dB)"
                    % (len(jobs), "/".join("%dx%d" % s for s in sorted(set((j.nu, j.nv) for j in jobs))),
                       min(j.P for j in jobs), max(j.P for j in jobs),
                       "/".join(str(s) for s in sorted(set(j.S for j in jobs))),
                       min(c["taylor"] for c in cfgs), max(c["taylor"] for c in cfgs)),
        "autotuned": {"tile": list(tune["tile"]), "pulse_chunk": tune["pulse_chunk"],
                      "stage_cap": tune.get("stage_cap", 0), "min_blocks": tune["min_blocks"],
                      "best_ms": tune_ms, "seconds": tune_s},
        "compare": {"graph_replay": g(ms_graph, steps),
                    "batched_call_no_graph": g(ms_batch, k2),
                    "loop_of_per_image_calls": g(ms_loop, k2),
                    "speedup_vs_loop": ms_loop / k2 / (ms_graph / steps)},
        "l2": "inputs+outputs %.1f GB per step (> 126 MB L2), no flush"
              % (sum(j.device_bytes() for j in jobs) / 1e9),
        "clocks": clk, "synthesis_seconds": synth_s,
    }
    if full:
        ms_naive = gmax(timed_ms(torch, stream,
                                 lambda: [ctx.run_jobs([j], precision=sb.PREC_NAIVE) for j in J], 1))
        ctx.synchronize()
        res["compare"]["loop_of_per_image_naive_fp32"] = g(ms_naive, 1)
        res["compare"]["speedup_vs_naive_loop"] = ms_naive / (ms_graph / steps)
        # end to end: phase histories, k_r, pos from pinned host memory in,
        # the complex images out, around each graph replay (one stream)
        h_in = [(t, t.cpu().pin_memory()) for j in jobs for t in (j.phs, j.k_r, j.pos)]
        h_out = [(j.out, torch.empty(j.out.shape, dtype=j.out.dtype).pin_memory()) for j in jobs]

        def e2e_step():
            for d, h in h_in:
                d.copy_(h, non_blocking=True)
            plan.launch(sp)
            for d, h in h_out:
                h.copy_(d, non_blocking=True)

        e2e_step()
        plan.wait()
        ms_e2e = gmax(timed_ms(torch, stream, e2e_step, e2e_steps))
        plan.wait()
        res["e2e_graph_serial_copies"] = {
            "value": g(ms_e2e, e2e_steps), "unit": "Gpixel*pulses/s",
            "h2d_bytes_per_step": int(sum(h.numel() * h.element_size() for _, h in h_in)),
            "d2h_bytes_per_step": int(sum(h.numel() * h.element_size() for _, h in h_out)),
            "ms_per_step": ms_e2e / e2e_steps, "steps": e2e_steps,
            "how": "inputs copied in, graph replayed, images copied out, one stream"}
        del h_in, h_out
    plan.close()
    if full:
        # end to end through the serving loop: the same jobs in pinned host
        # memory submitted at once, complex images back in pinned host
        # memory; a step is first submission -> last image on the host
        pin = lambda shape, dtype: torch.empty(
            shape, dtype=getattr(torch, np.dtype(dtype).name)).pin_memory().numpy()
        hjobs = [HostJob(j.cfg, alloc=pin, data=j.data) for j in jobs]
        houts = [hj.new_outputs()[0] for hj in hjobs]
        srv = sb.Server(ctx, hbm_cap_bytes=150e9, lanes=lanes, max_batch=32, max_batch_work=batch_work,
                        precision=sb.PREC_COMPAT)

        def burst():
            rids = [srv.submit(hj.job(o, precision=sb.PREC_COMPAT)) for hj, o in zip(hjobs, houts)]
            first = last = None
            for r in rids:
                rc = srv.wait(r)
                if rc != 0:
                    raise RuntimeError("request failed: %d %s" % (rc, sb.last_error()))
                ts, _, td = srv.times(r)
                first = ts if first is None else min(first, ts)
                last = td if last is None else max(last, td)
                srv.release(r)
            return (last - first) * 1e3

        try:
            burst()
            b0 = srv.stats()["batches"]
            ms_srv = gmax(sum(burst() for _ in range(e2e_steps)))
            srv_batches = (srv.stats()["batches"] - b0) / e2e_steps
        finally:
            srv.close()
        res["e2e"] = {
            "value": g(ms_srv, e2e_steps), "unit": "Gpixel*pulses/s",
            "h2d_bytes_per_step": int(sum(hj.phs.nbytes + hj.k32.nbytes + hj.p32.nbytes + hj.u.nbytes
                                          + hj.v.nbytes for hj in hjobs)),
            "d2h_bytes_per_step": int(sum(o.nbytes for o in houts)),
            "ms_per_step": ms_srv / e2e_steps, "steps": e2e_steps, "batches_per_step": srv_batches,
            "lanes": lanes,
            "how": "all jobs submitted at once to the serving loop (sarbp_server_*) from pinned "
                   "host memory; first submission to last image on the host"}
    res["tune"] = tune
    return res


def run_batch(args, rank, world, local_rank):
    """--config batch96: the batched form on its own (see batch_measure)."""
    import torch
    import torch.distributed as dist
    import sarbp_b200 as sb

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    ctx = sb.Context(local_rank)
    stream = torch.cuda.current_stream(dev)
    ctx.set_stream(stream.cuda_stream)

    def gmax(ms):
        if world > 1:
            t = torch.tensor([ms], device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ms = float(t.item())
        return ms

    if args.per_job or args.only_job >= 0:
        r = per_job_measure(torch, ctx, stream, dev, args.njobs, 7 + rank, args.only_job, args.steps)
        ctx.close()
        if rank == 0 and r is not None:
            print(json.dumps(r), flush=True)
        return
    tune = None
    if args.no_autotune:
        tune = dict(tile=tuple(int(x) for x in (args.tile or "32x32").split("x")),
                    pulse_chunk=args.chunk or 64, min_blocks=args.min_blocks or 3, stage_cap=args.stage_cap)
    if world > 1:
        dist.barrier()
    r = batch_measure(torch, ctx, stream, dev, args.njobs, 7 + rank, args.steps, args.warmup,
                      max(1, min(args.e2e_steps, args.steps)), tune=tune, lanes=args.serve_lanes,
                      batch_work=args.serve_batch_work, gmax=gmax, full=True)
    ctx.close()
    out = {
        "metric": "Gpixel*pulses/s (96 uneven jobs, batched)",
        "value": world * r["value"], "unit": "Gpixel*pulses/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": r["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 (split-precision; f64 per-pulse set-up)",
        "data": "synthetic (seeded uneven jobs)",
        "config": {"workload": "batch96: " + r["workload"],
                   "pixel_pulses_per_step": r["pixel_pulses_per_step"], "precision": "compat",
                   "parallelism": "replicas%d" % world, "l2": r["l2"]},
        "gpu_launches": r["gpu_launches"], "autotuned": r["autotuned"], "compare": r["compare"],
        "e2e": dict(r["e2e"], value=world * r["e2e"]["value"]),
        "e2e_graph_serial_copies": r["e2e_graph_serial_copies"],
        "clocks": r["clocks"], "synthesis_seconds": r["synthesis_seconds"],
    }
    if rank == 0:
        print(json.dumps(out), flush=True)


def metric_name(nu, nv, P):
    """The headline metric's name for an nu x nv image from P pulses
    ("Gpixel*pulses/s (2048^2 x 1999 backprojection)" for plain_large)."""
    img = "%d^2" % nu if nu == nv else "%dx%d" % (nu, nv)
    return "Gpixel*pulses/s (%s x %d backprojection)" % (img, P)


def per_job_measure(torch, ctx, stream, dev, njobs, seed, only, steps):
    """Each batch96 job alone through the device entry point (default launch
    shape): its backprojection ms from the library's stage events, with the
    job's tile regime (k_c x 32x32-tile half-diagonal: wide above 1024 rad;
    gm = half-diagonal / 2 R0, which sets the series order).  With `only`,
    runs that one job `steps` times and returns None (a profiling target)."""
    import sarbp_b200 as sb
    from sarbp_b200 import synth
    from sarbp_b200.batch import DeviceJob
    cfgs = synth.batch_jobs(njobs=njobs, seed=seed)
    if only >= 0:
        j = DeviceJob(cfgs[only], torch, dev)
        for _ in range(max(1, steps)):
            ctx.run_jobs([j.job])
        ctx.synchronize()
        return None
    c_light = 299792458.0
    rows = []
    for i, c in enumerate(cfgs):
        j = DeviceJob(c, torch, dev)
        for _ in range(2):
            ctx.run_jobs([j.job])
        ctx.set_timing(True)
        st = []
        for _ in range(3):
            ctx.run_jobs([j.job])
            st.append(ctx.last_stage_ms())
        ctx.set_timing(False)
        ctx.synchronize()
        bp = float(np.median(np.array(st), axis=0)[3])
        rho = 16 * math.sqrt(2) * c["extent"] / c["n"]
        kc = 4 * math.pi * (c["f0"] + c["S"] / 2 * c["df"]) / c_light
        rows.append({"job": i, "n": c["n"], "P": c["P"], "S": c["S"], "kc_rho": kc * rho,
                     "gm": rho / (2 * c["R0"]), "bp_ms": bp, "rate": c["n"] ** 2 * c["P"] / (bp * 1e-3) / 1e9})
        del j
    groups = {}
    for r in rows:
        key = "%d^2 %s" % (r["n"], "wide" if r["kc_rho"] > 1024 else "narrow")
        g = groups.setdefault(key, [0, 0.0, 0.0])
        g[0] += 1
        g[1] += r["n"] ** 2 * r["P"]
        g[2] += r["bp_ms"]
    return {"metric": "Gpixel*pulses/s of each batch96 job alone (backprojection stage)",
            "by_regime": {k: {"jobs": g[0], "rate": g[1] / (g[2] * 1e-3) / 1e9} for k, g in sorted(groups.items())},
            "sum_alone_ms": sum(r["bp_ms"] for r in rows), "jobs": rows}


def fp64_sample_rel_l2(pool, picks, seed, pixels=1000):
    """rel-L2 vs the FP64 oracle of the served images of the sampled requests
    (pool job k, image) at `pixels` random pixels each."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.lib()
    rng = np.random.default_rng(seed)
    errs = []
    for k, img in picks:
        hj = pool[k]
        d = hj.data
        r = O.pixel_locs(d["u"], d["v"], d["u_hat"], d["v_hat"])
        idx = rng.choice(hj.nu * hj.nv, min(pixels, hj.nu * hj.nv), replace=False)
        ref = O.backprojection(d["phs"], d["k_r"], d["taylor"], d["N_fft"], d["delta_r"], d["pos"], r,
                               hj.nu, hj.nv, mode=O.MODE_FP64, out_idx=idx,
                               taylor_mode=d.get("taylor_mode", 0))
        got = img.ravel()[idx]
        errs.append(float(np.linalg.norm(got - ref) / np.linalg.norm(ref)))
    return errs


def serve_measure(torch, ctx, dev, rates, nreq, lanes, batch_work, seed, sample_frac=0.05, resident=True):
    """The serving loop under Poisson arrivals.  A pool of 96 uneven jobs (the
    batch96 distribution) lives in pinned host memory; with `resident` their
    phase histories are registered once (uploaded and range-compressed
    once, kept on the device) and each request brings only its image plane;
    each request picks a pool job (seeded), is submitted at its arrival time
    and returns its complex image to pinned host memory.  Latency is
    submission to image-on-host on the server's clock; p50/p99 over `nreq`
    requests per rate.  PREC_PRECISE (f64 positions and k_r).  A seeded
    `sample_frac` of the requests keep their own output buffers and are
    checked against the FP64 oracle afterwards, outside the timed sweep."""
    import sarbp_b200 as sb
    from sarbp_b200 import synth
    from sarbp_b200.batch import HostJob

    pin = lambda shape, dtype: torch.empty(shape, dtype=getattr(torch, np.dtype(dtype).name)).pin_memory().numpy()
    cfgs = synth.batch_jobs(njobs=96, seed=seed)
    t0 = time.time()
    pool = [HostJob(c, alloc=pin) for c in cfgs]
    outs = [hj.new_outputs()[0] for hj in pool]  # shared image buffer per pool job
    synth_s = time.time() - t0
    clocks = Clocks(gpu_uuid(torch, dev))
    sweep, picks = [], []
    srng = np.random.default_rng(seed + 99)
    srv = sb.Server(ctx, hbm_cap_bytes=150e9, lanes=lanes, max_batch=32, max_batch_work=batch_work,
                    precision=sb.PREC_PRECISE)
    ap = [None] * len(pool)
    reg_s = 0.0
    try:
        if resident:  # phase histories uploaded and range-compressed once
            t0 = time.time()
            ap = [srv.register(hj.job(outs[k], precision=sb.PREC_PRECISE)) for k, hj in enumerate(pool)]
            reg_s = time.time() - t0

        def submit(k, o):
            job = pool[k].job(o, precision=sb.PREC_PRECISE)
            return srv.submit_on(ap[k], job) if resident else srv.submit(job)

        for k in range(len(pool)):  # warm-up: every pool job once
            r = submit(k, outs[k])
            srv.wait(r)
            srv.release(r)
        c0 = srv.counters()
        clocks.start()
        for rate in rates:
            rng = np.random.default_rng(int(rate * 1000) + seed)
            pick = rng.integers(0, len(pool), nreq)
            arrive = np.cumsum(rng.exponential(1.0 / rate, nreq))
            own = srng.choice(nreq, max(1, int(round(sample_frac * nreq))), replace=False).tolist()
            # the sampled requests' own (pinned) image buffers, made before
            # the arrivals start: pinning memory is slow and would stall them
            own = {i: pool[int(pick[i])].new_outputs()[0] for i in own}
            b0 = srv.stats()["batches"]
            rids = []
            start = time.perf_counter()
            for i in range(nreq):
                while True:
                    dt = arrive[i] - (time.perf_counter() - start)
                    if dt <= 0:
                        break
                    time.sleep(dt if dt > 2e-3 else 0)
                k = int(pick[i])
                o = own.get(i, outs[k])
                rids.append((submit(k, o), k, o, i in own))
            lat, first, last, units = [], None, None, 0.0
            for r, k, o, mine in rids:
                rc = srv.wait(r)
                if rc != 0:
                    raise RuntimeError("request failed: %d %s" % (rc, sb.last_error()))
                ts, ta, td = srv.times(r)
                lat.append((td - ts) * 1e3)
                first = ts if first is None else min(first, ts)
                last = td if last is None else max(last, td)
                units += pool[k].units
                srv.release(r)
                if mine:
                    picks.append((k, o))
            lat = np.array(lat)
            sweep.append({"rate_req_s": rate, "requests": nreq,
                          "achieved_rate_req_s": nreq / (arrive[-1] if arrive[-1] > 0 else 1.0),
                          "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
                          "mean_ms": float(lat.mean()),
                          "throughput_gpix_pulses_s": units / (last - first) / 1e9,
                          "batches": srv.stats()["batches"] - b0})
        clk = clocks.stop()
        peak = srv.stats()["peak_bytes"]
        c1 = srv.counters()
    finally:
        srv.close()
    t0 = time.time()
    errs = fp64_sample_rel_l2(pool, picks, seed)
    nall = nreq * len(rates)
    return {"sweep": sweep, "peak_device_bytes": peak, "clocks": clk, "synthesis_seconds": synth_s,
            "lanes": lanes,
            "residency": {
                "registered_apertures": len(pool) if resident else 0, "register_seconds": reg_s,
                "h2d_bytes_per_request": (c1["h2d_bytes"] - c0["h2d_bytes"]) / nall,
                "phase_history_bytes_per_request_if_uploaded": float(np.mean(
                    [pool[k].phs.nbytes + pool[k].k64.nbytes + pool[k].p64.nbytes + pool[k].k32.nbytes
                     + pool[k].p32.nbytes for k in range(len(pool))])),
                "range_compressed_pulses_during_sweep": c1["rc_pulses"] - c0["rc_pulses"],
                "requests_served_from_resident_apertures": c1["resident_requests"] - c0["resident_requests"]},
            "fp64_sample": {"requests": len(errs), "of": nreq * len(rates), "pixels_per_image": 1000,
                            "rel_l2_max": max(errs), "rel_l2_median": float(np.median(errs)),
                            "target": 1e-3, "oracle_seconds": time.time() - t0},
            "latency": "submission to complex image in pinned host memory",
            "workload": "%d requests per rate drawn from 96 uneven jobs (batch96 distribution), rates %s "
                        "req/s, %d lanes, batches <= 32, HBM budget 150 GB, PREC_PRECISE, %s"
                        % (nreq, "/".join("%g" % r for r in rates), lanes,
                           "phase histories registered once (resident range profiles)" if resident
                           else "each request uploads and range-compresses its phase history")}


def run_serve(args, rank, world, local_rank):
    """--config serve: the serving sweep on its own (see serve_measure)."""
    import torch
    import sarbp_b200 as sb

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    ctx = sb.Context(local_rank)
    rates = [float(x) for x in args.serve_rates.split(",")]
    try:
        s = serve_measure(torch, ctx, dev, rates, args.serve_requests, args.serve_lanes, args.serve_batch_work,
                          7 + rank)
        # the same top rate with every request uploading and range-compressing
        # its own phase history, for comparison
        u = serve_measure(torch, ctx, dev, rates[-1:], args.serve_requests, args.serve_lanes,
                          args.serve_batch_work, 7 + rank, resident=False)
    finally:
        ctx.close()
    top = s["sweep"][-1]
    out = {
        "metric": "serving p99 latency at %g req/s (ms)" % top["rate_req_s"],
        "value": top["p99_ms"], "unit": "ms", "n_gpus": world, "steps": args.serve_requests,
        "warmup": 96, "ms_per_step": top["mean_ms"], "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (split-precision; f64 per-pulse set-up, PREC_PRECISE)",
        "data": "synthetic (seeded uneven jobs, Poisson arrivals)",
        "config": {"workload": "serve: " + s["workload"], "parallelism": "replicas%d" % world,
                   "latency": s["latency"]},
        "sweep": s["sweep"], "fp64_sample": s["fp64_sample"], "residency": s["residency"],
        "peak_device_bytes": s["peak_device_bytes"],
        "uploading_each_request": {"sweep": u["sweep"], "residency": u["residency"]},
        "clocks": s["clocks"], "synthesis_seconds": s["synthesis_seconds"],
    }
    if rank == 0:
        print(json.dumps(out), flush=True)


# The reference's one-node Sandia run (exp/summit/darpa-demo2): its command
# line and the stage times its log reports, on 1 Summit node (2x POWER9, the
# CPU schedule, 42 and then 168 host threads).
SANDIA1_CMD = ["-d", "-45.0", "-D", "0.0", "-t", "30", "-u", "2"]
SANDIA1_PUBLISHED = {
    "hardware": "1 Summit node, 2x POWER9, the reference's -s cpu schedule (42 threads, then 168)",
    "data": "the Sandia phase history (1999 pulses x 1800 samples; not shipped with the reference)",
    "source": "exp/summit/darpa-demo2/logs/SARBP-Sandia-1.763157:182-201",
    "load_ms": 181, "image_plane_ms": 139, "backprojection_ms": [35528, 17448],
    "dB_ms": 41, "u8_ms": 16, "png_write_ms": 421,
}


def write_platform_dir(d, data):
    """A platform directory in the reference's .npy layout (PlatformData.cpp:
    phs complex128 [P][S], pos f32 [P][3], k_r f64 [S], delta_r, R_c f32 (the
    mid-aperture antenna position), npulses, nsamples) with the element
    types the Sandia run's log shows (the CLI downcasts phs and k_r)."""
    os.makedirs(d, exist_ok=True)
    P, S = data["phs"].shape
    np.save(os.path.join(d, "phs.npy"), data["phs"].astype(np.complex128))
    np.save(os.path.join(d, "pos.npy"), np.ascontiguousarray(data["pos"], np.float32))
    np.save(os.path.join(d, "k_r.npy"), np.ascontiguousarray(data["k_r"], np.float64))
    np.save(os.path.join(d, "delta_r.npy"), np.array(float(data["delta_r"])))
    np.save(os.path.join(d, "R_c.npy"), np.ascontiguousarray(data["pos"][P // 2], np.float32))
    np.save(os.path.join(d, "npulses.npy"), np.array(P, np.int64))
    np.save(os.path.join(d, "nsamples.npy"), np.array(S, np.int64))
    return d


def run_cli(args, rank, world, local_rank):
    """--config cli_sandia: the sarbp CLI end to end with the reference's
    one-node Sandia command line (-d -45 -D 0 -t 30 -u 2) on a seeded
    synthetic platform directory of that run's shape (1999 pulses x 1800
    samples; the CLI's image plane is then 2048^2 and N_fft 4096): load,
    image plane, `steps` + 1 backprojection calls from host buffers (the
    first one also creates the context), dB, u8 and the PNG write, each
    from the CLI's own progress lines, beside the times the reference's log
    reports for the same command on its Sandia data."""
    import re
    import shutil
    import tempfile
    import torch
    from sarbp_b200 import synth

    sarbp = os.path.join(ROOT, "halide-sar-app_b200", "bin", "sarbp")
    if not os.path.exists(sarbp):
        raise SystemExit("sarbp CLI not built (make -C halide-sar-app_b200)")
    data = synth.make("sandia_2048", seed=2 + rank, with_r=False)
    P, S = data["phs"].shape
    tmp = tempfile.mkdtemp(prefix="sarbp_cli_")
    try:
        pdir = write_platform_dir(os.path.join(tmp, "sandia"), data)
        iters = 1 + max(1, min(args.steps, 20))
        env = dict(os.environ, CUDA_VISIBLE_DEVICES=os.environ.get("CUDA_VISIBLE_DEVICES", str(local_rank)))
        clocks = Clocks(gpu_uuid(torch, torch.device("cuda", local_rank)))
        clocks.start()
        t0 = time.perf_counter()
        p = subprocess.run([sarbp, "-p", pdir, "-o", os.path.join(tmp, "sandia.png")] + SANDIA1_CMD +
                           ["-n", str(iters)], capture_output=True, text=True, timeout=600, env=env)
        wall = time.perf_counter() - t0
        clk = clocks.stop()
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    if p.returncode != 0:
        raise SystemExit("sarbp failed (%d): %s" % (p.returncode, p.stdout[-2000:] + p.stderr[-2000:]))
    out = p.stdout
    ms = lambda pat: [float(x) for x in re.findall(pat, out)]
    bp = ms(r"\(\d+\) Halide backprojection returned 0 in ([0-9.]+) ms")
    nu = int(re.search(r"X length: (\d+)", out).group(1))
    nv = int(re.search(r"Y length: (\d+)", out).group(1))
    warm = bp[1:]
    med = statistics.mean(warm)  # the lines give whole milliseconds: the mean resolves finer
    rate = lambda t: nu * nv * P / (t * 1e-3) / 1e9
    pub = SANDIA1_PUBLISHED
    stages = {"load": ms(r"Loaded platform data in ([0-9.]+) ms")[0],
              "image_plane": ms(r"Computed image plane parameters in ([0-9.]+) ms")[0],
              "backprojection_first": bp[0], "backprojection_warm": warm,
              "dB": ms(r"Halide dB conversion returned 0 in ([0-9.]+) ms")[0],
              "u8": ms(r"Halide PNG production returned 0 in ([0-9.]+) ms")[0],
              "png_write": ms(r"Wrote .* in ([0-9.]+) ms")[0]}
    h2d = P * S * 8 + P * 12 + S * 4 + (nu + nv) * 8
    res = {
        "metric": "Gpixel*pulses/s (sarbp CLI backprojection call, %dx%d image, %d pulses x %d samples)"
                  % (nu, nv, P, S),
        "value": rate(med), "unit": "Gpixel*pulses/s", "n_gpus": 1, "steps": len(warm), "warmup": 1,
        "ms_per_step": med, "higher_is_better": True, "scaling": "weak",
        # the faster of the two published calls (168 threads)
        "vs_baseline": rate(med) / rate(min(pub["backprojection_ms"])),
        "dtype": "f32 (split-precision; f64 per-pulse set-up, the reference's f32 positions)",
        "data": "synthetic (seeded; the Sandia run's shapes; complex128/f64 platform files as the Sandia data)",
        "config": {"workload": "cli_sandia: sarbp %s on %d pulses x %d samples -> %dx%d image, N_fft %d"
                               % (" ".join(SANDIA1_CMD), P, S, nu, nv, n_fft_of(S, 2)),
                   "parallelism": "replicas1", "l2": "host buffers; each call copies its inputs and image"},
        "e2e": {"value": rate(med), "unit": "Gpixel*pulses/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": nu * nv * 16},
        "stages_ms": stages, "cli_wall_s": wall,
        "published_reference": dict(pub, backprojection_gpix_pulses_s=[rate(t) for t in pub["backprojection_ms"]]),
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(res), flush=True)


def run_streamed(args, rank, world, local_rank):
    """--config streamed: one 4096^2 image from 4000 pulses x 2048 samples
    (N_fft 8192, 20 km, PREC_PRECISE) in host memory, formed by
    sarbp_backprojection_streamed under a device-memory cap smaller than
    its one-shot footprint (pulse chunks into a device-resident partial
    image, each chunk's rows uploaded under the previous chunk's kernels),
    against the same call with no cap (one chunk) and the device-resident
    one-shot call of the same job.  Host buffers are pinned; the streamed
    calls' wall time includes their copies and device allocations."""
    import torch
    import sarbp_b200 as sb
    from sarbp_b200 import synth
    from sarbp_b200.batch import HostJob

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    pin = lambda shape, dtype: torch.empty(shape, dtype=getattr(torch, np.dtype(dtype).name)).pin_memory().numpy()
    cfg = dict(synth.CONFIGS["precision"], nscat=40, clutter=0)
    d = synth.make("precision", seed=5 + rank, with_r=False, overrides=cfg)
    hj = HostJob(dict(cfg, seed=5 + rank), alloc=pin, data=d)
    out = hj.new_outputs()[0]
    job = hj.job(out, precision=sb.PREC_PRECISE)
    units = hj.units
    cap = float(args.cap_gb) * 1e9
    ctx = sb.Context(local_rank)
    clocks = Clocks(gpu_uuid(torch, dev))
    res = {}
    try:
        one_shot = sb.job_device_bytes(job, precision=sb.PREC_PRECISE)

        def timed(max_bytes):
            for _ in range(args.warmup):
                C, used = sb.backprojection_streamed(ctx, job, max_bytes, precision=sb.PREC_PRECISE)
            ts = []
            for _ in range(args.steps):
                t0 = time.perf_counter()
                C, used = sb.backprojection_streamed(ctx, job, max_bytes, precision=sb.PREC_PRECISE)
                ts.append(time.perf_counter() - t0)
            return C, used, statistics.median(ts)

        clocks.start()
        C, used, t_cap = timed(cap)
        C1, used1, t_one = timed(1e15)
        # the one-shot call with inputs resident on the device
        dv = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
        t = dict(phs=dv(d["phs"].view(np.float32)), k=dv(d["k_r"].astype(np.float32)),
                 pos=dv(d["pos"].astype(np.float32)), k64=dv(d["k_r"]), pos64=dv(d["pos"]),
                 u=dv(d["u"]), v=dv(d["v"]))
        o = torch.empty((d["nv"], d["nu"], 2), dtype=torch.float64, device=dev)
        jd = sb.make_job(d["S"], d["P"], d["N_fft"], d["taylor"], d["nu"], d["nv"], d["delta_r"],
                         t["phs"].data_ptr(), t["k"].data_ptr(), t["pos"].data_ptr(), o.data_ptr(),
                         u=t["u"].data_ptr(), v=t["v"].data_ptr(), u_hat=d["u_hat"], v_hat=d["v_hat"],
                         k_r64=t["k64"].data_ptr(), pos64=t["pos64"].data_ptr(), precision=sb.PREC_PRECISE)
        for _ in range(args.warmup):
            ctx.run_jobs([jd])
        ctx.synchronize()
        ts = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            ctx.run_jobs([jd])
            ctx.synchronize()
            ts.append(time.perf_counter() - t0)
        t_dev = statistics.median(ts)
        clk = clocks.stop()
    finally:
        ctx.close()
    rate = lambda sec: units / sec / 1e9
    res = {
        "metric": "Gpixel*pulses/s (4096^2 image, 4000 pulses, formed under a %.2f GB device-memory cap)"
                  % (cap / 1e9),
        "value": rate(t_cap), "unit": "Gpixel*pulses/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_cap * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32 (split-precision; f64 per-pulse set-up, PREC_PRECISE)",
        "data": "synthetic (seeded; 40 scatterers at 20 km)",
        "config": {"workload": "streamed: 4096x4096 image, 4000 pulses x 2048 samples, N_fft 8192, "
                               "host buffers (pinned), cap %.2f GB" % (cap / 1e9),
                   "parallelism": "replicas1", "l2": "inputs and outputs > 126 MB L2, no flush"},
        "e2e": {"value": rate(t_cap), "unit": "Gpixel*pulses/s",
                "h2d_bytes_per_step": hj.phs.nbytes + hj.k64.nbytes + hj.p64.nbytes + hj.u.nbytes + hj.v.nbytes,
                "d2h_bytes_per_step": out.nbytes},
        "chunk_pulses": C, "device_bytes_held": used, "one_shot_device_bytes": one_shot,
        "no_cap": {"chunk_pulses": C1, "device_bytes_held": used1, "ms": t_one * 1e3, "rate": rate(t_one)},
        "device_resident_one_shot": {"ms": t_dev * 1e3, "rate": rate(t_dev)},
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(res), flush=True)


def run_resize(args, rank, world, local_rank):
    """--config resize: the reference's data/resize.py resampling of a phase
    history of the one-node Sandia run's shape (1999 x 1800 complex128) to
    twice and to half its pulse and sample counts (resize.py -p 2 -s 2 and
    -p 0.5 -s 0.5), on the device (sarbp_resize_device, the real and
    imaginary parts as two interleaved f64 components; CUDA events on the
    context's stream), beside skimage's resize as restated on scipy in
    oracle/resize_oracle.py (host, one call per part), which also checks
    the device result.  HBM roofline on the input read plus the output
    written once."""
    import torch
    import sarbp_b200 as sb
    from sarbp_b200 import synth
    from sarbp_b200._lib import lib, check
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import resize_oracle as RO

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    d = synth.make("sandia_2048", seed=2 + rank, with_r=False)
    phs = d["phs"].astype(np.complex128)
    P, S = phs.shape
    peaks = {}
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peaks = json.load(f)
    except OSError:
        pass
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    ctx = sb.Context(local_rank)
    st = torch.cuda.current_stream()
    ctx.set_stream(st.cuda_stream)
    cases = []
    try:
        src = torch.from_numpy(phs.view(np.float64)).to(dev)
        for name, (po, so) in (("up2 (-p 2 -s 2)", (2 * P, 2 * S)), ("down2 (-p 0.5 -s 0.5)", (P // 2, S // 2))):
            dst = torch.empty((po, 2 * so), dtype=torch.float64, device=dev)

            def call():
                check(lib().sarbp_resize_device(ctx.handle, 8, 2, ctypes_ptr(src), P, S, po, so, ctypes_ptr(dst)))
            for _ in range(args.warmup):
                call()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            torch.cuda.synchronize()
            e0.record(st)
            for _ in range(args.steps):
                call()
            e1.record(st)
            torch.cuda.synchronize()
            ms = e0.elapsed_time(e1) / args.steps
            got = dst.cpu().numpy().view(np.complex128)
            t0 = time.perf_counter()
            ref = RO.sk_resize(phs.real, (po, so)) + 1j * RO.sk_resize(phs.imag, (po, so))
            cpu_s = time.perf_counter() - t0
            rng_ = max(np.ptp(phs.real), np.ptp(phs.imag))
            err = float(np.max(np.abs(got - ref)) / rng_)
            nbytes = P * S * 16 + po * so * 16
            cases.append({"case": name, "in": [P, S], "out": [po, so], "device_ms": ms,
                          "roofline": {"bound": "hbm", "achieved": nbytes / (ms * 1e-3) / 1e9, "peak": hbm_peak,
                                       "unit": "GB/s", "frac": nbytes / (ms * 1e-3) / 1e9 / hbm_peak,
                                       "traffic": None, "algorithmic_bytes": nbytes},
                          "cpu_ms": cpu_s * 1e3, "cpu_vs_device": cpu_s * 1e3 / ms,
                          "max_abs_diff_over_range": err})
    finally:
        ctx.close()
    res = {
        "metric": "resize device time (ms), phase history 1999x1800 complex128 to twice its size",
        "value": cases[0]["device_ms"], "unit": "ms", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": cases[0]["device_ms"], "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded; the one-node Sandia run's phase-history shape)",
        "config": {"workload": "resize: data/resize.py on a 1999x1800 complex128 phase history",
                   "parallelism": "replicas1", "l2": "inputs and outputs > 126 MB L2 (up2), no flush"},
        "cases": cases,
        "cpu_baseline": {"kind": "port", "cores": 1, "unit": "ms",
                         "sample": "the whole array, scipy.ndimage restatement of skimage's resize",
                         "value": cases[0]["cpu_ms"]},
    }
    if rank == 0:
        print(json.dumps(res), flush=True)


def run_distributed(args, rank, world, local_rank):
    """--config distributed: the reference's -s cuda_distributed schedule
    (backprojection.cpp:239-243) on plain_large through
    sarbp_b200.distributed: each rank forms its block of output rows into a
    device send buffer, NCCL gathers the blocks on rank 0, which copies the
    image to the host once.  One image per step, timed on the host clock
    between barriers (the call ends with rank 0's host copy), max over
    ranks; under torchrun each of N ranks forms nv / N rows (strong
    scaling); without it a one-rank NCCL group.  Rank 0's image is checked
    against the plain device call of the same job (bit for bit at N = 1)."""
    import datetime
    import torch
    import torch.distributed as dist
    import sarbp_b200 as sb
    from sarbp_b200 import synth
    from sarbp_b200.distributed import DeviceCompute, distributed_backprojection

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    own_group = not dist.is_initialized()
    if own_group:
        import socket
        with socket.socket() as so:
            so.bind(("127.0.0.1", 0))
            port = so.getsockname()[1]
        dist.init_process_group("nccl", init_method="tcp://127.0.0.1:%d" % port, rank=0, world_size=1,
                                timeout=datetime.timedelta(seconds=120), device_id=dev)
    try:
        d = synth.make("plain_large", seed=2, with_r=False)
        nu, nv, P = d["nu"], d["nv"], d["P"]
        ctx = sb.Context(local_rank)
        k32, p32 = d["k_r"].astype(np.float32), d["pos"].astype(np.float32)
        comp = DeviceCompute(ctx, d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], d["u"], d["v"], p32,
                             u_hat=d["u_hat"], v_hat=d["v_hat"])
        # rank 0's image lands in page-locked host memory, allocated once
        out = torch.empty((nv, nu, 2), dtype=torch.float64).pin_memory().numpy().view(np.complex128)[..., 0] \
            if rank == 0 else None
        img = None
        for _ in range(args.warmup):
            img = distributed_backprojection(comp, nu, nv, out=out)
        ts = []
        for _ in range(args.steps):
            dist.barrier(device_ids=[local_rank])
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            img = distributed_backprojection(comp, nu, nv, out=out)
            torch.cuda.synchronize()
            ts.append(time.perf_counter() - t0)
        t = torch.tensor([statistics.median(ts)], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        sec = float(t.item())
        same = None
        if rank == 0:
            ref = ctx.backprojection_plane(d["phs"], k32, d["taylor"], d["N_fft"], d["delta_r"], d["u"], d["v"],
                                           d["u_hat"], d["v_hat"], p32)
            same = bool(np.array_equal(img, ref)) if dist.get_world_size() == 1 else \
                float(np.linalg.norm(img - ref) / np.linalg.norm(ref))
        ctx.close()
        n = dist.get_world_size()
        if rank == 0:
            units = float(nu) * nv * P
            print(json.dumps({
                "metric": "Gpixel*pulses/s (2048^2 x 1999, distributed row blocks gathered to rank 0)",
                "value": units / sec / 1e9, "unit": "Gpixel*pulses/s", "n_gpus": n, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": sec * 1e3, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f32 (split-precision; f64 per-pulse set-up)",
                "data": "synthetic (seeded, plain_large shapes)",
                "config": {"workload": "distributed: plain_large, %d output-row block(s), NCCL gather to rank 0, "
                                       "one host copy of the image" % n, "parallelism": "rows%d" % n,
                           "l2": "inputs+outputs > 126 MB L2, no flush"},
                "timing": "host clock between barriers, median of steps, max over ranks",
                "image_vs_plain_call": same,
            }), flush=True)
    finally:
        if own_group:
            dist.destroy_process_group()


def ctypes_ptr(t):
    import ctypes
    return ctypes.c_void_p(t.data_ptr())


def n_fft_of(S, u):
    return int(math.pow(2, int(math.log2(S * u)) + 1))  # sarbp.cpp:258


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        run_reference(args, rank, world)  # rank 0 only, no process group
        return
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local_rank)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=torch.device("cuda", local_rank))
    try:
        import torch
        torch.cuda.set_device(local_rank)
        # one stream for the library, the torch copies and the timing events
        stream = torch.cuda.Stream(device=torch.device("cuda", local_rank))
        with torch.cuda.stream(stream):
            if args.config == "batch96":
                run_batch(args, rank, world, local_rank)
            elif args.config == "serve":
                run_serve(args, rank, world, local_rank)
            elif args.config == "cli_sandia":
                run_cli(args, rank, world, local_rank)
            elif args.config == "streamed":
                run_streamed(args, rank, world, local_rank)
            elif args.config == "resize":
                run_resize(args, rank, world, local_rank)
            elif args.config == "distributed":
                run_distributed(args, rank, world, local_rank)
            else:
                run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()
