#!/usr/bin/env python
"""Benchmark of the B200 spektralab render path: the 4K full render plus reprint workload.

Workload (one step): a 3840 x 2160 float32 linear ProPhoto RGB frame (synthetic, log-uniform in
[2^-8, 2^2], seed 0), synthetic 3-layer negative and paper stocks, halation as a 2-Gaussian mixture of
sigma 20 and 120 px (weight 0.03), scanner lens blur 1.5 px, grain on at a pixel pitch giving a mean
of 600 grains per pixel and sub-layer; one full render (develop + print at print_exposure 1.0), then a
reprint of the device-resident negative at print_exposure 1.2.

  value         steps / device time, one GPU or the whole job (replicas: every rank renders its own
                frames, no collective), time = CUDA events on the session stream, L2 flushed (256 MiB
                written) before every render and reprint, max over ranks
  e2e           the same workload through the C ABI with host buffers: spk_open from pinned host memory
                (host->device copy), spk_render, spk_set_params, spk_reprint, each result copied to
                pinned host memory, wall clock
  roofline      the dominant kernel: algorithmic bytes per launch / its mean CUDA-event duration
  cpu_baseline  the reference engine's own code (oracle/_ref) on this host's cores: three full 4K render
                + reprint steps, with the OpenMP thread count and the host's cores
  --impl reference  the reference engine alone on the host cores, same workload, metric and film format
                (from the reference's own grain set-up); the B200 library is not loaded
"""

from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(REPO, "spektralab-engine_b200"))

import numpy as np  # noqa: E402

import spk_ctypes as sc  # noqa: E402
import synth_resources  # noqa: E402

METRIC = "4K render/reprint frames/s"
UNIT = "frames/s"
W, H = 3840, 2160
BASE = {"film_stock": "synthetic_negative_400", "print_stock": "synthetic_paper", "auto_exposure": False,
        "dir_couplers_active": False, "glare_active": False, "scanner_lens_blur": 1.5}
HALATION = ([((1, 1, 1), (20, 20, 20)), ((1, 1, 1), (120, 120, 120))], (0.03, 0.03, 0.03))
TARGET_GRAINS = 600.0
MEASURED_PEAKS = os.path.join(REPO, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0

# Compulsory HBM bytes per pixel of each kernel in this workload (read + write of its planes; tables
# that stay in L2 are not counted): 12 bytes per RGB float32 plane pass, 8 per RGBA16 pixel.
N_HALATION = len(HALATION[0])
KERNEL_BYTES_PER_PX = {
    "expose": 24, "iir_h": 24, "iir_v": 36, "fir_v": 24, "fir_h": 24, "lincomb": 36, "copy": 24,
    "develop": 24, "develop_layers": 24, "print": 24, "encode": 32, "fir_tile": 24, "scan_encode": 20,
    "iir_rows": 12 + 12 * N_HALATION, "iir_cols": 12 * N_HALATION + 24,
}
N_SM = 148
# From the ncu capture summarised in profiles/render_kernels_2048x2048_ncu.md (one 2048 x 2048 render +
# reprint, --set full): DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) and warp instructions
# (smsp__inst_executed.sum) per pixel of each kernel's launch. Traffic scales with the pixels launched.
NCU_TRAFFIC_PER_PX = {"expose": 14.24, "iir_rows": 25.09, "iir_cols": 53.66,
                      "develop_layers": 13.98, "fir_tile": 14.42, "print": 13.08, "scan_encode": 13.39}
NCU_WARP_INST_PER_PX = {"expose": 10.73, "iir_rows": 18.37, "iir_cols": 11.89,
                        "develop_layers": 149.67, "fir_tile": 6.90, "print": 60.34, "scan_encode": 18.96}


def workload_name():
    return "4K full render + reprint" if (W, H) == (3840, 2160) else f"{W}x{H} full render + reprint"


def film_format_from_counts(counts, p0, long_edge):
    """film_format_mm giving a mean of TARGET_GRAINS grains per sub-layer and pixel, from the grain counts
    of a set-up at pixel pitch p0 (counts scale with the square of the pixel pitch), rounded to 0.1 um of
    film so that both arms open the same parameter set."""
    p = p0 * (TARGET_GRAINS / float(np.mean(counts))) ** 0.5
    return round(p * long_edge / 1000.0, 4)


def film_format_for_grains(lib, resources, long_edge):
    """The film format of the workload from this library's set-up."""
    p0 = 10.0
    out = ctypes.c_char_p()
    lib.check(lib.lib.spkx_setup_json(resources.encode(), json.dumps(BASE).encode(), p0, ctypes.byref(out)))
    return film_format_from_counts(lib.take_json(out)["f64"]["grain_count"], p0, long_edge)


def hbm_peak():
    try:
        with open(MEASURED_PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured (MEASURED_PEAKS.json hbm_gbs)"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback (no MEASURED_PEAKS.json: an earlier copy measurement on this B200 type)"


class Clocks:
    """nvidia-smi samples every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                          "-lms", "100", "-i", str(self.device)], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
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
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def dist_init(gpus, backend="nccl"):
    """One rank per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE / MASTER_*): (rank, local rank, world,
    process group or None, the device the group's tensors live on). backend "gloo" runs the same steps on
    the CPU (the tests' two-process check)."""
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    pg = None
    device = f"cuda:{local}" if backend == "nccl" else "cpu"
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
        pg = dist
    return rank, local, world, pg, device


def reduce_max(pg, device, value):
    """The maximum of value over the ranks (every rank gets it)."""
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg, device):
    if pg is None:
        return
    import torch
    if device.startswith("cuda"):
        idx = int(device.split(":")[1])
        pg.barrier(device_ids=[idx])
        torch.cuda.synchronize(idx)
    else:
        pg.barrier()


def replica_throughput(world, steps, dev_ms_max):
    """frames/s of the whole job: every rank renders and reprints `steps` frames of its own; the job takes
    the slowest rank's device time (replicas: no exchange between ranks)."""
    return world * steps / (dev_ms_max / 1000.0)


def host_threads():
    """(OpenMP threads the reference engine's parallel loops use, host cores this process may run on)."""
    try:
        omp = int(ctypes.CDLL("libgomp.so.1").omp_get_max_threads())
    except (OSError, AttributeError):
        omp = None
    try:
        nproc = len(os.sched_getaffinity(0))
    except AttributeError:
        nproc = os.cpu_count()
    return omp, nproc


def cpu_reference_run(resources, steps, warmup):
    """The reference engine alone (oracle/_ref: its own stage code and kernels built for the CPU, OpenMP over
    each kernel's grid) on the full workload: open the 3840 x 2160 frame with the workload's parameters,
    then per step a render (develop + print at print_exposure 1.0) and a reprint of its negative at 1.2.
    The film format comes from the reference's own grain set-up; nothing of the B200 library is loaded.
    Returns (frames/s, seconds per step, OpenMP threads, host cores, film format)."""
    ref = sc.load_reference()
    eng = ref.engine(resources)
    p0 = 10.0
    out = ctypes.c_char_p()
    ref.check(ref.lib.spkref_setup_json(eng.h, json.dumps(BASE).encode(), p0, ctypes.byref(out)))
    ff = film_format_from_counts(ref.take_json(out)["grain_count"], p0, W)
    img = sc.synthetic_image(W, H, 0)
    delta = dict(BASE, film_format_mm=ff)
    comps, strength = HALATION
    wts = (ctypes.c_double * 6)(*[float(v) for c in comps for v in c[0]])
    sig = (ctypes.c_double * 6)(*[float(v) for c in comps for v in c[1]])
    st = (ctypes.c_double * 3)(*strength)
    s = ref.lib.spkref_open(eng.h, img.ctypes.data_as(sc.FP), W, H, json.dumps(delta).encode(), 2, wts, sig, st)
    if not s:
        raise RuntimeError(ref.last_error())
    rgba = np.zeros((H, W, 4), np.uint16)
    rp = rgba.ctypes.data_as(ctypes.POINTER(ctypes.c_uint16))
    times = []
    for i in range(warmup + steps):
        t0 = time.perf_counter()
        ref.check(ref.lib.spkref_develop(s))
        ref.check(ref.lib.spkref_print(s, 1.0, rp))
        ref.check(ref.lib.spkref_print(s, 1.2, rp))
        if i >= warmup:
            times.append(time.perf_counter() - t0)
    ref.lib.spkref_close(s)
    eng.close()
    omp, nproc = host_threads()
    t = sum(times) / len(times)
    return 1.0 / t, t, omp, nproc, ff


def run_reference(args):
    """--impl reference: the reference engine's CPU build on this host's cores, the same 4K render + reprint
    workload, metric and units as the B200 arm; rank 0 alone (the other ranks exit without work)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    resources = synth_resources.ensure(sc.RESOURCES)
    steps = max(args.steps, 1)
    fps, t, omp, nproc, ff = cpu_reference_run(resources, steps, args.warmup)
    sample = (f"{steps} full {W}x{H} render + reprint steps (print_exposure 1.0 then 1.2), after {args.warmup} "
              f"untimed; {omp} OpenMP threads on {nproc} host cores")
    line = {"impl": "reference", "metric": METRIC, "value": fps, "unit": UNIT, "n_gpus": 0, "steps": steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * t, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(ff, 1),
            "cpu_baseline": {"value": fps, "unit": UNIT, "cores": omp, "nproc": nproc, "kind": "reference",
                             "sample": sample},
            "e2e": {"value": fps, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def workload_config(ff, world):
    return {"workload": workload_name(), "width": W, "height": H, "halation_sigma_px": [20, 120],
            "halation_weight": 0.03, "scanner_lens_blur_px": 1.5, "grains_per_px": TARGET_GRAINS,
            "film_format_mm": ff, "parallelism": f"replicas{world}",
            "l2": "flushed (256 MiB write) before each step"}


def run_e2e(args, eng, img, delta, pg, dev, world):
    """The workload through the C ABI with host buffers: spk_open from pinned host memory, spk_render,
    spk_set_params, spk_reprint, both results copied to pinned host memory and read in place."""
    import torch

    pinned = torch.empty((H, W, 3), dtype=torch.float32, pin_memory=True).numpy()
    pinned[...] = img

    def e2e_step():
        # spk_open copies the frame from pinned host memory; spk_render / spk_reprint copy each result to
        # pinned host memory (the pixels are read in place, as a caller of the C ABI reads them)
        with eng.open(pinned, delta) as s:
            s.set_halation(*HALATION)
            with s.render_result("full") as a:
                s.set_params({"print_exposure": 1.2})
                with s.render_result("full", reprint=True) as b:
                    checksum = int(a.pixels[H // 2, W // 2, 1]) + int(b.pixels[H // 2, W // 2, 1])
                    return a.row_stride_px, checksum

    for _ in range(args.warmup):
        e2e_step()
    barrier(pg, dev)
    t0 = time.perf_counter()
    stride = 0
    for _ in range(args.steps):
        stride, _ = e2e_step()
    e2e_s = reduce_max(pg, dev, time.perf_counter() - t0)
    barrier(pg, dev)
    e2e = {"value": world * args.steps / e2e_s, "unit": UNIT, "h2d_bytes_per_step": W * H * 3 * 4,
           "d2h_bytes_per_step": 2 * stride * H * 8}
    return e2e


VJP_SIZE = 1024
VJP_SEED = 7
VJP_HALATION = ([((0.02, 0.02, 0.02), (8, 8, 8)), ((0.02, 0.02, 0.02), (40, 40, 40))], (0.03, 0.03, 0.03))
# print_exposure, m_filter_shift, y_filter_shift, 2 halation weights, 2 halation sigmas, then 16
# density-curve parameters per film layer (hat functions over each layer's curve table)
VJP_PARAMS = 7 + 48


def run_vjp(args):
    """The render's adjoint (spk_render_vjp) on a 1024 x 1024 frame: the scanned linear RGB with the grain
    held fixed (film seed 7), the gradient of an L2 loss against a target rendered with perturbed
    parameters, with respect to the frame and 55 parameters. Wall time per call through the C ABI (host
    arrays in and out); the forward-only call (output alone) beside it."""
    resources = synth_resources.ensure(sc.RESOURCES)
    lib = sc.load()
    n = VJP_SIZE
    ff = film_format_for_grains(lib, resources, n)
    delta = dict(BASE, film_format_mm=ff)
    eng = lib.engine(resources, device=0)
    img = sc.synthetic_image(n, n, VJP_SEED)
    with eng.open(img, dict(delta, print_exposure=1.1)) as t:
        t.set_halation([((0.025,) * 3, (8, 8, 8)), ((0.015,) * 3, (44, 44, 44))], VJP_HALATION[1])
        target = t.render_linear(VJP_SEED)
    with eng.open(img, delta) as s:
        s.set_halation(*VJP_HALATION)
        y = s.render_linear(VJP_SEED)
        gy = y - target
        for _ in range(args.warmup):
            s.render_vjp(gy, VJP_SEED, VJP_PARAMS)
        fwd, bwd = [], []
        with Clocks(0) as clk:
            for _ in range(args.steps):
                t0 = time.perf_counter()
                s.render_linear(VJP_SEED)
                t1 = time.perf_counter()
                gx, gp = s.render_vjp(gy, VJP_SEED, VJP_PARAMS)
                t2 = time.perf_counter()
                fwd.append(t1 - t0)
                bwd.append(t2 - t1)
    eng.close()
    ms = 1000.0 * statistics.median(bwd)
    line = {"metric": "VJP ms/frame", "value": ms, "unit": "ms", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "render adjoint, 1024x1024, grain fixed (seed 7)", "width": n, "height": n,
                       "params": ["print_exposure", "m_filter_shift", "y_filter_shift", "halation_weight_0",
                                  "halation_weight_1", "halation_sigma_0", "halation_sigma_1"] +
                                 [f"curve_{c}_{j}" for c in range(3) for j in range(16)],
                       "halation_sigma_px": [8, 40]},
            "forward_ms": 1000.0 * statistics.median(fwd),
            "note": "wall time per spk_render_vjp call with host arrays (forward recomputed inside); "
                    "gradient accuracy is checked against binary64 central differences in tests/test_gpu_vjp.py",
            "grad_params": [float(v) for v in gp[:7]], "grad_curve_l1": float(np.abs(gp[7:]).sum()),
            "grad_input_l2": float(np.sqrt(np.sum(gx.astype(np.float64) ** 2))), "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


PREC_W, PREC_H = 6144, 4096
PREC_SEED = 0
PREC_MODES = ("fp32", "tf32", "bf16", "bf16x3", "fp64")


def tensor_flops_per_px(mode, bins):
    """Tensor-core FLOPs the spectral-mode kernel issues per pixel (both integrals): M x N x K MMAs with
    N = 16 and K the wavelengths padded to 32, twice for the BF16 hi + lo split of the A operand."""
    if mode not in ("tf32", "bf16", "bf16x3"):
        return 0
    k = (bins + 31) // 32 * 32
    return 2 * 2 * 16 * k * (2 if mode == "bf16x3" else 1)


def run_precision(args):
    """The print's spectral integrals in each arithmetic on a 6144 x 4096 frame of dye densities (uniform
    in [0, 3], seed 0), at 81 (5 nm) and 401 (1 nm) wavelengths. Per mode: the print kernel's device time
    (CUDA events around its launch, inputs resident on the device, L2 flushed before each call) and the
    error against the same print with both integrals in binary64 (mode fp64): the enlarger integral's
    max and mean over pixels of max_k |R - R64| / max_k |R64|, and the 16-bit output after the scan
    (LSB16). fp32 at 81 wavelengths is the binary32 print kernel, its integral taken from the
    spectral-mode kernel's binary32 path (the same operations); at 401 it is that path."""
    import torch

    resources = synth_resources.ensure(sc.RESOURCES)
    lib = sc.load()
    eng = lib.engine(resources, device=0)
    torch.cuda.set_device(0)
    w = args.width if args.width != 3840 else PREC_W
    h = args.height if args.height != 2160 else PREC_H
    gen = torch.Generator(device="cuda")
    gen.manual_seed(PREC_SEED)
    neg = torch.rand((h, w, 3), generator=gen, device="cuda", dtype=torch.float32) * 3.0
    stride = (w + 31) // 32 * 32
    out = torch.empty((h, stride, 4), dtype=torch.int16, device="cuda")
    ref_out = torch.empty_like(out)
    scratch = torch.empty_like(out)
    con = torch.empty((h, w, 3), dtype=torch.float32, device="cuda")
    ref_con = torch.empty_like(con)
    flush = torch.empty(64 << 20, dtype=torch.int32, device="cuda")
    mpx = w * h / 1e6
    s = eng.open(sc.synthetic_image(64, 48, 5), dict(BASE, grain_active=False))

    def run(mode, bins, contraction, rgba):
        s.set_print_mode(mode, bins)
        return s.print_negative(neg.data_ptr(), w, h, rgba.data_ptr(), stride,
                                contraction.data_ptr() if contraction is not None else None)

    def errors(R, rgba):
        R64 = ref_con.double()
        rel = (R.double() - R64).abs().amax(-1) / R64.abs().amax(-1)
        d = ((rgba[:, :w, :3].int() & 0xFFFF) - (ref_out[:, :w, :3].int() & 0xFFFF)).abs()
        return {"integral_rel_max": float(rel.max()), "integral_rel_mean": float(rel.mean()),
                "lsb16_max": int(d.max()), "lsb16_mean": float(d.float().mean()),
                "lsb16_frac_gt1": float((d > 1).float().mean())}

    modes = [m for m in args.modes.split(",") if m] if args.modes else list(PREC_MODES)
    bins_list = [int(b) for b in args.bins.split(",") if b]
    table = {}
    with Clocks(0) as clk:
        for bins in bins_list:
            run("fp64", bins, ref_con, ref_out)
            for mode in modes:
                times = []
                for k in range(args.warmup + args.steps):
                    flush.fill_(k)
                    ms = run(mode, bins, None, out)
                    if k >= args.warmup:
                        times.append(ms)
                row = {"print_ms": statistics.median(times)}
                row["mpx_s"] = mpx / (row["print_ms"] / 1000.0)
                tf = tensor_flops_per_px(mode, bins) * w * h
                if tf:
                    row["tensor_tflops_issued"] = tf / (row["print_ms"] / 1000.0) / 1e12
                if mode != "fp64":
                    if mode == "fp32" and bins == 81:
                        run("fp32_generic", bins, con, scratch)
                    else:
                        run(mode, bins, con, out)
                    row.update(errors(con, out))
                table[f"{mode}@{bins}"] = row
    s.close()
    eng.close()
    torch.cuda.synchronize()
    head = table.get("bf16x3@81") or next(iter(table.values()))
    head_key = "bf16x3@81" if "bf16x3@81" in table else next(iter(table))
    try:
        with open(MEASURED_PEAKS) as f:
            tpeak, tkind = float(json.load(f)["bf16_tflops"]), "measured (MEASURED_PEAKS.json bf16_tflops)"
    except (OSError, KeyError, ValueError):
        tpeak, tkind = 1590.0, "fallback (no MEASURED_PEAKS.json: an earlier cuBLAS bf16 measurement on this B200 type)"
    line = {"metric": "print Mpx/s, split-BF16 tensor cores, 81 wavelengths" if head_key == "bf16x3@81"
            else f"print Mpx/s, {head_key}", "value": head["mpx_s"],
            "unit": "Mpx/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": head["print_ms"], "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "bf16x3", "data": "synthetic",
            "config": {"workload": f"print spectral integrals, {w}x{h} dye densities uniform [0, 3] (seed 0), "
                                   "81 and 401 wavelengths", "width": w, "height": h,
                       "l2": "flushed (256 MiB write) before each call"},
            "modes": table,
            "roofline": {"bound": "tensor", "achieved": head.get("tensor_tflops_issued", 0.0), "peak": tpeak,
                         "unit": "TFLOP/s", "frac": head.get("tensor_tflops_issued", 0.0) / tpeak, "traffic": None,
                         "kernel": f"print_spectral ({head_key})", "peak_source": tkind,
                         "note": "tensor FLOPs issued (N padded to 16, K to 32); the kernel is bound by "
                                 "the exponentials and operand splits on the CUDA cores"},
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


BATCH_FRAMES = 64
BATCH_SEED = 3


def batch_workload():
    """64 frames, sizes uniform in [256, 4096] x [256, 2732], print_exposure uniform in [0.7, 1.4], a
    halation sigma pair (sigma0 in [5, 30], sigma1 in [40, 160] px, weight 1 each, strength 0.03), seed 3."""
    rng = np.random.default_rng(BATCH_SEED)
    frames = []
    for i in range(BATCH_FRAMES):
        w, h = int(rng.integers(256, 4097)), int(rng.integers(256, 2733))
        ex = float(rng.uniform(0.7, 1.4))
        s0, s1 = float(rng.uniform(5, 30)), float(rng.uniform(40, 160))
        frames.append((w, h, ex, s0, s1))
    return frames


def run_batch(args):
    """Batched renders (spkx_render_batch) of 64 frames of mixed sizes, then 64 batched reprints, against
    the same frames through per-frame spk_render / spk_reprint calls. Aggregate megapixels/s over wall
    time (results in pinned host memory); per-frame latency: a plain call's wall time, a batched frame's
    completion on the device from the batch's start."""
    resources = synth_resources.ensure(sc.RESOURCES)
    lib = sc.load()
    eng = lib.engine(resources, device=0)
    frames = batch_workload()
    mpx = sum(w * h for w, h, *_ in frames) / 1e6
    images = [sc.synthetic_image(w, h, i) for i, (w, h, *_) in enumerate(frames)]

    def open_all():
        ss = []
        for img, (w, h, ex, s0, s1) in zip(images, frames):
            s = eng.open(img, dict(BASE, film_format_mm=35.0, print_exposure=ex))
            s.set_halation([((1, 1, 1), (s0,) * 3), ((1, 1, 1), (s1,) * 3)], (0.03, 0.03, 0.03))
            ss.append(s)
        return ss

    def reprint_exposures(ss):
        for s, (w, h, ex, *_) in zip(ss, frames):
            s.set_params({"print_exposure": min(1.4, ex * 1.1)})

    def plain(ss, reprint):
        lat = []
        t0 = time.perf_counter()
        for s in ss:
            a = time.perf_counter()
            with s.render_result("full", reprint=reprint):
                pass
            lat.append(1000.0 * (time.perf_counter() - a))
        return time.perf_counter() - t0, lat

    def batched(ss, reprint):
        t0 = time.perf_counter()
        res, info = eng.render_batch(ss, "full", reprint=reprint)
        wall = time.perf_counter() - t0
        for r in res:
            r.free()
        return wall, info

    # warm-up and tuning: one plain pass and one batched pass of the same shape, untimed
    tuning = {}
    for mode in ("plain", "batch"):
        ss = open_all()
        if mode == "plain":
            plain(ss, False)
        else:
            _, tuning["render"] = batched(ss, False)
            reprint_exposures(ss)
            _, tuning["reprint"] = batched(ss, True)
        for s in ss:
            s.close()
    with Clocks(0) as clk:
        ss = open_all()
        p_render, lat_pr = plain(ss, False)
        reprint_exposures(ss)
        p_reprint, lat_pp = plain(ss, True)
        for s in ss:
            s.close()
        ss = open_all()
        b_render, info_r = batched(ss, False)
        reprint_exposures(ss)
        b_reprint, info_p = batched(ss, True)
        for s in ss:
            s.close()
    eng.close()

    def pct(v):
        return {"p50": float(np.percentile(v, 50)), "p99": float(np.percentile(v, 99))}

    line = {"metric": "batched render megapixels/s", "value": mpx / b_render, "unit": "Mpx/s", "n_gpus": 1,
            "steps": 1, "warmup": 1, "ms_per_step": 1000.0 * b_render, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "64 frames 256x256..4096x2732 (seed 3), render then reprint", "frames": BATCH_FRAMES,
                       "megapixels": mpx, "print_exposure": "uniform [0.7, 1.4]",
                       "halation_sigma_px": "uniform [5, 30] and [40, 160]"},
            "render": {"batched_mpx_s": mpx / b_render, "plain_mpx_s": mpx / p_render,
                       "batched_ms": 1000.0 * b_render, "plain_ms": 1000.0 * p_render,
                       "latency_ms_batched": pct(info_r["frame_done_ms"]), "latency_ms_plain": pct(lat_pr),
                       "plan": info_r.get("plan"),
                       "tuning_candidates_ms": tuning["render"].get("candidates_ms")},
            "reprint": {"batched_mpx_s": mpx / b_reprint, "plain_mpx_s": mpx / p_reprint,
                        "batched_ms": 1000.0 * b_reprint, "plain_ms": 1000.0 * p_reprint,
                        "latency_ms_batched": pct(info_p["frame_done_ms"]), "latency_ms_plain": pct(lat_pp),
                        "plan": info_p.get("plan"),
                        "tuning_candidates_ms": tuning["reprint"].get("candidates_ms")},
            "clocks": clk.summary()}
    print(json.dumps(line), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true", help="skip the end-to-end leg (profiling runs)")
    ap.add_argument("--width", type=int, default=3840, help="frame width (the benchmark workload is 3840)")
    ap.add_argument("--height", type=int, default=2160, help="frame height (the benchmark workload is 2160)")
    ap.add_argument("--modes", default="", help="precision: comma-separated print modes (default all)")
    ap.add_argument("--bins", default="81,401", help="precision: comma-separated wavelength counts (81, 401)")
    ap.add_argument("--config", default="render", choices=["render", "vjp", "batch", "precision"],
                    help="render: the 4K render + reprint (the headline); vjp: the render's adjoint on 1024x1024; "
                         "batch: 64 frames of mixed sizes, batched against per-frame calls; precision: the "
                         "print's spectral integrals in fp32 / tf32 / bf16 / split bf16 against binary64 on "
                         "6144x4096 densities")
    args = ap.parse_args()
    global W, H
    W, H = args.width, args.height
    if args.impl == "reference":
        return run_reference(args)
    args.warmup = max(args.warmup, 3)
    if args.config == "vjp":
        return run_vjp(args)
    if args.config == "batch":
        return run_batch(args)
    if args.config == "precision":
        return run_precision(args)

    rank, local, world, pg, dev = dist_init(args.gpus)
    resources = synth_resources.ensure(sc.RESOURCES)
    lib = sc.load()
    ff = film_format_for_grains(lib, resources, W)
    delta = dict(BASE, film_format_mm=ff)
    eng = lib.engine(resources, device=local)
    img = sc.synthetic_image(W, H, rank)

    # ---- device throughput ----
    sess = eng.open(img, delta)
    sess.set_halation(*HALATION)
    sess.set_params({"print_exposure": 1.0})
    sess.profile("full", False, args.warmup)
    sess.set_params({"print_exposure": 1.2})
    sess.profile("full", True, args.warmup)
    sess.set_params({"print_exposure": 1.0})
    barrier(pg, dev)
    # clocks are sampled every 100 ms from one second of untimed load before the timed steps to their end
    with Clocks(local) as clk:
        t_heat = time.perf_counter()
        while time.perf_counter() - t_heat < 1.0:
            sess.profile("full", False, 1)
        barrier(pg, dev)
        t0 = time.perf_counter()
        pr = sess.profile("full", False, args.steps)
        sess.set_params({"print_exposure": 1.2})
        pp = sess.profile("full", True, args.steps)
        wall = time.perf_counter() - t0
    barrier(pg, dev)
    dev_ms = sum(pr["total_ms"]) + sum(pp["total_ms"])
    dev_ms_max = reduce_max(pg, dev, dev_ms)
    value = replica_throughput(world, args.steps, dev_ms_max)
    render_ms = sum(pr["total_ms"]) / args.steps
    reprint_ms = sum(pp["total_ms"]) / args.steps
    launches = int(pr["launches"] + pp["launches"])

    # per-kernel times and the roofline of the dominant kernel
    kern = {}
    for prof in (pr, pp):
        for name, ms in prof["kernels"].items():
            k = kern.setdefault(name, [])
            k.extend(ms)
    table = {n: {"launches": len(v), "total_ms": sum(v), "mean_ms": sum(v) / len(v)} for n, v in kern.items()}
    dom = max(table, key=lambda n: table[n]["total_ms"])
    peak, peak_kind = hbm_peak()
    clk_sum = clk.summary()
    sm_ghz = (clk_sum["sm_mhz"] or 1965.0) / 1000.0
    issue_peak = N_SM * 4 * sm_ghz  # G warp-instructions/s: four schedulers per SM, one issue each per clock
    for n, t in table.items():
        t["hbm_gbs"] = KERNEL_BYTES_PER_PX.get(n, 24) * W * H / (t["mean_ms"] / 1000.0) / 1e9
        t["hbm_frac"] = t["hbm_gbs"] / peak
        if n in NCU_WARP_INST_PER_PX:
            t["issue_frac"] = NCU_WARP_INST_PER_PX[n] * W * H / (t["mean_ms"] / 1000.0) / 1e9 / issue_peak
    bytes_launch = KERNEL_BYTES_PER_PX.get(dom, 24) * W * H
    achieved = bytes_launch / (table[dom]["mean_ms"] / 1000.0) / 1e9
    traffic = NCU_TRAFFIC_PER_PX.get(dom)
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic * W * H if traffic else None, "kernel": dom,
                "algorithmic_bytes_per_launch": bytes_launch, "peak_source": peak_kind,
                # the render kernels are instruction-bound, not HBM-bound: the fraction of the SMs' issue
                # rate the kernel sustains (warp instructions per pixel from its ncu capture, the launch time
                # measured here, peak = 4 warp instructions per SM per clock at the sampled SM clock)
                "issue_frac": table[dom].get("issue_frac"),
                "step_hbm_gbs": (sum(KERNEL_BYTES_PER_PX.get(n, 24) * t["launches"] for n, t in table.items())
                                 * W * H / args.steps) / (dev_ms_max / args.steps / 1000.0) / 1e9}
    stage_ms = {}
    for prof in (pr, pp):
        for name, ms in prof["stages"].items():
            stage_ms[name] = stage_ms.get(name, 0.0) + sum(ms) / args.steps
    sess.close()

    # ---- end to end through the C ABI with host buffers ----
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(args, eng, img, delta, pg, dev, world)
    eng.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and os.path.exists(sc.REF_PATH):
        fps, t, omp, nproc, _ = cpu_reference_run(resources, steps=3, warmup=1)
        cpu = {"value": fps, "unit": UNIT, "cores": omp, "nproc": nproc, "kind": "reference",
               "sample": f"3 full {W}x{H} render + reprint steps after 1 untimed ({t:.2f} s per step), "
                         f"{omp} OpenMP threads on {nproc} host cores"}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": dev_ms_max / args.steps, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
                "config": workload_config(ff, world),
                "render_ms": render_ms, "reprint_ms": reprint_ms,
                "render_fps": 1000.0 / render_ms, "reprint_fps": 1000.0 / reprint_ms,
                "wall_s_timed": wall, "stage_ms": stage_ms, "kernels": table,
                "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
                "clocks": clk_sum}
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
