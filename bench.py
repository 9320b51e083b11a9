#!/usr/bin/env python3
"""Benchmark: span-3 HRRT OP-OSEM subset-iterations per second on B200.

Workload (the reference's span-3 configuration): HRRT model 999, span 3,
maxdel 67 (45 segments, 6367 planes x 288 views x 256 bins), image 256x256x207
at 1.21875 mm, 16 subsets, synthetic phantom study (seed 1 + rank, 3e8 counts,
per-bin lognormal norm sigma 0.1, scatter 15% of trues, randoms 25%).

One step = one OSEM subset-iteration: forward projection + OP ratio of the 9
view pairs of a subset, their back projection, rotate-back and the
multiplicative update (hrrt_osem3d_span3.cpp:4161-4260).

  value : device-resident throughput (inputs, sensitivity and image in HBM).
  e2e   : one full reconstruction through the C ABI (hrrt_reconstruct) from
          pinned host buffers (upload of prompts/randoms/norm/atten/scatter,
          sensitivity, 2 iterations x 16 subsets, image read back),
          subset-iterations per second of device time (CUDA events).

--impl reference times the reference's own CPU projector
(oracle/_ref/libhrrt_ref.so: forward_proj3d_thread1 / back_proj3d_thread1 /
rotate_image_buf and the -T thread grouping of CalculateOsem3d) on the host
cores, one OSEM subset per step.
With torchrun (N>1) every rank reconstructs its own frame (replicas, weak
scaling); there is no data-path collective.
"""
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

SPAN = 3
SUBSETS = 16
ITERATIONS = 2
METRIC = "span-3 OSEM subset-iters/s"
UNIT = "subset-iters/s"
STUDY = dict(total_counts=3e8, randoms_frac=0.25, scatter_frac=0.15, norm_sigma=0.1)


GEOMETRY = "hrrt"


def geom_dict():
    """HRRT model 999 at span 3; `--geometry small` selects a 24-ring test
    scanner that only the multi-process plumbing tests use."""
    if GEOMETRY == "small":
        return dict(nrings=24, nelements=64, nangles=96, ring_radius=58.625, plane_sep=1.21875, binsize=1.21875,
                    span=3, maxdel=13, subsets=SUBSETS)
    return dict(nrings=104, nelements=256, nangles=288, ring_radius=234.5, plane_sep=1.21875, binsize=1.21875,
                span=SPAN, maxdel=67, subsets=SUBSETS)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def init_dist(ws, backend):
    if ws <= 1:
        return None
    import datetime

    import torch.distributed as dist
    dist.init_process_group(backend=backend, timeout=datetime.timedelta(seconds=600))
    return dist


def barrier(dist, device=None):
    if dist is not None:
        if device is not None:
            dist.barrier(device_ids=[device])
        else:
            dist.barrier()


def max_over_ranks(dist, v, device=None):
    if dist is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=f"cuda:{device}" if device is not None else "cpu")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


class ClockSampler:
    """SM clocks and throttle reasons sampled while the timed region runs:
    through NVML every 10 ms (read-only queries), else nvidia-smi every
    200 ms."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.lines = []
        self.nvml = None
        self.samples = []  # (sm MHz, max MHz, reasons)
        self.stop_flag = threading.Event()

    def _nvml_handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        pr = torch.cuda.get_device_properties(self.device)
        bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
        return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus)

    def _poll(self):
        pynvml, h = self.nvml
        bits = {"hw_slowdown": pynvml.nvmlClocksThrottleReasonHwSlowdown,
                "hw_thermal_slowdown": pynvml.nvmlClocksThrottleReasonHwThermalSlowdown,
                "sw_thermal_slowdown": pynvml.nvmlClocksThrottleReasonSwThermalSlowdown,
                "sw_power_cap": pynvml.nvmlClocksThrottleReasonSwPowerCap}
        while not self.stop_flag.is_set():
            try:
                sm = pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM)
                mx = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
                r = pynvml.nvmlDeviceGetCurrentClocksThrottleReasons(h)
                self.samples.append((float(sm), float(mx), {n for n, b in bits.items() if r & b}))
            except Exception:
                break
            self.stop_flag.wait(0.01)

    def start(self):
        try:
            self.nvml = self._nvml_handle()
            self.t = threading.Thread(target=self._poll, daemon=True)
            self.t.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml is not None:
            self.stop_flag.set()
            self.t.join(timeout=5)
            if not self.samples:
                return None
            sm = [a for a, _, _ in self.samples]
            reasons = set().union(*(r for _, _, r in self.samples))
            return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": self.samples[-1][1], "reasons": sorted(reasons),
                    "samples": len(sm), "source": "nvml, 10 ms"}
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for n, v in zip(self.NAMES, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm),
                "source": "nvidia-smi, 200 ms"}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


FP32_TFLOPS_NOMINAL = 148 * 128 * 2 * 1.965e9 / 1e12


def ncu_traffic(kernel):
    """DRAM bytes (read + write) per launch of `kernel` at this workload, from
    the committed ncu summary profiles/traffic.txt (lines
    `<kernel> <bytes per launch> <source>`), or None."""
    p = os.path.join(ROOT, "profiles", "traffic.txt")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            parts = line.split(None, 2)
            if len(parts) >= 2 and parts[0] == kernel and not line.startswith("#"):
                try:
                    return float(parts[1]), (parts[2].strip() if len(parts) > 2 else "profiles/traffic.txt")
                except ValueError:
                    return None
    return None


def algorithmic_model(info, add_bytes=4):
    """Per-launch algorithmic bytes and FLOPs of the subset kernels.

    Bins per subset: 9 view pairs x 2 views x segmentsize x nbins.
    fp_kernel : image read once (nx*ny*nz*4) + prompts (2 B) + additive term
                (4 B, or 2 B stored as bf16) read + OP ratio (4 B) written
                per bin; FLOPs = 6 per
                lerp sample (2 adds, 2 muls, 2 accumulating adds for a sample
                pair, i.e. 3 per sample) x samples.
    bp_kernel : ratio read (4 B/bin) + correction image written once
                (nx*ny*nz*4); FLOPs = 4 per lerp sample (p + f*(q-p), summed).
    rotback_kernel: correction read + image read/write + inverse sensitivity
                read (4 image volumes).
    """
    nb = info.nbins
    pairs = info.sviews // 2
    bins = pairs * 2 * info.segmentsize * nb
    vol = info.nx * info.ny * info.nz * 4
    # lerp samples: every FOV column of every view contributes one sample to
    # every plane of its ray's segments
    samples = pairs * 2 * info.fov_columns * info.segmentsize
    return {
        "bins_per_subset": bins,
        "fp_kernel": {"bytes": vol + bins * (6 + add_bytes), "flops": samples * 3, "smem_bytes": samples * 8},
        "bp_kernel": {"bytes": bins * 4 + vol, "flops": samples * 4},
        "rotback_kernel": {"bytes": 4 * vol, "flops": info.fov_columns * info.zp * pairs * 16},
        # prompts + additive term read, ratio written and read back, image
        # read, inverse sensitivity read, image written
        "subset_bytes": bins * (2 + add_bytes + 8) + 3 * vol,
    }


DATA = "synthetic (seeded phantom study, Poisson prompts)"


def bench_config(storage, ws):
    """The workload both arms (ours and --impl reference) are measured on."""
    return {"workload": "HRRT span 3 (45 segments, 6367 planes x 288 views x 256 bins), image 256x256x207, "
                        "16 subsets, OP-OSEM (-W 3), 3e8 counts, lognormal norm 0.1, scatter 15%, randoms 25%",
            "parallelism": f"replicas x{ws}" if ws > 1 else "1 GPU",
            "l2": "inputs larger than L2 (1.9 GB prompts+additive per frame; 117 MB ratio per subset)",
            "storage": storage}


_PINNED = []  # page-locked tensors behind the numpy views handed to the C ABI


def pinned_copy(torch, a):
    """A numpy view of page-locked host memory holding a copy of `a`."""
    t = torch.empty(a.shape, dtype=getattr(torch, a.dtype.name), pin_memory=True)
    _PINNED.append(t)
    out = t.numpy()
    out[...] = a
    return out


def run_ours(args, ws, rank, local):
    import torch
    dist = init_dist(ws, "nccl")
    torch.cuda.set_device(local)
    import hrrt_reconstruction_b200 as H
    from hrrt_reconstruction_b200 import phantom

    geom = H.hrrt_geometry(**geom_dict())
    ctx = H.Context(geom, device=local)
    storage = H.STORE_16 if args.storage == "16" else H.STORE_F32
    t0 = time.time()
    st = phantom.study(ctx, seed=1 + rank, **STUDY)
    gen_s = time.time() - t0

    # ---- end-to-end through the C ABI from pinned host buffers ----
    e2e_subsets = ITERATIONS * SUBSETS
    names = ("prompts", "randoms", "norm", "atten", "scatter")
    host = {k: pinned_copy(torch, st[k]) for k in names if st[k] is not None}
    info = ctx.info
    img = pinned_copy(torch, np.zeros((info.nz, info.ny, info.nx), np.float32))
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    cs = torch.cuda.ExternalStream(ctx.stream)
    # one untimed pass sizes the library's staging buffers
    ctx.reconstruct(*(host.get(k) for k in names), storage=storage, iterations=1, out=img)
    barrier(dist, local)
    torch.cuda.synchronize()
    ev[0].record(cs)
    _, stats = ctx.reconstruct(*(host.get(k) for k in names), storage=storage, iterations=ITERATIONS, out=img)
    ev[1].record(cs)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(dist, ev[0].elapsed_time(ev[1]), local)
    h2d = sum(int(a.nbytes) for a in host.values())
    d2h = int(img.nbytes)
    e2e = {"value": ws * e2e_subsets / (e2e_ms / 1e3), "unit": UNIT,
           "h2d_bytes_per_step": h2d // e2e_subsets, "d2h_bytes_per_step": d2h // e2e_subsets,
           "ms_total": e2e_ms, "subset_iterations": e2e_subsets, "sum_image": stats.sum_image}

    # ---- device-resident steps ----
    ctx.init_image()
    ctx.osem_subsets(0, args.warmup)
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    barrier(dist, local)
    torch.cuda.synchronize()
    clocks.start()
    ctx.reset_kernel_stats()
    ctx.set_profiling(True)
    ev[0].record(cs)
    ctx.osem_subsets(args.warmup, args.steps)
    ev[1].record(cs)
    torch.cuda.synchronize()
    ctx.set_profiling(False)
    clk = clocks.stop()
    ms = max_over_ranks(dist, ev[0].elapsed_time(ev[1]), local)
    barrier(dist, local)
    kstats = {k: ctx.kernel_stats(k) for k in ("fp_kernel", "bp_kernel", "rotback_kernel")}
    launches = sum(n for n, _ in kstats.values())
    model = algorithmic_model(ctx.info, add_bytes=4 if storage == H.STORE_F32 else 2)
    dom = max(kstats, key=lambda k: kstats[k][1])
    n, tot = kstats[dom]
    avg_s = tot / max(n, 1) / 1e3
    peak, peak_kind = measured_peaks()
    achieved = model[dom]["bytes"] / avg_s / 1e9
    traffic = ncu_traffic(dom)
    sm_mhz = (clk or {}).get("sm_mhz") or 1965.0
    out = {
        "metric": METRIC, "value": ws * args.steps / (ms / 1e3), "unit": UNIT, "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32" if storage == H.STORE_F32 else "f32 compute, 16-bit stored inputs",
        "data": DATA,
        "config": bench_config(args.storage, ws),
        "e2e": e2e,
        "gpu_launches": launches,
        "kernels": {k: {"launches": v[0], "ms_total": v[1], "ms_avg": v[1] / max(v[0], 1)} for k, v in kstats.items()},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                     "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else
                     "fallback 6.65 TB/s", "unit": "GB/s", "frac": achieved / peak,
                     "traffic": traffic[0] if traffic else None,
                     "bytes_per_launch": model[dom]["bytes"],
                     "traffic_source": traffic[1] if traffic else None},
        # the projectors are bound by the FP32 pipe, not by HBM: the same
        # kernel against the FP32 CUDA-core peak (148 SMs x 128 lanes x 2 flop
        # per clock; nominal at 1965 MHz, and at the median SM clock sampled
        # during the timed region)
        "roofline_alu": {"bound": "fp32", "kernel": dom, "unit": "TFLOP/s",
                         "achieved": model[dom]["flops"] / avg_s / 1e12,
                         "flops_per_launch": model[dom]["flops"],
                         "peak_nominal": FP32_TFLOPS_NOMINAL,
                         "peak_at_clock": FP32_TFLOPS_NOMINAL * sm_mhz / 1965.0,
                         "frac_nominal": model[dom]["flops"] / avg_s / 1e12 / FP32_TFLOPS_NOMINAL,
                         "frac_at_clock": model[dom]["flops"] / avg_s / 1e12 / (FP32_TFLOPS_NOMINAL * sm_mhz / 1965.0)},
        # the bound the forward projector actually meets: every interpolation
        # sample reads its two row entries (4 B each) from shared memory;
        # peak = 148 SMs x 128 B per clock at the sampled SM clock
        "roofline_smem": {"bound": "shared memory", "kernel": "fp_kernel", "unit": "GB/s",
                          "bytes_per_launch": model["fp_kernel"]["smem_bytes"],
                          "achieved": model["fp_kernel"]["smem_bytes"] / (kstats["fp_kernel"][1] /
                                                                           max(kstats["fp_kernel"][0], 1) / 1e3) / 1e9,
                          "peak_nominal": 148 * 128 * sm_mhz * 1e6 / 1e9,
                          "frac": model["fp_kernel"]["smem_bytes"] / (kstats["fp_kernel"][1] /
                                                                       max(kstats["fp_kernel"][0], 1) / 1e3)
                          / (148 * 128 * sm_mhz * 1e6)},
        # the whole subset-iteration against HBM: algorithmic bytes per subset
        # (bins x (input bytes + 8) + 3 image volumes) over the step time
        "roofline_subset": {"bound": "hbm", "unit": "GB/s", "bytes_per_step": model["subset_bytes"],
                            "achieved": model["subset_bytes"] / (ms / args.steps / 1e3) / 1e9,
                            "frac": model["subset_bytes"] / (ms / args.steps / 1e3) / 1e9 / peak},
        "clocks": clk,
        "data_gen_s": gen_s,
    }
    if args.storage == "f32" and args.compare_16:
        out["storage16"] = run_storage16(args, torch, H, ctx, st, host, names, img, cs, dist, local, ws, ms)
        out["storage_f16"] = run_storage16(args, torch, H, ctx, st, host, names, img, cs, dist, local, ws, ms,
                                           storage=H.STORE_F16)
    out["adjoint"] = run_adjoint(args, torch, H, ctx, cs, dist, local, ws, ms)
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(args)
    if rank == 0 and ws == 1 and args.parity:
        out["parity"] = {"span3": run_parity(H, ctx, st, ITERATIONS, dict(seed=1, **STUDY))}
    ctx.close()
    del ctx, host, st
    if rank == 0 and ws == 1 and args.parity:
        out["parity"]["span9"] = run_parity_span9(H, local)
    _PINNED.clear()
    if args.dyn_frames > 0:
        out["dynamic"] = run_dynamic(args, torch, H, local, dist, ws)
    if args.lm_events > 0:
        out["listmode"] = run_listmode(args, torch, H, local, dist, ws, cpu=(rank == 0 and ws == 1 and
                                                                             not args.no_cpu_baseline))
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.destroy_process_group()


def run_storage16(args, torch, H, ctx, st, host, names, img_f32, cs, dist, local, ws, ms_f32, storage=None):
    """The same study with 1/(NA) and the additive term stored in 16 bits (bf16
    by default, fp16 with storage=STORE_F16; prompts int16; FP32 arithmetic):
    device-resident subset-iterations/s over the same steps, and the rel-L2
    of its image after the e2e reconstruction against the f32-stored image."""
    storage = H.STORE_16 if storage is None else storage
    img16 = pinned_copy(torch, np.zeros_like(img_f32))
    ctx.reconstruct(*(host.get(k) for k in names), storage=storage, iterations=ITERATIONS, out=img16)
    a = img16.astype(np.float64)
    b = img_f32.astype(np.float64)
    rel = float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))
    ctx.init_image()
    ctx.osem_subsets(0, args.warmup)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    barrier(dist, local)
    torch.cuda.synchronize()
    ev[0].record(cs)
    ctx.osem_subsets(args.warmup, args.steps)
    ev[1].record(cs)
    torch.cuda.synchronize()
    ms = max_over_ranks(dist, ev[0].elapsed_time(ev[1]), local)
    return {"value": ws * args.steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / args.steps,
            "speedup_vs_f32": ms_f32 / ms, "rel_l2_vs_f32_image": rel,
            "rel_l2_note": f"image after {ITERATIONS} iterations x {SUBSETS} subsets (hrrt_reconstruct), "
                           "16-bit-stored vs f32-stored inputs, same prompts",
            "storage": ("prompts int16, 1/(NA) and additive term " + ("fp16" if storage == H.STORE_F16 else "bf16")
                        + "; FP32 accumulation, FP64 image sum")}


def run_parity(H, ctx, st, iterations, study_kw):
    """Per-iteration parity of one whole study: hrrt_reconstruct from host
    buffers with f32, bf16 and fp16 terms, against the reference's own
    projector (oracle/_ref, stock -T) and the FP64 restatement run on the same
    prep (oracle/study_parity.py).  Outside every timed region."""
    from oracle import ref
    from oracle import study_parity as SP
    geom = dict(geom_dict(), span=int(ctx.geom.span))
    raw = [st[k] for k in ("prompts", "randoms", "norm", "atten", "scatter")]
    dev = {}
    for name, storage in (("f32", H.STORE_F32), ("bf16", H.STORE_16), ("fp16", H.STORE_F16)):
        dev[name] = [ctx.reconstruct(*raw, storage=storage, iterations=k + 1)[0] for k in range(iterations)]
    t0 = time.perf_counter()
    pre = SP.prep(geom, *raw)
    host = {}
    if ref.available():
        host["reference"] = SP.reconstruct("reference", geom, pre, iterations)
    host["fp64"] = SP.reconstruct("fp64", geom, pre, iterations)
    host_s = time.perf_counter() - t0
    res = {"workload": f"HRRT span {geom['span']}, 16 subsets x {iterations} iteration(s), phantom study "
                       + ", ".join(f"{k}={v}" for k, v in study_kw.items()),
           "metric": "image rel-L2 per iteration (whole [z][y][x] image)",
           "host": {k: {"threads": v[0]["threads"], "sensitivity_s": v[0]["sens_s"],
                        "iteration_s": [r["seconds"] for r in v], "sum_image": [r["sum"] for r in v]}
                    for k, v in host.items()},
           "host_s": host_s}
    for name, imgs in dev.items():
        d = {f"vs_{k}": v for k, v in SP.compare(imgs, host).items()}
        if name != "f32":
            d["vs_f32_device"] = [SP.rel_l2(a, b) for a, b in zip(imgs, dev["f32"])]
        res[name] = d
    if "reference" in host:
        res["reference_vs_fp64"] = [SP.rel_l2(a["image"], b["image"]) for a, b in zip(host["reference"], host["fp64"])]
    res["storage"] = {"f32": "prompts int16, terms f32", "bf16": "prompts int16, 1/(NA) and additive term bf16",
                      "fp16": "prompts int16, 1/(NA) and additive term fp16"}
    return res


def run_parity_span9(H, local):
    """The plain span-9 workload (seed-0 phantom, 1e8 counts, randoms 20 %,
    norm 1, water attenuation, 16 subsets x 1 iteration) and its 16-bit-stored
    form, through run_parity."""
    from hrrt_reconstruction_b200 import phantom
    kw = dict(seed=0, total_counts=1e8, randoms_frac=0.20)
    with H.Context(H.hrrt_geometry(**dict(geom_dict(), span=9)), device=local) as c9:
        st = phantom.study(c9, **kw)
        return run_parity(H, c9, st, 1, kw)


def run_adjoint(args, torch, H, ctx, cs, dist, local, ws, ms_ref):
    """The same device-resident subsets with the exact adjoint of the forward
    projector as the back projector (hrrt_set_backprojector(HRRT_BP_ADJOINT)):
    subset-iterations/s and each kernel's CUDA-event time, the adjoint pair
    against HBM with its algorithmic bytes (partial sums written and read
    back: the z-transpose reads the ratio (4 B/bin) and writes the column and
    row partials of every pair (2 volumes); the bilinear transpose reads them
    and reads/writes the image and reads the inverse sensitivity (2 x pairs +
    3 volumes)).  The back projector is set back to the reference's after."""
    ctx.set_backprojector(H.BP_ADJOINT)
    ctx.sensitivity()
    ctx.init_image()
    ctx.osem_subsets(0, args.warmup)
    torch.cuda.synchronize()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    barrier(dist, local)
    torch.cuda.synchronize()
    ctx.reset_kernel_stats()
    ctx.set_profiling(True)
    ev[0].record(cs)
    ctx.osem_subsets(args.warmup, args.steps)
    ev[1].record(cs)
    torch.cuda.synchronize()
    ctx.set_profiling(False)
    ms = max_over_ranks(dist, ev[0].elapsed_time(ev[1]), local)
    ks = {k: ctx.kernel_stats(k) for k in ("fp_kernel", "adj_kernel", "adj_rotate_kernel")}
    info = ctx.info
    pairs = info.sviews // 2
    bins = pairs * 2 * info.segmentsize * info.nbins
    vol = info.nx * info.ny * info.zp * 4
    algo = {"adj_kernel": bins * 4 + 2 * pairs * vol, "adj_rotate_kernel": 2 * pairs * vol + 3 * vol}
    peak, _ = measured_peaks()
    kern = {}
    for k, (n, tot) in ks.items():
        d = {"launches": n, "ms_total": tot, "ms_avg": tot / max(n, 1)}
        if k in algo and n:
            gbs = algo[k] / (tot / n / 1e3) / 1e9
            d.update({"bytes_per_launch": algo[k], "achieved_gbs": gbs, "frac_hbm": gbs / peak})
        kern[k] = d
    ctx.set_backprojector(H.BP_REF)
    ctx.sensitivity()
    return {"value": ws * args.steps / (ms / 1e3), "unit": UNIT, "ms_per_step": ms / args.steps,
            "vs_reference_backprojector": ms_ref / ms, "kernels": kern,
            "note": "exact adjoint of the forward projector (dot-product test to 1e-6 in tests/test_adjoint_gpu.py); "
                    "same study and steps as the headline"}


# Dynamic study: 24 span-9 frames of the config-0 phantom, sphere activity
# varying with time, counts log-uniform in [2e6, 2e8], 1-4 iterations each
# (seeded), 16-bit-stored terms, one batch (hrrt_batch_*).  The terms are
# stored as fp16: bf16 terms (8 bits of mantissa) miss the 1e-3 image bar on
# the highest-count frames (1.15e-3 against the f32-stored image at 1.86e8
# counts), fp16 terms (11 bits, range-checked on upload) hold it with 8x
# margin at the same 2 bytes; bf16's error is still reported.
DYN = dict(seed=4, counts=(2e6, 2e8), iterations=(1, 4), randoms_frac=0.20)


def dynamic_frames(nframes, seed):
    """Per frame: total counts, iterations, sphere activities (6 curves: uptake
    with time constant tau_k, washout over the study)."""
    rng = np.random.default_rng(seed)
    lo, hi = DYN["counts"]
    counts = np.exp(rng.uniform(np.log(lo), np.log(hi), nframes))
    iters = rng.integers(DYN["iterations"][0], DYN["iterations"][1] + 1, nframes)
    t = (np.arange(nframes) + 0.5) / nframes
    tau = np.linspace(0.05, 0.5, 6)
    act = 1.0 + 5.0 * (1.0 - np.exp(-t[:, None] / tau[None, :])) * np.exp(-t[:, None] / 1.5)
    return counts, iters, act


def run_dynamic(args, torch, H, local, dist, ws):
    from hrrt_reconstruction_b200 import phantom
    dev = f"cuda:{local}"
    nf = args.dyn_frames
    t0 = time.time()
    geom = H.hrrt_geometry(nrings=104, nelements=256, nangles=288, ring_radius=234.5, plane_sep=1.21875,
                           binsize=1.21875, span=9, maxdel=67, subsets=SUBSETS)
    ctx = H.Context(geom, device=local)
    counts, iters, act = dynamic_frames(nf, DYN["seed"] + 1000 * int(os.environ.get("RANK", "0")))
    # the frame images are linear in the sphere activities: forward-project
    # the cylinder and the six sphere indicators once
    base = phantom.phantom(ctx, seed=0, sphere_activity=1.0)
    parts = [ctx.forward_project(base)]
    for k in range(6):
        sc = np.zeros(6)
        sc[k] = 1.0
        ind = phantom.phantom(ctx, seed=0, activity=0.0, sphere_activity=1.0, sphere_scale=sc)
        parts.append(ctx.forward_project(ind))
    atten = np.exp(ctx.forward_project(phantom.mu_map(ctx)), dtype=np.float32)
    fps = torch.stack([torch.from_numpy(p) for p in parts]).to(dev)
    del parts
    atten_d = torch.from_numpy(atten).to(dev)
    valid = fps[0] > 0
    nvalid = int(valid.sum())
    g = torch.Generator(device=dev)
    g.manual_seed(DYN["seed"])
    host_p, host_r = [], []
    for f in range(nf):
        w = torch.tensor(np.concatenate([[1.0], act[f] - 1.0]), dtype=torch.float32, device=dev)
        t = torch.tensordot(w, fps, dims=1) / atten_d
        t_sum = float(t.sum(dtype=torch.float64))
        r_total = DYN["randoms_frac"] / (1.0 - DYN["randoms_frac"]) * t_sum
        scale = counts[f] / (t_sum + r_total)
        r_level = r_total * scale / nvalid
        mean = t * scale + valid * r_level
        pr = torch.poisson(mean, generator=g).clamp_(max=32767).to(torch.int16)
        hp = torch.empty(pr.shape, dtype=torch.int16, pin_memory=True)
        hp.copy_(pr)
        hr = torch.empty(pr.shape, dtype=torch.float32, pin_memory=True)
        hr.copy_(valid.float() * float(r_level))
        host_p.append(hp.numpy())
        host_r.append(hr.numpy())
        del t, mean, pr
    del fps, atten_d, valid
    torch.cuda.empty_cache()
    gen_s = time.time() - t0
    info = ctx.info
    imgs = [pinned_copy(torch, np.zeros((info.nz, info.ny, info.nx), np.float32)) for _ in range(nf)]
    cs = torch.cuda.ExternalStream(ctx.stream)
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    b = ctx.batch(nf, atten=atten, storage=H.STORE_F16)
    # untimed: prepare every frame, tune the launch shapes, capture the graphs
    for f in range(nf):
        b.set_frame(f, host_p[f], host_r[f], iterations=int(iters[f]))
    tune = b.autotune(repeats=3)
    b.run()
    torch.cuda.synchronize()
    # device-resident: every frame reconstructed from the uniform image
    clocks = ClockSampler(local)
    barrier(dist, local)
    clocks.start()
    bst = b.run()
    clk = clocks.stop()
    run_ms = max_over_ranks(dist, bst.ms_total, local)
    # end to end through the C ABI: every frame's inputs from pinned memory,
    # the reconstruction, every image back into pinned memory
    barrier(dist, local)
    torch.cuda.synchronize()
    ev[0].record(cs)
    for f in range(nf):
        b.set_frame(f, host_p[f], host_r[f], iterations=int(iters[f]))
    est = b.run()
    for f in range(nf):
        b.get_image(f, out=imgs[f])
    ev[1].record(cs)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(dist, ev[0].elapsed_time(ev[1]), local)
    sums = [b.get_image(f, out=imgs[f])[1] for f in range(nf)]
    # precision: two frames reconstructed alone with f32-stored terms (and,
    # for comparison, with bf16-stored terms)
    rel, rel_bf16 = {}, {}

    def rl2(a, b):
        a = a.astype(np.float64)
        b = b.astype(np.float64)
        return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))

    for f in (int(np.argmin(counts)), int(np.argmax(counts))):
        ctx2 = H.Context(geom, device=local)
        want, _ = ctx2.reconstruct(host_p[f], host_r[f], atten=atten, storage=H.STORE_F32,
                                   iterations=int(iters[f]))
        bf, _ = ctx2.reconstruct(host_p[f], host_r[f], atten=atten, storage=H.STORE_16,
                                 iterations=int(iters[f]))
        ctx2.close()
        key = f"frame{f} ({counts[f]:.3g} counts, {int(iters[f])} it)"
        rel[key] = rl2(imgs[f], want)
        rel_bf16[key] = rl2(bf, want)
    h2d = sum(int(a.nbytes) for a in host_p) + sum(int(a.nbytes) for a in host_r)
    d2h = sum(int(a.nbytes) for a in imgs)
    b.close()
    ctx.close()
    si = bst.subset_iterations
    return {
        "metric": "dynamic-study subset-iters/s (span 9, 24 frames, 16-bit-stored inputs)",
        "storage": "prompts int16, 1/(NA) and additive term fp16; FP32 accumulation",
        "unit": UNIT, "value": ws * si / (run_ms / 1e3), "ms_run": run_ms, "subset_iterations": si,
        "workload": f"{nf} span-9 HRRT frames (2209 planes x 288 views x 256 bins), image 256x256x207, phantom "
                    "seed 0 with time-varying sphere activity, counts log-uniform 2e6..2e8, 16 subsets x 1-4 "
                    "iterations per frame (seeded), randoms 20 %, water attenuation, norm 1",
        "frames": {"counts": [float(c) for c in counts], "iterations": [int(i) for i in iters],
                   "sum_image": sums},
        "batch": bst.as_dict(), "tuning": tune.as_dict(), "gpu_launches": bst.kernel_launches,
        "e2e": {"value": ws * est.subset_iterations / (e2e_ms / 1e3), "unit": UNIT, "ms": e2e_ms,
                "h2d_bytes_per_step": h2d // max(est.subset_iterations, 1),
                "d2h_bytes_per_step": d2h // max(est.subset_iterations, 1)},
        "rel_l2_vs_f32_stored": rel,
        "rel_l2_vs_f32_stored_bf16_terms": rel_bf16,
        "clocks": clk, "data_gen_s": gen_s,
    }


def run_listmode(args, torch, H, local, dist, ws, cpu=True):
    """l64 listmode -> span-3 prompt and delayed sinograms (16-bit), the
    config-5 workload: synthetic events from the config-1 phantom's LOR
    distribution, 10 % delayed, a time tag every 1000 events (1 ms)."""
    from hrrt_reconstruction_b200 import listmode_synth as LS
    n = args.lm_events
    t0 = time.time()
    with H.Context(H.hrrt_geometry(span=3), device=local) as c3:
        E = LS.expected_prompts(c3, seed=0)
    words = LS.synth_words(n, E, seed=0, device=f"cuda:{local}")
    del E
    gen_s = time.time() - t0
    nwords = words.numel()
    lm = H.Listmode(3, device=local)
    S = lm.sino_size
    ds = torch.zeros(S, dtype=torch.int16, device=f"cuda:{local}")
    dd = torch.zeros(S, dtype=torch.int16, device=f"cuda:{local}")
    cs = torch.cuda.current_stream()
    for _ in range(2):
        lm.reset_clock()
        lm.histogram_device(words.data_ptr(), nwords, ds.data_ptr(), dd.data_ptr(), stream=cs.cuda_stream)
    torch.cuda.synchronize()
    reps = 3
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    barrier(dist, local)
    ev[0].record(cs)
    dev_ms = []
    for _ in range(reps):
        lm.reset_clock()
        st = lm.histogram_device(words.data_ptr(), nwords, ds.data_ptr(), dd.data_ptr(), stream=cs.cuda_stream)
        dev_ms.append(st["ms"])
    ev[1].record(cs)
    torch.cuda.synchronize()
    ms = max_over_ranks(dist, ev[0].elapsed_time(ev[1]) / reps, local)
    # end to end: words from pinned host memory, sinograms back to pinned host memory
    hw = torch.empty(nwords, dtype=torch.int32, pin_memory=True)
    hw.copy_(words)
    del words, ds, dd
    torch.cuda.empty_cache()
    hs = torch.empty(S, dtype=torch.int16, pin_memory=True)
    hd = torch.empty(S, dtype=torch.int16, pin_memory=True)
    hwn = hw.numpy().view(np.uint32)
    out = (hs.numpy().view(np.uint16), hd.numpy().view(np.uint16))
    lm.reset_clock()
    lm.histogram(hwn, out=out)  # warm: grows the library's staging buffers
    ls = torch.cuda.ExternalStream(lm.stream)
    torch.cuda.synchronize()
    barrier(dist, local)
    ev[0].record(ls)
    lm.reset_clock()
    st = lm.histogram(hwn, out=out)[2]
    ev[1].record(ls)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(dist, ev[0].elapsed_time(ev[1]), local)
    peak, peak_kind = measured_peaks()
    algo = nwords * 4 + 2 * S * 2  # events read once + both 16-bit sinograms written once
    res = {
        "metric": "listmode events/s (l64 -> span-3 prompt + delayed sinograms, 16-bit)", "unit": "events/s",
        "value": ws * n / (ms / 1e3), "ms_per_frame": ms, "events": n, "words": nwords,
        "workload": "1 frame of synthetic l64 events (config-1 phantom LORs, 10 % delayed, 1 time tag / 1000 "
                    "events), histogram modes prompts + delayed, span 3",
        "stats": {k: st[k] for k in ("prompts", "delayed", "timetags", "unmapped", "invalid")},
        "e2e": {"value": ws * n / (e2e_ms / 1e3), "unit": "events/s", "ms": e2e_ms,
                "h2d_bytes_per_step": nwords * 4, "d2h_bytes_per_step": 2 * S * 2},
        "roofline": {"bound": "hbm", "kernel": "lm_map + lm_hist passes (whole call)", "unit": "GB/s",
                     "achieved": algo / (ms / 1e3) / 1e9, "peak": peak, "frac": algo / (ms / 1e3) / 1e9 / peak,
                     "bytes_per_launch": algo,
                     "note": "algorithmic bytes: the event words read once and both sinograms written once"},
        "device_ms_per_call": float(np.mean(dev_ms)),
        "data_gen_s": gen_s,
    }
    if cpu:
        res["cpu_baseline"] = listmode_cpu_baseline(hwn)
        res["parity"] = listmode_parity(H, hwn, local)
    lm.close()
    # the rest of the config-5 pipeline: OSEM (16 subsets x 2 iterations) of
    # the histogrammed prompts with the delayed sinogram as randoms, from the
    # pinned sinograms through the C ABI; the delayed counts become the float
    # randoms file on the host first, as lmhistogram's output does before
    # hrrt_osem3d reads it (not timed)
    del hw, hwn
    _PINNED.clear()
    prompts = out[0].view(np.int16)
    randoms = pinned_copy(torch, out[1].astype(np.float32))
    with H.Context(H.hrrt_geometry(span=3), device=local) as c3:
        info = c3.info
        img = pinned_copy(torch, np.zeros((info.nz, info.ny, info.nx), np.float32))
        c3.reconstruct(prompts, randoms, iterations=1, out=img)  # sizes the staging buffers
        rs = torch.cuda.ExternalStream(c3.stream)
        torch.cuda.synchronize()
        barrier(dist, local)
        ev[0].record(rs)
        _, rst = c3.reconstruct(prompts, randoms, iterations=ITERATIONS, out=img)
        ev[1].record(rs)
        torch.cuda.synchronize()
        rec_ms = max_over_ranks(dist, ev[0].elapsed_time(ev[1]), local)
    res["pipeline"] = {
        "metric": "listmode -> image events/s (1e9 events histogrammed, then 16 subsets x 2 iterations of OSEM)",
        "unit": "events/s", "value": ws * n / ((e2e_ms + rec_ms) / 1e3), "histogram_ms": e2e_ms,
        "reconstruct_ms": rec_ms, "subset_iterations": rst.subset_iterations, "sum_image": rst.sum_image,
        "note": "both stages end to end through the C ABI from pinned host memory (words -> sinograms -> image)"}
    return res


def listmode_cpu_baseline(words, n_sample_words=8_000_000):
    """The listmode restatement (oracle/lm_oracle.c, one thread) on the first
    `n_sample_words` words of the same stream."""
    from oracle.lm import LMOracle
    O = LMOracle(3)
    w = np.ascontiguousarray(words[:n_sample_words])
    s = np.zeros(O.sino_size, np.uint16)
    d = np.zeros(O.sino_size, np.uint16)
    t0 = time.perf_counter()
    _, _, st = O.histogram(w, sino=s, delayed=d)
    dt = time.perf_counter() - t0
    ev = st["prompts"] + st["delayed"]
    return {"value": ev / dt, "unit": "events/s", "cores": 1, "kind": "port",
            "sample": f"first {n_sample_words} words ({ev} events) of the stream on oracle/lm_oracle.c"}


def listmode_parity(H, words, local, npackets=4, duration=3):
    """The first `npackets` whole reader packets of the stream (1 Mi events
    each) histogrammed as one `duration`-second frame (prompts + delayed,
    span 3) by the device, by the restatement (oracle/lm_oracle.c) and by the
    reference's own histogrammer (oracle/_ref/lmhist_ref); bins that differ
    between them.  Outside every timed region."""
    from oracle import lm_ref
    from oracle.lm import LMOracle
    n = npackets * (2 << 20)
    w = np.ascontiguousarray(words[:n])
    with H.Listmode(3, device=local) as D:
        D.reset_clock()
        ds, dd, dst = D.histogram(w, duration=duration)
    O = LMOracle(3)
    O.reset_clock()
    os_, od, ost = O.histogram(w, duration=duration)
    res = {"prefix_words": n, "frame_s": duration, "events": int(ost["prompts"] + ost["delayed"]),
           "bins": 2 * int(ds.size), "device_vs_oracle_bins_differing": int((ds != os_).sum() + (dd != od).sum())}
    del os_, od
    if lm_ref.available():
        R = lm_ref.histogram(w, span=3, mode=1, duration=duration)
        res["device_vs_reference_bins_differing"] = int((ds.view(np.int16) != R["prompts"]).sum() +
                                                        (dd.view(np.int16) != R["delayed"]).sum())
        res["reference_frame"] = {"start_s": R["frame_start"], "duration_s": R["duration"],
                                  "prompts": R["total_prompts"], "randoms": R["total_randoms"]}
        res["device_frame"] = {"start_s": int(dst["frame_start"]), "duration_s": int(dst["duration"]),
                               "prompts": int(dst["prompts"]), "delayed": int(dst["delayed"])}
        res["reference"] = ("oracle/_ref/lmhist_ref: histogram_mp.cpp, LM_Reader_mp.cpp, LM_Rebinner_mp.cpp, "
                            "lor_sinogram_map.cpp, geometry_info.cpp, segment_info_fromarchive.cpp compiled "
                            "unmodified")
    return res


def ref_inputs(R, seed=0):
    """Cheap inputs for timing the reference CPU path: the phantom image and
    Poisson prompts; the projector's cost does not depend on the values."""
    rng = np.random.default_rng(seed)
    shape = (R.P, R.views, R.nx)
    prompts = rng.poisson(0.64, size=shape).astype(np.int16)
    add = np.full(shape, 0.1, np.float32)
    nf = np.ones(R.image_shape, np.float32)
    img = R.init_image()
    return img, nf, prompts, add


def ref_threads():
    """The reference's stock thread count: -T min(8, nproc).  Its projector
    threads are threads[Cal1 + thr] of a 16-entry array with Cal1 = 8
    (hrrt_osem3d_span3.cpp:189, :448, :4193), so -T cannot exceed 8."""
    return max(1, min(8, os.cpu_count() or 1))


def all_core_threads():
    """Every host core up to the harness's 16 thread slots (a labelled second
    figure: the stock binary does not run more than 8)."""
    return max(1, min(16, os.cpu_count() or 1))


def cpu_model():
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    import platform
    return platform.processor() or "unknown"


def time_ref_subsets(R, img, nf, prompts, add, order, first, count, T):
    t0 = time.perf_counter()
    for k in range(count):
        R.osem_subset(img, nf, prompts, add, int(order[(first + k) % SUBSETS]), T)
    return time.perf_counter() - t0


def cpu_baseline(args, subsets_in_sample=2):
    from oracle import ref
    if not ref.available():
        return oracle_port_baseline(subsets_in_sample)
    T, TA = ref_threads(), all_core_threads()
    R = ref.RefProjector(nthreads=max(T, TA), **geom_dict())
    img, nf, prompts, add = ref_inputs(R)
    order = R.order()
    dt = time_ref_subsets(R, img, nf, prompts, add, order, 0, subsets_in_sample, T)
    dta = time_ref_subsets(R, img, nf, prompts, add, order, subsets_in_sample, subsets_in_sample, TA)
    return {"value": subsets_in_sample / dt, "unit": UNIT, "cores": T, "kind": "reference",
            "nproc": os.cpu_count(), "cpu_model": cpu_model(),
            "sample": f"{subsets_in_sample} OP-OSEM subsets of the span-3 HRRT workload on the reference projector "
                      f"(oracle/_ref/libhrrt_ref.so) with the stock -T {T} thread grouping of CalculateOsem3d",
            "all_cores": {"value": subsets_in_sample / dta, "threads": TA,
                          "note": "the same with -T = min(16, nproc), beyond the stock maximum of 8"}}


def oracle_port_baseline(subsets_in_sample=1):
    """The C restatement (oracle/hrrt_oracle.c, f32 build) timed on the host
    cores when the reference build is absent."""
    from oracle.oracle import Oracle
    T = ref_threads()
    O = Oracle(precision="f32", nthreads=T, **geom_dict())
    rng = np.random.default_rng(0)
    shape = O.sino_shape
    prompts = rng.poisson(0.64, size=shape).astype(np.int16)
    add = np.full(shape, 0.1, np.float32)
    nf = np.ones(O.image_shape, np.float32)
    img = O.init_image()
    order = O.order()
    t0 = time.perf_counter()
    for k in range(subsets_in_sample):
        O.osem_subset(img, nf, prompts, add, int(order[k % SUBSETS]), T)
    dt = time.perf_counter() - t0
    return {"value": subsets_in_sample / dt, "unit": UNIT, "cores": min(T, O.sviews // 2), "kind": "port",
            "sample": f"{subsets_in_sample} OP-OSEM subset(s) of the span-3 HRRT workload on the C restatement "
                      f"(oracle/hrrt_oracle.c, {min(T, O.sviews // 2)} threads)"}


def run_reference(args, ws, rank, local):
    if rank != 0:
        return
    from oracle import ref
    if not ref.available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libhrrt_ref.so not built"}))
        return
    T, TA = ref_threads(), all_core_threads()
    R = ref.RefProjector(nthreads=max(T, TA), **geom_dict())
    img, nf, prompts, add = ref_inputs(R)
    order = R.order()
    time_ref_subsets(R, img, nf, prompts, add, order, 0, args.warmup, T)
    dt = time_ref_subsets(R, img, nf, prompts, add, order, args.warmup, args.steps, T)
    v = args.steps / dt
    # the labelled second figure: all host cores (up to 16 threads), a short sample
    na = min(args.steps, 4)
    dta = time_ref_subsets(R, img, nf, prompts, add, order, 0, na, TA)
    out = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": ws, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": dt * 1e3 / args.steps, "higher_is_better": True,
           "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": DATA,
           "config": bench_config(args.storage, ws),
           "cpu_baseline": {"value": v, "unit": UNIT, "cores": T, "kind": "reference", "nproc": os.cpu_count(),
                            "cpu_model": cpu_model(),
                            "sample": f"one OP-OSEM subset per step (9 view pairs), span-3 HRRT, on the reference "
                                      f"projector (oracle/_ref/libhrrt_ref.so) with the stock -T {T} thread "
                                      "grouping of CalculateOsem3d",
                            "all_cores": {"value": na / dta, "threads": TA, "steps": na,
                                          "note": "the same with -T = min(16, nproc), beyond the stock maximum "
                                                  "of 8"}},
           "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


# ---------------------------------------------------------------------------
# Kernel cases: compact workloads that launch one group of kernels a few
# times, for profiler captures (`--case`); they print per-kernel device times
# and no benchmark line.
# ---------------------------------------------------------------------------
OSEM_KERNELS = ("prep_kernel", "scale_pairs_kernel", "fp_kernel", "bp_kernel", "adj_kernel", "adj_rotate_kernel",
                "rotback_kernel", "post_iter_kernel", "psf_kernel", "apply_corr_kernel", "map_dpf_kernel")


def case_osem(args):
    """Seeded Poisson prompts, flat randoms and a lognormal normalisation at
    the HRRT geometry of `--span`: upload (prep), sensitivity, then
    `--subsets` OSEM subsets (and `--iterations` full iterations) with the
    chosen back projector, PSF and MAP options.  Holds the quad-layout inputs only (about 5 GB at span 3, 3 GB
    with 16-bit terms), so single launches of its kernels suit a profiler."""
    import hrrt_reconstruction_b200 as H
    ctx = H.Context(H.hrrt_geometry(span=args.span))
    rng = np.random.default_rng(7)
    shape = ctx.sino_shape
    prompts = rng.poisson(0.64, size=shape).astype(np.int16)
    randoms = np.full(shape, 0.1, np.float32)
    norm = np.exp(np.float32(0.1) * rng.standard_normal(shape, dtype=np.float32)).astype(np.float32)
    storage = {"f32": H.STORE_F32, "16": H.STORE_16, "f16": H.STORE_F16}[args.storage]
    if args.bp == "adjoint":
        ctx.set_backprojector(H.BP_ADJOINT)
    if args.psf:
        ctx.set_psf(True)
    ctx.set_profiling(True)
    ctx.upload_inputs(prompts, randoms, norm, storage=storage)
    ctx.sensitivity()
    ctx.init_image()
    if args.map:
        ctx.set_map(1, 0.02, first_subset=0)
    ctx.osem_subsets(0, args.subsets)
    if args.iterations:
        ctx.osem(args.iterations)
    ctx.set_profiling(False)
    for k in OSEM_KERNELS:
        n, ms = ctx.kernel_stats(k)
        if n:
            print(f"{k:18s} launches {n:4d}  total {ms:9.3f} ms  avg {ms / n:8.3f} ms", flush=True)
    ctx.close()


LM_PATHS = (("direct", 16), ("wide", 64), ("partitioned", 32))


def case_lm(args):
    """`--events` synthetic l64 events (the benchmark's generator) histogrammed
    `--reps` times through each device path into span-3 prompt and delayed
    sinograms; `--lm-extra randoms` also smooths randoms from the stream's
    coincidence histogram, `span9` folds the trues into span 9.  Holds the
    words (8 B per event) and the two 16-bit sinograms (1.9 GB)."""
    import torch

    import hrrt_reconstruction_b200 as H
    from hrrt_reconstruction_b200 import listmode_synth as LS
    with H.Context(H.hrrt_geometry(span=3)) as c3:
        E = LS.expected_prompts(c3, seed=0)
    words = LS.synth_words(int(args.events), E, seed=0)
    del E
    torch.cuda.synchronize()
    extra = set(args.lm_extra.split(",")) if args.lm_extra else set()
    with H.Listmode(3) as lm:
        ds = torch.zeros(lm.sino_size, dtype=torch.int16, device="cuda")
        dd = torch.zeros(lm.sino_size, dtype=torch.int16, device="cuda")
        stream = torch.cuda.current_stream().cuda_stream
        want = args.paths.split(",")
        for name, flag in LM_PATHS:
            if name not in want:
                continue
            ms = []
            for r in range(args.reps + 1):
                lm.reset_clock()
                st = lm.histogram_device(words.data_ptr(), words.numel(), ds.data_ptr(), dd.data_ptr(), flags=flag,
                                         stream=stream)
                if r > 0:
                    ms.append(st["ms"])
            print(f"{name:12s} {int(args.events)} events  " + " ".join(f"{m:.2f}" for m in ms) + " ms", flush=True)
        if "span9" in extra:
            d9 = torch.zeros(2209 * 288 * 256, dtype=torch.int16, device="cuda")
            for _ in range(args.reps + 1):
                lm.trues_span9_device(ds.data_ptr(), dd.data_ptr(), d9.data_ptr(), stream=stream)
            torch.cuda.synchronize()
            print("span9 trues folded", flush=True)
        if "randoms" in extra:
            lm.reset_clock()
            lm.histogram_device(words.data_ptr(), words.numel(), ds.data_ptr(), dd.data_ptr(),
                                flags=H.LM_CRYSTAL_COUNTS, stream=stream)
            torch.cuda.synchronize()
            counts = lm.crystal_counts().astype(np.int32)
            with H.Listmode(9) as l9:
                for _ in range(args.reps):
                    sino, it = l9.smooth_randoms(counts, scan_duration=max(1.0, args.events / 1e6 / 1e3))
            print(f"smoothed randoms: {it} iterations, sum {float(sino.sum(dtype=np.float64)):.6g}", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=48)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--storage", default="f32", choices=["f32", "16"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--lm-events", type=int, default=1_000_000_000,
                    help="listmode events of the l64 leg (0: skip it)")
    ap.add_argument("--geometry", default="hrrt", choices=["hrrt", "small"])
    ap.add_argument("--dyn-frames", type=int, default=24, help="frames of the dynamic-study leg (0: skip it)")
    ap.add_argument("--no-compare-16", dest="compare_16", action="store_false",
                    help="skip the 16-bit-storage leg of the span-3 workload")
    ap.add_argument("--no-parity", dest="parity", action="store_false",
                    help="skip the per-iteration parity of the span-3 and span-9 studies against the host checkers")
    ap.add_argument("--case", choices=["osem", "lm"], help="run a kernel case for a profiler instead of the bench")
    ap.add_argument("--span", type=int, default=3, choices=[3, 9], help="--case osem: span")
    ap.add_argument("--subsets", type=int, default=2, help="--case osem: OSEM subsets after the sensitivity")
    ap.add_argument("--case-storage", dest="case_storage", default="f32", choices=["f32", "16", "f16"],
                    help="--case osem: storage of the sinogram terms")
    ap.add_argument("--iterations", type=int, default=0,
                    help="--case osem: full iterations (every subset + the post-iteration pass) after the subsets")
    ap.add_argument("--bp", default="ref", choices=["ref", "adjoint"], help="--case osem: back projector")
    ap.add_argument("--psf", action="store_true", help="--case osem: PSF modelling (-B, HRRT defaults)")
    ap.add_argument("--map", action="store_true", help="--case osem: MAP technique 1 from the first subset")
    ap.add_argument("--events", type=float, default=1e8, help="--case lm: events")
    ap.add_argument("--reps", type=int, default=1, help="--case lm: timed calls per path")
    ap.add_argument("--paths", default="direct", help="--case lm: direct,wide,partitioned")
    ap.add_argument("--lm-extra", default="", help="--case lm: randoms,span9")
    args = ap.parse_args()
    if args.case == "osem":
        args.storage = args.case_storage
        return case_osem(args)
    if args.case == "lm":
        return case_lm(args)
    global GEOMETRY
    GEOMETRY = args.geometry
    if args.warmup < 3 and args.impl != "reference":
        args.warmup = 3
    ws, rank, local = dist_env()
    if args.impl == "reference":
        run_reference(args, ws, rank, local)
    else:
        run_ours(args, ws, rank, local)


if __name__ == "__main__":
    main()
