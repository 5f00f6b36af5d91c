"""Benchmark of the sm_100a splat rasterizer on the reference's headline workload.

Workloads (--config):
  plain  1.2M anisotropic degree-3 SH gaussians (seeded synthetic clusters,
         fp32), 1920x1080, 16x16 tiles, over the reference bench's orbit
         (src/bench.rs:38-111: distance 12, FOV 50 deg, yaw step 2 pi / 40,
         pitch 0.4 sin(0.1 i)). The default.
  fp16   the same scene with scales, rotations, opacities and SH stored as
         FP16 (positions f32), 3840x2160; the per-frame error against the
         FP64 naive rasterizer is stated for the first frames.
  learned
         the plain scene's 48 SH floats per splat replaced by 16 FP16 latents
         and a shared MLP (FP16 geometry), trained first on the device from
         exact SH at 256 Fibonacci directions per splat (batch 65536, Adam lr
         1e-3; the training is timed and reported separately), then rendered
         over the same 1080p orbit; PSNR against the exact-SH plain path, and
         the plain path's frames/s from the same run.
  batch  96 views of mixed resolution over three scenes, one CUDA graph.
  sharded
         the plain workload's frame drawn from splats sharded over the ranks:
         each rank holds a contiguous share of the scene and owns a window of
         tile rows; the projected splats cross in one all-to-all (NCCL) and
         the windows are gathered on the device. With one process, --shards
         ranks run one after another on the one GPU (the exchange becomes a
         concatenation): the line then also states each rank's part.
A step is one frame.

  value  frames/s with the scene resident in HBM and the frame written to
         device memory (CUDA events on the renderer's stream, max over ranks)
  e2e    frames/s through the public C ABI call splat_cuda_render with the
         frame copied to pinned host memory every step
  --impl reference
         the reference's CPU rasterizer (the oracle's C++ restatement of the
         `cpu` backend, all host threads) on the same workload

Under torchrun (N > 1) every rank renders its own share of the orbit views
(view-parallel replicas: no collective on the data path) and rank 0 prints
the aggregate.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_SPLATS = 1_200_000
ORBIT = 40
S_REC = 48  # bytes per projected-splat record
S_BIN = 16  # bytes per splat of tile rectangle, depth bits and pair count
CONFIGS = {
    "plain": {"metric": "frames/s at 1920x1080, 1.2M SH3 splats", "w": 1920, "h": 1080, "precision": "fp32",
              "s_in": 232,  # f32 position, opacity, colour, cov3d, 45 SH coefficients
              "workload": "1.2M SH-degree-3 gaussians (64 seeded clusters), 1920x1080, 16x16 tiles, 40-view orbit"},
    "batch": {"metric": "views/s, 96 views of mixed resolution over 3 scenes (50k SH0, 400k SH1, 3M SH3)",
              "workload": "3 seeded cluster scenes (50k SH0, 400k SH1, 3M SH3, f32), 96 views: resolution uniform "
                          "from 160x96..3840x2160, yaw U[0, 2pi), pitch U[-0.6, 0.6], FOV U[40, 70] deg, "
                          "distance 12; one CUDA graph per batch"},
    "learned": {"metric": "frames/s at 1920x1080, 1.2M splats, learned colour (16 FP16 latents + MLP)",
                "w": 1920, "h": 1080, "precision": "learned",
                "s_in": 64,  # f32 position + k, f16 scale/rotation/opacity, 16 f16 latents
                "workload": "1.2M gaussians of the SH3 workload with colour from 16 FP16 latents + a shared "
                            "19-64-64-3 MLP (FP16 geometry), 1920x1080, 16x16 tiles, 40-view orbit"},
    "sharded": {"metric": "frames/s at 1920x1080, 1.2M SH3 splats, one frame from splats sharded over the ranks",
                "w": 1920, "h": 1080, "precision": "fp32", "s_in": 232,
                "workload": "1.2M SH-degree-3 gaussians (64 seeded clusters), 1920x1080, 16x16 tiles, 40-view "
                            "orbit; splats sharded in contiguous runs, one window of tile rows per rank"},
    "fp16": {"metric": "frames/s at 3840x2160, 1.2M SH3 splats, FP16 storage", "w": 3840, "h": 2160,
             "precision": "fp16",
             "s_in": 124,  # f32 position; f16 scale, rotation, opacity, 48 SH coefficients
             "workload": "1.2M SH-degree-3 gaussians (64 seeded clusters) stored in FP16, 3840x2160, 16x16 tiles, "
                         "40-view orbit"},
}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=None,
                   help="timed steps (default: 4000 frames plain, 1000 fp16, 20 batches)")
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--config", default="plain", choices=sorted(CONFIGS))
    p.add_argument("--batch-views", type=int, default=96)
    p.add_argument("--batch-scale", type=float, default=1.0, help="batch: scale the three scene sizes")
    p.add_argument("--error-frames", type=int, default=2,
                   help="fp16: frames whose error against the FP64 naive rasterizer is stated")
    p.add_argument("--splats", type=int, default=N_SPLATS)
    p.add_argument("--shards", type=int, default=4, help="sharded, one process: ranks emulated one after another")
    p.add_argument("--cpu-sample-s", type=float, default=15.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--learn-epochs", type=float, default=30.0, help="learned: training epochs before rendering")
    p.add_argument("--psnr-frames", type=int, default=40, help="learned: orbit frames compared with exact SH")
    p.add_argument("--profile", action="store_true",
                   help="render --warmup then --steps frames and exit (a short command for ncu captures)")
    p.add_argument("--profile-io", action="store_true",
                   help="decode the workload's PLY and .splat bytes on the device (FP32 and FP16 storage) and draw "
                        "its home frame as terminal cells (half blocks, downsample 2; truecolor and ANSI-256), "
                        "--steps times each, then exit (a short command for ncu captures of k_decode_* and k_cells)")
    a = p.parse_args()
    if a.steps is None:
        a.steps = {"plain": 4000, "fp16": 1000, "batch": 20, "learned": 4000, "sharded": 500}[a.config]
    return a


from splat_b200.multi import dist_env, max_over_ranks, shard  # noqa: E402


_CLOCK_SAMPLER = r"""
import json, signal, sys, time
import pynvml
pynvml.nvmlInit()
bus, index, period = sys.argv[1], int(sys.argv[2]), float(sys.argv[3])
try:
    h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
except Exception:
    h = pynvml.nvmlDeviceGetHandleByIndex(index)
rows, stop = [], []
signal.signal(signal.SIGTERM, lambda *a: stop.append(1))
mx = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)  # a property of the part: read once
print("ready", flush=True)
while not stop:
    try:
        rows.append((pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM), mx,
                     pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)))
    except Exception:
        pass
    if period > 0:
        time.sleep(period)
print(json.dumps(rows), flush=True)
"""


class Clocks:
    """Samples the SM clock, its maximum and the clock-event (throttle)
    reasons of the GPU about every millisecond while the timed region runs.
    The sampler is a separate process querying NVML (read-only), so it takes
    nothing from the process that launches the frames and gets many samples
    even from a timed region of a few milliseconds; nvidia-smi one-shot
    queries from a thread are the fallback when NVML is not usable."""

    NAMES = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    BITS = [0x8, 0x40, 0x20, 0x4]  # nvmlClocksEventReason{HwSlowdown, HwThermalSlowdown, SwThermalSlowdown, SwPowerCap}
    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index, period=0.0002):
        self.index = index
        self.period = period
        self.rows = []  # (sm_mhz, max_mhz, reasons bitmask)
        self.stop = threading.Event()
        self.proc = None
        self.source = "nvml (sampler process)"

    def _bus(self):
        try:
            import torch

            p = torch.cuda.get_device_properties(self.index)
            return f"{p.pci_domain_id:08x}:{p.pci_bus_id:02x}:{p.pci_device_id:02x}.0"
        except Exception:
            return ""

    def _poll_smi(self):
        while not self.stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                for line in out.stdout.strip().splitlines():
                    c = [x.strip() for x in line.split(",")]
                    bits = sum(b for b, v in zip(self.BITS, c[3:7]) if v.lower().startswith("active"))
                    self.rows.append((float(c[0]), float(c[1]), bits))
            except Exception:
                pass
            self.stop.wait(0.2)

    def __enter__(self):
        try:
            self.proc = subprocess.Popen([sys.executable, "-c", _CLOCK_SAMPLER, self._bus(), str(self.index),
                                          str(self.period)], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL,
                                         text=True)
            if self.proc.stdout.readline().strip() != "ready":
                raise RuntimeError("clock sampler did not start")
        except Exception:
            if self.proc:
                self.proc.kill()
            self.proc = None
            self.source = "nvidia-smi"
            self.t = threading.Thread(target=self._poll_smi, daemon=True)
            self.t.start()
        self.t0 = time.perf_counter()
        return self

    def __exit__(self, *a):
        self.seconds = time.perf_counter() - self.t0
        if self.proc:
            import signal

            self.proc.send_signal(signal.SIGTERM)
            try:
                out, _ = self.proc.communicate(timeout=30)
                self.rows = [tuple(r) for r in json.loads(out.strip().splitlines()[-1])]
            except Exception:
                self.proc.kill()
        else:
            self.stop.set()
            self.t.join(timeout=10)

    def summary(self):
        sm = [float(r[0]) for r in self.rows]
        mx = [float(r[1]) for r in self.rows]
        reasons = sorted({nm for r in self.rows for nm, b in zip(self.NAMES, self.BITS) if int(r[2]) & b})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows), "source": self.source,
                "window_s": round(getattr(self, "seconds", 0.0), 4)}


def bench_config(cfg, n, w, h, world):
    """The workload's config dict, the same in both arms of the benchmark."""
    return {"workload": cfg["workload"], "splats": n, "width": w, "height": h, "tile": 16,
            "storage": cfg["precision"], "parallelism": f"view-parallel x{world}",
            "l2": f"inputs larger than L2 (scene {n * cfg['s_in'] / 1e6:.0f} MB > 126 MB)"}


def make_workload(n, cfg):
    """Scene (a Scene, or its HalfScene for the FP16 workload), the oracle's
    f32 form of what the device holds, and the orbit views."""
    from splat_b200 import synth

    scene = synth.cluster_scene(n, seed=0x5EED0001, sh_degree=3)
    cam = synth.orbit_camera(scene)
    home, warm, timed = synth.orbit_views(cam, ORBIT, 5)
    if cfg["precision"] == "learned":
        return scene, scene, scene, home, warm, timed
    if cfg["precision"] == "fp16":
        half = scene.to_fp16()
        return half, half.decoded_scene(), scene, home, warm, timed
    return scene, scene, scene, home, warm, timed


def scene_load(scene, dev):
    """The workload scene as a 3DGS PLY and as .splat records, loaded by the
    device decoders (header parse, one host-to-device copy, decode + finalize
    kernel, handle set-up; wall clock) beside the host path (the reader
    restated in numpy, Scene::finalize, splat_cuda_create's upload)."""
    import torch

    from oracle import scene_io as IO
    from splat_b200.render import CudaRenderer, from_ply_bytes, from_splat_bytes

    out = {}
    for kind, data, loader, parse in (("ply", IO.write_ply(scene), from_ply_bytes, IO.parse_ply),
                                      ("splat", IO.write_splat(scene), from_splat_bytes, IO.parse_splat)):
        loader(data, device=dev).close()  # warm-up
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = loader(data, device=dev)
        t_dev = time.perf_counter() - t0
        r.close()
        t0 = time.perf_counter()
        r = CudaRenderer(parse(data).finalize(), device=dev)
        t_host = time.perf_counter() - t0
        r.close()
        out[kind] = {"bytes": len(data), "device_decode_ms": 1e3 * t_dev, "device_gb_per_s": len(data) / t_dev / 1e9,
                     "host_parse_finalize_upload_ms": 1e3 * t_host}
    out["note"] = ("create_from_ply / create_from_splat (wall clock: header parse, copy, decode kernel, buffers) "
                   "against the reader restated in numpy + finalize + splat_cuda_create, same process")
    return out


def profile_traffic(config, stage):
    """The dominant kernel's DRAM bytes per launch measured by ncu for this
    workload (profiles/traffic.json) and where they come from, or None."""
    try:
        entry = json.load(open(os.path.join(ROOT, "profiles", "traffic.json"))).get(config, {})
        return entry.get(stage), entry.get("source")
    except Exception:
        return None, None


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def cpu_baseline(scene, views, w, h, sample_s, threads=0):
    """The reference's `cpu` backend (oracle restatement), all host threads,
    over a bounded sample of the orbit."""
    from oracle import oracle as O

    cpu = O.CpuTiled(scene, threads=threads)
    out = np.zeros((h, w, 3), np.uint8)
    cpu.render(views[0], w, h, (0, 0, 0), out)  # warm-up
    times = []
    t_end = time.perf_counter() + sample_s
    i = 0
    while time.perf_counter() < t_end or i < 2:
        t0 = time.perf_counter()
        cpu.render(views[i % len(views)], w, h, (0, 0, 0), out)
        times.append(time.perf_counter() - t0)
        i += 1
    threads_used = cpu.threads
    cpu.close()
    return len(times) / sum(times), threads_used, len(times)


def cpu_naive_baseline(scene, views, w, h, sample_s):
    """The reference's `cpu-naive` backend (oracle restatement of
    src/render/naive.rs: global depth sort, every splat over its bbox, one
    thread) over a bounded sample of the orbit."""
    from oracle import oracle as O

    times = []
    t_end = time.perf_counter() + sample_s
    i = 0
    while time.perf_counter() < t_end or i < 1:
        t0 = time.perf_counter()
        O.render_naive(scene, views[i % len(views)], w, h)
        times.append(time.perf_counter() - t0)
        i += 1
    return len(times) / sum(times), len(times)


def run_reference(args):
    rank, world, _ = dist_env()
    if world > 1 and rank != 0:
        return
    cfg = CONFIGS[args.config]
    W, H = cfg["w"], cfg["h"]
    _, f32_scene, _, home, warm, timed = make_workload(args.splats, cfg)
    from oracle import oracle as O

    cpu = O.CpuTiled(f32_scene, threads=0)
    out = np.zeros((H, W, 3), np.uint8)
    for i in range(args.warmup):
        cpu.render(warm[i % len(warm)], W, H, (0, 0, 0), out)
    # Each step renders one frame; bound the run to a few minutes.
    steps = args.steps
    t_start = time.perf_counter()
    times = []
    for i in range(steps):
        t0 = time.perf_counter()
        cpu.render(timed[i % len(timed)], W, H, (0, 0, 0), out)
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_start > 120.0:
            break
    fps = len(times) / sum(times)
    threads = cpu.threads
    cpu.close()
    line = {
        "impl": "reference", "metric": cfg["metric"], "value": fps, "unit": "frames/s", "n_gpus": 0,
        "steps": len(times), "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": bench_config(cfg, args.splats, W, H, world),
        "cpu_baseline": {"value": fps, "unit": "frames/s", "cores": threads, "kind": "port",
                         "sample": f"{len(times)} frames of the orbit (full {W}x{H} frames)"},
        "e2e": {"value": fps, "unit": "frames/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def fp64_errors(device_frames, source_scene, decoded_scene, views, w, h):
    """Per-frame error of the device frames against the FP64 naive
    rasterizer, run on the decoded FP16 values and on the f32 source."""
    from oracle import oracle as O

    def as_dict(sc):
        return {"positions": sc.positions, "scales": sc.scales, "rotations": sc.rotations,
                "opacities": sc.opacities, "colors": sc.colors, "sh_rest": sc.sh_rest, "sh_degree": sc.sh_degree}

    rows = []
    for i, (img, v) in enumerate(zip(device_frames, views)):
        row = {"frame": i}
        for key, sc in (("decoded_fp16", decoded_scene), ("f32_source", source_scene)):
            ref, _, _ = O.render_naive_f64(as_dict(sc), v, w, h)
            row[key] = {"psnr_db": O.psnr(img, ref),
                        "max_abs": int(np.max(np.abs(img.astype(int) - ref.astype(int))))}
        rows.append(row)
    return rows


def home_frame_check(r, scene, home, w, h, host):
    """The reference bench's PSNR (src/bench.rs:51-59, 153-170): the home
    frame of the orbit, drawn by the device (default and exact blends, into
    pinned host memory through splat_cuda_render) against the reference's
    `cpu` backend (the oracle's restatement)."""
    from oracle import oracle as O
    from splat_b200 import _native as Nat

    cpu = O.CpuTiled(scene, threads=0)
    want, _ = cpu.render(home, w, h, (0, 0, 0))
    cpu.close()
    r.render_into(home, w, h, (0, 0, 0), host.data_ptr(), host.numel())
    fast = host.numpy().reshape(h, w, 3).copy()
    r.set_option(Nat.SPLAT_OPT_EXACT_BLEND, 1)
    r.render_into(home, w, h, (0, 0, 0), host.data_ptr(), host.numel())
    exact = host.numpy().reshape(h, w, 3).copy()
    r.set_option(Nat.SPLAT_OPT_EXACT_BLEND, 0)
    return {"frame": "home (orbit frame 0)", "psnr_db": O.psnr(fast, want),
            "max_abs": int(np.max(np.abs(fast.astype(int) - want.astype(int)))),
            "exact_blend_identical": bool(np.array_equal(exact, want)),
            "against": "cpu backend (C++ restatement of src/render/cpu.rs), same scene and view"}


def run_ours(args):
    import torch

    rank, world, local = dist_env()
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    cfg = CONFIGS[args.config]
    W, H = cfg["w"], cfg["h"]

    from splat_b200 import _native as Nat
    from splat_b200.render import CudaRenderer

    stored, f32_scene, source, home, warm, timed = make_workload(args.splats, cfg)
    views = shard(timed, rank, world)
    r = CudaRenderer(stored, device=dev)
    stream = torch.cuda.ExternalStream(r.stream())
    out = torch.empty(W * H * 3, dtype=torch.uint8, device=dev)
    nbytes = out.numel()

    # Home frame and warm-up; capacity growth settles here.
    for v in [home] + warm[: max(args.warmup, 3)]:
        while True:
            r.render_device(v, W, H, (0, 0, 0), out.data_ptr(), nbytes)
            _, regrown = r.finish()
            if not regrown:
                break

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    if args.profile:
        for i in range(args.steps):
            r.render_device(views[i % len(views)], W, H, (0, 0, 0), out.data_ptr(), nbytes)
            s, _ = r.finish()
        # The last profiled frame again, with the blend counting its evaluations
        # (launched after the profiled frames: outside a capture of their launches).
        r.set_option(Nat.SPLAT_OPT_COUNT_EVALS, 1)
        r.render_device(views[(args.steps - 1) % len(views)], W, H, (0, 0, 0), out.data_ptr(), nbytes)
        r.finish()
        evals = r.get_option(Nat.SPLAT_OPT_BLEND_EVALS)
        if rank == 0:
            print(json.dumps({"profile_frames": args.steps, "visible": s.visible, "pairs": s.overlaps,
                              "last_frame_blend_evaluations": evals}), flush=True)
        r.close()
        return

    # Timed region: K frames enqueued back to back on the renderer's stream.
    K = args.steps
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    launches0 = r.get_option(Nat.SPLAT_OPT_KERNEL_LAUNCHES)
    with Clocks(dev) as clk:
        start.record(stream)
        for i in range(K):
            r.render_device(views[i % len(views)], W, H, (0, 0, 0), out.data_ptr(), nbytes)
        end.record(stream)
        st_last, regrown = r.finish()
        barrier()
    launches = (r.get_option(Nat.SPLAT_OPT_KERNEL_LAUNCHES) - launches0) % (1 << 32)
    assert not regrown, "pair buffers overflowed inside the timed region"
    ms = start.elapsed_time(end)
    t_max = max_over_ranks(ms, dev)
    ms_max = t_max
    frames_total = K * world
    value = frames_total / (ms_max / 1e3)

    # Per-stage device times (the library's CUDA events on its stream), one
    # frame at a time over the orbit.
    sums = {"project_ms": 0.0, "sort_ms": 0.0, "raster_ms": 0.0}
    vis = ovl = 0
    for v in views:
        r.render_device(v, W, H, (0, 0, 0), out.data_ptr(), nbytes)
        s, _ = r.finish()
        sums["project_ms"] += s.project_ms
        sums["sort_ms"] += s.sort_ms
        sums["raster_ms"] += s.raster_ms
        vis += s.visible
        ovl += s.overlaps
    nv = len(views)
    stage = {k: v / nv for k, v in sums.items()}
    V, P = vis / nv, ovl / nv

    # The blend's work: pixel/splat evaluations after early termination
    # (a counting instantiation of the blend, outside the timed region).
    r.set_option(Nat.SPLAT_OPT_COUNT_EVALS, 1)
    evals = 0
    for v in views:
        r.render_device(v, W, H, (0, 0, 0), out.data_ptr(), nbytes)
        r.finish()
        evals += r.get_option(Nat.SPLAT_OPT_BLEND_EVALS)
    r.set_option(Nat.SPLAT_OPT_COUNT_EVALS, 0)
    E = evals / nv

    # End to end through the public C ABI: splat_cuda_render into pinned host memory.
    host = torch.empty(W * H * 3, dtype=torch.uint8).pin_memory()
    for v in warm[:3]:
        r.render_into(v, W, H, (0, 0, 0), host.data_ptr(), host.numel())
    barrier()
    t0 = time.perf_counter()
    for i in range(K):
        r.render_into(views[i % len(views)], W, H, (0, 0, 0), host.data_ptr(), host.numel())
    e2e_s = time.perf_counter() - t0
    te_max = max_over_ranks(e2e_s, dev)
    e2e = frames_total / te_max
    # Where an end-to-end frame's time goes: the device stages (frames written
    # through the host buffer's device mapping) and the call's wall time.
    e2e_stages = {"project_ms": 0.0, "sort_ms": 0.0, "raster_ms": 0.0, "call_ms": 0.0}
    for v in views:
        st_e = r.render_into(v, W, H, (0, 0, 0), host.data_ptr(), host.numel())
        e2e_stages["project_ms"] += st_e.project_ms / len(views)
        e2e_stages["sort_ms"] += st_e.sort_ms / len(views)
        e2e_stages["raster_ms"] += st_e.raster_ms / len(views)
        e2e_stages["call_ms"] += st_e.total_ms / len(views)

    errors = None
    if rank == 0 and cfg["precision"] == "fp16" and args.error_frames > 0:
        frames = []
        for v in views[: args.error_frames]:
            r.render_into(v, W, H, (0, 0, 0), host.data_ptr(), host.numel())
            frames.append(host.numpy().reshape(H, W, 3).copy())
        errors = fp64_errors(frames, source, f32_scene, views[: args.error_frames], W, H)

    if rank == 0:
        peak, peak_kind = measured_peaks()
        N = args.splats
        tiles = ((W + 15) // 16) * ((H + 15) // 16)
        # Algorithmic bytes per frame and stage:
        #   project: scene read once, tile rectangle per splat and record per visible splat written
        #   sort:    rectangles read by the count and scatter passes, pair words written by the
        #            scatter, read and written once by the per-tile sort
        #   raster:  pair words read, one record gathered per pair, ranges, u8 frame written
        bytes_stage = {
            "project": N * cfg["s_in"] + N * S_BIN + V * S_REC,
            "sort": 2 * N * S_BIN + P * 8 + 2 * P * 8,
            "raster": P * (8 + S_REC) + tiles * 8 + W * H * 3,
        }
        times = {"project": stage["project_ms"], "sort": stage["sort_ms"], "raster": stage["raster_ms"]}
        dom = max(times, key=times.get)
        achieved = bytes_stage[dom] / (times[dom] / 1e3) / 1e9
        traffic, traffic_src = profile_traffic(args.config, dom)
        load = scene_load(source, dev) if cfg["precision"] == "fp32" else None
        cpu = None
        if not args.no_cpu_baseline:
            fps, cores, frames = cpu_baseline(f32_scene, timed, W, H, args.cpu_sample_s)
            cpu = {"value": fps, "unit": "frames/s", "cores": cores, "kind": "port",
                   "sample": f"{frames} full {W}x{H} frames of the orbit (~{args.cpu_sample_s:.0f} s)"}
            nfps, nframes = cpu_naive_baseline(f32_scene, timed, W, H, min(args.cpu_sample_s, 10.0))
            cpu_naive = {"value": nfps, "unit": "frames/s", "cores": 1, "kind": "port",
                         "sample": f"{nframes} full {W}x{H} frames of the orbit",
                         "backend": "cpu-naive (src/render/naive.rs), one thread"}
        home_check = home_frame_check(r, f32_scene, home, W, H, host) if cfg["precision"] == "fp32" else None
        line = {
            "metric": cfg["metric"], "value": value, "unit": "frames/s", "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": bench_config(cfg, N, W, H, world),
            "frame": {"visible": V, "pairs": P},
            "gsplat_tiles_per_s": P * value / world / 1e9,
            "stages_ms": stage,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "traffic_source": traffic_src,
                         "peak_kind": peak_kind, "algorithmic_bytes": bytes_stage[dom]},
            "frame_hbm": {"bytes": sum(bytes_stage.values()),
                          "achieved_gbs": sum(bytes_stage.values()) * value / world / 1e9},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": "frames/s", "h2d_bytes_per_step": 56,
                    "d2h_bytes_per_step": W * H * 3 + 32,
                    "note": "input per step: the 56-byte view, passed as kernel parameters (the scene stays "
                            "resident); output: the u8 frame, written by the blend straight into the caller's "
                            "pinned host buffer through its device mapping, plus the 32-byte frame state",
                    "stages_ms": e2e_stages},
            "clocks": clk.summary(),
            "gpu_launches": launches,
        }
        if errors is not None:
            line["error_vs_fp64_naive"] = errors
        if home_check is not None:
            line["psnr_vs_cpu"] = home_check
        issue = profile_traffic(args.config, "blend_issue")[0]
        line["blend_work"] = {
            "evaluations_per_frame": E, "evaluations_per_pair": E / P if P else None,
            "bound_pairs_x_256": P * 256, "evaluations_per_s": E / (stage["raster_ms"] / 1e3),
            "note": "pixel/splat evaluations of the default blend after early termination (counted on the device "
                    "over the orbit, outside the timed region); the blend is bound by instruction issue, not HBM",
        }
        if issue:
            line["blend_work"]["issue"] = issue
        if load is not None:
            line["scene_load"] = load
        if cpu is not None:
            line["cpu_naive_baseline"] = cpu_naive
        print(json.dumps(line), flush=True)
    r.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def run_sharded(args):
    """The frame of the plain workload from splats sharded over the ranks
    (splat_cuda_shard_records -> all-to-all of the records ->
    splat_cuda_render_records -> all_gather of the windows). Timed with CUDA
    events on the current stream around whole frames (the library's calls
    block, so the span holds every rank part and exchange), max over ranks."""
    import datetime

    import torch
    import torch.distributed as dist

    from splat_b200 import _native as Nat
    from splat_b200 import multi
    from splat_b200.render import CudaRenderer, Frame

    rank, world, local = dist_env()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    cfg = CONFIGS["sharded"]
    W, H, RB = cfg["w"], cfg["h"], Nat.SPLAT_RECORD_BYTES
    scene, _, _, home, warm, timed = make_workload(args.splats, cfg)
    S = world if world > 1 else max(1, args.shards)
    mine = [rank] if world > 1 else list(range(S))
    n = len(scene)
    shards = {q: CudaRenderer(scene.shard(*multi.shard_range(n, q, S)), device=dev) for q in mine}
    wins = multi.row_windows(H, S)
    bounds = [r0 for r0, _ in wins] + [H]
    most = max(rows for _, rows in wins)
    outs = {q: torch.zeros((most, W, 3), dtype=torch.uint8, device=dev) for q in mine}
    sends = {q: torch.empty(max(n // S, 1) * RB * 2, dtype=torch.uint8, device=dev) for q in mine}
    gathered = [torch.empty((most, W, 3), dtype=torch.uint8, device=dev) for _ in range(S)]
    parts = {"select_ms": [], "draw_ms": [], "sent_bytes": []}

    def frame(v, record=False):
        res = {}
        for q in mine:
            t0 = time.perf_counter()
            res[q] = shards[q].shard_records(v, W, H, bounds, send=sends[q])
            if record:
                parts["select_ms"].append(1e3 * (time.perf_counter() - t0))
                parts["sent_bytes"].append(sum(res[q][1]) * RB)
            if res[q][0].numel() > sends[q].numel():
                sends[q] = res[q][0]
        for q in mine:
            row0, rows = wins[q]
            if world > 1:
                recs, _ = multi.exchange_records(res[q][0], res[q][1], RB, world)
            else:
                runs = []
                for p in mine:
                    send, counts, _ = res[p]
                    off = sum(counts[:q]) * RB
                    runs.append(send[off:off + counts[q] * RB])
                recs = torch.cat(runs)
            t0 = time.perf_counter()
            if rows:
                shards[q].render_records(v, W, H, (0, 0, 0), recs, row0, rows, out=outs[q][:rows])
            if record:
                parts["draw_ms"].append(1e3 * (time.perf_counter() - t0))
        if world > 1:
            dist.all_gather(gathered, outs[rank])
        else:
            for q in mine:
                gathered[q].copy_(outs[q])

    def assemble():
        f = np.empty((H, W, 3), np.uint8)
        for (r0, rows), g in zip(wins, gathered):
            if rows:
                f[r0:r0 + rows] = g[:rows].cpu().numpy()
        return f

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    for v in [home] + warm[: max(args.warmup, 3)] + timed[:8]:  # record buffers settle here
        frame(v)
    torch.cuda.synchronize()
    match = None
    if rank == 0:  # the home frame against the one-device frame of the whole scene
        frame(home)
        torch.cuda.synchronize()
        whole = CudaRenderer(scene, device=dev)
        f = Frame()
        whole.render(home, W, H, (0, 0, 0), f)
        whole.close()
        match = bool(np.array_equal(assemble(), f.pixels))
    elif world > 1:
        frame(home)
    views = timed
    K = args.steps
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = sum(r.get_option(Nat.SPLAT_OPT_KERNEL_LAUNCHES) for r in shards.values())
    barrier()
    with Clocks(dev) as clk:
        start.record()
        for i in range(K):
            frame(views[i % len(views)])
        end.record()
        barrier()
    launches = sum(r.get_option(Nat.SPLAT_OPT_KERNEL_LAUNCHES) for r in shards.values()) - launches0
    ms = max_over_ranks(start.elapsed_time(end), dev)
    value = K / (ms / 1e3)
    # End to end: each frame then also reaches pinned host memory on rank 0.
    host = torch.empty((H, W, 3), dtype=torch.uint8).pin_memory()
    barrier()
    t0 = time.perf_counter()
    for i in range(min(K, 200)):
        frame(views[i % len(views)])
        if rank == 0:
            for (r0, rows), g in zip(wins, gathered):
                if rows:
                    host[r0:r0 + rows].copy_(g[:rows], non_blocking=True)
            torch.cuda.synchronize()
    e2e = min(K, 200) / max_over_ranks(time.perf_counter() - t0, dev)
    for v in views[:8]:
        frame(v, record=True)
    if rank == 0:
        line = {
            "metric": cfg["metric"], "value": value, "unit": "frames/s", "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": ms / K, "higher_is_better": True, "scaling": "strong",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": dict(bench_config(cfg, n, W, H, world), parallelism=f"splat-sharded x{S}"
                           + ("" if world > 1 else " (emulated one after another on one GPU)")),
            "matches_whole_frame": match,
            "parts": {"select_ms_per_rank": float(np.median(parts["select_ms"])),
                      "draw_ms_per_window": float(np.median(parts["draw_ms"])),
                      "records_bytes_per_rank": float(np.median(parts["sent_bytes"])),
                      "note": "wall time of the blocking calls (this process's ranks), medians over 8 views"},
            "e2e": {"value": e2e, "unit": "frames/s", "h2d_bytes_per_step": 56 * S, "d2h_bytes_per_step": W * H * 3,
                    "note": "each frame also copied from the gathered windows to pinned host memory on rank 0"},
            "clocks": clk.summary(),
            "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    for r in shards.values():
        r.close()
    if world > 1:
        dist.destroy_process_group()


def learned_quality_correlated(args, W, H, dev):
    """The learned colour's quality where the SH carries structure: the same
    1.2M-splat geometry with the 45 higher coefficients generated from a
    4-dimensional code per splat (synth.cluster_scene(sh_code_dim=4)),
    trained as the main workload for twice its epochs, PSNR against exact
    SH over orbit frames."""
    from oracle import oracle as O
    from splat_b200 import Frame, synth
    from splat_b200.learned import LearnConfig, Learner, learned_renderer
    from splat_b200.render import CudaRenderer

    scene = synth.cluster_scene(args.splats, seed=0x5EED0001, sh_degree=3, sh_code_dim=4)
    cam = synth.orbit_camera(scene)
    _, _, timed = synth.orbit_views(cam, ORBIT, 5)
    exact = CudaRenderer(scene, device=dev)
    learner = Learner(exact, LearnConfig(directions=256, batch=65536, lr=1e-3, seed=1))
    ts = learner.train(max(1, int(round(2 * args.learn_epochs * learner.steps_per_epoch))))
    p16, lat16 = learner.params_f16()
    learner.close()
    r = learned_renderer(scene.to_fp16(), lat16, p16, device=dev)
    ps = []
    fe, fl = Frame(), Frame()
    for v in timed[: max(1, args.psnr_frames // 4)]:
        exact.render(v, W, H, (0, 0, 0), fe)
        r.render(v, W, H, (0, 0, 0), fl)
        ps.append(O.psnr(fl.pixels, fe.pixels))
    r.close()
    exact.close()
    return {"mean_db": float(np.mean(ps)), "min_db": float(np.min(ps)), "frames": len(ps), "epochs": ts.epochs,
            "scene": "the workload's geometry; SH rest coefficients from a 4-dim code per splat (std 0.08 each)"}


def run_learned(args):
    """Learned colour: train on the device, then time the learned renderer
    (and the exact-SH plain renderer of the same scene) over the orbit."""
    import torch

    rank, world, local = dist_env()
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    cfg = CONFIGS["learned"]
    W, H = cfg["w"], cfg["h"]
    from oracle import oracle as O  # PSNR and the CPU baseline only
    from splat_b200 import _native as Nat
    from splat_b200.learned import LearnConfig, Learner, learned_renderer
    from splat_b200.render import CudaRenderer

    scene, _, _, home, warm, timed = make_workload(args.splats, cfg)
    views = shard(timed, rank, world)
    exact = CudaRenderer(scene, device=dev)

    # Training (every rank trains its own replica: no exchange).
    learner = Learner(exact, LearnConfig(directions=256, batch=65536, lr=1e-3, seed=1))
    learner.train(1)  # warm-up: graph capture, clocks
    learner.set_params(*learner.params())
    steps = max(1, int(round(args.learn_epochs * learner.steps_per_epoch)))
    with Clocks(dev) as clk_train:
        ts = learner.train(steps)
    train_ctas = learner.option(Nat.LEARN_TRAIN_CTAS)
    p16, lat16 = learner.params_f16()
    learner.close()
    samples = ts.epochs * ts.samples_per_epoch
    flop_per_sample = 3 * 11008  # forward 11,008 FLOP; backward ~2x (activation and weight gradients)
    train_tflops = samples * flop_per_sample / (ts.ms / 1e3) / 1e12

    half = scene.to_fp16()
    r = learned_renderer(half, lat16, p16, device=dev)
    base = scene.to_fp16()
    base.sh = base.sh[:, :1, :].copy()
    base.sh_degree = 0
    rbase = CudaRenderer(base, device=dev)
    out = torch.empty(W * H * 3, dtype=torch.uint8, device=dev)
    nbytes = out.numel()

    def settle(rr):
        for v in [home] + warm[: max(args.warmup, 3)]:
            while True:
                rr.render_device(v, W, H, (0, 0, 0), out.data_ptr(), nbytes)
                if not rr.finish()[1]:
                    break

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    def timed_frames(rr, K):
        stream = torch.cuda.ExternalStream(rr.stream())
        start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        barrier()
        l0 = rr.get_option(Nat.SPLAT_OPT_KERNEL_LAUNCHES)
        start.record(stream)
        for i in range(K):
            rr.render_device(views[i % len(views)], W, H, (0, 0, 0), out.data_ptr(), nbytes)
        end.record(stream)
        _, regrown = rr.finish()
        barrier()
        assert not regrown, "pair buffers overflowed inside the timed region"
        t_max = max_over_ranks(start.elapsed_time(end), dev)
        return t_max, (rr.get_option(Nat.SPLAT_OPT_KERNEL_LAUNCHES) - l0) % (1 << 32)

    if args.profile:  # a short command for ncu: the training above, then --steps learned frames
        for i in range(args.steps):
            r.render_device(views[i % len(views)], W, H, (0, 0, 0), out.data_ptr(), nbytes)
            s, _ = r.finish()
        if rank == 0:
            print(json.dumps({"profile_train_steps": ts.steps, "profile_frames": args.steps, "visible": s.visible,
                              "pairs": s.overlaps}), flush=True)
        for x in (r, rbase, exact):
            x.close()
        return
    settle(r)
    settle(exact)
    K = args.steps
    with Clocks(dev) as clk:
        ms_max, launches = timed_frames(r, K)
    value = K * world / (ms_max / 1e3)
    ms_plain, _ = timed_frames(exact, K)
    plain_fps = K * world / (ms_plain / 1e3)

    sums = {"project_ms": 0.0, "sort_ms": 0.0, "raster_ms": 0.0}
    vis = ovl = 0
    for v in views:
        r.render_device(v, W, H, (0, 0, 0), out.data_ptr(), nbytes)
        s, _ = r.finish()
        for k in sums:
            sums[k] += getattr(s, k)
        vis += s.visible
        ovl += s.overlaps
    nv = len(views)
    stage = {k: v / nv for k, v in sums.items()}
    V, P = vis / nv, ovl / nv

    # End to end through the public C ABI into pinned host memory.
    host = torch.empty(W * H * 3, dtype=torch.uint8).pin_memory()
    for v in warm[:3]:
        r.render_into(v, W, H, (0, 0, 0), host.data_ptr(), host.numel())
    barrier()
    t0 = time.perf_counter()
    for i in range(K):
        r.render_into(views[i % len(views)], W, H, (0, 0, 0), host.data_ptr(), host.numel())
    te_max = max_over_ranks(time.perf_counter() - t0, dev)
    e2e = K * world / te_max

    # The batched form: the rank's orbit views as one recorded batch (one
    # graph replay draws them all), learned colour and FP16 geometry.
    from splat_b200.batch import BatchRenderer, BatchView

    bat = BatchRenderer([r], [BatchView(0, v, W, H) for v in views])
    bat.render()
    bstream = torch.cuda.ExternalStream(bat.stream())
    reps = max(1, K // max(len(views), 1))
    bs, be = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    bs.record(bstream)
    for _ in range(reps):
        bat.run()
    be.record(bstream)
    _, _, regrown = bat.finish()
    barrier()
    assert not regrown
    tb_max = max_over_ranks(bs.elapsed_time(be), dev)
    batched_fps = reps * len(views) * world / (tb_max / 1e3)
    bat.close()

    line = None
    if rank == 0:
        # Quality over the orbit: learned and base-colour-only against exact SH.
        from splat_b200 import Frame

        ps_l, ps_b, mx_l = [], [], []
        fe, fl, fb = Frame(), Frame(), Frame()
        for v in timed[: args.psnr_frames]:
            exact.render(v, W, H, (0, 0, 0), fe)
            r.render(v, W, H, (0, 0, 0), fl)
            rbase.render(v, W, H, (0, 0, 0), fb)
            ps_l.append(O.psnr(fl.pixels, fe.pixels))
            ps_b.append(O.psnr(fb.pixels, fe.pixels))
            mx_l.append(int(np.abs(fl.pixels.astype(int) - fe.pixels.astype(int)).max()))
        correlated = learned_quality_correlated(args, W, H, dev)
        peak, peak_kind = measured_peaks()
        try:
            tpeak = float(json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))["bf16_tflops_sustained"])
            tpeak_kind = "measured (sustained dense bf16 GEMM; fp16 runs at the same rate)"
        except Exception:
            tpeak, tpeak_kind = 1400.0, "fallback"
        N = args.splats
        tiles = ((W + 15) // 16) * ((H + 15) // 16)
        bytes_stage = {
            "project": N * cfg["s_in"] + N * S_BIN + V * S_REC,
            "sort": 2 * N * S_BIN + P * 8 + 2 * P * 8,
            "raster": P * (8 + S_REC) + tiles * 8 + W * H * 3,
        }
        times = {"project": stage["project_ms"], "sort": stage["sort_ms"], "raster": stage["raster_ms"]}
        dom = max(times, key=times.get)
        achieved = bytes_stage[dom] / (times[dom] / 1e3) / 1e9
        cpu = None
        if not args.no_cpu_baseline:
            fps, cores, frames = cpu_baseline(scene, timed, W, H, args.cpu_sample_s)
            cpu = {"value": fps, "unit": "frames/s", "cores": cores, "kind": "port",
                   "sample": f"{frames} full {W}x{H} frames of the orbit with exact SH (~{args.cpu_sample_s:.0f} s)"}
        line = {
            "metric": cfg["metric"], "value": value, "unit": "frames/s", "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (fp16 MLP operands, fp32 accumulate)", "data": "synthetic",
            "config": {"workload": cfg["workload"], "splats": N, "width": W, "height": H, "tile": 16,
                       "storage": "fp16 geometry + 16 fp16 latents", "visible": V, "pairs": P,
                       "parallelism": f"view-parallel x{world}",
                       "l2": f"inputs larger than L2 (scene {N * cfg['s_in'] / 1e6:.0f} MB + records)"},
            "plain_exact_sh_frames_per_s": plain_fps,
            "vs_plain": value / plain_fps,
            "batched_learned_frames_per_s": batched_fps,
            "batched_vs_plain": batched_fps / plain_fps,
            "psnr_vs_exact_sh": {"mean_db": float(np.mean(ps_l)), "min_db": float(np.min(ps_l)),
                                 "max_abs": int(max(mx_l)), "frames": len(ps_l)},
            "psnr_base_colour_vs_exact_sh": {"mean_db": float(np.mean(ps_b)), "min_db": float(np.min(ps_b))},
            "psnr_vs_exact_sh_correlated": correlated,
            "training": {"epochs": ts.epochs, "steps": ts.steps, "samples": int(samples), "ms": ts.ms,
                         "samples_per_s": samples / (ts.ms / 1e3), "final_loss": ts.last_loss,
                         "mean_loss_last_call": ts.mean_loss, "train_ctas": train_ctas,
                         "roofline": {"bound": "tensor", "achieved": train_tflops, "peak": tpeak,
                                      "unit": "TFLOP/s", "frac": train_tflops / tpeak, "peak_kind": tpeak_kind,
                                      "algorithmic_flop_per_sample": flop_per_sample},
                         "clocks": clk_train.summary()},
            "gsplat_tiles_per_s": P * value / world / 1e9,
            "stages_ms": stage,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": profile_traffic("learned", dom)[0],
                         "traffic_source": profile_traffic("learned", dom)[1], "peak_kind": peak_kind,
                         "algorithmic_bytes": bytes_stage[dom]},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": "frames/s", "h2d_bytes_per_step": 56,
                    "d2h_bytes_per_step": W * H * 3 + 32,
                    "note": "input per step: the 56-byte view (the trained scene stays resident); output: the u8 "
                            "frame, written by the blend straight into the caller's pinned host buffer through its "
                            "device mapping, plus the 32-byte frame state"},
            "clocks": clk.summary(),
            "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    for x in (r, rbase, exact):
        x.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def batch_workload(args):
    from splat_b200 import synth

    n = max(args.batch_scale, 1e-6)
    sizes = tuple(max(int(x * n), 1000) for x in (50_000, 400_000, 3_000_000))
    scenes = synth.batch_scenes(sizes=sizes)
    views = synth.batch_views(scenes, n_views=args.batch_views)
    return scenes, views


def run_batch_reference(args):
    """The oracle's cpu backend over the batch's views, one after another,
    all host threads, for a bounded time."""
    rank, world, _ = dist_env()
    if world > 1 and rank != 0:
        return
    cfg = CONFIGS["batch"]
    scenes, views = batch_workload(args)
    from oracle import oracle as O

    cpus = [O.CpuTiled(s, threads=0) for s in scenes]
    t_start = time.perf_counter()
    times, pixels = [], 0
    i = 0
    while i < len(views) * max(args.steps, 1):
        k, v, w, h = views[i % len(views)]
        out = np.zeros((h, w, 3), np.uint8)
        t0 = time.perf_counter()
        cpus[k].render(v, w, h, (0, 0, 0), out)
        times.append(time.perf_counter() - t0)
        pixels += w * h
        i += 1
        if time.perf_counter() - t_start > 120.0:
            break
    vps = len(times) / sum(times)
    threads = cpus[0].threads
    for c in cpus:
        c.close()
    line = {
        "impl": "reference", "metric": cfg["metric"], "value": vps, "unit": "views/s", "n_gpus": 0,
        "steps": len(times), "warmup": 0, "ms_per_step": 1e3 * sum(times) / len(times), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": cfg["workload"], "views": len(views)},
        "cpu_baseline": {"value": vps, "unit": "views/s", "cores": threads, "kind": "port",
                         "sample": f"{len(times)} views of the batch, one at a time"},
        "e2e": {"value": vps, "unit": "views/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_batch(args):
    """The batching workload: every view rendered one at a time through the
    single-view path (the baseline), then the whole batch as one recorded
    CUDA graph after the tuner picked its tile shape and block size."""
    import torch

    rank, world, local = dist_env()
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()
    cfg = CONFIGS["batch"]
    from splat_b200 import _native as Nat
    from splat_b200.batch import BatchRenderer, BatchView
    from splat_b200.render import CudaRenderer

    scenes, views_all = batch_workload(args)
    views = shard(views_all, rank, world)
    rends = [CudaRenderer(s, device=dev) for s in scenes]
    stream = torch.cuda.Stream(device=dev)
    for r in rends:
        r.set_stream(stream.cuda_stream)
    max_bytes = max(w * h * 3 for _, _, w, h in views)
    out = torch.empty(max_bytes, dtype=torch.uint8, device=dev)

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    if args.profile:
        # A short command for ncu: the batch with the default configuration,
        # --warmup + --steps replays.
        b = BatchRenderer(rends, [BatchView(k, v, w, h) for k, v, w, h in views])
        for _ in range(args.warmup + args.steps):
            stats, _ = b.render()
        if rank == 0:
            print(json.dumps({"profile_batches": args.steps, "visible": sum(x.visible for x in stats),
                              "pairs": sum(x.overlaps for x in stats)}), flush=True)
        b.close()
        for r in rends:
            r.close()
        return

    # Baseline: the single-view path, one view after another on one stream.
    for k, v, w, h in views:  # capacity growth settles here
        while True:
            rends[k].render_device(v, w, h, (0, 0, 0), out.data_ptr(), max_bytes)
            _, regrown = rends[k].finish()
            if not regrown:
                break
    K1 = max(1, args.steps // 10)
    s0, s1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    s0.record(stream)
    for _ in range(K1):
        for k, v, w, h in views:
            rends[k].render_device(v, w, h, (0, 0, 0), out.data_ptr(), max_bytes)
    s1.record(stream)
    barrier()
    single_vps = len(views) * K1 / (s0.elapsed_time(s1) / 1e3)

    # The batch: tuner, then K replays of the recorded graph.
    b = BatchRenderer(rends, [BatchView(k, v, w, h) for k, v, w, h in views])
    tune = b.autotune(reps=3)
    bstream = torch.cuda.ExternalStream(b.stream(), device=dev)
    for _ in range(max(args.warmup, 3)):
        b.render()
    K = args.steps
    launches0 = b.get_option(Nat.SPLAT_OPT_KERNEL_LAUNCHES)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    barrier()
    with Clocks(dev) as clk:
        start.record(bstream)
        for _ in range(K):
            b.run()
        end.record(bstream)
        stats, batch_ms, regrown = b.finish()
        barrier()
    launches = (b.get_option(Nat.SPLAT_OPT_KERNEL_LAUNCHES) - launches0) % (1 << 32)
    assert not regrown, "pair buffers overflowed inside the timed region"
    ms = start.elapsed_time(end)
    t_max = max_over_ranks(ms, dev)
    ms_max = t_max
    views_total = len(views_all) if world > 1 else len(views)
    value = views_total * K / (ms_max / 1e3)
    stats, _ = b.render()  # stage times of one batch
    stage = {"project_ms": stats[0].project_ms, "sort_ms": stats[0].sort_ms, "raster_ms": stats[0].raster_ms}

    # End to end: the batch plus every frame copied to pinned host memory.
    host = torch.empty(b.frames_dev.numel(), dtype=torch.uint8).pin_memory()
    barrier()
    t0 = time.perf_counter()
    for _ in range(K):
        b.run()
        with torch.cuda.stream(bstream):
            host.copy_(b.frames_dev, non_blocking=True)
        b.finish()
    e2e_s = time.perf_counter() - t0
    te_max = max_over_ranks(e2e_s, dev)
    e2e = views_total * K / te_max

    if rank == 0:
        peak, peak_kind = measured_peaks()
        N_in = sum(len(scenes[k].opacities) for k, _, _, _ in views)
        s_in = {0: 32, 1: 68, 2: 128, 3: 232}
        B_in = sum(len(scenes[k].opacities) * s_in[scenes[k].sh_degree] for k, _, _, _ in views)
        V = sum(s.visible for s in stats)
        P = sum(s.overlaps for s in stats)
        px = sum(w * h for _, _, w, h in views)
        tiles = sum(((w + 15) // 16) * ((h + 15) // 16) for _, _, w, h in views)
        bytes_stage = {
            "project": B_in + N_in * S_BIN + V * S_REC,
            "sort": 2 * N_in * S_BIN + P * 8 + 2 * P * 8,
            "raster": P * (8 + S_REC) + tiles * 8 + px * 3,
        }
        times = {"project": stage["project_ms"], "sort": stage["sort_ms"], "raster": stage["raster_ms"]}
        dom = max(times, key=times.get)
        achieved = bytes_stage[dom] / (times[dom] / 1e3) / 1e9
        cpu = None
        if not args.no_cpu_baseline:
            from oracle import oracle as O

            cpus = [O.CpuTiled(s, threads=0) for s in scenes]
            t_end = time.perf_counter() + args.cpu_sample_s
            n_cpu, t_cpu, i = 0, 0.0, 0
            while time.perf_counter() < t_end or n_cpu < 2:
                k, v, w, h = views[i % len(views)]
                o = np.zeros((h, w, 3), np.uint8)
                t1 = time.perf_counter()
                cpus[k].render(v, w, h, (0, 0, 0), o)
                t_cpu += time.perf_counter() - t1
                n_cpu += 1
                i += 1
            cpu = {"value": n_cpu / t_cpu, "unit": "views/s", "cores": cpus[0].threads, "kind": "port",
                   "sample": f"the first {n_cpu} views of the batch, one at a time (~{args.cpu_sample_s:.0f} s)"}
            for c in cpus:
                c.close()
        line = {
            "metric": cfg["metric"], "value": value, "unit": "views/s", "n_gpus": world, "steps": K,
            "warmup": args.warmup, "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": cfg["workload"], "views": views_total, "splats_projected": N_in,
                       "pixels": px, "visible": V, "pairs": P, "parallelism": f"view-parallel x{world}",
                       "blend_config": list(b.config), "l2": "inputs larger than L2 (scenes 0.8 GB > 126 MB)"},
            "single_view_path_views_per_s": single_vps,
            "batch_speedup_vs_single_view_path": value / world / single_vps if world == 1 else None,
            "tuner": [{"tile": [c[0], c[1]], "threads": c[2], "ms": m} for c, m in tune],
            "stages_ms": stage,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "peak_kind": peak_kind,
                         "algorithmic_bytes": bytes_stage[dom]},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e, "unit": "views/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": int(b.frames_dev.numel()),
                    "note": "the recorded batch replayed (views fixed in the graph), then every view's frame "
                            "copied to pinned host memory"},
            "clocks": clk.summary(),
            "gpu_launches": launches,
        }
        print(json.dumps(line), flush=True)
    # Free what torch used on the batch's and the renderers' streams before
    # those streams are destroyed.
    torch.cuda.synchronize()
    del host, out, bstream
    b.close()
    for r in rends:
        r.close()
    if world > 1:
        torch.distributed.destroy_process_group()


def run_profile_io(args):
    """The scene-file decoders and the terminal-cell kernel on the plain
    workload (see --profile-io)."""
    import torch

    from oracle import scene_io as IO
    from splat_b200 import _native as Nat
    from splat_b200.render import CudaRenderer, from_ply_bytes, from_splat_bytes

    torch.cuda.set_device(0)
    cfg = CONFIGS["plain"]
    scene, _, _, home, _, _ = make_workload(args.splats, cfg)
    ply, spl = IO.write_ply(scene), IO.write_splat(scene)
    for _ in range(args.steps):
        for data, loader in ((ply, from_ply_bytes), (spl, from_splat_bytes)):
            for prec in (Nat.SPLAT_PRECISION_FP32, Nat.SPLAT_PRECISION_FP16):
                loader(data, precision=prec).close()
    r = CudaRenderer(scene)
    for _ in range(args.steps):
        for mode in (Nat.SPLAT_CELLS_TRUECOLOR, Nat.SPLAT_CELLS_ANSI256):
            r.render_cells(home, cfg["w"], cfg["h"], (0, 0, 0), downsample=2, mode=mode)
    r.close()
    print(json.dumps({"profile_io": args.steps, "ply_bytes": len(ply), "splat_bytes": len(spl)}), flush=True)


def main():
    args = parse()
    if args.profile_io:
        run_profile_io(args)
        return
    if args.config == "batch":
        if args.impl == "reference":
            run_batch_reference(args)
        else:
            run_batch(args)
    elif args.impl == "reference":
        run_reference(args)
    elif args.config == "learned":
        run_learned(args)
    elif args.config == "sharded":
        run_sharded(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
