#!/usr/bin/env python
"""Benchmark of the B200 point-cloud compute rasteriser.

Workload (default): HQS frames of a 100,000,000-point fractal heightfield
(4 km x 4 km, 6 octaves, amplitude 200 m, 5% volumetric outliers, RGB8 from a
height ramp + N(0, 10)), packed on the GPU into 10,240-point Morton batches
(30-bit keys), rendered at 1920x1080 from 32 seeded poses 300 m above the
local terrain (yaw uniform, pitch -20..-45 deg, 60 deg vertical fov).  A step
is one frame (cull, clear, depth, colour, resolve) at the next pose.

Prints one JSON line (rank 0):
  value   cloud points per second over the timed frames (Gpts/s), device
          timed with CUDA events on the library's stream, max over ranks;
  e2e     the same metric through the public API per frame: camera upload
          (file table from pinned memory), render, RGBA8 read-back into
          pinned host memory (asynchronous, overlapped with the next frame's
          render; the blocking read-back is reported beside it), wall-clock;
  roofline  the dominant pass (largest average device time): algorithmic
          bytes per launch (level bytes + split-precision words of every
          survivor point [+ colour words]) / its average duration from the
          per-pass CUDA events of the timed frames, against the measured
          HBM copy bandwidth;
  cpu_baseline  the CPU oracle (single-threaded C++ restatement of the
          reference passes) on whole frames of the same cloud, with a
          bit-exact comparison of the first frame against the GPU.
`--impl reference` times the oracle with every host thread instead.
Multi-GPU (torchrun): every rank renders its own poses of its own copy of the
cloud; no collective on the data path (weak scaling).
"""
from __future__ import annotations

import argparse
import importlib
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Gpts/s HQS 1080p @100M pts (%HBM roofline); 64-view batched vs per-view, bit-exact"
PASS_NAMES = ("clear", "cull", "depth", "color", "resolve", "hole_fill")


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=64)
    ap.add_argument("--warmup", type=int, default=8)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--points", type=int, default=100_000_000)
    ap.add_argument("--width", type=int, default=1920)
    ap.add_argument("--height", type=int, default=1080)
    ap.add_argument("--poses", type=int, default=32)
    ap.add_argument("--mode", default="hqs", choices=["hqs", "nearest"])
    ap.add_argument("--seed", type=lambda s: int(s, 0), default=0xC0FFEE02)
    ap.add_argument("--cpu-seconds", type=float, default=12.0,
                    help="target CPU time of the baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--parity-poses", type=int, default=-1,
                    help="timed poses compared bit for bit with the oracle in both modes "
                         "(-1 = all of them, 0 = none)")
    ap.add_argument("--pack-check-points", type=int, default=100_000_000,
                    help="points of the packer's bit-exact comparison with the oracle's "
                         "pack (0 = skip it)")
    ap.add_argument("--chunk-points", type=int, default=None,
                    help="points per work record of the point passes (launch tuning)")
    ap.add_argument("--tiles", type=int, default=None, choices=[0, 1],
                    help="shared-memory screen tiles on/off (launch tuning)")
    ap.add_argument("--mv-views", type=int, default=64,
                    help="views of the batched multi-view comparison (0 = skip it)")
    ap.add_argument("--mv-points", type=int, default=50_000_000)
    ap.add_argument("--mv-reps", type=int, default=5)
    ap.add_argument("--diff-points", type=int, default=20_000_000,
                    help="points of the differentiable-colour leg (0 = skip it)")
    ap.add_argument("--diff-views", type=int, default=32)
    ap.add_argument("--diff-check", type=int, default=1000,
                    help="points whose gradient is checked against the FP64 oracle (0 = none)")
    ap.add_argument("--pack-points", type=int, default=400_000_000,
                    help="points of the 63-bit packer leg (0 = skip it)")
    ap.add_argument("--stream-points", type=int, default=20_000_000,
                    help="points of the streaming-residency leg (0 = skip it)")
    ap.add_argument("--stream-frames", type=int, default=96)
    ap.add_argument("--ply-points", type=int, default=20_000_000,
                    help="points of the PLY leg's binary file (ASCII: a tenth; 0 = skip it)")
    ap.add_argument("--shard", default="frames", choices=["frames", "points"],
                    help="N>1: every rank renders its own frames of its own copy of the cloud "
                         "(frames, weak scaling), or every frame is split by batches over the "
                         "ranks with a depth max and a colour sum all-reduce (points, strong "
                         "scaling)")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# Multi-process plumbing
# ---------------------------------------------------------------------------
def pose_order(rank: int, world: int, n: int, poses: int) -> list:
    """The poses rank `rank` renders, in order: ranks interleave over the pose
    list, so each renders its own frames (weak scaling)."""
    return [(rank + world * k) % poses for k in range(n)]


class Dist:
    """Ranks from the torchrun environment; NCCL on GPUs (one per rank), gloo
    for the CPU tests of the multi-rank helpers."""

    def __init__(self, backend: str = "nccl", group_of_one: bool = False):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.pg = None
        if self.world > 1 or group_of_one:
            if self.world == 1:  # a process group of one rank (frames split by points)
                os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
                if "MASTER_PORT" not in os.environ:
                    import socket
                    with socket.socket() as sk:
                        sk.bind(("127.0.0.1", 0))
                        os.environ["MASTER_PORT"] = str(sk.getsockname()[1])
                os.environ.setdefault("RANK", "0")
                os.environ.setdefault("WORLD_SIZE", "1")
            import datetime

            import torch
            import torch.distributed as dist
            kw = {}
            if backend == "nccl":
                torch.cuda.set_device(self.local)
                kw["device_id"] = torch.device("cuda", self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120), **kw)
            self.pg = dist

    def barrier(self):
        if self.pg:
            self.pg.barrier()

    def max(self, x: float) -> float:
        if not self.pg:
            return x
        import torch
        dev = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        t = torch.tensor([x], dtype=torch.float64, device=dev)
        self.pg.all_reduce(t, op=self.pg.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.pg.destroy_process_group()


# ---------------------------------------------------------------------------
# Workload
# ---------------------------------------------------------------------------
class Camera:
    """A benchmark pose: a right-handed view looking down -Z and a reverse-Z
    perspective projection (near -> 1, far -> 0), both column-major
    float32[16], computed in float64 and rounded once, as the library's
    PerspectiveCamera computes them.  Defined here so that both arms build
    identical matrices and the reference arm needs nothing from the library."""

    def __init__(self, position, target, up=(0.0, 0.0, 1.0), near=1.0, far=10000.0,
                 fov=60.0, aspect=1.0):
        self.position = np.asarray(position, np.float64)
        self.target = np.asarray(target, np.float64)
        self.up = np.asarray(up, np.float64)
        self.near, self.far, self.fov, self.aspect = near, far, fov, aspect
        f = self.target - self.position
        f = f / np.linalg.norm(f)
        s = np.cross(f, self.up)
        s = s / np.linalg.norm(s)
        u = np.cross(s, f)
        m = np.eye(4)
        m[0, :3], m[1, :3], m[2, :3] = s, u, -f
        m[0, 3], m[1, 3], m[2, 3] = -s @ self.position, -u @ self.position, f @ self.position
        self._view = np.ascontiguousarray(m.astype(np.float32).T.reshape(16))

    @property
    def viewMatrix(self) -> np.ndarray:
        return self._view.copy()

    @property
    def projectionMatrix(self) -> np.ndarray:
        t = 1.0 / math.tan(math.radians(self.fov) * 0.5)
        n, fa = self.near, self.far
        m = np.zeros((4, 4))
        m[0, 0] = t / self.aspect
        m[1, 1] = t
        m[2, 2] = n / (fa - n)
        m[2, 3] = fa * n / (fa - n)
        m[3, 2] = -1.0
        return np.ascontiguousarray(m.astype(np.float32).T.reshape(16))


def make_poses(height, extent, n, seed, aspect):
    """n seeded cameras 300 m above the local terrain (height(x, y)), looking
    20-45 deg down."""
    rng = np.random.default_rng(seed ^ 0x5EED)
    cams = []
    for _ in range(n):
        x, y = rng.uniform(0.15, 0.85, 2) * extent
        z = height(x, y) + 300.0
        yaw = rng.uniform(0.0, 2.0 * math.pi)
        pitch = math.radians(rng.uniform(-45.0, -20.0))
        d = np.array([math.cos(pitch) * math.cos(yaw), math.cos(pitch) * math.sin(yaw),
                      math.sin(pitch)])
        cams.append(Camera((x, y, z), np.array([x, y, z]) + d, aspect=aspect))
    return cams


def lib_poses(cr, params, n, seed, aspect):
    """make_poses over the library's terrain height."""
    return make_poses(lambda x, y: cr.terrain_height(params, x, y), params.extent, n, seed,
                      aspect)


def words_per_point(level):
    return np.where(level == 0, 3, np.where(level == 1, 2, 1))


def pass_bytes(visible):
    """Algorithmic HBM bytes of the depth and colour passes for one frame's
    survivor list: every survivor point reads its level byte and 4 B per
    split-precision word of the batch's level (3/2/1 words at level 0/1/>=2);
    the colour pass also reads its 4 B colour."""
    if len(visible) == 0:
        return 0, 0, 0
    act = visible["activePoints"].astype(np.int64)
    w = words_per_point(visible["level"])
    depth = int(np.sum(act * (1 + 4 * w)))
    color = int(np.sum(act * (1 + 4 * w + 4)))
    return depth, color, int(act.sum())


class ClockSampler:
    """SM clock and clock-event reasons sampled during the timed region.

    NVML (the device found by its PCI bus id, so the index CUDA sees does not
    matter) polled every millisecond in a thread; only samples between
    begin() and end() count.  Falls back to nvidia-smi at 200 ms."""
    REASONS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
               "hw_thermal_slowdown": 0x40, "hw_power_brake_slowdown": 0x80}
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.samples = []  # (t, sm_mhz, reasons mask)
        self.max_mhz = None
        self._stop = threading.Event()
        self._t = None
        self._t0 = self._t1 = None
        self._nvml = None
        self.proc = None
        self.lines = []

    def _handle(self):
        import pynvml
        import torch
        pynvml.nvmlInit()
        pr = torch.cuda.get_device_properties(self.device)
        bus = f"{pr.pci_domain_id:08x}:{pr.pci_bus_id:02x}:{pr.pci_device_id:02x}.0"
        return pynvml, pynvml.nvmlDeviceGetHandleByPciBusId(bus.encode())

    def start(self):
        try:
            nv, h = self._handle()
            self._nvml = nv
            self.max_mhz = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            get_reasons = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons

            def poll():
                while not self._stop.is_set():
                    self.samples.append((time.perf_counter(),
                                         float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                         int(get_reasons(h))))
                    time.sleep(0.001)

            self._t = threading.Thread(target=poll, daemon=True)
            self._t.start()
            while not self.samples:
                time.sleep(0.001)
        except Exception:  # no NVML: nvidia-smi
            self._nvml = None
            try:
                self.proc = subprocess.Popen(
                    ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.QUERY}",
                     "--format=csv,noheader,nounits", "-lms", "200"],
                    stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
                self._t = threading.Thread(target=self._read, daemon=True)
                self._t.start()
                time.sleep(0.3)
            except (FileNotFoundError, OSError):
                self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def begin(self):
        self._t0 = time.perf_counter()

    def end(self):
        self._t1 = time.perf_counter()
        time.sleep(0.003)  # one more sample after the region

    def stop(self) -> dict:
        if self._nvml is not None:
            self._stop.set()
            self._t.join(timeout=2)
            inside = [x for x in self.samples if self._t0 <= x[0] <= self._t1]
            if not inside:  # region shorter than one poll: the first sample after it
                inside = [x for x in self.samples if x[0] > self._t1][:1]
            reasons = sorted(n for n, bit in self.REASONS.items()
                             if any(m & bit for _, _, m in inside))
            return {"sm_mhz": statistics.median(x[1] for x in inside) if inside else None,
                    "sm_max_mhz": self.max_mhz, "reasons": reasons, "samples": len(inside),
                    "source": "nvml 1 ms"}
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi 200 ms"}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def ncu_traffic(workload: str, kernel: str):
    """DRAM bytes per launch of `kernel` on `workload` from a committed ncu summary."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            d = json.load(f)
        return d[workload][kernel]
    except (OSError, KeyError, ValueError):
        return None


def ncu_kernel_figures(kernel: str):
    """Issue and L2-atomic figures of `kernel` from a committed ncu summary
    (profiles/kernel_figures.json: one small-case capture of that kernel)."""
    try:
        with open(os.path.join(ROOT, "profiles", "kernel_figures.json")) as f:
            return json.load(f)[kernel]
    except (OSError, KeyError, ValueError):
        return None


def build_cloud(cr, ctx, args, params):
    ppb = 10240
    nb = (args.points + ppb - 1) // ppb
    recs = cr.synth_terrain(ctx, params, args.points)
    cloud = cr.ComputeRasteriserPointCloud(ctx, cr.ComputeRasteriserCapacity(nb, ppb))
    t0 = time.perf_counter()
    cr.GPUPacker(ctx).pack(records=recs, into=cloud)
    ctx.synchronize()
    pack_s = time.perf_counter() - t0
    recs.close()
    ctx.trim()
    return cloud, pack_s


def oracle_cloud(orc, cloud):
    pts = cloud.points()
    return orc.Cloud(batches=cloud.batches(), files=cloud.files(), xyzLow=pts["xyzLow"],
                     xyzMed=pts["xyzMed"], xyzHigh=pts["xyzHigh"], colors=pts["colors"],
                     levels=pts["levels"])


def oracle_config(orc, cfg):
    return orc.Config(mode=cfg.mode, depthTolerance=cfg.depthTolerance,
                      backgroundColor=tuple(cfg.backgroundColor),
                      enableFrustumCulling=cfg.enableFrustumCulling, lodBias=cfg.lodBias,
                      enableCLOD=cfg.enableCLOD, enableLODDither=cfg.enableLODDither,
                      holeFillIterations=cfg.holeFillIterations,
                      pointSizeMode=cfg.pointSizeMode, minimumPointSize=cfg.minimumPointSize,
                      maximumPointSize=cfg.maximumPointSize, pointSizeScale=cfg.pointSizeScale)


def config_dict(args):
    return {"workload": f"{args.mode}_{args.width}x{args.height}_{args.points // 1_000_000}M"
                        "_heightfield",
            "points": args.points, "width": args.width, "height": args.height,
            "poses": args.poses, "points_per_batch": 10240, "morton_bits": 30,
            "mode": args.mode, "shard": args.shard,
            "l2": "inputs larger than L2 (1.7 GB resident slot pool per 100M points)"}


# ---------------------------------------------------------------------------
# Our arm
# ---------------------------------------------------------------------------
def run_ours(args, dist):
    cr = importlib.import_module("satin-computerasteriser_b200")
    import torch
    ctx = cr.Context(dist.local)
    ctx.set_tuning(chunkPoints=args.chunk_points, useTiles=None if args.tiles is None
                   else bool(args.tiles))
    params = cr.TerrainParams(seed=args.seed)
    cloud, pack_s = build_cloud(cr, ctx, args, params)
    W, H = args.width, args.height
    ras = cr.ComputeRasteriser(ctx)
    ras.configuration = cr.ComputeRasteriserConfiguration(
        mode=cr.MODE_HQS if args.mode == "hqs" else cr.MODE_NEAREST)
    ras.addPointCloud(cloud)
    ras.resize((W, H))
    cams = lib_poses(cr, params, args.poses, args.seed, W / H)
    frame_encoder = ras
    if args.shard == "points":
        if args.mode != "hqs":
            raise SystemExit("--shard points needs --mode hqs")
        # Every rank keeps its contiguous part of the batches (slot layout and
        # point indices as in the whole cloud) and renders every frame; the
        # planes are combined over NCCL between the stages.
        sharded = importlib.import_module("satin-computerasteriser_b200.sharded")
        nb = cloud.residentBatchCount
        lo, hi = sharded.shard_range(nb, dist.rank, dist.world)
        drop = [b for b in range(nb) if not lo <= b < hi]
        if drop:
            cloud.removeBatches(drop)
        frame_encoder = sharded.PointShardedRasteriser(ras)
        order = pose_order(0, 1, args.warmup + args.steps, args.poses)
    else:
        order = pose_order(dist.rank, dist.world, args.warmup + args.steps, args.poses)

    # Survivor lists of every pose (untimed) for the algorithmic byte counts.
    pose_bytes = {}
    for p in sorted(set(order)):
        ras.update(cams[p])
        ras.encode()
        pose_bytes[p] = pass_bytes(cloud.visibleBatches())
    for k in range(args.warmup):
        ras.update(cams[order[k]])
        frame_encoder.encode()
    ctx.synchronize()

    stream = torch.cuda.ExternalStream(ctx.stream(), device=f"cuda:{dist.local}")
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(dist.local)
    dist.barrier()
    ctx.synchronize()
    sampler.start()
    timed = order[args.warmup:]
    sampler.begin()
    ev0.record(stream)
    for p in timed:
        ras.update(cams[p])
        frame_encoder.encode()
    ev1.record(stream)
    ev1.synchronize()
    sampler.end()
    clocks = sampler.stop()
    ctx.synchronize()
    dist.barrier()
    ms = ev0.elapsed_time(ev1)
    # Per-pass times from a second run of the same frames with a CUDA event
    # around every pass; the timed run above records none, so that the
    # passes follow one another as they do for a user.
    ctx.set_profiling(True)
    for p in timed:
        ras.update(cams[p])
        frame_encoder.encode()
    ctx.synchronize()
    times = ctx.pass_times(len(timed))
    ctx.set_profiling(False)
    ms_max = dist.max(ms)
    # Points drawn per frame by all ranks: their own frames' clouds (frames),
    # or one cloud split over them (points).
    units = args.points * (dist.world if args.shard == "frames" else 1)
    value = units * args.steps / (ms_max / 1e3) / 1e9

    # Dominant pass and its roofline.
    avg = times.mean(axis=0)
    dom = int(np.argmax(avg))
    b_depth = np.array([pose_bytes[p][0] for p in timed], np.float64)
    b_color = np.array([pose_bytes[p][1] for p in timed], np.float64)
    active = np.array([pose_bytes[p][2] for p in timed], np.float64)
    dom_bytes = b_depth if PASS_NAMES[dom] == "depth" else b_color
    dom_ms = times[:, dom].astype(np.float64)
    achieved = float(dom_bytes.mean() / (dom_ms.mean() / 1e3) / 1e9)
    peak, peak_kind = measured_peaks()
    # Single-pixel footprints: the depth pass emits fragments (PASS_DEPTH_FRAG
    # = 3) and the colour pass reads them (color_hash_kernel).
    kernel = {"depth": "depth_kernel<3>", "color": "color_hash_kernel"}.get(PASS_NAMES[dom],
                                                                           PASS_NAMES[dom])
    roofline = {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(achieved / peak, 4), "peak_source": peak_kind,
                "kernel": kernel, "pass": PASS_NAMES[dom],
                "bytes_per_launch": int(dom_bytes.mean()),
                "launch_ms": round(float(dom_ms.mean()), 4),
                "traffic": ncu_traffic(config_dict(args)["workload"], PASS_NAMES[dom])}
    # The whole frame against the same peak: both point passes' algorithmic
    # bytes plus 48 B per pixel (clear 20, resolve read 20, RGBA8 write 4,
    # float depth write 4) over the device-timed frame.
    frame_bytes = float((b_depth + b_color).mean()) + 48.0 * W * H
    frame_gbs = frame_bytes / (ms_max / len(timed) / 1e3) / 1e9
    roofline["frame"] = {"bytes_per_frame": int(frame_bytes), "achieved": round(frame_gbs, 1),
                         "frac": round(frame_gbs / peak, 4)}
    # The instruction-issue bound and the L2 atomic rate of the same kernel,
    # from its small-case ncu capture (instructions per survivor point, the
    # fraction of the SMs' issue slots used, L2 reduction/atomic throughput
    # as a fraction of its peak).
    figures = ncu_kernel_figures(kernel)
    if figures:
        roofline["issue"] = {k: figures[k] for k in ("inst_per_survivor_point", "issue_frac",
                                                     "source") if k in figures}
        if "l2_atomic_frac" in figures:
            roofline["l2_atomic_frac"] = figures["l2_atomic_frac"]

    # End to end through the public API: per frame camera upload, render,
    # RGBA8 read-back into pinned host memory.  Pipelined: frame k's image is
    # copied (outputRGBA8Async, three pinned buffers) while frame k+1
    # renders; the host sets the next frame's camera (encode has already
    # captured frame k's), then waits until at most the latest copy (frame
    # k-1's) is still travelling, so that frame k-2's image is complete and
    # its buffer free, and enqueues frame k's.  (Waiting for frame k-1's copy
    # instead left the GPU idle between frames whenever that copy ended
    # later in frame k than the host's 77 µs of per-frame work allowed.)  The
    # clock stops after the last copy.
    # One untimed frame first creates the copy stream and events, then the
    # loop runs three times and the median is reported (host-side noise).
    pinned = [cr.HostBuffer((H, W, 4), np.uint8) for _ in range(3)]
    ras.update(cams[timed[0]])
    frame_encoder.encode()
    ras.outputRGBA8Async(pinned[0].array)
    ras.waitOutput()

    waits = []  # host seconds spent waiting for read-backs, per run

    def e2e_loop():
        dist.barrier()
        ctx.synchronize()
        t0 = time.perf_counter()
        waited = 0.0
        ras.update(cams[timed[0]])
        for k in range(len(timed)):
            frame_encoder.encode()
            if k + 1 < len(timed):
                ras.update(cams[timed[k + 1]])
            tw = time.perf_counter()
            ras.waitOutput(keep=1)
            waited += time.perf_counter() - tw
            ras.outputRGBA8Async(pinned[k % 3].array)
        ras.waitOutput()
        waits.append(waited)
        return dist.max(time.perf_counter() - t0)

    e2e_runs = [e2e_loop() for _ in range(3)]
    e2e_max = statistics.median(e2e_runs)
    last_ok = bool(np.array_equal(pinned[(len(timed) - 1) % 3].array, ras.outputRGBA8()))
    # The same loop with a blocking read-back per frame, for comparison.
    dist.barrier()
    ctx.synchronize()
    t0 = time.perf_counter()
    for p in timed:
        ras.update(cams[p])
        frame_encoder.encode()
        ras.outputRGBA8(out=pinned[0].array)
    blocking_max = dist.max(time.perf_counter() - t0)
    e2e = {"value": round(units * args.steps / e2e_max / 1e9, 4),
           "unit": "Gpts/s", "h2d_bytes_per_step": 256, "d2h_bytes_per_step": W * H * 4,
           "ms_per_step": round(e2e_max * 1e3 / args.steps, 4),
           "readback": "asynchronous, overlapped with the next frame (3 pinned buffers; "
                       "the host waits for frame k-2's copy before enqueuing frame k's)",
           "timing": "wall clock, median of 3 runs of the timed poses (max over ranks)",
           "runs_ms_per_step": [round(x * 1e3 / args.steps, 4) for x in e2e_runs],
           # Host time per frame outside the read-back waits (camera update,
           # encode, enqueueing the copy): when it exceeds the part of a
           # frame the wait leaves, the GPU idles between frames.
           "host_ms_per_step": round(statistics.median(
               [(r - w) * 1e3 / args.steps for r, w in zip(e2e_runs, waits)]), 4),
           "last_image_matches_blocking_read": last_ok,
           "blocking_readback": {
               "value": round(units * args.steps / blocking_max / 1e9, 4),
               "ms_per_step": round(blocking_max * 1e3 / args.steps, 4)}}

    out = {"metric": METRIC, "value": round(value, 4), "unit": "Gpts/s", "n_gpus": dist.world,
           "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(ms_max / args.steps, 4), "higher_is_better": True,
           "scaling": "weak" if args.shard == "frames" else "strong",
           "vs_baseline": None, "dtype": "f32+u32",
           "data": "synthetic (seeded fractal heightfield, generated and packed on the GPU)",
           "config": config_dict(args), "e2e": e2e, "roofline": roofline, "clocks": clocks,
           # HQS: the cull (whose trailing CTAs clear the frame), depth,
           # colour, resolve, and the exact re-run, which returns at once
           # unless a pixel passed 16,843,009 samples.  A frame split by
           # points has no re-run (its colour adds are unpacked) but two
           # depth-order flips.  Nearest: cull, nearest pass, resolve.
           "gpu_launches": int(args.steps * (
               (6 if args.shard == "points" else 5) if args.mode == "hqs" else 3)),
           "pass_ms": {n: round(float(v), 4) for n, v in zip(PASS_NAMES, avg)},
           "survivor_points_per_frame": int(active.mean()),
           "survivors_by_pose": {int(p): int(pose_bytes[p][2]) for p in sorted(pose_bytes)},
           "tuning": ctx.tuning(),
           "pack_s": round(pack_s, 3)}

    out["timed_poses"] = [int(p) for p in timed]
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        out["cpu_baseline"] = cpu_baseline(args, cr, ctx, ras, cloud, cams)
    if dist.world == 1 and args.mode == "hqs" and args.shard == "frames":
        out["nearest"] = run_nearest(args, cr, ctx, ras, cloud, cams, timed, stream)
    if dist.world == 1 and args.shard == "frames" and args.parity_poses != 0:
        chk = timed if args.parity_poses < 0 else timed[:args.parity_poses]
        modes = ("hqs", "nearest") if args.mode == "hqs" else ("nearest",)
        out["parity"] = {m: parity_poses(args, cr, ras, cloud, cams, chk,
                                         cr.MODE_HQS if m == "hqs" else cr.MODE_NEAREST)
                         for m in modes}
    for b in pinned:
        b.close()
    if args.mv_views > 0:
        out["multiview"] = run_multiview(args, cr, ctx, torch, dist)
    if args.diff_points > 0:
        out["differentiable"] = run_differentiable(args, cr, ctx, torch, dist)
    if args.stream_points > 0:
        out["streaming"] = run_streaming(args, cr, ctx, dist)
    if args.ply_points > 0 and dist.rank == 0:
        out["ply"] = run_ply(args, cr, ctx)
    if args.pack_points > 0:
        cloud.close()
        out["packer"] = run_packer(args, cr, ctx, torch, dist)
    return out


def run_ply(args, cr, ctx):
    """PLY input: a binary little-endian file of --ply-points vertices (float
    x, y, z; uchar red, green, blue, alpha: 16 B each) and an ASCII file of a
    tenth as many, written to a temporary directory; parsed with every host
    thread and with one (the reference's loader is single-threaded), and the
    binary file loaded end to end (parse + GPU pack into a slot pool)."""
    import os
    import tempfile
    rng = np.random.default_rng(args.seed ^ 0x91)
    n = args.ply_points
    rec = np.zeros(n, np.dtype([("p", "<f4", 3), ("c", "u1", 4)]))
    rec["p"] = rng.normal(0.0, 100.0, (n, 3))
    rec["c"] = rng.integers(0, 256, (n, 4))
    head = ("ply\nformat {fmt} 1.0\nelement vertex {n}\nproperty float x\nproperty float y\n"
            "property float z\nproperty uchar red\nproperty uchar green\nproperty uchar blue\n"
            "property uchar alpha\nend_header\n")
    threads = os.cpu_count() or 1
    out = {"threads": threads}
    with tempfile.TemporaryDirectory() as d:
        bpath, apath = os.path.join(d, "b.ply"), os.path.join(d, "a.ply")
        with open(bpath, "wb") as f:
            f.write(head.format(fmt="binary_little_endian", n=n).encode())
            rec.tofile(f)
        m = max(1, n // 10)
        with open(apath, "wb") as f:
            f.write(head.format(fmt="ascii", n=m).encode())
            np.savetxt(f, np.column_stack([rec["p"][:m].astype(np.float64),
                                           rec["c"][:m].astype(np.float64)]),
                       fmt=["%.7g"] * 3 + ["%d"] * 4)
        for name, path, cnt in (("binary", bpath, n), ("ascii", apath, m)):
            size = os.path.getsize(path)
            cr.PLYPointCloudLoader.read(path, threads=threads)  # page cache warm
            res = {"points": cnt, "mb": round(size / 1e6, 1)}
            for key, th in (("all_threads", threads), ("one_thread", 1)):
                t0 = time.perf_counter()
                pos, col = cr.PLYPointCloudLoader.read(path, threads=th)
                dt = time.perf_counter() - t0
                res[key] = {"s": round(dt, 4), "mb_per_s": round(size / 1e6 / dt, 1),
                            "mpts_per_s": round(cnt / 1e6 / dt, 2)}
            res["speedup"] = round(res["one_thread"]["s"] / res["all_threads"]["s"], 2)
            out[name] = res
        pos = col = None
        t0 = time.perf_counter()
        cloud = cr.PLYPointCloudLoader.load(ctx, bpath, pointsPerBatch=10240, threads=threads)
        ctx.synchronize()
        out["binary_load_s"] = round(time.perf_counter() - t0, 4)
        out["binary_load_points"] = cloud.pointCount
        cloud.close()
    out["timing"] = "wall clock; files in the page cache; load = parse + GPU pack"
    return out


class _SyncUploads:
    """A cloud whose adapter uploads copy synchronously (the reference's
    addBatches, ComputeRasteriserPointCloud.swift:410-452): the comparison arm
    of the streaming leg."""

    def __init__(self, cloud):
        self.cloud = cloud

    def __getattr__(self, name):
        return getattr(self.cloud, name)

    def addBatchesAsync(self, low, med, high, colors, levels, batches, borrow=False):
        return self.cloud.addBatches(low, med, high, colors, levels, batches, commit=False)

    def pollUploads(self, commit=True):
        return 0, 0


def run_streaming(args, cr, ctx, dist):
    """Streaming residency: a camera flight at 300 m over a --stream-points
    terrain whose chunks (8 batches of 10,240 points, Morton-contiguous) stream
    from host memory into a pool of 40 % of the batches; the in-memory source
    wants the nearest chunks within a budget of 50 % of the cloud (the pool is
    over-subscribed).  The chunks sit in page-locked host memory.  Per frame:
    StreamingAdapter.update (up to 8 chunk uploads), render, wait for the
    frame.  Timed twice on the same path, with asynchronous uploads that
    borrow the chunks' arrays (addBatchesAsync) and with synchronous ones
    (the reference's addBatches); the
    adapter's invariant (source's resident chunks = resident + queued) is
    checked every frame."""
    streaming = importlib.import_module("satin-computerasteriser_b200.streaming")
    params = cr.TerrainParams(seed=args.seed ^ 0x57)
    sargs = argparse.Namespace(**vars(args))
    sargs.points = args.stream_points
    src_cloud, _ = build_cloud(cr, ctx, sargs, params)
    packed = argparse.Namespace(batches=src_cloud.batches(), **src_cloud.points())
    src_cloud.close()
    ctx.trim()
    chunks = streaming.chunks_from_packed(packed, 8)
    del packed
    nb = sum(len(c.batches) for c in chunks)
    total_bytes = sum(c.totalPointCount for c in chunks) * streaming.BYTES_PER_POINT
    W, H = 1280, 720
    e = params.extent
    path = []
    for k in range(args.stream_frames):
        t = k / max(args.stream_frames - 1, 1)
        x, y = e * (0.1 + 0.8 * t), e * (0.3 + 0.4 * t)
        z = cr.terrain_height(params, x, y) + 300.0
        cam = cr.PerspectiveCamera(position=(x, y, z), near=1.0, far=10000.0, fov=60.0,
                                   aspect=W / H)
        cam.lookAt((x + 600.0, y + 300.0, z - 400.0), up=(0.0, 0.0, 1.0))
        path.append(cam)

    # Chunks in page-locked host memory: the asynchronous uploads read them
    # directly; the synchronous arm copies the same arrays.
    arena = streaming.pin_chunks(chunks)

    def fly(sync: bool):
        cloud = cr.ComputeRasteriserPointCloud(
            ctx, cr.ComputeRasteriserCapacity(int(0.4 * nb), 10240))
        src = streaming.InMemoryStreamingSource(chunks, budget_bytes=int(0.5 * total_bytes))
        ad = streaming.StreamingAdapter(src, _SyncUploads(cloud) if sync else cloud)
        ad.maxChunkUploadsPerTick = 8
        ras = cr.ComputeRasteriser(ctx)
        ras.addPointCloud(cloud)
        ras.resize((W, H))
        ok, full, uploads, t_ad, per_frame = True, False, 0, 0.0, []
        ctx.synchronize()
        dist.barrier()
        t0 = time.perf_counter()
        for cam in path:
            tf = time.perf_counter()
            had = set(ad.slotsByChunk)
            ta = time.perf_counter()
            ad.update(cam, (W, H))
            t_ad += time.perf_counter() - ta
            uploads += len(set(ad.slotsByChunk) - had)
            ras.update(cam)
            ras.encode()
            ctx.synchronize()
            ok &= len(src.believed) - ad.residentChunks - ad.pendingUploadCount == 0
            ok &= ad.residentPoints == cloud.pointCount
            full |= ad.lastError is not None
            per_frame.append(time.perf_counter() - tf)
        s = time.perf_counter() - t0
        cloud.waitUploads()
        res = {"ms_per_frame": round(dist.max(s) * 1e3 / len(path), 4),
               "p95_frame_ms": round(float(np.percentile(per_frame, 95)) * 1e3, 4),
               "max_frame_ms": round(max(per_frame) * 1e3, 4),
               "adapter_update_ms_per_frame": round(t_ad * 1e3 / len(path), 4),
               "chunks_uploaded": uploads,
               "resident_chunks_end": ad.residentChunks, "invariants_hold": bool(ok),
               "pool_pressure": bool(full)}
        ras.removePointCloud(cloud)
        cloud.close()
        return res

    fly(False)  # warm-up (streams)
    a = fly(False)
    b = fly(True)
    arena.close()
    return {"points": args.stream_points, "chunks": len(chunks), "batches_per_chunk": 8,
            "pool_slots": int(0.4 * nb), "frames": len(path), "size": f"{W}x{H}",
            "max_chunk_uploads_per_tick": 8, "async": a, "sync": b,
            "speedup": round(b["ms_per_frame"] / max(a["ms_per_frame"], 1e-9), 3),
            "timing": "wall clock per frame: adapter update + render + wait for the frame"}


def decoded_positions(cloud, first=0, n=None):
    """Full-precision (level 0, 30-bit) positions of pool points [first, first+n):
    a freshly packed pool holds batch k's points from slot k * pointsPerBatch."""
    pts = cloud.points(first, n)
    ppb = cloud.capacity.pointsPerBatch
    b = cloud.batches()
    idx = np.arange(first, first + len(pts["xyzLow"]), dtype=np.int64)
    slot = idx // ppb
    lo, me, hi = (pts[k].astype(np.uint64) for k in ("xyzLow", "xyzMed", "xyzHigh"))
    out = np.zeros((len(idx), 3), np.float64)
    for a, (mn, mx) in enumerate((("minX", "maxX"), ("minY", "maxY"), ("minZ", "maxZ"))):
        s = 10 * a
        q = (((lo >> s) & 1023) << 20) | (((me >> s) & 1023) << 10) | ((hi >> s) & 1023)
        size = np.maximum(b[mx][slot].astype(np.float64) - b[mn][slot], 1e-6)
        out[:, a] = q.astype(np.float64) * size / 1073741824.0 + b[mn][slot]
    return out


def run_differentiable(args, cr, ctx, torch, dist):
    """Differentiable HQS colour fitting: a heightfield of --diff-points points
    (seed 0xC0FFEE05) with learnable FP32 colours initialised to 0.5, --diff-views
    views at 512 x 512 (seeded poses), targets rendered from the hidden field
    c(x) = 0.5 + 0.5 sin(k . x / 400 m + phi).  A step is, for every view, the FP32
    forward, the L2 loss gradient and the adjoint (gradients accumulate over the
    views); timed with CUDA events.  The gradient of --diff-check seeded points
    visible in some view is compared with the FP64 oracle's adjoint and central
    differences (step 1e-3)."""
    seed = 0xC0FFEE05
    params = cr.TerrainParams(seed=seed)
    cloud, _ = build_cloud(cr, ctx, argparse.Namespace(points=args.diff_points), params)
    n = cloud.capacity.maxResidentPoints
    W = H = 512
    cams = lib_poses(cr, params, args.diff_views, seed ^ dist.rank, 1.0)
    xyz = decoded_positions(cloud)
    k = np.array([[3.1, -2.3, 1.7], [-1.9, 2.7, 2.2], [2.4, 1.3, -3.0]]) / 400.0
    phi = np.array([0.3, 1.1, -0.7])
    hidden = (0.5 + 0.5 * np.sin(xyz @ k.T + phi)).astype(np.float32)
    del xyz
    learn = np.full((n, 3), 0.5, np.float32)
    ras = cr.ComputeRasteriser(ctx)
    ras.addPointCloud(cloud)
    ras.resize((W, H))
    d_col = cr.DeviceBuffer(ctx, n * 12, (n, 3), np.float32)
    d_grad = cr.DeviceBuffer(ctx, n * 12, (n, 3), np.float32)
    d_img = cr.DeviceBuffer(ctx, H * W * 12, (H, W, 3), np.float32)
    d_dl = cr.DeviceBuffer(ctx, H * W * 12, (H, W, 3), np.float32)
    tgts = [cr.DeviceBuffer(ctx, H * W * 12, (H, W, 3), np.float32) for _ in cams]
    d_col.upload(hidden)
    for cam, t in zip(cams, tgts):
        ras.update(cam)
        ras.forwardF32(cloud, d_col, t)
    d_col.upload(learn)
    scale = 1.0 / (3.0 * W * H * len(cams))

    def step():
        for cam, t in zip(cams, tgts):
            ras.update(cam)
            ras.forwardF32(cloud, d_col, d_img)
            cr.l2_loss(ctx, d_img, t, scale, d_dl, want_loss=False)
            ras.backwardColors(cloud, d_dl, d_grad)

    stream = torch.cuda.ExternalStream(ctx.stream(), device=f"cuda:{dist.local}")
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for _ in range(2):
        step()
    reps = 3
    ctx.synchronize()
    ev0.record(stream)
    for _ in range(reps):
        step()
    ev1.record(stream)
    ev1.synchronize()
    step_ms = ev0.elapsed_time(ev1) / reps
    out = {"points": args.diff_points, "views": len(cams), "size": f"{W}x{H}",
           "step_ms": round(step_ms, 3),
           "views_per_s": round(len(cams) / (step_ms / 1e3), 1),
           "gpts_per_s": round(args.diff_points * len(cams) / (step_ms / 1e3) / 1e9, 2),
           "step": "per view: FP32 forward + L2 loss gradient + adjoint (accumulated)"}
    if args.diff_check > 0 and dist.rank == 0:
        out["gradient_check"] = diff_gradient_check(args, cr, ctx, ras, cloud, cams, tgts, d_col,
                                                    d_grad, learn, scale)
    for b in [d_col, d_grad, d_img, d_dl] + tgts:
        b.close()
    cloud.close()
    return out


def diff_gradient_check(args, cr, ctx, ras, cloud, cams, tgts, d_col, d_grad, learn, scale):
    import oracle as orc
    orc.build()
    n = len(learn)
    d_col.upload(learn)
    d_grad.upload(np.zeros((n, 3), np.float32))
    d_img = cr.DeviceBuffer(ctx, tgts[0].nbytes, tgts[0].shape, np.float32)
    d_dl = cr.DeviceBuffer(ctx, tgts[0].nbytes, tgts[0].shape, np.float32)
    for cam, t in zip(cams, tgts):
        ras.update(cam)
        ras.forwardF32(cloud, d_col, d_img)
        cr.l2_loss(ctx, d_img, t, scale, d_dl, want_loss=False)
        ras.backwardColors(cloud, d_dl, d_grad)
    g = d_grad.download().astype(np.float64)
    cand = np.flatnonzero(np.abs(g).max(axis=1) > 0)
    pts = np.sort(np.random.default_rng(0x5EED).choice(cand, min(args.diff_check, len(cand)),
                                                        replace=False))
    ocl = oracle_cloud(orc, cloud)
    ocfg = oracle_config(orc, ras.configuration)
    threads = os.cpu_count() or 1
    grad64 = np.zeros((n, 3))
    fd = np.zeros((len(pts), 3))
    t0 = time.perf_counter()
    W, H = ras.viewportSize
    for cam, t in zip(cams, tgts):
        ras.update(cam)
        ocl.files = cloud.files()
        orc.hqs_grad_f64(ocl, ocfg, cam.viewMatrix, cam.projectionMatrix, W, H,
                         learn.astype(np.float64), t.download().astype(np.float64), scale,
                         grad=grad64, fd_points=pts.astype(np.uint32), fd_h=1e-3, fd=fd,
                         threads=threads)
    floor = 1e-2 * np.abs(grad64[pts]).max()

    def rel(a, b):
        return float((np.abs(a - b).max(axis=1) / np.maximum(np.abs(b).max(axis=1), floor)).max())

    d_img.close()
    d_dl.close()
    return {"points": int(len(pts)), "fd_step": 1e-3,
            "max_rel_err_vs_fp64_fd": rel(g[pts], fd),
            "max_rel_err_vs_fp64_adjoint": rel(g[pts], grad64[pts]),
            "fd_vs_adjoint_fp64": rel(fd, grad64[pts]),
            "rel_err": "max over points of max_c |g - ref| / max(max_c |ref|, 1e-2 max |ref|)",
            "oracle_threads": threads, "oracle_s": round(time.perf_counter() - t0, 1)}


def run_packer(args, cr, ctx, torch, dist):
    """The 63-bit packer at --pack-points points (seed 0xC0FFEE03): GPU-synthesised
    16-byte records packed with 21 bits per axis (64-bit keys, 32-bit index) into
    10,240-point batches, timed with CUDA events (mean of 3 packs after one).  The
    result is checked by size-independent invariants: point count, colour
    checksum, per-batch level counts against the cumulative LOD words, and every
    decoded point of 64 seeded batches inside its batch AABB.  (Bit-exact parity
    with the CPU pack at smaller sizes is a GPU test.)"""
    n = args.pack_points
    ppb = 10240
    params = cr.TerrainParams(seed=0xC0FFEE03)
    recs = cr.synth_terrain(ctx, params, n)
    cloud = cr.ComputeRasteriserPointCloud(ctx, cr.ComputeRasteriserCapacity((n + ppb - 1) // ppb,
                                                                             ppb))
    packer = cr.GPUPacker(ctx, mortonBits=21)
    stream = torch.cuda.ExternalStream(ctx.stream(), device=f"cuda:{dist.local}")
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    packer.pack(records=recs, into=cloud)
    ctx.synchronize()
    reps = 3
    ev0.record(stream)
    for _ in range(reps):
        packer.pack(records=recs, into=cloud)
    ev1.record(stream)
    ev1.synchronize()
    ms = ev0.elapsed_time(ev1) / reps
    # Colour checksums (sum and sum of squares, modulo 2^64) of the input on
    # the device, and of the packed pool read back in 10M-point chunks.
    mask = (1 << 64) - 1
    rc = torch.as_tensor(recs, device=f"cuda:{dist.local}")[:, 3].contiguous()
    rc = rc.view(torch.int32).to(torch.int64) & 0xFFFFFFFF
    in_sum, in_sq = int(rc.sum().item()) & mask, int((rc * rc).sum().item()) & mask
    del rc
    recs.close()
    ctx.trim()
    b = cloud.batches()
    res = b[b["state"] != 0]
    checks = {"points": int(res["numPoints"].astype(np.int64).sum()) == n}
    cap = cloud.capacity.maxResidentPoints
    out_sum = out_sq = 0
    for first in range(0, cap, 10_000_000):
        m = min(10_000_000, cap - first)
        col = cloud.points(first, m)["colors"].astype(np.uint64)
        idx = np.arange(first, first + m, dtype=np.int64)
        slot = idx // ppb
        valid = (b["state"][slot] != 0) & (idx - b["firstPoint"][slot] < b["numPoints"][slot])
        c = col[valid]
        out_sum = (out_sum + int(c.sum())) & mask
        out_sq = (out_sq + int((c * c).sum())) & mask
    checks["colour_checksum"] = bool(in_sum == out_sum and in_sq == out_sq)
    rng = np.random.default_rng(3)
    lod_ok = aabb_ok = True
    for i in rng.choice(len(res), min(64, len(res)), replace=False):
        f, c = int(res["firstPoint"][i]), int(res["numPoints"][i])
        lv = cloud.points(f, c)["levels"] & 7
        cum = []
        for w in ("lodCum01", "lodCum23", "lodCum45", "lodCum67"):
            cum += [int(res[w][i]) & 0xFFFF, int(res[w][i]) >> 16]
        lod_ok &= all(cum[L] == int((lv <= L).sum()) for L in range(8))
        p = decoded_positions(cloud, f, c)
        for a, (mn, mx) in enumerate((("minX", "maxX"), ("minY", "maxY"), ("minZ", "maxZ"))):
            aabb_ok &= bool((p[:, a] >= res[mn][i] - 1e-3).all() and
                            (p[:, a] <= res[mx][i] + 1e-3).all())
    checks["lod_cumulative_counts"] = bool(lod_ok)
    checks["points_inside_batch_aabb"] = bool(aabb_ok)
    cloud.close()
    ctx.trim()
    bit_exact = pack_parity(args, cr, ctx) if args.pack_check_points > 0 else None
    # Algorithmic bytes per point (63-bit keys, 4 LOD levels): 8 radix passes
    # moving a 64-bit key and a 32-bit index in and out (192 B), the gather
    # (16 B in, 12 B of sorted position out), 3 LOD levels (12 B each), the
    # quantisation (12 B in, 12 B out) and the colour (4 B): 284 B.
    bpp = 8 * 2 * (8 + 4) + (16 + 12) + 3 * 12 + (12 + 12) + 4
    peak, peak_kind = measured_peaks()
    achieved = n * bpp / (ms / 1e3) / 1e9
    return {"points": n, "morton_bits": 63, "batches": int(len(res)),
            "pack_ms": round(ms, 2), "gpts_per_s": round(n / (ms / 1e3) / 1e9, 3),
            "roofline": {"bound": "hbm", "bytes_per_point": bpp,
                         "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 4), "peak_source": peak_kind},
            "checks": checks, "bit_exact": bit_exact,
            "timing": "CUDA events, mean of 3 packs after one warm-up pack"}


def pack_parity(args, cr, ctx):
    """The 63-bit GPU pack of --pack-check-points heightfield points (the
    packer configuration's generator, seed 0xC0FFEE03) against the oracle's
    pack of the same records on every host thread (bit-identical to its
    single-threaded pack): sorted order (source indices), per-batch records
    (AABB, counts, cumulative LOD counts), split-precision words, levels and
    colours, compared bit for bit.  The oracle's host generator must also
    reproduce the device's records."""
    import oracle as orc
    orc.build()
    threads = len(os.sched_getaffinity(0)) or 1
    n, ppb = args.pack_check_points, 10240
    seed = 0xC0FFEE03
    recs = cr.synth_terrain(ctx, cr.TerrainParams(seed=seed), n)
    dev_recs = recs.download()
    cloud = cr.ComputeRasteriserPointCloud(ctx, cr.ComputeRasteriserCapacity((n + ppb - 1) // ppb,
                                                                             ppb))
    src = cr.GPUPacker(ctx, mortonBits=21).pack(records=recs, into=cloud, sourceIndices=True)
    recs.close()
    t0 = time.perf_counter()
    host_recs = orc.synth_terrain(orc.Terrain(seed=seed), n, threads=threads)
    same = {"records": host_recs.tobytes() == dev_recs.tobytes()}
    del host_recs
    ref = orc.pack(dev_recs[:, :3], colors_rgba8=dev_recs[:, 3].view(np.uint32),
                   pointsPerBatch=ppb, morton_bits=21, threads=threads)
    del dev_recs
    cpu_s = time.perf_counter() - t0
    same["source_order"] = bool(np.array_equal(src, ref.sourceIndices))
    same["batches"] = cloud.batches().tobytes() == ref.batches.tobytes()
    for k in ("xyzLow", "xyzMed", "xyzHigh", "colors", "levels"):
        same[k] = True
    for first in range(0, n, 20_000_000):
        m = min(20_000_000, n - first)
        pts = cloud.points(first, m)
        for k in ("xyzLow", "xyzMed", "xyzHigh", "colors", "levels"):
            same[k] &= bool(np.array_equal(pts[k], getattr(ref, k)[first:first + m]))
    cloud.close()
    ctx.trim()
    return {"points": n, "morton_bits": 63, "bit_exact": all(same.values()),
            "outputs": {k: bool(v) for k, v in same.items()},
            "oracle": f"orc_pack_threads on {threads} host threads", "oracle_s": round(cpu_s, 1)}


MV_SIZES = ((256, 256), (512, 512), (1280, 720), (1920, 1080))


def run_multiview(args, cr, ctx, torch, dist):
    """Batched views against per-view renders: a heightfield of
    --mv-points points (seed 0xC0FFEE04), --mv-views cameras at seeded poses
    with sizes drawn uniformly from 256^2, 512^2, 1280x720 and 1920x1080.
    Per-view: one ComputeRasteriser update + encode per view.  Batched: one
    MultiViewRasteriser.render of all views (one CUDA-graph launch), launch
    shape from the autotuner.  Both timed with CUDA events on the library
    stream over --mv-reps repetitions; every view's RGBA8, depth and R, G, B,
    count planes are compared bit for bit."""
    seed = 0xC0FFEE04
    params = cr.TerrainParams(seed=seed)
    mv_args = argparse.Namespace(points=args.mv_points)
    cloud, _ = build_cloud(cr, ctx, mv_args, params)
    rng = np.random.default_rng(seed ^ dist.rank)
    sizes = [MV_SIZES[i] for i in rng.integers(0, len(MV_SIZES), args.mv_views)]
    cams = lib_poses(cr, params, args.mv_views, seed ^ dist.rank, 1.0)
    for cam, (w, h) in zip(cams, sizes):
        cam.aspect = w / h
    saved = ctx.tuning()
    stream = torch.cuda.ExternalStream(ctx.stream(), device=f"cuda:{dist.local}")
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    ras = cr.ComputeRasteriser(ctx)
    ras.addPointCloud(cloud)

    def per_view():
        for cam, size in zip(cams, sizes):
            ras.resize(size)
            ras.update(cam)
            ras.encode()

    for _ in range(2):
        per_view()
    ctx.synchronize()
    ev0.record(stream)
    for _ in range(args.mv_reps):
        per_view()
    ev1.record(stream)
    ev1.synchronize()
    per_view_ms = ev0.elapsed_time(ev1) / args.mv_reps
    # Pass times of the per-view renders (a separate run with a CUDA event
    # around every pass): the depth and colour work is the same in both
    # forms, so (all passes) / (depth + colour) bounds what batching can gain.
    ctx.set_profiling(True)
    per_view()
    ctx.synchronize()
    pt = ctx.pass_times(len(cams))
    ctx.set_profiling(False)
    names = list(PASS_NAMES)
    work = float(pt[:, names.index("depth")].sum() + pt[:, names.index("color")].sum())
    by_size = {}
    for w, h in MV_SIZES:
        idx = [i for i, sz in enumerate(sizes) if sz == (w, h)]
        if idx:
            by_size[f"{w}x{h}"] = {n: round(float(pt[idx, k].mean()), 4)
                                   for k, n in enumerate(names) if pt[idx, k].any()}

    mv = cr.MultiViewRasteriser(ctx, sizes)
    mv.addPointCloud(cloud)
    tuned = mv.autotune(cams, reps=3)
    for _ in range(2):
        mv.render(cams)
    ctx.synchronize()
    ev0.record(stream)
    for _ in range(args.mv_reps):
        mv.render(cams)
    ev1.record(stream)
    ev1.synchronize()
    batched_ms = ev0.elapsed_time(ev1) / args.mv_reps

    exact = True
    for i, (cam, size) in enumerate(zip(cams, sizes)):
        ras.resize(size)
        ras.update(cam)
        ras.encode()
        a, b = ras.pixels(), mv.pixels(i)
        exact &= all(np.array_equal(a[f], b[f]) for f in ("depth", "red", "green", "blue",
                                                          "count"))
        exact &= bool(np.array_equal(ras.outputRGBA8(), mv.outputRGBA8(i)))
        exact &= bool(np.array_equal(ras.depthTexture().view(np.uint32),
                                     mv.depthTexture(i).view(np.uint32)))
    ctx.set_tuning(chunkPoints=saved["chunkPoints"], useTiles=saved["useTiles"],
                   viewGroupPixels=saved["viewGroupPixels"])
    mv.close()
    cloud.close()
    n = args.mv_views
    return {"views": n, "points": args.mv_points,
            "sizes": {f"{w}x{h}": sizes.count((w, h)) for w, h in MV_SIZES},
            "per_view_ms": round(per_view_ms, 4), "batched_ms": round(batched_ms, 4),
            "speedup": round(per_view_ms / batched_ms, 3),
            "per_view_pass_ms": by_size,
            "ceiling": {"value": round(float(pt.sum()) / max(work, 1e-9), 3),
                        "why": "per-view pass time over its depth + colour time: the "
                               "per-(point, view) work that batching cannot share"},
            "batched_gpts_per_s": round(n * args.mv_points / (batched_ms / 1e3) / 1e9, 2),
            "bit_exact": bool(exact), "tuning": tuned,
            "timing": "CUDA events on the library stream, mean of --mv-reps repetitions "
                      "after 2 warm-ups; per-view includes each view's host calls"}


def cpu_baseline(args, cr, ctx, ras, cloud, cams):
    """The single-threaded oracle timed on whole frames of the same cloud (a
    bounded sample of about --cpu-seconds)."""
    import oracle as orc
    orc.build()
    cfg = oracle_config(orc, ras.configuration)
    W, H = args.width, args.height
    frames, cpu_s = 0, 0.0
    p = 0
    ocl = oracle_cloud(orc, cloud)  # the device pool, read back once
    while True:
        ras.update(cams[p])
        ocl.files = cloud.files()
        t0 = time.perf_counter()
        orc.render(ocl, cfg, cams[p].viewMatrix, cams[p].projectionMatrix, W, H, threads=1)
        cpu_s += time.perf_counter() - t0
        frames += 1
        p = (p + 1) % args.poses
        if cpu_s >= args.cpu_seconds or frames >= 8:
            break
    value = args.points * frames / cpu_s / 1e9
    return {"value": round(value, 6), "unit": "Gpts/s", "cores": 1, "kind": "port",
            "sample": f"{frames} whole frame(s) of the {args.points:,}-point "
                      f"{W}x{H} workload (poses 0..{frames - 1}), single-threaded C++ oracle",
            "seconds": round(cpu_s, 2)}


def parity_poses(args, cr, ras, cloud, cams, poses, mode):
    """Every pose in `poses` rendered again through the library in `mode` and
    compared bit for bit with the oracle on every host thread: HQS the depth
    plane, the R, G, B, count planes, the survivor list, RGBA8 and the float
    depth; nearest the nearest depth and index planes and RGBA8."""
    import oracle as orc
    orc.build()
    threads = len(os.sched_getaffinity(0)) or 1
    saved = ras.configuration
    ras.configuration = cr.ComputeRasteriserConfiguration(mode=mode)
    ocfg = oracle_config(orc, ras.configuration)
    ocl = oracle_cloud(orc, cloud)
    W, H = args.width, args.height
    matched, failed = [], {}
    t0 = time.perf_counter()
    try:
        for p in sorted(set(poses)):
            ras.update(cams[p])
            ras.encode()
            ocl.files = cloud.files()
            ref = orc.render(ocl, ocfg, cams[p].viewMatrix, cams[p].projectionMatrix, W, H,
                             threads=threads)
            same = {"rgba8": np.array_equal(ras.outputRGBA8(), ref.rgba)}
            if mode == cr.MODE_HQS:
                px = ras.pixels()
                acc = np.stack([px["red"], px["green"], px["blue"], px["count"]], -1)
                same["depth"] = np.array_equal(px["depth"], ref.depth)
                same["accum"] = np.array_equal(acc, ref.accum)
                same["visible"] = np.array_equal(cloud.visibleBatches(), ref.visible[0])
                same["depth_f32"] = np.array_equal(ras.depthTexture().view(np.uint32),
                                                   ref.depthf.view(np.uint32))
            else:
                same["nearest_depth"] = np.array_equal(ras.nearestDepths(), ref.nearest_depth)
                same["nearest_index"] = np.array_equal(ras.nearestIndices(), ref.nearest_index)
            if all(same.values()):
                matched.append(int(p))
            else:
                failed[int(p)] = sorted(k for k, v in same.items() if not v)
    finally:
        ras.configuration = saved
    return {"poses_checked": len(set(poses)), "poses_bit_exact": len(matched),
            "bit_exact": not failed, "poses": sorted(int(p) for p in set(poses)),
            "failed": failed,
            "planes": ["depth", "accum", "visible", "rgba8", "depth_f32"] if mode == cr.MODE_HQS
            else ["nearest_depth", "nearest_index", "rgba8"],
            "oracle_threads": threads, "seconds": round(time.perf_counter() - t0, 1)}


def run_nearest(args, cr, ctx, ras, cloud, cams, timed, stream):
    """The nearest-point mode on the same cloud and frames: the timed HQS
    frames' poses drawn again with .nearestPoint (device time, CUDA events
    around the whole run)."""
    import torch
    hqs = ras.configuration
    ras.configuration = cr.ComputeRasteriserConfiguration(mode=cr.MODE_NEAREST)
    try:
        for p in timed[:3]:
            ras.update(cams[p])
            ras.encode()
        ctx.synchronize()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ev0.record(stream)
        for p in timed:
            ras.update(cams[p])
            ras.encode()
        ev1.record(stream)
        ev1.synchronize()
        ms = ev0.elapsed_time(ev1) / len(timed)
        return {"value": round(args.points / (ms / 1e3) / 1e9, 4), "unit": "Gpts/s",
                "ms_per_step": round(ms, 4), "frames": len(timed),
                "timing": "CUDA events around the run; the HQS run's poses"}
    finally:
        ras.configuration = hqs


# ---------------------------------------------------------------------------
# Reference arm: the CPU oracle with every host thread
# ---------------------------------------------------------------------------
def run_reference(args, dist):
    """The reference arm: the CPU oracle (the reference's pass semantics restated
    in C++) renders the same workload with every host thread.  It builds its
    inputs on the CPU without the library: the oracle's host restatement of the
    seeded heightfield generator (bit-identical records), the oracle's pack on
    every host thread (bit-identical to the single-threaded pack, which the
    library's GPU pack also equals), and the same camera poses."""
    if dist.rank != 0:
        return None
    import oracle as orc
    orc.build()
    threads = len(os.sched_getaffinity(0)) or 1
    terrain = orc.Terrain(seed=args.seed)
    t0 = time.perf_counter()
    recs = orc.synth_terrain(terrain, args.points, threads=threads)
    packed = orc.pack(recs[:, :3], colors_rgba8=recs[:, 3].view(np.uint32), pointsPerBatch=10240,
                      threads=threads)
    del recs
    build_s = time.perf_counter() - t0
    W, H = args.width, args.height
    cams = make_poses(lambda x, y: orc.terrain_height(terrain, x, y), terrain.extent, args.poses,
                      args.seed, W / H)
    base = packed.cloud()
    cfg = orc.Config(mode=0 if args.mode == "hqs" else 1)
    eye = np.eye(4, dtype=np.float32)
    vp_files = [orc.update_files(base.files, orc.mat4_mul(c.projectionMatrix, c.viewMatrix), eye)
                for c in cams]

    def frame(p, cl):
        cl.files = vp_files[p]
        t0 = time.perf_counter()
        orc.render(cl, cfg, cams[p].viewMatrix, cams[p].projectionMatrix, W, H, threads=threads)
        return time.perf_counter() - t0

    # Size the per-step sample (every m-th batch slot resident) so the whole
    # run stays within a few minutes.
    t_full = frame(0, base)
    budget = 150.0 / max(args.steps + args.warmup, 1)
    m = max(1, int(math.ceil(t_full / budget)))
    sample = orc.Cloud(**{k: getattr(base, k) for k in
                          ("batches", "files", "xyzLow", "xyzMed", "xyzHigh", "colors",
                           "levels")})
    if m > 1:
        b = base.batches.copy()
        keep = np.zeros(len(b), bool)
        keep[::m] = True
        b["state"][~keep] = 0
        sample.batches = b
    pts = int(sample.batches["numPoints"][sample.batches["state"] != 0].sum())
    for k in range(args.warmup):
        frame(k % args.poses, sample)
    total = 0.0
    for k in range(args.steps):
        total += frame((args.warmup + k) % args.poses, sample)
    value = pts * args.steps / total / 1e9
    samp = (f"whole {W}x{H} frames over every {m}-th batch slot ({pts:,} of "
            f"{args.points:,} points), {threads} host threads")
    return {"metric": METRIC, "value": round(value, 6), "unit": "Gpts/s", "impl": "reference",
            "n_gpus": dist.world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(total * 1e3 / args.steps, 3), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+u32",
            "data": "synthetic (seeded fractal heightfield, generated and packed on the host "
                    "by the oracle)",
            "config": config_dict(args),
            "cpu_baseline": {"value": round(value, 6), "unit": "Gpts/s", "cores": threads,
                             "kind": "port", "sample": samp},
            "e2e": {"value": round(value, 6), "unit": "Gpts/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "inputs_build_s": round(build_s, 1)}


def main():
    args = parse_args()
    dist = Dist(group_of_one=args.shard == "points" and args.impl == "ours")
    try:
        out = run_reference(args, dist) if args.impl == "reference" else run_ours(args, dist)
        if out is not None and dist.rank == 0:
            print(json.dumps(out), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
