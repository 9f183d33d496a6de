"""Benchmark: the plain CUDA frame (primary -> godray -> composite) on B200.

Workload (N = 1): the full plain pipeline at 1920x1080 present / 960x540
internal over a streamed world of 16x4x16 chunks with 3D caves, a 5-level
256^2 toroidal clipmap and a seeded 64-frame Catmull-Rom camera path with a
+1 chunk grid shift every 16 frames.  One step = one frame.

* ``value``  Mrays/s (primary rays = internal pixels) with every input
  resident in HBM: all chunks the path needs are uploaded before timing and a
  grid shift is a 4 KiB grid rewrite; per-step device time from CUDA events on
  the compute stream, L2 flushed (512 MiB memset) between steps.
* ``e2e``    the same frames through the C ABI with host buffers: camera,
  clipmap patches, streamed chunk uploads at grid shifts (host -> device) and
  the RGBA32F present image read back (device -> host) inside the timed region.
* ``--gpus N``: replicas only -- each rank renders the same workload on its own
  GPU, no data-path collective; value = all ranks' rays / max-over-ranks time.
* ``--impl reference``: the reference cannot run here (Rust + WGSL, no
  graphics stack), so the reference arm is the C++ scalar restatement of its
  WGSL (oracle/) on all host cores, one full frame per step.
"""
from __future__ import annotations

import argparse
import ctypes as C
import contextlib
import gc
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO / "voxel-engine-v0_b200"))
sys.path.insert(0, str(REPO))

METRIC = "Mrays/s + 1080p frame ms on 1×B200, served p50/p99 latency, vs plain CUDA pass"
UNIT = "Mrays/s"
WORKLOAD = ("config2 plain pipeline: 16x4x16 chunks (caves > 0.6), 5-level 256^2 clipmap, 1920x1080 present / "
            "960x540 internal, primary+godray+composite per frame, 64-frame Catmull-Rom path, grid shift every 16 frames")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=48)
    ap.add_argument("--warmup", type=int, default=4)
    ap.add_argument("--impl", default="vxe", choices=["vxe", "reference"])
    ap.add_argument("--present", default="1920x1080")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batch", action="store_true", help="skip the batched / served workloads")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--profile-steps", type=int, default=0, help="render N steps only (for ncu), no JSON")
    ap.add_argument("--build-profile", type=int, default=0,
                    help="build the first N config-2 chunks (a counting build, then the full build) only, for ncu")
    return ap.parse_args()


@contextlib.contextmanager
def no_gc():
    """Timed regions run without the cyclic garbage collector: a collection
    over the host's world objects would pause the host loop that feeds the
    GPU.  Collected before, re-enabled after."""
    gc.collect()
    gc.disable()
    try:
        yield
    finally:
        gc.enable()


class ClockSampler:
    """Samples the SM clock and the clock-event (throttle) reasons while the
    timed region runs: NVML every 10 ms (read-only queries), nvidia-smi
    every 200 ms where NVML is unavailable."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")
    REASONS = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.samples = []  # (sm MHz, max sm MHz, set of active reason names)
        self._stop = threading.Event()
        self._t = None
        self._nvml = None

    def _nvml_handle(self):
        try:
            import pynvml
            import torch

            # this CUDA device's NVML handle by its PCI address, as the bytes
            # "dddddddd:bb:dd.0" (the binding passes an integer through as a
            # pointer, so only a bytes string goes in)
            pr = torch.cuda.get_device_properties(self.index)
            ids = (getattr(pr, "pci_domain_id", None), getattr(pr, "pci_bus_id", None),
                   getattr(pr, "pci_device_id", None))
            if not all(isinstance(v, int) for v in ids):
                return None
            bus = f"{ids[0]:08X}:{ids[1]:02X}:{ids[2]:02X}.0".encode()
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            bits = {"hw_slowdown": pynvml.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": pynvml.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": pynvml.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": pynvml.nvmlClocksEventReasonSwPowerCap}
            return pynvml, h, bits
        except Exception:
            return None

    def _run(self):
        nv = self._nvml_handle()
        while not self._stop.is_set():
            try:
                if nv is not None:
                    pynvml, h, bits = nv
                    sm = float(pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM))
                    mx = float(pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM))
                    r = pynvml.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.samples.append((sm, mx, {n for n, b in bits.items() if r & b}))
                else:
                    out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits"], capture_output=True, text=True,
                                         timeout=5)
                    if out.returncode == 0 and out.stdout.strip():
                        f = [v.strip() for v in out.stdout.strip().split(",")]
                        num = lambda v: float(v) if v.replace(".", "").isdigit() else None  # noqa: E731
                        self.samples.append((num(f[1]), num(f[2]), {self.REASONS[i] for i in range(4)
                                                                     if len(f) > 5 + i and f[5 + i].lower() == "active"}))
            except Exception:
                pass
            self._stop.wait(0.01 if nv is not None else 0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [s[0] for s in self.samples if s[0] is not None]
        mx = [s[1] for s in self.samples if s[1] is not None]
        reasons = sorted(set().union(*(s[2] for s in self.samples)))
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


def run_vxe(args, rank: int, world_size: int):
    import torch

    from vxe import _abi as A
    from vxe.renderer import Renderer
    from vxe.world import Clipmap

    dev = rank if torch.cuda.device_count() > rank else 0
    torch.cuda.set_device(dev)
    present = tuple(int(v) for v in args.present.split("x"))
    from vxe.scenes import ResidentPathDriver, config2

    sc = config2(present=present)
    drv = ResidentPathDriver(sc)
    ups = drv.initial_uploads()
    world = drv.world
    r = Renderer(sc.present[0], sc.present[1], sc.render_scale, node_capacity=world.node_capacity,
                 chunk_capacity=world.chunk_capacity, grid_capacity=int(np.prod(sc.grid_dims)),
                 clip_levels=sc.clip_levels, clip_res=sc.clip_res, flags=A.FLAG_GODRAY_MACRO_ALIAS, device=dev)
    r.apply_chunk_uploads(ups)
    rays_per_frame = sc.internal[0] * sc.internal[1]

    def submit(step):
        cam, params, patches, grid = drv.inputs(step)
        if grid is not None:
            r.write_chunk_grid(grid)
        r.write_clipmap_updates(params, patches)
        r.write_camera(cam)
        r.encode_compute(sync=False)

    if args.profile_steps:
        for s in range(args.profile_steps):
            submit(s)
        r.synchronize()
        return None

    flush = torch.empty(512 << 20, dtype=torch.uint8, device=f"cuda:{dev}")
    for s in range(args.warmup):
        submit(s)
    r.synchronize()
    # ---- device-resident timing: per-step kernel time from the context's events
    if world_size > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    step_ms, prim_ms, god_ms, comp_ms, tile_ms, trace_ms, grass_ms, walk_ms = [], [], [], [], [], [], [], []
    with ClockSampler(dev) as clocks, no_gc():
        for s in range(args.steps):
            flush.zero_()
            torch.cuda.synchronize()
            submit(args.warmup + s)
            t = r.read_gpu_timings_ms_blocking()
            step_ms.append(t["total"])
            prim_ms.append(t["primary"])
            god_ms.append(t["godray"])
            comp_ms.append(t["composite"])
            tile_ms.append(t["tiles"])
            trace_ms.append(t["primary_trace"])
            walk_ms.append(t["trace_kernel"])
            grass_ms.append(t["grass_cells"])
    torch.cuda.synchronize()
    if world_size > 1:
        torch.distributed.barrier()
    total_ms = float(sum(step_ms))
    err = r.read_error_word()
    r.close()
    del r, drv, world, ups, flush  # the device-resident workload's host objects
    # ---- end to end through the C ABI with host buffers (streaming world)
    if args.no_e2e:
        e2e = {"seconds": float("nan"), "rays": 0, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
               "serial_seconds": float("nan")}
    else:
        e2e = run_e2e(args, sc, dev, world_size)
    return {
        "total_ms": total_ms, "step_ms": step_ms, "primary_ms": prim_ms, "godray_ms": god_ms,
        "composite_ms": comp_ms, "tiles_ms": tile_ms, "trace_ms": trace_ms, "grass_ms": grass_ms, "walk_ms": walk_ms,
        "rays_per_frame": rays_per_frame,
        "internal": list(sc.internal),
        "clocks": clocks.summary(), "e2e": e2e, "error_word": err, "device": torch.cuda.get_device_name(dev),
    }


# Served runs depend on host timing (which arrivals share a batch) and on the
# shared host's load: each served figure is the median of this many runs.
SERVE_RUNS = 5


def run_batch_serve(dev):
    """Batched and served workloads (mixed viewport / query batches; Poisson request serving) on the config-2 world.

    batch: the config-3 request mix (24 viewports 128^2-1920x1080, 40 query
    batches 1e3-1e6 rays, seeded) as one persistent batch vs one plain launch
    per request (the single-launch pass with the reference's inline grass
    probes), device time from the lane's CUDA events, best of 3.
    serve: 120 Poisson requests at 1000 req/s (70 % viewports 256^2-1920x1080,
    30 % query batches 1k-256k rays), continuous batching over 2 lanes with a
    4 GiB admission budget, vs the plain one-request-at-a-time server; both
    re-upload 10 resident chunks per 16 ms tick; latency = completion -
    arrival (host clock).
    serve.sessions: the same with session frames (resident histories) at a
    saturating (1000 req/s) and a light (200 req/s) load.
    """
    import torch

    from vxe import _abi as A
    from vxe.batch import make_batch
    from vxe.renderer import Renderer
    from vxe.scenes import FrameDriver, config2
    from vxe.serve import make_arrivals, make_sessions, serve, serve_plain

    sc = config2()
    drv = FrameDriver(sc)
    ups = drv.initial_uploads()
    _, _, clip, cam = drv.step()
    w = drv.world
    r = Renderer(sc.present[0], sc.present[1], sc.render_scale, node_capacity=w.node_capacity,
                 chunk_capacity=w.chunk_capacity, grid_capacity=w.grid_capacity, clip_levels=sc.clip_levels,
                 clip_res=sc.clip_res, device=dev)
    try:
        r.upload_world(w, ups)
        r.write_clipmap_updates(*clip)
        r.write_camera(cam)
        b = make_batch(w, torch, seed=3)
        out = {}
        for mode, name in [(A.BATCH_PLAIN, "plain"), (A.BATCH_PERSISTENT, "persistent"), (A.BATCH_GRAPH, "graph")]:
            ms = min(r.submit_batch(b.requests, (8, 4), 1, mode).ms for _ in range(3))
            out[name] = {"ms": round(ms, 3), "mrays_per_s": round(b.rays / ms / 1e3, 3)}
        # the B200 schedule (deferred probes, finishing queues, coherent
        # query order) one request at a time: separates the schedule's gain
        # from the batching's
        ms = min(sum(r.submit_batch([q], (8, 4), 1, A.BATCH_PERSISTENT).ms for q in b.requests) for _ in range(2))
        out["per_request_b200_schedule"] = {"ms": round(ms, 3), "mrays_per_s": round(b.rays / ms / 1e3, 3)}
        batch = {"workload": "config-3 mix: 24 viewports + 40 query batches, seed 3", "rays": int(b.rays),
                 "tile": [8, 4], "rays_per_thread": 1, **out,
                 "plain": {**out["plain"], "mode": "one plain launch per request, the reference's inline probes"},
                 "speedup_vs_plain": round(out["plain"]["ms"] / out["persistent"]["ms"], 3),
                 "speedup_vs_per_request_b200_schedule":
                     round(out["per_request_b200_schedule"]["ms"] / out["persistent"]["ms"], 3)}
        reqs = make_arrivals(w, 2000.0, 20, seed=1)
        serve(r, w, reqs, torch, mem_budget=4 << 30, lanes=2)  # warm-up
        # The served run depends on host timing (which arrivals share a batch):
        # three runs each, the median one by completion time is reported.
        def median_run(fn):
            with no_gc():
                runs = sorted((fn() for _ in range(SERVE_RUNS)), key=lambda x: x.seconds)
            return runs[SERVE_RUNS // 2], [round(x.seconds, 4) for x in runs]

        rep, rep_s = median_run(lambda: serve(r, w, make_arrivals(w, 1000.0, 120, seed=7), torch,
                                              mem_budget=4 << 30, lanes=2, max_batch=32))
        base, base_s = median_run(lambda: serve_plain(r, w, make_arrivals(w, 1000.0, 120, seed=7), torch))
        srv = {"workload": "120 Poisson requests at 1000 req/s, 70 % viewports / 30 % query batches, "
                           "10 chunk re-uploads per 16 ms tick in both servers; median of 5 runs",
               "batched": {**rep.summary(), "runs_seconds": rep_s}, "plain": {**base.summary(), "runs_seconds": base_s},
               "speedup_vs_plain": round(base.seconds / rep.seconds, 3)}
        # Sessions: frames of 16 clients whose TAA / godray / shadow histories
        # stay resident between requests (one view each), with query batches.
        sess = {}
        for rate in (1000.0, 200.0):
            def sess_served():
                ss = make_sessions(w, 16, seed=3)
                return serve(r, w, make_arrivals(w, rate, 240, seed=7, sessions=ss), torch, mem_budget=None,
                             lanes=2, max_batch=16, sessions=ss)

            def sess_plain():
                ss = make_sessions(w, 16, seed=3)
                return serve_plain(r, w, make_arrivals(w, rate, 240, seed=7, sessions=ss), torch, sessions=ss)

            def sess_single_launch():
                ss = make_sessions(w, 16, seed=3)
                return serve_plain(r, w, make_arrivals(w, rate, 240, seed=7, sessions=ss), torch, sessions=ss,
                                   single_launch_pass=True)

            rep, _ = median_run(sess_served)
            base, _ = median_run(sess_plain)
            single = sess_single_launch()
            sess[f"{int(rate)}_per_s"] = {"batched": rep.summary(), "plain": base.summary(),
                                          "plain_single_launch_pass": single.summary(),
                                          "speedup_vs_plain": round(base.seconds / rep.seconds, 3),
                                          "speedup_vs_plain_single_launch_pass": round(single.seconds / rep.seconds, 3)}
        srv["sessions"] = {"workload": "240 Poisson requests, 70 % frames of 16 sessions (256^2-1920x1080 "
                                       "present at render scale 0.5, histories resident) / 30 % query batches; "
                                       "median of 5 runs; plain = one request at a time in the wavefront "
                                       "schedule, plain_single_launch_pass = one request at a time, one kernel "
                                       "per pass (one run); every server re-uploads 10 resident chunks per 16 ms "
                                       "tick",
                           **sess}
        return batch, srv
    finally:
        r.close()


def run_serve_config4(dev, count: int = 120):
    """Config 4: Poisson serving at 200 / 500 / 1000 / 2000 req/s (70 %
    one-off viewports 256^2-1920x1080, 30 % query batches 1k-256k rays) over a
    4096-chunk resident arena (32x4x32 chunks of the config-2 terrain, built on
    the device), 10 chunk re-uploads per 16 ms tick on the upload stream,
    admission by the device's free memory (cudaMemGetInfo) less 4 GiB.
    Batched (continuous batching over 2 lanes) vs the plain one-request-at-a-
    time server (one plain launch per request); median of 5 runs per rate."""
    import torch

    from vxe.renderer import Renderer
    from vxe.scenes import config2
    from vxe.serve import device_memory_budget, make_arrivals, serve, serve_plain
    from vxe.world import World

    sc = config2(present=(64, 36))
    dims = (32, 4, 32)
    w = World(sc.spec, (0, 0, 0), dims, 48 << 20, chunk_capacity=int(np.prod(dims)), mirror=False)
    r = Renderer(64, 36, 1.0, node_capacity=w.node_capacity, chunk_capacity=w.chunk_capacity,
                 grid_capacity=w.grid_capacity, clip_levels=sc.clip_levels, clip_res=sc.clip_res, device=dev)
    out = {}
    try:
        w.populate_device(r)
        w.prebuild(list(w.slot_to_key))  # host copies the re-uploads send
        pos = np.array([102.4, 9.0, 102.4])
        from vxe.world import build_camera

        cam = build_camera(pos, 0.3, -0.1, (64, 36), (64, 36), frame_index=1, time_s=0.0, world=w, jitter=False)
        r.write_camera(cam)
        r.synchronize()
        budget = device_memory_budget(torch, device=dev)
        serve(r, w, make_arrivals(w, 2000.0, 20, seed=1), torch, mem_budget=budget, lanes=2)  # warm-up

        def median_run(fn):
            with no_gc():
                runs = sorted((fn() for _ in range(SERVE_RUNS)), key=lambda x: x.seconds)
            return runs[SERVE_RUNS // 2]

        for rate in (200.0, 500.0, 1000.0, 2000.0):
            rep = median_run(lambda: serve(r, w, make_arrivals(w, rate, count, seed=7), torch, mem_budget=budget,
                                           lanes=2, max_batch=32))
            base = median_run(lambda: serve_plain(r, w, make_arrivals(w, rate, count, seed=7), torch))
            out[f"{int(rate)}_per_s"] = {"batched": rep.summary(), "plain": base.summary(),
                                         "speedup_vs_plain": round(base.seconds / rep.seconds, 3)}
        out["workload"] = (f"{count} Poisson requests per rate, 70 % viewports / 30 % query batches, 4096-chunk "
                           "arena (32x4x32), 10 re-uploads per 16 ms tick in both servers, admission budget = free "
                           "device memory - 4 GiB; median of 5 runs")
        out["admission_budget_bytes"] = int(budget)
    finally:
        r.close()
    return out


def config5_with_queries(dev, frames: int = 128, seed: int = 5):
    """Config 5 as specified: the 128-frame camera path over the 32x8x32-chunk
    world at 3840x2160 present / 1920x1080 internal, with a served ray-query
    batch of 64k-1M incoherent rays (log-uniform) issued on a batch lane
    before each frame so the two overlap on the device.  Wall clock over the
    whole run (every frame and batch complete when it stops)."""
    import math

    import torch

    from vxe import _abi as A
    from vxe import scenes
    from vxe.renderer import Renderer
    from vxe.scenes import FrameDriver

    sc = scenes.config5()
    cells = int(np.prod(sc.grid_dims))
    r = Renderer(sc.present[0], sc.present[1], sc.render_scale, node_capacity=sc.node_capacity,
                 chunk_capacity=cells, grid_capacity=cells, clip_levels=sc.clip_levels,
                 clip_res=sc.clip_res, flags=A.FLAG_GODRAY_MACRO_ALIAS, device=dev)
    rng = np.random.default_rng(seed)
    try:
        drv = FrameDriver(sc, device_renderer=r, mirror=False)  # the world built on the device
        drv.initial_uploads()
        w = drv.world
        lo, hi = w.world_aabb_m()
        # path frame 0 (the clipmap's first full build) untimed
        _, _, clip, cam = drv.step()
        r.write_clipmap_updates(*clip)
        r.write_camera(cam)
        r.encode_compute()
        frames -= 1
        batches = []
        for _ in range(frames):
            n = int(round(math.exp(rng.uniform(math.log(64e3), math.log(1e6)))))
            o = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
            d = rng.normal(size=(n, 3))
            d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
            to, td = torch.from_numpy(o).to(f"cuda:{dev}"), torch.from_numpy(d).to(f"cuda:{dev}")
            res = torch.empty(n * 32, dtype=torch.uint8, device=f"cuda:{dev}")
            q = A.Request()
            q.kind, q.ray_count, q.tmax = A.REQ_QUERY, n, 120.0
            q.d_origins, q.d_dirs, q.d_out = to.data_ptr(), td.data_ptr(), res.data_ptr()
            batches.append((q, (to, td, res)))
        torch.cuda.synchronize(dev)
        frame_ms, q_rays = [], 0
        t0 = time.perf_counter()
        for f in range(frames):
            uploads, grid_changed, clip, cam = drv.step()
            if f > 0:
                r.batch_wait(0, block=True)
            q = batches[f][0]
            r.submit_batch_async(0, [q], (8, 4), 1, A.BATCH_PERSISTENT)
            q_rays += q.ray_count
            r.write_clipmap_updates(*clip)
            r.write_camera(cam)
            r.encode_compute(sync=False)
            frame_ms.append(r.read_gpu_timings_ms_blocking()["total"])
        r.batch_wait(0, block=True)
        r.synchronize()
        dt = time.perf_counter() - t0
        assert r.read_error_word() == 0
    finally:
        r.close()
    frays = frames * sc.internal[0] * sc.internal[1]
    return {"workload": "config5: 32x8x32 chunks (caves > 0.5), 6-level 512^2 clipmap, 3840x2160 present / "
                        "1920x1080 internal, 128-frame path (frames 1..127 timed), one 64k-1M-ray query batch per "
                        "frame on a lane",
            "frames": frames, "frame_ms_mean": round(statistics.mean(frame_ms), 3),
            "frame_ms_p99": round(float(np.percentile(frame_ms, 99)), 3),
            "query_rays": int(q_rays), "frame_rays": int(frays), "seconds": round(dt, 4),
            "mrays_per_s": round((frays + q_rays) / dt / 1e6, 3),
            "note": "wall clock over the run; frame_ms from the context's events (the query batches overlap)"}


def frame_series(sc, dev, steps: int, warmup: int, present=None):
    """Frames of scene `sc` (static grid) timed by the context's events; returns ms per frame (mean) and rays."""
    import torch

    from vxe import _abi as A
    from vxe.renderer import Renderer
    from vxe.scenes import FrameDriver

    drv = FrameDriver(sc)
    ups = drv.initial_uploads()
    w = drv.world
    r = Renderer(sc.present[0], sc.present[1], sc.render_scale, node_capacity=w.node_capacity,
                 chunk_capacity=w.chunk_capacity, grid_capacity=w.grid_capacity, clip_levels=sc.clip_levels,
                 clip_res=sc.clip_res, flags=A.FLAG_GODRAY_MACRO_ALIAS, device=dev)
    flush = torch.empty(512 << 20, dtype=torch.uint8, device=f"cuda:{dev}")
    try:
        r.upload_world(w, ups)
        ms = []
        for f in range(warmup + steps):
            _, _, clip, cam = drv.step()
            r.write_clipmap_updates(*(clip if clip is not None else (drv.empty_clip(), [])))  # config 1: none
            r.write_camera(cam)
            if f >= warmup:
                flush.zero_()
                torch.cuda.synchronize()
                r.encode_compute(sync=False)
                ms.append(r.read_gpu_timings_ms_blocking()["total"])
            else:
                r.encode_compute(sync=False)
        r.synchronize()
        assert r.read_error_word() == 0
        return statistics.mean(ms), sc.internal[0] * sc.internal[1]
    finally:
        r.close()


def run_clipmap(dev):
    """Clipmap patch generation, config 5's 6 x 512^2 clipmap: a full rebuild
    (every level new) and a one-texel scroll, on the host (the reference's
    path: CPU texels, then an upload) vs on the device (texels written in place)."""
    import time

    import torch

    from vxe import scenes
    from vxe.renderer import Renderer
    from vxe.world import Clipmap

    sc = scenes.config5(present=(64, 36))
    r = Renderer(64, 36, 1.0, node_capacity=1 << 12, chunk_capacity=4, grid_capacity=4, clip_levels=6, clip_res=512,
                 device=dev)
    out = {}
    try:
        for name, moves in (("full_rebuild", [(100.0, 100.0)]), ("scroll_1m", [(100.0, 100.0), (101.0, 100.0)])):
            cpu, gpu = Clipmap(sc.spec, 6, 512, 1.0), Clipmap(sc.spec, 6, 512, 1.0)
            for x, z in moves[:-1]:
                r.write_clipmap_updates(*cpu.update(x, z))
                gpu.update_device(r, x, z)
            torch.cuda.synchronize(dev)
            x, z = moves[-1]
            t0 = time.perf_counter()
            params, patches = cpu.update(x, z)
            r.write_clipmap_updates(params, patches)
            torch.cuda.synchronize(dev)  # the upload stream's copies have landed
            t1 = time.perf_counter()
            gpu.update_device(r, x, z)
            torch.cuda.synchronize(dev)
            t2 = time.perf_counter()
            texels = int(sum(p[3] * p[4] for p in patches))
            out[name] = {"texels": texels, "host_ms": round((t1 - t0) * 1e3, 3), "device_ms": round((t2 - t1) * 1e3, 3),
                         "note": "host: CPU texels + upload; device: plan + kernel; wall clock to completion"}
    finally:
        r.close()
    return out


def run_builder(dev, steps: int = 3, warmup: int = 2):
    """Chunk builds, all 1024 chunks of the config-2 world (16 x 4 x 16, caves
    above 0.6): the device builder (ground + material fill + octree/ropes
    kernels, two calls of 512 chunks, device events per kernel) against the
    host builder (the C++ port of svo/builder.rs) on all host cores on a
    bounded sample.  e2e: World.prebuild_device, host copies of every chunk
    included, wall clock."""
    import os
    import time

    import torch

    from vxe import _abi as A
    from vxe import scenes
    from vxe.renderer import Renderer
    from vxe.world import World

    sc = scenes.config2(present=(64, 36))
    keys = [(x, y, z) for z in range(16) for y in range(4) for x in range(16)]
    r = Renderer(64, 36, 1.0, node_capacity=1 << 12, chunk_capacity=4, grid_capacity=4, clip_levels=1, clip_res=16,
                 device=dev)
    wp = sc.spec.params()
    parts = [torch.tensor(keys[i:i + A.BUILD_BATCH_MAX], dtype=torch.int32, device=f"cuda:{dev}")
             for i in range(0, len(keys), A.BUILD_BATCH_MAX)]
    try:
        counts = [r.build_chunks(wp, c, node_cap=0)["counts"] for c in parts]
        cap = int(max(int(c[:, 0].max()) for c in counts))
        solid = int(sum(int(c[:, 1].sum()) for c in counts))
        working = int(sum(int((c[:, 1] > 0).sum()) for c in counts))  # all-air chunks return at once
        nodes_total = int(sum(int(c[:, 0].sum()) for c in counts))
        per = {"columns": [], "svo": []}
        for it in range(warmup + steps):
            step = {"columns": 0.0, "svo": 0.0}
            for c in parts:
                r.build_chunks(wp, c, node_cap=cap)
                for k, v in r.build_timings().items():
                    step[k] += v
            if it >= warmup:
                for k in per:
                    per[k].append(step[k])
        dev_ms = statistics.mean(per["columns"]) + statistics.mean(per["svo"])
        wd = World(sc.spec, sc.grid_origin, sc.grid_dims, sc.node_capacity)
        wd.prebuild_device(r, keys[:64], batch=64)  # warm
        wd = World(sc.spec, sc.grid_origin, sc.grid_dims, sc.node_capacity)
        t0 = time.perf_counter()
        wd.prebuild_device(r, keys, batch=256)
        e2e_s = time.perf_counter() - t0
    finally:
        r.close()
    # streaming the whole grid into a renderer's world: device builds straight
    # into the arenas (World.populate_device) vs host builds on every core plus
    # the upload (World.populate + Renderer.upload_world); wall clock to the
    # world being resident, median of 3
    kw = dict(node_capacity=sc.node_capacity, chunk_capacity=len(keys), grid_capacity=len(keys), clip_levels=1,
              clip_res=16, device=dev)
    res_s, host_s2 = [], []
    for _ in range(3):
        rr = Renderer(64, 36, 1.0, **kw)
        try:
            wr = World(sc.spec, sc.grid_origin, sc.grid_dims, sc.node_capacity)
            rr.synchronize()
            t0 = time.perf_counter()
            wr.populate_device(rr)
            rr.synchronize()
            res_s.append(time.perf_counter() - t0)
            wh2 = World(sc.spec, sc.grid_origin, sc.grid_dims, sc.node_capacity)
            t0 = time.perf_counter()
            ups = wh2.populate()
            rr.upload_world(wh2, ups)
            rr.synchronize()
            host_s2.append(time.perf_counter() - t0)
        finally:
            rr.close()
    # host builder on every host core, a bounded sample of 128 chunks spread over the grid
    threads = os.cpu_count() or 1
    sample = keys[::8]
    wh = World(sc.spec, sc.grid_origin, sc.grid_dims, sc.node_capacity)
    t0 = time.perf_counter()
    wh.prebuild(sample, threads=threads)
    host_s = time.perf_counter() - t0
    # bytes the octree kernel must move per chunk that holds a solid voxel
    # (an all-air chunk writes its lone air root and returns): the 64^3
    # materials read, 32^3 level-5 state and offset words written and read
    # back, colinfo and macro words, node (16 B) and rope (32 B) records written
    svo_bytes = working * (64 ** 3 + 32 ** 3 * 4 * 4 + 2048 * 4 + 16 * 4) + nodes_total * 48
    return {
        "workload": "1024 chunks of the config-2 world (16x4x16, 64^3 voxels each)",
        "chunks_per_s": round(len(keys) / (dev_ms * 1e-3), 1),
        "device_ms": round(dev_ms, 3),
        "kernel_ms": {k: round(statistics.mean(v), 3) for k, v in per.items()},
        "steps": steps, "warmup": warmup,
        "nodes_total": nodes_total, "solid_voxels": solid, "node_cap": cap, "chunks_with_solid_voxels": working,
        "svo_kernel_gbs": round(svo_bytes / (statistics.mean(per["svo"]) * 1e-3) / 1e9, 2),
        "svo_kernel_gbs_note": "algorithmic bytes of the chunks holding solid voxels / k_build_svo time",
        "e2e": {"resident_chunks_per_s": round(len(keys) / statistics.median(res_s), 1),
                "resident_seconds": round(statistics.median(res_s), 4),
                "host_build_upload_chunks_per_s": round(len(keys) / statistics.median(host_s2), 1),
                "host_build_upload_seconds": round(statistics.median(host_s2), 4),
                "host_copies_chunks_per_s": round(len(keys) / e2e_s, 1),
                "note": "resident: World.populate_device (counting build, count readback, slot/arena "
                        "bookkeeping, resident build, grid write); host_build_upload: World.populate on "
                        f"{os.cpu_count()} host threads + Renderer.upload_world; host_copies: "
                        "World.prebuild_device (device build, chunk records copied to the host)"},
        "cpu_baseline": {"chunks_per_s": round(len(sample) / host_s, 2), "cores": threads, "kind": "port",
                         "sample": f"{len(sample)} chunks (every 8th of the grid), World.prebuild thread pool"},
    }


def build_profile(n: int) -> None:
    """The chunk builder on the first n chunks of the config-2 grid: a counting
    build (node_cap 0), then the full build; prints the kernels' device ms."""
    import torch

    from vxe import scenes
    from vxe.renderer import Renderer

    sc = scenes.config2(present=(64, 36))
    keys = [(x, y, z) for z in range(16) for y in range(4) for x in range(16)][:n]
    r = Renderer(64, 36, 1.0, node_capacity=1 << 12, chunk_capacity=4, grid_capacity=4, clip_levels=1, clip_res=16)
    try:
        c = torch.tensor(keys, dtype=torch.int32, device="cuda:0")
        wp = sc.spec.params()
        cap = int(r.build_chunks(wp, c, node_cap=0)["counts"][:, 0].max())
        r.build_chunks(wp, c, node_cap=cap)
        print(json.dumps({"chunks": len(keys), "node_cap": cap, "kernel_ms": r.build_timings()}))
    finally:
        r.close()


def run_configs(dev):
    """Secondary frame lines: config 1 (one 64^3 chunk, 256x144 frames),
    config 5 (32x8x32 chunks, 6-level 512^2 clipmap, 3840x2160 present /
    1920x1080 internal) and config 2 at render scale 1.0."""
    from vxe import scenes

    out = {}
    for key, sc, steps in (("config1", scenes.config1(), 32), ("config5_4k", scenes.config5(), 8),
                           ("config2_scale1", scenes.config2(present=(1920, 1080), render_scale=1.0), 8)):
        sc.shift_every = 0
        ms, rays = frame_series(sc, dev, steps=steps, warmup=4)
        out[key] = {"present": list(sc.present), "internal": list(sc.internal), "frame_ms": round(ms, 4),
                    "mrays_per_s": round(rays / ms / 1e3, 3), "steps": steps, "warmup": 4,
                    "l2": "flushed between steps"}
    return out


# Frames the e2e loop keeps in flight: step i waits for step i - depth's
# output, so a step's host work hides behind the frames queued before it.
# Two were measured slower for host streaming (7.75 vs 7.37 ms): a grid
# shift's uploads wait for every frame in flight, and the queue drains there.
PIPELINE_DEPTH = 1


def run_e2e(args, sc, dev, world_size):
    import torch

    from vxe import _abi as A
    from vxe.renderer import Renderer
    from vxe.scenes import FrameDriver

    drv = r = None

    def setup(device_streaming=False):
        """A fresh driver, world and renderer: every mode runs the same frames.
        Host streaming: chunks entering the grid at the shifts are built on the
        host before timing (the reference builds them on its worker pool) and
        their upload is timed.  Device streaming: they are built resident on
        the device inside the timed region and slots move on the device."""
        nonlocal drv, r
        cap = int(np.prod(sc.grid_dims))
        r = Renderer(sc.present[0], sc.present[1], sc.render_scale, node_capacity=sc.node_capacity,
                     chunk_capacity=cap, grid_capacity=cap, clip_levels=sc.clip_levels, clip_res=sc.clip_res,
                     flags=A.FLAG_GODRAY_MACRO_ALIAS, device=dev)
        drv = FrameDriver(sc, device_renderer=r if device_streaming else None, mirror=False)
        ups = drv.initial_uploads()
        if not device_streaming:
            for ox in range(1, 4):
                for iz in range(sc.grid_dims[2]):
                    for iy in range(sc.grid_dims[1]):
                        drv.world.chunk((ox + sc.grid_dims[0] - 1, iy, iz))
            r.upload_world(drv.world, ups)

    pw, ph = sc.present
    host_out = [torch.empty((ph, pw, 4), dtype=torch.float32).pin_memory().numpy()
                for _ in range(PIPELINE_DEPTH + 1)]
    h2d = d2h = 0

    def one(i, pipelined):
        """Step i: this step's world writes, camera and clipmap from host
        memory, the frame, and the read-back of its output -- synchronous, or
        queued on the copy stream (returns the ticket)."""
        nonlocal h2d, d2h
        back = []
        b = 464
        drv.last_shift = None
        if drv.frame >= 64:
            # restart the path: the grid returns to its first origin
            drv.frame = 0
            if drv.device is not None:
                built, moved = drv.world.shift_device(r, -drv.world.grid_origin[0], 0, 0)
                # coords + places + slot moves + grid in, node counts out
                b += 36 * built + 8 * moved + drv.world.grid.nbytes
                d2h += 8 * built
            else:
                back = drv.world.shift(-drv.world.grid_origin[0], 0, 0)
        uploads, grid_changed, clip, cam = drv.step()
        if drv.last_shift is not None:
            built, moved = drv.last_shift
            b += 36 * built + 8 * moved + drv.world.grid.nbytes
            d2h += 8 * built
        if back:
            uploads, grid_changed = back + uploads, True
        if uploads:
            r.apply_chunk_uploads(uploads)
            b += sum(48 + (len(u.data.nodes) * 48 + 16 * 4 + 2048 * 4 if u.data is not None else 0) for u in uploads)
        if grid_changed:
            r.write_chunk_grid(drv.world.grid)
            b += drv.world.grid.nbytes
        params, patches = clip
        r.write_clipmap_updates(params, patches)
        b += 528 + sum(p[5].nbytes for p in patches)
        r.write_camera(cam)
        r.encode_compute(sync=False)
        out = host_out[i % (PIPELINE_DEPTH + 1)]
        h2d += b
        d2h += out.nbytes
        if pipelined:
            return r.read_image_async(A.IMG_OUTPUT, out)
        r._check(r._lib.vxe_read_image(r._ctx, A.IMG_OUTPUT, out.ctypes.data, out.nbytes), "read")
        return None

    def timed(pipelined):
        nonlocal h2d, d2h
        for i in range(args.warmup):
            t = one(i, pipelined)
            if t is not None:
                r.read_image_wait(t)
        r.synchronize()
        h2d = d2h = 0
        if world_size > 1:
            torch.distributed.barrier()
        with no_gc():
            t0 = time.perf_counter()
            pending = []  # tickets of the outputs not yet waited for, oldest first
            for i in range(args.steps):
                t = one(i, pipelined)
                if t is not None:
                    pending.append(t)
                if len(pending) > PIPELINE_DEPTH:
                    r.read_image_wait(pending.pop(0))  # step i - depth's output is in host memory
            for t in pending:
                r.read_image_wait(t)
            r.synchronize()
            dt = time.perf_counter() - t0
        if world_size > 1:
            torch.distributed.barrier()
        return dt

    setup()
    dt = timed(True)
    bytes_host = (h2d, d2h)
    r.close()
    setup()
    serial_s = timed(False)
    r.close()
    setup(device_streaming=True)
    dev_s = timed(True)
    bytes_dev = (h2d, d2h)
    r.close()
    h2d, d2h = bytes_host
    rays = sc.internal[0] * sc.internal[1] * args.steps
    return {"seconds": dt, "rays": rays, "h2d_bytes_per_step": h2d // args.steps,
            "d2h_bytes_per_step": d2h // args.steps, "serial_seconds": serial_s,
            "device_streaming": {"seconds": dev_s, "h2d_bytes_per_step": bytes_dev[0] // args.steps,
                                 "d2h_bytes_per_step": bytes_dev[1] // args.steps}}


def device_streaming_line(e2e: dict, steps: int, n: int):
    """The e2e frames with the world streamed on the device (resident builds of
    the entering chunks and device slot moves inside the timed region)."""
    ds = e2e.get("device_streaming")
    if not ds or not ds["seconds"] == ds["seconds"]:
        return None
    return {"value": round(replica_value(e2e["rays"], n, ds["seconds"]), 3), "unit": UNIT,
            "frame_ms": round(ds["seconds"] * 1e3 / steps, 3), "h2d_bytes_per_step": ds["h2d_bytes_per_step"],
            "d2h_bytes_per_step": ds["d2h_bytes_per_step"],
            "note": "pipelined read-back; chunks entering at the grid shifts built resident on the device "
                    "(counting build + count read-back + resident build) and slots moved on the device, "
                    "inside the timed region"}


def cpu_sample(seconds: float, present, threads: int):
    """Times the oracle (scalar C++ restatement of the WGSL) on full frames of
    the path.  The frame inputs (camera, clipmap patches, streamed chunks) are
    produced between the timed renders; only the passes are timed."""
    from oracle import oracle as O
    from vxe.scenes import FrameDriver, config2

    sc = config2(present=present)
    drv = FrameDriver(sc)
    drv.initial_uploads()
    runner = O.OracleFrameRunner(drv.world, sc.internal, sc.present, drv.clip.tex, sc.clip_res)
    frames = 0
    ctr = None
    elapsed = 0.0
    while elapsed < seconds or frames == 0:
        if drv.frame >= 64:
            drv.frame = 0
        uploads, gc, clip, cam = drv.step()
        t0 = time.perf_counter()
        runner.render(cam, clip[0], threads=threads)
        elapsed += time.perf_counter() - t0
        if ctr is None:
            ctr = (runner.primary_ctr.as_dict(), runner.godray_ctr.as_dict(), runner.trace_ctr.as_dict())
        frames += 1
    rays = frames * sc.internal[0] * sc.internal[1]
    return {"rays": rays, "seconds": elapsed, "frames": frames, "counters": ctr}


def cpu_table(threads: int) -> dict:
    """The oracle's rays/s on 1 host thread and on `threads`, bounded samples:
    config 1 (one 64^3 chunk, 256x144 rays, cold full frames) and the config-2
    1080p frame's primary pass over tile rows 30..37 (path frame 5, after four
    warm frames on all threads)."""
    from oracle import oracle as O
    from vxe.scenes import FrameDriver, config1, config2

    out = {}
    sc = config1()
    drv = FrameDriver(sc)
    drv.initial_uploads()
    _, _, _, cam = drv.step()
    clip = drv.empty_clip()
    row = {}
    for nt in (1, threads):
        runner = O.OracleFrameRunner(drv.world, sc.internal, sc.present, None, sc.clip_res)
        frames, t0 = 0, time.perf_counter()
        while frames < 3 or time.perf_counter() - t0 < 1.0:
            runner.ping = 0  # cold frames
            runner.render(cam, clip, threads=nt)
            frames += 1
        dt = time.perf_counter() - t0
        row[f"{nt}_threads"] = round(frames * sc.internal[0] * sc.internal[1] / dt / 1e6, 4)
    out["config1_full_frame_mrays_per_s"] = row
    sc = config2()
    drv = FrameDriver(sc)
    drv.initial_uploads()
    runner = O.OracleFrameRunner(drv.world, sc.internal, sc.present, drv.clip.tex, sc.clip_res)
    for _ in range(5):
        _, _, clip, cam = drv.step()
        runner.render(cam, clip[0], threads=threads)
    _, _, clip, cam = drv.step()
    row = {}
    for nt in (1, threads):
        t0 = time.perf_counter()
        rays = runner.primary_rows(cam, clip[0], 30, 38, threads=nt)
        row[f"{nt}_threads"] = round(rays / (time.perf_counter() - t0) / 1e6, 4)
    out["config2_1080p_primary_rows_30_37_mrays_per_s"] = row
    return out


def record_bytes(c: dict) -> int:
    """Full record sizes of the loads the oracle counted: node 16, rope 32, meta 48, grid / macro / colinfo
    words and clip texels 4."""
    return int(16 * c["node_loads"] + 32 * c["rope_loads"] + 48 * c["meta_loads"] + 4 * c["grid_loads"] +
               4 * c["macro_loads"] + 4 * c["colinfo_loads"] + 4 * c["clip_loads"])


def algorithmic_primary_bytes(counters: dict, pixels: int) -> int:
    """Primary pass: record bytes the reference algorithm loads + compulsory image I/O."""
    # outputs: color 16 + depth 4 + hist 16 + shadow 4 + local_hist 16; inputs: hist 16 + shadow 4 + local_hist 16
    io = pixels * (16 + 4 + 16 + 4 + 16 + 16 + 4 + 16)
    return record_bytes(counters) + int(io)


def algorithmic_trace_bytes(trace_counters: dict, pixels: int) -> int:
    """Voxel trace phase (k_primary_trace): its record loads + the two history texels the hit-distance
    hint reads per pixel (own + reprojected, 16 B each)."""
    return record_bytes(trace_counters) + 32 * int(pixels)


def max_over_ranks(values, device="cpu"):
    """Element-wise max of per-rank timings (replicas: the job ends with the slowest rank)."""
    import torch
    import torch.distributed as dist

    t = torch.tensor(list(values), dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def replica_value(rays_per_rank: int, world_size: int, max_seconds: float) -> float:
    """Whole-job Mrays/s: every rank traces the same workload on its own GPU."""
    return rays_per_rank * world_size / max_seconds / 1e6


def peaks():
    p = REPO / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def l2_peak(dev: int) -> float:
    """L2 read bandwidth of this GPU (vxe_measure_l2_bandwidth: a 48 MiB
    L2-resident buffer read 20 times with 16-byte loads), GB/s."""
    import ctypes as C

    from vxe import _abi as A

    g = C.c_double()
    st = A.lib().vxe_measure_l2_bandwidth(dev, 48 << 20, 20, C.byref(g))
    if st != A.VXE_OK:
        raise A.VxeError(st, "vxe_measure_l2_bandwidth")
    return float(g.value)


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world_size = int(os.environ.get("WORLD_SIZE", "1"))
    if args.impl == "reference":
        return main_reference(args, rank, world_size)
    if args.build_profile:
        return build_profile(args.build_profile)
    if world_size > 1:
        import datetime

        import torch

        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    res = run_vxe(args, rank, world_size)
    if res is None:
        return
    batch = srv = configs = None
    if not args.no_batch and world_size == 1:  # one GPU: the batched, served, secondary-config and builder lines
        batch, srv = run_batch_serve(0)
        srv["config4"] = run_serve_config4(0)
        configs = run_configs(0)
        configs["config5_with_queries"] = config5_with_queries(0)
        configs["clipmap_patches"] = run_clipmap(0)
        configs["chunk_builder"] = run_builder(0)
    if world_size > 1:
        import torch

        total_ms, e2e_s = max_over_ranks([res["total_ms"], res["e2e"]["seconds"]], device="cuda")
        torch.distributed.destroy_process_group()
    else:
        total_ms, e2e_s = res["total_ms"], res["e2e"]["seconds"]
    if rank != 0:
        return
    n = max(1, world_size)
    value = replica_value(res["rays_per_frame"] * args.steps, n, total_ms * 1e-3)
    e2e_val = replica_value(res["e2e"]["rays"], n, e2e_s)
    line = {
        "metric": METRIC, "value": round(value, 3), "unit": UNIT, "n_gpus": n, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(total_ms / args.steps, 4), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded value-noise world)",
        "config": bench_config(tuple(map(int, args.present.split("x"))), res["internal"], n),
        "frame_ms": {"tiles": round(statistics.mean(res["tiles_ms"]), 4),
                     "primary": round(statistics.mean(res["primary_ms"]), 4),
                     "primary_trace": round(statistics.mean(res["trace_ms"]), 4),
                     "k_primary_trace": round(statistics.mean(res["walk_ms"]), 4),
                     "grass_cells": round(statistics.mean(res["grass_ms"]), 4),
                     "godray": round(statistics.mean(res["godray_ms"]), 4),
                     "composite": round(statistics.mean(res["composite_ms"]), 4)},
        "e2e": {"value": round(e2e_val, 3), "unit": UNIT, "h2d_bytes_per_step": res["e2e"]["h2d_bytes_per_step"],
                "d2h_bytes_per_step": res["e2e"]["d2h_bytes_per_step"],
                "frame_ms": round(e2e_s * 1e3 / args.steps, 3),
                "mode": f"pipelined: step i's output read back on the copy stream while later frames run "
                        f"(vxe_read_image_async, waited {PIPELINE_DEPTH} steps later, {PIPELINE_DEPTH + 1} pinned "
                        "host buffers; every output lands inside the timed region)",
                "serial_frame_ms": round(res["e2e"]["serial_seconds"] * 1e3 / args.steps, 3),
                "device_streaming": device_streaming_line(res["e2e"], args.steps, n)},
        # per frame: k_grass_wind, k_tiles, k_primary_trace, k_probe_dda, k_slab_eval, k_slab_pick,
        # k_gov_eval, k_primary_resolve, k_shade_prep, k_shade_shadow, k_shade_lights, k_shade_vox,
        # k_shade_far x 2 and k_godray_far (side stream), k_godray, k_composite
        "gpu_launches": 17 * args.steps,
        "batch": batch,
        "serve": srv,
        "configs": configs,
        "clocks": res["clocks"],
        "device_error_word": res["error_word"],
    }
    peak, peak_kind = peaks()
    l2 = l2_peak(0)
    prim_s = statistics.mean(res["primary_ms"]) * 1e-3
    trace_s = statistics.mean(res["trace_ms"]) * 1e-3
    # The reference's voxel trace runs here as five launches (the walk, then the
    # grass probes' column DDAs, slab marches, pick and resolve); the roofline
    # unit is that stage, timed by the events around it.
    roof = {"bound": "hbm", "achieved": None, "peak": peak, "unit": "GB/s", "frac": None, "traffic": None,
            "kernel": "trace stage: k_primary_trace + k_probe_dda + k_slab_eval + k_slab_pick + k_primary_resolve",
            "peak_kind": peak_kind, "launch_ms": round(trace_s * 1e3, 4),
            "walk_kernel_ms": round(statistics.mean(res["walk_ms"]), 4)}
    present = tuple(int(v) for v in args.present.split("x"))
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        cs = cpu_sample(args.cpu_seconds, present, threads)
        line["cpu_baseline"] = {"value": round(cs["rays"] / cs["seconds"] / 1e6, 4), "unit": UNIT, "cores": threads,
                                "kind": "port",
                                "sample": f"{cs['frames']} full frames of the same workload (path frames 0..{cs['frames'] - 1})",
                                "table": cpu_table(threads)}
        tb = algorithmic_trace_bytes(cs["counters"][2], res["rays_per_frame"])
        achieved = tb / trace_s / 1e9
        roof.update({"achieved": round(achieved, 2), "frac": round(achieved / peak, 5),
                     "algorithmic_bytes_per_launch": tb,
                     "bytes_per_ray": round(tb / res["rays_per_frame"], 2)})
        if l2:
            roof["l2"] = {"peak": round(l2, 1), "unit": "GB/s", "frac": round(achieved / l2, 5),
                          "note": "measured here: vxe_measure_l2_bandwidth, 48 MiB L2-resident buffer, 16-byte loads"}
        ab = algorithmic_primary_bytes(cs["counters"][0], res["rays_per_frame"])
        pa = ab / prim_s / 1e9
        roof["primary_pass"] = {"kernels": "k_primary_trace + k_shade_vox + k_shade_far",
                                "achieved": round(pa, 2), "frac": round(pa / peak, 5),
                                "algorithmic_bytes_per_frame": ab, "ms": round(prim_s * 1e3, 4)}
    # DRAM bytes of the trace stage per 1080p frame: one ncu capture of the
    # same five kernels on this workload (data file beside the profiles)
    traffic = REPO / "profiles" / "trace_stage_config2_1080p_dram.json"
    if traffic.exists() and present == (1920, 1080):
        roof["traffic"] = int(json.loads(traffic.read_text())["dram_bytes_per_stage"])
        roof["traffic_source"] = "ncu dram__bytes_read.sum + dram__bytes_write.sum, frame 1 of this path"
    line["roofline"] = roof
    print(json.dumps(line))


def _ref_wgsl_frames(drv, sc, threads):
    """The reference's own five compute passes, translated mechanically from
    its WGSL to C++ (oracle/_ref/libref_wgsl.so, built by vxe_build where the
    reference's sources are), as a per-step frame function; None where that
    library is absent.  The world is bound once, the camera and clipmap per
    frame (not timed); the histories ping-pong as the reference's do."""
    import vxe_build

    if not vxe_build.REF_WGSL_LIB.exists():
        return None
    try:
        ref = C.CDLL(str(vxe_build.REF_WGSL_LIB))
    except OSError as e:  # built on another machine and unusable here: the port runs instead
        print(f"reference arm: {vxe_build.REF_WGSL_LIB.name} does not load ({e}); timing the port", file=sys.stderr)
        return None
    ref.ref_wgsl_frame.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_void_p, C.c_uint32]
    w = drv.world
    iw, ih = sc.internal
    pw, ph = sc.present
    z = lambda *shape: np.zeros(shape, np.float32)
    stride = ((iw * 4 + 255) & ~255) // 4
    io = [z(ih, iw, 4), z(ih, iw), z(ih, iw, 4), z(ih, iw, 4), z(ih, iw, 4), z(ih, iw), z(ih, stride),
          z(ih, iw, 4), z(ih, iw, 4), z(ih, iw, 4), z(ih, iw, 4), z(ph, pw, 4), z(ph, pw, 4), z(ph, pw, 4),
          z(ph, pw, 4)]
    u64 = C.c_uint64
    keep = {}

    def frame(cam, clip_params):
        keep["cam"], keep["clip"] = cam, clip_params
        keep["tex"] = np.ascontiguousarray(drv.clip.tex, np.float32)
        ref.ref_wgsl_set_scene(C.c_void_p(w.metas.ctypes.data), u64(w.metas.shape[0]),
                               C.c_void_p(w.nodes.ctypes.data), u64(len(w.nodes)), C.c_void_p(w.grid.ctypes.data),
                               u64(len(w.grid)), C.c_void_p(w.macro.ctypes.data), u64(len(w.macro)),
                               C.c_void_p(w.ropes.ctypes.data), u64(len(w.ropes)),
                               C.c_void_p(w.colinfo.ctypes.data), u64(len(w.colinfo)), C.c_void_p(C.addressof(cam)))
        t = keep["tex"]
        ref.ref_wgsl_set_clip(C.c_void_p(C.addressof(clip_params)), t.ctypes.data_as(C.POINTER(C.c_float)),
                              C.c_int32(t.shape[1]), C.c_int32(t.shape[0]))
        ptrs = (C.c_void_p * 15)(*[a.ctypes.data for a in io])
        t0 = time.perf_counter()
        ref.ref_wgsl_frame(iw, ih, pw, ph, ptrs, threads)
        dt = time.perf_counter() - t0
        io[3], io[4] = io[4], io[3]  # this frame's histories are the next one's inputs
        io[5][:] = io[6][:, :iw]  # the shadow buffer -> texture copy
        io[7], io[8] = io[8], io[7]
        io[9], io[10] = io[10], io[9]
        io[12], io[14] = io[14], io[12]
        return dt

    return frame


def main_reference(args, rank, world_size):
    """The reference arm, on all host cores, one full frame of the same
    workload per step.  Where the reference's sources were present at build
    time it runs the reference's own compute passes -- its WGSL translated
    mechanically to C++ (oracle/wgsl_to_cpp.py), shown bit-identical to the
    oracle's frames -- else the oracle's C++ restatement of them (oracle/).
    Its frame inputs come from a host-only build of the producers
    (oracle/libref_producer.so), so this process maps no CUDA library of this
    repository; the producer work between frames is not timed."""
    if rank != 0:
        return
    from vxe import _abi as A

    import vxe_build

    A.use_host_library(vxe_build.build_ref_producer())
    threads = os.cpu_count() or 1
    present = tuple(int(v) for v in args.present.split("x"))
    from oracle import oracle as O
    from vxe.scenes import FrameDriver, config2

    sc = config2(present=present)
    drv = FrameDriver(sc)
    drv.initial_uploads()
    ref_frame = _ref_wgsl_frames(drv, sc, threads)
    runner = None if ref_frame is not None else O.OracleFrameRunner(drv.world, sc.internal, sc.present,
                                                                    drv.clip.tex, sc.clip_res)

    def step():
        if drv.frame >= 64:
            drv.frame = 0
        _, _, clip, cam = drv.step()
        if ref_frame is not None:
            return ref_frame(cam, clip[0])
        t0 = time.perf_counter()
        runner.render(cam, clip[0], threads=threads)
        return time.perf_counter() - t0

    for _ in range(args.warmup):
        step()
    dt = sum(step() for _ in range(args.steps))
    rays = sc.internal[0] * sc.internal[1] * args.steps
    v = rays / dt / 1e6
    kind = "reference" if ref_frame is not None else "port"
    note = ("the reference's own WGSL compute passes (main_primary, main_local_taa, main_godray, main_composite, "
            "main_composite_taa) translated mechanically to C++ and run on the host cores; no Rust toolchain or "
            "graphics stack here to run them as they are" if ref_frame is not None else
            "reference is Rust+WGSL; no Rust toolchain or graphics stack here, so this arm runs the C++ scalar "
            "restatement of its WGSL (oracle/) on the host cores")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(v, 4), "unit": UNIT, "n_gpus": max(1, world_size),
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(dt * 1e3 / args.steps, 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded value-noise world)",
        "config": bench_config(present, sc.internal, max(1, world_size)),
        "cpu_baseline": {"value": round(v, 4), "unit": UNIT, "cores": threads, "kind": kind,
                         "sample": "full frames of the same workload, one per step (path frames "
                                   f"{args.warmup}..{args.warmup + args.steps - 1}); passes timed, producers not"},
        "e2e": {"value": round(v, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": note,
    }))


def bench_config(present, internal, n):
    """The `config` object of both arms' lines (the same workload keys)."""
    return {"workload": WORKLOAD, "present": list(present), "internal": list(internal),
            "parallelism": "replicas" if n > 1 else "single",
            "l2": "GPU arm: flushed between steps (512 MiB memset), per-step CUDA events"}


if __name__ == "__main__":
    main()
