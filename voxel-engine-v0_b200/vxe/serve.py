"""Continuous-batching request server over the batch lanes of one context.

Requests arrive by a seeded Poisson process: 70 % viewport renders (width and
height uniform in [256, 1920] x [256, 1080], primary hit records), 30 % ray
query batches (log-uniform 1k-256k rays, origins uniform in the world, uniform
directions).  The server loop

  * admits waiting requests in arrival order while their device footprint fits
    the memory budget (outputs, query inputs, and for a viewport the history
    textures a renderer keeps for it: 5 RGBA32F + 2 R32F at internal size and
    2 RGBA32F at present size),
  * starts a batch on any free lane with everything admitted so far, so work
    that arrives while other batches run overlaps with them on the device,
  * frees a batch's memory when its lane reports completion,
  * re-uploads chunks on the context's upload stream every tick (the reference
    applies streamed uploads every frame),
  * records per-request latency = completion - arrival (host clock).

`serve_plain` is the baseline: one request at a time, one plain launch each.
"""
from __future__ import annotations

import math
import time
from collections import deque
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A
from .world import Upload, World, build_camera


@dataclass
class SRequest:
    rid: int
    kind: str            # "v" or "q"
    arrival: float       # seconds from start
    w: int = 0
    h: int = 0
    n: int = 0
    cam: object = None
    o: np.ndarray | None = None
    d: np.ndarray | None = None
    done: float = -1.0
    out: object = None
    tin: tuple = ()

    @property
    def rays(self) -> int:
        return self.w * self.h if self.kind == "v" else self.n

    def footprint(self) -> int:
        if self.kind == "v":
            internal = (self.w // 2) * (self.h // 2)
            return self.w * self.h * 32 + internal * (5 * 16 + 2 * 4) + self.w * self.h * 2 * 16
        return self.n * (24 + 32)


def make_arrivals(world: World, rate: float, count: int, seed: int = 1, vp_frac: float = 0.7,
                  vp_range=((256, 1920), (256, 1080)), q_range=(1e3, 256e3)):
    rng = np.random.default_rng(seed)
    lo, hi = world.world_aabb_m()
    t = 0.0
    out = []
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        if rng.uniform() < vp_frac:
            w = int(rng.integers(vp_range[0][0], vp_range[0][1] + 1))
            h = int(rng.integers(vp_range[1][0], vp_range[1][1] + 1))
            pos = np.array([rng.uniform(lo[0] + 10, hi[0] - 10), rng.uniform(6.0, 12.0),
                            rng.uniform(lo[2] + 10, hi[2] - 10)])
            cam = build_camera(pos, rng.uniform(0, 2 * math.pi), rng.uniform(-0.45, 0.05), (w, h), (w, h),
                               frame_index=1, time_s=0.0, world=world, jitter=False)
            out.append(SRequest(i, "v", t, w=w, h=h, cam=cam))
        else:
            n = int(round(math.exp(rng.uniform(math.log(q_range[0]), math.log(q_range[1])))))
            o = rng.uniform(lo, hi, size=(n, 3)).astype(np.float32)
            d = rng.normal(size=(n, 3))
            d = (d / np.linalg.norm(d, axis=1, keepdims=True)).astype(np.float32)
            out.append(SRequest(i, "q", t, n=n, o=o, d=d))
    return out


def _to_request(r: SRequest, torch, device="cuda") -> A.Request:
    q = A.Request()
    r.out = torch.empty(r.rays * 32, dtype=torch.uint8, device=device)
    if r.kind == "v":
        q.kind, q.width, q.height, q.camera = A.REQ_VIEWPORT, r.w, r.h, r.cam
    else:
        to = torch.from_numpy(r.o).to(device, non_blocking=True)
        td = torch.from_numpy(r.d).to(device, non_blocking=True)
        r.tin = (to, td)
        q.kind, q.ray_count, q.tmax = A.REQ_QUERY, r.n, 120.0
        q.d_origins, q.d_dirs = to.data_ptr(), td.data_ptr()
    q.d_out = r.out.data_ptr()
    return q


@dataclass
class ServeReport:
    latencies_ms: list
    rays: int
    seconds: float
    batches: int
    max_inflight: int
    uploads: int
    extra: dict = field(default_factory=dict)

    def summary(self) -> dict:
        lat = np.asarray(self.latencies_ms)
        return {"requests": len(lat), "p50_ms": round(float(np.percentile(lat, 50)), 3),
                "p99_ms": round(float(np.percentile(lat, 99)), 3), "mrays_per_s": round(self.rays / self.seconds / 1e6, 3),
                "seconds": round(self.seconds, 4), "batches": self.batches, "max_batches_in_flight": self.max_inflight,
                "chunk_reuploads": self.uploads, **self.extra}


def serve(renderer, world: World, requests, torch, mem_budget: int, lanes: int = 2, tile=(8, 4), rpt: int = 1,
          max_batch: int = 64, reuploads_per_tick: int = 10, tick_s: float = 0.016, keep_outputs: bool = False,
          mode: int = A.BATCH_PERSISTENT) -> ServeReport:
    reqs = sorted(requests, key=lambda r: r.arrival)
    pending = deque(reqs)
    waiting = deque()
    inflight = {}
    reserved = 0
    rng = np.random.default_rng(99)
    resident = [k for k in world.slot_to_key if not world.chunk(k).macro_empty]
    batches = uploads = max_inflight = 0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    next_tick = 0.0
    while pending or waiting or inflight:
        now = time.perf_counter() - t0
        while pending and pending[0].arrival <= now:
            waiting.append(pending.popleft())
        if reuploads_per_tick and now >= next_tick and (pending or waiting or inflight):
            # re-upload resident chunks (same bytes) on the upload stream
            picks = rng.choice(len(resident), size=min(reuploads_per_tick, len(resident)), replace=False)
            ups = []
            for i in picks:
                key = resident[int(i)]
                slot = world.key_to_slot[key]
                base, _ = world.alloc[key]
                ups.append(Upload(slot, world.metas[slot].copy(), base, world.chunk(key)))
            renderer.apply_chunk_uploads(ups)
            uploads += len(ups)
            next_tick += tick_s
        for lane in list(inflight):
            st = renderer.batch_wait(lane, block=False)
            if st is None:
                continue
            done = time.perf_counter() - t0
            for r in inflight.pop(lane):
                r.done = done
                reserved -= r.footprint()
                if not keep_outputs:
                    r.out = None
                    r.tin = ()
        free = [l for l in range(lanes) if l not in inflight]
        if free and waiting:
            batch = []
            while waiting and len(batch) < max_batch and reserved + waiting[0].footprint() <= mem_budget:
                r = waiting.popleft()
                reserved += r.footprint()
                batch.append(r)
            if not batch and not inflight and waiting:
                # a single request larger than the whole budget still runs, alone
                r = waiting.popleft()
                reserved += r.footprint()
                batch.append(r)
            if batch:
                rq = [_to_request(r, torch) for r in batch]
                torch.cuda.current_stream().synchronize()  # query inputs are on the device
                renderer.submit_batch_async(free[0], rq, tile, rpt, mode)
                inflight[free[0]] = batch
                batches += 1
                max_inflight = max(max_inflight, len(inflight))
                continue
        if not (pending and pending[0].arrival <= time.perf_counter() - t0):
            time.sleep(0.0002)
    seconds = time.perf_counter() - t0
    lat = [(r.done - r.arrival) * 1e3 for r in reqs]
    return ServeReport(lat, sum(r.rays for r in reqs), seconds, batches, max_inflight, uploads)


def serve_plain(renderer, world: World, requests, torch, keep_outputs: bool = False) -> ServeReport:
    """Baseline: FIFO, one request at a time, each as its own plain launch."""
    reqs = sorted(requests, key=lambda r: r.arrival)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for r in reqs:
        now = time.perf_counter() - t0
        if r.arrival > now:
            time.sleep(r.arrival - now)
        q = _to_request(r, torch)
        torch.cuda.current_stream().synchronize()
        renderer.submit_batch([q], (8, 4), 1, A.BATCH_PLAIN)
        r.done = time.perf_counter() - t0
        if not keep_outputs:
            r.out = None
            r.tin = ()
    seconds = time.perf_counter() - t0
    lat = [(r.done - r.arrival) * 1e3 for r in reqs]
    return ServeReport(lat, sum(r.rays for r in reqs), seconds, len(reqs), 1, 0)
