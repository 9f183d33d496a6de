"""Continuous-batching request server over the batch lanes of one context.

Requests arrive by a seeded Poisson process: 70 % render requests, 30 % ray
query batches (log-uniform 1k-256k rays, origins uniform in the world,
uniform directions).  A render request is either

  * the next frame of a client session ("f"): a viewport with its own size
    and camera path whose images and histories (primary hit, shadow, local
    light, godray, output TAA) stay resident on the device in a vxe_view
    between its frames, or
  * a one-off viewport ("v"): primary hit records of a cold frame, traced in
    the batch kernel.

The server loop

  * admits waiting requests in arrival order while their device footprint fits
    the memory budget (by default the device's free memory at start, from
    cudaMemGetInfo, less a reserve): a session's view (its history footprint: 5 RGBA32F +
    2 R32F at internal size and 2 RGBA32F at present size, plus scratch) is
    created when the session is first admitted and stays until memory is
    needed by another session (least recently used idle view first); a
    one-off viewport or query counts its outputs and inputs,
  * starts work on any free lane with everything admitted so far -- one
    persistent batch for viewports and queries, then the session frames on the
    same lane's stream, every pass of up to 8 sessions' frames in one launch
    (vxe_view_render_batch_async) -- so work that arrives while other lanes
    run overlaps with them on the device,
  * keeps a session's frames in order (one in flight at a time),
  * re-uploads chunks on the context's upload stream every tick (the reference
    applies streamed uploads every frame),
  * records per-request latency = completion - arrival (host clock).

`serve_plain` is the baseline: one request at a time (a frame rendered alone
on lane 0, a viewport or query batch as one plain launch).
"""
from __future__ import annotations

import math
import time
from collections import OrderedDict, deque
from dataclasses import dataclass, field

import numpy as np

from . import _abi as A
from .world import Upload, World, build_camera


@dataclass
class Session:
    """A client viewport: fixed size, a straight camera path from a seeded start."""

    sid: int
    w: int
    h: int
    pos: np.ndarray
    yaw: float
    pitch: float
    speed: float = 0.15           # metres per frame
    render_scale: float = 0.5
    frame: int = 0
    prev_vp: object = None

    def camera(self, world: World, frame: int, prev_vp=None):
        fwd = np.array([math.sin(self.yaw), 0.0, math.cos(self.yaw)])
        pos = self.pos + fwd * (self.speed * frame)
        internal = tuple(max(1, int(np.floor(np.float32(v) * np.float32(self.render_scale) + np.float32(0.5))))
                         for v in (self.w, self.h))
        # the world's wind clock is the server's, not the client's: one grass
        # table serves every lane
        return build_camera(pos, self.yaw + 0.002 * frame, self.pitch, (self.w, self.h), internal,
                            frame_index=frame + 1, time_s=0.0, world=world, jitter=True, prev_view_proj=prev_vp)


def make_sessions(world: World, count: int, seed: int = 3, size_range=((256, 1920), (256, 1080)),
                  render_scale: float = 0.5):
    rng = np.random.default_rng(seed)
    lo, hi = world.world_aabb_m()
    out = []
    for i in range(count):
        w = int(rng.integers(size_range[0][0], size_range[0][1] + 1))
        h = int(rng.integers(size_range[1][0], size_range[1][1] + 1))
        pos = np.array([rng.uniform(lo[0] + 15, hi[0] - 15), rng.uniform(6.0, 12.0), rng.uniform(lo[2] + 15, hi[2] - 15)])
        out.append(Session(i, w, h, pos, rng.uniform(0, 2 * math.pi), rng.uniform(-0.35, 0.0),
                           render_scale=render_scale))
    return out


@dataclass
class SRequest:
    rid: int
    kind: str            # "f" session frame, "v" one-off viewport, "q" query batch
    arrival: float       # seconds from start
    w: int = 0
    h: int = 0
    n: int = 0
    cam: object = None
    o: np.ndarray | None = None
    d: np.ndarray | None = None
    session: int = -1
    frame: int = -1
    done: float = -1.0
    out: object = None
    tin: tuple = ()

    @property
    def rays(self) -> int:  # primary rays: present pixels of a viewport, internal pixels of a frame
        return self.w * self.h if self.kind == "v" else self.n

    def footprint(self) -> int:
        if self.kind == "v":
            internal = (self.w // 2) * (self.h // 2)
            return self.w * self.h * 32 + internal * (5 * 16 + 2 * 4) + self.w * self.h * 2 * 16
        if self.kind == "q":
            return self.n * (24 + 32)
        return 0  # session frames are charged through their view


def make_arrivals(world: World, rate: float, count: int, seed: int = 1, vp_frac: float = 0.7,
                  vp_range=((256, 1920), (256, 1080)), q_range=(1e3, 256e3), sessions=None):
    """Poisson arrivals; with `sessions`, render requests are session frames (a
    seeded client picks its next frame), else one-off viewports."""
    rng = np.random.default_rng(seed)
    lo, hi = world.world_aabb_m()
    t = 0.0
    out = []
    frames = [0] * (len(sessions) if sessions else 0)
    for i in range(count):
        t += rng.exponential(1.0 / rate)
        if rng.uniform() < vp_frac:
            if sessions:
                sid = int(rng.integers(0, len(sessions)))
                s = sessions[sid]
                iw, ih = (max(1, int(np.floor(np.float32(v) * np.float32(s.render_scale) + np.float32(0.5))))
                          for v in (s.w, s.h))
                out.append(SRequest(i, "f", t, w=s.w, h=s.h, n=iw * ih, session=sid, frame=frames[sid]))
                frames[sid] += 1
                continue
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


class _Views:
    """Resident session views under a byte budget (least recently used idle view evicted first)."""

    def __init__(self, renderer, sessions):
        self.r = renderer
        self.sessions = sessions
        self.live = OrderedDict()  # sid -> View
        self.bytes = {}
        self.evictions = 0
        self.created = 0

    def need(self, sid) -> int:
        if sid in self.live:
            return 0
        s = self.sessions[sid]
        return self.r.view_bytes(s.w, s.h, s.render_scale)

    def used(self) -> int:
        return sum(self.bytes.values())

    def make_room(self, nbytes, budget, reserved, busy) -> bool:
        while reserved + self.used() + nbytes > budget:
            idle = [sid for sid in self.live if sid not in busy]
            if not idle:
                return False
            sid = idle[0]
            self.live.pop(sid).close()
            self.bytes.pop(sid)
            self.sessions[sid].frame = 0  # history is gone: the session restarts cold
            self.sessions[sid].prev_vp = None
            self.evictions += 1
        return True

    def get(self, sid):
        if sid not in self.live:
            s = self.sessions[sid]
            self.live[sid] = self.r.view(s.w, s.h, s.render_scale)
            self.bytes[sid] = self.r.view_bytes(s.w, s.h, s.render_scale)
            self.created += 1
        self.live.move_to_end(sid)
        return self.live[sid]

    def close(self):
        for v in self.live.values():
            v.close()
        self.live.clear()
        self.bytes.clear()


def _reupload(renderer, world, resident, rng, count):
    """Re-uploads `count` resident chunks with their own contents: the upload
    traffic of a streaming loader without changing the world, so the uploads
    may overlap the passes in flight (FLAG_UPLOADS_UNORDERED)."""
    picks = rng.choice(len(resident), size=min(count, len(resident)), replace=False)
    ups = []
    for i in picks:
        key = resident[int(i)]
        slot = world.key_to_slot[key]
        base, _ = world.alloc[key]
        data = world.chunk(key)
        # the meta from the slot's bookkeeping (a world built on the device
        # keeps no host meta records)
        ups.append(Upload(slot, world._meta_for(slot, key, base, data), base, data, key=key))
    renderer.apply_chunk_uploads(ups)
    return len(ups)


def _frame_camera(world, sessions, r: SRequest):
    s = sessions[r.session]
    cam = s.camera(world, s.frame, s.prev_vp)
    s.prev_vp = cam.view_proj
    s.frame += 1
    return cam


def device_memory_budget(torch, reserve: int = 4 << 30, device: int = 0) -> int:
    """Admission budget from the device's free memory (cudaMemGetInfo) less a
    reserve for everything the server does not count (the context's lanes
    growing, the allocator's slack)."""
    free, _total = torch.cuda.mem_get_info(device)
    return max(0, int(free) - int(reserve))


def serve(renderer, world: World, requests, torch, mem_budget: int | None, lanes: int = 2, tile=(8, 4), rpt: int = 1,
          max_batch: int = 64, reuploads_per_tick: int = 10, tick_s: float = 0.016, keep_outputs: bool = False,
          mode: int = A.BATCH_PERSISTENT, sessions=None) -> ServeReport:
    if mem_budget is None:
        mem_budget = device_memory_budget(torch, device=renderer.device)
    reqs = sorted(requests, key=lambda r: r.arrival)
    pending = deque(reqs)
    waiting = deque()
    inflight = {}       # lane -> requests
    busy_sessions = set()
    # each lane that renders session frames holds one set of working buffers
    # per view of a launch, each for the largest session
    lane_bytes = max((renderer.view_lane_bytes(s.w, s.h, s.render_scale) for s in sessions or []), default=0)
    per_launch = min(max_batch, A.MAX_VIEWS_PER_LAUNCH, len(sessions or []))
    reserved = lanes * lane_bytes * max(1, per_launch)
    views = _Views(renderer, sessions or [])
    rng = np.random.default_rng(99)
    resident = [k for k in world.slot_to_key if not world.chunk(k).macro_empty]
    batches = uploads = max_inflight = 0
    flags0 = renderer.flags
    renderer.set_flags(flags0 | A.FLAG_UPLOADS_UNORDERED)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    next_tick = 0.0
    try:
        while pending or waiting or inflight:
            now = time.perf_counter() - t0
            while pending and pending[0].arrival <= now:
                waiting.append(pending.popleft())
            if reuploads_per_tick and now >= next_tick and (pending or waiting or inflight):
                uploads += _reupload(renderer, world, resident, rng, reuploads_per_tick)
                next_tick += tick_s
            for lane in list(inflight):
                if renderer.batch_wait(lane, block=False) is None:
                    continue
                done = time.perf_counter() - t0
                for r in inflight.pop(lane):
                    r.done = done
                    reserved -= r.footprint()
                    if r.kind == "f":
                        busy_sessions.discard(r.session)
                        if keep_outputs:
                            r.out = views.get(r.session).read_image(A.IMG_OUTPUT)
                    elif not keep_outputs:
                        r.out = None
                        r.tin = ()
            free = [l for l in range(lanes) if l not in inflight]
            if free and waiting:
                batch, frames, skipped = [], [], deque()
                while waiting and len(batch) + len(frames) < max_batch:
                    r = waiting.popleft()
                    if r.kind == "f":
                        if r.session in busy_sessions or any(f.session == r.session for f in frames):
                            skipped.append(r)  # a session's frames run one at a time, in order
                            continue
                        if not views.make_room(views.need(r.session), mem_budget, reserved,
                                               busy_sessions | {f.session for f in frames}):
                            skipped.append(r)
                            break
                        views.get(r.session)
                        frames.append(r)
                    else:
                        if reserved + views.used() + r.footprint() > mem_budget and (batch or frames or inflight):
                            skipped.append(r)
                            break
                        reserved += r.footprint()
                        batch.append(r)
                waiting.extendleft(reversed(skipped))
                if batch or frames:
                    lane = free[0]
                    if batch:
                        rq = [_to_request(r, torch) for r in batch]
                        torch.cuda.current_stream().synchronize()  # query inputs are on the device
                        renderer.submit_batch_async(lane, rq, tile, rpt, mode)
                    # the admitted frames of every session: each pass launched
                    # once for up to MAX_VIEWS_PER_LAUNCH views
                    renderer.render_views_async(lane, [(views.get(r.session), _frame_camera(world, sessions, r))
                                                       for r in frames])
                    busy_sessions.update(r.session for r in frames)
                    inflight[lane] = batch + frames
                    batches += 1
                    max_inflight = max(max_inflight, len(inflight))
                    continue
            if not (pending and pending[0].arrival <= time.perf_counter() - t0):
                time.sleep(0.0002)
        seconds = time.perf_counter() - t0
    finally:
        views.close()
        renderer.set_flags(flags0)
    lat = [(r.done - r.arrival) * 1e3 for r in reqs]
    extra = ({"views_created": views.created, "view_evictions": views.evictions, "lane_bytes": lane_bytes}
             if sessions else {})
    extra["admission_budget_bytes"] = int(mem_budget)
    return ServeReport(lat, sum(r.rays for r in reqs), seconds, batches, max_inflight, uploads, extra)


def serve_plain(renderer, world: World, requests, torch, keep_outputs: bool = False, sessions=None,
                single_launch_pass: bool = False, reuploads_per_tick: int = 10,
                tick_s: float = 0.016) -> ServeReport:
    """Baseline: FIFO, one request at a time (frames alone on lane 0, batches as
    plain launches), with the same chunk re-upload ticks as `serve` between
    requests.  `single_launch_pass`: frames in the one-kernel-per-pass
    schedule (VXE_FLAG_PRIMARY_MEGAKERNEL: the reference's pass structure)
    instead of the wavefront."""
    reqs = sorted(requests, key=lambda r: r.arrival)
    views = _Views(renderer, sessions or [])
    flags0 = renderer.flags
    flags = flags0 | A.FLAG_UPLOADS_UNORDERED
    if single_launch_pass:
        flags |= A.FLAG_PRIMARY_MEGAKERNEL
    renderer.set_flags(flags)
    rng = np.random.default_rng(99)
    resident = [k for k in world.slot_to_key if not world.chunk(k).macro_empty]
    uploads = 0
    next_tick = 0.0
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    try:
        for r in reqs:
            now = time.perf_counter() - t0
            if r.arrival > now:
                time.sleep(r.arrival - now)
                now = time.perf_counter() - t0
            while reuploads_per_tick and now >= next_tick:
                uploads += _reupload(renderer, world, resident, rng, reuploads_per_tick)
                next_tick += tick_s
            if r.kind == "f":
                v = views.get(r.session)
                v.render_async(0, _frame_camera(world, sessions, r))
                renderer.batch_wait(0, block=True)
                if keep_outputs:
                    r.out = v.read_image(A.IMG_OUTPUT)
            else:
                q = _to_request(r, torch)
                torch.cuda.current_stream().synchronize()
                renderer.submit_batch([q], (8, 4), 1, A.BATCH_PLAIN)
                if not keep_outputs:
                    r.out = None
                    r.tin = ()
            r.done = time.perf_counter() - t0
        seconds = time.perf_counter() - t0
    finally:
        views.close()
        renderer.set_flags(flags0)
    lat = [(r.done - r.arrival) * 1e3 for r in reqs]
    return ServeReport(lat, sum(r.rays for r in reqs), seconds, len(reqs), 1, uploads)
