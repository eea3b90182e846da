"""Render and SDF/normal-query serving over resident scenes with continuous batching.

Semantics follow the reference's inference paths: a render request is `render_full_image`
(scripts/render.py:35-54: RaySampler(64, 64, perturb=False), near/far from the unit sphere,
outputs rgb and depth); a query request is the batched `query_normals` of
`compute_mesh_normals` (geometry/mesh.py:80-114) plus `query_sdf`.

Design:
* SceneStore keeps every scene's parameters resident on the device (grid, hash table, MLP,
  variance, occupancy mask).
* Work is cut into chunks of a few fixed size buckets; each (scene, kind, bucket) has a CUDA
  graph captured once (the bulk graphs share one memory pool: they replay on one stream, one at
  a time), so a chunk costs one graph launch whatever kernels it contains.
* Two lanes. Requests of at most EXPRESS_CHUNKS chunks of the smallest bucket take the express
  lane: a higher-priority stream with its own graphs of the smallest buckets (their own memory
  pool), served first come first served with about EXPRESS_AHEAD_MS of work queued, so their
  kernels run beside the bulk chunks on the device (the block scheduler prefers the higher
  priority) instead of behind them. The other requests take the bulk lane.
* The engine thread admits pending requests while the reserved device memory stays under the
  budget (a fraction of the free HBM measured at start), between every two chunks it queues. It
  keeps about AHEAD_MS of estimated bulk work queued on the compute stream (each bucket's graph
  is timed once at start) and fills it with chunks of the active request with the least
  remaining work, chosen again for every chunk, so a request that arrives behind large ones runs
  after at most that much queued work, while the queue still covers pauses of the engine thread;
  input copies run on a separate copy stream ahead of the compute streams. Results for
  host requests come back through a fixed ring of pinned staging blocks on the copy stream and
  are copied into ordinary host tensors by the engine thread as each block lands (allocating
  pinned memory per request would cost milliseconds and synchronise the device).
* Requests share launches: a bulk chunk that its request cannot fill (its last one) takes the
  next rays of the other active requests of the same scene and kind, through a segment table
  (request, first ray, count, offset in the bucket) applied by the copies into and out of the
  graph's buffers.
* A result is the same alone and in any mix: every ray and point is computed independently,
  with the same kernels and launch shapes, whatever chunk (and whichever neighbours) it falls in.
* Failures stay on the host: malformed requests are rejected at submission, a request larger
  than the budget is rejected, and an exception inside the engine fails the affected requests
  and stops the engine cleanly.
"""

from __future__ import annotations

import collections
import math
import queue
import threading
import time
from dataclasses import dataclass, field
from typing import Dict, List, Optional, Tuple

import torch

from . import ops
from .models import VoxNeuS
from .rendering import RaySampler


class RequestError(RuntimeError):
    pass


@dataclass(eq=False)  # requests compare by identity (the engine removes them from lists)
class Request:
    scene: str
    kind: str  # "render" or "query"
    inputs: Tuple[torch.Tensor, ...]  # render: (rays_o, rays_d) (n,3); query: (points,) (n,3); host or device
    rid: int = -1
    arrival: float = 0.0
    admitted: float = 0.0
    finished: float = 0.0
    n: int = 0
    outputs: Dict[str, torch.Tensor] = field(default_factory=dict)
    error: Optional[str] = None
    done: threading.Event = field(default_factory=threading.Event)
    # engine state
    _dev_in: Tuple[torch.Tensor, ...] = ()
    _dev_out: Dict[str, torch.Tensor] = field(default_factory=dict)
    _next: int = 0
    _reserved: int = 0
    _copy_evt: Optional[torch.cuda.Event] = None
    _out_evt: Optional[torch.cuda.Event] = None
    _pieces_left: int = 0
    _express: bool = False

    @property
    def latency(self) -> float:
        return self.finished - self.arrival

    def wait(self, timeout: Optional[float] = None) -> "Request":
        if not self.done.wait(timeout):
            raise TimeoutError(f"request {self.rid} not finished within {timeout}s")
        if self.error:
            raise RequestError(self.error)
        return self


class SceneStore:
    """Resident scenes keyed by name."""

    def __init__(self, device):
        dev = torch.device(device)
        if dev.type == "cuda" and dev.index is None:
            dev = torch.device("cuda", torch.cuda.current_device())
        self.device = dev
        self.scenes: Dict[str, VoxNeuS] = {}

    def add(self, name: str, model: VoxNeuS) -> None:
        model = model.to(self.device).eval()
        for p in model.parameters():
            p.requires_grad_(False)
        self.scenes[name] = model

    def load_checkpoint(self, name: str, path: str, **model_kw) -> int:
        """Load a checkpoint written by the reference's save_checkpoint (training/checkpoint.py:11-33:
        {"step", "model_state", "grid_res", ...}) into the store; returns its step.

        The grid resolution comes from "grid_res" (else the grid's shape), the hash table's levels,
        features and size, the MLP width and the occupancy resolution from the state_dict's shapes
        (the reference's load_checkpoint rescales a model built at another resolution,
        :48-54; here the model is built at the saved one). Only tensors and plain containers are
        unpickled (weights_only). model_kw overrides the inferred constructor arguments."""
        ck = torch.load(path, map_location="cpu", weights_only=True)
        sd = ck["model_state"]
        emb = sd["radiance_hash.encoder.embeddings"]
        res = ck.get("grid_res") or list(sd["sdf_grid.grid"].shape[-3:])
        kw = dict(grid_res=[int(r) for r in res], hash_n_levels=int(emb.shape[0]), hash_n_features=int(emb.shape[2]),
                  hash_log2_size=int(emb.shape[1]).bit_length() - 1,
                  mlp_hidden_dim=int(sd["radiance_mlp.net.0.weight"].shape[0]),
                  occupancy_res=int(sd["occupancy_grid.occupancy_mask"].shape[0]))
        kw.update(model_kw)
        m = VoxNeuS(**kw)
        m.load_state_dict(sd)
        self.add(name, m)
        return int(ck.get("step", 0))

    def bytes(self) -> int:
        return sum(sum(t.numel() * t.element_size() for t in m.state_dict().values()) for m in self.scenes.values())


class _GraphBucket:
    """A captured render or query pipeline for one scene and one chunk size."""

    def __init__(self, model: VoxNeuS, kind: str, size: int, sampler: RaySampler, pool, stream):
        self.kind, self.size = kind, size
        dev = model.sdf_grid.grid.device
        if kind == "render":
            self.inp = (torch.zeros(size, 3, device=dev), torch.zeros(size, 3, device=dev))
            self.inp[0][:, 2] = 3.0
            self.inp[1][:, 2] = -1.0
        else:
            self.inp = (torch.zeros(size, 3, device=dev),)
        self.model, self.sampler = model, sampler
        with torch.cuda.stream(stream), torch.no_grad():
            self._run()  # warm caches (tables, scratch) outside capture
            stream.synchronize()
            self.graph = torch.cuda.CUDAGraph()
            with torch.cuda.graph(self.graph, pool=pool, stream=stream):
                self.out = self._run()

    def _run(self):
        m = self.model
        if self.kind == "render":
            out = m.render(self.inp[0], self.inp[1], self.sampler, None, None, extras=False)
            return {"rgb": out["rgb"], "depth": out["depth"]}
        lo, hi = m.sdf_grid.bounds()
        sdf, _, nrm, _, _ = ops.field_query(m.sdf_grid.grid, lo, hi, self.inp[0], sdf=True, normal=True)
        return {"sdf": sdf.unsqueeze(-1), "normal": nrm}


class ServingEngine:
    RENDER_BUCKETS = (4096, 16384, 65536)
    QUERY_BUCKETS = (65536, 262144, 1048576)
    STAGE_BYTES = 16 << 20  # pinned staging block
    STAGE_BLOCKS = 8
    AHEAD_MS = 20.0  # estimated device time kept queued on the compute stream
    EXPRESS_CHUNKS = 2  # requests of at most this many smallest-bucket chunks take the express lane
    EXPRESS_AHEAD_MS = 2.0  # estimated device time kept queued on the express stream

    def __init__(self, store: SceneStore, memory_fraction: float = 0.5, n_samples: int = 64,
                 n_importance: int = 64, budget_bytes: Optional[int] = None, fault_injector=None,
                 render_buckets: Optional[Tuple[int, ...]] = None, query_buckets: Optional[Tuple[int, ...]] = None,
                 tc_wait_polls: Optional[int] = None, express: bool = True):
        if render_buckets:
            self.RENDER_BUCKETS = tuple(sorted(render_buckets))
        if query_buckets:
            self.QUERY_BUCKETS = tuple(sorted(query_buckets))
        self.store = store
        self.device = store.device
        self.sampler = RaySampler(n_samples, n_importance, perturb=False)
        self.compute = torch.cuda.Stream(self.device)
        self.copy = torch.cuda.Stream(self.device)
        self.pool = torch.cuda.graph_pool_handle()
        self.graphs: Dict[Tuple[str, str, int], _GraphBucket] = {}
        # the express lane: a higher-priority stream whose own graphs (smallest buckets, their own
        # memory pool) let small requests run beside the bulk chunks instead of behind them
        self.express = torch.cuda.Stream(self.device, priority=torch.cuda.Stream.priority_range()[1]) \
            if express else None
        self.xpool = torch.cuda.graph_pool_handle() if express else None
        self.xgraphs: Dict[Tuple[str, str, int], _GraphBucket] = {}
        # blocks of the MLP kernels that gave up waiting on the tensor core (every graph is captured
        # with this status word); a request whose completion sees it nonzero stops the engine
        self.tc_status = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._status_host = torch.zeros(4096, dtype=torch.int32).pin_memory()
        with ops.tc_guard(self.tc_status, tc_wait_polls):
            for name, m in store.scenes.items():
                for size in self.RENDER_BUCKETS:
                    self.graphs[(name, "render", size)] = _GraphBucket(m, "render", size, self.sampler, self.pool,
                                                                       self.compute)
                for size in self.QUERY_BUCKETS:
                    self.graphs[(name, "query", size)] = _GraphBucket(m, "query", size, self.sampler, self.pool,
                                                                      self.compute)
                if self.express is not None:
                    for kind, size in (("render", self.RENDER_BUCKETS[0]), ("query", self.QUERY_BUCKETS[0])):
                        self.xgraphs[(name, kind, size)] = _GraphBucket(m, kind, size, self.sampler, self.xpool,
                                                                        self.express)
        # one replay of every graph before serving: the first launch of a graph uploads it to the
        # device, which would otherwise stall the engine thread on the first request of each scene
        for graphs, stream in ((self.graphs, self.compute), (self.xgraphs, self.express)):
            if graphs:
                with torch.cuda.stream(stream):
                    for gb in graphs.values():
                        gb.graph.replay()
        torch.cuda.synchronize(self.device)
        # device time of one replay of each bucket (the first scene's graphs stand for all scenes)
        self._cost_ms: Dict[Tuple[str, int], float] = {}
        first = next(iter(store.scenes))
        with torch.cuda.stream(self.compute):
            for (name, kind, size), gb in self.graphs.items():
                if name != first:
                    continue
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                gb.graph.replay()
                e0.record(self.compute)
                gb.graph.replay()
                e1.record(self.compute)
                e1.synchronize()
                self._cost_ms[(kind, size)] = max(e0.elapsed_time(e1), 1e-3)
        if budget_bytes is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            budget_bytes = int(free * memory_fraction)
        self.budget = budget_bytes
        self.reserved = 0
        self.pending: "queue.Queue[Request]" = queue.Queue()
        self.waiting: List[Request] = []
        self.active: List[Request] = []
        self._inflight: List[Tuple[torch.cuda.Event, Request]] = []
        # device -> host results go through a fixed ring of pinned staging blocks (allocating pinned
        # memory per request is slow and synchronising); the engine thread copies each landed block
        # into the request's ordinary host tensor
        self._stage = [torch.empty(self.STAGE_BYTES, dtype=torch.uint8, pin_memory=True)
                       for _ in range(self.STAGE_BLOCKS)]
        self._free_stage: List[int] = list(range(self.STAGE_BLOCKS))
        self._pieces: "collections.deque" = collections.deque()  # (req, src flat view, dst flat view)
        self._pieces_inflight: List[Tuple[torch.cuda.Event, int, Request, torch.Tensor, int]] = []
        self._ahead: "collections.deque" = collections.deque()  # (completion event, cost ms) of queued chunks
        self._ahead_ms = 0.0
        self._xahead: "collections.deque" = collections.deque()  # the same for the express stream
        self._xahead_ms = 0.0
        self.packed_launches = 0  # bulk launches that carried rays of more than one request
        self._rid = 0
        self._stop = threading.Event()
        self._failed: Optional[str] = None
        self._fault = fault_injector
        self._thread = threading.Thread(target=self._loop, name="voxneus-serving", daemon=True)
        self._thread.start()

    # ---------------------------------------------------------------- submission

    @staticmethod
    def _bytes_for(kind: str, n: int) -> int:
        return n * 4 * (6 + 4) if kind == "render" else n * 4 * (3 + 4)

    def submit(self, req: Request) -> Request:
        if self._failed:
            raise RequestError(f"engine stopped: {self._failed}")
        if req.scene not in self.store.scenes:
            raise RequestError(f"unknown scene {req.scene!r}")
        if req.kind not in ("render", "query"):
            raise RequestError(f"unknown request kind {req.kind!r}")
        want = 2 if req.kind == "render" else 1
        if len(req.inputs) != want:
            raise RequestError(f"{req.kind} needs {want} input tensor(s)")
        n = req.inputs[0].shape[0]
        for t in req.inputs:
            if t.dim() != 2 or t.shape[1] != 3 or t.shape[0] != n or t.dtype != torch.float32:
                raise RequestError("inputs must be float32 (n, 3) tensors of equal length")
            # one float64 reduction: finite iff every element is (float32 magnitudes cannot overflow it)
            if not math.isfinite(float(t.sum(dtype=torch.float64))):
                raise RequestError("inputs contain NaN or Inf")
        if n == 0:
            raise RequestError("empty request")
        if self._bytes_for(req.kind, n) > self.budget:
            raise RequestError(f"request needs {self._bytes_for(req.kind, n)} bytes, budget is {self.budget}")
        req.n = n
        req.rid = self._rid
        self._rid += 1
        req.arrival = req.arrival or time.perf_counter()
        self.pending.put(req)
        return req

    # ---------------------------------------------------------------- engine loop

    def _admit(self):
        while True:
            try:
                self.waiting.append(self.pending.get_nowait())
            except queue.Empty:
                break
        still = []
        for req in self.waiting:
            need = self._bytes_for(req.kind, req.n)
            if self.reserved + need > self.budget:
                still.append(req)
                continue
            self.reserved += need
            req._reserved = need
            req.admitted = time.perf_counter()
            smallest = self.RENDER_BUCKETS[0] if req.kind == "render" else self.QUERY_BUCKETS[0]
            req._express = self.express is not None and req.n <= self.EXPRESS_CHUNKS * smallest
            with torch.cuda.stream(self.copy):
                req._dev_in = tuple(t.to(self.device, non_blocking=True) for t in req.inputs)
                if req.kind == "render":
                    req._dev_out = {"rgb": torch.empty(req.n, 3, device=self.device),
                                    "depth": torch.empty(req.n, 1, device=self.device)}
                else:
                    req._dev_out = {"sdf": torch.empty(req.n, 1, device=self.device),
                                    "normal": torch.empty(req.n, 3, device=self.device)}
                req._copy_evt = torch.cuda.Event()
                req._copy_evt.record(self.copy)
            self.active.append(req)
        self.waiting = still

    def _bucket(self, kind: str, remaining: int) -> int:
        buckets = self.RENDER_BUCKETS if kind == "render" else self.QUERY_BUCKETS
        for b in buckets:
            if remaining <= b:
                return b
        return buckets[-1]

    def _run_chunk(self, req: Request) -> List[Request]:
        """Queue one bucket launch for req's next rays (or points). A bulk chunk that req cannot fill
        takes the next rays of other active requests of the same scene and kind, in admission order
        (a segment table: request, first ray, count, offset in the bucket). Returns the requests of
        the launch."""
        if req._express:
            size = self.RENDER_BUCKETS[0] if req.kind == "render" else self.QUERY_BUCKETS[0]
            gb = self.xgraphs[(req.scene, req.kind, size)]
            s = self.express
        else:
            size = self._bucket(req.kind, req.n - req._next)
            gb = self.graphs[(req.scene, req.kind, size)]
            s = self.compute
        segs = [(req, req._next, min(size, req.n - req._next), 0)]
        room = size - segs[0][2]
        if room > 0 and not req._express:
            for other in self.active:
                if room == 0:
                    break
                if other is req or other._express or other.scene != req.scene or other.kind != req.kind:
                    continue
                take = min(room, other.n - other._next)
                if take > 0:
                    segs.append((other, other._next, take, size - room))
                    room -= take
        if len(segs) > 1:
            self.packed_launches += 1
        for r, _, _, _ in segs:
            s.wait_event(r._copy_evt)
        with torch.cuda.stream(s):
            for a, dst in enumerate(gb.inp):
                for r, start, cnt, off in segs:
                    dst[off:off + cnt].copy_(r._dev_in[a][start:start + cnt])
                if room > 0:  # pad with the last ray of the launch
                    r, start, cnt, off = segs[-1]
                    dst[size - room:].copy_(r._dev_in[a][start + cnt - 1:start + cnt].expand(room, 3))
            gb.graph.replay()
            for k, v in gb.out.items():
                for r, start, cnt, off in segs:
                    r._dev_out[k][start:start + cnt].copy_(v[off:off + cnt])
            evt = torch.cuda.Event()
            evt.record(s)
        cost = self._cost_ms[(req.kind, size)]
        if req._express:
            self._xahead.append((evt, cost))
            self._xahead_ms += cost
        else:
            self._ahead.append((evt, cost))
            self._ahead_ms += cost
        for r, start, cnt, _ in segs:
            r._next = start + cnt
        return [r for r, _, _, _ in segs]

    def _room(self) -> bool:
        """Less than AHEAD_MS of estimated work still queued on the compute stream."""
        while self._ahead and self._ahead[0][0].query():
            self._ahead_ms -= self._ahead.popleft()[1]
        return self._ahead_ms < self.AHEAD_MS

    def _xroom(self) -> bool:
        """Less than EXPRESS_AHEAD_MS of estimated work still queued on the express stream."""
        while self._xahead and self._xahead[0][0].query():
            self._xahead_ms -= self._xahead.popleft()[1]
        return self._xahead_ms < self.EXPRESS_AHEAD_MS

    def _remaining(self, req: Request) -> float:
        size = self._bucket(req.kind, req.n - req._next)
        return (req.n - req._next) / size * self._cost_ms[(req.kind, size)]

    def _finish(self, req: Request):
        """All chunks of req are queued on its stream: queue its results for the host."""
        s = self.express if req._express else self.compute
        with torch.cuda.stream(s):  # the status word as of the request's last chunk
            k = req.rid % self._status_host.numel()
            self._status_host[k:k + 1].copy_(self.tc_status, non_blocking=True)
        evt = torch.cuda.Event()
        evt.record(s)
        if req.inputs[0].device.type != "cpu":
            req.outputs = dict(req._dev_out)
            self._inflight.append((evt, req))
            return
        req._out_evt = evt
        req.outputs = {}
        req._pieces_left = 0
        for k, v in req._dev_out.items():
            h = torch.empty(v.shape, dtype=v.dtype)
            req.outputs[k] = h
            src, dst = v.reshape(-1).view(torch.uint8), h.reshape(-1).view(torch.uint8)
            for a in range(0, src.numel(), self.STAGE_BYTES):
                b = min(a + self.STAGE_BYTES, src.numel())
                self._pieces.append((req, src[a:b], dst[a:b]))
                req._pieces_left += 1
        self._issue_pieces()

    def _issue_pieces(self):
        while self._pieces and self._free_stage:
            req, src, dst = self._pieces.popleft()
            i = self._free_stage.pop()
            n = src.numel()
            with torch.cuda.stream(self.copy):
                self.copy.wait_event(req._out_evt)
                self._stage[i][:n].copy_(src, non_blocking=True)
                evt = torch.cuda.Event()
                evt.record(self.copy)
            self._pieces_inflight.append((evt, i, req, dst, n))

    def _complete(self, req: Request):
        bad = int(self._status_host[req.rid % self._status_host.numel()])
        if bad:  # raised into the loop's handler: every pending request fails and the engine stops
            raise RuntimeError(f"{bad} block(s) of the MLP kernels gave up waiting on the tensor core")
        req.finished = time.perf_counter()
        self.reserved -= req._reserved
        req._dev_in, req._dev_out = (), {}
        req.done.set()

    def _poll(self):
        keep = []
        for evt, req in self._inflight:
            if evt.query():
                self._complete(req)
            else:
                keep.append((evt, req))
        self._inflight = keep
        keep_p = []
        for evt, i, req, dst, n in self._pieces_inflight:
            if evt.query():
                dst.copy_(self._stage[i][:n])
                self._free_stage.append(i)
                req._pieces_left -= 1
                if req._pieces_left == 0:
                    self._complete(req)
            else:
                keep_p.append((evt, i, req, dst, n))
        self._pieces_inflight = keep_p
        self._issue_pieces()

    def _step(self, req: Request) -> None:
        """Queue the next chunk of req; hand every request of the launch that it completed to the
        output path."""
        if self._fault is not None:
            self._fault(req)
        for r in self._run_chunk(req):
            if r._next >= r.n:
                self.active.remove(r)
                self._finish(r)

    def _busy(self) -> bool:
        return bool(self.active or self._inflight or self._pieces or self._pieces_inflight)

    def _loop(self):
        try:
            torch.cuda.set_device(self.device)
            while not self._stop.is_set():
                self._admit()
                self._poll()
                progressed = False
                # small requests first, on the express stream (FIFO), while it has room
                while self._xroom():
                    req = next((r for r in self.active if r._express), None)
                    if req is None:
                        break
                    progressed = True
                    self._step(req)
                    self._admit()
                    self._poll()
                # then the bulk lane: least remaining work first, re-chosen after every chunk so a
                # request admitted meanwhile competes for the next one
                while self._room():
                    bulk = [r for r in self.active if not r._express]
                    if not bulk:
                        break
                    progressed = True
                    self._step(min(bulk, key=self._remaining))
                    self._admit()
                    self._poll()
                    if any(r._express for r in self.active) and self._xroom():
                        break
                if not progressed:
                    time.sleep(0.0002)
        except Exception as e:  # host-side failure: fail every request and stop
            self._failed = f"{type(e).__name__}: {e}"
            in_copy = [p[0] for p in self._pieces] + [p[2] for p in self._pieces_inflight]
            for req in self.active + self.waiting + [r for _, r in self._inflight] + in_copy:
                req.error = self._failed
                req.done.set()
            while True:
                try:
                    r = self.pending.get_nowait()
                    r.error = self._failed
                    r.done.set()
                except queue.Empty:
                    break

    def close(self):
        self._stop.set()
        self._thread.join(timeout=30)
        torch.cuda.synchronize(self.device)

    @property
    def failed(self) -> Optional[str]:
        return self._failed


def latency_stats(reqs: List[Request]) -> Dict[str, float]:
    lat = sorted(r.latency * 1e3 for r in reqs if not r.error)
    if not lat:
        return {}

    def pct(p):
        return lat[min(len(lat) - 1, max(0, int(math.ceil(p / 100.0 * len(lat))) - 1))]

    wait = [(r.admitted - r.arrival) * 1e3 for r in reqs if not r.error]
    return {"p50_ms": pct(50), "p99_ms": pct(99), "mean_ms": sum(lat) / len(lat), "n": len(lat),
            "admission_wait_share": sum(wait) / max(sum(lat), 1e-9)}
