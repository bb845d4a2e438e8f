"""Continuous-batching request loop for SPEEDY physics tendency and VJP requests.

A request names 1..n members (grid instances, each a key into a member source) and asks either
for their tendencies (``SpeedyPhysics.compute_tendencies``, jcm/physics/speedy/
speedy_physics.py:88-127) or for the VJP of those tendencies (``jax.vjp`` of the same function)
under a cotangent the request seeds.  The reference has no serving layer; this module is the
layer a forecast service would put in front of the physics:

* Admission by free HBM.  Every device byte the loop holds (resident member state, result and
  cotangent buffers, the adjoint's scratch) is counted against ``budget_bytes``, and a request
  must also fit the device memory the backend can still hand out (its pool's free bytes, plus
  the driver's free memory when the pool would have to grow).  A request is admitted, in arrival order,
  when its new members and its result buffers fit; idle resident members are evicted
  least-recently-used to make room.  A request that can never fit is
  rejected; a failed device allocation leaves the request waiting and is counted.
* Device-resident column state.  A member's state, forcing and geometry are uploaded once, as
  one packed buffer from pinned host memory on a copy stream, and stay on the device while any
  request uses them (and afterwards, until evicted).
* Continuous batching.  Requests admitted while earlier batches run are merged into the next
  batch of their kind: one ragged-ensemble launch over all their members
  (``spd_ensemble_fwd`` for tendencies, ``spd_ensemble_vjp`` for VJPs), enqueued while up to
  ``max_inflight`` earlier batches of that kind are still on the device.  VJP batches run on
  their own stream, so their work overlaps the tendency batches on the device, and uploads
  overlap both; the tendency stream has the higher priority.
* Latency.  Completion times are device timestamps (CUDA events) mapped onto the host clock on
  which arrivals are stamped; p50/p99 latency and columns/s are reported per run.

``mode="plain"`` is the per-request drop-in on the same GPU: one request at a time in arrival
order, every member through ``spd_fwd`` (or ``spd_vjp``) on one stream.  A VJP request's
cotangents are N(0, 1) drawn once over its contiguous cotangent buffer from a generator seeded
by the request, in either mode.

The scheduler (``Scheduler``) is independent of the device; ``CudaBackend`` performs the device
work through the C ABI.  Failures a caller can cause are handled on the host: malformed
requests and requests larger than the budget are rejected at submission, allocation failures
are retried, and ``cancel`` drops a waiting request or discards an in-flight one's results.
"""
from __future__ import annotations

import collections
import ctypes as C
import gc
import resource
import time
from dataclasses import dataclass, field
from typing import Callable, Dict, Hashable, List, Optional

import numpy as np

from . import _lib

TENDENCY = "tendency"
VJP = "vjp"
KINDS = (TENDENCY, VJP)

_ALIGN = 256

# Instance attribute of each ABI input field (synthetic.Instance naming).
_INSTANCE_FIELDS = dict(u_wind="u", v_wind="v", temperature="t", specific_humidity="q",
                        geopotential="phi", normalized_surface_pressure="psa", alb0="alb0",
                        sice_am="sice", snowc_am="snowc", soilw_am="soilw", stl_am="stl",
                        sea_surface_temperature="sst", fmask="fmask", orog="orog",
                        phis0="phis0", sia="sia", coa="coa")
_LEVEL_FIELDS = ("u_wind", "v_wind", "temperature", "specific_humidity", "geopotential")
_LAT_FIELDS = ("sia", "coa")


def _round_up(n, a=_ALIGN):
    return (n + a - 1) // a * a


def member_layout(kx, ix, il):
    """Byte offsets of the 17 input fields in a member's packed buffer, and its size."""
    c = ix * il
    off, pos = {}, 0
    for name in _lib.INPUT_FIELDS:
        n = kx * c if name in _LEVEL_FIELDS else (il if name in _LAT_FIELDS else c)
        off[name] = (pos, n)
        pos = _round_up(pos + 4 * n)
    return off, pos


def tendency_result_floats(kx, ix, il):
    """Floats of one member's tendency result: four tendency planes and two precipitation
    fields."""
    return (4 * kx + 2) * ix * il


def vjp_result_floats(kx, ix, il):
    """Floats of one member's VJP result and cotangent: gradients of u, v, T, q, phi and psa,
    the 12 parameter gradients, and the four cotangent planes."""
    return (5 * kx + 1) * ix * il + 12 + 4 * kx * ix * il


@dataclass
class HostMember:
    """One member's inputs packed in one host buffer (pinned when torch can pin), in the
    layout of ``member_layout``."""
    kx: int
    ix: int
    il: int
    lfluxland: bool
    buffer: object          # torch uint8 tensor (CPU)
    nbytes: int

    @property
    def columns(self):
        return self.ix * self.il

    @classmethod
    def from_instance(cls, inst, pin=True):
        import torch
        off, nbytes = member_layout(inst.kx, inst.ix, inst.il)
        buf = torch.zeros(nbytes, dtype=torch.uint8, pin_memory=pin and torch.cuda.is_available())
        flat = buf.view(torch.float32) if nbytes % 4 == 0 else None
        for name, (pos, n) in off.items():
            a = np.ascontiguousarray(getattr(inst, _INSTANCE_FIELDS[name]), np.float32).ravel()
            if a.size != n:
                raise ValueError(f"field {name}: {a.size} values, expected {n}")
            flat[pos // 4: pos // 4 + n] = torch.from_numpy(a)
        return cls(inst.kx, inst.ix, inst.il, bool(inst.lfluxland), buf, nbytes)


@dataclass
class Request:
    """A tendency or VJP request over ``members`` (keys of the member source)."""
    kind: str
    members: List[Hashable]
    arrival: float = 0.0              # seconds after the stream's start
    seed: int = 0                     # cotangent seed (VJP)
    rid: int = -1
    status: str = "new"               # new, waiting, admitted, running, done, rejected, cancelled
    reason: str = ""
    columns: int = 0
    t_submit: float = float("nan")
    t_admit: float = float("nan")
    t_launch: float = float("nan")
    t_done: float = float("nan")
    result: Optional[list] = None     # per member: dict of device tensors (valid in on_complete)
    _shapes: list = field(default_factory=list, repr=False)
    _outputs: object = field(default=None, repr=False)
    _out_bytes: int = 0
    _out_handle: object = field(default=None, repr=False)
    _views: object = field(default=None, repr=False)
    _ct: object = field(default=None, repr=False)
    _base: int = 0

    @property
    def latency(self):
        return self.t_done - self.arrival


@dataclass
class _Resident:
    key: Hashable
    host: HostMember
    dev: object = None
    refs: int = 0
    last_use: int = 0


@dataclass
class WorkItem:
    kind: str
    requests: List[Request]
    handle: object = None
    interval: tuple = (float("nan"), float("nan"))   # device (start, end) on the loop's clock


class Scheduler:
    """Admission, residency, batching and completion; the device work goes to ``backend``.

    ``backend`` provides: ``member_bytes(host)``, ``output_bytes(kind, host)``,
    ``fixed_bytes()``, ``now()``, ``upload(host)`` -> device member, ``release(dev)``,
    ``alloc_outputs(request, hosts)`` (raises MemoryError when the device refuses),
    ``free_outputs(request)``, ``launch(kind, requests, devs)`` -> handle,
    ``done(handle)``, ``completion_time(handle)``, ``device_interval(handle)``,
    ``retire(handle)``, ``results(request)``, ``start_clock()``, ``synchronize()``.

    ``freeze_gc`` (default on) keeps the garbage collector's full collections off the loop
    during ``run``; a caller that drives ``step`` itself can do the same with ``gc.freeze``.

    ``slow_passes`` (filled by ``run``): every pass of the loop that took longer than
    ``slow_pass_ms`` of wall time, with the time spent in submission, ``poll``, ``admit`` and
    ``launch``, the loop thread's CPU time over the pass and its voluntary and involuntary
    context switches (a pass whose CPU time is far below its wall time, with involuntary
    switches, was descheduled by the operating system; one with voluntary switches waited in
    a blocking call).
    """

    def __init__(self, backend, source: Callable[[Hashable], HostMember], budget_bytes: int,
                 mode: str = "batched", max_inflight: int = 2, max_batch_columns: int = 1 << 24,
                 on_complete: Optional[Callable[[Request], None]] = None,
                 max_admit_per_step: int = 8, freeze_gc: bool = True,
                 slow_pass_ms: float = 5.0):
        if mode not in ("batched", "plain"):
            raise ValueError("mode is 'batched' or 'plain'")
        self.b = backend
        self.source = source
        self.budget = int(budget_bytes)
        self.mode = mode
        self.max_inflight = max_inflight
        self.max_batch_columns = max_batch_columns
        self.on_complete = on_complete
        self.max_admit_per_step = max_admit_per_step
        self.freeze_gc = freeze_gc
        self.used = self.b.fixed_bytes()
        if self.used > self.budget:
            raise ValueError(f"budget {self.budget} below the fixed device bytes {self.used}")
        self.peak = self.used
        self.resident: Dict[Hashable, _Resident] = {}
        self.hosts: Dict[Hashable, HostMember] = {}
        self.waiting = collections.deque()
        self.admitted = {TENDENCY: collections.deque(), VJP: collections.deque()}
        self.inflight: List[WorkItem] = []
        self.items: List[WorkItem] = []
        self.finished: List[Request] = []
        self.cancelled = set()
        self._rid = 0
        self._tick = 0
        self.stats = collections.Counter()
        self.slow_pass_ms = float(slow_pass_ms)
        self.slow_passes: List[dict] = []
        self._phase = (0.0, 0.0, 0.0)

    # -- submission -----------------------------------------------------------------------------
    def _host(self, key):
        h = self.hosts.get(key)
        if h is None:
            h = self.source(key)
            self.hosts[key] = h
        return h

    def submit(self, req: Request) -> Request:
        req.rid = self._rid
        self._rid += 1
        req.t_submit = self.b.now()
        try:
            if req.kind not in KINDS:
                raise ValueError(f"unknown request kind {req.kind!r}")
            if not req.members:
                raise ValueError("request names no members")
            hosts = [self._host(k) for k in req.members]
        except Exception as e:  # malformed request: unknown member, bad kind, bad data
            return self._reject(req, f"malformed: {e}")
        req._shapes = [(h.kx, h.ix, h.il) for h in hosts]
        req.columns = sum(h.columns for h in hosts)
        req._out_bytes = sum(self.b.output_bytes(req.kind, h) for h in hosts)
        distinct = {k: self.hosts[k] for k in req.members}
        need = req._out_bytes + sum(self.b.member_bytes(h) for h in distinct.values())
        if self.b.fixed_bytes() + need > self.budget:
            return self._reject(req, f"needs {need} bytes, budget {self.budget}")
        req.status = "waiting"
        self.waiting.append(req)
        return req

    def _reject(self, req, why):
        req.status, req.reason = "rejected", why
        self.stats["rejected"] += 1
        self.finished.append(req)
        return req

    def cancel(self, rid) -> bool:
        for r in list(self.waiting):
            if r.rid == rid:
                self.waiting.remove(r)
                r.status = "cancelled"
                self.finished.append(r)
                self.stats["cancelled"] += 1
                return True
        for q in self.admitted.values():
            for r in list(q):
                if r.rid == rid:
                    q.remove(r)
                    self._unpin(r)
                    self.b.free_outputs(r)
                    self.used -= r._out_bytes
                    r.status = "cancelled"
                    self.finished.append(r)
                    self.stats["cancelled"] += 1
                    return True
        for it in self.inflight:
            for r in it.requests:
                if r.rid == rid and r.status == "running":
                    self.cancelled.add(rid)
                    return True
        return False

    # -- residency and admission ----------------------------------------------------------------
    def _fits(self, nbytes):
        """Within the budget, and within the device memory the backend can still hand out
        (free HBM: its pool's free bytes plus what the driver reports free), when the backend
        measures it."""
        if self.budget - self.used < nbytes:
            return False
        avail = getattr(self.b, "available_bytes", None)
        return avail is None or avail(nbytes) >= nbytes

    def _evict_for(self, nbytes, keep):
        idle = sorted((r for r in self.resident.values() if r.refs == 0 and r.key not in keep),
                      key=lambda r: r.last_use)
        for r in idle:
            if self._fits(nbytes):
                break
            self.b.release(r.dev)
            self.used -= self.b.member_bytes(r.host)
            del self.resident[r.key]
            self.stats["evictions"] += 1
        return self._fits(nbytes)

    def _admit_one(self, req) -> bool:
        keys = list(dict.fromkeys(req.members))
        new = [k for k in keys if k not in self.resident]
        need = req._out_bytes + sum(self.b.member_bytes(self.hosts[k]) for k in new)
        if not self._evict_for(need, set(keys)):
            return False
        try:
            self.b.alloc_outputs(req, [self.hosts[k] for k in req.members])
        except MemoryError:
            self.stats["alloc_failures"] += 1
            return False
        self.used += req._out_bytes
        for k in new:
            h = self.hosts[k]
            try:
                dev = self.b.upload(h)
            except MemoryError:
                self.stats["alloc_failures"] += 1
                self.b.free_outputs(req)
                self.used -= req._out_bytes
                return False
            self.resident[k] = _Resident(k, h, dev)
            self.used += self.b.member_bytes(h)
            self.stats["uploads"] += 1
            self.stats["upload_bytes"] += h.nbytes
        self._tick += 1
        for k in req.members:
            r = self.resident[k]
            r.refs += 1
            r.last_use = self._tick
        self.peak = max(self.peak, self.used)
        req.status = "admitted"
        req.t_admit = self.b.now()
        self.admitted[req.kind].append(req)
        return True

    def _unpin(self, req):
        for k in req.members:
            r = self.resident.get(k)
            if r is not None:
                r.refs -= 1

    def admit(self):
        """Admits waiting requests in arrival order while they fit, at most
        ``max_admit_per_step`` per call so that launches interleave with a large burst."""
        n = 0
        while (self.waiting and n < self.max_admit_per_step and
               self._admit_one(self.waiting[0])):
            self.waiting.popleft()
            n += 1
        return n

    def prefetch(self, keys):
        """Makes the members ``keys`` resident ahead of traffic (as far as the budget allows,
        evicting idle members least-recently-used) and waits for the uploads.  Returns the
        number uploaded."""
        n = 0
        for k in dict.fromkeys(keys):
            if k in self.resident:
                continue
            h = self._host(k)
            if not self._evict_for(self.b.member_bytes(h), {k}):
                break
            self.resident[k] = _Resident(k, h, self.b.upload(h))
            self.used += self.b.member_bytes(h)
            self.peak = max(self.peak, self.used)
            self.stats["prefetched"] += 1
            n += 1
        self.b.synchronize()
        return n

    # -- launching ------------------------------------------------------------------------------
    def _inflight_of(self, kind):
        return sum(1 for it in self.inflight if it.kind == kind)

    def _launch(self, kind, reqs):
        devs = [[self.resident[k].dev for k in r.members] for r in reqs]
        handle = self.b.launch(kind, reqs, devs)
        t = self.b.now()
        for r in reqs:
            r.status, r.t_launch = "running", t
        self.inflight.append(WorkItem(kind, reqs, handle))
        self.stats[f"launches_{kind}"] += 1

    def launch(self):
        n = 0
        if self.mode == "plain":
            if self.inflight:
                return 0
            # one request at a time, in admission (= arrival) order across both kinds
            cands = [q[0] for q in self.admitted.values() if q]
            if cands:
                r = min(cands, key=lambda x: x.rid)
                self.admitted[r.kind].popleft()
                self._launch(r.kind, [r])
                n += 1
            return n
        # continuous batching: everything admitted of one kind (up to max_batch_columns)
        # becomes one batched launch while fewer than max_inflight of that kind are on the GPU
        for kind in KINDS:
            q = self.admitted[kind]
            while q and self._inflight_of(kind) < self.max_inflight:
                batch, cols = [], 0
                while q and (not batch or cols + q[0].columns <= self.max_batch_columns):
                    r = q.popleft()
                    batch.append(r)
                    cols += r.columns
                self._launch(kind, batch)
                n += 1
        return n

    # -- completion -----------------------------------------------------------------------------
    def poll(self):
        n = 0
        for it in list(self.inflight):
            if not self.b.done(it.handle):
                continue
            t = self.b.completion_time(it.handle)
            it.interval = self.b.device_interval(it.handle)
            self.inflight.remove(it)
            self.items.append(it)
            for r in it.requests:
                r.t_done = t
                if r.rid in self.cancelled:
                    r.status = "cancelled"
                    self.stats["cancelled"] += 1
                else:
                    r.status = "done"
                    if self.on_complete is not None:
                        r.result = self.b.results(r)
                        self.on_complete(r)
                        r.result = None
                self._unpin(r)
                self.b.free_outputs(r)
                self.used -= r._out_bytes
                self.finished.append(r)
                n += 1
            self.b.retire(it.handle)
        return n

    def busy(self):
        return bool(self.waiting or self.inflight or any(self.admitted.values()))

    def step(self):
        """One pass of the loop: retire, admit, launch.  Returns the amount of work done."""
        t0 = time.perf_counter()
        a = self.poll()
        t1 = time.perf_counter()
        b = self.admit()
        t2 = time.perf_counter()
        c = self.launch()
        self._phase = (t1 - t0, t2 - t1, time.perf_counter() - t2)
        return a + b + c

    def run(self, requests: List[Request], timeout_s: float = 600.0):
        """Serve ``requests`` (their ``arrival`` times in seconds after the start) in real time
        and return the finished requests.

        With ``freeze_gc`` the objects alive when the run starts are moved out of the garbage
        collector's generations (``gc.freeze``) until it ends.  A full collection scans every
        tracked object of the process and stops this loop meanwhile: in a process holding
        ~190 k objects one took 36 ms, and the requests arriving during it waited that long
        to be submitted.  Frozen, a collection scans only the loop's own young objects.  The
        end of the run unfreezes every frozen object, including any frozen before it (they
        are then scanned by full collections again, as unfrozen objects are)."""
        pending = collections.deque(sorted(requests, key=lambda r: r.arrival))
        if self.freeze_gc:
            gc.collect()
            gc.freeze()
        try:
            self.b.start_clock()
            t_end = time.perf_counter() + timeout_s
            wall, cpu, sw = time.perf_counter(), time.thread_time(), _switches()
            while pending or self.busy():
                now = self.b.now()
                while pending and pending[0].arrival <= now:
                    self.submit(pending.popleft())
                t_sub = time.perf_counter()
                idle = self.step() == 0
                w1 = time.perf_counter()
                if (w1 - wall) * 1e3 > self.slow_pass_ms:
                    self._slow_pass(now, wall, cpu, sw, t_sub, w1)
                wall, cpu, sw = w1, time.thread_time(), _switches()
                if idle and w1 > t_end:
                    raise TimeoutError(f"serving loop exceeded {timeout_s} s "
                                       f"({len(pending)} pending, {len(self.inflight)} in flight)")
            self.b.synchronize()
        finally:
            if self.freeze_gc:
                gc.unfreeze()
        return self.finished

    def _slow_pass(self, now, wall, cpu, sw, t_sub, w1):
        sw1 = _switches()
        poll, admit, launch = self._phase
        self.slow_passes.append(dict(
            at_s=round(now, 4), wall_ms=round((w1 - wall) * 1e3, 3),
            cpu_ms=round((time.thread_time() - cpu) * 1e3, 3),
            submit_ms=round((t_sub - wall) * 1e3, 3), poll_ms=round(poll * 1e3, 3),
            admit_ms=round(admit * 1e3, 3), launch_ms=round(launch * 1e3, 3),
            voluntary=sw1[0] - sw[0], involuntary=sw1[1] - sw[1]))


def _switches():
    """(voluntary, involuntary) context switches of the calling thread so far."""
    try:
        r = resource.getrusage(resource.RUSAGE_THREAD)
    except (AttributeError, OSError):
        return (0, 0)
    return (r.ru_nvcsw, r.ru_nivcsw)


def latency_stats(finished: List[Request]):
    """p50/p99 latency (ms) overall and per kind, and columns/s over the run."""
    done = [r for r in finished if r.status == "done"]
    if not done:
        return dict(requests=0)
    lat = np.array([r.latency for r in done]) * 1e3
    t0 = min(r.arrival for r in done)
    t1 = max(r.t_done for r in done)
    out = dict(requests=len(done), p50_ms=float(np.percentile(lat, 50)),
               p99_ms=float(np.percentile(lat, 99)), mean_ms=float(lat.mean()),
               max_ms=float(lat.max()), columns=int(sum(r.columns for r in done)),
               makespan_s=float(t1 - t0))
    out["columns_per_s"] = out["columns"] / max(t1 - t0, 1e-9)
    for kind in KINDS:
        sel = np.array([r.latency for r in done if r.kind == kind]) * 1e3
        if sel.size:
            out[f"{kind}_p50_ms"] = float(np.percentile(sel, 50))
            out[f"{kind}_p99_ms"] = float(np.percentile(sel, 99))
            out[f"{kind}_requests"] = int(sel.size)
            out[f"{kind}_columns"] = int(sum(r.columns for r in done if r.kind == kind))
    return out


def overlap_stats(items: List[WorkItem]):
    """Device time of the tendency and VJP work items, and how much of the VJP time ran
    while a tendency batch was also on the device."""
    iv = {k: sorted(it.interval for it in items if it.kind == k) for k in KINDS}
    busy = {k: float(sum(b - a for a, b in v)) for k, v in iv.items()}
    both = 0.0
    for a, b in iv[VJP]:
        for c, d in iv[TENDENCY]:
            if c >= b:
                break
            both += max(0.0, min(b, d) - max(a, c))
    return dict(tendency_busy_s=busy[TENDENCY], vjp_busy_s=busy[VJP], overlap_s=both,
                vjp_overlap_fraction=both / busy[VJP] if busy[VJP] > 0 else 0.0)


# Resolutions and level counts of the request stream (spectral truncation -> (ix, il)).
STREAM_GRIDS = {21: (64, 32), 31: (96, 48), 42: (128, 64), 85: (256, 128), 170: (512, 256)}


def poisson_stream(seed=0, rate=200.0, n=400, vjp_fraction=0.2, max_members=32,
                   truncations=(21, 31, 42, 85, 170), levels=(8, 16), member_pool=8):
    """Requests of the serving workload: Poisson arrivals at ``rate`` per second, tendency or
    VJP (``vjp_fraction``), 1..``max_members`` members at one resolution and level count drawn
    uniformly.  Member keys are (truncation, kx, seed) with seeds from a pool of
    ``member_pool`` per (truncation, kx), so member state is shared across requests."""
    rng = np.random.default_rng(seed)
    t = np.cumsum(rng.exponential(1.0 / rate, n)) if rate > 0 else np.zeros(n)
    reqs = []
    for i in range(n):
        trunc = int(rng.choice(truncations))
        kx = int(rng.choice(levels))
        m = int(rng.integers(1, max_members + 1))
        s0 = int(rng.integers(0, member_pool))
        kind = VJP if rng.uniform() < vjp_fraction else TENDENCY
        keys = [(trunc, kx, (s0 + j) % member_pool) for j in range(m)]
        reqs.append(Request(kind, keys, arrival=float(t[i]), seed=int(rng.integers(1 << 30))))
    return reqs


def synthetic_member(key, base_seed=5000):
    """The synthetic land member (an Instance) that a ``poisson_stream`` key names."""
    from . import synthetic
    trunc, kx, s = key
    ix, il = STREAM_GRIDS[trunc]
    return synthetic.land_instance(base_seed + 1000 * trunc + 100 * kx + s, ix, il, kx)


def synthetic_source(base_seed=5000, pin=True):
    """Member source for ``poisson_stream`` keys: land members of the synthetic generator."""
    cache = {}

    def source(key):
        if key not in cache:
            cache[key] = HostMember.from_instance(synthetic_member(key, base_seed), pin=pin)
        return cache[key]
    return source


# ---------------------------------------------------------------------------------------------
# Device arena
# ---------------------------------------------------------------------------------------------
class DeviceArena:
    """Best-fit allocator over a few large device chunks, so that serving never calls into the
    driver's allocator on the request path (a cudaMalloc of a fresh segment takes milliseconds).

    The scheduler frees a buffer only after every kernel that used it has completed (member
    state when no admitted request references it, results after the completion event), so a
    freed range can be handed out again at once, on any stream.  Chunks are added on demand
    (``chunk_bytes`` or the request, whichever is larger) and kept."""

    ALIGN = 256

    def __init__(self, device, chunk_bytes=8 << 30, alloc=None):
        import torch
        self.torch = torch
        self.device = device
        self.chunk_bytes = int(chunk_bytes)
        self._alloc = alloc or (lambda n: torch.empty(n, dtype=torch.uint8, device=device))
        self.chunks = []          # uint8 tensors
        self.free = []            # per chunk: sorted list of [offset, size]
        self.reserved = 0
        self.in_use = 0

    def reserve(self, nbytes):
        """Adds a chunk of at least nbytes."""
        n = self.chunk_bytes if nbytes <= self.chunk_bytes else _round_up(int(nbytes), 2 << 20)
        t = self._alloc(n)
        self.chunks.append(t)
        self.free.append([[0, n]])
        self.reserved += n
        return len(self.chunks) - 1

    def alloc(self, nbytes):
        """A uint8 device tensor of nbytes (256-byte aligned), and its handle for release()."""
        n = _round_up(max(int(nbytes), 1), self.ALIGN)
        best = None
        for ci, fl in enumerate(self.free):
            for j, (off, size) in enumerate(fl):
                if size >= n and (best is None or size < best[3]):
                    best = (ci, j, off, size)
        if best is None:
            ci = self.reserve(n)
            best = (ci, 0, 0, self.free[ci][0][1])
        ci, j, off, size = best
        if size == n:
            del self.free[ci][j]
        else:
            self.free[ci][j] = [off + n, size - n]
        self.in_use += n
        return self.chunks[ci][off:off + n], (ci, off, n)

    def release(self, handle):
        ci, off, n = handle
        fl = self.free[ci]
        lo, hi = 0, len(fl)
        while lo < hi:
            mid = (lo + hi) // 2
            if fl[mid][0] < off:
                lo = mid + 1
            else:
                hi = mid
        fl.insert(lo, [off, n])
        # coalesce with the neighbours
        if lo + 1 < len(fl) and fl[lo][0] + fl[lo][1] == fl[lo + 1][0]:
            fl[lo][1] += fl[lo + 1][1]
            del fl[lo + 1]
        if lo > 0 and fl[lo - 1][0] + fl[lo - 1][1] == fl[lo][0]:
            fl[lo - 1][1] += fl[lo][1]
            del fl[lo]
        self.in_use -= n


class PinnedCache:
    """Reusable pinned host buffers for plans (a pinned allocation costs milliseconds)."""

    def __init__(self):
        import torch
        self.torch = torch
        self.pool = []

    def get(self, nbytes):
        for i, t in enumerate(self.pool):
            if t.numel() >= nbytes:
                return self.pool.pop(i)
        return self.torch.empty(max(int(nbytes), 1 << 20) * 2, dtype=self.torch.uint8,
                                pin_memory=True)

    def put(self, t):
        self.pool.append(t)
        self.pool.sort(key=lambda x: x.numel())


# ---------------------------------------------------------------------------------------------
# CUDA backend
# ---------------------------------------------------------------------------------------------
class _DevMember:
    __slots__ = ("host", "buf", "inputs", "ready", "handle")

    def __init__(self, host, buf, inputs, ready):
        self.host, self.buf, self.inputs, self.ready = host, buf, inputs, ready


class _Handle:
    __slots__ = ("stream", "start", "done", "keep")

    def __init__(self, stream, start, done, keep):
        self.stream, self.start, self.done, self.keep = stream, start, done, keep


class CudaBackend:
    """Device work of the serving loop through the C ABI (ensemble, plain and VJP calls)."""

    def __init__(self, device="cuda", date=None, parameters=None, mode="batched",
                 arena_chunk_bytes=8 << 30, reserve_bytes=0,
                 tendency_grid=_lib.GRID_PER_TILE):
        import torch
        from .physics import DateData, SpeedyPhysics, initialize_vertical
        self.torch = torch
        self.lib = _lib.load()
        self.dev = torch.device(device)
        if self.dev.index is None:
            self.dev = torch.device("cuda", torch.cuda.current_device())
        _lib.preload(self.dev.index)
        self.mode = mode
        # grid_blocks of the batched forward.  One block per tile by default: tendency batches
        # share the GPU with adjoint batches, and a persistent block that starts late still owns
        # its whole stride of tiles (measured at saturation: 1.59 G columns/s per tile against
        # 1.47 G persistent).  0 = persistent grids.
        self.tendency_grid = tendency_grid
        self.date = date or DateData(80.0 / 365.2425, 1950, 0, 1800.0)
        self.phys = SpeedyPhysics(parameters, diagnostics=False)
        # tendency batches on the highest-priority stream: when an adjoint batch shares the
        # GPU, the block scheduler hands freed SMs to tendency blocks first
        self.compute = torch.cuda.Stream(self.dev, priority=-10)
        self.vjp_stream = torch.cuda.Stream(self.dev) if mode == "batched" else self.compute
        self.copy = torch.cuda.Stream(self.dev) if mode == "batched" else self.compute
        self._vg = {}
        self._vert = initialize_vertical
        # adjoint scratch: one buffer, reused in stream order on the VJP stream
        self._vjp_bytes = max(self._vjp_scratch_bytes(kx) for kx in (8, 16))
        self._fwd_bytes = self._fwd_scratch_bytes()
        with torch.cuda.stream(self.vjp_stream):
            self.vjp_scratch = torch.empty(self._vjp_bytes, dtype=torch.uint8, device=self.dev)
        with torch.cuda.stream(self.compute):
            self.fwd_scratch = torch.empty(self._fwd_bytes, dtype=torch.uint8, device=self.dev)
        self.arena = DeviceArena(self.dev, chunk_bytes=arena_chunk_bytes)
        if reserve_bytes > 0:  # a service sizes its pool once, at startup
            self.arena.reserve(reserve_bytes)
        self.pinned = PinnedCache()
        self._free_at, self._free_reserved, self._dev_free = None, None, 0
        self._t0 = None
        self._h0 = 0.0

    # -- sizes ----------------------------------------------------------------------------------
    def _desc(self, kx, ix, il, lfluxland, forward=False):
        """The instance descriptor.  Forward calls form the cloud-top level set before the
        columns (SPD_NO_SPECULATION): every tendency batch is a new plan and the plain calls
        share one scratch across members, so there is no previous call of the same instance to
        predict it from."""
        from types import SimpleNamespace
        d = self.phys.desc(SimpleNamespace(nodal_shape=(kx, ix, il)), self.date, lfluxland)
        if forward:
            d.flags |= _lib.SPD_NO_SPECULATION
        return d

    def _vjp_scratch_bytes(self, kx):
        # 512 x 256 columns reach the adjoint's thread cap, hence its largest scratch
        d = self._desc(kx, 512, 256, True)
        return int(self.lib.spd_vjp_scratch_bytes(C.byref(d)))

    def _fwd_scratch_bytes(self):
        d = self._desc(16, 512, 256, True)
        return int(self.lib.spd_fwd_scratch_bytes(C.byref(d)))

    def vgrid(self, kx):
        if kx not in self._vg:
            from .physics import Geometry
            g = Geometry.__new__(Geometry)
            vert = self._vert(kx)
            for n, v in zip(("hsg", "fsg", "dhs", "sigl", "grdsig", "grdscp", "wvi"), vert):
                setattr(g, n, v)
            g.nodal_shape = (kx, 1, 1)
            g._vgrid = None
            self._vg[kx] = g.vgrid()
        return self._vg[kx]

    def fixed_bytes(self):
        return self._vjp_bytes + self._fwd_bytes

    def member_bytes(self, h):
        return h.nbytes

    def output_bytes(self, kind, h):
        f = tendency_result_floats if kind == TENDENCY else vjp_result_floats
        return _round_up(4 * f(h.kx, h.ix, h.il))

    # -- clock ----------------------------------------------------------------------------------
    def start_clock(self):
        torch = self.torch
        torch.cuda.synchronize(self.dev)
        self._t0 = torch.cuda.Event(enable_timing=True)
        self._t0.record(self.compute)
        self._t0.synchronize()
        self._h0 = time.perf_counter()

    def now(self):
        return time.perf_counter() - self._h0

    def synchronize(self):
        self.torch.cuda.synchronize(self.dev)

    # -- memory ---------------------------------------------------------------------------------
    def upload(self, h):
        torch = self.torch
        try:
            buf, handle = self.arena.alloc(h.nbytes)
        except torch.cuda.OutOfMemoryError as e:
            raise MemoryError(str(e))
        with torch.cuda.stream(self.copy):
            buf[:h.nbytes].copy_(h.buffer, non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(self.copy)
        base = buf.data_ptr()
        off, _ = member_layout(h.kx, h.ix, h.il)
        inputs = _lib.Inputs(**{n: base + off[n][0] for n in _lib.INPUT_FIELDS})
        dm = _DevMember(h, buf, inputs, ev)
        dm.handle = handle
        return dm

    def available_bytes(self, need=None):
        """Device bytes this backend can still hand out: its pool's free bytes, plus the
        device's free memory (the pool grows into it), less a 1 GiB margin for the driver and
        other users of the device.  When the pool's own free bytes cover ``need`` that figure
        is returned as it is: the driver's free memory (cudaMemGetInfo) is asked for only when
        the pool may have to grow, because the query waits on the device -- in the request
        loop it blocked a pass for 6-16 ms while batches ran.  The driver's figure is measured
        at most every half second and after the pool grows, the pool's own figure exactly."""
        pool_free = self.arena.reserved - self.arena.in_use
        if need is not None and pool_free >= need:
            return pool_free
        now = time.perf_counter()
        if (self._free_at is None or now - self._free_at > 0.5 or
                self._free_reserved != self.arena.reserved):
            self._dev_free = int(self.torch.cuda.mem_get_info(self.dev)[0])
            self._free_at, self._free_reserved = now, self.arena.reserved
        return pool_free + max(0, self._dev_free - (1 << 30))

    def release(self, dm):
        # The member's upload may still be running on the copy stream (a prefetched member, or
        # one left over by an admission that failed part way): the range must not go to
        # another request's outputs, which a compute stream writes, before that copy ends.
        if dm.ready is not None:
            dm.ready.synchronize()
        self.arena.release(dm.handle)
        dm.buf = None

    def alloc_outputs(self, req, hosts):
        """One device buffer per request: every member's result planes, then (VJP) every
        member's cotangent planes in one contiguous region, each region 256-byte aligned.  Only
        offsets are recorded here; tensor views are made when results are read."""
        if req.kind == TENDENCY:
            names3 = ("u_wind", "v_wind", "temperature", "specific_humidity")
            names2 = ("precnv", "precls")
        else:
            names3 = ("u_wind", "v_wind", "temperature", "specific_humidity", "geopotential")
            names2 = ("normalized_surface_pressure",)
        layout, pos = [], 0
        for h in hosts:
            c, kx = h.columns, h.kx
            d, p = {}, pos
            for k in names3:
                d[k] = (p, (kx, h.ix, h.il))
                p += kx * c
            for k in names2:
                d[k] = (p, (h.ix, h.il))
                p += c
            if req.kind == VJP:
                d["params"] = (p, (12,))
                p += 12
            layout.append(d)
            pos += _round_up(4 * (p - pos)) // 4
        ct0 = pos
        if req.kind == VJP:
            for h, d in zip(hosts, layout):
                c, kx = h.columns, h.kx
                for k in ("u_wind", "v_wind", "temperature", "specific_humidity"):
                    d["ct_" + k] = (pos, (kx, h.ix, h.il))
                    pos += kx * c
                pos = _round_up(4 * pos) // 4
        try:
            raw, req._out_handle = self.arena.alloc(4 * pos)
        except self.torch.cuda.OutOfMemoryError as e:
            raise MemoryError(str(e))
        req._outputs = raw[:4 * pos].view(self.torch.float32)
        req._ct = req._outputs[ct0:] if req.kind == VJP else None
        req._base = req._outputs.data_ptr()
        req._views = layout

    def free_outputs(self, req):
        h = req._out_handle
        if h is not None:
            self.arena.release(h)
            req._out_handle = None
        req._outputs = None
        req._views = None
        req._ct = None

    def results(self, req):
        """Per member, a dict of tensor views of its results (and cotangents, for a VJP)."""
        out = req._outputs
        res = []
        for d in req._views:
            v = {}
            for k, (off, shape) in d.items():
                n = 1
                for x in shape:
                    n *= x
                v[k] = out[off:off + n].view(shape)
            res.append(v)
        return res

    # -- launches -------------------------------------------------------------------------------
    def launch(self, kind, reqs, devs):
        torch = self.torch
        if kind == VJP:
            stream = self.vjp_stream
        else:
            stream = self.compute
        start = torch.cuda.Event(enable_timing=True)
        done = torch.cuda.Event(enable_timing=True)
        keep = []
        with torch.cuda.stream(stream):
            seen = set()
            for dl in devs:
                for dm in dl:
                    if id(dm) not in seen:
                        seen.add(id(dm))
                        stream.wait_event(dm.ready)
            start.record(stream)
            if kind == VJP and self.mode == "plain":
                for r, dl in zip(reqs, devs):
                    self._vjp_plain(r, dl, stream)
            elif kind == VJP:
                keep.append(self._vjp_batch(reqs, devs, stream))
            elif self.mode == "plain":
                for r, dl in zip(reqs, devs):
                    for dm, d in zip(dl, r._views):
                        self._fwd_plain(dm, r, d, stream)
            else:
                keep.append(self._ensemble(reqs, devs, stream))
            done.record(stream)
        return _Handle(stream, start, done, keep)

    @staticmethod
    def _ptrs(req, d, names):
        return {k: (req._base + 4 * d[k][0] if k in d else None) for k in names}

    def _outputs_struct(self, req, d):
        return _lib.Outputs(**self._ptrs(req, d, _lib.OUTPUT_FIELDS))

    def _fwd_plain(self, dm, req, d, stream):
        h = dm.host
        desc = self._desc(h.kx, h.ix, h.il, h.lfluxland, forward=True)
        rc = self.lib.spd_fwd(C.byref(desc), C.byref(self.vgrid(h.kx)),
                              C.byref(self.phys._pstruct), C.byref(dm.inputs),
                              C.byref(self._outputs_struct(req, d)),
                              C.c_void_p(self.fwd_scratch.data_ptr()), self._fwd_bytes,
                              C.c_void_p(stream.cuda_stream))
        _lib.check(rc, "spd_fwd")

    def _cotangents(self, req):
        """The request's cotangents: N(0, 1), one draw over its contiguous cotangent region from
        a generator seeded by the request (so a request draws the same cotangents alone or in a
        mix)."""
        g = self.torch.Generator(device=self.dev)
        g.manual_seed(int(req.seed))
        req._ct.normal_(generator=g)

    def _grads_struct(self, req, d):
        return _lib.Grads(**self._ptrs(req, d, ("u_wind", "v_wind", "temperature",
                                                "specific_humidity", "geopotential",
                                                "normalized_surface_pressure", "params")))

    def _ct_struct(self, req, d):
        p = self._ptrs(req, d, ("ct_u_wind", "ct_v_wind", "ct_temperature",
                                "ct_specific_humidity"))
        return _lib.Cotangents(**{k[3:]: v for k, v in p.items()})

    def _vjp_plain(self, req, dl, stream):
        self._cotangents(req)
        for dm, d in zip(dl, req._views):
            h = dm.host
            desc = self._desc(h.kx, h.ix, h.il, h.lfluxland)
            rc = self.lib.spd_vjp(C.byref(desc), C.byref(self.vgrid(h.kx)),
                                  C.byref(self.phys._pstruct), C.byref(dm.inputs),
                                  C.byref(self._ct_struct(req, d)),
                                  C.byref(self._grads_struct(req, d)),
                                  C.c_void_p(self.vjp_scratch.data_ptr()), self._vjp_bytes,
                                  C.c_void_p(stream.cuda_stream))
            _lib.check(rc, "spd_vjp")

    def _classes(self, members, forward=False):
        classes, cls_of = [], {}
        for h in members:
            key = (h.kx, h.lfluxland)
            if key not in cls_of:
                c = _lib.Class()
                c.desc = self._desc(h.kx, h.ix, h.il, h.lfluxland, forward)
                c.vgrid = self.vgrid(h.kx)
                c.params = self.phys._pstruct
                cls_of[key] = len(classes)
                classes.append(c)
        if len(classes) > _lib.MAX_CLASSES:
            raise ValueError("more member classes than one ensemble launch takes")
        return (_lib.Class * len(classes))(*classes), cls_of

    def _plan(self, bytes_fn, plan_fn, classes, mem, n):
        nbytes = int(bytes_fn(mem, n))
        host = self.pinned.get(nbytes)
        plan, handle = self.arena.alloc(nbytes)
        info = _lib.PlanInfo()
        rc = plan_fn(classes, len(classes), mem, n, C.c_void_p(host.data_ptr()),
                     C.c_void_p(plan.data_ptr()), nbytes, C.byref(info))
        _lib.check(rc, "ensemble plan")
        plan[:nbytes].copy_(host[:nbytes], non_blocking=True)
        return host, handle, info

    def _vjp_batch(self, reqs, devs, stream):
        pairs = [(dm, r, d) for r, dl in zip(reqs, devs) for dm, d in zip(dl, r._views)]
        for r in reqs:
            self._cotangents(r)
        cl, cls_of = self._classes([dm.host for dm, _, _ in pairs])
        mem = (_lib.VjpMember * len(pairs))()
        for i, (dm, r, d) in enumerate(pairs):
            h = dm.host
            mem[i].inp = dm.inputs
            mem[i].ct = self._ct_struct(r, d)
            mem[i].grads = self._grads_struct(r, d)
            mem[i].ix, mem[i].il, mem[i].cls = h.ix, h.il, cls_of[(h.kx, h.lfluxland)]
        host, handle, info = self._plan(self.lib.spd_ensemble_vjp_plan_bytes,
                                        self.lib.spd_ensemble_vjp_plan, cl, mem, len(pairs))
        plan = self.arena.chunks[handle[0]].data_ptr() + handle[1]
        rc = self.lib.spd_ensemble_vjp(cl, len(cl), C.c_void_p(plan), C.byref(info), 0,
                                       C.c_void_p(stream.cuda_stream))
        _lib.check(rc, "spd_ensemble_vjp")
        return (host, handle, cl, mem)

    def _ensemble(self, reqs, devs, stream):
        pairs = [(dm, r, d) for r, dl in zip(reqs, devs) for dm, d in zip(dl, r._views)]
        cl, cls_of = self._classes([dm.host for dm, _, _ in pairs], forward=True)
        mem = (_lib.Member * len(pairs))()
        for i, (dm, r, d) in enumerate(pairs):
            h = dm.host
            mem[i].inp = dm.inputs
            mem[i].out = self._outputs_struct(r, d)
            mem[i].ix, mem[i].il, mem[i].cls = h.ix, h.il, cls_of[(h.kx, h.lfluxland)]
        host, handle, info = self._plan(self.lib.spd_ensemble_plan_bytes,
                                        self.lib.spd_ensemble_plan, cl, mem, len(pairs))
        plan = self.arena.chunks[handle[0]].data_ptr() + handle[1]
        rc = self.lib.spd_ensemble_fwd(cl, len(cl), C.c_void_p(plan), C.byref(info),
                                       int(self.tendency_grid), C.c_void_p(stream.cuda_stream))
        _lib.check(rc, "spd_ensemble_fwd")
        return (host, handle, cl, mem)

    def done(self, handle):
        return handle.done.query()

    def completion_time(self, handle):
        """Device completion of the work item, in seconds on the loop's clock (``now``)."""
        return self._t0.elapsed_time(handle.done) / 1e3

    def device_interval(self, handle):
        """(start, end) of the work item in seconds on the loop's clock."""
        return (self._t0.elapsed_time(handle.start) / 1e3,
                self._t0.elapsed_time(handle.done) / 1e3)

    def retire(self, handle):
        for host, arena_handle, _, _ in handle.keep:
            self.pinned.put(host)
            self.arena.release(arena_handle)
        handle.keep = None
