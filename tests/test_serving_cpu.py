"""Serving loop logic on the CPU: admission by budget, residency and eviction, continuous
batching, plain (one request at a time) order, rejection of malformed and oversized requests,
allocation failures, cancellation, and the request stream generator.  The device is a fake
backend on a virtual clock: a launched work item takes (columns x cost) seconds on its stream."""
import importlib

import numpy as np
import pytest

pkg = importlib.import_module("jax-gcm_b200")
S = pkg.serving


class FakeBackend:
    def __init__(self, fixed=0, per_col=1e-6, fail_alloc=0, realtime=False):
        self.t = 0.0
        self.fixed = fixed
        self.per_col = per_col
        self.fail_alloc = fail_alloc
        self.realtime = realtime
        self.uploaded, self.released, self.launched = [], [], []
        self.stream_free = {S.TENDENCY: 0.0, S.VJP: 0.0}
        self._h0 = 0.0

    def fixed_bytes(self):
        return self.fixed

    def member_bytes(self, h):
        return h.nbytes

    def output_bytes(self, kind, h):
        return 4 * h.columns * (4 * h.kx + 2 if kind == S.TENDENCY else 9 * h.kx + 1)

    def now(self):
        if self.realtime:
            import time
            return time.perf_counter() - self._h0
        return self.t

    def start_clock(self):
        import time
        self._h0 = time.perf_counter()

    def synchronize(self):
        pass

    def upload(self, h):
        self.uploaded.append(h)
        return ("dev", id(h))

    def release(self, d):
        self.released.append(d)

    def alloc_outputs(self, req, hosts):
        if self.fail_alloc > 0:
            self.fail_alloc -= 1
            raise MemoryError("injected allocation failure")
        req._outputs = [dict(n=h.columns) for h in hosts]

    def free_outputs(self, req):
        req._outputs = None

    def results(self, req):
        return req._outputs

    def launch(self, kind, reqs, devs):
        cols = sum(r.columns for r in reqs)
        start = max(self.now(), self.stream_free[kind])
        end = start + cols * self.per_col
        self.stream_free[kind] = end
        self.launched.append((kind, [r.rid for r in reqs]))
        return dict(start=start, end=end)

    def done(self, h):
        return self.now() >= h["end"]

    def completion_time(self, h):
        return h["end"]

    def device_interval(self, h):
        return (h["start"], h["end"])

    def retire(self, h):
        pass


def host(kx=8, ix=64, il=32, nbytes=None):
    n = nbytes if nbytes is not None else S.member_layout(kx, ix, il)[1]
    return S.HostMember(kx, ix, il, True, None, n)


def make_source(**shapes):
    hosts = {k: host(*v) if isinstance(v, tuple) else v for k, v in shapes.items()}

    def source(key):
        return hosts[key]
    return source, hosts


def test_member_layout_is_aligned_and_complete():
    off, n = S.member_layout(16, 96, 48)
    assert [k for k in off] == list(pkg._lib.INPUT_FIELDS)
    for name, (pos, cnt) in off.items():
        assert pos % 256 == 0
        exp = 16 * 96 * 48 if name in ("u_wind", "v_wind", "temperature", "specific_humidity",
                                       "geopotential") else (48 if name in ("sia", "coa")
                                                             else 96 * 48)
        assert cnt == exp, name
    assert n >= 4 * (5 * 16 * 96 * 48 + 10 * 96 * 48 + 2 * 48)


def test_host_member_packs_instance_fields():
    inst = pkg.synthetic.land_instance(3, 8, 4, 8)
    h = S.HostMember.from_instance(inst, pin=False)
    off, n = S.member_layout(8, 8, 4)
    flat = h.buffer.view(-1).numpy().view(np.float32)
    pos, cnt = off["temperature"]
    assert np.array_equal(flat[pos // 4: pos // 4 + cnt], inst.t.ravel())
    pos, cnt = off["coa"]
    assert np.array_equal(flat[pos // 4: pos // 4 + cnt], inst.coa)
    assert h.nbytes == n and h.columns == 32


def test_continuous_batching_merges_arrivals_while_busy():
    src, _ = make_source(a=(8, 64, 32), b=(16, 64, 32), c=(8, 96, 48))
    be = FakeBackend(per_col=1e-6)
    sch = S.Scheduler(be, src, budget_bytes=1 << 30, max_inflight=2)
    for k in ("a", "b", "c"):
        sch.submit(S.Request(S.TENDENCY, [k]))
    sch.step()
    assert be.launched == [(S.TENDENCY, [0, 1, 2])]          # one batch of three
    sch.submit(S.Request(S.TENDENCY, ["a", "b"]))
    sch.submit(S.Request(S.TENDENCY, ["c"]))
    sch.step()
    assert be.launched[-1] == (S.TENDENCY, [3, 4])            # second batch while first runs
    sch.submit(S.Request(S.TENDENCY, ["a"]))
    sch.step()
    assert len(be.launched) == 2                              # two in flight: waits
    assert [r.rid for r in sch.admitted[S.TENDENCY]] == [5]
    be.t = 1.0
    sch.step()
    assert be.launched[-1] == (S.TENDENCY, [5])
    be.t = 2.0
    sch.step()
    assert not sch.busy()
    assert [r.status for r in sch.finished] == ["done"] * 6
    assert len(be.uploaded) == 3                              # members stay resident


def test_vjp_requests_run_on_their_own_stream_and_overlap():
    src, _ = make_source(a=(8, 128, 64), b=(16, 128, 64))
    be = FakeBackend(per_col=1e-6)
    sch = S.Scheduler(be, src, budget_bytes=1 << 30)
    sch.submit(S.Request(S.TENDENCY, ["a"]))
    sch.submit(S.Request(S.VJP, ["b"]))
    sch.step()
    kinds = sorted(k for k, _ in be.launched)
    assert kinds == [S.TENDENCY, S.VJP]
    be.t = 10.0
    sch.step()
    ov = S.overlap_stats(sch.items)
    assert ov["overlap_s"] > 0 and 0 < ov["vjp_overlap_fraction"] <= 1


def test_plain_mode_is_one_request_at_a_time_in_arrival_order():
    src, _ = make_source(a=(8, 64, 32), b=(16, 64, 32))
    be = FakeBackend(per_col=1e-6)
    sch = S.Scheduler(be, src, budget_bytes=1 << 30, mode="plain")
    sch.submit(S.Request(S.VJP, ["a"]))
    sch.submit(S.Request(S.TENDENCY, ["b"]))
    sch.submit(S.Request(S.TENDENCY, ["a"]))
    for step in range(10):
        be.t = float(step)
        sch.step()
        assert len(sch.inflight) <= 1
    order = [ids for _, ids in be.launched]
    assert order == [[0], [1], [2]]


def test_budget_admission_eviction_and_fifo():
    out = 4 * (4 * 8 + 2) * 64 * 32       # one member's tendency outputs
    m = 10 * out                          # one member's resident state
    hosts = dict(a=host(8, 64, 32, nbytes=m), b=host(8, 64, 32, nbytes=m),
                 c=host(8, 64, 32, nbytes=m))
    src = hosts.__getitem__
    budget = 2 * m + 2 * out + 10         # r0's members and outputs; no room for r1 beside
    be = FakeBackend(per_col=1e-3)
    sch = S.Scheduler(be, src, budget_bytes=budget)
    r0 = sch.submit(S.Request(S.TENDENCY, ["a", "b"]))
    r1 = sch.submit(S.Request(S.TENDENCY, ["c"]))
    sch.step()
    assert r0.status == "running" and r1.status == "waiting"
    assert sch.used <= budget
    be.t = 100.0
    sch.step()                            # r0 done; r1 admitted after evicting an idle member
    assert r0.status == "done" and r1.status in ("running", "done")
    assert sch.stats["evictions"] >= 1
    assert sch.peak <= budget
    be.t = 200.0
    sch.step()
    assert r1.status == "done" and sch.used == be.fixed_bytes() + sum(
        h.nbytes for k, h in hosts.items() if k in sch.resident)


def test_resident_members_in_use_are_never_evicted():
    hosts = dict(a=host(nbytes=1000), b=host(nbytes=1000))
    out = 4 * (4 * 8 + 2) * 64 * 32
    be = FakeBackend(per_col=1e-3)
    sch = S.Scheduler(be, hosts.__getitem__, budget_bytes=1000 + out + 500)
    r0 = sch.submit(S.Request(S.TENDENCY, ["a"]))
    r1 = sch.submit(S.Request(S.TENDENCY, ["b"]))
    sch.step()
    assert r0.status == "running" and r1.status == "waiting"
    assert "a" in sch.resident and sch.resident["a"].refs == 1
    assert not be.released


def test_rejections_malformed_and_oversized():
    hosts = dict(a=host(nbytes=1000))
    be = FakeBackend()
    sch = S.Scheduler(be, hosts.__getitem__, budget_bytes=10_000)
    r = sch.submit(S.Request(S.TENDENCY, ["missing"]))
    assert r.status == "rejected" and r.reason.startswith("malformed")
    r = sch.submit(S.Request("forecast", ["a"]))
    assert r.status == "rejected" and "kind" in r.reason
    r = sch.submit(S.Request(S.TENDENCY, []))
    assert r.status == "rejected"
    r = sch.submit(S.Request(S.TENDENCY, ["a"]))      # outputs alone exceed the budget
    assert r.status == "rejected" and "budget" in r.reason
    assert sch.stats["rejected"] == 4 and not sch.busy()


def test_allocation_failure_is_retried():
    src, _ = make_source(a=(8, 64, 32))
    be = FakeBackend(fail_alloc=2)
    sch = S.Scheduler(be, src, budget_bytes=1 << 30)
    r = sch.submit(S.Request(S.TENDENCY, ["a"]))
    sch.step()
    assert r.status == "waiting"
    sch.step()
    assert r.status == "waiting"
    sch.step()
    assert r.status == "running"
    assert sch.stats["alloc_failures"] == 2


def test_cancel_waiting_and_inflight():
    src, hosts = make_source(a=(8, 64, 32), b=(8, 64, 32))
    seen = []
    be = FakeBackend(per_col=1e-3)
    sch = S.Scheduler(be, src, budget_bytes=1 << 30, mode="plain", on_complete=seen.append)
    r0 = sch.submit(S.Request(S.TENDENCY, ["a"]))
    r1 = sch.submit(S.Request(S.TENDENCY, ["b"]))
    sch.step()
    assert r0.status == "running"
    assert sch.cancel(r1.rid) and r1.status == "cancelled"
    assert sch.cancel(r0.rid)
    be.t = 100.0
    sch.step()
    assert r0.status == "cancelled" and not seen
    assert not sch.busy() and sch.used == sum(
        h.nbytes for k, h in hosts.items() if k in sch.resident)
    assert not sch.cancel(12345)


def test_run_loop_real_time_with_fake_device():
    src, _ = make_source(a=(8, 64, 32), b=(16, 96, 48))
    be = FakeBackend(per_col=1e-8, realtime=True)
    sch = S.Scheduler(be, src, budget_bytes=1 << 30)
    reqs = [S.Request(S.TENDENCY if i % 3 else S.VJP, ["a", "b"][: 1 + i % 2],
                      arrival=0.002 * i) for i in range(20)]
    fin = sch.run(reqs, timeout_s=30)
    st = S.latency_stats(fin)
    assert st["requests"] == 20 and st["p99_ms"] >= st["p50_ms"] >= 0
    assert all(r.t_done >= r.arrival for r in fin)


def test_slow_passes_name_the_phase_and_the_wait():
    """A launch that blocks for 30 ms shows as one slow pass: its time in launch, little
    CPU time, and a voluntary context switch (a blocking wait, not a preemption)."""
    import time
    src, _ = make_source(a=(8, 64, 32))
    blocked = []

    class Blocking(FakeBackend):
        def launch(self, kind, reqs, devs):
            if not blocked:
                blocked.append(True)
                time.sleep(0.03)
            return super().launch(kind, reqs, devs)

    sch = S.Scheduler(Blocking(per_col=1e-8, realtime=True), src, 1 << 30, slow_pass_ms=20.0)
    sch.run([S.Request(S.TENDENCY, ["a"], arrival=0.001 * i) for i in range(4)], timeout_s=30)
    assert len(sch.slow_passes) >= 1
    p = max(sch.slow_passes, key=lambda p: p["wall_ms"])
    assert p["wall_ms"] >= 29.0 and p["launch_ms"] >= 29.0
    assert p["cpu_ms"] < 0.5 * p["wall_ms"]
    assert p["voluntary"] >= 1
    assert set(p) >= {"at_s", "submit_ms", "poll_ms", "admit_ms", "involuntary"}


def test_run_freezes_the_collector_for_its_duration():
    import gc
    src, _ = make_source(a=(8, 64, 32))
    seen = []

    class Probe(FakeBackend):
        def launch(self, kind, reqs, devs):
            seen.append(gc.get_freeze_count())
            return super().launch(kind, reqs, devs)

    reqs = lambda: [S.Request(S.TENDENCY, ["a"], arrival=0.001 * i) for i in range(4)]
    n_objects = len(gc.get_objects())
    S.Scheduler(Probe(per_col=1e-8, realtime=True), src, 1 << 30).run(reqs(), timeout_s=30)
    assert seen and min(seen) >= n_objects // 2   # objects alive at the start were frozen
    assert gc.get_freeze_count() == 0             # and released at the end
    seen.clear()
    S.Scheduler(Probe(per_col=1e-8, realtime=True), src, 1 << 30,
                freeze_gc=False).run(reqs(), timeout_s=30)
    assert seen and max(seen) == 0


def test_poisson_stream_shape():
    reqs = S.poisson_stream(seed=4, rate=200.0, n=2000)
    t = np.array([r.arrival for r in reqs])
    assert np.all(np.diff(t) >= 0)
    assert abs(np.mean(np.diff(t)) - 1 / 200) < 0.0005
    frac = np.mean([r.kind == S.VJP for r in reqs])
    assert 0.17 < frac < 0.23
    sizes = [len(r.members) for r in reqs]
    assert min(sizes) == 1 and max(sizes) == 32
    assert {k[0] for r in reqs for k in r.members} == {21, 31, 42, 85, 170}
    assert {k[1] for r in reqs for k in r.members} == {8, 16}
    assert S.poisson_stream(seed=4, n=5)[3].members == S.poisson_stream(seed=4, n=5)[3].members


def test_latency_stats():
    rs = []
    for i in range(100):
        r = S.Request(S.TENDENCY, ["a"], arrival=i * 0.01)
        r.status, r.t_done, r.columns = "done", i * 0.01 + 0.001 * (i + 1), 10
        rs.append(r)
    st = S.latency_stats(rs)
    assert st["requests"] == 100
    assert st["p50_ms"] == pytest.approx(50.5, rel=1e-6)
    assert st["p99_ms"] == pytest.approx(99.01, rel=1e-6)
    assert st["columns"] == 1000


def test_device_arena_best_fit_coalescing_and_growth():
    import torch
    made = []

    def alloc(n):
        made.append(n)
        return torch.zeros(n, dtype=torch.uint8)

    A = S.DeviceArena("cpu", chunk_bytes=1 << 20, alloc=alloc)
    a, ha = A.alloc(1000)
    b, hb = A.alloc(5000)
    c, hc = A.alloc(300)
    assert made == [1 << 20] and a.numel() == 1024 and b.numel() == 5120
    offs = sorted(h[1] for h in (ha, hb, hc))
    assert all(o % 256 == 0 for o in offs) and len(set(offs)) == 3
    A.release(hb)
    d, hd = A.alloc(4096)                      # best fit: reuses b's hole
    assert hd[1] == hb[1]
    A.release(ha)
    A.release(hc)
    A.release(hd)
    assert A.free == [[[0, 1 << 20]]] and A.in_use == 0   # all coalesced back
    big, hbig = A.alloc(3 << 20)               # larger than a chunk: a new chunk
    assert len(made) == 2 and made[1] >= 3 << 20 and hbig[0] == 1
    A.release(hbig)
    e, he = A.alloc(100)
    assert he[0] == 0                          # smallest fitting hole is in chunk 0


def test_device_arena_reuse_never_overlaps():
    import torch
    rng = np.random.default_rng(1)
    A = S.DeviceArena("cpu", chunk_bytes=1 << 22,
                      alloc=lambda n: torch.zeros(n, dtype=torch.uint8))
    live = {}
    for step in range(400):
        if live and rng.uniform() < 0.45:
            k = list(live)[int(rng.integers(len(live)))]
            A.release(live.pop(k))
        else:
            _, h = A.alloc(int(rng.integers(1, 200_000)))
            live[step] = h
        spans = sorted((h[0], h[1], h[1] + h[2]) for h in live.values())
        for (c0, a0, b0), (c1, a1, b1) in zip(spans, spans[1:]):
            assert c0 != c1 or b0 <= a1
    for h in live.values():
        A.release(h)
    assert A.in_use == 0 and all(len(f) == 1 for f in A.free)


def test_prefetch_makes_members_resident_within_budget():
    hosts = dict(a=host(nbytes=1000), b=host(nbytes=1000), c=host(nbytes=1000))
    be = FakeBackend()
    sch = S.Scheduler(be, hosts.__getitem__, budget_bytes=2500)
    assert sch.prefetch(["a", "b", "a"]) == 2
    assert set(sch.resident) == {"a", "b"} and sch.used == 2000
    assert sch.prefetch(["c"]) == 1            # evicts the least recently used idle member
    assert "c" in sch.resident and len(sch.resident) == 2 and sch.used <= 2500
    r = sch.submit(S.Request(S.TENDENCY, ["c"]))
    assert r.status == "rejected"              # outputs do not fit beside any member


def test_admission_is_capped_per_step():
    src, _ = make_source(a=(8, 64, 32))
    be = FakeBackend(per_col=1e-6)
    sch = S.Scheduler(be, src, budget_bytes=1 << 30, max_admit_per_step=3)
    for _ in range(7):
        sch.submit(S.Request(S.TENDENCY, ["a"]))
    sch.admit()
    assert len(sch.waiting) == 4


def test_cuda_backend_release_waits_for_the_upload_before_freeing():
    """CudaBackend.release returns a member's range to the arena only after the member's
    upload event has completed (recorded order: the event's synchronize, then the arena
    release); no device is touched (the event and the arena are fakes)."""
    S = pkg.serving
    order = []

    class Ev:
        def synchronize(self):
            order.append("upload done")

    class Arena:
        def release(self, handle):
            order.append(("arena release", handle))

    be = S.CudaBackend.__new__(S.CudaBackend)
    be.arena = Arena()
    dm = S._DevMember(None, object(), None, Ev())
    dm.handle = 7
    be.release(dm)
    assert order == ["upload done", ("arena release", 7)]
    assert dm.buf is None


def test_cuda_backend_asks_the_driver_only_when_the_pool_may_grow():
    """CudaBackend.available_bytes answers from its pool while the pool's free bytes cover the
    request; the driver's free memory (a query that waits on the device) is asked for only
    when they do not.  No device is touched (the arena and torch are fakes)."""
    S = pkg.serving
    asked = []

    class Cuda:
        @staticmethod
        def mem_get_info(dev):
            asked.append(dev)
            return (10 << 30, 80 << 30)

    class Torch:
        cuda = Cuda

    class Arena:
        reserved, in_use = 4 << 30, 1 << 30

    be = S.CudaBackend.__new__(S.CudaBackend)
    be.arena, be.torch, be.dev = Arena(), Torch(), 0
    be._free_at, be._free_reserved, be._dev_free = None, None, 0
    assert be.available_bytes(2 << 30) == 3 << 30 and asked == []
    assert be.available_bytes(5 << 30) == (3 << 30) + (9 << 30) and asked == [0]
    assert be.available_bytes() == (3 << 30) + (9 << 30) and asked == [0]   # half-second cache


def test_admission_waits_for_free_device_memory_below_the_budget():
    """A backend that measures its free device memory below what the budget would allow:
    requests are admitted only as far as that memory goes (idle members evicted first), the
    rest wait until memory frees up; the budget alone would have admitted both at once."""
    class Measured(FakeBackend):
        def __init__(self, limit, **kw):
            super().__init__(**kw)
            self.limit = limit
            self.held = {}

        def available_bytes(self, need=None):
            return self.limit - sum(self.held.values())

        def upload(self, h):
            d = super().upload(h)
            self.held[d] = h.nbytes
            return d

        def release(self, d):
            self.held.pop(d, None)
            return super().release(d)

    out = 4 * (4 * 8 + 2) * 64 * 32
    m = 10 * out
    hosts = dict(a=host(8, 64, 32, nbytes=m), b=host(8, 64, 32, nbytes=m))
    be = Measured(limit=m + 2 * out, per_col=1e-3)
    sch = S.Scheduler(be, hosts.__getitem__, budget_bytes=1 << 40)
    r0 = sch.submit(S.Request(S.TENDENCY, ["a"]))
    r1 = sch.submit(S.Request(S.TENDENCY, ["b"]))
    sch.step()
    assert r0.status == "running" and r1.status == "waiting"
    be.t = 100.0
    sch.step()                            # r0 done: "a" evicted to make room for "b"
    assert r0.status == "done" and r1.status in ("running", "done")
    assert sch.stats["evictions"] == 1
    be.t = 200.0
    sch.step()
    assert r1.status == "done"
