"""Batched ragged ensembles: many grid instances of mixed resolution and level count run in
one pair of persistent launches (``spd_ensemble_fwd``), optionally captured in a CUDA graph.

Each member gives the same tendencies as ``SpeedyPhysics.compute_tendencies`` on it alone
(jcm/physics/speedy/speedy_physics.py:88-127); the batching has no reference counterpart.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from typing import List, Optional

import torch

from . import _lib
from .physics import Parameters, SpeedyPhysics


@dataclass
class Member:
    state: object      # PhysicsState
    forcing: object    # ForcingData (2-D or daily 3-D fields)
    geometry: object   # Geometry
    out: Optional[dict] = None


_TUNE_CACHE = {}


class Ensemble:
    """A fixed set of members whose buffers stay in place between calls.

    ``forward()`` recomputes every member's tendencies into ``member.out`` (dicts with
    ``u_wind, v_wind, temperature, specific_humidity, precnv, precls``).  Members are grouped
    into at most four classes by (level count, land-flux switch, vertical grid).
    """

    def __init__(self, members: List[Member], date, parameters: Optional[Parameters] = None,
                 fuse_verify=False, time_step=None, q_tend_scale=1.0,
                 orographic_correction=False, low_level_winds=False, speculate=True):
        lib = _lib.load()
        self.low_level_winds = low_level_winds
        self.speculate = speculate
        self.members = members
        self.date = date
        self.phys = SpeedyPhysics(parameters, fuse_verify=fuse_verify, time_step=time_step,
                                  q_tend_scale=q_tend_scale, diagnostics=False,
                                  orographic_correction=orographic_correction,
                                  speculate=speculate)
        dev = members[0].state.temperature.device
        self.device = dev
        _lib.preload(dev.index if dev.index is not None else torch.cuda.current_device())
        keys, classes = {}, []
        cls_of = []
        day = date.model_day()
        self._keep = []
        for m in members:
            g = m.geometry
            kx = g.nodal_shape[0]
            key = (kx, bool(m.forcing.lfluxland), tuple(float(x) for x in g.hsg))
            if key not in keys:
                if len(classes) == _lib.MAX_CLASSES:
                    raise ValueError("at most 4 member classes (level count, land flux, grid)")
                keys[key] = len(classes)
                c = _lib.Class()
                c.desc = self.phys.desc(g, date, m.forcing.lfluxland)
                if low_level_winds:  # u, v and their tendencies as lowest-level planes
                    c.desc.flags |= _lib.SPD_LOW_LEVEL_WINDS
                c.vgrid = g.vgrid()
                c.params = self.phys._pstruct
                classes.append(c)
            cls_of.append(keys[key])
        self.nclasses = len(classes)
        self.classes = (_lib.Class * self.nclasses)(*classes)
        mem = (_lib.Member * len(members))()
        for i, m in enumerate(members):
            kx, ix, il = m.geometry.nodal_shape
            f2 = m.forcing.day_slice(day)
            self._keep.append(f2)
            st, g = m.state, m.geometry
            tensors = dict(u_wind=st.u_wind, v_wind=st.v_wind, temperature=st.temperature,
                           specific_humidity=st.specific_humidity, geopotential=st.geopotential,
                           normalized_surface_pressure=st.normalized_surface_pressure,
                           alb0=f2.alb0, sice_am=f2.sice_am, snowc_am=f2.snowc_am,
                           soilw_am=f2.soilw_am, stl_am=f2.stl_am,
                           sea_surface_temperature=f2.sea_surface_temperature, fmask=g.fmask,
                           orog=g.orog, phis0=g.phis0, sia=g.sia, coa=g.coa)
            for k, v in tensors.items():
                if v.dtype != torch.float32 or not v.is_contiguous() or v.device != dev:
                    raise ValueError(f"member {i}: field {k} must be contiguous float32 on {dev}")
            wind_numel = ix * il if low_level_winds else kx * ix * il
            for k in ("u_wind", "v_wind"):
                if tensors[k].numel() != wind_numel:
                    raise ValueError(f"member {i}: {k} must have {wind_numel} elements")
            if m.out is None:
                e3 = lambda: torch.empty((kx, ix, il), dtype=torch.float32, device=dev)
                e2 = lambda: torch.empty((ix, il), dtype=torch.float32, device=dev)
                ew = e2 if low_level_winds else e3
                m.out = dict(u_wind=ew(), v_wind=ew(), temperature=e3(), specific_humidity=e3(),
                             precnv=e2(), precls=e2())
            mem[i].inp = _lib.Inputs(**{k: tensors[k].data_ptr() for k in _lib.INPUT_FIELDS})
            mem[i].out = _lib.Outputs(**{k: (m.out[k].data_ptr() if k in m.out else None)
                                         for k in _lib.OUTPUT_FIELDS})
            mem[i].ix, mem[i].il, mem[i].cls = ix, il, cls_of[i]
        self._members_c = mem
        nbytes = lib.spd_ensemble_plan_bytes(mem, len(members))
        self.plan = torch.empty(nbytes, dtype=torch.uint8, device=dev)
        host = (C.c_ubyte * nbytes)()
        self.info = _lib.PlanInfo()
        rc = lib.spd_ensemble_plan(self.classes, self.nclasses, mem, len(members),
                                   C.cast(host, C.c_void_p), C.c_void_p(self.plan.data_ptr()),
                                   nbytes, C.byref(self.info))
        _lib.check(rc, "spd_ensemble_plan")
        self.plan.copy_(torch.frombuffer(bytearray(host), dtype=torch.uint8))
        self.grid_blocks = 0
        self.columns = sum(m.geometry.nodal_shape[1] * m.geometry.nodal_shape[2] for m in members)

    def signature(self):
        return tuple(sorted((m.geometry.nodal_shape for m in self.members)))

    def forward(self, grid_blocks=None, marker=None):
        """Runs every member.  ``marker`` (a torch.cuda.Event) is recorded between the two
        launches, for timing them separately: after the fused launch (before the fixup) when
        ``speculate``, after the level-set launch (before the fused one) otherwise.  With
        ``speculate`` each member's cloud-top level set is predicted from the previous call
        (the plan keeps it), checked on the device, and only members whose prediction missed
        are computed again (``redone()`` counts them)."""
        lib = _lib.load()
        gb = self.grid_blocks if grid_blocks is None else grid_blocks
        stream = torch.cuda.current_stream(self.device).cuda_stream
        ev = C.c_void_p(marker.cuda_event) if marker is not None else None
        rc = lib.spd_ensemble_fwd_marked(self.classes, self.nclasses,
                                         C.c_void_p(self.plan.data_ptr()), C.byref(self.info),
                                         int(gb), C.c_void_p(stream), ev)
        _lib.check(rc, "spd_ensemble_fwd")
        return [m.out for m in self.members]

    def redone(self):
        """Members the forward has computed a second time because their predicted level set
        missed, over every call on this plan (the first call misses for every member)."""
        nw = (self.info.nmembers + 3) & ~3
        off = int(self.info.levelset_offset) + 16 + 12 * nw
        return int(self.plan[off:off + 4].view(torch.int32).item())

    def autotune(self, candidates=None, reps=5):
        """Picks the launch shape by timing the candidates (CUDA events): persistent grids of
        0 (SMs x resident blocks), 1-4 blocks per SM, or one block per tile
        (``_lib.GRID_PER_TILE``); cached per ensemble signature."""
        sig = self.signature()
        if sig in _TUNE_CACHE:
            self.grid_blocks = _TUNE_CACHE[sig]
            return self.grid_blocks
        sms = torch.cuda.get_device_properties(self.device).multi_processor_count
        cands = candidates or [0, sms, 2 * sms, 3 * sms, 4 * sms, _lib.GRID_PER_TILE]
        best, best_ms = 0, float("inf")
        for gb in cands:
            self.forward(gb)
            torch.cuda.synchronize(self.device)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            for _ in range(reps):
                self.forward(gb)
            b.record()
            torch.cuda.synchronize(self.device)
            ms = a.elapsed_time(b) / reps
            if ms < best_ms:
                best, best_ms = gb, ms
        self.grid_blocks = best
        _TUNE_CACHE[sig] = best
        return best

    def capture(self, calls=1):
        """A CUDA graph of ``calls`` consecutive forwards (replay with ``graph.replay()``)."""
        s = torch.cuda.Stream(self.device)
        s.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(s):
            self.forward()
        torch.cuda.current_stream(self.device).wait_stream(s)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            for _ in range(calls):
                self.forward()
        return g


STATE_FIELDS = ("u_wind", "v_wind", "temperature", "specific_humidity", "geopotential",
                "normalized_surface_pressure")
RESULT_FIELDS = ("u_wind", "v_wind", "temperature", "specific_humidity", "precnv", "precls")


def _packed_layout(members, fields, level_fields):
    """Offsets (in floats, each field 64-float aligned) of every member's fields in one flat
    buffer; returns ([{field: (offset, shape)}], total floats)."""
    off, out = 0, []
    for m in members:
        kx, ix, il = m.geometry.nodal_shape
        d = {}
        for f in fields:
            shape = (kx, ix, il) if f in level_fields else (ix, il)
            n = 1
            for s in shape:
                n *= s
            d[f] = (off, shape)
            off += (n + 63) // 64 * 64
        out.append(d)
    return out, off


class HostPipeline:
    """Ensemble steps whose state comes from, and whose results go to, pinned host memory.

    Every member's state (T, q and phi at every level, u and v at the lowest level, psa) lives
    in one packed host buffer and every member's results (the T and q tendency planes, the
    lowest-level u and v tendencies, precnv, precls) in another, so a step is one host-to-device
    copy, one ``spd_ensemble_fwd`` and one device-to-host copy.  Only the lowest wind level
    crosses PCIe in either direction: the physics reads the winds there alone
    (surface_flux.py:57-58) and its wind tendencies are zero above it (surface_flux.py:294-295),
    so the ensemble runs with SPD_LOW_LEVEL_WINDS.  ``depth`` sets of device buffers (each with
    its own plan) rotate over three streams: while step n computes, step n+1's state uploads and
    step n-1's results download (PCIe carries both directions at once).  Forcing and geometry
    stay resident.

    ``host_state`` (pack into it with ``set_state``) is read by every step; ``submit()`` enqueues
    one step and returns the index of the host result buffer it writes; ``wait(i)`` blocks until
    that buffer is complete and ``results(i)`` views it per member (u and v tendencies as the
    lowest-level [ix, il] plane; ``dense_winds`` gives the reference's [kx, ix, il] form).
    """

    def __init__(self, members: List[Member], date, depth: int = 2, **ensemble_kw):
        dev = members[0].state.temperature.device
        self.device, self.depth = dev, depth
        level = {"temperature", "specific_humidity", "geopotential"}
        self.kx = [m.geometry.nodal_shape[0] for m in members]
        self.in_layout, n_in = _packed_layout(members, STATE_FIELDS, level)
        self.out_layout, n_out = _packed_layout(members, RESULT_FIELDS, level)
        self.host_state = torch.empty(n_in, dtype=torch.float32, pin_memory=True)
        self.host_results = [torch.empty(n_out, dtype=torch.float32, pin_memory=True)
                             for _ in range(depth)]
        self.dev_state = [torch.empty(n_in, dtype=torch.float32, device=dev)
                          for _ in range(depth)]
        self.dev_results = [torch.empty(n_out, dtype=torch.float32, device=dev)
                            for _ in range(depth)]
        self.ensembles = []
        for b in range(depth):
            mem = []
            for m, li, lo in zip(members, self.in_layout, self.out_layout):
                sv = {f: self._view(self.dev_state[b], *li[f]) for f in STATE_FIELDS}
                ov = {f: self._view(self.dev_results[b], *lo[f]) for f in RESULT_FIELDS}
                st = type(m.state)(*(sv[f] for f in STATE_FIELDS))
                mem.append(Member(st, m.forcing, m.geometry, ov))
            self.ensembles.append(Ensemble(mem, date, low_level_winds=True, **ensemble_kw))
        self.h2d = torch.cuda.Stream(dev)
        self.compute = torch.cuda.Stream(dev)
        self.d2h = torch.cuda.Stream(dev)
        ev = lambda: [torch.cuda.Event() for _ in range(depth)]
        self.uploaded, self.computed, self.downloaded = ev(), ev(), ev()
        self.used = [False] * depth
        self.n = 0

    @staticmethod
    def _view(flat, off, shape):
        n = 1
        for s in shape:
            n *= s
        return flat[off:off + n].view(shape)

    def set_state(self, i, state):
        """Packs member i's state (a PhysicsState of CPU or CUDA tensors, winds at every level)
        into host_state; of u and v only the lowest level is kept."""
        for f in STATE_FIELDS:
            x = getattr(state, f)
            if f in ("u_wind", "v_wind"):
                x = x[-1]
            self._view(self.host_state, *self.in_layout[i][f]).copy_(x)

    def begin(self):
        """Orders the pipeline's streams after the work already on the current stream."""
        cur = torch.cuda.current_stream(self.device)
        for s in (self.h2d, self.compute, self.d2h):
            s.wait_stream(cur)

    def submit(self):
        b = self.n % self.depth
        if self.used[b]:
            self.h2d.wait_event(self.computed[b])      # the buffer's previous step read it
        with torch.cuda.stream(self.h2d):
            self.dev_state[b].copy_(self.host_state, non_blocking=True)
            self.uploaded[b].record(self.h2d)
        self.compute.wait_event(self.uploaded[b])
        if self.used[b]:
            self.compute.wait_event(self.downloaded[b])  # its previous results were read out
        with torch.cuda.stream(self.compute):
            self.ensembles[b].forward()
            self.computed[b].record(self.compute)
        self.d2h.wait_event(self.computed[b])
        with torch.cuda.stream(self.d2h):
            self.host_results[b].copy_(self.dev_results[b], non_blocking=True)
            self.downloaded[b].record(self.d2h)
        self.used[b] = True
        self.n += 1
        return b

    def end(self):
        """Orders the current stream after every submitted step."""
        cur = torch.cuda.current_stream(self.device)
        for s in (self.h2d, self.compute, self.d2h):
            cur.wait_stream(s)

    def wait(self, i):
        self.downloaded[i].synchronize()

    def results(self, i):
        """Member views of host result buffer i: [{field: tensor}] (valid after wait(i))."""
        return [{f: self._view(self.host_results[i], *lo[f]) for f in RESULT_FIELDS}
                for lo in self.out_layout]

    def dense_winds(self, i, plane):
        """The reference's dense [kx, ix, il] wind tendency of member i from its lowest-level
        plane (zeros above)."""
        out = torch.zeros((self.kx[i],) + tuple(plane.shape), dtype=plane.dtype)
        out[-1] = plane
        return out

    @property
    def h2d_bytes(self):
        return self.host_state.numel() * 4

    @property
    def d2h_bytes(self):
        return self.host_results[0].numel() * 4
