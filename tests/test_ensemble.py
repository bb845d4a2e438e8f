"""Batched ragged ensemble: the host-side plan (CPU) and per-member equality with the plain
per-instance forward plus oracle parity (GPU)."""
import ctypes as C
import importlib

import numpy as np
import pytest

from oracle import speedy_oracle as O
from tests.helpers import compare_fields, fake_fields, to_device


@pytest.fixture(scope="module")
def pkg():
    return importlib.import_module("jax-gcm_b200")


def _fake_member(L, ix, il, cls):
    m = L.Member()
    m.inp, m.out = fake_fields(L)  # never dereferenced by the plan
    m.ix, m.il, m.cls = ix, il, cls
    return m


def test_plan_layout_and_tile_order(pkg):
    """The plan (host side, no device work): tiles cover every column once, 16-level members
    first, each member's level-set word and solar table at distinct aligned offsets."""
    L = pkg._lib
    lib = L.load()
    classes = (L.Class * 2)()
    classes[0].desc.kx, classes[1].desc.kx = 8, 16
    shapes = [(64, 32, 0), (96, 48, 1), (64, 32, 1), (7, 3, 0)]
    mem = (L.Member * len(shapes))(*[_fake_member(L, *s) for s in shapes])
    n = lib.spd_ensemble_plan_bytes(mem, len(shapes))
    host = (C.c_ubyte * n)()
    info = L.PlanInfo()
    dev_base = 1 << 32
    rc = lib.spd_ensemble_plan(classes, 2, mem, len(shapes), C.cast(host, C.c_void_p),
                               C.c_void_p(dev_base), n, C.byref(info))
    assert rc == 0
    want_tiles = sum((ix * il + 127) // 128 for ix, il, _ in shapes)
    assert info.ntiles == want_tiles and info.nmembers == 4
    raw = bytes(host)
    member_bytes = (n - 256)  # not used beyond sanity
    assert member_bytes > 0
    # tiles are (member, col0) int pairs after the member table
    msize = C.sizeof(L.Inputs) + C.sizeof(L.Outputs) + 4 * 4 + 2 * 8
    tiles_off = 256 + ((4 * msize + 255) // 256) * 256
    tiles = np.frombuffer(raw, dtype=np.int32, count=2 * info.ntiles, offset=tiles_off)
    tiles = tiles.reshape(-1, 2)
    kx_of = [8, 16, 16, 8]
    order = [kx_of[m] for m in tiles[:, 0]]
    assert order == sorted(order, reverse=True)
    covered = {}
    for m, c0 in tiles:
        covered.setdefault(int(m), []).append(int(c0))
    for i, (ix, il, _) in enumerate(shapes):
        assert covered[i] == list(range(0, ix * il, 128))
    assert info.levelset_offset % 256 == 0
    # the level-set region: launch words, then each member's T, R and P words (the member
    # count rounded up to 4 apart), then the count of redone members
    nw = 4
    assert info.levelset_bytes == 16 + 12 * nw + 16
    head = C.sizeof(L.Inputs) + C.sizeof(L.Outputs) + 4 * 4
    for i in range(len(shapes)):
        rec = 256 + i * msize
        s_ptr = int(np.frombuffer(raw, np.uint64, 1, rec + head)[0])
        stride = int(np.frombuffer(raw, np.int32, 1, rec + head + 8)[0])
        assert s_ptr == dev_base + info.levelset_offset + 16 + 4 * i and stride == nw


def test_plan_rejects_bad_class(pkg):
    L = pkg._lib
    lib = L.load()
    classes = (L.Class * 1)()
    classes[0].desc.kx = 8
    mem = (L.Member * 1)(_fake_member(L, 64, 32, 3))
    n = lib.spd_ensemble_plan_bytes(mem, 1)
    host = (C.c_ubyte * n)()
    info = L.PlanInfo()
    rc = lib.spd_ensemble_plan(classes, 1, mem, 1, C.cast(host, C.c_void_p),
                               C.c_void_p(1 << 32), n, C.byref(info))
    assert rc == 2


CT_FIELDS = ("u_wind", "v_wind", "temperature", "specific_humidity")
GRAD_FIELDS = ("u_wind", "v_wind", "temperature", "specific_humidity", "geopotential",
               "normalized_surface_pressure", "params")


def _fake_vjp_member(L, ix, il, cls, slot):
    m = L.VjpMember()
    m.inp, _ = fake_fields(L)  # never dereferenced by the plan
    base = (1 << 40) + slot * (1 << 34)
    m.ct = L.Cotangents(**{k: base + i * (1 << 28) for i, k in enumerate(CT_FIELDS)})
    m.grads = L.Grads(**{k: base + (4 + i) * (1 << 28) for i, k in enumerate(GRAD_FIELDS)})
    m.ix, m.il, m.cls = ix, il, cls
    return m


def test_vjp_plan_layout_tiles_and_records(pkg):
    """The adjoint's plan (host side): every column once, 16-level members first, and each
    member record carrying its column count, level count, class, level-set word and table."""
    L = pkg._lib
    lib = L.load()
    classes = (L.Class * 2)()
    classes[0].desc.kx, classes[1].desc.kx = 8, 16
    shapes = [(64, 32, 0), (96, 48, 1), (64, 32, 1), (7, 3, 0)]
    mem = (L.VjpMember * len(shapes))(*[_fake_vjp_member(L, *s, i)
                                        for i, s in enumerate(shapes)])
    n = lib.spd_ensemble_vjp_plan_bytes(mem, len(shapes))
    host = (C.c_ubyte * n)()
    info = L.PlanInfo()
    dev_base = 1 << 32
    rc = lib.spd_ensemble_vjp_plan(classes, 2, mem, len(shapes), C.cast(host, C.c_void_p),
                                   C.c_void_p(dev_base), n, C.byref(info))
    assert rc == 0
    assert info.ntiles == sum((ix * il + 127) // 128 for ix, il, _ in shapes)
    raw = bytes(host)
    head = C.sizeof(L.Inputs) + C.sizeof(L.Cotangents) + C.sizeof(L.Grads)
    msize = head + 4 * 4 + 2 * 8
    kx_of = [8, 16, 16, 8]
    tables = set()
    for i, (ix, il, cls) in enumerate(shapes):
        rec = 256 + i * msize
        cols, il_, kx, cls_ = np.frombuffer(raw, np.int32, 4, rec + head)
        assert (cols, il_, kx, cls_) == (ix * il, il, kx_of[i], cls)
        s_ptr, table = np.frombuffer(raw, np.uint64, 2, rec + head + 16)
        assert s_ptr == dev_base + info.levelset_offset + 16 + 4 * i
        tables.add(int(table))
    assert len(tables) == len(shapes) and all(t % 256 == 0 for t in tables)
    tiles_off = 256 + ((len(shapes) * msize + 255) // 256) * 256
    tiles = np.frombuffer(raw, np.int32, 2 * info.ntiles, tiles_off).reshape(-1, 2)
    order = [kx_of[m] for m in tiles[:, 0]]
    assert order == sorted(order, reverse=True)
    covered = {}
    for m, c0 in tiles:
        covered.setdefault(int(m), []).append(int(c0))
    for i, (ix, il, _) in enumerate(shapes):
        assert covered[i] == list(range(0, ix * il, 128))


def test_vjp_plan_rejects_missing_cotangent_and_bad_class(pkg):
    L = pkg._lib
    lib = L.load()
    classes = (L.Class * 1)()
    classes[0].desc.kx = 8

    def plan(m):
        mem = (L.VjpMember * 1)(m)
        n = lib.spd_ensemble_vjp_plan_bytes(mem, 1)
        host = (C.c_ubyte * n)()
        return lib.spd_ensemble_vjp_plan(classes, 1, mem, 1, C.cast(host, C.c_void_p),
                                         C.c_void_p(1 << 32), n, C.byref(L.PlanInfo()))

    m = _fake_vjp_member(L, 64, 32, 0, 0)
    assert plan(m) == 0
    m.ct.temperature = None
    assert plan(m) == 1
    assert plan(_fake_vjp_member(L, 64, 32, 2, 0)) == 2


def _members(pkg, device):
    insts = [pkg.synthetic.land_instance(500 + i, ix, il, kx)
             for i, (ix, il, kx) in enumerate([(64, 32, 8), (64, 32, 16), (96, 48, 16),
                                               (128, 64, 8), (7, 5, 16)])]
    members, plain = [], []
    for inst in insts:
        state, forcing, geom, date = to_device(pkg, inst, device)
        members.append(pkg.Member(state, forcing, geom))
        plain.append((state, forcing, geom, date))
    return insts, members, plain


@pytest.mark.gpu
def test_ensemble_matches_plain_and_oracle(pkg):
    import torch
    insts, members, plain = _members(pkg, "cuda")
    date = plain[0][3]
    ens = pkg.Ensemble(members, date)
    outs = ens.forward()
    torch.cuda.synchronize()
    phys = pkg.SpeedyPhysics(diagnostics=False)
    for inst, out, (st, fo, ge, da) in zip(insts, outs, plain):
        tend, data = phys.compute_tendencies(st, fo, ge, da)
        for k, ref in (("temperature", tend.temperature), ("specific_humidity", tend.specific_humidity),
                       ("u_wind", tend.u_wind), ("v_wind", tend.v_wind),
                       ("precnv", data.convection.precnv), ("precls", data.condensation.precls)):
            assert torch.equal(out[k], ref), (inst.name, k)
    # one member against the oracle, through the ensemble path
    inst, out = insts[2], outs[2]
    tend, data = O.compute_tendencies(*inst.oracle_args(O.default_parameters()))
    got = {k: out[k].cpu().numpy() for k in ("u_wind", "v_wind", "temperature",
                                              "specific_humidity", "precnv", "precls")}
    rep = compare_fields(got, tend, data)
    bad_cols = np.zeros((inst.ix, inst.il), bool)
    for v in rep.values():
        b = v["bad"]
        while b.ndim > 2:
            b = b.any(0)
        bad_cols |= b
    assert bad_cols.sum() <= 2, {k: v["nbad"] for k, v in rep.items()}


@pytest.mark.gpu
def test_ensemble_graph_replay_and_autotune(pkg):
    import torch
    insts, members, plain = _members(pkg, "cuda")
    ens = pkg.Ensemble(members, plain[0][3])
    ref = [{k: v.clone() for k, v in o.items()} for o in ens.forward()]
    # one block per tile instead of persistent grids: the same columns, bitwise
    for o, r in zip(ens.forward(grid_blocks=pkg._lib.GRID_PER_TILE), ref):
        for k in r:
            assert torch.equal(o[k], r[k]), k
    gb = ens.autotune(reps=2)
    assert gb >= 0 or gb == pkg._lib.GRID_PER_TILE
    for o in ens.forward():
        for v in o.values():
            v.fill_(float("nan"))
    g = ens.capture(calls=3)
    g.replay()
    torch.cuda.synchronize()
    for o, r in zip([m.out for m in ens.members], ref):
        for k in r:
            assert torch.equal(o[k], r[k]), k


@pytest.mark.gpu
def test_host_pipeline_matches_ensemble(pkg):
    """HostPipeline (state from and results to pinned host memory, steps overlapped over
    double buffers) gives every member the results Ensemble.forward gives, bitwise, on each of
    three consecutive steps (both buffer sets, one reused)."""
    import torch
    insts, members, plain = _members(pkg, "cuda")
    ref = [{k: v.clone() for k, v in o.items()}
           for o in pkg.Ensemble(members, plain[0][3]).forward()]
    pipe = pkg.batched.HostPipeline(
        [pkg.Member(m.state, m.forcing, m.geometry) for m in members], plain[0][3])
    for i, m in enumerate(members):
        pipe.set_state(i, m.state)
    pipe.begin()
    bufs = [pipe.submit() for _ in range(3)]
    pipe.end()
    torch.cuda.synchronize()
    assert bufs == [0, 1, 0]
    for b in (0, 1):
        pipe.wait(b)
        for i, (got, want) in enumerate(zip(pipe.results(b), ref)):
            for k in want:
                g = got[k]
                if k in ("u_wind", "v_wind"):  # the lowest level crosses PCIe
                    g = pipe.dense_winds(i, g)
                assert torch.equal(g, want[k].cpu()), k
    # only the lowest wind level moves: T, q, phi at every level, u, v, psa once per column
    cols = [(m.kx, m.columns) for m in insts]
    assert pipe.h2d_bytes >= 4 * sum((3 * kx + 3) * c for kx, c in cols)
    assert pipe.h2d_bytes < 4 * sum((3 * kx + 3) * c + 6 * 64 for kx, c in cols)
    assert pipe.d2h_bytes < 4 * sum((2 * kx + 4) * c + 6 * 64 for kx, c in cols)
