"""The serving loop on the GPU: each request's result is the same served alone and in a mix
of concurrent tendency and VJP requests, the same in batched and plain mode, the same under a
budget that forces evictions, and equal to the per-member drop-in call.

Tendencies and VJP state gradients are bitwise equal (every column is computed by one thread
with the same instructions whatever else runs).  The 12 parameter gradients are sums over
columns accumulated with atomics, whose order varies run to run: they agree within
1e-5 x max|g| per member."""
import importlib

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu

pkg = importlib.import_module("jax-gcm_b200")
S = pkg.serving
PARAM_TOL = 1e-5


def stream(n=16, seed=3):
    return S.poisson_stream(seed=seed, rate=4000.0, n=n, truncations=(21, 31, 42),
                            max_members=4, member_pool=3)


def fresh(reqs, arrival=None):
    return [S.Request(r.kind, list(r.members), r.arrival if arrival is None else arrival, r.seed)
            for r in reqs]


_SOURCE = S.synthetic_source()


def serve(reqs, mode="batched", budget=16 << 30):
    res = {}

    def keep(r):
        res[r.rid] = [{k: v.detach().cpu().clone() for k, v in d.items()} for d in r.result]

    be = S.CudaBackend("cuda", mode=mode)
    sch = S.Scheduler(be, _SOURCE, budget, mode=mode, on_complete=keep)
    fin = sch.run(reqs, timeout_s=300)
    assert all(r.status == "done" for r in fin), [(r.status, r.reason) for r in fin]
    return res, sch


def assert_same(kind, a, b, what):
    for ma, mb in zip(a, b):
        for k in ma:
            if k == "params":
                scale = float(ma[k].abs().max()) or 1.0
                err = float((ma[k] - mb[k]).abs().max())
                assert err <= PARAM_TOL * scale, (what, kind, k, err, scale)
            else:
                assert torch.equal(ma[k], mb[k]), (what, kind, k)


def test_alone_equals_in_mix():
    reqs = stream()
    assert {r.kind for r in reqs} == {S.TENDENCY, S.VJP}
    mix, sch = serve(fresh(reqs))
    assert sch.stats["launches_tendency"] < sum(r.kind == S.TENDENCY for r in reqs), \
        "the mix should have batched some tendency requests together"
    for i, r in enumerate(reqs):
        alone, _ = serve(fresh([r], arrival=0.0))
        assert_same(r.kind, mix[i], alone[0], f"request {i}")


def test_plain_mode_and_evicting_budget_give_the_same_results():
    reqs = stream(n=12, seed=8)
    base, _ = serve(fresh(reqs))
    plain, _ = serve(fresh(reqs), mode="plain")
    # room for the adjoint scratch, the largest request and a little more: forces evictions
    be = S.CudaBackend("cuda")
    largest = max(sum(_SOURCE(k).nbytes for k in set(r.members)) +
                  sum(be.output_bytes(r.kind, _SOURCE(k)) for k in r.members) for r in reqs)
    budget = be.fixed_bytes() + largest + (1 << 20)
    del be
    tight, sch = serve(fresh(reqs), budget=budget)
    assert sch.stats["evictions"] > 0 and sch.peak <= budget
    for i, r in enumerate(reqs):
        assert_same(r.kind, base[i], plain[i], f"plain {i}")
        assert_same(r.kind, base[i], tight[i], f"tight budget {i}")


def test_served_tendencies_equal_the_drop_in_call():
    reqs = [S.Request(S.TENDENCY, [(21, 8, 0), (31, 16, 1), (42, 8, 2)])]
    res, _ = serve(fresh(reqs))
    phys = pkg.SpeedyPhysics(diagnostics=False)
    for key, got in zip(reqs[0].members, res[0]):
        inst = S.synthetic_member(key)
        st, fo, ge, da = pkg.instance_to_device(inst, "cuda")
        tend, data = phys.compute_tendencies(st, fo, ge, da)
        torch.cuda.synchronize()
        for k in ("u_wind", "v_wind", "temperature", "specific_humidity"):
            assert torch.equal(got[k], getattr(tend, k).cpu()), (key, k)
        assert torch.equal(got["precnv"], data.convection.precnv.cpu())
        assert torch.equal(got["precls"], data.condensation.precls.cpu())


def test_served_vjp_equals_the_adjoint_call():
    reqs = [S.Request(S.VJP, [(21, 8, 0), (31, 16, 1)], seed=77)]
    res, _ = serve(fresh(reqs))
    phys = pkg.SpeedyPhysics(diagnostics=False)
    for key, got in zip(reqs[0].members, res[0]):
        inst = S.synthetic_member(key)
        st, fo, ge, da = pkg.instance_to_device(inst, "cuda")
        ct = pkg.PhysicsTendency(*(got["ct_" + k].cuda() for k in
                                   ("u_wind", "v_wind", "temperature", "specific_humidity")))
        gs, gp = pkg.adjoint.vjp(phys, st, fo, ge, da, ct)
        torch.cuda.synchronize()
        for k in ("u_wind", "v_wind", "temperature", "specific_humidity", "geopotential",
                  "normalized_surface_pressure"):
            assert torch.equal(got[k], getattr(gs, k).cpu()), (key, k)
        scale = float(gp.abs().max())
        assert float((got["params"] - gp.cpu()).abs().max()) <= PARAM_TOL * scale
