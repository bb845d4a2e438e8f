"""The GPU adjoint (spd_vjp) against the host build of the same generic column code, and
autograd through the torch op.

The host float64 VJP is the finite-difference-checked one (tests/test_adjoint_cpu.py); the
GPU computes in float32.  Bar, per gradient field, column by column: |gpu - host64| <=
max(1e-4, 3x the host float32 VJP's own largest distance from float64) of the field's max.  A
column outside that bar is a branch flip (a convection, condensation or cloud threshold
decided differently in float32) and is explained when the GPU agrees with the host float32
VJP there, or when the host float32 VJP is itself outside the bar; at most 1 % of the columns
may flip and none may be unexplained.  Parameter gradients: each of the 12 within 1e-4
relative of the float64 host sum over the columns (the flipped columns' contributions taken
from the float32 host), except where float32 itself cannot reach that: the bar is then twice
the host float32 build's per-column distances from float64 summed over the columns (measured:
a single column's float32 sensitivity puts the host float32 sum 8.7e-5 from float64 at
32x16x8 seed 708, and a sum that cancels 115-fold puts it 4.7e-5 away at 32x16x16 seed 716;
the GPU's 1.4e-4 and 1.9e-4 there are the same arithmetic, unchanged without contraction).
"""
import importlib

import numpy as np
import pytest

from tests.test_adjoint_cpu import (VJP_HAND32, VJP_HAND64, vjp_any)
from tests.test_adjoint_cpu import (HostOut, _flags, _loss_and_grads, build_host, column_of,
                                    run_oracle, structs)

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pkg():
    return importlib.import_module("jax-gcm_b200")


@pytest.fixture(scope="module")
def host(tmp_path_factory):
    return build_host(tmp_path_factory.mktemp("hostcol") / "libhostcol.so")


def _gpu_vjp(pkg, inst, cts, fuse_verify=False, orographic=False):
    import torch
    state, forcing, geom, date = pkg.instance_to_device(inst, "cuda")
    phys = pkg.SpeedyPhysics(diagnostics=False, fuse_verify=fuse_verify, time_step=1800.0,
                             orographic_correction=orographic)
    t = lambda a: torch.as_tensor(a, dtype=torch.float32, device="cuda")
    cot = pkg.PhysicsTendency(t(cts["u"]), t(cts["v"]), t(cts["t"]), t(cts["q"]))
    gs, gp = pkg.adjoint.vjp(phys, state, forcing, geom, date, cot)
    torch.cuda.synchronize()
    c = lambda x: x.cpu().numpy().astype(np.float64)
    return dict(t=c(gs.temperature), q=c(gs.specific_humidity), phi=c(gs.geopotential),
                psa=c(gs.normalized_surface_pressure), u=c(gs.u_wind), v=c(gs.v_wind)), c(gp)


CASES = [  # (kx, seed, lfluxland, fused verify with some negative humidity, orographic term)
    (8, 708, True, False, False), (16, 716, True, False, False), (7, 707, True, False, False),
    (8, 808, False, False, False), (8, 908, True, True, False), (16, 916, True, True, False),
    (16, 926, True, True, True)]


@pytest.mark.parametrize("kx,seed,lfluxland,verify,oro", CASES)
def test_gpu_vjp_matches_host(pkg, host, kx, seed, lfluxland, verify, oro):
    inst = pkg.synthetic.land_instance(seed, 32, 16, kx)
    inst.lfluxland = lfluxland
    if verify:
        mask = np.random.default_rng(seed).uniform(size=inst.q.shape) < 0.05
        inst.q = np.where(mask, -np.abs(inst.q) * 0.01 - 1e-4, inst.q).astype(np.float32)
    if verify:  # the level set and solar rows the GPU sees: those of the verified state
        import copy
        vinst = copy.deepcopy(inst)
        vinst.q = np.where(vinst.q < 0, np.float32(0), vinst.q).astype(np.float32)
        tend, data, S = run_oracle(vinst)
    else:
        tend, data, S = run_oracle(inst)
    vg, pr = structs(pkg, inst)
    rng = np.random.default_rng(kx)
    shape = (kx, inst.ix, inst.il)
    cts = dict(t=rng.normal(size=shape), q=rng.normal(size=shape), u=rng.normal(size=shape),
               v=rng.normal(size=shape))
    g_gpu, p_gpu = _gpu_vjp(pkg, inst, cts, fuse_verify=verify, orographic=oro)
    flags = _flags(inst) | (16 if verify else 0) | (32 if oro else 0)
    h64 = {k: np.zeros_like(v) for k, v in g_gpu.items()}
    h32 = {k: np.zeros_like(v) for k, v in g_gpu.items()}
    pc = {False: np.zeros((inst.ix, inst.il, 12)), True: np.zeros((inst.ix, inst.il, 12))}
    for i in range(inst.ix):
        for j in range(inst.il):
            h = column_of(inst, data, S, i, j, flags)
            ct = (list(cts["t"][:, i, j]) + [0.0] * (16 - kx),
                  list(cts["q"][:, i, j]) + [0.0] * (16 - kx),
                  float(cts["u"][-1, i, j]), float(cts["v"][-1, i, j]))
            for f32, dst in ((False, h64), (True, h32)):
                if oro:  # the taped host forward has no orographic term: the hand-written
                    # host pass (the kernel's own source) in float64 and float32
                    g = vjp_any(host, VJP_HAND32 if f32 else VJP_HAND64, vg, pr, h, ct)
                    g = dict(g, psa=g["psa"][0], u=g["u"][0], v=g["v"][0])
                else:
                    g, _ = _loss_and_grads(host, vg, pr, h, *ct, f32=f32)
                dst["t"][:, i, j], dst["q"][:, i, j], dst["phi"][:, i, j] = g["t"], g["q"], g["phi"]
                dst["psa"][i, j] = g["psa"]
                dst["u"][-1, i, j], dst["v"][-1, i, j] = g["u"], g["v"]
                pc[f32][i, j] = g["params"]
    report = {}
    flipped = np.zeros((inst.ix, inst.il), bool)
    for k in ("t", "q", "phi", "psa", "u", "v"):
        scale = max(np.max(np.abs(h64[k])), 1e-30)
        e_gpu = np.abs(g_gpu[k] - h64[k]) / scale
        e_32 = np.abs(h32[k] - h64[k]) / scale
        report[k] = (float(e_gpu.max()), float(e_32.max()))
        # columns where float32 rounding flips a branch differ by O(1)
        tol = max(1e-4, 3 * float(np.median(e_32.reshape(-1, inst.ix, inst.il).max(axis=0))))
        colmax = lambda e: e.reshape(-1, inst.ix, inst.il).max(axis=0)
        bad = colmax(e_gpu) > tol
        agrees32 = colmax(np.abs(g_gpu[k] - h32[k]) / scale) <= tol
        flips32 = colmax(e_32) > tol
        unexplained = bad & ~agrees32 & ~flips32
        assert unexplained.sum() == 0, (k, report[k], np.argwhere(unexplained))
        assert bad.sum() <= max(2, 0.01 * inst.ix * inst.il), (k, report[k], bad.sum())
        flipped |= bad
    print(inst.name, report)
    # the float64 sum, with the flipped columns' contributions from the float32 host (the GPU
    # takes their float32 branch)
    p64 = np.where(flipped[..., None], pc[True], pc[False]).sum(axis=(0, 1))
    # the float32 noise of that sum: the host float32 build's per-column distances from float64,
    # added up over the columns that did not flip
    e32 = np.where(flipped[..., None], 0.0, np.abs(pc[True] - pc[False])).sum(axis=(0, 1))
    err = np.abs(p_gpu - p64)
    rel = err / np.maximum(np.abs(p64), 1e-30)
    print("parameter gradients, relative error", np.array2string(rel, precision=1))
    print("host float32 noise, relative", np.array2string(e32 / np.maximum(np.abs(p64), 1e-30),
                                                          precision=1))
    assert np.all(err <= np.maximum(1e-4 * np.abs(p64), 2 * e32)), (p_gpu, p64, rel)


def test_large_batch_budget_matches_host(pkg, host):
    """A 256 x 256 instance with 16 levels is 512 tiles, more than two blocks per SM hold at
    once, so the VJP runs the 128-register (four blocks per SM) budget of the adjoint kernel;
    the small cases above run the 255-register one.  Sampled columns against the host VJP under
    the bar above (the float64 host within max(1e-4, 3x the float32 host's own distance) of the
    field's sampled maximum, flips explained by the float32 host)."""
    kx = 16
    inst = pkg.synthetic.land_instance(4242, 256, 256, kx)
    tend, data, S = run_oracle(inst)
    vg, pr = structs(pkg, inst)
    rng = np.random.default_rng(5)
    shape = (kx, inst.ix, inst.il)
    cts = dict(t=rng.normal(size=shape), q=rng.normal(size=shape), u=rng.normal(size=shape),
               v=rng.normal(size=shape))
    g_gpu, _ = _gpu_vjp(pkg, inst, cts)
    flags = _flags(inst)
    cols = [(int(i), int(j)) for i, j in zip(rng.integers(0, inst.ix, 48),
                                               rng.integers(0, inst.il, 48))]
    h64s, h32s = {k: [] for k in ("t", "q", "phi")}, {k: [] for k in ("t", "q", "phi")}
    for (i, j) in cols:
        h = column_of(inst, data, S, i, j, flags)
        ct = (list(cts["t"][:, i, j]), list(cts["q"][:, i, j]),
              float(cts["u"][-1, i, j]), float(cts["v"][-1, i, j]))
        g64, _ = _loss_and_grads(host, vg, pr, h, *ct, f32=False)
        g32, _ = _loss_and_grads(host, vg, pr, h, *ct, f32=True)
        for k in h64s:
            h64s[k].append(np.asarray(g64[k])[:kx])
            h32s[k].append(np.asarray(g32[k])[:kx])
    for k in h64s:
        a64, a32 = np.array(h64s[k]), np.array(h32s[k])
        gps = np.array([g_gpu[k][:, i, j] for (i, j) in cols])
        scale = max(np.max(np.abs(a64)), 1e-30)
        e_gpu = np.abs(gps - a64).max(axis=1) / scale
        e_32 = np.abs(a32 - a64).max(axis=1) / scale
        tol = max(1e-4, 3 * float(np.median(e_32)))
        bad = e_gpu > tol
        explained = (np.abs(gps - a32).max(axis=1) / scale <= tol) | (e_32 > tol)
        assert np.all(~bad | explained), (k, float(e_gpu.max()), tol)
        assert bad.sum() <= 1, (k, int(bad.sum()))


def test_autograd_through_torch_op(pkg):
    import torch
    inst = pkg.synthetic.land_instance(55, 32, 16, 8)
    state, forcing, geom, date = pkg.instance_to_device(inst, "cuda")
    phys = pkg.SpeedyPhysics(diagnostics=False)
    for f in ("u_wind", "v_wind", "temperature", "specific_humidity", "geopotential",
              "normalized_surface_pressure"):
        getattr(state, f).requires_grad_(True)
    params = pkg.adjoint.parameter_vector(device="cpu").requires_grad_(True)
    tend = pkg.adjoint.tendencies(phys, state, forcing, geom, date, params)
    ref, _ = phys.compute_tendencies(pkg.PhysicsState(*(getattr(state, f).detach() for f in (
        "u_wind", "v_wind", "temperature", "specific_humidity", "geopotential",
        "normalized_surface_pressure"))), forcing, geom, date)
    assert torch.equal(tend.temperature.detach(), ref.temperature)
    w = torch.randn_like(tend.temperature)
    loss = (tend.temperature * w).sum() + tend.specific_humidity.sum()
    loss.backward()
    cot = pkg.PhysicsTendency(torch.zeros_like(w), torch.zeros_like(w), w,
                              torch.ones_like(w))
    gs, gp = pkg.adjoint.vjp(phys, state, forcing, geom, date, cot)
    assert torch.allclose(state.temperature.grad, gs.temperature)
    assert torch.allclose(state.geopotential.grad, gs.geopotential)
    assert torch.allclose(params.grad, gp.cpu())
