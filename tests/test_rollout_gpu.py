"""The 48-step column rollout and its checkpointed adjoint on the GPU (jax-gcm_b200/rollout.py):

* checkpoints every 8 steps give bitwise the state gradient of storing every state (the
  recomputed forward is deterministic), and the parameter gradient up to the order of its
  atomic sums;
* on single-column instances (whose cloud-top level set is the column's own), the float32 GPU
  rollout's gradients agree with the float64 host rollout (tests/host/host_column.cpp)
  normwise within 1e-4, state and parameters alike, after 48 steps of float32 against float64
  through threshold-driven physics (measured: ~1e-6 for the state, ~1e-5 for the parameters).
"""
import ctypes as C
import importlib

import numpy as np
import pytest
import torch

from tests.test_adjoint_cpu import build_host, column_of, run_oracle, structs

pytestmark = pytest.mark.gpu

pkg = importlib.import_module("jax-gcm_b200")
R = pkg.rollout


@pytest.fixture(scope="module")
def host(tmp_path_factory):
    lib = build_host(tmp_path_factory.mktemp("hostroll") / "libhostroll.so")
    d = C.POINTER(C.c_double)
    lib.hc_rollout.restype = C.c_double
    lib.hc_rollout.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, d, C.c_int, C.c_double, d, d, d]
    return lib


def cotangent(shape, seed, device="cuda"):
    g = torch.Generator(device="cpu").manual_seed(seed)
    return pkg.PhysicsTendency(*(torch.randn(shape, generator=g).to(device) for _ in range(4)))


def test_checkpointed_equals_stored():
    inst = pkg.synthetic.land_instance(41, 32, 16, 8)
    st, fo, ge, da = pkg.instance_to_device(inst, "cuda")
    ct = cotangent(tuple(st.temperature.shape), 1)
    f8, g8, p8 = R.rollout_vjp(None, st, fo, ge, da, ct, nsteps=48, checkpoint_every=8)
    f1, g1, p1 = R.rollout_vjp(None, st, fo, ge, da, ct, nsteps=48, checkpoint_every=1)
    for k in ("u_wind", "v_wind", "temperature", "specific_humidity"):
        assert torch.equal(getattr(f8, k), getattr(f1, k))
    for k in ("u_wind", "v_wind", "temperature", "specific_humidity", "geopotential",
              "normalized_surface_pressure"):
        assert torch.equal(getattr(g8, k), getattr(g1, k)), k
    # the parameter gradient sums every column's contribution with atomics (order not fixed),
    # and some of its entries cancel: compare normwise
    assert float((p8 - p1).abs().max()) <= 1e-5 * float(p1.abs().max())


def one_column(inst, i, j):
    sub = pkg.synthetic.land_instance(0, 1, 1, inst.kx)
    for n in ("u", "v", "t", "q", "phi"):
        setattr(sub, n, np.ascontiguousarray(getattr(inst, n)[:, i:i + 1, j:j + 1]))
    for n in ("psa", "sst", "stl", "soilw", "snowc", "sice", "alb0", "fmask", "orog", "phis0"):
        setattr(sub, n, np.ascontiguousarray(getattr(inst, n)[i:i + 1, j:j + 1]))
    for n in ("lat", "sia", "coa"):
        setattr(sub, n, np.ascontiguousarray(getattr(inst, n)[j:j + 1]))
    return sub


def rollout_columns_against_host(host, inst, columns, seed, params=None):
    """48-step rollout VJPs of single-column instances cut from ``inst`` on the GPU (float32)
    and on the host (float64), with the parameter overrides ``params`` ({"group.name": value});
    returns the normwise errors of the state gradients by field and of the 12 parameter
    gradients."""
    kx = inst.kx
    if params:
        P = pkg.Parameters.default().with_values(
            **{k.replace(".", "__"): v for k, v in params.items()})
        from oracle import speedy_oracle as O
        tend, data = O.compute_tendencies(*inst.oracle_args(O.default_parameters(**params)))
        S = int(sum(1 << int(l) for l in np.nonzero(O.cloud_top_level_set(
            data.shortwave_rad.icltop, kx))[0]))
    else:
        P = pkg.Parameters.default()
        tend, data, S = run_oracle(inst)
    phys = pkg.SpeedyPhysics(P)
    vg, _ = structs(pkg, inst)
    pr = P.to_struct()
    rng = np.random.default_rng(seed)
    G, H, PG, PH = [], [], [], []
    for (i, j) in columns:
        sub = one_column(inst, i, j)
        st, fo, ge, da = pkg.instance_to_device(sub, "cuda")
        ctv = np.zeros((4, kx))
        ctv[0, -1], ctv[1, -1] = rng.normal(size=2)
        ctv[2], ctv[3] = rng.normal(size=kx), rng.normal(size=kx)
        ct = pkg.PhysicsTendency(*(torch.tensor(ctv[n], dtype=torch.float32, device="cuda")
                                   .view(kx, 1, 1) for n in range(4)))
        _, g, gp = R.rollout_vjp(phys, st, fo, ge, da, ct, nsteps=48)
        h = column_of(inst, data, S, i, j, 1 | 2 | 4)
        x0 = np.zeros(51)
        x0[:kx], x0[16:16 + kx], x0[32:32 + kx] = inst.t[:, i, j], inst.q[:, i, j], inst.phi[:, i, j]
        x0[48], x0[49], x0[50] = inst.psa[i, j], inst.u[-1, i, j], inst.v[-1, i, j]
        cth = np.zeros(34)
        cth[:kx], cth[16:16 + kx], cth[32], cth[33] = ctv[2], ctv[3], ctv[0, -1], ctv[1, -1]
        arr = lambda a: (C.c_double * len(a))(*a)
        hg, hp = (C.c_double * 51)(), (C.c_double * 12)()
        host.hc_rollout(C.byref(vg), C.byref(pr), C.byref(h), arr(x0), 48, 1800.0, arr(cth), hg,
                        hp)
        c = lambda t: t.detach().cpu().numpy().ravel().astype(np.float64)
        G.append(np.concatenate([c(g.temperature), c(g.specific_humidity), c(g.geopotential),
                                 c(g.normalized_surface_pressure), c(g.u_wind)[-1:],
                                 c(g.v_wind)[-1:]]))
        hg = np.array(hg[:])
        H.append(np.concatenate([hg[:kx], hg[16:16 + kx], hg[32:32 + kx], hg[48:51]]))
        PG.append(c(gp))
        PH.append(np.array(hp[:]))
    G, H, PG, PH = map(np.array, (G, H, PG, PH))
    segs = {"t": slice(0, kx), "q": slice(kx, 2 * kx), "phi": slice(2 * kx, 3 * kx),
            "psa": slice(3 * kx, 3 * kx + 1), "uv": slice(3 * kx + 1, 3 * kx + 3)}
    errs = {k: float(np.max(np.abs(G[:, s] - H[:, s])) / max(np.max(np.abs(H[:, s])), 1e-30))
            for k, s in segs.items()}
    perr = float(np.max(np.abs(PG - PH)) / np.max(np.abs(PH)))
    return errs, perr


@pytest.mark.parametrize("kx", [8, 16])
def test_single_column_rollout_matches_float64_host(host, kx):
    inst = pkg.synthetic.land_instance(700 + kx, 16, 8, kx)
    errs, perr = rollout_columns_against_host(
        host, inst, [(1, 2), (5, 3), (9, 6), (13, 1), (3, 7), (11, 4)], seed=kx)
    print("normwise errors", errs, "params", perr)
    assert all(e <= 1e-4 for e in errs.values()), errs
    assert perr <= 1e-4, perr


def test_t42_rollout_with_perturbed_parameters_matches_float64_host(host):
    """The adjoint workload's rollout: columns of the T42 instance (128 x 64, 8 levels, land and
    sea ice) with the 12 differentiated parameters scaled by seeded U(0.8, 1.2) factors, a
    48-step rollout VJP with checkpoints every 8 steps on the GPU against the float64 host
    rollout, column by column."""
    from tests.test_adjoint_config2_gpu import perturbed_parameters
    inst = pkg.synthetic.land_instance(42, 128, 64, 8, sst_noise=1.5)
    params = perturbed_parameters(pkg, seed=6)
    cols = [(3, 5), (17, 60), (40, 31), (77, 12), (101, 47), (126, 20), (64, 2), (90, 58)]
    errs, perr = rollout_columns_against_host(host, inst, cols, seed=42, params=params)
    print("T42 perturbed rollout normwise errors", errs, "params", perr)
    assert all(e <= 1e-4 for e in errs.values()), errs
    assert perr <= 1e-4, perr
