"""The checkpointed reverse of the column rollout (jax-gcm_b200/rollout.py) and the float64
rollout reference of the host harness:

* ``checkpointed_reverse`` gives the same gradient for every checkpoint spacing and matches
  the analytic gradient of a toy map, holding ceil(N / spacing) + spacing - 1 states at most;
* the float64 48-step rollout VJP (hand-written reverse pass, fused verify step) agrees with
  float64 central differences of the rollout along random directions of the state and for the
  12 tuning parameters.
"""
import ctypes as C
import importlib
import math

import numpy as np
import pytest

from tests.test_adjoint_cpu import build_host, column_of, run_oracle, structs

pkg = importlib.import_module("jax-gcm_b200")
R = pkg.rollout


@pytest.fixture(scope="module")
def host(tmp_path_factory):
    lib = build_host(tmp_path_factory.mktemp("hostroll") / "libhostroll.so")
    d = C.POINTER(C.c_double)
    lib.hc_rollout.restype = C.c_double
    lib.hc_rollout.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, d, C.c_int, C.c_double, d, d, d]
    return lib


def toy_problem(n=5, seed=0):
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(n, n)) * 0.3
    b = rng.normal(size=n)

    def step(x, k):
        return x + 0.1 * np.sin(A @ x + b + 0.01 * k)

    def step_vjp(x, k, xb):
        return xb + 0.1 * A.T @ (np.cos(A @ x + b + 0.01 * k) * xb)

    return step, step_vjp, rng.normal(size=n), rng.normal(size=n)


@pytest.mark.parametrize("every", [1, 3, 8, 48, 100])
def test_checkpointed_reverse_spacing_invariant(every):
    step, step_vjp, x0, ct = toy_problem()
    N = 48
    ref_final, ref, _ = R.checkpointed_reverse(step, step_vjp, x0, ct, N, 1)
    final, xb, held = R.checkpointed_reverse(step, step_vjp, x0, ct, N, every)
    assert np.array_equal(final, ref_final)
    assert np.array_equal(xb, ref)
    e = min(every, N)
    assert held <= math.ceil(N / e) + e - 1


def test_checkpointed_reverse_matches_finite_differences():
    step, step_vjp, x0, ct = toy_problem(seed=2)
    N = 48
    _, xb, _ = R.checkpointed_reverse(step, step_vjp, x0, ct, N, 8)

    def loss(x):
        for k in range(N):
            x = step(x, k)
        return ct @ x

    h = 1e-6
    fd = np.array([(loss(x0 + h * e) - loss(x0 - h * e)) / (2 * h) for e in np.eye(len(x0))])
    assert np.allclose(fd, xb, rtol=1e-6, atol=1e-9)


def test_checkpointed_reverse_rejects_bad_spacing():
    step, step_vjp, x0, ct = toy_problem()
    with pytest.raises(ValueError):
        R.checkpointed_reverse(step, step_vjp, x0, ct, 4, 0)


def _column(kx, seed, i, j):
    inst = pkg.synthetic.land_instance(seed, 16, 8, kx)
    tend, data, S = run_oracle(inst)
    vg, pr = structs(pkg, inst)
    h = column_of(inst, data, S, i, j, 1 | 2 | 4)
    x0 = np.zeros(51)
    x0[:kx] = inst.t[:, i, j]
    x0[16:16 + kx] = inst.q[:, i, j]
    x0[32:32 + kx] = inst.phi[:, i, j]
    x0[48], x0[49], x0[50] = inst.psa[i, j], inst.u[-1, i, j], inst.v[-1, i, j]
    return vg, pr, h, x0


def _rollout(host, vg, pr, h, x0, ct, n, dt, grad=False):
    arr = lambda a: (C.c_double * len(a))(*a)
    g, gp = (C.c_double * 51)(), (C.c_double * 12)()
    loss = host.hc_rollout(C.byref(vg), C.byref(pr), C.byref(h), arr(x0), n, dt, arr(ct),
                           g if grad else None, gp if grad else None)
    return loss, np.array(g[:]), np.array(gp[:])


@pytest.mark.parametrize("kx", [8, 16])
def test_rollout_vjp_matches_float64_central_differences(host, kx):
    """48 steps of 1800 s.  Directional check with d = 1e-6 |x| r along the state; a column
    whose rollout crosses a threshold inside the step is not differentiable there, so 3 of 4
    columns must agree to 1e-4."""
    rng = np.random.default_rng(kx)
    good = 0
    for n_col, (i, j) in enumerate([(1, 2), (5, 3), (9, 6), (13, 1)]):
        vg, pr, h, x0 = _column(kx, 700 + kx, i, j)
        ct = np.zeros(34)
        ct[:kx] = rng.normal(size=kx)
        ct[16:16 + kx] = rng.normal(size=kx)
        ct[32:34] = rng.normal(size=2)
        _, g, _ = _rollout(host, vg, pr, h, x0, ct, 48, 1800.0, grad=True)
        d = 1e-6 * np.abs(x0) * rng.normal(size=51)
        d[np.abs(x0) == 0] = 0.0
        lp = _rollout(host, vg, pr, h, x0 + d, ct, 48, 1800.0)[0]
        lm = _rollout(host, vg, pr, h, x0 - d, ct, 48, 1800.0)[0]
        fd = (lp - lm) / 2
        ad = float(g @ d)
        if abs(fd - ad) <= 1e-4 * max(abs(fd), abs(ad)):
            good += 1
    assert good >= 3, good


def test_rollout_parameter_gradients_match_central_differences(host):
    kx = 8
    vg, pr, h, x0 = _column(kx, 910, 4, 5)
    rng = np.random.default_rng(9)
    ct = np.zeros(34)
    ct[:kx] = rng.normal(size=kx)
    ct[16:16 + kx] = rng.normal(size=kx)
    _, _, gp = _rollout(host, vg, pr, h, x0, ct, 48, 1800.0, grad=True)
    names = ["psmin", "trcnv", "rhil", "rhbl", "entmax", "smf", "trlsc", "rhlsc", "drhlsc",
             "rhblsc", "albcl", "albcls"]
    good = 0
    for n, name in enumerate(names):
        base = getattr(pr, name)
        vals = []
        for sgn in (1, -1):
            setattr(pr, name, base + sgn * 1e-5 * abs(base))
            vals.append((_rollout(host, vg, pr, h, x0, ct, 48, 1800.0)[0], getattr(pr, name)))
        setattr(pr, name, base)
        fd = (vals[0][0] - vals[1][0]) / (vals[0][1] - vals[1][1])
        if abs(fd - gp[n]) <= 2e-3 * max(abs(fd), abs(gp[n])) + 1e-12:
            good += 1
    assert good >= 10, good
