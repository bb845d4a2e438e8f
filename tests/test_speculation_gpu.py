"""The forward's prediction of the cloud-top level set (the one cross-column dependency,
shortwave_radiation.py:62-68): a call uses the level set of the previous call on the same
scratch (or plan), checks it on the device and redoes the instance when it missed.  Whatever
the prediction, the results must equal those of the non-speculating forward (which forms the
level set first) bitwise: on a first call (nothing to predict from), on repeated calls, and
after a call on another instance whose level set differs."""
import importlib

import numpy as np
import pytest
import torch

from tests.helpers import run_gpu_instance, to_device

pytestmark = pytest.mark.gpu
FIELDS = ("u_wind", "v_wind", "temperature", "specific_humidity", "precnv", "precls")


@pytest.fixture(scope="module")
def pkg():
    return importlib.import_module("jax-gcm_b200")


def two_instances(pkg):
    """Two 4x2-column instances whose level sets differ: {1} (every column's cloud top at level
    1), and {1, 4} (one column moistened fivefold in its upper five levels condenses from level
    4 down, which moves its cloud top there)."""
    a = pkg.synthetic.config0_instance(seed=2, ix=4, il=2, lfluxland=True)
    b = pkg.synthetic.config0_instance(seed=2, ix=4, il=2, lfluxland=True)
    b.q[:5, 0, 0] = b.q[:5, 0, 0] * 5.0
    return a, b


def level_set(got, kx):
    return {int(min(max(x, 0), kx - 1)) for x in np.asarray(got["icltop"]).ravel()}


def test_plain_calls_equal_the_non_speculating_forward(pkg):
    a, b = two_instances(pkg)
    ref_a = run_gpu_instance(pkg, a, speculate=False)
    ref_b = run_gpu_instance(pkg, b, speculate=False)
    assert level_set(ref_a, a.kx) != level_set(ref_b, b.kx)
    phys = pkg.SpeedyPhysics(speculate=True)
    seq = [(a, ref_a), (a, ref_a), (b, ref_b), (b, ref_b), (a, ref_a)]
    for inst, ref in seq:  # first call, a hit, a miss, a hit, a miss
        st, fo, ge, da = to_device(pkg, inst, "cuda")
        tend, data = phys.compute_tendencies(st, fo, ge, da)
        torch.cuda.synchronize()
        got = dict(u_wind=tend.u_wind, v_wind=tend.v_wind, temperature=tend.temperature,
                   specific_humidity=tend.specific_humidity, precnv=data.convection.precnv,
                   precls=data.condensation.precls)
        for k in FIELDS:
            assert np.array_equal(got[k].cpu().numpy(), ref[k]), (inst.name, k)


def test_ensemble_prediction_misses_only_on_the_first_call(pkg):
    insts = [pkg.synthetic.land_instance(700 + i, ix, il, kx)
             for i, (ix, il, kx) in enumerate([(64, 32, 8), (64, 32, 16), (96, 48, 16),
                                               (7, 5, 8)])]

    def ensemble(speculate):
        members, date = [], None
        for inst in insts:
            st, fo, ge, date = to_device(pkg, inst, "cuda")
            members.append(pkg.Member(st, fo, ge))
        return pkg.Ensemble(members, date, speculate=speculate)

    ref = [{k: v.clone() for k, v in o.items()} for o in ensemble(False).forward()]
    ens = ensemble(True)
    for call in range(3):
        outs = ens.forward()
        torch.cuda.synchronize()
        for o, r in zip(outs, ref):
            for k in r:
                assert torch.equal(o[k], r[k]), (call, k)
        # the first call has no prediction: every member is redone once, and never again
        assert ens.redone() == len(insts)
    g = ens.capture(calls=2)
    g.replay()
    torch.cuda.synchronize()
    assert ens.redone() == len(insts)
    for o, r in zip([m.out for m in ens.members], ref):
        for k in r:
            assert torch.equal(o[k], r[k]), k


def test_large_instance_redo_strides_over_the_tiles(pkg):
    """A 1024-tile instance (more tiles than the GPU holds blocks at once): its first call
    misses, and the fixup launch -- one resident wave of blocks striding over the tiles --
    redoes every tile; a second call hits.  Both equal the non-speculating forward bitwise."""
    inst = pkg.synthetic.land_instance(77, 512, 256, 16)
    ref = run_gpu_instance(pkg, inst, speculate=False)
    phys = pkg.SpeedyPhysics(speculate=True)
    st, fo, ge, da = to_device(pkg, inst, "cuda")
    for call in range(2):
        tend, data = phys.compute_tendencies(st, fo, ge, da)
        torch.cuda.synchronize()
        got = dict(u_wind=tend.u_wind, v_wind=tend.v_wind, temperature=tend.temperature,
                   specific_humidity=tend.specific_humidity, precnv=data.convection.precnv,
                   precls=data.condensation.precls)
        for k in FIELDS:
            assert np.array_equal(got[k].cpu().numpy(), ref[k]), (call, k)
