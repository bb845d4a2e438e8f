"""spd_fwd_noalloc: the forward for callers that cannot allocate device scratch.

A foreign-function bridge that only forwards the buffers it was handed, or a process whose
device memory is owned by another runtime's allocator, cannot provide spd_fwd's scratch
buffer.  spd_fwd_noalloc keeps that scratch in a fixed array inside the library instead.  The
GPU test calls it through the C ABI twice in a row, on two different instances (so the
second call runs over the first call's leftovers in the shared array), and checks that both
results equal spd_fwd's bitwise: both entry points run the same two kernels over the same
one-member plan, so any difference would be a scratch offset or leftover-state fault.  This
file is collected last on purpose.
"""
import ctypes as C
import importlib

import numpy as np
import pytest

from tests.helpers import fake_fields, to_device


@pytest.fixture(scope="module")
def pkg():
    return importlib.import_module("jax-gcm_b200")


def _structs(pkg, inst, device):
    import torch
    state, forcing, geom, date = to_device(pkg, inst, device)
    phys = pkg.SpeedyPhysics(diagnostics=False)
    tensors = dict(u_wind=state.u_wind, v_wind=state.v_wind, temperature=state.temperature,
                   specific_humidity=state.specific_humidity, geopotential=state.geopotential,
                   normalized_surface_pressure=state.normalized_surface_pressure,
                   alb0=forcing.alb0, sice_am=forcing.sice_am, snowc_am=forcing.snowc_am,
                   soilw_am=forcing.soilw_am, stl_am=forcing.stl_am,
                   sea_surface_temperature=forcing.sea_surface_temperature, fmask=geom.fmask,
                   orog=geom.orog, phis0=geom.phis0, sia=geom.sia, coa=geom.coa)
    inp = pkg._lib.Inputs(**{k: tensors[k].data_ptr() for k in pkg._lib.INPUT_FIELDS})
    kx, ix, il = geom.nodal_shape
    out = {k: torch.full((kx, ix, il) if k in ("u_wind", "v_wind", "temperature",
                                               "specific_humidity") else (ix, il),
                         float("nan"), device=device)
           for k in ("u_wind", "v_wind", "temperature", "specific_humidity", "precnv",
                     "precls")}
    outs = pkg._lib.Outputs(**{k: (out[k].data_ptr() if k in out else None)
                               for k in pkg._lib.OUTPUT_FIELDS})
    desc = phys.desc(geom, date, forcing.lfluxland)
    return phys, (state, forcing, geom, date), tensors, inp, out, outs, desc


@pytest.mark.gpu
def test_noalloc_matches_spd_fwd_on_two_calls_in_a_row(pkg):
    import torch
    lib = pkg._lib.load()
    dev = torch.device("cuda", 0)
    insts = [pkg.synthetic.land_instance(41, 96, 48, 16),
             pkg.synthetic.land_instance(42, 64, 32, 8, sst_noise=1.5)]
    prepared = [_structs(pkg, inst, dev) for inst in insts]
    # the existing entry point (caller-provided scratch), as the reference result
    want = []
    for phys, args, _, _, _, _, _ in prepared:
        tend, data = phys.compute_tendencies(*args)
        want.append({"u_wind": tend.u_wind, "v_wind": tend.v_wind,
                     "temperature": tend.temperature,
                     "specific_humidity": tend.specific_humidity,
                     "precnv": data.convection.precnv, "precls": data.condensation.precls})
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    # two calls in a row through the C ABI, each over the shared fixed scratch
    for (phys, args, _, inp, out, outs, desc), ref in zip(prepared, want):
        geom = args[2]
        rc = lib.spd_fwd_noalloc(C.byref(desc), C.byref(geom.vgrid()),
                                 C.byref(phys._pstruct), C.byref(inp), C.byref(outs), stream)
        assert rc == 0, lib.spd_status_string(rc)
        torch.cuda.synchronize()
        for k, r in ref.items():
            g = out[k].cpu().numpy()
            assert np.all(np.isfinite(g)), k
            assert np.array_equal(g, r.cpu().numpy()), k


def test_noalloc_rejects_too_many_latitudes(pkg):
    """The fixed scratch bounds the latitude count; larger instances get a clear error
    before any device work."""
    lib = pkg._lib.load()
    L = pkg._lib
    il = L.NOALLOC_MAX_IL + 2
    desc = L.Desc(8, 4, il, 0, 0.2, 1950, 0, 1950, 1800.0, 1.0)
    # aligned, never dereferenced: the call returns before touching the GPU
    inp, outs = fake_fields(L)
    vg, pr = L.VGrid(), L.Params()
    rc = lib.spd_fwd_noalloc(C.byref(desc), C.byref(vg), C.byref(pr), C.byref(inp),
                             C.byref(outs), None)
    assert rc == 8
    assert "SPD_NOALLOC_MAX_IL" in lib.spd_status_string(rc).decode()
