"""CPU checks of the C ABI: the library loads, exports every declared entry point, validates
arguments before touching a GPU, and its parameter defaults agree with the reference's."""
import ctypes as C
import importlib
import os
import re

import numpy as np
import pytest

from tests.helpers import fake_fields

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def pkg():
    return importlib.import_module("jax-gcm_b200")


@pytest.fixture(scope="module")
def lib(pkg):
    path = pkg._lib.LIB_PATH
    if not os.path.exists(path):
        import __graft_entry__
        __graft_entry__.build()
    return pkg._lib.load()


def declared_functions():
    names = []
    for fn in sorted(os.listdir(os.path.join(ROOT, "include"))):
        if fn.endswith(".h"):
            text = open(os.path.join(ROOT, "include", fn)).read()
            text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
            names += re.findall(r"^\s*(?:const\s+)?[a-z_0-9]+\s*\*?\s*(spd_[a-z_0-9]+)\s*\(",
                                text, flags=re.M)
    return sorted(set(names))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "spd_fwd" in names and "spd_fwd_scratch_bytes" in names


def test_library_exports_every_declared_symbol(lib):
    for name in declared_functions():
        assert hasattr(lib, name), name


def test_abi_version(lib):
    assert lib.spd_abi_version() == 1


def test_default_params_match_reference_defaults(pkg, lib):
    from oracle import speedy_oracle as O
    p = pkg._lib.Params()
    lib.spd_default_params(C.byref(p))
    mine = pkg.Parameters.default().to_struct()
    flat = {}
    for g, d in O.PARAM_DEFAULTS.items():
        flat.update(d)
    for name in pkg._lib.PARAM_FIELDS:
        assert getattr(p, name) == np.float32(flat[name]), name
        assert getattr(mine, name) == np.float32(flat[name]), name


def test_struct_sizes_match_header(pkg):
    L = pkg._lib
    assert C.sizeof(L.Desc) == 40
    assert C.sizeof(L.VGrid) == 4 * (17 + 5 * 16 + 32)
    assert C.sizeof(L.Params) == 4 * 57
    assert C.sizeof(L.Inputs) == 8 * 17
    assert C.sizeof(L.Outputs) == 8 * 21


def test_scratch_bytes(pkg, lib):
    """The forward's scratch is one 256-byte header (launch words and the instance's level-set
    state), whatever the grid; the adjoint's holds a one-member plan and grows with it."""
    for shape in ((8, 96, 48), (16, 1280, 640)):
        d = pkg._lib.Desc(*shape, 0, 0.2, 1950, 0, 1950, 1800.0, 1.0)
        assert lib.spd_fwd_scratch_bytes(C.byref(d)) == 256
    small = pkg._lib.Desc(8, 96, 48, 0, 0.2, 1950, 0, 1950, 1800.0, 1.0)
    large = pkg._lib.Desc(16, 1280, 640, 0, 0.2, 1950, 0, 1950, 1800.0, 1.0)
    a, b = lib.spd_vjp_scratch_bytes(C.byref(small)), lib.spd_vjp_scratch_bytes(C.byref(large))
    assert a % 256 == 0 and b > a


def test_argument_validation_needs_no_gpu(pkg, lib):
    L = pkg._lib
    d = L.Desc(8, 96, 48, 0, 0.2, 1950, 0, 1950, 1800.0, 1.0)
    vg, pr, inp, out = L.VGrid(), L.Params(), L.Inputs(), L.Outputs()
    rc = lib.spd_fwd(None, C.byref(vg), C.byref(pr), C.byref(inp), C.byref(out), None, 0, None)
    assert rc == 1
    rc = lib.spd_fwd(C.byref(d), C.byref(vg), C.byref(pr), C.byref(inp), C.byref(out), None, 0,
                     None)
    assert rc == 1  # null field pointers
    d.kx = 9
    rc = lib.spd_fwd(C.byref(d), C.byref(vg), C.byref(pr), C.byref(inp), C.byref(out), None, 0,
                     None)
    assert rc == 3
    assert lib.spd_status_string(3).decode().startswith("unsupported")


def test_overlapping_outputs_are_rejected(pkg, lib):
    L = pkg._lib
    d = L.Desc(8, 16, 8, 0, 0.2, 1950, 0, 1950, 1800.0, 1.0)
    vg, pr = L.VGrid(), L.Params()
    call = lambda i, o: lib.spd_fwd(C.byref(d), C.byref(vg), C.byref(pr), C.byref(i), C.byref(o),
                                    None, 0, None)
    inp, out = fake_fields(L)
    assert call(inp, out) == 4  # disjoint: reaches the scratch check
    inp, out = fake_fields(L)
    out.temperature = inp.temperature  # in-place update
    assert call(inp, out) == 9
    inp, out = fake_fields(L)
    out.cbmf = out.precls + 16
    assert call(inp, out) == 9  # a diagnostic overlapping a required output
    inp, out = fake_fields(L)
    out.evap = inp.coa - 16
    assert call(inp, out) == 9  # a diagnostic running into a latitude table
    assert lib.spd_status_string(9).decode().startswith("an output field overlaps")


def test_vjp_argument_validation_needs_no_gpu(pkg, lib):
    """spd_vjp's checks, in order: null arguments, the instance and its cotangent and gradient
    planes, the scratch (present, 256-byte aligned, large enough), the level count.  Every call
    here fails a check, so no device work is attempted on the fake addresses."""
    L = pkg._lib
    d = L.Desc(8, 16, 8, 0, 0.2, 1950, 0, 1950, 1800.0, 1.0)
    vg, pr = L.VGrid(), L.Params()
    inp, _ = fake_fields(L)
    base = 1 << 40
    cts = ("u_wind", "v_wind", "temperature", "specific_humidity")
    grs = cts + ("geopotential", "normalized_surface_pressure", "params")
    ct = L.Cotangents(**{k: base + i * (1 << 28) for i, k in enumerate(cts)})
    gr = L.Grads(**{k: base + (4 + i) * (1 << 28) for i, k in enumerate(grs)})
    n = lib.spd_vjp_scratch_bytes(C.byref(d))
    assert n > 0 and n % 256 == 0

    def call(desc, scratch, nbytes):
        return lib.spd_vjp(C.byref(desc) if desc is not None else None, C.byref(vg),
                           C.byref(pr), C.byref(inp), C.byref(ct), C.byref(gr),
                           C.c_void_p(scratch) if scratch else None, nbytes, None)

    assert call(None, 1 << 32, n) == 1
    assert call(d, None, n) == 4
    assert call(d, (1 << 32) + 16, n) == 4      # misaligned
    assert call(d, 1 << 32, n - 256) == 4       # too small
    d.kx = 9
    assert call(d, 1 << 32, n) == 3
    d.kx = 8
    ct.temperature = None
    assert call(d, 1 << 32, n) == 1


def test_product_path_fails_loudly_without_library(pkg, monkeypatch):
    monkeypatch.setattr(pkg._lib, "_lib", None)
    monkeypatch.setattr(pkg._lib, "LIB_PATH", "/nonexistent/libspeedy_b200.so")
    with pytest.raises(pkg._lib.SpeedyLibraryError):
        pkg._lib.load()


def test_vertical_tables_match_oracle(pkg):
    from oracle import speedy_oracle as O
    for kx in (7, 8, 16):
        a = pkg.physics.initialize_vertical(kx)
        b = O.vertical_tables(kx)
        for x, y in zip(a, b):
            np.testing.assert_array_equal(x, y)
