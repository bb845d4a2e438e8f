"""The forward's packed float32 pieces (sm_100 .f32x2 pairs) against the scalar expressions
they pair, bit for bit (spd_selftest_packed, compiled with the forward's flags).  The forward's
results rest on this: the packed build gives the bits of the separately rounded scalar
arithmetic the parity tests pin."""
import ctypes as C
import importlib

import pytest

pytestmark = pytest.mark.gpu

PIECES = ["longwave down", "longwave up", "band fractions", "half-level temperatures",
          "blackbody terms", "shortwave band 1", "shortwave band 2", "heating-rate scaling"]


@pytest.mark.parametrize("seed", [1, 20261204])
def test_packed_pieces_equal_scalar_expressions(seed):
    lib = importlib.import_module("jax-gcm_b200._lib").load()
    out = (C.c_uint * len(PIECES))()
    assert lib.spd_selftest_packed(1 << 20, seed, out) == 0
    assert dict(zip(PIECES, out)) == {p: 0 for p in PIECES}


def test_selftest_argument_errors():
    lib = importlib.import_module("jax-gcm_b200._lib").load()
    out = (C.c_uint * len(PIECES))()
    assert lib.spd_selftest_packed(0, 1, out) == 2      # SPD_ERR_SHAPE
    assert lib.spd_selftest_packed(16, 1, None) == 1    # SPD_ERR_NULL
