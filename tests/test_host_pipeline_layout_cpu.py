"""The packed host/device layout of ``batched.HostPipeline`` (one flat buffer for every
member's state, one for every member's results) on the CPU: every field of every member gets
its own 256-byte-aligned range of the right shape, the ranges do not overlap, and the buffer
holds nothing else beyond the alignment padding."""
import importlib
from types import SimpleNamespace

pkg = importlib.import_module("jax-gcm_b200")
B = pkg.batched

SHAPES = [(8, 64, 32), (16, 96, 48), (8, 3, 5), (16, 512, 256), (7, 1, 1)]
LEVEL = {"temperature", "specific_humidity", "geopotential"}  # winds: lowest level only


def members():
    return [SimpleNamespace(geometry=SimpleNamespace(nodal_shape=s)) for s in SHAPES]


def check(fields):
    layout, total = B._packed_layout(members(), fields, LEVEL)
    assert len(layout) == len(SHAPES)
    ranges, payload = [], 0
    for (kx, ix, il), d in zip(SHAPES, layout):
        assert list(d) == list(fields)
        for f, (off, shape) in d.items():
            want = (kx, ix, il) if f in LEVEL else (ix, il)
            assert shape == want
            n = 1
            for s in shape:
                n *= s
            assert off % 64 == 0          # 64 floats = 256 bytes
            ranges.append((off, off + n))
            payload += n
    ranges.sort()
    for (a0, a1), (b0, b1) in zip(ranges, ranges[1:]):
        assert a1 <= b0                   # no two fields share a float
    assert ranges[-1][1] <= total
    assert total - payload < 64 * len(ranges)   # only alignment padding besides the fields


def test_state_layout():
    check(B.STATE_FIELDS)


def test_result_layout():
    check(B.RESULT_FIELDS)
