"""The static operation count of the column physics (``oracle/op_count.py``): per column it is
affine in the level count, and its headline figures are the ones the roofline discussion
quotes (8 exponentials per level and 6 per column; 6 divisions per level and 16 per column)."""
import pytest

from oracle import op_count


@pytest.fixture(scope="module")
def fit():
    return op_count.per_level_fit(8, 16)


def test_counts_are_affine_in_the_level_count(fit):
    c7 = op_count.count(7)
    for name, (a, b) in fit.items():
        if name in ("sin", "cos", "arccos", "arcsin"):  # per-latitude work, level-independent
            continue
        assert c7.get(name, 0.0) == pytest.approx(a * 7 + b, abs=0.15), name


def test_transcendental_and_division_counts(fit):
    a, b = fit["exp"]
    assert (round(a, 2), round(b, 2)) == (8.0, 6.0)
    a, b = fit["divide"]
    assert round(a) == 6 and round(b) == 16
    assert fit["sqrt"][0] == pytest.approx(0.0, abs=1e-6)


def test_counting_follows_every_operation():
    ops = op_count.count(8, ix=8, il=4)
    tr, dv, other = op_count.classes(ops)
    assert tr > 60 and dv > 40 and other > 2000
