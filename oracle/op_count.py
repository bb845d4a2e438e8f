"""Static operation count of the column physics, taken from the NumPy restatement.

TEST INFRASTRUCTURE ONLY (like the rest of ``oracle/``): it runs ``speedy_oracle`` once on a
small grid with every input array wrapped in a counting ndarray subclass, and tallies the
elements each NumPy operation produces (``exp``, ``log``, ``divide``, ``multiply`` ...).
Divided by the column count, these are the operations per column of the reference's
arithmetic; two level counts give each operation as ``a * kx + b`` per column.

What the counts mean: the restatement evaluates both branches of every ``where`` (as the
reference's jax.numpy code does), so branch-heavy terms (convection's trigger levels, the
surface's land/sea branches, the cloud-top level set) are counted for every column; a
per-column kernel that branches executes fewer.  The per-latitude work (insolation, ozone,
zenith) is counted once per latitude and spread over the columns.  Reductions count one
operation per input element.

    python -m oracle.op_count          # the table for 8 and 16 levels
"""
from __future__ import annotations

import collections

import numpy as np

from oracle import speedy_oracle as O

# operation classes: what a GPU executes for them
TRANSCENDENTAL = ("exp", "log", "sqrt", "power", "sin", "cos", "arcsin", "arccos", "tanh")
DIVISION = ("divide", "true_divide", "reciprocal")


class _Tally:
    def __init__(self):
        self.ops = collections.Counter()


_TALLY = _Tally()


def _plain(x):
    return x.view(np.ndarray) if isinstance(x, Counted) else x


def _wrap(x):
    if isinstance(x, np.ndarray) and not isinstance(x, Counted):
        return x.view(Counted)
    if isinstance(x, tuple):
        return tuple(_wrap(v) for v in x)
    if isinstance(x, list):
        return [_wrap(v) for v in x]
    return x


class Counted(np.ndarray):
    """An ndarray that adds the size of every operation's result to the running tally."""

    def __array_ufunc__(self, ufunc, method, *inputs, **kwargs):
        args = [_plain(a) for a in inputs]
        if "out" in kwargs:
            kwargs["out"] = tuple(_plain(o) for o in kwargs["out"])
        res = getattr(ufunc, method)(*args, **kwargs)
        if method == "__call__":
            n = max((np.size(r) for r in (res if isinstance(res, tuple) else (res,))), default=0)
        else:  # reduce / accumulate: one operation per input element
            n = np.size(args[0])
        _TALLY.ops[ufunc.__name__] += int(n)
        return _wrap(res)

    def __array_function__(self, func, types, args, kwargs):
        def unwrap(v):
            if isinstance(v, Counted):
                return v.view(np.ndarray)
            if isinstance(v, (list, tuple)):
                return type(v)(unwrap(x) for x in v)
            return v
        res = func(*unwrap(args), **{k: unwrap(v) for k, v in kwargs.items()})
        if func is np.where and len(args) == 3:
            _TALLY.ops["where"] += int(np.size(res))
        elif func in (np.cumsum, np.sum, np.max, np.min, np.diff):
            _TALLY.ops[func.__name__] += int(np.size(args[0]))
        return _wrap(res)


def _counted(ns):
    for k, v in list(vars(ns).items()):
        if isinstance(v, np.ndarray):
            setattr(ns, k, v.view(Counted))
    return ns


def count(kx, ix=16, il=8, seed=3, orographic=False):
    """Operations per column, {name: count}, of one compute_tendencies call on a synthetic
    land column set (shortwave on) with ``kx`` levels."""
    import importlib
    pkg = importlib.import_module("jax-gcm_b200")
    inst = pkg.synthetic.land_instance(seed, ix, il, kx)
    st, fo, ge, da, params = inst.oracle_args(O.default_parameters())
    st, fo, ge = _counted(st), _counted(fo), _counted(ge)
    saved = np.asarray
    np.asarray = np.asanyarray  # keep the counting subclass through the restatement's asarray
    try:
        _TALLY.ops.clear()
        O.compute_tendencies(st, fo, ge, da, params, orographic=orographic)
        ops = dict(_TALLY.ops)
    finally:
        np.asarray = saved
    cols = ix * il
    return {k: v / cols for k, v in sorted(ops.items())}


def per_level_fit(kx_a=8, kx_b=16, **kw):
    """{name: (a, b)} with count(kx) = a * kx + b per column, from two level counts."""
    ca, cb = count(kx_a, **kw), count(kx_b, **kw)
    out = {}
    for k in sorted(set(ca) | set(cb)):
        ya, yb = ca.get(k, 0.0), cb.get(k, 0.0)
        a = (yb - ya) / (kx_b - kx_a)
        out[k] = (a, ya - a * kx_a)
    return out


def classes(ops):
    """(transcendental, division, other) totals of one count()."""
    tr = sum(v for k, v in ops.items() if k in TRANSCENDENTAL)
    dv = sum(v for k, v in ops.items() if k in DIVISION)
    other = sum(ops.values()) - tr - dv
    return tr, dv, other


if __name__ == "__main__":
    fit = per_level_fit()
    print(f"{'operation':<16}{'per level':>12}{'per column':>12}{'kx=8':>10}{'kx=16':>10}")
    for k, (a, b) in fit.items():
        print(f"{k:<16}{a:>12.2f}{b:>12.2f}{a * 8 + b:>10.1f}{a * 16 + b:>10.1f}")
    for kx in (8, 16):
        tr, dv, other = classes(count(kx))
        print(f"kx={kx}: transcendental {tr:.1f}, division {dv:.1f}, other {other:.1f} per column")
