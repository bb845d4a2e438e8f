"""Builds ``tests/golden/reference_goldens.npz`` from the JAX-GCM sources.

The reference's own known-answer tests for the SPEEDY physics hold their expected values as
literal arrays inside ``jcm/physics/speedy/*_test.py`` and as Fortran-derived ``.npy`` files in
``jcm/data/test``.  This script reads the test files as text with :mod:`ast` (nothing in them
is executed), collects every numeric list literal of each test function in source order, and
stores it under ``"<file>::<function>::<n>"``; the ``.npy`` arrays are stored under
``"npy::<name>"``.  The fixture is small and committed, because the reference tree is not
available where the GPU tests run.

Usage:  python tests/golden/make_golden.py /path/to/jax-gcm
"""
import ast
import json
import sys
from pathlib import Path

import numpy as np

FILES = ["convection_test.py", "large_scale_condensation_test.py",
         "shortwave_radiation_test.py", "longwave_radiation_test.py", "surface_flux_test.py",
         "vertical_diffusion_test.py", "orographic_correction_test.py"]
NPY = ["iptop", "qdif", "cbmf", "precnv", "dfse", "dfqa"]


def _numeric(node):
    try:
        val = ast.literal_eval(node)
    except Exception:
        return None
    arr = np.asarray(val)
    if arr.dtype.kind in "if" and arr.size > 0:
        return arr.astype(np.float64)
    return None


def _outermost_lists(fn):
    """Numeric list literals of a function body, outermost only, in source order."""
    found = []

    def visit(node):
        if isinstance(node, ast.List):
            arr = _numeric(node)
            if arr is not None:
                found.append((node.lineno, node.col_offset, arr))
                return
        for child in ast.iter_child_nodes(node):
            visit(child)

    visit(fn)
    found.sort(key=lambda t: (t[0], t[1]))
    return found


def _scalar_assignments(fn):
    """``name = <number>`` and ``name = jnp.array(<number>)`` assignments of a function."""
    out = {}
    for node in ast.walk(fn):
        if isinstance(node, ast.Assign) and len(node.targets) == 1 and isinstance(
                node.targets[0], ast.Name):
            val = node.value
            if isinstance(val, ast.Call) and len(val.args) == 1:
                val = val.args[0]
            try:
                v = ast.literal_eval(val)
            except Exception:
                continue
            if isinstance(v, (int, float)) and not isinstance(v, bool):
                out[node.targets[0].id] = np.float64(v)
    return out


def _float_constants(fn):
    """Every float literal of a function body, in source order."""
    consts = [(n.lineno, n.col_offset, n.value) for n in ast.walk(fn)
              if isinstance(n, ast.Constant) and isinstance(n.value, float)]
    consts.sort()
    return np.asarray([c[2] for c in consts], dtype=np.float64)


def main(root):
    root = Path(root)
    speedy = root / "jcm" / "physics" / "speedy"
    out, manifest = {}, {}
    for fname in FILES:
        tree = ast.parse((speedy / fname).read_text())
        for node in ast.walk(tree):
            if isinstance(node, ast.FunctionDef) and node.name.startswith("test"):
                for n, (line, _, arr) in enumerate(_outermost_lists(node)):
                    key = f"{fname[:-3]}::{node.name}::{n}"
                    out[key] = arr
                    manifest[key] = {"shape": list(arr.shape), "line": line}
                for name, v in _scalar_assignments(node).items():
                    key = f"{fname[:-3]}::{node.name}::assign::{name}"
                    out[key] = v
                    manifest[key] = {"value": float(v)}
                consts = _float_constants(node)
                if consts.size:
                    key = f"{fname[:-3]}::{node.name}::floats"
                    out[key] = consts
                    manifest[key] = {"shape": list(consts.shape)}
    for name in NPY:
        arr = np.load(root / "jcm" / "data" / "test" / f"{name}.npy")
        out[f"npy::{name}"] = arr
        manifest[f"npy::{name}"] = {"shape": list(arr.shape), "dtype": str(arr.dtype)}
    here = Path(__file__).resolve().parent
    np.savez_compressed(here / "reference_goldens.npz", **out)
    (here / "reference_goldens_manifest.json").write_text(json.dumps(manifest, indent=1) + "\n")
    print(f"wrote {len(out)} arrays")


if __name__ == "__main__":
    if len(sys.argv) != 2:
        sys.exit("usage: python tests/golden/make_golden.py <path of the JAX-GCM checkout>")
    main(sys.argv[1])
