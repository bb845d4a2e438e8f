"""Parity of the batched ragged ensemble the benchmark times (32xT21, 16xT31, 8xT42, 4xT85 and
1xT170, 466,944 columns, members alternating 8 and 16 levels, seeds 1000 + member) with the
float32 and float64 oracles, member by member, through one spd_ensemble_fwd call and under
the bar of tests/helpers.py (elementwise 1e-5 above per-field floors, trigger flips counted)."""
import importlib

import numpy as np
import pytest

from tests.helpers import check_against_oracle, to_device

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pkg():
    return importlib.import_module("jax-gcm_b200")


def test_benchmark_ensemble_every_member(pkg):
    import torch
    insts = pkg.synthetic.ensemble_members(base_seed=1000)
    assert len(insts) == 61 and sum(m.columns for m in insts) == 466944
    members = []
    for inst in insts:
        st, fo, ge, da = to_device(pkg, inst, "cuda")
        kx, ix, il = inst.kx, inst.ix, inst.il
        out = {k: torch.empty((kx, ix, il), dtype=torch.float32, device="cuda")
               for k in ("u_wind", "v_wind", "temperature", "specific_humidity")}
        for k in ("precnv", "precls", "cloudc", "rsds", "rlds"):
            out[k] = torch.empty((ix, il), dtype=torch.float32, device="cuda")
        for k in ("iptop", "icltop"):
            out[k] = torch.empty((ix, il), dtype=torch.int32, device="cuda")
        members.append(pkg.Member(st, fo, ge, out))
    ens = pkg.Ensemble(members, da)
    ens.forward()
    torch.cuda.synchronize()
    totals = dict(columns=0, flip_columns=0, flip_columns_le_1ulp=0)
    worst = {}
    for inst, m in zip(insts, members):
        got = {k: v.cpu().numpy() for k, v in m.out.items()}
        _, summ = check_against_oracle(inst, got)
        for k in totals:
            totals[k] += summ[k]
        for k, f in summ["required_floors"].items():
            worst[k] = max(worst.get(k, 0.0), f)
    print("ensemble totals", totals, "largest required floors", worst)
    assert totals["columns"] == 466944
    assert totals["flip_columns"] <= 2e-3 * totals["columns"]
