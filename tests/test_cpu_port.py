"""The compiled CPU restatement of the reference (oracle/cpu_port.cpp), which the benchmark
times as its CPU baseline and reference arm, against the NumPy oracle under the same parity
bar as the CUDA path (tests/helpers.py): it must compute what it claims to time."""
import importlib

import numpy as np
import pytest

from oracle import cpu_port
from tests.helpers import check_against_oracle


@pytest.fixture(scope="module")
def pkg():
    return importlib.import_module("jax-gcm_b200")


@pytest.mark.parametrize("lfluxland", [False, True])
def test_t31_aquaplanet(pkg, lfluxland):
    inst = pkg.synthetic.config0_instance(seed=11, lfluxland=lfluxland)
    got = cpu_port.Prepared(inst).run()
    check_against_oracle(inst, got)


@pytest.mark.parametrize("kx", [8, 16])
def test_land_member_with_sea_ice(pkg, kx):
    inst = pkg.synthetic.land_instance(300 + kx, 128, 64, kx, sst_noise=1.5)
    got = cpu_port.Prepared(inst).run(nthreads=2)
    check_against_oracle(inst, got)


def test_repeat_runs_and_thread_counts_agree(pkg):
    inst = pkg.synthetic.land_instance(5, 64, 32, 16)
    p = cpu_port.Prepared(inst)
    a = {k: v.copy() for k, v in p.run(nthreads=1).items()}
    b = p.run(nthreads=4)
    for k in a:
        assert np.array_equal(a[k], b[k]), k


def test_batch_equals_single_instances(pkg):
    """One parallel region over several instances of mixed level counts gives each instance
    exactly what its own call gives."""
    insts = [pkg.synthetic.land_instance(600 + i, ix, il, kx)
             for i, (ix, il, kx) in enumerate([(64, 32, 8), (32, 16, 16), (96, 48, 16)])]
    single = [{k: v.copy() for k, v in cpu_port.Prepared(i).run(nthreads=3).items()}
              for i in insts]
    b = cpu_port.Batch(insts)
    b.run(nthreads=5)
    for s, p in zip(single, b.items):
        for k, name in (("u_wind", "du"), ("temperature", "dt"), ("specific_humidity", "dq"),
                        ("precnv", "precnv"), ("icltop", "icltop")):
            assert np.array_equal(s[k], p.out[name]), k
