"""The K2+Kf operation census (oracle/census.py) behind the benchmark's roofline: its
restatement of the oracle's FP64 path returns the oracle's values, and bench.py's
census constants are the census of the headline workload."""

from __future__ import annotations

import math

import numpy as np

import bench
import oracle
from oracle import census


def test_census_restatement_returns_the_oracles_values():
    r = oracle.r_grid(1e-7, 1e2, 399)
    N = oracle.mv_amplitude(r, 0.6)
    sp = oracle.loglog_spline(r, N, 1)
    sspl = census.Spline(sp.x, sp.a, sp.b, sp.c, sp.d, sp.rmin, sp.rmax)
    phys = oracle.physics(bench.workload_config())
    lower, width = oracle.nlo_box(r)
    rng = np.random.default_rng(11)
    for parent in (12, 150, 260, 330):
        for u in rng.uniform(0.0, 1.0, (40, 4)):
            x = lower + width * u
            want = oracle.k2kf_integrand(float(r[parent]), x, sp, phys)
            got = census.integrand(float(r[parent]), x, sspl, census.Physics())
            for a, b in zip(got, want):
                assert math.isclose(a, b, rel_tol=1e-12, abs_tol=1e-300), (parent, x, got, want)


def test_bench_census_constants_are_the_workload_census():
    c = census.workload_census()
    assert bench.CENSUS_EVAL_FLOPS == c["eval_arithmetic"]
    assert bench.CENSUS_EVAL_TRANSCENDENTALS == c["eval_special"]
    assert bench.CENSUS_SAMPLE_FLOPS == c["sample_arithmetic"]
    assert bench.CENSUS_SAMPLE_TRANSCENDENTALS == c["sample_special"]


def test_bench_dis_census_constants_are_the_workload_census():
    from oracle import census_dis

    c = census_dis.workload_census()
    assert bench.DIS_CENSUS == {"I2N": c["I2n"], "I3N": c["I3n"]}
