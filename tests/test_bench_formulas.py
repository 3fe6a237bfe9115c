"""The algorithmic work per pixel that bench.py divides by the measured
time (the roofline numerators), against the stated formulas at N = 10, 30
and 60: Gram 8 L N(N+1)/2, EVD 16N^3/3 + 8N^2 + 320N, EMI adds N^3 + 2N^2,
normalisation and gamma 30 N(N-1)/2; and the workloads' names.
"""

import pytest

import bench


@pytest.mark.parametrize("n,gram147,evd,emi", [
    (10, 64_680, 9_333.3, 10_533.3),
    (30, 546_840, 160_800.0, 189_600.0),
    (60, 2_152_080, 1_200_000.0, 1_423_200.0),
])
def test_flops_per_pixel(n, gram147, evd, emi):
    g, link_evd = bench.flops_per_pixel(n, 147, False)
    _, link_emi = bench.flops_per_pixel(n, 147, True)
    norm_gamma = 30.0 * n * (n - 1) / 2
    assert g == pytest.approx(gram147)
    assert link_evd - norm_gamma == pytest.approx(evd, rel=1e-4)
    assert link_emi - norm_gamma == pytest.approx(emi, rel=1e-4)


def test_workloads_are_named_by_their_settings():
    for key, w in bench.WORKLOADS.items():
        name = bench.workload_name(w["rows"], w["cols"], w)
        assert name.startswith("N=%d %dx%d %s/%s" % (w["n"], w["rows"], w["cols"], w["shp_test"],
                                                      w["estimator"]))
    assert bench.metric_name(bench.WORKLOAD) == bench.METRIC
