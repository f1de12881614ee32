"""The reference arm's CPU sample (bench.py): the reference spends more per
PML point than per interior point, so the 160 x 160 x 100 sub-grid it times
runs the PML thickness whose share of PML points matches the full
400 x 400 x 200 workload's (12 layers there) instead of the workload's own
12 layers, which would make PML points 36 % of the sample against 17 %."""

import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_pml_point_fraction_counts_five_faces():
    # x and y both sides, z only at the bottom (the top is the free surface)
    assert bench.pml_point_fraction(10, 10, 10, 0) == 0.0
    assert bench.pml_point_fraction(10, 10, 10, 1) == pytest.approx(1 - 8 * 8 * 9 / 1000)
    assert bench.pml_point_fraction(400, 400, 200, 12) == pytest.approx(0.169416)


def test_sample_pml_matches_workload_share():
    n = bench.sample_npml((160, 160, 100))
    assert n == 5
    full = bench.pml_point_fraction(400, 400, 200, 12)
    got = bench.pml_point_fraction(160, 160, 100, n)
    assert abs(got - full) < 0.01
    # every other thickness is further from the workload's share
    for m in range(1, 13):
        assert abs(bench.pml_point_fraction(160, 160, 100, m) - full) >= abs(got - full)
