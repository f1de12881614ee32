"""The reference's CPU-runnable benchmark case at full size and length.

128 x 128 x 96 points, homogeneous half-space with a flat free surface,
12-layer PML, an Mxy point source (finite-fault file) with a 2 Hz Ricker rate
at 3 km depth, 1000 RK4 steps, 16 surface stations.  tests/golden/
c1_halfspace.npz holds the reference's own CPU build's results for it and the
FP64 oracle's (tests/golden/make_golden_c1.py made both).

The exact build must reproduce the reference bit for bit over all 1000 steps;
the fast build (the benched one, FMA contraction) stays within 1e-5 relative
L2 on seismograms, and on the final surface velocities (a residue after the
waves have left) within twice the reference FP32 build's own distance from
FP64.  Against the FP64 oracle:
the library's FP64 run agrees to the fixture's float32 rounding, the FP32
builds are within 1e-5 (as close as the reference's own FP32 build), and the
mixed-precision storage within 1e-3.
"""

import json
import os
import tempfile

import numpy as np
import pytest

import parity_util as pu
from cgfdm import Session, cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLD = os.path.join(ROOT, "tests", "golden", "c1_halfspace.npz")


@pytest.fixture(scope="module")
def c1():
    if not os.path.exists(GOLD):
        pytest.skip("tests/golden/c1_halfspace.npz not generated")
    gold = np.load(GOLD)
    d = tempfile.mkdtemp(prefix="c1_")
    cases.write_case(cases.halfspace_case(), d)
    return d, gold


def _run(d, flavor, options=None):
    with Session(d, options=options, flavor=flavor) as s:
        assert s.info.NT == 1000
        s.run(s.info.NT)
        W = s.wavefield()
        return s.stations(), s.pgv(), W[W.shape[0] - 4]


@pytest.mark.gpu
def test_c1_exact_bitwise(c1):
    d, gold = c1
    st, pgv, wz = _run(d, "exact")
    np.testing.assert_array_equal(st, gold["stations"])
    np.testing.assert_array_equal(pgv, gold["PGV"])
    np.testing.assert_array_equal(wz, gold["W_plane_z"])


@pytest.mark.gpu
def test_c1_fast_tolerance(c1):
    """Seismograms within 1e-5 of the reference.  The final surface plane is a
    residue 1e-4 of the peak velocity after the waves have left through the
    PML; there the reference's own FP32 build is 7e-5 from the FP64 oracle, so
    the fast build is held to being as close to FP64 as that (within 2x)."""
    d, gold = c1
    st, pgv, wz = _run(d, "fast")
    e_st = pu.rel_l2(st[:, :, :3], gold["stations"][:, :, :3])
    w64 = gold["W_plane_z64"].astype(np.float64)
    e_w = pu.rel_l2(wz[:, :, :3], w64)
    e_w_ref = pu.rel_l2(gold["W_plane_z"][:, :, :3], w64)
    print(f"C1 fast vs reference: stations {e_st:.2e}; final surface velocity vs FP64: fast {e_w:.2e}, "
          f"reference FP32 {e_w_ref:.2e}")
    assert e_st <= 1e-5
    assert e_w <= 2 * e_w_ref


@pytest.mark.gpu
def test_c1_against_fp64(c1):
    d, gold = c1
    st64_ref = gold["stations64"].astype(np.float64)
    with Session(d) as s:
        st64, _, _ = s.run_precise(s.info.NT, bits=64)
    e_gpu64 = pu.rel_l2(st64[:, :, :3], st64_ref)
    e_ref32 = pu.rel_l2(gold["stations"][:, :, :3], st64_ref)
    errs = {}
    for name, flavor, opts in (("fast", "fast", None), ("exact", "exact", None),
                               ("fp16 storage", "fast", json.dumps({"storage": "fp16"}))):
        st, _, _ = _run(d, flavor, opts)
        errs[name] = pu.rel_l2(st[:, :, :3], st64_ref)
    print(f"C1 vs FP64 oracle: GPU FP64 {e_gpu64:.2e}, reference FP32 {e_ref32:.2e}, "
          + ", ".join(f"{k} {v:.2e}" for k, v in errs.items()))
    assert e_gpu64 <= 1e-6
    assert errs["fast"] <= 1e-5 and errs["exact"] <= 1e-5
    assert errs["exact"] <= 2 * e_ref32 + 1e-9
    assert errs["fp16 storage"] <= 1e-3
