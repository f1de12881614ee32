"""The oracle's C restatement of the time-stepping path (oracle/restated/
stepper.c) against the reference's own CPU build, on the CPU.

In FP32 the CGFDM restatement reproduces the reference bit for bit (station
traces, final wavefield, PGV).  The ME-AWENO restatement differs only where
the characteristic free surface is restated with the inverse surface basis
instead of the reference's expanded float formulas, so it is held to 1e-6
relative L2.  The FP64 build, the FP64 oracle used for precision reports,
must agree with the reference's FP32 results to 1e-5 (the FP32 rounding
error over these short runs).  The mixed-storage build (FP16 stage and
accumulator deltas from the FP32 step state), the oracle of the library's
"storage": "fp16" path, must stay within the 1e-3 seismogram bound of the
FP64 oracle while differing from the FP32 build (it does round).
"""

import os

import numpy as np
import pytest

import parity_util as pu
import refrun
import restated
from cgfdm import cases

CASES = {
    "cg_multi_fault": (lambda: pu.multi_fault(steps=24), "CGFDM"),
    "cg_double_couple": (lambda: pu.double_couple(steps=24), "CGFDM"),
    "cg_hill": (lambda: pu.small_hill(steps=24), "CGFDM"),
    "sc_halfspace": (lambda: pu.small_halfspace(steps=16, courant=0.5), "SCFDM"),
    "sc_hill": (lambda: pu.small_hill(steps=16), "SCFDM"),
}


@pytest.fixture(scope="module")
def runs(tmp_path_factory):
    if not (restated.available() and refrun.available("CGFDM") and refrun.available("SCFDM")):
        pytest.skip("oracle builds (oracle/build, oracle/_ref) not present")
    root = tmp_path_factory.mktemp("rs")
    dirs = {}
    for name, (mk, scheme) in CASES.items():
        d = str(root / name)
        cases.write_case(mk(), d, scheme=scheme)
        dirs[name] = d
    for scheme in ("CGFDM", "SCFDM"):
        refrun.run_many([d for n, d in dirs.items() if CASES[n][1] == scheme], scheme)
    out = {}
    for name, d in dirs.items():
        scheme = CASES[name][1]
        b = restated.make_bundle(d, os.path.join(d, "bundle"), scheme)
        out[name] = (refrun.read_outputs(d, scheme), restated.run(b, "f32"), restated.run(b, "f64"))
    return out


@pytest.mark.parametrize("name", list(CASES))
def test_restated_fp32_matches_reference(runs, name):
    ref, r32, _ = runs[name]
    assert np.abs(ref["W"]).max() > 0
    if CASES[name][1] == "CGFDM":
        np.testing.assert_array_equal(r32["stations"], ref["stations"])
        np.testing.assert_array_equal(r32["W"], ref["W"])
        np.testing.assert_array_equal(r32["PGV"], ref["PGV"])
    else:
        assert pu.rel_l2(r32["stations"][:, :, :3], ref["stations"][:, :, :3]) <= 1e-6
        assert pu.rel_l2(r32["W"], ref["W"]) <= 1e-6
        assert pu.rel_l2(r32["PGV"], ref["PGV"]) <= 1e-6


@pytest.mark.parametrize("name", list(CASES))
def test_restated_fp64_near_reference(runs, name):
    ref, _, r64 = runs[name]
    assert pu.rel_l2(r64["stations"][:, :, :3], ref["stations"][:, :, :3]) <= 1e-5
    assert pu.rel_l2(r64["W"], ref["W"]) <= 1e-5



def test_restated_mixed_storage_near_fp64(tmp_path):
    """200 steps on the curvilinear hill, long enough for the direct waves to
    reach the stations (in the first few tens of steps the station signals
    are small beside the FP16 rounding noise radiated from the source)."""
    if not (restated.available() and refrun.available("CGFDM") and os.access(restated.binary("m16"), os.X_OK)):
        pytest.skip("oracle builds (oracle/build, oracle/_ref) not present")
    d = str(tmp_path / "hill")
    cases.write_case(pu.small_hill(steps=200), d)
    refrun.run(d, "CGFDM")
    b = restated.make_bundle(d, os.path.join(d, "bundle"), "CGFDM")
    r32, r64, m16 = restated.run(b, "f32"), restated.run(b, "f64"), restated.run(b, "m16")
    e = pu.rel_l2(m16["stations"][:, :, :3], r64["stations"][:, :, :3])
    print(f"mixed storage vs FP64: stations {e:.2e}")
    assert e <= 1e-3
    assert pu.rel_l2(m16["stations"][:, :, :3], r32["stations"][:, :, :3]) > 0.0
