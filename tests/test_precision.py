"""FP32 results of the library against the FP64 oracle.

The FP64 oracle is the C restatement of the time-stepping path
(oracle/restated/stepper.c) built with REAL = double, run on the model the
reference's CPU build set up (metric, medium, sources).  Every FP32 result
of this library is reported with its error against it; the bound here is
the FP32 rounding level over these short runs (1e-5 relative L2 on the
velocity seismograms and on the final wavefield), and the test also checks
that the library is no further from FP64 than the reference's own FP32
build is, within a factor of 4.
"""

import os

import numpy as np
import pytest

import parity_util as pu
import refrun
import restated
from cgfdm import Session, cases

CASES = {
    "cg_multi_fault": (lambda: pu.multi_fault(steps=40), "CGFDM"),
    "cg_hill": (lambda: pu.small_hill(steps=40), "CGFDM"),
    "sc_hill": (lambda: pu.small_hill(steps=24), "SCFDM"),
    "sc_double_couple": (lambda: pu.double_couple(steps=24, courant=0.5), "SCFDM"),
}


@pytest.fixture(scope="module")
def runs(tmp_path_factory):
    if not (restated.available() and refrun.available("CGFDM") and refrun.available("SCFDM")):
        pytest.skip("oracle builds (oracle/build, oracle/_ref) not present")
    root = tmp_path_factory.mktemp("prec")
    dirs = {}
    for name, (mk, scheme) in CASES.items():
        dirs[name] = str(root / name)
        cases.write_case(mk(), dirs[name], scheme=scheme)
    for scheme in ("CGFDM", "SCFDM"):
        refrun.run_many([d for n, d in dirs.items() if CASES[n][1] == scheme], scheme)
    out = {}
    for name, d in dirs.items():
        scheme = CASES[name][1]
        b = restated.make_bundle(d, os.path.join(d, "bundle"), scheme)
        out[name] = (d, refrun.read_outputs(d, scheme), restated.run(b, "f64"))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("flavor", ["fast", "exact"])
@pytest.mark.parametrize("name", list(CASES))
def test_fp32_error_against_fp64(runs, name, flavor):
    d, ref32, ref64 = runs[name]
    with Session(d, flavor=flavor) as s:
        s.run(s.info.NT)
        st, W = s.stations(), s.wavefield()
    e_st = pu.rel_l2(st[:, :, :3], ref64["stations"][:, :, :3])
    e_w = pu.rel_l2(W, ref64["W"])
    r_st = pu.rel_l2(ref32["stations"][:, :, :3], ref64["stations"][:, :, :3])
    r_w = pu.rel_l2(ref32["W"], ref64["W"])
    print(f"{name} {flavor}: vs FP64 stations {e_st:.2e} W {e_w:.2e} | reference FP32 vs FP64 {r_st:.2e} {r_w:.2e}")
    assert e_st <= 1e-5 and e_w <= 1e-5
    assert e_st <= 4 * r_st + 1e-7 and e_w <= 4 * r_w + 1e-7
