"""Mixed-precision storage of the CGFDM path ("storage": "fp16").

The step-start state stays FP32; each RK stage's delta from it and the RK
accumulator's delta are stored in FP16 with per-field power-of-two scales,
and every stage reads the delta back into its FP32 stencil input.  The
oracle is the C restatement built with the same storage (oracle/build/
stepper_m16, run on the model the reference's own CPU build set up): the
"exact" library build must reproduce it bit for bit.  The fast build is held
to the north-star bound, 1e-3 relative L2 on the station seismograms against
the FP64 run, on a case long enough for the direct waves to reach the
stations.
"""

import json
import os

import numpy as np
import pytest

import parity_util as pu
import refrun
import restated
from cgfdm import CgfdmError, Session, cases

FP16 = json.dumps({"storage": "fp16"})
E_OPTIONS = 180


def _terrain_fault(d):
    from cgfdm import configs

    configs.terrain_fault(d, steps=60, NX=64, NY=60, NZ=40, nPML=6)


CASES = {
    "halfspace": lambda d: cases.write_case(pu.small_halfspace(steps=48), d),
    "hill_200": lambda d: cases.write_case(pu.small_hill(steps=200), d),
    "multi_fault": lambda d: cases.write_case(pu.multi_fault(steps=48), d),
    "ricker_point": lambda d: cases.write_case(pu.ricker_point(steps=48), d),
    "double_couple": lambda d: cases.write_case(pu.double_couple(steps=48), d),
    "terrain_fault": _terrain_fault,
}


@pytest.fixture(scope="module")
def oracle_runs(tmp_path_factory):
    if not (refrun.available("CGFDM") and os.access(restated.binary("m16"), os.X_OK)):
        pytest.skip("oracle builds (oracle/build/stepper_m16, oracle/_ref) not present")
    root = tmp_path_factory.mktemp("mix")
    dirs = {}
    for name, write in CASES.items():
        dirs[name] = str(root / name)
        write(dirs[name])
    refrun.run_many(list(dirs.values()), "CGFDM")
    out = {}
    for name, d in dirs.items():
        b = restated.make_bundle(d, os.path.join(d, "bundle"), "CGFDM")
        out[name] = (d, restated.run(b, "m16"))
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_exact_build_matches_mixed_oracle(oracle_runs, name):
    d, ref = oracle_runs[name]
    with Session(d, options=FP16, flavor="exact") as s:
        s.run(s.info.NT)
        st, W, pgv = s.stations(), s.wavefield(), s.pgv()
    diff_st = np.abs(st - ref["stations"]).max()
    diff_w = np.abs(W - ref["W"]).max()
    assert diff_st == 0.0 and diff_w == 0.0, (
        f"{name}: max |stations diff| {diff_st}, max |W diff| {diff_w}, rel L2 stations "
        f"{pu.rel_l2(st, ref['stations']):.3e}, W {pu.rel_l2(W, ref['W']):.3e}")
    np.testing.assert_array_equal(pgv, ref["PGV"])


@pytest.mark.gpu
def test_fast_build_error_against_fp64(tmp_path):
    d = str(tmp_path / "hill")
    cases.write_case(pu.small_hill(steps=300), d)
    with Session(d, options=FP16) as s:
        NT = s.info.NT
        s.run(NT)
        st = s.stations()
        st64, _, _ = s.run_precise(NT, bits=64)
    with Session(d) as s:
        s.run(NT)
        st32 = s.stations()
    e16 = pu.rel_l2(st[:, :, :3], st64[:, :, :3])
    e32 = pu.rel_l2(st32[:, :, :3], st64[:, :, :3])
    print(f"stations vs FP64: fp16 storage {e16:.2e}, fp32 {e32:.2e}")
    assert e16 <= 1e-3
    assert e32 < e16


@pytest.mark.gpu
def test_fp16_storage_limits(tmp_path):
    d = str(tmp_path / "sc")
    cases.write_case(pu.small_hill(steps=8), d, scheme="SCFDM")
    with pytest.raises(CgfdmError) as e:
        Session(d, options=FP16)
    assert e.value.code == E_OPTIONS
    d2 = str(tmp_path / "cg")
    cases.write_case(pu.small_halfspace(steps=8), d2)
    with Session(d2, options=FP16) as s:
        s.run(3)
        with pytest.raises(CgfdmError) as e:
            s.checkpoint()
        assert e.value.code == E_OPTIONS
