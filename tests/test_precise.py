"""The reference-form run in a chosen precision (cgfdm_run_precise).

bits = 32, exact build: the same time loop, written one thread per point on
the session's model, must reproduce the fused session bit for bit (CGFDM;
ME-AWENO within 1e-6, the fused passes share smoothness indicators in the
fast build and differ in the last bits of the characteristic surface).
That pins the restatement to the session's algorithm.

bits = 64: the FP64 run on the GPU must agree with the CPU FP64 oracle
(oracle/restated/stepper.c built with REAL = double, run on the model the
reference's own CPU build set up) to 1e-10 relative L2 on the station
traces: both are the same FP64 algorithm, differing only in where FMA
contraction rounds.
"""

import os

import numpy as np
import pytest

import parity_util as pu
import refrun
import restated
from cgfdm import Session, cases

CG = {
    "halfspace": lambda: pu.small_halfspace(steps=40),
    "gauss_hill": lambda: pu.small_hill(steps=40),
    "multi_fault": lambda: pu.multi_fault(steps=40),
    "ricker_point": lambda: pu.ricker_point(steps=40),
    "double_couple": lambda: pu.double_couple(steps=40),
}
SC = {
    "sc_hill": lambda: pu.small_hill(steps=24),
    "sc_double_couple": lambda: pu.double_couple(steps=24, courant=0.5),
    "sc_multi_fault": lambda: pu.multi_fault(steps=24, courant=0.5),
}


def _write(tmp, name, mk, scheme):
    d = str(tmp / name)
    cases.write_case(mk(), d, scheme=scheme)
    return d


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CG) + list(SC))
def test_fp32_form_matches_session(tmp_path, name):
    scheme = "CGFDM" if name in CG else "SCFDM"
    d = _write(tmp_path, name, (CG if name in CG else SC)[name], scheme)
    with Session(d, flavor="exact") as s:
        NT = s.info.NT
        st_p, pgv_p, W_p = s.run_precise(NT, bits=32, wavefield=True)
        s.run(NT)
        st, W, pgv = s.stations(), s.wavefield(), s.pgv()
    if scheme == "CGFDM":
        np.testing.assert_array_equal(st_p.astype(np.float32), st)
        np.testing.assert_array_equal(W_p.astype(np.float32), W)
        np.testing.assert_array_equal(pgv_p.astype(np.float32), pgv[:, :, :2])
    else:
        assert pu.rel_l2(st_p[:, :, :3], st[:, :, :3]) <= 1e-6
        assert pu.rel_l2(W_p, W) <= 1e-6


@pytest.fixture(scope="module")
def fp64_runs(tmp_path_factory):
    if not (restated.available() and refrun.available("CGFDM") and refrun.available("SCFDM")):
        pytest.skip("oracle builds (oracle/build, oracle/_ref) not present")
    root = tmp_path_factory.mktemp("fp64")
    dirs = {}
    for name, mk in list(CG.items()) + list(SC.items()):
        dirs[name] = _write(root, name, mk, "CGFDM" if name in CG else "SCFDM")
    for scheme, names in (("CGFDM", CG), ("SCFDM", SC)):
        refrun.run_many([dirs[n] for n in names], scheme)
    out = {}
    for name, d in dirs.items():
        scheme = "CGFDM" if name in CG else "SCFDM"
        b = restated.make_bundle(d, os.path.join(d, "bundle"), scheme)
        r = restated.run(b, "f64")
        nst, NT = r["stations"].shape[:2]
        st64 = np.fromfile(os.path.join(b, "out_stations64.bin"), np.float64).reshape(nst, NT, 9)
        out[name] = (d, st64, r["W"])
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("flavor", ["fast", "exact"])
@pytest.mark.parametrize("name", list(CG) + list(SC))
def test_fp64_run_matches_cpu_fp64_oracle(fp64_runs, name, flavor):
    d, st64, W64 = fp64_runs[name]
    with Session(d, flavor=flavor) as s:
        st, _, W = s.run_precise(s.info.NT, bits=64, wavefield=True)
    e_st = pu.rel_l2(st[:, :, :3], st64[:, :, :3])
    e_w = pu.rel_l2(W.astype(np.float32), W64)   # the oracle's wavefield file is float32
    print(f"{name} {flavor}: GPU FP64 vs CPU FP64 stations {e_st:.2e}, W {e_w:.2e}")
    assert e_st <= 1e-10
    assert e_w <= 1e-6
