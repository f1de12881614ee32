"""The oracles against the committed golden fixtures (tests/golden/, made
by tests/golden/make_golden.py from the reference's own CPU build), on the
CPU: the reference build must reproduce them exactly (the fixtures pin the
build across machines), and the C restatement in FP32 must reproduce the
CGFDM ones bit for bit and the ME-AWENO one to 1e-6 (its free surface is
restated, see stepper.c)."""

import os

import numpy as np
import pytest

import golden_cases
import parity_util as pu
import refrun
import restated
from cgfdm import cases

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("name", list(golden_cases.CASES))
def test_oracles_reproduce_golden(tmp_path, name):
    mk, scheme = golden_cases.CASES[name]
    if not (refrun.available(scheme) and restated.available()):
        pytest.skip("oracle builds not present")
    gold = np.load(os.path.join(HERE, "golden", f"{name}.npz"))
    d = str(tmp_path / name)
    cases.write_case(mk(), d, scheme=scheme)
    refrun.run(d, scheme)
    ref = refrun.read_outputs(d, scheme)
    np.testing.assert_array_equal(ref["stations"], gold["stations"])
    np.testing.assert_array_equal(ref["PGV"], gold["PGV"])
    np.testing.assert_array_equal(ref["W"][ref["W"].shape[0] - 4], gold["W_plane_z"])
    r = restated.run(restated.make_bundle(d, os.path.join(d, "bundle"), scheme), "f32")
    if scheme == "CGFDM":
        np.testing.assert_array_equal(r["stations"], gold["stations"])
        np.testing.assert_array_equal(r["PGV"], gold["PGV"])
    else:
        assert pu.rel_l2(r["stations"][:, :, :3], gold["stations"][:, :, :3]) <= 1e-6
        assert pu.rel_l2(r["PGV"], gold["PGV"]) <= 1e-6
