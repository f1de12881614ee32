"""Snapshot and model-slice files against the reference's CPU build.

With IT_SKIP, sliceX/Y/Z and sliceFreeSurf set, the reference writes
velocity slices after every step s with s % IT_SKIP == 0 and the model
slices (coordinates, Vs, Vp, rho) before the loop (src/propagate.cpp:289-309,
src/run.cpp:70, src/data_io.cpp:332-626).  The library writes the same files
during cgfdm_run and in cgfdm_write_outputs.  The exact build must match the
CGFDM reference bit for bit; SCFDM slices hold velocity converted from
momentum and are held to the scheme's parity tolerance.
"""

import glob
import os
import shutil

import numpy as np
import pytest

import parity_util as pu
import refrun
from cgfdm import Session, cases


def _case(scheme):
    c = pu.multi_fault(steps=24, **({} if scheme == "CGFDM" else {"courant": 0.5}))
    c.it_skip = 10
    c.slice_xyz = (16, 12, c.NZ - 5)
    c.slice_free_surface = 1
    return c


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", ["CGFDM", "SCFDM"])
def test_snapshot_files(tmp_path, scheme):
    if not refrun.available(scheme):
        pytest.skip("reference CPU build not present")
    ref_dir, lib_dir = str(tmp_path / "ref"), str(tmp_path / "lib")
    cases.write_case(_case(scheme), ref_dir, scheme=scheme)
    shutil.copytree(ref_dir, lib_dir)
    refrun.run(ref_dir, scheme)
    with Session(lib_dir, flavor="exact") as s:
        s.run(s.info.NT)
        s.write_outputs()
    names = sorted(os.path.basename(p) for p in glob.glob(os.path.join(ref_dir, "output", "*_mpi_0_0_0.bin")))
    snaps = [n for n in names if n.startswith(("Vx_", "Vy_", "Vz_", "FreeSurfV"))]
    model = [n for n in names if n.startswith(("coord", "Vs_", "Vp_", "rho_"))]
    assert len(snaps) == 3 * 3 * 3 + 3 * 3   # 3 snapshot steps x (3 components x 3 planes + 3 surface)
    assert len(model) == 6 * 3
    for n in snaps + model:
        a = np.fromfile(os.path.join(lib_dir, "output", n), np.float32)
        b = np.fromfile(os.path.join(ref_dir, "output", n), np.float32)
        assert a.shape == b.shape, n
        if scheme == "CGFDM" or n in model:
            np.testing.assert_array_equal(a, b, err_msg=n)
        else:
            assert pu.rel_l2(a, b) <= 1e-5, (n, pu.rel_l2(a, b))
