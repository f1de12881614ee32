"""Peak ground acceleration (SOLVE_PGA) against the reference's CPU build
compiled with that flag: the PGV file then holds four fields per surface
point, PGVh, PGV, PGAh, PGA (src/PGV.cpp:61-175).  The reference's PGA is
|V| / (10 DT) at every tenth step (its previous-velocity copy never reaches
the surface, src/propagate.cpp:26-58); the library reproduces it.  The exact
build matches the CGFDM reference bit for bit; SCFDM is held to the
scheme's parity tolerance."""

import os
import shutil

import numpy as np
import pytest

import parity_util as pu
import refrun
from cgfdm import Session, cases


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", ["CGFDM", "SCFDM"])
def test_pga_file(tmp_path, scheme):
    if not refrun.available(scheme, pga=True):
        pytest.skip("reference CPU build with SOLVE_PGA not present")
    c = pu.multi_fault(steps=41, **({} if scheme == "CGFDM" else {"courant": 0.5}))
    c.extra = dict(c.extra, SOLVE_PGA=1)
    ref_dir, lib_dir = str(tmp_path / "ref"), str(tmp_path / "lib")
    cases.write_case(c, ref_dir, scheme=scheme)
    shutil.copytree(ref_dir, lib_dir)
    refrun.run(ref_dir, scheme, pga=True)
    with Session(lib_dir, flavor="exact") as s:
        assert s.info.pgv_fields == 4
        s.run(s.info.NT)
        s.write_outputs()
        mine = s.pgv()
    ref = refrun.read_outputs(ref_dir, scheme)["PGV"]
    assert ref.shape == mine.shape and ref.shape[2] == 4
    assert np.abs(ref[..., 2:]).max() > 0, "the case must accelerate the surface"
    f = np.fromfile(os.path.join(lib_dir, "output", "PGV_Z_mpi_0_0_0.bin"), np.float32)
    np.testing.assert_array_equal(f.reshape(mine.shape), mine)
    if scheme == "CGFDM":
        np.testing.assert_array_equal(mine, ref)
    else:
        for c in range(4):
            assert pu.rel_l2(mine[..., c], ref[..., c]) <= 1e-5, (c, pu.rel_l2(mine[..., c], ref[..., c]))
