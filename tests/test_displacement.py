"""Surface displacement (SOLVE_DISPLACEMENT) against the reference's CPU build
compiled with that flag.

The reference integrates Dis += v * DT after every step, v the velocity
(CGFDM) or momentum times buoyancy (SCFDM), after the free surface and the
sponge (src/solve_displacement.cpp:27-63, src/propagate.cpp:264-266), and
writes its surface layer as FreeSurfUx/Uy/Uz with the free-surface
velocity snapshots (src/data_io.cpp:619-633, src/propagate.cpp:305-307).
The library takes the flag as the params.json switch SOLVE_DISPLACEMENT.
The exact build must match the CGFDM reference bit for bit; SCFDM is held
to the scheme's parity tolerance.
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
    c.slice_free_surface = 1
    c.extra = dict(c.extra, SOLVE_DISPLACEMENT=1)
    return c


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", ["CGFDM", "SCFDM"])
def test_free_surface_displacement(tmp_path, scheme):
    if not refrun.available(scheme, displacement=True):
        pytest.skip("reference CPU build with SOLVE_DISPLACEMENT not present")
    ref_dir, lib_dir = str(tmp_path / "ref"), str(tmp_path / "lib")
    cases.write_case(_case(scheme), ref_dir, scheme=scheme)
    shutil.copytree(ref_dir, lib_dir)
    refrun.run(ref_dir, scheme, displacement=True)
    with Session(lib_dir, flavor="exact") as s:
        s.run(s.info.NT)
        s.write_outputs()
    names = sorted(os.path.basename(p) for p in glob.glob(os.path.join(ref_dir, "output", "FreeSurf*_mpi_0_0_0.bin")))
    disp = [n for n in names if n.startswith("FreeSurfU")]
    assert len(disp) == 3 * 3        # 3 snapshot steps x 3 components
    assert len(names) == 2 * 3 * 3   # and the velocity snapshots beside them
    for n in names:
        a = np.fromfile(os.path.join(lib_dir, "output", n), np.float32)
        b = np.fromfile(os.path.join(ref_dir, "output", n), np.float32)
        assert a.shape == b.shape, n
        if scheme == "CGFDM":
            np.testing.assert_array_equal(a, b, err_msg=n)
        elif np.abs(b).max() > 0:
            assert pu.rel_l2(a, b) <= 1e-5, (n, pu.rel_l2(a, b))
        else:
            assert np.abs(a).max() == 0, n
    last = np.fromfile(os.path.join(ref_dir, "output", disp[-1]), np.float32)
    assert np.abs(last).max() > 0, "the case must move the surface"
