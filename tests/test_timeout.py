"""The stage kernel's bounded waits, made to run out on purpose.

Every wait of the CGFDM stage kernel for a plane copy is bounded; a wait
that gives up sets a device error word, the CTA waits (bounded) for the
copies it did issue and returns, and the next cgfdm_run reports
CGFDM_E_TIMEOUT.  The reference has no such path: its CHECK macro prints a
CUDA error and carries on (src/macro.h:94-103).

The test hook cgfdm_test_stall makes one work item leave one plane copy
unissued: nothing is in flight for that slot and its barrier phase never
completes, so the wait runs out after a short limit (about 2 ms here).  The
drain then waits for the copies that were issued, including the one for the
same slot's missing plane, which also runs out.  No copy is left landing in
shared memory, and the device stays usable: a fresh session on it then
matches the golden fixture of the reference's CPU build.
"""

import os
import tempfile

import numpy as np
import pytest

import golden_cases
from cgfdm import CgfdmError, Session, cases

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
E_TIMEOUT = 20002
WAIT_CYCLES = 1 << 22


def _fresh_session_matches_golden():
    mk, scheme = golden_cases.CASES["cg_halfspace"]
    gold = np.load(os.path.join(ROOT, "tests", "golden", "cg_halfspace.npz"))
    with tempfile.TemporaryDirectory() as d:
        cases.write_case(mk(), d, scheme=scheme)
        with Session(d, device=0, flavor="exact") as s:
            s.run(s.info.NT)
            st = s.stations()
    assert np.array_equal(st, gold["stations"])


@pytest.mark.gpu
@pytest.mark.parametrize("fill", [2, 7], ids=["first_window", "in_loop"])
def test_stage_wait_gives_up_and_device_recovers(tmp_path, fill):
    # fill 2: a plane of the item's first window (issued before the loop);
    # fill 7: a plane the loop issues, with later copies already in flight
    c = cases.halfspace_case(NX=64, NY=60, NZ=40, nPML=6, steps=16, n_stations=2)
    cases.write_case(c, str(tmp_path))
    with Session(str(tmp_path), device=0) as s:
        s.run(1)
        s.test_stall(item=0, fill=fill, wait_cycles=WAIT_CYCLES)
        with pytest.raises(CgfdmError) as e:
            s.run(9)
        assert e.value.code == E_TIMEOUT
        assert "gave up" in str(e.value)
    _fresh_session_matches_golden()
