"""Checkpoint and restore through the C ABI (cgfdm_checkpoint / cgfdm_restore).

A run interrupted at a step boundary, checkpointed, and continued in a new
session from that checkpoint must give exactly the traces, wavefield and PGV
of an uninterrupted run, for both schemes (the CGFDM case includes PML
auxiliaries and the finite-fault source, the SCFDM case the sponge).
A checkpoint of a different grid is refused with CGFDM_E_ARG.
"""

import numpy as np
import pytest

import parity_util as pu
from cgfdm import CgfdmError, Session, cases


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", ["CGFDM", "SCFDM"])
def test_restart_is_bit_identical(tmp_path, scheme):
    d = str(tmp_path / "run")
    c = pu.multi_fault(steps=37, **({} if scheme == "CGFDM" else {"courant": 0.5}))
    cases.write_case(c, d, scheme=scheme)
    with Session(d) as s:
        s.run(s.info.NT)
        full = (s.stations(), s.wavefield(), s.pgv())
    with Session(d) as s:
        s.run(13)                      # not a multiple of the 8-step graph
        ck = s.checkpoint()
    with Session(d) as s:
        s.restore(ck)
        assert s.info.steps_done == 13
        s.run(s.info.NT)
        part = (s.stations(), s.wavefield(), s.pgv())
    for a, b in zip(full, part):
        np.testing.assert_array_equal(a, b)


@pytest.mark.gpu
def test_restore_rejects_other_grid(tmp_path):
    d1, d2 = str(tmp_path / "a"), str(tmp_path / "b")
    cases.write_case(pu.small_halfspace(steps=8), d1)
    cases.write_case(pu.small_halfspace(steps=8, NX=36), d2)
    with Session(d1) as s:
        ck = s.checkpoint()
    with Session(d2) as s:
        with pytest.raises(CgfdmError) as e:
            s.restore(ck)
        assert e.value.code == 20003
