"""The autotuner of the CGFDM stage launch (cgfdm_autotune,
cgfdm_batch_autotune): tuning times candidate work decompositions on trial
steps from a copy of the state and puts the state back, so a run tuned in
the middle gives exactly the traces, wavefield and PGV of an untuned run,
and the chosen tiling is one of the candidates."""

import numpy as np
import pytest

import parity_util as pu
from cgfdm import Batch, Session, cases, configs


@pytest.mark.gpu
def test_session_autotune_keeps_results(tmp_path):
    d = cases.write_case(pu.multi_fault(steps=30), str(tmp_path / "run"))
    with Session(d) as s:
        s.run(s.info.NT)
        ref = (s.stations(), s.wavefield(), s.pgv())
    with Session(d) as s:
        s.run(7)
        kc, ctas, ms = s.autotune(3)
        assert s.info.steps_done == 7
        assert s.tiling() == (kc, ctas) and 1 <= kc <= s.info.nz and ctas >= 1 and ms > 0
        s.run(s.info.NT)
        for a, r in zip((s.stations(), s.wavefield(), s.pgv()), ref):
            np.testing.assert_array_equal(a, r)
        # any tiling, same numbers
        s2 = Session(d)
        s2.set_tiling(5, 37)
        assert s2.tiling() == (5, 37)
        s2.run(s2.info.NT)
        np.testing.assert_array_equal(s2.stations(), ref[0])
        s2.close()


@pytest.mark.gpu
def test_batch_autotune_keeps_results(tmp_path):
    dirs = configs.batch_shots(str(tmp_path), n=3, steps=21, sizes=((40, 72), (36, 64), (28, 44)), nPML=6,
                               n_stations=6)
    alone = []
    for d in dirs:
        with Session(d) as s:
            s.run(s.info.NT)
            alone.append((s.stations(), s.wavefield(), s.pgv()))
    sessions = [Session(d) for d in dirs]
    try:
        with Batch(sessions) as b:
            b.run(3)
            kc, ctas, ms = b.autotune(2)
            assert kc >= 0 and ctas >= 1 and ms > 0
            b.run(100)
        for s, ref in zip(sessions, alone):
            for a, r in zip((s.stations(), s.wavefield(), s.pgv()), ref):
                np.testing.assert_array_equal(a, r)
    finally:
        for s in sessions:
            s.close()
