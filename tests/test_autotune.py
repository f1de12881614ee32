"""The autotuner of the CGFDM stage launch (cgfdm_autotune,
cgfdm_batch_autotune): tuning times candidate work decompositions on trial
steps from a copy of the state and puts the state back, so a run tuned in
the middle gives exactly the traces, wavefield and PGV of an untuned run,
and the chosen tiling is one of the candidates."""

import numpy as np
import pytest

import parity_util as pu
from cgfdm import Batch, CgfdmError, Session, cases, configs

E_ARG, E_OPTIONS = 20003, 180


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
def test_stage_tile_heights(tmp_path):
    """32 x 8 tiles by default on the FP32 split pipeline, 4 rows on the ring
    pipeline and with FP16 storage (8 refused there); switching the height
    in the middle of a run changes no number."""
    d = cases.write_case(pu.multi_fault(steps=30), str(tmp_path / "run"))
    with Session(d) as s:
        assert s.stage_tile() == 8
        s.run(s.info.NT)
        ref = (s.stations(), s.wavefield(), s.pgv())
    with Session(d) as s:
        s.run(11)
        s.set_stage_tile(4)
        assert s.stage_tile() == 4
        s.run(6)
        s.set_stage_tile(8)
        s.run(s.info.NT)
        for a, r in zip((s.stations(), s.wavefield(), s.pgv()), ref):
            np.testing.assert_array_equal(a, r)
        with pytest.raises(CgfdmError) as e:
            s.set_stage_tile(6)
        assert e.value.code == E_ARG
    with Session(d, options='{"stagePipeline": "ring"}') as s:
        # the ring pipeline runs 32 x 4 tiles unless asked for 8 rows
        assert s.stage_tile() == 4
        s.run(9)
        s.set_stage_tile(8)
        s.run(s.info.NT)
        for a, r in zip((s.stations(), s.wavefield(), s.pgv()), ref):
            np.testing.assert_array_equal(a, r)
    with Session(d, options='{"storage": "fp16"}') as s:
        assert s.stage_tile() == 4
        with pytest.raises(CgfdmError) as e:
            s.set_stage_tile(8)
        assert e.value.code == E_OPTIONS
    for opts in ('{"storage": "fp16", "stageTile": 8}', '{"stageTile": 6}'):
        with pytest.raises(CgfdmError) as e:
            Session(d, options=opts)
        assert e.value.code == E_OPTIONS


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
            assert kc >= 0 and ctas >= 1 and ms > 0 and b.stage_tile() in (4, 8)
            b.run(4)
            b.set_stage_tile(12 - b.stage_tile())   # the other height, mid-run
            b.run(100)
        for s, ref in zip(sessions, alone):
            for a, r in zip((s.stations(), s.wavefield(), s.pgv()), ref):
                np.testing.assert_array_equal(a, r)
    finally:
        for s in sessions:
            s.close()
