"""Batched CGFDM sessions (cgfdm_batch_*): three shots of different grid
sizes, media and sources advanced together by one persistent stage launch
per RK stage must give each shot exactly the traces, wavefield and PGV of
running it alone; a batched session stepped on its own is detected."""

import numpy as np
import pytest

from cgfdm import Batch, CgfdmError, Session, configs


def _shots(root):
    return configs.batch_shots(str(root), n=3, steps=21, sizes=((40, 72), (36, 64), (28, 44)), nPML=6,
                               n_stations=6)


@pytest.mark.gpu
def test_batch_matches_single_runs(tmp_path):
    dirs = _shots(tmp_path)
    alone = []
    for d in dirs:
        with Session(d) as s:
            s.run(s.info.NT)
            alone.append((s.stations(), s.wavefield(), s.pgv()))
    sessions = [Session(d) for d in dirs]
    try:
        with Batch(sessions) as b:
            b.run(5)          # off the 8-step graph phase
            b.run(100)        # the rest, clipped to NT
        for s, ref in zip(sessions, alone):
            assert s.info.steps_done == s.info.NT
            for a, r in zip((s.stations(), s.wavefield(), s.pgv()), ref):
                np.testing.assert_array_equal(a, r)
    finally:
        for s in sessions:
            s.close()


@pytest.mark.gpu
def test_batch_detects_solo_step(tmp_path):
    dirs = _shots(tmp_path)
    sessions = [Session(d) for d in dirs]
    try:
        with Batch(sessions) as b:
            sessions[1].run(1)
            with pytest.raises(CgfdmError) as e:
                b.run(1)
            assert e.value.code == 20004
    finally:
        for s in sessions:
            s.close()


@pytest.mark.gpu
def test_fp16_storage_batch_matches_single_runs(tmp_path):
    """Sessions with FP16 storage (FP32 step state, per-field-scaled FP16
    stage and accumulator deltas) batched together: each shot's traces,
    wavefield and PGV are bit-identical to its own run with the same
    storage; the per-field scales and the bounds they come from stay per
    session inside the shared launch.  A batch mixing both storages is
    refused."""
    fp16 = '{"storage": "fp16"}'
    dirs = _shots(tmp_path)
    alone = []
    for d in dirs:
        with Session(d, options=fp16) as s:
            s.run(s.info.NT)
            alone.append((s.stations(), s.wavefield(), s.pgv()))
    sessions = [Session(d, options=fp16) for d in dirs]
    try:
        with Batch(sessions) as b:
            b.run(5)
            b.run(100)
        for s, ref in zip(sessions, alone):
            assert s.info.steps_done == s.info.NT
            for a, r in zip((s.stations(), s.wavefield(), s.pgv()), ref):
                np.testing.assert_array_equal(a, r)
    finally:
        for s in sessions:
            s.close()
    both = [Session(dirs[0], options=fp16), Session(dirs[1])]
    try:
        with pytest.raises(CgfdmError) as e:
            Batch(both)
        assert e.value.code == 180
    finally:
        for s in both:
            s.close()
