"""Sessions created and run from several host threads at once.

Uploads of large model volumes go through a process-wide set of pinned
staging slots (one pipelined upload at a time, the others wait), and every
session holds its arrays in its own device block; two sessions made
concurrently in two threads must give the same traces and wavefield as the
same sessions made one after the other.  The grid is large enough
(256 x 256 x 128: a 110 MB medium volume) for the pipelined upload."""

import threading

import numpy as np
import pytest

from cgfdm import Session, configs

STEPS = 10


@pytest.fixture(scope="module")
def run_dirs(tmp_path_factory):
    root = tmp_path_factory.mktemp("thr")
    dirs = []
    for n, seed in enumerate((2, 5)):
        d = str(root / f"tf{n}")
        configs.terrain_fault(d, steps=STEPS, NX=256, NY=256, NZ=128, seed=seed, source="double_couple")
        dirs.append(d)
    return dirs


def _run(d):
    with Session(d) as s:
        s.run(s.info.NT)
        return s.stations(), s.wavefield()


@pytest.mark.gpu
def test_concurrent_sessions_match_sequential(run_dirs):
    seq = [_run(d) for d in run_dirs]
    out = [None] * len(run_dirs)
    errors = []

    def work(n):
        try:
            out[n] = _run(run_dirs[n])
        except Exception as e:  # reported below, in the main thread
            errors.append(e)

    th = [threading.Thread(target=work, args=(n,)) for n in range(len(run_dirs))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errors, errors
    for got, want in zip(out, seq):
        for a, b in zip(got, want):
            np.testing.assert_array_equal(a, b)
    # the two models differ, so the check would see a swapped upload
    assert not np.array_equal(seq[0][1], seq[1][1])
