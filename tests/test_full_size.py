"""Properties of the full-size benchmark workload (terrain_fault, 400 x 400 x
200, 12-layer PML, 40 x 20 finite fault, 400 stations), which is too large
for the CPU oracles: checks that do not depend on a reference result.

* a run interrupted, checkpointed and restored in a new session ends
  bit-identical to the uninterrupted run;
* the same grid decomposed into two parts on the GPU, with the halo stores
  fused into the stage kernels, ends bit-identical too;
* the state is finite and the source has put energy into it;
* the device medium (mu, lambda, buoyancy), made from the medium volume the
  session uploads through its pinned staging slots (the path only arrays of
  more than 64 MB take), agrees with the host model of the same run
  directory point for point."""

import os

import numpy as np
import pytest

from cgfdm import Session, configs, domain, model_medium

STEPS = 12


@pytest.fixture(scope="module")
def run_dir(tmp_path_factory):
    d = str(tmp_path_factory.mktemp("full") / "terrain_fault")
    configs.terrain_fault(d, steps=STEPS)
    return d


@pytest.fixture(scope="module")
def reference(run_dir):
    with Session(run_dir) as s:
        assert (s.info.nx, s.info.ny, s.info.nz) == (400, 400, 200)
        s.run(s.info.NT)
        assert s.check_finite() == (0, -1)
        return s.wavefield()[3:-3, 3:-3, 3:-3].copy(), s.stations(), s.pgv()[..., :2].copy()


@pytest.mark.gpu
def test_full_size_restart_is_bit_identical(run_dir, reference):
    with Session(run_dir) as s:
        s.run(5)
        ck = s.checkpoint()
    with Session(run_dir) as s:
        s.restore(ck)
        s.run(s.info.NT)
        got = (s.wavefield()[3:-3, 3:-3, 3:-3], s.stations(), s.pgv()[..., :2])
    for a, b in zip(got, reference):
        np.testing.assert_array_equal(a, b)
    assert np.abs(reference[0]).max() > 0


@pytest.mark.gpu
def test_full_size_two_parts_fused_match(run_dir, reference):
    got = domain.run_local(run_dir, (2, 1, 1), fused=True)
    for a, b in zip(got, reference):
        np.testing.assert_array_equal(a, b)


@pytest.mark.gpu
def test_full_size_medium_upload(run_dir):
    """The 408 MB medium volume crosses to the device in 8 MB slots filled by
    several host threads; a slot landing in the wrong place would move a
    whole block of the model.  Checked against the host model: mu = rho vs^2,
    lambda = rho (vp^2 - 2 vs^2), buoyancy = 1 / rho at every interior point,
    to FP32 rounding."""
    med = model_medium(run_dir).astype(np.float64)
    with Session(run_dir) as s:
        cjm = s.cjm()
    vs, vp, rho = med[..., 0], med[..., 1], med[..., 2]
    want = {10: rho * vs * vs, 11: rho * (vp * vp - 2.0 * vs * vs), 12: 1.0 / rho}
    inner = (slice(3, -3), slice(3, -3), slice(3, -3))
    for ch, w in want.items():
        got = cjm[inner + (ch,)].astype(np.float64)
        w = w[inner]
        rel = np.abs(got - w) / np.abs(w)
        assert rel.max() < 1e-5, (ch, float(rel.max()), np.unravel_index(np.argmax(rel), rel.shape))
