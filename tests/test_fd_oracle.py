"""CPU checks of the finite-difference oracle the adjoint tests use
(oracle/fd_gradient.py over the FP64 restatement, oracle/restated).

* a zero perturbation changes nothing;
* a zero perturbation at a surface point, which recomputes that point's
  free-surface matrices in FP64 from the restated formula, agrees with the
  reference's own FP32 matrices to FP32 rounding;
* central differences with steps 1e-3 and 1e-4 of the parameter agree (the
  misfit is smooth and the differences are not noise).
"""

import os
import shutil

import numpy as np
import pytest

import fd_gradient
import refrun
import restated
import test_adjoint as ta
from cgfdm import cases


@pytest.fixture(scope="module")
def bundle(tmp_path_factory):
    if not (refrun.available("CGFDM") and restated.available()):
        pytest.skip("reference CPU build or restatement not built")
    root = tmp_path_factory.mktemp("fdo")
    c = ta._grad_case(steps=40)
    d = cases.write_case(c, str(root / "run"))
    med = ta._medium(c, 11, False)
    med.tofile(os.path.join(d, "medium.bin"))
    refrun.run(d, "CGFDM")
    b = restated.make_bundle(d, str(root / "bundle"))
    return c, med, b, root


def _stations(b, work, lines):
    return fd_gradient._run_one(b, work, lines)


def test_zero_perturbations(bundle):
    c, med, b, root = bundle
    base = _stations(b, str(root / "z0"), [])
    same = _stations(b, str(root / "z1"), ["20 18 25 0.0 0.0 0.0"])
    np.testing.assert_array_equal(base, same)
    top = c.NZ + 2
    surf = _stations(b, str(root / "z2"), [f"20 18 {top} 0.0 0.0 0.0", f"14 22 {top} 0.0 0.0 0.0"])
    scale = np.abs(base).max()
    assert np.abs(surf - base).max() <= 1e-5 * scale


def test_central_differences_converge(bundle):
    c, med, b, root = bundle
    rng = np.random.default_rng(1)
    obs = (rng.standard_normal(_stations(b, str(root / "o"), [])[:, :, :3].shape) * 1e-9).astype(np.float32)
    cells = [(20, 18, 25), (17, 15, c.NZ + 2)]
    g3 = fd_gradient.fd_gradient(b, str(root / "fd3"), med, cells, obs, rel_step=1e-3)
    g4 = fd_gradient.fd_gradient(b, str(root / "fd4"), med, cells, obs, rel_step=1e-4)
    for p in fd_gradient.PARAMS:
        assert np.all(np.abs(g3[p] - g4[p]) <= 1e-4 * np.abs(g4[p]) + 1e-30), (p, g3[p], g4[p])
    shutil.rmtree(str(root), ignore_errors=True)
