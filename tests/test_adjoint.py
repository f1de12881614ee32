"""The CGFDM adjoint: dot-product test of the transposed step and the misfit
gradient against FP64 central finite differences.

Dot-product test: for A the forward map of n steps without sources
(cgfdm_set_wavefield -> cgfdm_run -> cgfdm_get_wavefield) and A^T its
transpose from cgfdm_adjoint_apply, <A x, y> = <x, A^T y> for random
interior states x, y, over a flat and a curvilinear (Gauss hill) grid with
the PML on, so the stencil, the traction-image free surface and the PML
auxiliaries are all exercised.

Gradient: dJ/d(Vp, Vs, rho) of J = 1/2 sum (v - d)^2 from cgfdm_gradient at
20 seeded grid points (four of them in the surface layers) against central
differences of the FP64 restatement of the time loop (oracle/restated,
oracle/fd_gradient.py) on the reference's own model of the same run.
"""

import dataclasses
import json
import os
import shutil

import numpy as np
import pytest

import fd_gradient
import parity_util as pu
import refrun
import restated
from cgfdm import Session, cases

NPML = 6


def _scaled_state(rng, shape, v_scale, t_scale):
    x = rng.standard_normal(shape).astype(np.float32)
    x[..., :3] *= v_scale
    x[..., 3:] *= t_scale
    x[:3], x[-3:], x[:, :3], x[:, -3:], x[:, :, :3], x[:, :, -3:] = 0, 0, 0, 0, 0, 0
    return x


def _source_free(hill: bool, steps: int) -> cases.Case:
    """A run whose source adds nothing (a finite fault of zero rate; a run
    needs a source), so a step is a linear map of the state."""
    c = pu.small_hill(steps=steps) if hill else pu.small_halfspace(steps=steps)
    c.fault = [dataclasses.replace(p, rate=np.zeros_like(p.rate)) for p in c.fault]
    return c


@pytest.mark.gpu
@pytest.mark.parametrize("kernel", ["two-pass", "fused"])
@pytest.mark.parametrize("flavor", ["fast", "exact"])
@pytest.mark.parametrize("hill", [False, True], ids=["flat", "hill"])
def test_dot_product(tmp_path, hill, flavor, kernel):
    n = 12
    d = cases.write_case(_source_free(hill, n), str(tmp_path / "run"))
    rng = np.random.default_rng(3 + hill)
    with Session(d, options=json.dumps({"adjointKernel": kernel}), flavor=flavor) as s:
        i = s.info
        shape = (i.nzp, i.nyp, i.nxp, 9)
        zr = 2670.0 * 6000.0   # impedance: balances velocity and stress entries
        x = _scaled_state(rng, shape, 1.0, zr)
        y = _scaled_state(rng, shape, 1.0, 1.0 / zr)
        s.set_wavefield(x)
        s.run(n)
        ax = s.wavefield()
        aty = s.adjoint_apply(y, n)
    inner = (slice(3, -3),) * 3
    lhs = float(np.sum(ax[inner].astype(np.float64) * y[inner]))
    rhs = float(np.sum(x[inner].astype(np.float64) * aty[inner]))
    print(f"dot product: <Ax,y> = {lhs:.9e}, <x,A^T y> = {rhs:.9e}, rel diff {abs(lhs - rhs) / abs(lhs):.2e}")
    assert np.abs(aty[:3]).max() == 0 and np.abs(aty[:, :, -3:]).max() == 0
    assert abs(lhs - rhs) <= 2e-5 * abs(lhs), (lhs, rhs, abs(lhs - rhs) / abs(lhs))


def _medium(c: cases.Case, seed: int, anomaly: bool) -> np.ndarray:
    """Smooth +-5% heterogeneity over the half-space, optionally a +8% Vs
    ball of radius 600 m near the centre: [nzp][nyp][nxp][3] (Vs, Vp, rho)."""
    rng = np.random.default_rng(seed)
    nzp, nyp, nxp = c.NZ + 6, c.NY + 6, c.NX + 6
    noise = rng.standard_normal((3, nzp, nyp, nxp))
    k = np.exp(-0.5 * (np.arange(-6, 7) / 2.5) ** 2)
    k /= k.sum()
    for ax in (1, 2, 3):
        noise = np.apply_along_axis(lambda v: np.convolve(v, k, mode="same"), ax, noise)
    noise /= np.abs(noise).max()
    med = np.empty((nzp, nyp, nxp, 3), np.float64)
    med[..., 0] = 3464.0 * (1 + 0.05 * noise[0])
    med[..., 1] = 6000.0 * (1 + 0.05 * noise[1])
    med[..., 2] = 2670.0 * (1 + 0.05 * noise[2])
    if anomaly:
        kk, jj, ii = np.meshgrid(np.arange(nzp), np.arange(nyp), np.arange(nxp), indexing="ij")
        r = np.sqrt((ii - nxp / 2) ** 2 + (jj - nyp / 2) ** 2 + (kk - (nzp - 10)) ** 2) * c.DH
        med[..., 0] *= np.where(r < 600.0, 1.08, 1.0)
    return med.astype(np.float32)


def _grad_case(steps=90):
    c = pu.ricker_point(steps=steps, NX=36, NY=32, NZ=28, nPML=NPML, courant=0.45)
    c.gauss_hill = 1
    c.stations = [(x, y, c.NZ - 1) for x in (9, 15, 21, 27) for y in (9, 16, 23)]
    c.extra = dict(c.extra, mediumFile="medium.bin", useMedium=1)
    return c


def _cells(c, rng, n=16):
    _nx, _ny, _nz = c.NX + 3, c.NY + 3, c.NZ + 3
    lo = 3 + NPML
    cells = [(int(rng.integers(lo, _nx - NPML)), int(rng.integers(lo, _ny - NPML)), int(rng.integers(lo, _nz - 3)))
             for _ in range(n)]
    for kk in (_nz - 1, _nz - 1, _nz - 2, _nz - 3):
        cells.append((int(rng.integers(lo, _nx - NPML)), int(rng.integers(lo, _ny - NPML)), kk))
    return cells


@pytest.mark.gpu
def test_gradient_against_fp64_finite_differences(tmp_path):
    if not (refrun.available("CGFDM") and restated.available()):
        pytest.skip("reference CPU build or restatement not built")
    c = _grad_case()
    d = cases.write_case(c, str(tmp_path / "run"))
    true_med, start_med = _medium(c, 11, True), _medium(c, 11, False)
    start_med.tofile(os.path.join(d, "medium.bin"))
    # observed data: the true model's seismograms (FP32 forward)
    with Session(d) as s:
        s.set_medium(true_med)
        s.run(s.info.NT)
        observed = s.stations()[:, :, :3].copy()
        s.set_medium(start_med)
        J, grad = s.gradient(observed, checkpoint_every=25)
        # one segment instead of four: the same stored RHS, the same result
        s.set_medium(start_med)
        J1, grad1 = s.gradient(observed, checkpoint_every=s.info.NT)
    assert J1 == J and np.array_equal(grad1, grad)
    # the fused kernel (Phi in shared memory) agrees with the default two passes
    with Session(d, options=json.dumps({"adjointKernel": "fused"})) as s2:
        s2.set_medium(start_med)
        J2, grad2 = s2.gradient(observed, checkpoint_every=25)
    assert J2 == J
    print(f"fused vs two-pass gradient: rel L2 {pu.rel_l2(grad, grad2):.2e}")
    assert 0.0 < pu.rel_l2(grad, grad2) <= 1e-5   # another summation order, the same gradient
    assert np.abs(grad[:, :NPML]).max() == 0 and np.abs(grad[:, :, :, -NPML:]).max() == 0
    # the reference's model of the starting medium, and FP64 differences
    ref_dir = str(tmp_path / "ref")
    shutil.copytree(d, ref_dir)
    refrun.run(ref_dir, "CGFDM")
    bundle = restated.make_bundle(ref_dir, str(tmp_path / "bundle"))
    rng = np.random.default_rng(5)
    cells = _cells(c, rng)
    fd = fd_gradient.fd_gradient(bundle, str(tmp_path / "fd"), start_med, cells, observed)
    assert abs(J - fd["J"][0]) <= 1e-3 * fd["J"][0], (J, fd["J"][0])
    rows = []
    for p_i, p in enumerate(fd_gradient.PARAMS):
        g = np.array([grad[p_i, k - 3, j - 3, i - 3] for (i, j, k) in cells], np.float64)
        rows.append((p, pu.rel_l2(g, fd[p]), g, fd[p]))
    for p, e, g, f in rows:
        worst = np.max(np.abs(g - f)) / np.max(np.abs(f))
        print(f"d J / d {p}: rel L2 vs FP64 central differences {e:.2e} over {len(cells)} points "
              f"(max abs err / max abs {worst:.2e})")
    for p, e, g, f in rows:
        assert e <= 1e-3, (p, e, list(zip(cells, g, f)))


@pytest.mark.gpu
def test_autograd_function_matches_session_gradient(tmp_path):
    import torch

    from cgfdm.autograd import misfit

    c = _grad_case(steps=40)
    d = cases.write_case(c, str(tmp_path / "run"))
    med = _medium(c, 11, False)
    med.tofile(os.path.join(d, "medium.bin"))
    rng = np.random.default_rng(2)
    with Session(d) as s:
        obs = (rng.standard_normal((s.info.n_stations, s.info.NT, 3)) * 1e-9).astype(np.float32)
        inner = med[3:-3, 3:-3, 3:-3]
        vs, vp, rho = (torch.tensor(inner[..., c].copy(), requires_grad=True) for c in range(3))
        J = misfit(vp, vs, rho, s, torch.from_numpy(obs), 10)
        (2.0 * J).backward()
        J = J.item()
        s.set_medium(med)
        J0, g0 = s.gradient(obs, 10)
    assert J == J0
    for t, g in zip((vp, vs, rho), g0):
        np.testing.assert_array_equal(t.grad.numpy(), 2.0 * g)
