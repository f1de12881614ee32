"""The per-function entry points (include/cgfdm_shims.h, cgfdm.shims) driven
by a Python restatement of the reference's time loop, src/propagate.cpp:
186-309 -- source, then per RK stage waveDeriv, freeSurfaceDeriv, pmlDeriv,
pmlFreeSurfaceDeriv, waveRk, pmlRk, then displacement, stations and PGV --
on device arrays in the reference's layouts (torch CUDA tensors), as a
patched propagate.cpp would call them.  Against the session's fused path
(itself bit-exact against the reference's CPU build): the final wavefield,
the station traces and the PGV must agree bit for bit in the exact build,
on a curvilinear grid (Gaussian hill) with PML on five faces, the traction
free surface and each source kind (finite fault of several cells, Ricker
and double-couple point sources); for ME-AWENO the same with the
characteristic free surface and the sponge.

CPU-only checks: every entry point the header declares is exported, and
argument errors come back as CGFDM_E_ARG without touching a GPU."""

import ctypes
import os
import re

import numpy as np
import pytest

import parity_util as pu
from cgfdm import CgfdmError, Session, cases, lib_path

# the MacCormack sign table, src/propagate.cpp:158-168
FB_TABLE = [(-1, -1, -1), (1, 1, -1), (1, 1, 1), (-1, -1, 1), (-1, 1, -1), (1, -1, -1), (1, -1, 1), (-1, 1, 1)]
HEADER = os.path.join(os.path.dirname(__file__), "..", "include", "cgfdm_shims.h")


def _add_point(sh, g, c, W, CJM, it, DT, DH, scheme):
    """The single point source of case c at stage 0 of step it, as
    src/propagate.cpp:195-198 calls it."""
    f32 = lambda x: float(np.float32(x))
    if c.ricker_point is not None:
        X, Y, Z, fc = c.ricker_point
        sh.loadPointSource_ricker(g, (X + 3, Y + 3, Z + 3), W, CJM, it, 0, DT, DH, f32(fc), scheme)
    if c.double_couple is not None:
        d = c.double_couple
        sh.loadPointSource_double_couple(g, (d["X"] + 3, d["Y"] + 3, d["Z"] + 3), W, CJM, it, 0, DT, DH,
                                         f32(d["strike"]), f32(d["dip"]), f32(d["rake"]), f32(d["Mw"]),
                                         f32(d["duration"]), scheme)


def propagate(sh, s, torch, nsteps, nPML, fault_dt, c=None):
    """The reference's loop over the entry points, for a CGFDM session with
    PML, free surface, a finite fault or point source, and stations."""
    from cgfdm.shims import Grid

    info = s.info
    nx, ny, nz, NT = info.nx, info.ny, info.nz, info.NT
    DT, DH = info.DT, info.DH
    g = Grid(info.nxp, info.nyp, info.nzp, float(np.float32(1.0 / np.float64(np.float32(DH)))))
    dev = torch.device("cuda:0")
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    npad = info.nxp * info.nyp * info.nzp
    h_W, W, t_W, m_W = (torch.zeros(npad * 9, dtype=torch.float32, device=dev) for _ in range(4))
    CJM = T(s.cjm())
    DX, DY = T(s.array("rDZ_DX")), T(s.array("rDZ_DY"))
    pml = [T(s.array(f"pml_{q}_{ax}")) for ax in "xyz" for q in ("alpha", "beta", "d")]
    beta = (pml[1], pml[4], pml[7])
    sizes = [nPML * ny * nz, nPML * nx * nz, nPML * nx * ny]
    aux = []
    for face in range(6):
        n = sizes[face % 3] * 9 if face != 5 else 0
        aux += [torch.zeros(max(n, 1), dtype=torch.float32, device=dev) for _ in range(4)] if n else [None] * 4
    border = [1, 1, 1, 1, 1, 1]
    idx = T(s.array("srcIndex"))
    npts = idx.numel()
    rate = T(s.array("momentRate"))
    nt_src = rate.numel() // max(npts * 6, 1)
    slice_ = torch.zeros(max(npts, 1) * 6, dtype=torch.float32, device=dev)
    XYZ = T(s.array("stationXYZ"))
    nst = XYZ.numel() // 3
    wave = torch.zeros(nst * NT * 9, dtype=torch.float32, device=dev)
    pgv = torch.zeros(nx * ny * 2, dtype=torch.float32, device=dev)
    Dis = torch.zeros(npad * 3, dtype=torch.float32, device=dev)

    sh.calculateMomentRate(npts, nt_src, CJM, rate, idx, DH)
    for it in range(nsteps):
        FB = list(FB_TABLE[it % 8])
        if c is not None:
            _add_point(sh, g, c, W, CJM, it, DT, DH, 0)
        sh.addMomenteRate(npts, nt_src, fault_dt, W, idx, rate, slice_, it, 0, DT)
        for irk in range(4):
            sh.waveDeriv(g, h_W, W, CJM, beta, FB, DT)
            sh.freeSurfaceDeriv(g, h_W, W, CJM, DX, DY, beta, FB, DT)
            sh.pmlDeriv(g, nPML, h_W, W, CJM, aux, pml, border, True, FB, DT)
            sh.pmlFreeSurfaceDeriv(g, nPML, W, CJM, aux, DX, DY, pml[2], pml[5], border, FB, DT)
            sh.waveRk(g, irk, h_W, W, t_W, m_W)
            sh.pmlRk(nx, ny, nz, nPML, irk, aux, border, True)
            FB = [-f for f in FB]
        sh.SolveDisplacement(g, W, Dis, DT)
        sh.storageStation(g, NT, nst, XYZ, wave, W, it)
        sh.comparePGV(nx, ny, nz, W, pgv, DT, it)
    torch.cuda.synchronize()
    return (W.cpu().numpy().reshape(info.nzp, info.nyp, info.nxp, 9),
            wave.cpu().numpy().reshape(nst, NT, 9), pgv.cpu().numpy().reshape(ny, nx, 2))


def _source_case(kind, steps, **kw):
    c = {"fault": pu.multi_fault, "ricker": pu.ricker_point, "double_couple": pu.double_couple}[kind](
        steps=steps, courant=0.45, **kw)
    c.gauss_hill = 1
    return c


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["fault", "ricker", "double_couple"])
def test_reference_loop_on_entry_points_matches_session(tmp_path, kind):
    import torch

    from cgfdm.shims import Shims

    c = _source_case(kind, 24)
    d = cases.write_case(c, str(tmp_path / "run"))
    with Session(d, flavor="exact") as s:
        assert s.info.scheme == 0
        W, st, pgv = propagate(Shims("exact"), s, torch, s.info.NT, c.nPML, float(np.float32(c.fault_dt)), c)
        assert (s.info.n_fault_cells > 1) == (kind == "fault") and s.info.n_stations > 0
        s.run(s.info.NT)
        np.testing.assert_array_equal(W, s.wavefield())
        np.testing.assert_array_equal(st, s.stations())
        np.testing.assert_array_equal(pgv, s.pgv()[..., :2])
    assert np.abs(W).max() > 0


def propagate_scfdm(sh, s, torch, nsteps, fault_dt, c=None):
    """The reference's ME-AWENO loop (src/propagate.cpp:186-296 with SCFDM,
    LF, EXP_DECAY, FREE_SURFACE) over the entry points."""
    from cgfdm.shims import Grid

    info = s.info
    nx, ny, nz, NT = info.nx, info.ny, info.nz, info.NT
    DT, DH = info.DT, info.DH
    g = Grid(info.nxp, info.nyp, info.nzp, float(np.float32(1.0 / np.float64(np.float32(DH)))))
    dev = torch.device("cuda:0")
    T = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(dev)
    npad = info.nxp * info.nyp * info.nzp
    h_W, W, RF, m_W = (torch.zeros(npad * 9, dtype=torch.float32, device=dev) for _ in range(4))
    CJM = T(s.cjm())
    idx = T(s.array("srcIndex"))
    npts = idx.numel()
    rate = T(s.array("momentRate"))
    nt_src = rate.numel() // max(npts * 6, 1)
    slice_ = torch.zeros(max(npts, 1) * 6, dtype=torch.float32, device=dev)
    XYZ = T(s.array("stationXYZ"))
    nst = XYZ.numel() // 3
    wave = torch.zeros(nst * NT * 9, dtype=torch.float32, device=dev)
    pgv = torch.zeros(nx * ny * 2, dtype=torch.float32, device=dev)
    Dis = torch.zeros(npad * 3, dtype=torch.float32, device=dev)

    sh.calculateMomentRate(npts, nt_src, CJM, rate, idx, DH, scheme=1)
    for it in range(nsteps):
        if c is not None:
            _add_point(sh, g, c, W, CJM, it, DT, DH, 1)
        sh.addMomenteRate(npts, nt_src, fault_dt, W, idx, rate, slice_, it, 0, DT, scheme=1, CJM=CJM)
        for irk in range(3):
            sh.waveDeriv_alternative_flux_FD(g, h_W, W, RF, CJM, info.Vp_max, DT)
            sh.waveRk_tvd(g, irk, h_W, W, m_W)
        sh.charfreeSurfaceDeriv(g, W, CJM)
        sh.expDecayLayers(g, W, True)
        sh.SolveDisplacement(g, W, Dis, DT, scheme=1, CJM=CJM)
        sh.storageStation(g, NT, nst, XYZ, wave, W, it, scheme=1, CJM=CJM)
        sh.comparePGV(nx, ny, nz, W, pgv, DT, it, scheme=1, CJM=CJM)
    torch.cuda.synchronize()
    return (W.cpu().numpy().reshape(info.nzp, info.nyp, info.nxp, 9),
            wave.cpu().numpy().reshape(nst, NT, 9), pgv.cpu().numpy().reshape(ny, nx, 2))


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["fault", "double_couple"])
def test_reference_scfdm_loop_on_entry_points_matches_session(tmp_path, kind):
    """The same for ME-AWENO: WENO5-JS Lax-Friedrichs fluxes and their
    corrected differences, TVD-RK3, the characteristic free surface and the
    sponge, against the session's exact build (which evaluates the
    characteristic condition with the same restatement)."""
    import torch

    from cgfdm.shims import Shims

    c = _source_case(kind, 20)
    d = cases.write_case(c, str(tmp_path / "run"), scheme="SCFDM")
    with Session(d, flavor="exact") as s:
        assert s.info.scheme == 1
        W, st, pgv = propagate_scfdm(Shims("exact"), s, torch, s.info.NT, float(np.float32(c.fault_dt)), c)
        s.run(s.info.NT)
        np.testing.assert_array_equal(st, s.stations())
        np.testing.assert_array_equal(pgv, s.pgv()[..., :2])
        np.testing.assert_array_equal(W, s.wavefield())
    assert np.abs(W).max() > 0


def test_header_symbols_exported():
    names = re.findall(r"^(?:int|const char \*)\s*(cgfdm_\w+)\(", open(HEADER).read(), re.M)
    assert len(names) >= 13
    for flavor in ("fast", "exact"):
        L = ctypes.CDLL(lib_path(flavor))
        for n in names:
            assert hasattr(L, n), (flavor, n)


def test_argument_errors_without_gpu():
    from cgfdm.shims import Grid, Shims

    sh = Shims("fast")
    g = Grid(10, 10, 10, 0.01)
    with pytest.raises(CgfdmError) as e:
        sh.waveDeriv(g, None, None, None, None, (1, 1, 1), 0.01)
    assert e.value.code == 20003
    with pytest.raises(CgfdmError) as e:
        sh.waveRk(g, 4, None, None, None, None)
    assert e.value.code == 20003
