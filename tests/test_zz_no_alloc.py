"""The allocation-free entry point, cgfdm_hrange_noalloc, against the session.

Some callers cannot allocate device memory when they need the CFL spacing
check.  Examples are an application whose other streams run a live
simulation, where cudaMalloc and cudaFree may synchronize the device, and an
embedder whose pool allocator owns the GPU memory.  cgfdm_hrange_noalloc
serves them from a static device array.  This test calls it through the C
ABI, twice in a row on the same static scratch.  Each result is checked
against H_min from cgfdm_create, the existing entry point, for a flat grid
and a terrain-following grid, and a smaller grid after a larger one is
checked exactly against a float64 restatement.  The file is named so that
pytest collects it last.
"""

import ctypes
import os

import numpy as np
import pytest

import cgfdm
from cgfdm import cases, configs

HALO = 3
TOL = 1e-5  # relative, as the parity tests


def _flat_xy(NX, NY, DH, cx, cy):
    DHf = np.float32(DH)
    x = ((np.arange(NX + 2 * HALO) - HALO).astype(np.float32) * DHf - np.float32(cx) * DHf).astype(np.float32)
    y = ((np.arange(NY + 2 * HALO) - HALO).astype(np.float32) * DHf - np.float32(cy) * DHf).astype(np.float32)
    return x, y


def _coords(NX, NY, NZ, DH, terrain=None):
    """The library's coordinate array, [nz+6][ny+6][nx+6][3] float32."""
    x, y = _flat_xy(NX, NY, DH, NX // 2, NY // 2)
    nzp = NZ + 2 * HALO
    if terrain is None:
        K = (np.arange(nzp) - HALO + 1).astype(np.float32)
        z1 = (K * np.float32(DH) - np.float32(NZ) * np.float32(DH)).astype(np.float32)
        z = np.broadcast_to(z1[:, None, None], (nzp, NY + 2 * HALO, NX + 2 * HALO))
    else:
        z = configs._coords_z(terrain, NZ, DH)
    c = np.empty((nzp, NY + 2 * HALO, NX + 2 * HALO, 3), np.float32)
    c[..., 0] = x[None, None, :]
    c[..., 1] = y[None, :, None]
    c[..., 2] = z
    return c


def _hrange_f64(coord):
    """Smallest and largest point-to-plane distance of the interior points to
    their six diagonal-neighbour planes (src/calc_CFL.cpp:56-163), in float64
    with the library's operation order; numpy rounds every operation as the
    device's explicitly rounded intrinsics do, so the result is exact."""
    c = coord.astype(np.float64)
    nzp, nyp, nxp, _ = c.shape
    I = slice(HALO, nxp - HALO)
    J = slice(HALO, nyp - HALO)
    K = slice(HALO, nzp - HALO)
    P = c[K, J, I]
    lo, hi = np.inf, 0.0

    def sh(di, dj, dk):
        return c[HALO + dk:nzp - HALO + dk, HALO + dj:nyp - HALO + dj, HALO + di:nxp - HALO + di]

    for ii in (-1, 1):
        for jj in (-1, 1):
            for kk in (-1, 1):
                A, B, C = sh(-ii, 0, 0), sh(0, -jj, 0), sh(0, 0, -kk)
                AB, AC, PA = B - A, C - A, P - A
                n0 = AB[..., 1] * AC[..., 2] - AB[..., 2] * AC[..., 1]
                n1 = AB[..., 2] * AC[..., 0] - AB[..., 0] * AC[..., 2]
                n2 = AB[..., 0] * AC[..., 1] - AB[..., 1] * AC[..., 0]
                nd = np.sqrt((n0 * n0 + n1 * n1) + n2 * n2)
                n0, n1, n2 = n0 / nd, n1 / nd, n2 / nd
                d = np.abs((PA[..., 0] * n0 + PA[..., 1] * n1) + PA[..., 2] * n2)
                lo, hi = min(lo, d.min()), max(hi, d.max())
    return lo, hi


def _lib():
    L = cgfdm.load("fast")
    L.cgfdm_hrange_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                                       ctypes.c_void_p]
    L.cgfdm_hrange_noalloc.restype = ctypes.c_int
    L.cgfdm_noalloc_last_error.restype = ctypes.c_char_p
    return L


def _check(run_dir, coord, NX, NY, NZ):
    import torch

    L = _lib()
    with cgfdm.Session(run_dir) as s:
        h_session = s.info.H_min
    d_coord = torch.from_numpy(np.ascontiguousarray(coord)).cuda()
    stream = torch.cuda.current_stream()
    for call in range(2):
        d_out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
        rc = L.cgfdm_hrange_noalloc(ctypes.c_void_p(d_coord.data_ptr()), NX, NY, NZ,
                                    ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, L.cgfdm_noalloc_last_error().decode()
        torch.cuda.synchronize()
        hmin, hmax = d_out.cpu().numpy()
        assert abs(float(np.float32(hmin)) - h_session) <= TOL * h_session, (call, hmin, h_session)
        assert hmax >= hmin > 0.0
    return hmin, hmax


@pytest.mark.gpu
def test_noalloc_matches_session_flat(tmp_path):
    c = cases.halfspace_case(NX=40, NY=36, NZ=30, nPML=6, steps=4, n_stations=2)
    cases.write_case(c, str(tmp_path))
    hmin, hmax = _check(str(tmp_path), _coords(40, 36, 30, 100.0), 40, 36, 30)
    assert abs(hmin - 100.0 / np.sqrt(3.0)) < 1e-9 * 100


@pytest.mark.gpu
def test_noalloc_matches_session_terrain(tmp_path):
    d = str(tmp_path)
    configs.terrain_fault(d, steps=4, NX=64, NY=60, NZ=40, nPML=6)
    terrain = np.fromfile(os.path.join(d, "terrain.bin"), np.float32).reshape(60 + 2 * HALO, 64 + 2 * HALO)
    _check(d, _coords(64, 60, 40, 100.0, terrain), 64, 60, 40)


@pytest.mark.gpu
def test_noalloc_smaller_grid_after_larger():
    """A larger grid, then a smaller one, then the larger again, on the same
    static scratch: the smaller call must not pick up partials the larger one
    left behind.  Both H_min and H_max are checked exactly against a float64
    restatement computed here."""
    import torch

    L = _lib()
    rng = np.random.default_rng(7)
    big = (72, 64, 48)
    small = (24, 20, 18)
    terrain = (rng.standard_normal((big[1] + 2 * HALO, big[0] + 2 * HALO)) * 60.0).astype(np.float32)
    cbig = _coords(*big, 100.0, terrain)
    csmall = _coords(*small, 50.0)
    stream = torch.cuda.current_stream()
    for coord, (NX, NY, NZ) in ((cbig, big), (csmall, small), (cbig, big)):
        want = _hrange_f64(coord)
        d_coord = torch.from_numpy(np.ascontiguousarray(coord)).cuda()
        d_out = torch.full((2,), -1.0, dtype=torch.float64, device="cuda")
        rc = L.cgfdm_hrange_noalloc(ctypes.c_void_p(d_coord.data_ptr()), NX, NY, NZ,
                                    ctypes.c_void_p(d_out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))
        assert rc == 0, L.cgfdm_noalloc_last_error().decode()
        torch.cuda.synchronize()
        got = d_out.cpu().numpy()
        assert got[0] == want[0] and got[1] == want[1], (NX, got, want)


@pytest.mark.gpu
def test_noalloc_rejects_too_many_blocks_along_y():
    import torch

    L = _lib()
    d_coord = torch.zeros(3 * 8 * 8 * 8, dtype=torch.float32, device="cuda")
    d_out = torch.zeros(2, dtype=torch.float64, device="cuda")
    # 1 x 65536 x 1 blocks: within the scratch's 65536 pairs, above the launch limit along y
    rc = L.cgfdm_hrange_noalloc(ctypes.c_void_p(d_coord.data_ptr()), 32, 8 * 65536, 16,
                                ctypes.c_void_p(d_out.data_ptr()), None)
    assert rc == 20003
    assert b"65535" in L.cgfdm_noalloc_last_error()


@pytest.mark.gpu
def test_noalloc_rejects_oversized_grid():
    import torch

    L = _lib()
    d_coord = torch.zeros(3 * 8 * 8 * 8, dtype=torch.float32, device="cuda")
    d_out = torch.zeros(2, dtype=torch.float64, device="cuda")
    rc = L.cgfdm_hrange_noalloc(ctypes.c_void_p(d_coord.data_ptr()), 100000, 100000, 1000,
                                ctypes.c_void_p(d_out.data_ptr()), None)
    assert rc == 20003
    assert b"static scratch" in L.cgfdm_noalloc_last_error()
