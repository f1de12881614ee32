"""Synthetic benchmark workloads, written as reference-format run directories.

* ``halfspace``      homogeneous half-space, flat free surface, 128x128x96,
                     DH = 100 m, 12-layer PML, one Mxy point source (M0 =
                     1e16 N m, 2 Hz Ricker moment rate) at 3 km depth, 1000
                     RK4 steps at 0.8 of the stability bound, 16 surface
                     stations on a line: the reference's CPU-runnable case.
* ``terrain_fault``  400x400x200, DH = 100 m, curvilinear grid under a sum of
                     eight Gaussian hills (heights 200-1500 m, widths 2-8 km),
                     four layers over a half-space (Vp 4500 -> 7800 m/s,
                     Vs = Vp / 1.73, Gardner density) with +-3 % Gaussian-
                     correlated perturbations (correlation length 1 km), a
                     40x20 finite fault (strike 30, dip 60, rake 90, k^-2 slip,
                     rupture at 0.8 Vs), 400 surface stations, 3000 steps.
* ``aweno_basin``    the ME-AWENO (SCFDM, TVD-RK3, exponential sponge)
                     workload: 512x512x256, DH = 50 m, terrain as above, a
                     discontinuous medium of seven layers separated by six
                     planar interfaces with seeded dips up to 20 degrees
                     (Vs 1200-3600 m/s, a 3:1 contrast), an ellipsoidal
                     low-velocity basin (Vs = 400 m/s, semi-axes 8 x 5 x 1 km)
                     under the centre of the surface, one 5 Hz Ricker point
                     source, 100 surface stations, 4000 steps.

Everything is drawn from numpy ``default_rng(seed)``.  The terrain and the
heterogeneous medium are raw arrays ("terrainFile", "mediumFile"), which the
library maps through the reference's own terrain-following and medium
conventions; the reference program has no reader for them, so the oracle
build routes them in through its construction hooks.
"""

from __future__ import annotations

import math
import os
from typing import Tuple

import numpy as np

from . import cases

HALO = cases.HALO


def _coords_z(terrain: np.ndarray, NZ: int, DH: float) -> np.ndarray:
    """Terrain-following z of every padded point, float32, as
    src/coord.cpp:228-234 computes it (cal_depth = DH * NZ)."""
    cal = np.float32(np.float32(DH * NZ * 1e-3) * 1000)
    nzp = NZ + 2 * HALO
    DZ = ((terrain.astype(np.float32) + np.abs(cal)).astype(np.float64) / float(NZ - 1)).astype(np.float32)
    K = (np.arange(nzp) - HALO).astype(np.float32)
    return (-np.abs(cal) + DZ[None, :, :] * K[:, None, None]).astype(np.float32)


def hmin_terrain(terrain: np.ndarray, NX: int, NY: int, NZ: int, DH: float, centerX: int, centerY: int) -> float:
    """Smallest point-to-plane distance over the interior (src/calc_CFL.cpp:
    94-163), evaluated slab by slab in float64."""
    nxp, nyp = NX + 2 * HALO, NY + 2 * HALO
    DHf = np.float32(DH)
    x = ((np.arange(nxp) - HALO).astype(np.float32) * DHf - np.float32(centerX) * DHf).astype(np.float64)
    y = ((np.arange(nyp) - HALO).astype(np.float32) * DHf - np.float32(centerY) * DHf).astype(np.float64)
    z = _coords_z(terrain, NZ, DH).astype(np.float64)
    X = np.broadcast_to(x[None, :], (nyp, nxp))
    Y = np.broadcast_to(y[:, None], (nyp, nxp))
    best = np.inf
    I = slice(HALO, nxp - HALO)
    J = slice(HALO, nyp - HALO)
    for k in range(HALO, NZ + HALO):
        P = np.stack([X[J, I], Y[J, I], z[k][J, I]], -1)
        for ii in (-1, 1):
            for jj in (-1, 1):
                for kk in (-1, 1):
                    Ia = slice(HALO - ii, nxp - HALO - ii)
                    Jb = slice(HALO - jj, nyp - HALO - jj)
                    A = np.stack([X[J, Ia], Y[J, Ia], z[k][J, Ia]], -1)
                    B = np.stack([X[Jb, I], Y[Jb, I], z[k][Jb, I]], -1)
                    C = np.stack([X[J, I], Y[J, I], z[k - kk][J, I]], -1)
                    n = np.cross(B - A, C - A)
                    n /= np.linalg.norm(n, axis=-1, keepdims=True)
                    d = np.abs(((P - A) * n).sum(-1))
                    best = min(best, float(d.min()))
    return best


def gaussian_hills(NX: int, NY: int, DH: float, rng: np.random.Generator, n: int = 8,
                   hrange=(200.0, 1500.0), wrange=(2000.0, 8000.0)) -> np.ndarray:
    """Surface height [nyp][nxp] (metres) as a sum of n Gaussian hills."""
    nxp, nyp = NX + 2 * HALO, NY + 2 * HALO
    x = (np.arange(nxp) - HALO - NX // 2) * DH
    y = (np.arange(nyp) - HALO - NY // 2) * DH
    X, Y = np.meshgrid(x, y)
    h = np.zeros((nyp, nxp))
    for _ in range(n):
        cx, cy = rng.uniform(-0.4, 0.4) * NX * DH, rng.uniform(-0.4, 0.4) * NY * DH
        amp = rng.uniform(*hrange)
        w = rng.uniform(*wrange)
        h += amp * np.exp(-((X - cx) ** 2 + (Y - cy) ** 2) / (2 * w * w))
    return h.astype(np.float32)


def layered_perturbed_medium(z: np.ndarray, rng: np.random.Generator, DH: float,
                             vp_layers=(4500.0, 5400.0, 6200.0, 7000.0, 7800.0),
                             depths_m=(2000.0, 6000.0, 12000.0, 18000.0), corr_m=1000.0,
                             sigma=0.01, clip=0.03) -> np.ndarray:
    """(Vs, Vp, rho) volume [nzp][nyp][nxp][3]: layers by depth below the top
    of the model, Vs = Vp / 1.73, Gardner rho = 310 Vp^0.25, times (1 + delta)
    with delta a Gaussian random field of correlation length corr_m."""
    from scipy.ndimage import gaussian_filter

    ztop = z[-HALO - 1].max()
    depth = ztop - z
    vp = np.full(z.shape, vp_layers[-1], np.float32)
    for d, v in zip(reversed(depths_m), reversed(vp_layers[:-1])):
        vp[depth < d] = v
    noise = rng.standard_normal(z.shape).astype(np.float32)
    field = gaussian_filter(noise, sigma=corr_m / DH / math.sqrt(2.0), mode="wrap")
    field *= sigma / max(float(field.std()), 1e-12)
    delta = np.clip(field, -clip, clip)
    vp = vp * (1.0 + delta)
    vs = vp / 1.73
    rho = 310.0 * vp ** 0.25
    return np.stack([vs, vp, rho], -1).astype(np.float32)


def k2_slip(nl: int, nw: int, rng: np.random.Generator, mean_slip: float = 1.0) -> np.ndarray:
    """Random slip with a k^-2 amplitude spectrum beyond the corner wavenumber."""
    kx = np.fft.fftfreq(nl)[None, :]
    ky = np.fft.fftfreq(nw)[:, None]
    k = np.sqrt(kx ** 2 + ky ** 2)
    kc = 1.0 / max(nl, nw)
    amp = 1.0 / (1.0 + (k / kc) ** 2)
    spec = amp * np.exp(2j * np.pi * rng.random((nw, nl)))
    s = np.real(np.fft.ifft2(spec))
    s -= s.min()
    s *= mean_slip / max(float(s.mean()), 1e-12)
    return s.astype(np.float32)


def finite_fault(case_steps: int, DT: float, center_lon: float, center_lat: float, rng: np.random.Generator,
                 nl: int = 40, nw: int = 20, sub_m: float = 500.0, strike=30.0, dip=60.0, rake=90.0,
                 top_depth_m: float = 1000.0, vs: float = 3464.0, rise_s: float = 1.0, fault_dt: float = 0.01):
    """Sub-faults of a planar fault centred under the grid centre."""
    nt = int(math.ceil((case_steps + 2) * DT / fault_dt)) + 4
    t = np.arange(nt) * fault_dt
    slip = k2_slip(nl, nw, rng)
    s_r, d_r = math.radians(strike), math.radians(dip)
    ustrike = np.array([math.sin(s_r), math.cos(s_r), 0.0])          # x east, y north
    udip = np.array([math.cos(s_r) * math.cos(d_r), -math.sin(s_r) * math.cos(d_r), -math.sin(d_r)])
    hypo = (nl // 2, int(nw * 0.7))
    vr = 0.8 * vs
    pts = []
    for iw in range(nw):
        for il in range(nl):
            p = (il - nl / 2 + 0.5) * sub_m * ustrike + (iw + 0.5) * sub_m * udip
            lon, lat = cases.aeqd_inv(center_lon, center_lat, float(p[0]), float(p[1]))
            z = float(p[2]) - top_depth_m
            dist = math.hypot((il - hypo[0]) * sub_m, (iw - hypo[1]) * sub_m)
            tr = dist / vr
            tri = np.clip(1.0 - np.abs(t - tr - rise_s / 2) / (rise_s / 2), 0.0, None) * (2.0 / rise_s)
            rate = (slip[iw, il] * tri).astype(np.float32)
            pts.append(cases.FaultPoint(lon, lat, z, sub_m * sub_m, strike, dip, np.full(nt, rake, np.float32), rate))
    # zero-rate companion at the top of the model: depths in a fault file are
    # measured from its shallowest point (src/multiSource.cpp:209-223)
    pts.append(cases.FaultPoint(center_lon, center_lat, 0.0, 1.0, strike, dip, np.full(nt, rake, np.float32),
                                np.zeros(nt, np.float32)))
    return pts


def surface_stations(NX: int, NY: int, NZ: int, nPML: int, n_side: int) -> list:
    xs = np.linspace(nPML + 4, NX - nPML - 5, n_side).round().astype(int)
    ys = np.linspace(nPML + 4, NY - nPML - 5, n_side).round().astype(int)
    return [(int(x), int(y), NZ - 1) for y in ys for x in xs]


def halfspace(steps: int = 1000) -> cases.Case:
    c = cases.halfspace_case(NX=128, NY=128, NZ=96, DH=100.0, steps=steps, nPML=12)
    return c


def terrain_fault(directory: str, steps: int = 3000, NX: int = 400, NY: int = 400, NZ: int = 200,
                  DH: float = 100.0, nPML: int = 12, seed: int = 2, courant: float = 0.8,
                  scheme: str = "CGFDM", source: str = "fault") -> Tuple[cases.Case, dict]:
    """Writes the curvilinear finite-fault workload into ``directory``.

    ``source="double_couple"`` replaces the finite fault by a point double
    couple 8 cells below the centre of the surface (for small grids, where
    the rupture would not reach the grid within a short run)."""
    rng = np.random.default_rng(seed)
    os.makedirs(directory, exist_ok=True)
    terrain = gaussian_hills(NX, NY, DH, rng)
    z = _coords_z(terrain, NZ, DH)
    med = layered_perturbed_medium(z, rng, DH)
    vp_max = float(med[..., 1].max())
    hmin = hmin_terrain(terrain, NX, NY, NZ, DH, NX // 2, NY // 2)
    DT = cases.cfl_dt(DH, vp_max, courant, hmin=hmin)
    terrain.tofile(os.path.join(directory, "terrain.bin"))
    med.tofile(os.path.join(directory, "medium.bin"))
    fault = finite_fault(steps, DT, 100.0, 30.0, rng)
    c = cases.Case(NX=NX, NY=NY, NZ=NZ, DH=DH, DT=DT, steps=steps, nPML=nPML, layers=(),
                   fault=fault, stations=surface_stations(NX, NY, NZ, nPML, 20),
                   extra={"terrainFile": "terrain.bin", "mediumFile": "medium.bin", "useMedium": 1})
    if source == "double_couple":
        c.fault = []
        c.double_couple = dict(X=NX // 2, Y=NY // 2, Z=NZ - 8, strike=30.0, dip=60.0, rake=90.0, Mw=4.0,
                               duration=0.3)
    cases.write_case(c, directory, scheme=scheme)
    return c, {"hmin": hmin, "vp_max": vp_max, "DT": DT}


def dipping_layers_basin(z: np.ndarray, NX: int, NY: int, DH: float, rng: np.random.Generator,
                         n_interfaces: int = 6, max_dip_deg: float = 20.0, vs_range=(1200.0, 3600.0),
                         basin_vs: float = 400.0, basin_axes_m=(8000.0, 5000.0, 1000.0)) -> np.ndarray:
    """(Vs, Vp, rho) volume [nzp][nyp][nxp][3] with sharp planar dipping
    interfaces and an ellipsoidal basin.  Interface i passes through depth
    d_i under the grid centre with a seeded dip (<= max_dip_deg) and dip
    direction; Vs rises layer by layer from vs_range[0] to vs_range[1];
    Vp = 1.73 Vs, Gardner rho = 310 Vp^0.25.  The basin is centred under the
    centre of the free surface and measured from the local surface."""
    nzp, nyp, nxp = z.shape
    x = ((np.arange(nxp) - HALO - NX // 2) * DH).astype(np.float64)
    y = ((np.arange(nyp) - HALO - NY // 2) * DH).astype(np.float64)
    ztop_col = z[-HALO - 1].astype(np.float64)                  # surface height per column
    depth_total = float(ztop_col.max() - z[HALO].min())
    d0 = np.sort(rng.uniform(0.08, 0.85, n_interfaces)) * depth_total
    dips = np.radians(rng.uniform(0.0, max_dip_deg, n_interfaces))
    az = rng.uniform(0.0, 2.0 * np.pi, n_interfaces)
    vs_layers = np.sort(rng.uniform(vs_range[0], vs_range[1], n_interfaces + 1))
    vs_layers[0], vs_layers[-1] = vs_range
    X, Y = np.meshgrid(x, y)
    zref = float(ztop_col.max())
    vs = np.full(z.shape, vs_layers[0], np.float32)
    for n in range(n_interfaces):
        # interface depth below zref, a plane dipping along azimuth az
        dint = d0[n] + np.tan(dips[n]) * (np.cos(az[n]) * X + np.sin(az[n]) * Y)
        below = (zref - z) > dint[None, :, :]
        vs[below] = vs_layers[n + 1]
    ax, ay, az_ = basin_axes_m
    dsurf = ztop_col[None, :, :] - z
    inside = (X[None] / ax) ** 2 + (Y[None] / ay) ** 2 + (dsurf / az_) ** 2 <= 1.0
    vs[inside] = basin_vs
    vp = (vs * 1.73).astype(np.float32)
    rho = (310.0 * vp.astype(np.float64) ** 0.25).astype(np.float32)
    return np.stack([vs, vp, rho], -1).astype(np.float32)


def aweno_basin(directory: str, steps: int = 4000, NX: int = 512, NY: int = 512, NZ: int = 256,
                DH: float = 50.0, seed: int = 3, courant: float = 0.5, fc: float = 5.0,
                n_side: int = 10) -> Tuple[cases.Case, dict]:
    """Writes the ME-AWENO basin workload (SCFDM scheme) into ``directory``."""
    rng = np.random.default_rng(seed)
    os.makedirs(directory, exist_ok=True)
    # hills scaled with the model: heights 200-1500 m, widths 2-8 km
    terrain = gaussian_hills(NX, NY, DH, rng)
    z = _coords_z(terrain, NZ, DH)
    med = dipping_layers_basin(z, NX, NY, DH, rng)
    vp_max = float(med[..., 1].max())
    hmin = hmin_terrain(terrain, NX, NY, NZ, DH, NX // 2, NY // 2)
    DT = cases.cfl_dt(DH, vp_max, courant, hmin=hmin)
    terrain.tofile(os.path.join(directory, "terrain.bin"))
    med.tofile(os.path.join(directory, "medium.bin"))
    c = cases.Case(NX=NX, NY=NY, NZ=NZ, DH=DH, DT=DT, steps=steps, nPML=12, layers=(), fault=[],
                   stations=surface_stations(NX, NY, NZ, 20, n_side),
                   extra={"terrainFile": "terrain.bin", "mediumFile": "medium.bin", "useMedium": 1})
    # 2 km below the surface, or half the model depth on small grids
    c.ricker_point = (NX // 2, NY // 2, NZ - 1 - min(int(round(2000.0 / DH)), NZ // 2), fc)
    cases.write_case(c, directory, scheme="SCFDM")
    return c, {"hmin": hmin, "vp_max": vp_max, "DT": DT}


def batch_shots(root: str, n: int = 32, steps: int = 1500, seed: int = 5, sizes=((64, 256), (64, 256), (64, 128)),
                DH: float = 100.0, nPML: int = 12, n_stations: int = 32, courant: float = 0.8) -> list:
    """Writes ``n`` independent CGFDM run directories root/shot_<i> for the
    batched workload: grid sizes drawn from ``sizes`` (NX, NY, NZ ranges),
    a random layered medium (3-6 layers, Vs 1500-4500 m/s increasing with
    depth, Vp = 1.73 Vs, Gardner density), Gaussian-hill terrain of random
    amplitude up to 1 km, one point moment tensor (random strike, dip, rake;
    M0 = 1e16 N m with a Ricker moment rate of 1-4 Hz) at 30 % of the model
    depth, ``n_stations`` surface stations.  Returns the directories."""
    rng = np.random.default_rng(seed)
    dirs = []
    for s in range(n):
        NX = int(rng.integers(sizes[0][0], sizes[0][1] + 1))
        NY = int(rng.integers(sizes[1][0], sizes[1][1] + 1))
        NZ = int(rng.integers(sizes[2][0], sizes[2][1] + 1))
        d = os.path.join(root, f"shot_{s:02d}")
        os.makedirs(d, exist_ok=True)
        terrain = gaussian_hills(NX, NY, DH, rng)
        amp = float(rng.uniform(0.0, 1000.0))
        terrain = (terrain * (amp / max(float(terrain.max()), 1e-6))).astype(np.float32)
        nl = int(rng.integers(3, 7))
        depth_total = NZ * DH
        tops = np.concatenate([[0.0], np.sort(rng.uniform(0.1, 0.9, nl - 1)) * depth_total]) / 1000.0
        vs = np.sort(rng.uniform(1500.0, 4500.0, nl))
        vp = 1.73 * vs
        rho = 310.0 * vp ** 0.25
        layers = tuple((float(tops[i]), float(vs[i] / 1000), float(vp[i] / 1000), float(rho[i] / 1000))
                       for i in range(nl))
        vp_max = float(vp.max())
        hmin = hmin_terrain(terrain, NX, NY, NZ, DH, NX // 2, NY // 2)
        DT = cases.cfl_dt(DH, vp_max, courant, hmin=hmin)
        depth_src = 0.3 * depth_total
        li = int(np.searchsorted(tops * 1000.0, depth_src, side="right") - 1)
        mu = float(rho[li] * vs[li] ** 2)
        fault, _ = cases.moment_fault(steps, DT, 0.01, 100.0, 30.0, depth_src, 1e16, float(rng.uniform(1.0, 4.0)),
                                      mu, strike=float(rng.uniform(0, 360)), dip=float(rng.uniform(10, 90)),
                                      rake=float(rng.uniform(-180, 180)))
        xs = rng.integers(nPML + 4, NX - nPML - 4, n_stations)
        ys = rng.integers(nPML + 4, NY - nPML - 4, n_stations)
        stations = [(int(x), int(y), NZ - 1) for x, y in zip(xs, ys)]
        terrain.tofile(os.path.join(d, "terrain.bin"))
        c = cases.Case(NX=NX, NY=NY, NZ=NZ, DH=DH, DT=DT, steps=steps, nPML=nPML, layers=layers, fault=fault,
                       stations=stations, extra={"terrainFile": "terrain.bin"})
        cases.write_case(c, d)
        dirs.append(d)
    return dirs


def adjoint_layers(NX: int, NY: int, NZ: int, DH: float, anomaly: bool, radius: float = 2000.0,
                   dvs: float = 0.08) -> np.ndarray:
    """Medium of the adjoint workload, [nzp][nyp][nxp][3] (Vs, Vp, rho):
    four layers over a half-space under a flat surface (Vp 4500 -> 7000 m/s,
    Vs = Vp / 1.73, Gardner density), and, with ``anomaly``, a ball of
    radius ``radius`` (2 km) of Vs + ``dvs`` (8 %) centred at 40 % of the
    model depth."""
    nxp, nyp, nzp = NX + 2 * HALO, NY + 2 * HALO, NZ + 2 * HALO
    depth = (NZ - 1 - (np.arange(nzp) - HALO)) * DH          # metres below the surface
    tops = np.array([0.0, 0.15, 0.3, 0.5, 0.7]) * NZ * DH
    vps = np.array([4500.0, 5200.0, 5900.0, 6500.0, 7000.0])
    li = np.clip(np.searchsorted(tops, depth, side="right") - 1, 0, len(tops) - 1)
    vp = np.broadcast_to(vps[li][:, None, None], (nzp, nyp, nxp)).astype(np.float64)
    vs = vp / 1.73
    rho = 310.0 * vp ** 0.25
    if anomaly:
        kk, jj, ii = np.meshgrid(np.arange(nzp), np.arange(nyp), np.arange(nxp), indexing="ij")
        zc = (NZ - 1) - 0.4 * NZ + HALO
        r = np.sqrt((ii - (nxp - 1) / 2) ** 2 + (jj - (nyp - 1) / 2) ** 2 + (kk - zc) ** 2) * DH
        vs = vs * np.where(r < radius, 1.0 + dvs, 1.0)
    return np.stack([vs, vp, rho], -1).astype(np.float32)


def adjoint_shots(root: str, steps: int = 2000, NX: int = 192, NY: int = 192, NZ: int = 128, DH: float = 100.0,
                  nPML: int = 12, n_shots: int = 4, n_side: int = 8, courant: float = 0.8, seed: int = 9) -> dict:
    """The adjoint workload: ``n_shots`` run directories root/shot_<i> over
    one model (the starting medium, no anomaly, as medium.bin; the true
    medium with the Vs ball beside it as medium_true.bin), each with one 2 Hz
    Ricker point source at a seeded position at 1/4 of the model depth and
    the same n_side x n_side surface stations (64).  Returns the shot
    directories, DT and the two media."""
    rng = np.random.default_rng(seed)
    start = adjoint_layers(NX, NY, NZ, DH, False)
    true = adjoint_layers(NX, NY, NZ, DH, True)
    vp_max = float(true[..., 1].max())
    DT = cases.cfl_dt(DH, vp_max, courant)
    stations = surface_stations(NX, NY, NZ, nPML, n_side)
    dirs = []
    for s in range(n_shots):
        d = os.path.join(root, f"shot_{s}")
        os.makedirs(d, exist_ok=True)
        X = int(rng.integers(nPML + 16, NX - nPML - 16))
        Y = int(rng.integers(nPML + 16, NY - nPML - 16))
        c = cases.Case(NX=NX, NY=NY, NZ=NZ, DH=DH, DT=DT, steps=steps, nPML=nPML, stations=stations,
                       ricker_point=(X, Y, int(NZ * 0.75), 2.0),
                       extra={"mediumFile": "medium.bin", "useMedium": 1})
        cases.write_case(c, d)
        start.tofile(os.path.join(d, "medium.bin"))
        dirs.append(d)
    return {"dirs": dirs, "DT": DT, "start": start, "true": true}
