"""Writers for run directories in the reference's own input formats.

A run directory holds what the reference program reads from its working
directory: ``params.json`` (keys read by src/getParams.cpp:58-232),
``station.json`` (src/station.cpp:92-292), an optional layered-medium file
(src/medium.cpp:143-267) and an optional finite-fault source file
(src/multiSource.cpp:24-94,345-396).  The same directory drives the library
(``cgfdm.Session``) and the reference CPU build used as the oracle, so both
see byte-identical inputs.

Formats (little-endian):
  * layered model: int32 layers, then per layer float32 depth[km], Vs[km/s],
    Vp[km/s], rho[g/cm^3] (src/medium.cpp:163-186);
  * finite fault: int32 npts, int32 nt, float32 dt, then per point float32
    lon, lat, z[m], area[m^2], strike, dip, rake[nt], rate[nt]
    (src/multiSource.cpp:36-47,363-379);
  * stations: {"station(point)": {"name": [X, Y, Z], ...}} with global grid
    indices (src/station.cpp:136-183).

All synthetic inputs are generated from seeded numpy generators.
"""

from __future__ import annotations

import json
import math
import os
import struct
from dataclasses import dataclass, field
from typing import List, Optional, Sequence, Tuple

import numpy as np

HALO = 3

# params.json keys the reference reads; every one is written so that no field
# of the reference's PARAMS struct is left uninitialised (src/main.cpp:20).
_DEFAULT_PARAMS = {
    "TMAX": 1.0, "DT": 0.01, "DH": 100.0,
    "NX": 32, "NY": 32, "NZ": 32,
    "PX": 1, "PY": 1, "PZ": 1,
    "centerX": 16, "centerY": 16,
    "centerLatitude": 30.0, "centerLongitude": 100.0,
    "IT_SKIP": 1000000,
    "sliceX": 16, "sliceY": 16, "sliceZ": 16, "sliceFreeSurf": 0,
    "nPML": 6,
    "gauss_hill": 0, "useTerrain": 0, "useMedium": 0, "useMultiSource": 0,
    "LayeredModel": 0, "LayeredFileName": "./layered.bin",
    "useSingleSource(ricker)": 0, "useSingleSource(double_couple)": 0,
    "rickerfc": 2.0, "strike": 0.0, "dip": 90.0, "rake": 0.0, "Mw": 5.0, "duration": 1.0,
    "ShenModel": 0, "Crust_1Model": 0,
    "itSlice": 0, "itStep": 1, "waveOutput": "v", "sliceName": "s",
    "itStart": 0, "itEnd": 0, "igpu": 0,
    "OUT": "./output",
    "TerrainDir": "./terrain", "SRTM90": 0,
    "lonStart": 100, "latStart": 30, "blockX": 1, "blockY": 1,
    "Depth(km)": 10.0,
    "MLonStart": 0.0, "MLatStart": 0.0, "MLonEnd": 0.0, "MLatEnd": 0.0,
    "MLonStep": 0.5, "MLatStep": 0.5, "CrustLonStep": 1.0, "CrustLatStep": 1.0,
    "MVeticalStep": 500.0, "MediumDir": "./medium", "CrustDir": "./crust",
    "sourceX": 16, "sourceY": 16, "sourceZ": 16,
    "sourceFile": "source.bin", "sourceDir": ".",
    "degree2radian": 1,
}


_WGS84_A = 6378137.0
_WGS84_F = 1.0 / 298.257223563


def aeqd_inv(lon0_deg: float, lat0_deg: float, x: float, y: float) -> Tuple[float, float]:
    """Longitude/latitude (degrees) of the point x east, y north (metres) of
    the centre: the direct geodesic problem on WGS84 (Vincenty 1975), the
    inverse of the azimuthal-equidistant projection the library and the
    reference use to place sub-faults (src/multiSource.cpp:122-171)."""
    a, f = _WGS84_A, _WGS84_F
    b = a * (1 - f)
    lon0, lat0 = math.radians(lon0_deg), math.radians(lat0_deg)
    s = math.hypot(x, y)
    if s == 0.0:
        return lon0_deg, lat0_deg
    alpha1 = math.atan2(x, y)
    sA1, cA1 = math.sin(alpha1), math.cos(alpha1)
    tanU1 = (1 - f) * math.tan(lat0)
    cosU1 = 1 / math.sqrt(1 + tanU1 * tanU1)
    sinU1 = tanU1 * cosU1
    sig1 = math.atan2(tanU1, cA1)
    sinAl = cosU1 * sA1
    cos2Al = 1 - sinAl * sinAl
    u2 = cos2Al * (a * a - b * b) / (b * b)
    A = 1 + u2 / 16384 * (4096 + u2 * (-768 + u2 * (320 - 175 * u2)))
    B = u2 / 1024 * (256 + u2 * (-128 + u2 * (74 - 47 * u2)))
    sig = s / (b * A)
    for _ in range(200):
        c2m = math.cos(2 * sig1 + sig)
        ss, cs = math.sin(sig), math.cos(sig)
        dS = B * ss * (c2m + B / 4 * (cs * (-1 + 2 * c2m * c2m) - B / 6 * c2m * (-3 + 4 * ss * ss) *
                                      (-3 + 4 * c2m * c2m)))
        new = s / (b * A) + dS
        if abs(new - sig) < 1e-14:
            sig = new
            break
        sig = new
    c2m = math.cos(2 * sig1 + sig)
    ss, cs = math.sin(sig), math.cos(sig)
    tmp = sinU1 * ss - cosU1 * cs * cA1
    phi2 = math.atan2(sinU1 * cs + cosU1 * ss * cA1, (1 - f) * math.sqrt(sinAl * sinAl + tmp * tmp))
    lam = math.atan2(ss * sA1, cosU1 * cs - sinU1 * ss * cA1)
    C = f / 16 * cos2Al * (4 + f * (4 - 3 * cos2Al))
    L = lam - (1 - C) * f * sinAl * (sig + C * ss * (c2m + C * cs * (-1 + 2 * c2m * c2m)))
    return math.degrees(lon0 + L), math.degrees(phi2)


def ricker(t: np.ndarray, fc: float, t0: Optional[float] = None) -> np.ndarray:
    """Ricker wavelet of peak frequency fc, delayed by t0 (default 1/fc)."""
    if t0 is None:
        t0 = 1.0 / fc
    a = (math.pi * fc * (t - t0)) ** 2
    return (1.0 - 2.0 * a) * np.exp(-a)


def cfl_dt(DH: float, vp_max: float, courant: float = 0.8, hmin: Optional[float] = None) -> float:
    """Time step at a fraction of the reference's stability bound.

    The reference accepts DT <= 1.34 * H_min / Vp_max (src/calc_CFL.cpp:325-345),
    where H_min is the smallest point-to-plane distance through diagonal
    neighbours, DH/sqrt(3) on a flat grid (src/calc_CFL.cpp:94-163).
    """
    if hmin is None:
        hmin = DH / math.sqrt(3.0)
    return courant * 1.34 * hmin / vp_max


@dataclass
class FaultPoint:
    lon: float
    lat: float
    z: float          # metres, positive up; depth is referenced to the shallowest point
    area: float
    strike: float
    dip: float
    rake: np.ndarray  # [nt]
    rate: np.ndarray  # [nt]


@dataclass
class Case:
    """A complete run description, written out by :func:`write_case`."""

    NX: int
    NY: int
    NZ: int
    DH: float
    DT: float
    steps: int
    nPML: int = 6
    layers: Sequence[Tuple[float, float, float, float]] = ((0.0, 3.464, 6.0, 2.67), (1000.0, 3.464, 6.0, 2.67))
    gauss_hill: int = 0
    center_lon: float = 100.0
    center_lat: float = 30.0
    fault_dt: float = 0.01
    fault: List[FaultPoint] = field(default_factory=list)
    ricker_point: Optional[Tuple[int, int, int, float]] = None   # X, Y, Z, fc
    double_couple: Optional[dict] = None                         # X, Y, Z, strike, dip, rake, Mw, duration
    stations: List[Tuple[int, int, int]] = field(default_factory=list)
    it_skip: int = 1000000
    slice_xyz: Tuple[int, int, int] = (-1, -1, -1)
    slice_free_surface: int = 0
    extra: dict = field(default_factory=dict)

    @property
    def TMAX(self) -> float:
        # NT = (int)(TMAX / DT) with DT rounded to float (src/propagate.cpp:88);
        # half a step of margin keeps the truncation on the intended count.
        return (self.steps + 0.5) * float(np.float32(self.DT))


def write_layered(path: str, layers: Sequence[Tuple[float, float, float, float]]) -> None:
    with open(path, "wb") as f:
        f.write(struct.pack("<i", len(layers)))
        for depth_km, vs, vp, rho in layers:
            f.write(struct.pack("<ffff", depth_km, vs, vp, rho))


def write_fault(path: str, points: Sequence[FaultPoint], nt: int, dt: float) -> None:
    with open(path, "wb") as f:
        f.write(struct.pack("<iif", len(points), nt, dt))
        for p in points:
            f.write(struct.pack("<ffffff", p.lon, p.lat, p.z, p.area, p.strike, p.dip))
            f.write(np.asarray(p.rake, dtype="<f4").tobytes())
            f.write(np.asarray(p.rate, dtype="<f4").tobytes())


def write_stations(path: str, stations: Sequence[Tuple[int, int, int]]) -> None:
    obj = {"station(point)": {str(i): [int(x), int(y), int(z)] for i, (x, y, z) in enumerate(stations)}}
    with open(path, "w") as f:
        json.dump(obj, f, indent=1)


def write_case(case: Case, directory: str, scheme: str = "CGFDM") -> str:
    """Write params.json, station.json and the input files into ``directory``."""
    os.makedirs(directory, exist_ok=True)
    os.makedirs(os.path.join(directory, "output"), exist_ok=True)
    p = dict(_DEFAULT_PARAMS)
    p.update({
        "TMAX": case.TMAX, "DT": case.DT, "DH": case.DH,
        "NX": case.NX, "NY": case.NY, "NZ": case.NZ,
        "centerX": case.NX // 2, "centerY": case.NY // 2,
        "centerLongitude": case.center_lon, "centerLatitude": case.center_lat,
        "IT_SKIP": case.it_skip,
        "sliceX": case.slice_xyz[0], "sliceY": case.slice_xyz[1], "sliceZ": case.slice_xyz[2],
        "sliceFreeSurf": case.slice_free_surface,
        "nPML": case.nPML, "gauss_hill": case.gauss_hill,
        "Depth(km)": case.DH * case.NZ * 1e-3,
        "scheme": scheme,
    })
    if case.layers:
        write_layered(os.path.join(directory, "layered.bin"), case.layers)
        p.update({"useMedium": 1, "LayeredModel": 1, "LayeredFileName": "./layered.bin"})
    if case.fault:
        nt = len(case.fault[0].rate)
        write_fault(os.path.join(directory, "source.bin"), case.fault, nt, case.fault_dt)
        p.update({"useMultiSource": 1, "sourceDir": ".", "sourceFile": "source.bin"})
    if case.ricker_point is not None:
        X, Y, Z, fc = case.ricker_point
        p.update({"useSingleSource(ricker)": 1, "sourceX": X, "sourceY": Y, "sourceZ": Z, "rickerfc": fc})
    if case.double_couple is not None:
        dc = case.double_couple
        p.update({"useSingleSource(double_couple)": 1, "sourceX": dc["X"], "sourceY": dc["Y"],
                  "sourceZ": dc["Z"], "strike": dc["strike"], "dip": dc["dip"], "rake": dc["rake"],
                  "Mw": dc["Mw"], "duration": dc["duration"]})
    p.update(case.extra)
    with open(os.path.join(directory, "params.json"), "w") as f:
        json.dump(p, f, indent=1)
    write_stations(os.path.join(directory, "station.json"), case.stations)
    return directory


def moment_fault(case_steps: int, DT: float, fault_dt: float, lon: float, lat: float, depth_m: float,
                 m0: float, fc: float, mu: float, area: float = 1.0e6,
                 strike: float = 0.0, dip: float = 90.0, rake: float = 0.0,
                 with_dummy: bool = True) -> Tuple[List[FaultPoint], int]:
    """A point moment-tensor source written as a finite-fault file.

    Moment rate M0 * Ricker(t; fc) is encoded as rate = M0 * r(t) / (mu *
    area), because the reference scales rate*area by mu/(J*DH^3)
    (src/multiSource.cpp:514-519, src/addMoment.cpp:52-61).  Depth in a
    fault file is measured from its shallowest point (src/multiSource.cpp:
    209-223), so a zero-rate companion point ``depth_m`` shallower fixes the
    real point's depth below the top of the model.  The table is long enough
    that the reference never reaches its end-of-table branch
    (src/addMoment.cpp:296-302).
    """
    nt = int(math.ceil((case_steps + 2) * DT / fault_dt)) + 4
    t = np.arange(nt) * fault_dt
    rate = (m0 * ricker(t, fc) / (mu * area)).astype(np.float32)
    pts = [FaultPoint(lon, lat, -depth_m, area, strike, dip, np.full(nt, rake, np.float32), rate)]
    if with_dummy:
        pts.append(FaultPoint(lon, lat, 0.0, area, strike, dip, np.full(nt, rake, np.float32),
                              np.zeros(nt, np.float32)))
    return pts, nt


def halfspace_case(NX=128, NY=128, NZ=96, DH=100.0, steps=1000, nPML=12, courant=0.8,
                   vp=6000.0, vs=3464.0, rho=2670.0, depth_m=3000.0, m0=1e16, fc=2.0,
                   n_stations=16, gauss_hill=0, DT=None) -> Case:
    """Homogeneous half-space with a flat free surface and one Mxy point source.

    The 128x128x96, DH=100 m, nPML=12, 1000-step configuration is the
    reference's CPU-runnable benchmark case; smaller sizes are parity cases.
    """
    if DT is None:
        DT = cfl_dt(DH, vp, courant)
    mu = rho * vs * vs
    fault, _ = moment_fault(steps, DT, 0.01, 100.0, 30.0, depth_m, m0, fc, mu)
    j = NY // 2
    step = max(1, (NX - 2 * nPML - 8) // max(1, n_stations))
    i0 = nPML + 4
    stations = [(i0 + step * n, j, NZ - 1) for n in range(n_stations) if i0 + step * n < NX - nPML]
    layer = (vs / 1000.0, vp / 1000.0, rho / 1000.0)
    return Case(NX=NX, NY=NY, NZ=NZ, DH=DH, DT=DT, steps=steps, nPML=nPML,
                layers=((0.0,) + layer, (1000.0,) + layer), gauss_hill=gauss_hill,
                fault=fault, stations=stations)
