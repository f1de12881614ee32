"""Shared helpers for the parity tests: case construction and error norms."""

from __future__ import annotations

import math
import os

import numpy as np

from cgfdm import cases


def rel_l2(a: np.ndarray, b: np.ndarray) -> float:
    """||a - b|| / ||b|| over all entries (0 if both vanish)."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    if nb == 0.0:
        return float(np.linalg.norm(a))
    return float(np.linalg.norm(a - b) / nb)


def small_halfspace(steps=60, NX=32, NY=32, NZ=24, nPML=6, **kw) -> cases.Case:
    return cases.halfspace_case(NX=NX, NY=NY, NZ=NZ, nPML=nPML, steps=steps, n_stations=6,
                                depth_m=1000.0, **kw)


def small_hill(steps=60, NX=36, NY=32, NZ=28, nPML=6) -> cases.Case:
    """The reference's single Gauss hill (src/coord.cpp:136-177): height
    0.2 * Depth, width 0.1 * Depth, so a curvilinear grid with steep slopes."""
    c = small_halfspace(steps=steps, NX=NX, NY=NY, NZ=NZ, nPML=nPML, courant=0.45)
    c.gauss_hill = 1
    return c


def multi_fault(steps=60, NX=34, NY=30, NZ=26, nPML=6, seed=7, **kw) -> cases.Case:
    """Several sub-faults of varying mechanism around the centre, some of them
    sharing a grid cell, so the duplicate-cell merge is exercised
    (src/multiSource.cpp:537-592)."""
    rng = np.random.default_rng(seed)
    c = small_halfspace(steps=steps, NX=NX, NY=NY, NZ=NZ, nPML=nPML, **kw)
    DT = c.DT
    nt = int(math.ceil((steps + 2) * DT / 0.01)) + 4
    t = np.arange(nt) * 0.01
    pts = []
    lon0, lat0 = c.center_lon, c.center_lat
    for n in range(9):
        dx, dy = rng.uniform(-350, 350, 2)
        lon, lat = _inv(lon0, lat0, dx, dy)
        depth = float(rng.uniform(600, 1400))
        mu = 2670.0 * 3464.0 ** 2
        rate = (1e15 * cases.ricker(t, rng.uniform(1.5, 3.0), 0.6) / (mu * 1e6)).astype(np.float32)
        rake = np.full(nt, rng.uniform(-180, 180), np.float32)
        pts.append(cases.FaultPoint(lon, lat, -depth, 1e6, float(rng.uniform(0, 360)), float(rng.uniform(20, 90)),
                                    rake, rate))
    # two sub-faults in one cell: identical location
    pts.append(cases.FaultPoint(pts[0].lon, pts[0].lat, pts[0].z, 5e5, 45.0, 60.0, np.full(nt, 30.0, np.float32),
                                pts[0].rate * 0.5))
    pts.append(cases.FaultPoint(lon0, lat0, 0.0, 1e6, 0.0, 90.0, np.zeros(nt, np.float32), np.zeros(nt, np.float32)))
    c.fault = pts
    return c


def ricker_point(steps=60, **kw) -> cases.Case:
    c = small_halfspace(steps=steps, **kw)
    c.fault = []
    c.ricker_point = (c.NX // 2, c.NY // 2, c.NZ - 8, 2.0)
    return c


def double_couple(steps=60, **kw) -> cases.Case:
    c = small_halfspace(steps=steps, **kw)
    c.fault = []
    c.double_couple = dict(X=c.NX // 2 - 2, Y=c.NY // 2 + 1, Z=c.NZ - 9, strike=30.0, dip=60.0, rake=90.0, Mw=4.0,
                           duration=0.3)
    return c


def _inv(lon0, lat0, x, y):
    """lon/lat (degrees) of a point x, y metres from the centre, through the
    same projection the library and the oracle's PROJ stand-in use."""
    return cases.aeqd_inv(lon0, lat0, x, y)
