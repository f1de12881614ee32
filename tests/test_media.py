"""Real-data medium inputs against the reference's CPU build: Weisen Shen's
Vs model (ShenModel, src/dealMedium.cpp:49-360) read from per-node ".mod"
text files, interpolated to the grid's longitudes and latitudes (inverse
azimuthal-equidistant projection about the centre), layered by depth below
the model top, Vp and rho from Vs.  The packed medium (mu, lambda,
buoyancy of every padded point) must equal the reference's bit for bit.

The node files are synthetic: seeded Vs profiles of the published format
(depth, Vs, error per line, km and km/s) on a 0.1-degree grid around the
model, whose 12 x 10 km extent spans several nodes."""

import os

import numpy as np
import pytest

import parity_util as pu
import refrun
from cgfdm import Session, cases


def write_shen_nodes(directory, lon0, lon1, lat0, lat1, step, nlayer, dz_km, seed=4):
    rng = np.random.default_rng(seed)
    os.makedirs(directory, exist_ok=True)
    nlon = int(round((lon1 - lon0) / step)) + 1
    nlat = int(round((lat1 - lat0) / step)) + 1
    for j in range(nlat):
        for i in range(nlon):
            lon = np.float32(np.float32(lon0) + np.float32(i) * np.float32(step))
            lat = np.float32(np.float32(lat0) + np.float32(j) * np.float32(step))
            base = rng.uniform(2.2, 3.0)
            grad = rng.uniform(0.03, 0.06)
            with open(os.path.join(directory, f"{float(lon):.1f}_{float(lat):.1f}.mod"), "w") as f:
                for k in range(nlayer):
                    dep = k * dz_km
                    vs = min(4.6, base + grad * dep + 0.05 * np.sin(0.7 * k + i - j))
                    f.write(f"{dep:.3f} {vs:.4f} {0.01:.3f}\n")


def _case(steps=6):
    c = pu.small_halfspace(steps=steps, NX=60, NY=50, NZ=40, DH=200.0, vp=8500.0)
    c.fault = []
    c.double_couple = dict(X=30, Y=25, Z=30, strike=30.0, dip=60.0, rake=90.0, Mw=4.0, duration=0.3)
    c.stations = [(20, 20, c.NZ - 1), (40, 30, c.NZ - 1)]
    c.layers = ()
    c.extra = dict(c.extra, useMedium=1, LayeredModel=0, ShenModel=1, MLonStart=99.8, MLonEnd=100.2,
                   MLatStart=29.8, MLatEnd=30.2, MLonStep=0.1, MLatStep=0.1, MVeticalStep=500.0,
                   MediumDir="./MediumDir")
    return c


@pytest.mark.gpu
@pytest.mark.parametrize("scheme", ["CGFDM", "SCFDM"])
def test_shen_medium_matches_reference(tmp_path, scheme):
    if not refrun.available(scheme):
        pytest.skip("reference CPU build not present")
    c = _case()
    d = cases.write_case(c, str(tmp_path / "run"), scheme=scheme)
    depth_km = c.DH * c.NZ * 1e-3
    nlayer = int((depth_km * 1e3 + 3e4) / 500.0)
    write_shen_nodes(os.path.join(d, "MediumDir"), 99.8, 100.2, 29.8, 30.2, 0.1, nlayer, 0.5)
    refrun.run(d, scheme)
    ref = refrun.read_outputs(d, scheme)["CJM"]
    with Session(d, flavor="exact") as s:
        mine = s.cjm()
    med = slice(10, 13)   # mu, lambda, buoyancy
    assert np.unique(ref[..., 10]).size > 20, "the medium must vary"
    np.testing.assert_array_equal(mine[..., med], ref[..., med])


def _cjm_medium(med):
    """mu, lambda, buoyancy from (Vs, Vp, rho) with the float32 operations of
    the reference's CJM fill (src/CJM.cpp:52-77)."""
    vs, vp, rho = (med[..., c].astype(np.float32) for c in range(3))
    mu = rho * (vs * vs)
    lam = rho * (vp * vp - (np.float32(2) * vs) * vs)
    return np.stack([mu, lam, np.float32(1) / rho], -1)


def test_shen_medium_host_matches_reference(tmp_path):
    """The same comparison on the CPU: the library builds the medium on the
    host (cgfdm_model_medium), the reference's CPU build packs it into CJM."""
    from cgfdm import model_medium

    if not refrun.available("CGFDM"):
        pytest.skip("reference CPU build not present")
    c = _case(steps=2)
    d = cases.write_case(c, str(tmp_path / "run"))
    nlayer = int((c.DH * c.NZ + 3e4) / 500.0)
    write_shen_nodes(os.path.join(d, "MediumDir"), 99.8, 100.2, 29.8, 30.2, 0.1, nlayer, 0.5)
    med = model_medium(d)
    refrun.run(d, "CGFDM")
    ref = refrun.read_outputs(d)["CJM"][..., 10:13]
    assert np.unique(med[..., 0]).size > 20
    np.testing.assert_array_equal(_cjm_medium(med), ref)


def write_crust1(directory, seed=6):
    """Synthetic CRUST1.0 files (crust1.vs/.vp/.rho/.bnds): 64800 one-degree
    cells from 179.5 W, 89.5 N, longitude fastest, 9 layers per cell (water,
    ice, three sediment, three crust layers, mantle), smooth in space."""
    rng = np.random.default_rng(seed)
    os.makedirs(directory, exist_ok=True)
    lon = -179.5 + np.arange(360)
    lat = 89.5 - np.arange(180)
    LO, LA = np.meshgrid(np.radians(lon), np.radians(lat))
    f = lambda a, b: np.sin(a * LO + rng.uniform(0, 6)) * np.cos(b * LA + rng.uniform(0, 6))
    topo = 0.4 + 0.3 * f(7, 5)
    thick = [np.zeros_like(topo), np.zeros_like(topo), 0.4 + 0.3 * f(11, 9) ** 2, 0.9 + 0.6 * f(5, 13) ** 2,
             1.5 + 0.8 * f(9, 3) ** 2, 11 + 3 * f(3, 4), 10 + 2 * f(4, 6), 12 + 2 * f(6, 2)]
    bnds = [topo]
    for t in thick:
        bnds.append(bnds[-1] - t)
    vs0 = [0.0, 1.9, 1.0, 1.7, 2.4, 3.5, 3.7, 3.9, 4.5]
    vp0 = [1.5, 3.8, 2.5, 3.4, 4.4, 6.0, 6.4, 6.9, 8.1]
    rho0 = [1.02, 0.92, 2.0, 2.3, 2.5, 2.7, 2.85, 3.0, 3.35]
    vs = [v + 0.1 * f(3 + n, 2 + n) * (v > 0) for n, v in enumerate(vs0)]
    vp = [v + 0.15 * f(2 + n, 3 + n) for n, v in enumerate(vp0)]
    rho = [v + 0.05 * f(4 + n, 5 + n) for n, v in enumerate(rho0)]
    for name, arr in (("vs", vs), ("vp", vp), ("rho", rho), ("bnds", bnds)):
        a = np.stack([x.reshape(-1) for x in arr], axis=1)   # [cell][layer]
        np.savetxt(os.path.join(directory, f"crust1.{name}"), a, fmt="%.4f")


def _crust_case(steps=2):
    c = _case(steps)
    c.extra = dict(c.extra, ShenModel=0, Crust_1Model=1, CrustLonStep=1.0, CrustLatStep=1.0, CrustDir="./crust")
    return c


def test_crust1_medium_host_matches_reference(tmp_path):
    """CRUST1.0 (Crust_1Model, src/crustMedium.cpp:67-370), on the CPU."""
    from cgfdm import model_medium

    if not refrun.available("CGFDM"):
        pytest.skip("reference CPU build not present")
    c = _crust_case()
    d = cases.write_case(c, str(tmp_path / "run"))
    write_crust1(os.path.join(d, "crust"))
    med = model_medium(d)
    refrun.run(d, "CGFDM")
    ref = refrun.read_outputs(d)["CJM"][..., 10:13]
    assert np.unique(med[..., 0]).size > 20
    np.testing.assert_array_equal(_cjm_medium(med), ref)


# ------------------------------------------------------------ SRTM terrain
def write_srtm_tile(directory, lat, lon, seed=8):
    """One synthetic SRTM90 tile "srtm_<lat>N<lon>E.bin": 6000 x 6000
    float32 heights (m), longitude fastest, rows from the tile's southern
    edge, 5/6000 degree apart; smooth hills plus scattered single-point
    spikes around the tile's centre, which the despiking replaces."""
    rng = np.random.default_rng(seed)
    os.makedirs(directory, exist_ok=True)
    n = 6000
    x = (np.arange(n, dtype=np.float32) * np.float32(5.0 / n))
    sx = np.sin(x * np.float32(2 * np.pi / 0.37)).astype(np.float32)
    cy = np.cos(x * np.float32(2 * np.pi / 0.29)).astype(np.float32)
    h = np.float32(1200) + np.float32(600) * cy[:, None] * sx[None, :]
    h += np.float32(150) * np.sin(x * np.float32(2 * np.pi / 0.05)).astype(np.float32)[None, :]
    ii = rng.integers(2850, 3150, 3000)
    jj = rng.integers(2850, 3150, 3000)
    h[jj, ii] += rng.choice([-400.0, 400.0], 3000).astype(np.float32)
    h.astype(np.float32).tofile(os.path.join(directory, f"srtm_{lat}N{lon}E.bin"))


def _terrain_case(kind):
    c = pu.small_halfspace(steps=2, NX=60, NY=50, NZ=40, DH=200.0, vp=8500.0)
    c.fault = []
    c.double_couple = dict(X=30, Y=25, Z=30, strike=30.0, dip=60.0, rake=90.0, Mw=4.0, duration=0.3)
    c.stations = [(20, 20, c.NZ - 1), (40, 30, c.NZ - 1)]
    c.layers = ()
    c.center_lon, c.center_lat = 102.5, 32.5
    c.extra = dict(c.extra, useTerrain=int(kind != "gauss_float"), SRTM90=int(kind == "srtm"),
                   TerrainDir="./terrain", lonStart=100, latStart=30, blockX=1, blockY=1)
    if kind in ("gauss", "gauss_float"):
        c.gauss_hill = 1
    return c


@pytest.mark.parametrize("kind", ["flat", "gauss", "srtm", "gauss_float"])
def test_terrain_host_matches_reference(tmp_path, kind):
    """useTerrain (src/coord.cpp:325-328, src/terrain.cpp:772-858) on the
    CPU: the SRTM90 surface (tiles read, despiked and smoothed around the
    model, interpolated to every column and smoothed again) and the
    terrain-following z of every point, against the reference's CPU build,
    bit for bit; "flat" and "gauss" apply only the z mapping, and
    "gauss_float" the Gauss hill without useTerrain (the terrain-following z
    in float, src/coord.cpp:204-255)."""
    from cgfdm import model_coord

    if not refrun.available("CGFDM"):
        pytest.skip("reference CPU build not present")
    c = _terrain_case(kind)
    d = cases.write_case(c, str(tmp_path / "run"))
    if kind == "srtm":
        write_srtm_tile(os.path.join(d, "terrain"), 30, 100)
    terrain, coord = model_coord(d)
    refrun.run(d, "CGFDM")
    out = os.path.join(d, "output")
    ref_coord = np.fromfile(os.path.join(out, "oracle_coord.bin"), np.float32).reshape(coord.shape)
    ref_terrain = np.fromfile(os.path.join(out, "oracle_terrain.bin"), np.float32).reshape(terrain.shape)
    np.testing.assert_array_equal(coord, ref_coord)
    np.testing.assert_array_equal(terrain, ref_terrain)
    if kind == "srtm":
        assert np.unique(terrain).size > 1000 and terrain.max() - terrain.min() > 100.0
        written = np.fromfile(os.path.join(out, "terrain_mpi_0_0_0.bin"), np.float32)
        np.testing.assert_array_equal(written.reshape(c.NY, c.NX), terrain[3:-3, 3:-3])


def test_srtm_outside_tiles_is_an_error(tmp_path):
    """A model whose corners leave the tiles fails as the reference aborts
    (error 1001, src/terrain.cpp:512-519)."""
    from cgfdm import CgfdmError, model_coord

    c = _terrain_case("srtm")
    c.center_lon = 100.02
    d = cases.write_case(c, str(tmp_path / "run"))
    write_srtm_tile(os.path.join(d, "terrain"), 30, 100)
    with pytest.raises(CgfdmError):
        model_coord(d)


@pytest.mark.gpu
def test_srtm_terrain_metrics_match_reference(tmp_path):
    """The SRTM90 surface through the whole setup on the GPU: the packed
    metric and medium (CJM) of the exact build against the reference's."""
    if not refrun.available("CGFDM"):
        pytest.skip("reference CPU build not present")
    c = _terrain_case("srtm")
    d = cases.write_case(c, str(tmp_path / "run"))
    write_srtm_tile(os.path.join(d, "terrain"), 30, 100)
    refrun.run(d, "CGFDM")
    ref = refrun.read_outputs(d)["CJM"]
    ref_out = os.path.join(d, "output")
    mine_out = os.path.join(d, "mine")
    with Session(d, options='{"OUT": "%s"}' % mine_out, flavor="exact") as s:
        mine = s.cjm()
        s.write_outputs()
    np.testing.assert_array_equal(mine, ref)
    for name in ("lon", "lat", "terrain"):   # the projection data files
        f = f"{name}_mpi_0_0_0.bin"
        a = np.fromfile(os.path.join(mine_out, f), np.float32)
        np.testing.assert_array_equal(a, np.fromfile(os.path.join(ref_out, f), np.float32), err_msg=f)
