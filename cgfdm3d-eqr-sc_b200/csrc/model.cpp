// Host-side setup: parameters, grid, coordinates, medium, PML profiles,
// finite-fault and point sources, stations.  Each function follows the
// reference routine cited beside it and keeps its float/double mix so the
// arrays are bit-identical to the reference's (this file is compiled with
// -ffp-contract=off).
#include "model.hpp"

#include <algorithm>
#include <fcntl.h>
#include <unistd.h>
#include <chrono>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <thread>
#ifdef __linux__
#include <sched.h>
#endif

#include "aeqd.h"

namespace cgfdm {

// f(k) for k = 0 .. n-1 on the host's cores: the model's per-plane loops
// (every point's value depends on its own inputs only, so the result does
// not depend on the split).
template <class F>
static void par_for(int n, F f)
{
    unsigned T = std::max(1u, std::min(std::thread::hardware_concurrency(), 32u));
#ifdef __linux__
    {
        cpu_set_t set;   // the cores this process may run on, not all the machine's
        if (sched_getaffinity(0, sizeof set, &set) == 0) T = std::max(1u, std::min(T, (unsigned)CPU_COUNT(&set)));
    }
#endif
    if (n < 2 || T == 1) {
        for (int k = 0; k < n; k++) f(k);
        return;
    }
    std::atomic<int> next(0);
    std::vector<std::thread> th;
    for (unsigned t = 0; t < std::min<unsigned>(T, (unsigned)n); t++)
        th.emplace_back([&] {
            for (int k; (k = next++) < n;) f(k);
        });
    for (auto &x : th) x.join();
}


// Constants as the reference defines them (src/macro.h:70-73): PI is a float
// literal, DEGREE2RADIAN is PI converted to double over 180.0.
static const float REF_PI = 3.141592657f;
static const double REF_DEG2RAD = (double)REF_PI / 180.0;

static std::string join(const std::string &dir, const std::string &f)
{
    if (f.empty()) return f;
    if (f[0] == '/') return f;
    std::string d = dir;
    if (!d.empty() && d.back() != '/') d += '/';
    return d + f;
}

// ----------------------------------------------------------------- params
int read_params(const std::string &path, Params &p, std::string &err)
{
    JsonValue root;
    {
        std::ifstream f(path);
        if (!f) {
            err = "there is no params file " + path;
            return ST_NO_PARAMS;
        }
    }
    if (!json_parse_file(path, root, err) || root.kind != JsonValue::Object) {
        err = "cannot parse json file " + path + ": " + err;
        return ST_JSON;
    }
    const JsonValue *it;
#define GETD(key, field) if ((it = root.get(key))) p.field = it->num
#define GETF(key, field) if ((it = root.get(key))) p.field = (float)it->num
#define GETI(key, field) if ((it = root.get(key))) p.field = it->as_int()
#define GETS(key, field) if ((it = root.get(key)) && it->kind == JsonValue::String) p.field = it->str
    GETD("TMAX", TMAX);
    GETD("DT", DT);
    GETD("DH", DH);
    GETI("NX", NX);
    GETI("NY", NY);
    GETI("NZ", NZ);
    GETI("PX", PX);
    GETI("PY", PY);
    GETI("PZ", PZ);
    GETI("centerX", centerX);
    GETI("centerY", centerY);
    GETD("centerLongitude", centerLongitude);
    GETD("centerLatitude", centerLatitude);
    GETI("IT_SKIP", IT_SKIP);
    GETI("sliceX", sliceX);
    GETI("sliceY", sliceY);
    GETI("sliceZ", sliceZ);
    GETI("sliceFreeSurf", sliceFreeSurf);
    GETI("nPML", nPML);
    GETI("gauss_hill", gauss_hill);
    GETI("useTerrain", useTerrain);
    GETI("useMedium", useMedium);
    GETI("useMultiSource", useMultiSource);
    GETI("LayeredModel", LayeredModel);
    GETS("LayeredFileName", LayeredFileName);
    GETI("useSingleSource(ricker)", useSingleSource_ricker);
    GETI("useSingleSource(double_couple)", useSingleSource_double_couple);
    GETF("strike", strike);
    GETF("dip", dip);
    GETF("rake", rake);
    GETF("Mw", Mw);
    GETF("duration", duration);
    GETF("rickerfc", rickerfc);
    GETI("ShenModel", ShenModel);
    GETI("Crust_1Model", Crust_1Model);
    GETF("MLonStart", MLonStart);
    GETF("MLatStart", MLatStart);
    GETF("MLonEnd", MLonEnd);
    GETF("MLatEnd", MLatEnd);
    GETF("MLonStep", MLonStep);
    GETF("MLatStep", MLatStep);
    GETF("CrustLonStep", CrustLonStep);
    GETF("CrustLatStep", CrustLatStep);
    GETF("MVeticalStep", MVeticalStep);
    GETS("MediumDir", MediumDir);
    GETI("SRTM90", SRTM90);
    GETS("TerrainDir", TerrainDir);
    GETI("lonStart", lonStart);
    GETI("latStart", latStart);
    GETI("blockX", blockX);
    GETI("blockY", blockY);
    GETS("CrustDir", CrustDir);
    GETS("OUT", OUT);
    GETF("Depth(km)", Depth);
    GETI("sourceX", sourceX);
    GETI("sourceY", sourceY);
    GETI("sourceZ", sourceZ);
    GETS("sourceFile", sourceFile);
    GETS("sourceDir", sourceDir);
    GETI("degree2radian", degree2radian);
    // run-time switches (names of the reference's compile-time flags)
    if ((it = root.get("scheme")) && it->kind == JsonValue::String) {
        std::string s = it->str;
        for (auto &c : s) c = (char)std::toupper((unsigned char)c);
        if (s == "SCFDM" || s == "AWENO" || s == "ME-AWENO") p.scheme = SCHEME_SCFDM;
        else if (s == "CGFDM") p.scheme = SCHEME_CGFDM;
        else {
            err = "unknown scheme " + it->str;
            return ST_OPTIONS;
        }
    }
    // defaults of the two reference builds (Makefile_CGFDM / Makefile_SCFDM:
    // PML or EXP_DECAY by scheme, SOLVE_DISPLACEMENT on in both)
    p.pml = p.scheme == SCHEME_CGFDM ? 1 : 0;
    p.exp_decay = p.scheme == SCHEME_SCFDM ? 1 : 0;
    p.solve_displacement = 1;
    GETI("PML", pml);
    GETI("EXP_DECAY", exp_decay);
    GETI("SOLVE_DISPLACEMENT", solve_displacement);
    GETI("SOLVE_PGA", solve_pga);
    if ((it = root.get("metricPrecision")) && it->kind == JsonValue::String) p.metric_fp64 = it->str == "fp64";
    GETS("storage", storage);
    GETS("terrainFile", terrainFile);
    GETS("mediumFile", mediumFile);
#undef GETD
#undef GETF
#undef GETI
#undef GETS
    if (!p.useTerrain) p.Depth = (float)(p.DH * p.NZ * 1e-3);  // src/getParams.cpp:234-237
    return ST_OK;
}

// ------------------------------------------------------------------- grid
Grid make_grid(const Params &p)
{
    Grid g;
    g.NX = p.NX, g.NY = p.NY, g.NZ = p.NZ;
    g.nx = p.NX, g.ny = p.NY, g.nz = p.NZ;
    g._nx_ = g.nx + 2 * HALO, g._ny_ = g.ny + 2 * HALO, g._nz_ = g.nz + 2 * HALO;
    g._nx = g.nx + HALO, g._ny = g.ny + HALO, g._nz = g.nz + HALO;
    g.originalX = p.centerX, g.originalY = p.centerY;
    g.nPML = p.nPML;
    g.DH = (float)p.DH;
    g.rDH = (float)(1.0 / g.DH);  // src/init_grid.cpp:89
    return g;
}

// ------------------------------------------------------------ coordinates
// Flat grid (src/coord.cpp:99-134), single Gauss hill (:136-177) and the
// terrain-following z of src/coord.cpp:204-255.  Each coordinate is
// computed by coord_at from the grid, the terrain and the mode, in the same
// operations and types as the filled volume, so both ways give the same
// floats.
float Model::coord_at(int i, int j, int k, int c) const
{
    if (!coord_lazy) return coord[(size_t)g.idx(i, j, k) * 3 + c];
    const float DH = g.DH;
    const int NZ = g.NZ;
    if (c == 0) return (i - HALO) * DH - g.originalX * DH;
    if (c == 1) return (j - HALO) * DH - g.originalY * DH;
    if (coord_mode == 0) return (k - HALO + 1) * DH - NZ * DH;
    const int K = k - HALO;
    if (coord_mode == 1) {
        const float cal_depth = coord_depth_f;
        const float height = terrain[(size_t)i + (size_t)j * g._nx_];
        const float DZ = (float)(double(height + std::fabs(cal_depth)) / double(NZ - 1));
        return -std::fabs(cal_depth) + DZ * K;
    }
    const double Depth = coord_depth_d;
    const double DZ = double(terrain[(size_t)i + (size_t)j * g._nx_] + std::fabs(Depth)) / double(NZ - 1);
    return (float)(-std::fabs(Depth) + DZ * K);
}

void materialize_coords(Model &m)
{
    if (!m.coord_lazy) return;
    const Grid &g = m.g;
    m.coord.resize((size_t)g.npad() * 3);   // every value written below
    par_for(g._nz_, [&](int k) {
        for (int j = 0; j < g._ny_; j++)
            for (int i = 0; i < g._nx_; i++)
                for (int c = 0; c < 3; c++) m.coord[(size_t)g.idx(i, j, k) * 3 + c] = m.coord_at(i, j, k, c);
    });
    m.coord_lazy = false;
}

// lazy: leave the volume to coord_at (the flat mode's terrain is still made)
static void build_coords(Model &m, bool lazy)
{
    const Grid &g = m.g;
    const float DH = g.DH;
    const int NZ = g.NZ;
    m.coord_mode = 0;
    m.terrain.assign((size_t)g._nx_ * g._ny_, 0.f);
    if (lazy) {
        const int K = NZ + HALO - 1;
        for (int j = 0; j < g._ny_; j++)
            for (int i = 0; i < g._nx_; i++) m.terrain[(size_t)i + (size_t)j * g._nx_] = (K - HALO + 1) * DH - NZ * DH;
        m.coord.clear();
        m.coord_lazy = true;
        return;
    }
    m.coord.resize((size_t)g.npad() * 3);   // every value written below
    m.coord_lazy = false;
    par_for(g._nz_, [&](int k) {
        for (int j = 0; j < g._ny_; j++)
            for (int i = 0; i < g._nx_; i++) {
                long long id = g.idx(i, j, k) * 3;
                int I = i, J = j, K = k;
                if (K == NZ + HALO - 1) m.terrain[(size_t)i + (size_t)j * g._nx_] = (K - HALO + 1) * DH - NZ * DH;
                m.coord[id + 0] = (I - HALO) * DH - g.originalX * DH;
                m.coord[id + 1] = (J - HALO) * DH - g.originalY * DH;
                m.coord[id + 2] = (K - HALO + 1) * DH - NZ * DH;
            }
    });
}

static void terrain_following_z(Model &m, float cal_depth)
{
    const Grid &g = m.g;
    m.coord_mode = 1;
    m.coord_depth_f = cal_depth;
    if (m.coord_lazy) return;
    par_for(g._nz_, [&](int k) {
        for (int j = 0; j < g._ny_; j++)
            for (int i = 0; i < g._nx_; i++) {
                long long id = g.idx(i, j, k);
                int K = k - HALO;
                float height = m.terrain[(size_t)i + (size_t)j * g._nx_];
                float DZ = (float)(double(height + std::fabs(cal_depth)) / double(g.NZ - 1));
                m.coord[id * 3 + 2] = -std::fabs(cal_depth) + DZ * K;
            }
    });
}

static void gauss_hill(Model &m)
{
    const Grid &g = m.g;
    const float DH = g.DH;
    float cal_depth = m.p.Depth * 1000;
    float h = (float)(0.2 * cal_depth);
    float a = (float)(0.1 * cal_depth), b = (float)(0.1 * cal_depth);
    for (int j = 0; j < g._ny_; j++)
        for (int i = 0; i < g._nx_; i++) {
            float x = (i - HALO) * DH - g.originalX * DH;
            float y = (j - HALO) * DH - g.originalY * DH;
            float height = h * expf(-0.5f * (x * x / (a * a) + y * y / (b * b)));
            m.terrain[(size_t)i + (size_t)j * g._nx_] = height;
        }
    terrain_following_z(m, cal_depth);
}

// Extension: a raw float32 [_ny_][_nx_] surface height map in metres, mapped
// by the reference's terrain-following formula (src/coord.cpp:228-234).
static int terrain_file(Model &m, const std::string &path, std::string &err)
{
    const Grid &g = m.g;
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        err = "cannot open terrain file " + path;
        return ST_IO;
    }
    f.read((char *)m.terrain.data(), (std::streamsize)(m.terrain.size() * sizeof(float)));
    if (!f) {
        err = "terrain file too short: " + path;
        return ST_IO;
    }
    terrain_following_z(m, m.p.Depth * 1000);
    (void)g;
    return ST_OK;
}

// ---------------------------------------------------------- SRTM terrain
// Two-point Lagrange (bilinear) interpolation in double, the evaluation
// order of src/terrain.cpp:563-600: z = {A, C, B, D} for the corners
// (x1, y1), (x1, y2), (x2, y1), (x2, y2).
static double interp2d(const double x[2], const double y[2], const double z[4], double x_, double y_)
{
    double Lx[2], Ly[2];
    Lx[0] = 1.0 * (x_ - x[1]) / (x[0] - x[1]);
    Lx[1] = 1.0 * (x_ - x[0]) / (x[1] - x[0]);
    Ly[0] = 1.0 * (y_ - y[1]) / (y[0] - y[1]);
    Ly[1] = 1.0 * (y_ - y[0]) / (y[1] - y[0]);
    double Li = 0.0;
    for (int jj = 0; jj < 2; jj++)
        for (int ii = 0; ii < 2; ii++) Li = Li + Lx[ii] * Ly[jj] * z[ii * 2 + jj];
    return Li;
}

// The projection centre as the reference hands it to PROJ: a float printed
// with "%lf" (src/terrain.cpp:325-331, 490-505), in radians.
static void proj_centre(const Params &p, double *lon0, double *lat0)
{
    char buf[64];
    std::snprintf(buf, sizeof buf, "%lf", (double)(float)p.centerLongitude);
    *lon0 = std::atof(buf) * (3.14159265358979323846 / 180.0);
    std::snprintf(buf, sizeof buf, "%lf", (double)(float)p.centerLatitude);
    *lat0 = std::atof(buf) * (3.14159265358979323846 / 180.0);
}

// 11-point Gaussian of the terrain smoothing (Terrain_Smooth, on in the
// reference's builds): GAUSS_FUN(n - 5, 2.5, 0) of src/macro.h:37.
static void smooth_weights(double Dg[11])
{
    const double ra = 5 * 0.5;
    for (int n = 0; n < 11; n++) {
        const double t = ((n - 5) - 0.0) / ra;
        Dg[n] = std::exp(-(t * t)) / (ra * 1.772453850905516);
    }
}

static int column_lonlat(const Model &m, float lonMin, float lonMax, float latMin, float latMax,
                         std::vector<double> &lon, std::vector<double> &lat, std::string &err);

// SRTM90 surface (src/terrain.cpp:206-290, 307-447, 602-770): 5 x 5 degree
// tiles "<TerrainDir>/srtm_<lat>N<lon>E.bin" of 6000 x 6000 float heights
// (blockX x blockY of them from lonStart, latStart), joined with one shared
// row and column; around the model, points whose central-difference
// gradient exceeds 100 m take the mean of their four neighbours, then an
// 11 x 11 Gaussian smooths the map; each column's height is interpolated
// at its longitude and latitude (on a grid widened by 5 points) and smoothed
// again with the same Gaussian.  The reference's third corner value is
// taken at (I + 1, J + 1) as well as the fourth; kept.
static int srtm_terrain(Model &m, const std::string &run_dir, std::string &err)
{
    const Params &p = m.p;
    const Grid &g = m.g;
    const int PPB = 6000, DPB = 5;
    if (p.blockX < 1 || p.blockY < 1) {
        err = "SRTM90 needs blockX, blockY >= 1";
        return ST_OPTIONS;
    }
    const int TX = (PPB - 1) * p.blockX + 1, TY = (PPB - 1) * p.blockY + 1;
    std::vector<float> total((size_t)TX * TY, 0.0f), tile((size_t)PPB * PPB);
    const std::string dir = join(run_dir, p.TerrainDir);
    for (int jb = 0; jb < p.blockY; jb++)
        for (int ib = 0; ib < p.blockX; ib++) {
            const int lat = p.latStart + jb * DPB, lon = p.lonStart + ib * DPB;
            char name[96];
            std::snprintf(name, sizeof name, "srtm_%dN%dE.bin", lat, lon);
            const std::string path = dir + "/" + name;
            FILE *f = std::fopen(path.c_str(), "rb");
            if (!f) {
                err = "There is no such file " + path;
                return ST_IO;
            }
            const size_t got = std::fread(tile.data(), sizeof(float), tile.size(), f);
            std::fclose(f);
            if (got != tile.size()) {
                err = "SRTM tile too short: " + path;
                return ST_IO;
            }
            for (int jj = 0; jj < PPB - 1; jj++)
                for (int ii = 0; ii < PPB - 1; ii++)
                    total[(size_t)(ib * (PPB - 1) + ii) + (size_t)(jb * (PPB - 1) + jj) * TX] =
                        tile[(size_t)ii + (size_t)jj * PPB];
        }

    double lon0, lat0;
    proj_centre(p, &lon0, &lat0);
    const double r2d = 180.0 / (double)REF_PI;
    const float DH = g.DH;
    const double lonStart = p.lonStart, latStart = p.latStart;
    const double dLon = double(DPB * p.blockX) / double(TX), dLat = double(DPB * p.blockY) / double(TY);
    double Dg[11];
    smooth_weights(Dg);

    // despiking and smoothing of the tiles around the model (callibrateTotalTerrain)
    {
        const double xs[2] = {(double)((0 - HALO) * DH - g.originalX * DH), (double)((g._nx_ - HALO) * DH - g.originalX * DH)};
        const double ys[2] = {(double)((0 - HALO) * DH - g.originalY * DH), (double)((g._ny_ - HALO) * DH - g.originalY * DH)};
        float maxLon = -1000.0f, maxLat = -1000.0f, minLon = 1000.0f, minLat = 1000.0f;
        const double cx[4] = {xs[0], xs[0], xs[1], xs[1]}, cy[4] = {ys[0], ys[1], ys[0], ys[1]};
        for (int c = 0; c < 4; c++) {
            double la, ph;
            cgfdm_aeqd_inv(lon0, lat0, cx[c], cy[c], &la, &ph);
            const double Lon = la * r2d, Lat = ph * r2d;
            if (maxLon <= Lon) maxLon = (float)Lon;
            if (maxLat <= Lat) maxLat = (float)Lat;
            if (minLon >= Lon) minLon = (float)Lon;
            if (minLat >= Lat) minLat = (float)Lat;
        }
        const int I0 = int((minLon - lonStart) / dLon) - 10, J0 = int((minLat - latStart) / dLat) - 10;
        const int I1 = int((maxLon - lonStart) / dLon) + 10, J1 = int((maxLat - latStart) / dLat) + 10;
        if (I0 - 5 < 0 || J0 - 5 < 0 || I1 + 5 > TX || J1 + 5 > TY) {
            err = "the model lies too close to the edge of the SRTM tiles";
            return 1001;
        }
        std::vector<float> next(total);
        for (int j = J0; j < J1; j++)
            for (int i = I0; i < I1; i++) {
                const float a = total[(size_t)(i + 1) + (size_t)j * TX], b = total[(size_t)(i - 1) + (size_t)j * TX];
                const float c = total[(size_t)i + (size_t)(j + 1) * TX], d = total[(size_t)i + (size_t)(j - 1) * TX];
                const float gx = a - b, gy = c - d;
                const float grad = std::sqrt(gx * gx + gy * gy);
                if (grad > 100.0) next[(size_t)i + (size_t)j * TX] = (float)((a + b + c + d) * 0.25);
            }
        total = next;
        for (int j = J0; j < J1; j++)
            for (int i = I0; i < I1; i++) {
                double sum = 0.0;
                for (int jj = j - 5; jj < j + 6; jj++)
                    for (int ii = i - 5; ii < i + 6; ii++) {
                        const double amp = Dg[ii + 5 - i] * Dg[jj + 5 - j] / 0.996768;
                        sum += amp * total[(size_t)ii + (size_t)jj * TX];
                    }
                next[(size_t)i + (size_t)j * TX] = (float)sum;
            }
        total.swap(next);
    }

    // the model with its 2-point margin inside the tiles, and the columns'
    // longitude and latitude for the projection output (projTrans)
    {
        const float lonMax = (float)(p.lonStart + p.blockX * DPB), latMax = (float)(p.latStart + p.blockY * DPB);
        if (int st = column_lonlat(m, (float)p.lonStart, lonMax, (float)p.latStart, latMax, m.lon, m.lat, err))
            return st;
    }

    // the columns' heights (terrainInterp), on a grid widened by 5 points
    const int ng = 5, enx = g._nx_ + 2 * ng, eny = g._ny_ + 2 * ng;
    std::vector<float> ex((size_t)enx * eny);
    for (int j = -ng; j < g._ny_ + ng; j++)
        for (int i = -ng; i < g._nx_ + ng; i++) {
            const double px = (double)((i - HALO) * DH - g.originalX * DH);
            const double py = (double)((j - HALO) * DH - g.originalY * DH);
            double la, ph;
            cgfdm_aeqd_inv(lon0, lat0, px, py, &la, &ph);
            const double x_ = la * r2d, y_ = ph * r2d;
            const int I = int((x_ - lonStart) / dLon), J = int((y_ - latStart) / dLat);
            if (I < 0 || J < 0 || I + 1 >= TX || J + 1 >= TY) {
                err = "the model extends beyond the SRTM tiles";
                return 1001;
            }
            const double x1 = I * dLon + lonStart, y1 = J * dLat + latStart;
            const double x[2] = {x1, x1 + dLon}, y[2] = {y1, y1 + dLat};
            auto T = [&](int a, int b) { return (double)total[(size_t)a + (size_t)b * TX]; };
            const double z[4] = {T(I, J), T(I + 1, J + 1), T(I + 1, J), T(I + 1, J + 1)};
            ex[(size_t)(i + ng) + (size_t)(j + ng) * enx] = (float)interp2d(x, y, z, x_, y_);
        }
    for (int j = ng; j < g._ny_ + ng; j++)
        for (int i = ng; i < g._nx_ + ng; i++) {
            double sum = 0.0;
            for (int jj = j - ng; jj < j + ng + 1; jj++)
                for (int ii = i - ng; ii < i + ng + 1; ii++) {
                    const double amp = Dg[ii + ng - i] * Dg[jj + ng - j] / 0.996768;
                    sum += amp * ex[(size_t)ii + (size_t)jj * enx];
                }
            m.terrain[(size_t)(i - ng) + (size_t)(j - ng) * g._nx_] = (float)sum;
        }
    return ST_OK;
}

// z of every point below a surface of the reference's useTerrain path
// (src/terrain.cpp:834-858), in double: -|Depth| + K (h + |Depth|) / (NZ - 1).
static void terrain_z_double(Model &m)
{
    const Grid &g = m.g;
    const double Depth = m.p.Depth * 1e3;
    m.coord_mode = 2;
    m.coord_depth_d = Depth;
    if (m.coord_lazy) return;
    par_for(g._nz_, [&](int k) {
        for (int j = 0; j < g._ny_; j++)
            for (int i = 0; i < g._nx_; i++) {
                const int K = k - HALO;
                const double DZ = double(m.terrain[(size_t)i + (size_t)j * g._nx_] + std::fabs(Depth)) / double(g.NZ - 1);
                m.coord[g.idx(i, j, k) * 3 + 2] = (float)(-std::fabs(Depth) + DZ * K);
            }
    });
}

// ----------------------------------------------------------------- medium
// Longitude and latitude (degrees) of every column of the padded grid: the
// inverse azimuthal-equidistant projection about the centre of the x, y of
// its top interior point (src/terrain.cpp:450-536, cart2LonLat), after the
// check that the model corners with a 2-point margin lie inside the data's
// range (calculateCutLonLat, :120-157; MPI_Abort 1001 there).
static int column_lonlat(const Model &m, float lonMin, float lonMax, float latMin, float latMax,
                         std::vector<double> &lon, std::vector<double> &lat, std::string &err)
{
    const Grid &g = m.g;
    double lon0, lat0;
    proj_centre(m.p, &lon0, &lat0);
    const double r2d = 180.0 / (double)REF_PI;
    const int NX_ = m.p.NX + 2 * HALO, NY_ = m.p.NY + 2 * HALO;
    const int ox = g.originalX + HALO, oy = g.originalY + HALO;
    const double corner[4][2] = {{(double)(-(ox + 2) * g.DH), (double)(-(oy + 2) * g.DH)},
                                 {(double)(-(ox + 2) * g.DH), (double)(((NY_ - oy) + 2) * g.DH)},
                                 {(double)(((NX_ - ox) + 2) * g.DH), (double)(-(oy + 2) * g.DH)},
                                 {(double)(((NX_ - ox) + 2) * g.DH), (double)(((NY_ - oy) + 2) * g.DH)}};
    for (int c = 0; c < 4; c++) {
        double la, ph;
        cgfdm_aeqd_inv(lon0, lat0, corner[c][0], corner[c][1], &la, &ph);
        const float lo = (float)(la * r2d), at = (float)(ph * r2d);
        if (lo > lonMax || lo < lonMin || at > latMax || at < latMin) {
            err = "the longitude or latitude range of the model extends beyond the medium data's range";
            return 1001;
        }
    }
    lon.assign((size_t)g._nx_ * g._ny_, 0.0);
    lat.assign((size_t)g._nx_ * g._ny_, 0.0);
    const int k = g._nz - 1;
    for (int j = 0; j < g._ny_; j++)
        for (int i = 0; i < g._nx_; i++) {
            double la, ph;
            cgfdm_aeqd_inv(lon0, lat0, (double)m.coord_at(i, j, k, 0), (double)m.coord_at(i, j, k, 1), &la, &ph);
            lon[(size_t)i + (size_t)j * g._nx_] = la * r2d;
            lat[(size_t)i + (size_t)j * g._nx_] = ph * r2d;
        }
    return ST_OK;
}

// Weisen Shen's Vs model (src/dealMedium.cpp:49-360): one text file per
// node "<MediumDir>/<lon %.1f>_<lat %.1f>.mod" on MLonStart..MLonEnd x
// MLatStart..MLatEnd by MLonStep x MLatStep, NLayer = int((Depth + 30 km) /
// MVeticalStep) lines "depth vs error" (km/s).  Per layer, Vs is
// interpolated to each column's longitude and latitude; the first layer
// takes the second's values (DealWithFirstLayer, on in the reference's
// builds); a point takes layer K = int(-(z - top)) / MVeticalStep below the
// model top DZ (NZ - 1) - Depth (StructureTerrain), Vp and rho from Vs by
// the relations of src/dealMedium.cpp:186-189.
static int shen_medium(Model &m, const std::string &run_dir, std::string &err)
{
    const Params &p = m.p;
    const Grid &g = m.g;
    const float LonStart = p.MLonStart, LatStart = p.MLatStart, LonStep = p.MLonStep, LatStep = p.MLatStep;
    if (!(LonStep > 0.0f) || !(LatStep > 0.0f) || !(p.MVeticalStep > 0.0f)) {
        err = "ShenModel needs positive MLonStep, MLatStep and MVeticalStep";
        return ST_OPTIONS;
    }
    const int nLon = int((p.MLonEnd - LonStart) / LonStep + 0.5 + 1);
    const int nLat = int((p.MLatEnd - LatStart) / LatStep + 0.5 + 1);
    const float Depth = (float)(p.Depth * 1e3 + 3e4);
    const int NLayer = int(Depth / p.MVeticalStep);
    if (nLon < 2 || nLat < 2 || NLayer < 2) {
        err = "ShenModel grid too small";
        return ST_OPTIONS;
    }
    std::vector<float> VModel((size_t)nLon * nLat * NLayer);
    const std::string dir = join(run_dir, p.MediumDir);
    for (int j = 0; j < nLat; j++)
        for (int i = 0; i < nLon; i++) {
            char name[64];
            std::snprintf(name, sizeof name, "%.1f_%.1f.mod", (double)(LonStart + i * LonStep),
                          (double)(LatStart + j * LatStep));
            const std::string path = dir + "/" + name;
            FILE *f = std::fopen(path.c_str(), "r");
            if (!f) {
                err = "cannot open Shen model file " + path;
                return ST_IO;
            }
            for (int K = 0; K < NLayer; K++) {
                double dep, vs, e;
                if (std::fscanf(f, "%lf %lf %lf", &dep, &vs, &e) != 3) {
                    std::fclose(f);
                    err = "Shen model file too short: " + path;
                    return ST_IO;
                }
                VModel[(size_t)K + ((size_t)i + (size_t)j * nLon) * NLayer] = (float)(vs * 1e3);
            }
            std::fclose(f);
        }
    std::vector<double> lon, lat;
    if (int st = column_lonlat(m, LonStart, p.MLonEnd, LatStart, p.MLatEnd, lon, lat, err)) return st;

    const size_t plane = (size_t)g._nx_ * g._ny_;
    std::vector<float> Vs(plane * NLayer);
    for (int K = 0; K < NLayer; K++)
        for (int j = 0; j < g._ny_; j++)
            for (int i = 0; i < g._nx_; i++) {
                const size_t c = (size_t)i + (size_t)j * g._nx_;
                const double x_ = lon[c], y_ = lat[c];
                const int I = int((x_ - (double)LonStart) / LonStep);
                const int J = int((y_ - (double)LatStart) / LatStep);
                if (I < 0 || J < 0 || I + 1 >= nLon || J + 1 >= nLat) {
                    err = "a grid column falls outside the Shen model's nodes";
                    return 1001;
                }
                const double x1 = (float)(I * LonStep) + (double)LonStart;
                const double y1 = (float)(J * LatStep) + (double)LatStart;
                const double x[2] = {x1, x1 + LonStep}, y[2] = {y1, y1 + LatStep};
                auto at = [&](int a, int b) { return (double)VModel[(size_t)K + ((size_t)a + (size_t)b * nLon) * NLayer]; };
                const double z[4] = {at(I, J), at(I, J + 1), at(I + 1, J), at(I + 1, J + 1)};
                Vs[(size_t)K * plane + c] = (float)interp2d(x, y, z, x_, y_);
            }
    for (size_t c = 0; c < plane; c++) Vs[c] = Vs[plane + c];   // DealWithFirstLayer

    const int NZ = p.NZ;
    const double DepthM = p.Depth * 1e3;
    for (int k = 0; k < g._nz_; k++)
        for (int j = 0; j < g._ny_; j++)
            for (int i = 0; i < g._nx_; i++) {
                const long long id = g.idx(i, j, k);
                const double DZ = (double)(m.coord_at(i, j, 4, 2) - m.coord_at(i, j, 3, 2));
                const double top = DZ * double(NZ - 1) - std::fabs(DepthM);
                int K = (int)((float)int(-((double)m.coord_at(i, j, k, 2) - top)) / p.MVeticalStep);
                if (K <= 0) K = 0;
                if (K >= NLayer) {
                    err = "a grid point lies below the Shen model's deepest layer";
                    return ST_OPTIONS;
                }
                const float VS = (float)(Vs[(size_t)K * plane + (size_t)i + (size_t)j * g._nx_] * 1e-3);
                const float VP = (float)(0.9409 + 2.0947 * VS - 0.8206 * std::pow((double)VS, 2.0) +
                                         0.2683 * std::pow((double)VS, 3.0) - 0.0251 * std::pow((double)VS, 4.0));
                const float RHO = (float)(1.6612 * VP - 0.4721 * std::pow((double)VP, 2.0) +
                                          0.0671 * std::pow((double)VP, 3.0) - 0.0043 * std::pow((double)VP, 4.0) +
                                          0.000106 * std::pow((double)VP, 5.0));
                float *md = &m.medium[id * 3];
                md[0] = (float)(VS * 1e3);
                md[1] = (float)(VP * 1e3);
                md[2] = (float)(RHO * 1e3);
            }
    return ST_OK;
}

// CRUST1.0 (src/crustMedium.cpp:67-370): the text files crust1.vs, .vp,
// .rho, .bnds of CrustDir, 64800 one-degree cells (from 179.5 W, 89.5 N,
// longitude fastest) x 9 layers each (km/s, g/cm^3, km), read cell by cell;
// every layer's values are interpolated to each column's longitude and
// latitude on the CrustLonStep x CrustLatStep grid; a point takes the layer
// whose boundaries (m) bracket its height, skipping layers less than 1 km
// thick below the boundary it falls under (BoundaryDifference).
static int crust_medium(Model &m, const std::string &run_dir, std::string &err)
{
    const Params &p = m.p;
    const Grid &g = m.g;
    const int nLon = 360, nLat = 180, nLayer = 9, nLL = nLon * nLat;
    const std::string dir = join(run_dir, p.CrustDir);
    const char *names[4] = {"crust1.vs", "crust1.vp", "crust1.rho", "crust1.bnds"};
    std::vector<float> file[4];
    FILE *fp[4] = {};
    for (int f = 0; f < 4; f++) {
        const std::string path = dir + "/" + names[f];
        fp[f] = std::fopen(path.c_str(), "r");
        if (!fp[f]) {
            for (int q = 0; q < f; q++) std::fclose(fp[q]);
            err = "cannot open CRUST1.0 file " + path;
            return ST_IO;
        }
        file[f].assign((size_t)nLL * nLayer, 0.0f);
    }
    bool ok = true;
    for (int i = 0; i < nLL && ok; i++)
        for (int n = 0; n < nLayer && ok; n++)
            for (int f = 0; f < 4 && ok; f++) ok = std::fscanf(fp[f], "%f", &file[f][(size_t)i + (size_t)n * nLL]) == 1;
    for (int f = 0; f < 4; f++) std::fclose(fp[f]);
    if (!ok) {
        err = "CRUST1.0 files too short in " + dir;
        return ST_IO;
    }
    if (!(p.CrustLonStep > 0.0f) || !(p.CrustLatStep > 0.0f)) {
        err = "Crust_1Model needs positive CrustLonStep and CrustLatStep";
        return ST_OPTIONS;
    }
    std::vector<double> lon, lat;
    if (int st = column_lonlat(m, -180.0f, 180.0f, -90.0f, 90.0f, lon, lat, err)) return st;

    const size_t plane = (size_t)g._nx_ * g._ny_;
    std::vector<float> interp[4];
    for (int f = 0; f < 4; f++) interp[f].assign(plane * nLayer, 0.0f);
    const float LonStart = -179.5f, LatStart = 89.5f, LonStep = p.CrustLonStep, LatStep = p.CrustLatStep;
    for (int K = 0; K < nLayer; K++)
        for (int j = 0; j < g._ny_; j++)
            for (int i = 0; i < g._nx_; i++) {
                const size_t c = (size_t)i + (size_t)j * g._nx_;
                const double x_ = lon[c], y_ = lat[c];
                const int I = int((x_ - LonStart) / LonStep);
                const int J = int((LatStart - y_) / LatStep) + 1;
                if (I < 0 || I + 1 >= nLon || J < 1 || J >= nLat) {
                    err = "a grid column falls outside the CRUST1.0 cells";
                    return 1001;
                }
                const double x1 = I * LonStep + LonStart, y1 = LatStart - J * LatStep;
                const double x[2] = {x1, x1 + LonStep}, y[2] = {y1, y1 + LatStep};
                auto at = [&](int f, int a, int b) {
                    return (double)file[f][(size_t)a + (size_t)b * nLon + (size_t)K * nLL];
                };
                for (int f = 0; f < 4; f++) {
                    const double z[4] = {at(f, I, J), at(f, I, J - 1), at(f, I + 1, J), at(f, I + 1, J - 1)};
                    interp[f][(size_t)K * plane + c] = (float)interp2d(x, y, z, x_, y_);
                }
            }
    std::vector<float> &bnds = interp[3];
    for (size_t e = 0; e < bnds.size(); e++) bnds[e] = (float)(bnds[e] * 1e3);

    const float BoundaryDifference = 1000.0f;
    float vs = 0.0f, vp = 0.0f, rho = 0.0f;
    for (int k = 0; k < g._nz_; k++)
        for (int j = 0; j < g._ny_; j++)
            for (int i = 0; i < g._nx_; i++) {
                const long long id = g.idx(i, j, k);
                const size_t c = (size_t)i + (size_t)j * g._nx_;
                const float coordZ = m.coord_at(i, j, k, 2);
                auto B = [&](int l) { return bnds[(size_t)l * plane + c]; };
                // the layer above the first boundary at least 1 km below boundary `from`
                auto take_below = [&](int from) {
                    int l = from;
                    while (l < nLayer && std::fabs(B(from) - B(l)) < BoundaryDifference) l++;
                    const size_t q = (size_t)(l - 1) * plane + c;
                    vs = interp[0][q], vp = interp[1][q], rho = interp[2][q];
                };
                if (coordZ > B(0)) take_below(0);
                if (coordZ <= B(nLayer - 1)) {
                    const size_t q = (size_t)(nLayer - 1) * plane + c;
                    vs = interp[0][q], vp = interp[1][q], rho = interp[2][q];
                }
                if (coordZ <= B(0) && coordZ > B(nLayer - 1))
                    for (int mm = 0; mm < nLayer - 1; mm++)
                        if (coordZ <= B(mm) && coordZ > B(mm + 1)) take_below(mm);
                float *md = &m.medium[id * 3];
                md[0] = (float)(vs * 1e3);
                md[1] = (float)(vp * 1e3);
                md[2] = (float)(rho * 1e3);
            }
    return ST_OK;
}

// Homogeneous default (src/medium.cpp:115-140), then the media the switches
// select in the reference's order (src/medium.cpp:251-295): CRUST1.0, Shen,
// the 1-D layered model (LayeredStructureTerrain on as in Makefile_CGFDM).
static int build_medium(Model &m, const std::string &run_dir, std::string &err)
{
    const Grid &g = m.g;
    m.medium.resize((size_t)g.npad() * 3);
    const long long plane = (long long)g._nx_ * g._ny_;
    par_for(g._nz_, [&](int k) {
        for (long long n = k * plane; n < (k + 1) * plane; n++) {
            m.medium[n * 3 + 0] = 3300.0f;
            m.medium[n * 3 + 1] = 5716.0f;
            m.medium[n * 3 + 2] = 2700.0f;
        }
    });
    if (!m.p.useMedium) return ST_OK;
    if (m.p.Crust_1Model)
        if (int st = crust_medium(m, run_dir, err)) return st;
    if (m.p.ShenModel)
        if (int st = shen_medium(m, run_dir, err)) return st;
    if (!m.p.LayeredModel) return ST_OK;
    std::string path = join(run_dir, m.p.LayeredFileName);
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        err = "cannot open Layered Model file " + path;
        return ST_IO;
    }
    int layers = 0;
    f.read((char *)&layers, 4);
    if (!f || layers < 0 || layers > 100000) {
        err = "bad layered model file " + path;
        return ST_IO;
    }
    std::vector<float> hgt(layers), vsd(layers), vpd(layers), rhod(layers);
    for (int F = 0; F < layers; ++F) {
        float v[4];
        f.read((char *)v, 16);
        if (!f) {
            err = "layered model file too short: " + path;
            return ST_IO;
        }
        hgt[F] = v[0] * 1000.0f;
        if (F != 0) hgt[F] += 0.0f;
        vsd[F] = v[1] * 1000.f;
        vpd[F] = v[2] * 1000.f;
        rhod[F] = v[3] * 1000.f;
    }
    const float tolerance = 1.0f;
    par_for(g._nz_, [&](int k) {
        for (int j = 0; j < g._ny_; j++)
            for (int i = 0; i < g._nx_; i++) {
                long long id = g.idx(i, j, k);
                double terrain = m.terrain[(size_t)i + (size_t)j * g._nx_];
                float coordz = m.coord_at(i, j, k, 2);
                float *md = &m.medium[id * 3];
                for (int F = 1; F < layers; ++F) {
                    float h0 = (float)(-hgt[0] + terrain);
                    float h1 = (float)(-hgt[F - 1] + terrain);
                    float h2 = (float)(-hgt[F] + terrain);
                    if (coordz > (h0 - tolerance)) md[0] = vsd[0], md[1] = vpd[0], md[2] = rhod[0];
                    if ((h1 - tolerance) > coordz && coordz > (h2 - tolerance))
                        md[0] = vsd[F - 1], md[1] = vpd[F - 1], md[2] = rhod[F - 1];
                    if ((h2 - tolerance) > coordz) md[0] = vsd[F], md[1] = vpd[F], md[2] = rhod[F];
                }
            }
    });
    return ST_OK;
}

// Extension: raw float32 [_nz_][_ny_][_nx_][3] (Vs, Vp, rho) volume.
// A raw float32 volume, read by the process's cores in plane-sized pieces
// (pread at independent offsets), each piece landing in the pages that the
// reading thread first touches.
static int medium_file(Model &m, const std::string &path, std::string &err)
{
    const int fd = open(path.c_str(), O_RDONLY);
    if (fd < 0) {
        err = "cannot open medium file " + path;
        return ST_IO;
    }
    const long long plane_bytes = (long long)m.g._nx_ * m.g._ny_ * 3 * (long long)sizeof(float);
    std::atomic<bool> short_read(false);
    par_for(m.g._nz_, [&](int k) {
        char *dst = (char *)m.medium.data() + (size_t)k * plane_bytes;
        long long done = 0;
        while (done < plane_bytes) {
            const ssize_t r = pread(fd, dst + done, (size_t)(plane_bytes - done), (off_t)(k * plane_bytes + done));
            if (r <= 0) {
                short_read = true;
                return;
            }
            done += r;
        }
    });
    close(fd);
    if (short_read) {
        err = "medium file too short: " + path;
        return ST_IO;
    }
    return ST_OK;
}

static void value_ranges(Model &m)
{
    // src/calc_CFL.cpp:165-180,283-285: ranges over the whole padded grid
    // min and max per plane, then over planes (the order does not matter)
    const int nz = m.g._nz_;
    const long long plane = (long long)m.g._nx_ * m.g._ny_;
    std::vector<float> pmn((size_t)nz * 3, 1.0e20f), pmx((size_t)nz * 3, -1.0e20f);
    par_for(nz, [&](int k) {
        float lo[3] = {1.0e20f, 1.0e20f, 1.0e20f}, hi[3] = {-1.0e20f, -1.0e20f, -1.0e20f};
        const float *md = m.medium.data();
        for (long long q = k * plane; q < (k + 1) * plane; q++)
            for (int c = 0; c < 3; c++) {
                float v = md[q * 3 + c];
                if (v < lo[c]) lo[c] = v;
                if (v > hi[c]) hi[c] = v;
            }
        for (int c = 0; c < 3; c++) pmn[k * 3 + c] = lo[c], pmx[k * 3 + c] = hi[c];
    });
    float mn[3] = {1.0e20f, 1.0e20f, 1.0e20f}, mx[3] = {-1.0e20f, -1.0e20f, -1.0e20f};
    for (int k = 0; k < nz; k++)
        for (int c = 0; c < 3; c++) {
            if (pmn[k * 3 + c] < mn[c]) mn[c] = pmn[k * 3 + c];
            if (pmx[k * 3 + c] > mx[c]) mx[c] = pmx[k * 3 + c];
        }
    m.Vs_min = mn[0], m.Vs_max = mx[0];
    m.Vp_min = mn[1], m.Vp_max = mx[1];
    m.rho_min = mn[2], m.rho_max = mx[2];
}

// ------------------------------------------------------------------- PML
// src/init_pml_para.cpp:97-239, all six borders on a single rank; the top
// face is not absorbing under FREE_SURFACE.
static void build_pml(Model &m)
{
    const Grid &g = m.g;
    const int _nx_ = g._nx_, _ny_ = g._ny_, _nz_ = g._nz_;
    const int _nx = g._nx, _ny = g._ny, _nz = g._nz;
    const float DH = g.DH;
    const int nPML = g.nPML;
    const float P_alpha = 1.0f, P_beta = 2.0f, P_d = 2.0f;
    float Cp = 6000.0;
    float pml_fc = 0.5;
    float L = DH * (nPML - 1);
    float R = (float)std::pow(10.0, -(std::log10((double)nPML) - 1.0) / std::log10(2.0) - 3.0);
    float d0 = -(P_d + 1.0f) * Cp / (2.0f * L) * logf(R);
    float pml_alpha0 = REF_PI * pml_fc;
    float pml_beta0 = 3.0;
    auto cal_alpha = [&](float l) { return (l < 0.0f) ? 0.0f : (pml_alpha0 * (1.0f - powf(l / L, P_alpha))); };
    auto cal_beta = [&](float l) { return (l < 0.0f) ? 1.0f : (1.0f + (pml_beta0 - 1.0f) * powf(l / L, P_beta)); };
    auto cal_d = [&](float l) { return (l < 0.0f) ? 0.0f : (d0 * powf(l / L, P_d)); };

    auto axis = [&](int n_, int n_in, bool lo, bool hi, bool allow_hi, std::vector<float> &al,
                    std::vector<float> &be, std::vector<float> &dd) {
        std::vector<float> Ls(n_, -1.0f);
        for (int i = HALO; i < n_in; ++i) {
            if (i < HALO + nPML && lo) Ls[i] = (HALO + nPML - 1 - i) * DH;
            if (allow_hi && i >= n_in - nPML && hi) Ls[i] = (i - (n_in - nPML)) * DH;
        }
        al.assign(n_, 0.0f);
        be.assign(n_, 1.0f);
        dd.assign(n_, 0.0f);
        for (int i = HALO; i < n_in; ++i) {
            al[i] = cal_alpha(Ls[i]);
            be[i] = cal_beta(Ls[i]);
            dd[i] = cal_d(Ls[i]);
        }
        for (int i = 0; i < n_; ++i) {
            dd[i] /= be[i];
            be[i] = 1.0f / be[i];
        }
    };
    axis(_nx_, _nx, m.border[0], m.border[1], true, m.pml_alpha_x, m.pml_beta_x, m.pml_d_x);
    axis(_ny_, _ny, m.border[2], m.border[3], true, m.pml_alpha_y, m.pml_beta_y, m.pml_d_y);
    axis(_nz_, _nz, m.border[4], m.border[5], false, m.pml_alpha_z, m.pml_beta_z, m.pml_d_z);
}

// ---------------------------------------------------------- point sources
// Gaussian spatial weights of the 7x7x7 smoothed point source
// (src/singleSource.cpp:134-143, GAUSS_FUN of src/macro.h:37).
std::vector<float> point_gauss_weights(int nGauss)
{
    std::vector<float> amp;
    float ra = (float)(nGauss * 0.5);
    for (int dk = -nGauss; dk <= nGauss; dk++)
        for (int dj = -nGauss; dj <= nGauss; dj++)
            for (int di = -nGauss; di <= nGauss; di++) {
                auto gf = [&](int t) {
                    double q = ((t) - (0.0)) / (ra);
                    return (float)(std::exp(-(q * q)) / (ra * 1.772453850905516));
                };
                float D1 = gf(di), D2 = gf(dj), D3 = gf(dk);
                float a = D1 * D2 * D3;
                a = (float)(a / 0.998125703461425);
                amp.push_back(a);
            }
    return amp;
}

// Source time of stage irk of step it (src/singleSource.cpp:47-59).
static float stage_time(int it, int irk, float DT)
{
    if (irk == 0) return (it + 0.0f) * DT;
    if (irk == 3) return (it + 1.0f) * DT;
    return (it + 0.5f) * DT;
}

float point_ricker(float rickerfc, int it, int irk, float DT)
{
    float t = stage_time(it, irk, DT);
    float tdelay = 1.0f / rickerfc;
    float r = REF_PI * rickerfc * (t - tdelay);
    float rr = r * r;
    float s = (float)(r * (3.0 - 2.0f * rr) * expf(-rr) * sqrtf(REF_PI) * 0.5 * rickerfc * REF_PI);
    float M0 = 1e9;
    s *= M0;
    return s;
}

float point_gauss_stf(float duration, int it, int irk, float DT)
{
    float t = stage_time(it, irk, DT);
    float tdelay = duration / 2 + 1;
    return expf(-(t - tdelay) * (t - tdelay) / (duration * duration)) / (sqrtf(REF_PI) * duration);
}

// Moment-tensor components from strike/dip/rake in radians, in the
// reference's float/double mix (src/multiSource.cpp:507-519,
// src/singleSource.cpp:257-269), returned as (Mxx, Myy, Mzz, Mxy, Mxz, Myz)
// = (M22, M11, M33, M12, -M23, -M13) before scaling.
struct MT {
    float M11, M22, M33, M12, M13, M23;
};
static MT moment_tensor(float s, float d, float r)
{
    MT t;
    double sdcr = (double)(sinf(d) * cosf(r));
    t.M11 = (float)(-(sdcr * std::sin(2.0 * s) + std::sin(2.0 * d) * sinf(r) * sinf(s) * sinf(s)));
    t.M22 = (float)(sdcr * std::sin(2.0 * s) - std::sin(2.0 * d) * sinf(r) * cosf(s) * cosf(s));
    t.M33 = -(t.M11 + t.M22);
    t.M12 = (float)(sdcr * std::cos(2.0 * s) + 0.5 * std::sin(2.0 * d) * sinf(r) * std::sin(2.0 * s));
    t.M13 = (float)(-((double)(cosf(d) * cosf(r) * cosf(s)) + std::cos(2.0 * d) * sinf(r) * sinf(s)));
    t.M23 = (float)(-((double)(cosf(d) * cosf(r) * sinf(s)) - std::cos(2.0 * d) * sinf(r) * cosf(s)));
    return t;
}

static void build_point_source(Model &m)
{
    const Grid &g = m.g;
    PointSource &ps = m.point;
    if (!m.p.useSingleSource_ricker && !m.p.useSingleSource_double_couple) return;
    ps.kind = m.p.useSingleSource_ricker ? 1 : 2;
    // src/singleSource.cpp:25-40 (locateSource), single rank
    ps.X = m.p.sourceX + HALO, ps.Y = m.p.sourceY + HALO, ps.Z = m.p.sourceZ + HALO;
    ps.inside = ps.X >= HALO && ps.X < g._nx && ps.Y >= HALO && ps.Y < g._ny && ps.Z >= HALO && ps.Z < g._nz;
    ps.amp = point_gauss_weights(3);
    float DT = (float)m.p.DT;
    ps.stf.resize(m.NT);
    if (ps.kind == 1) {
        for (int it = 0; it < m.NT; it++) ps.stf[it] = point_ricker(m.p.rickerfc, it, 0, DT);
    } else {
        for (int it = 0; it < m.NT; it++) ps.stf[it] = point_gauss_stf(m.p.duration, it, 0, DT);
        point_moment(m.p.strike, m.p.dip, m.p.rake, m.p.Mw, ps.mom, &ps.m0);
    }
}

void point_moment(float strike, float dip, float rake, float Mw, float mom[6], float *m0)
{
    float s = (float)(strike * REF_DEG2RAD), d = (float)(dip * REF_DEG2RAD);
    float r = (float)(rake * REF_DEG2RAD);
    MT t = moment_tensor(s, d, r);
    mom[0] = t.M22, mom[1] = t.M11, mom[2] = t.M33;
    mom[3] = t.M12, mom[4] = -t.M23, mom[5] = -t.M13;
    *m0 = (float)(1.5 * powf(10, Mw + 6));
}

// ----------------------------------------------------- finite-fault source
// src/multiSource.cpp:24-868 for one rank, up to (but not including) the
// mu/(J DH^3) scaling, which needs the metric and runs on the GPU.
static int build_fault(Model &m, const std::string &run_dir, std::string &err)
{
    const Grid &g = m.g;
    FaultSource &fs = m.fault;
    std::string path = join(join(run_dir, m.p.sourceDir), m.p.sourceFile);
    if (!m.p.sourceDir.empty() && m.p.sourceDir[0] == '/') path = join(m.p.sourceDir, m.p.sourceFile);
    std::ifstream f(path, std::ios::binary);
    if (!f) {
        err = "can't open source file " + path;
        return ST_IO;
    }
    int npts_i = 0, nt = 0;
    float dt = 0;
    f.read((char *)&npts_i, 4);
    f.read((char *)&nt, 4);
    f.read((char *)&dt, 4);
    if (!f || npts_i < 0 || nt < 0) {
        err = "bad source file header " + path;
        return ST_IO;
    }
    const long long npts = npts_i;
    const long long rec = 6 * 4 + 2LL * 4 * nt;
    std::vector<float> x(npts), y(npts), z(npts);
    for (long long i = 0; i < npts; i++) {
        float v[3];
        f.seekg(12 + rec * i, std::ios::beg);
        f.read((char *)v, 12);
        if (!f) {
            err = "source file too short: " + path;
            return ST_IO;
        }
        x[i] = v[0], y[i] = v[1], z[i] = v[2];
    }
    // projection (src/multiSource.cpp:96-171): the centre goes through the
    // "%lf" formatting of a float, source points through DEGREE2RADIAN
    {
        char buf[64];
        float lon_0 = (float)m.p.centerLongitude, lat_0 = (float)m.p.centerLatitude;
        std::snprintf(buf, sizeof buf, "%lf", (double)lon_0);
        double lon0 = std::atof(buf) * (3.14159265358979323846 / 180.0);
        std::snprintf(buf, sizeof buf, "%lf", (double)lat_0);
        double lat0 = std::atof(buf) * (3.14159265358979323846 / 180.0);
        for (long long i = 0; i < npts; i++) {
            double px, py;
            cgfdm_aeqd_fwd(lon0, lat0, x[i] * REF_DEG2RAD, y[i] * REF_DEG2RAD, &px, &py);
            x[i] = (float)px;
            y[i] = (float)py;
        }
    }
    // cell location (src/multiSource.cpp:173-314, NO_SOURCE_SMOOTH branch)
    float Depth = m.p.Depth * 1000;
    const float DH = g.DH;
    float maxCoordZ = -Depth;
    for (long long jj = 0; jj < npts; jj++)
        if (maxCoordZ < z[jj]) maxCoordZ = z[jj];
    for (long long jj = 0; jj < npts; jj++) z[jj] = z[jj] - maxCoordZ;
    std::map<long long, long long> point_index;
    long long pointNum = 0;
    for (long long i = 0; i < npts; i++) {
        int srcX = int(x[i] / DH + 0.5) + g.originalX + HALO;
        int srcY = int(y[i] / DH + 0.5) + g.originalY + HALO;
        if (srcX >= HALO && srcX < g._nx && srcY >= HALO && srcY < g._ny) {
            double DZ = m.coord_at(srcX, srcY, 4, 2) - m.coord_at(srcX, srcY, 3, 2);
            double terrain = DZ * double(g.NZ - 1) - std::fabs(Depth);
            z[i] = (float)(terrain + z[i]);
            for (int k = HALO; k < g._nz; k++) {
                long long index = g.idx(srcX, srcY, k);
                const float zk = m.coord_at(srcX, srcY, k, 2);
                double dz1 = (zk - m.coord_at(srcX, srcY, k - 1, 2)) * 0.5;
                double dz2 = (m.coord_at(srcX, srcY, k + 1, 2) - zk) * 0.5;
                if (zk - dz1 <= z[i] && z[i] < dz2 + zk) {
                    point_index[i] = index;
                    pointNum++;
                }
            }
        }
    }
    // parameters of the located points, in sub-fault order (:345-396)
    std::vector<float> area(pointNum, 0.f), strike(pointNum, 0.f), dip(pointNum, 0.f);
    std::vector<float> rake((size_t)pointNum * nt, 0.f), rate((size_t)pointNum * nt, 0.f);
    {
        long long i = 0;
        for (auto &pi : point_index) {
            f.clear();
            f.seekg(12 + rec * pi.first + 12, std::ios::beg);
            f.read((char *)&area[i], 4);
            f.read((char *)&strike[i], 4);
            f.read((char *)&dip[i], 4);
            f.read((char *)&rake[(size_t)i * nt], 4LL * nt);
            f.read((char *)&rate[(size_t)i * nt], 4LL * nt);
            if (!f) {
                err = "source file too short: " + path;
                return ST_IO;
            }
            i++;
        }
    }
    // moment rate per point and sample (:450-535)
    std::vector<float> mr((size_t)pointNum * nt * 6, 0.f);
    for (long long p = 0; p < pointNum; p++) {
        float s = (float)(strike[p] * REF_DEG2RAD), d = (float)(dip[p] * REF_DEG2RAD), a = area[p];
        for (int it = 0; it < nt; it++) {
            long long index = it + p * nt;
            float r = m.p.degree2radian == 0 ? rake[index] : (float)(rake[index] * REF_DEG2RAD);
            float rt = rate[index];
            MT t = moment_tensor(s, d, r);
            mr[index * 6 + 0] = t.M22 * a * rt;
            mr[index * 6 + 1] = t.M11 * a * rt;
            mr[index * 6 + 2] = t.M33 * a * rt;
            mr[index * 6 + 3] = t.M12 * a * rt;
            mr[index * 6 + 4] = -t.M23 * a * rt;
            mr[index * 6 + 5] = -t.M13 * a * rt;
        }
    }
    // sub-faults sharing a cell are summed into the last of them (:537-592)
    std::map<long long, long long> index_point;
    {
        long long i = 0;
        for (auto &pi : point_index) index_point[pi.second] = i++;
        i = 0;
        for (auto &pi : point_index) {
            long long ii = index_point[pi.second];
            if (ii > i)
                for (int t = 0; t < nt; t++)
                    for (int c = 0; c < 6; c++)
                        mr[((size_t)t + ii * nt) * 6 + c] += mr[((size_t)t + i * nt) * 6 + c];
            i++;
        }
    }
    // reorder to [t][cell] with cells ascending by grid index (:706-752)
    fs.npts = (long long)index_point.size();
    fs.nt = nt;
    fs.dt = dt;
    fs.index.resize(fs.npts);
    fs.rate.assign((size_t)fs.npts * nt * 6, 0.f);
    long long J = 0;
    for (auto &ip : index_point) {
        fs.index[J] = ip.first;
        long long ii = ip.second;
        for (int t = 0; t < nt; t++)
            for (int c = 0; c < 6; c++)
                fs.rate[((size_t)J + (size_t)t * fs.npts) * 6 + c] = mr[((size_t)ii * nt + t) * 6 + c];
        J++;
    }
    return ST_OK;
}

// --------------------------------------------------------------- stations
// src/station.cpp:92-292: global [X, Y, Z] indices, kept when inside the
// interior; a missing file means no stations, a malformed entry stops reading.
static int read_stations(Model &m, const std::string &run_dir, std::string &err)
{
    std::string path = join(run_dir, "station.json");
    std::ifstream f(path);
    if (!f) return ST_OK;
    JsonValue root;
    std::string e;
    if (!json_parse_file(path, root, e)) return ST_OK;  // reference: "Can't parse json file!", no stations
    const JsonValue *arr = root.get("station(point)");
    if (!arr) return ST_OK;
    const Grid &g = m.g;
    std::vector<int> loc, glob;
    const size_t cnt = arr->kind == JsonValue::Object ? arr->members.size() : arr->items.size();
    for (size_t i = 0; i < cnt; i++) {
        const JsonValue &s = arr->kind == JsonValue::Object ? arr->members[i].second : arr->items[i];
        size_t a = s.kind == JsonValue::Object ? s.members.size() : s.items.size();
        if (a != 3) {
            err = "station entry without 3 indices";
            m.stations.clear();
            m.stations_global.clear();
            return ST_OK;
        }
        auto at = [&](int q) { return s.kind == JsonValue::Object ? s.members[q].second.as_int() : s.items[q].as_int(); };
        int X = at(0), Y = at(1), Z = at(2);
        int tx = X + HALO, ty = Y + HALO, tz = Z + HALO;
        if (tx >= HALO && tx < g._nx && ty >= HALO && ty < g._ny && tz >= HALO && tz < g._nz) {
            loc.insert(loc.end(), {tx, ty, tz});
            glob.insert(glob.end(), {X, Y, Z});
        }
    }
    m.stations = loc;
    m.stations_global = glob;
    return ST_OK;
}

// ------------------------------------------------------------------ model
int build_model(const std::string &run_dir, const std::string &options_json, Model &m, std::string &err)
{
    return build_model(run_dir, options_json, m, err, {});
}

int build_model(const std::string &run_dir, const std::string &options_json, Model &m, std::string &err,
                const std::function<void(const Model &)> &medium_ready)
{
    int st = read_params(join(run_dir, "params.json"), m.p, err);
    if (st) return st;
    if (!options_json.empty()) {
        // run-time overrides as a JSON object with the same keys
        JsonValue o;
        if (!json_parse(options_json, o, err) || o.kind != JsonValue::Object) {
            err = "bad options json: " + err;
            return ST_JSON;
        }
        const JsonValue *it;
        if ((it = o.get("scheme")) && it->kind == JsonValue::String) {
            std::string s = it->str;
            for (auto &c : s) c = (char)std::toupper((unsigned char)c);
            m.p.scheme = (s == "SCFDM" || s == "AWENO") ? SCHEME_SCFDM : SCHEME_CGFDM;
            m.p.pml = m.p.scheme == SCHEME_CGFDM;
            m.p.exp_decay = m.p.scheme == SCHEME_SCFDM;
        }
        if ((it = o.get("PML"))) m.p.pml = it->as_int();
        if ((it = o.get("EXP_DECAY"))) m.p.exp_decay = it->as_int();
        if ((it = o.get("SOLVE_DISPLACEMENT"))) m.p.solve_displacement = it->as_int();
        if ((it = o.get("SOLVE_PGA"))) m.p.solve_pga = it->as_int();
        if ((it = o.get("metricPrecision")) && it->kind == JsonValue::String) m.p.metric_fp64 = it->str == "fp64";
        if ((it = o.get("storage")) && it->kind == JsonValue::String) m.p.storage = it->str;
        if ((it = o.get("adjointKernel")) && it->kind == JsonValue::String) m.p.adj_fused = it->str == "fused";
        if ((it = o.get("adjointStoreSegments"))) m.p.adj_store_max = it->as_int();
        if ((it = o.get("OUT")) && it->kind == JsonValue::String) m.p.OUT = it->str;
        if ((it = o.get("checkFinite"))) m.p.check_finite = std::max(0, it->as_int());
        if ((it = o.get("stagePipeline")) && it->kind == JsonValue::String) m.p.stage_split = it->str != "ring";
        if ((it = o.get("stageTile"))) m.p.stage_tile = it->as_int();
    }
    Params &p = m.p;
    if (p.NX <= 0 || p.NY <= 0 || p.NZ <= 0 || p.DH <= 0 || p.DT <= 0) {
        err = "NX, NY, NZ, DH and DT must be positive";
        return ST_OPTIONS;
    }
    if (p.PX != 1 || p.PY != 1 || p.PZ != 1) {
        // a session runs the whole grid on one device; a decomposition is
        // explicit (cgfdm_create_part, partition.cpp)
        p.PX = p.PY = p.PZ = 1;
    }
    // src/modelChecking.cpp:17-61
    if (p.useSingleSource_ricker && p.useSingleSource_double_couple) {
        err = "useSingleSource(ricker) and useSingleSource(double_couple) set at the same time";
        return ST_OPTIONS;
    }
    if (!(p.useMultiSource || p.useSingleSource_ricker || p.useSingleSource_double_couple)) {
        err = "no source set";
        return ST_OPTIONS;
    }
    if (p.gauss_hill && !p.terrainFile.empty()) {
        err = "gauss_hill and terrainFile are exclusive";
        return ST_OPTIONS;
    }
    if (p.storage != "fp32" && p.storage != "fp16" && p.storage != "bf16") {
        err = "storage must be fp32, fp16 or bf16";
        return ST_OPTIONS;
    }
    m.g = make_grid(p);
    const Grid &g = m.g;
    float DT = (float)p.DT;
    m.NT = (int)(p.TMAX / DT);  // src/propagate.cpp:88
    if (m.NT < 0) m.NT = 0;
    if (p.pml && p.scheme == SCHEME_CGFDM) {
        if (g.nPML >= g.nx || g.nPML >= g.ny || g.nPML >= g.nz) {
            err = "The PML layer(nPML) is not smaller than nx/ny/nz";
            return ST_PML_SIZE;
        }
        if (g.nPML < 2) {
            err = "nPML must be at least 2";
            return ST_PML_SIZE;
        }
    }
    auto tick = std::chrono::steady_clock::now();
    auto lap = [&](int ph) {
        const auto now = std::chrono::steady_clock::now();
        m.phase_ms[ph] = std::chrono::duration<double, std::milli>(now - tick).count();
        tick = now;
    };
    build_coords(m, true);
    if (p.gauss_hill) gauss_hill(m);
    else if (!p.terrainFile.empty()) {
        if ((st = terrain_file(m, join(run_dir, p.terrainFile), err))) return st;
    }
    if (p.useTerrain) {   // src/coord.cpp:325-328
        if (p.SRTM90 == 1)
            if ((st = srtm_terrain(m, run_dir, err))) return st;
        terrain_z_double(m);
    }
    lap(0);
    if (p.mediumFile.empty()) {
        if ((st = build_medium(m, run_dir, err))) return st;
    } else {
        // a raw volume replaces whatever the switches would build
        m.medium.resize((size_t)g.npad() * 3);
        if ((st = medium_file(m, join(run_dir, p.mediumFile), err))) return st;
    }
    lap(1);
    if (medium_ready) medium_ready(m);
    value_ranges(m);
    build_pml(m);
    lap(2);
    build_point_source(m);
    if (p.useMultiSource)
        if ((st = build_fault(m, run_dir, err))) return st;
    lap(3);
    if ((st = read_stations(m, run_dir, err))) return st;
    lap(4);
    return ST_OK;
}

}  // namespace cgfdm
