// Host-side model description: run parameters, grid, coordinates, medium,
// PML profiles, sources and stations.  Everything here mirrors the
// reference's setup stage (src/run.cpp:28-138) for a single rank and is
// computed on the host in the reference's own float/double mix, so the
// arrays handed to the GPU are bit-identical to what the reference builds.
#pragma once

#include <cstdint>
#include <functional>
#include <memory>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>
#include <cstdlib>
#include <new>
#include <sys/mman.h>

#include "json.hpp"

namespace cgfdm {

// An allocator whose value-less construct leaves the element uninitialised:
// resize() of a FieldVec does not write the hundreds of megabytes of a
// padded volume from one thread; the parallel loops that fill it first touch
// its pages on the cores that use them.
template <class T>
struct DefaultInitAlloc : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = DefaultInitAlloc<U>;
    };
    DefaultInitAlloc() = default;
    template <class U>
    DefaultInitAlloc(const DefaultInitAlloc<U> &) noexcept {}
    // Volumes of 32 MB and more on 2 MB boundaries, marked for transparent
    // huge pages: their first touch (the parallel file read or fill) then
    // faults a 2 MB page at a time instead of a 4 KB one.
    static constexpr size_t HUGE_MIN = size_t(32) << 20, HUGE_ALIGN = size_t(2) << 20;
    T *allocate(size_t n)
    {
        const size_t bytes = n * sizeof(T);
        if (bytes < HUGE_MIN) return std::allocator<T>::allocate(n);
        const size_t rounded = (bytes + HUGE_ALIGN - 1) / HUGE_ALIGN * HUGE_ALIGN;
        void *p = std::aligned_alloc(HUGE_ALIGN, rounded);
        if (!p) throw std::bad_alloc();
        madvise(p, rounded, MADV_HUGEPAGE);   // advice only: no error if refused
        return static_cast<T *>(p);
    }
    void deallocate(T *p, size_t n)
    {
        if (n * sizeof(T) < HUGE_MIN) std::allocator<T>::deallocate(p, n);
        else std::free(p);
    }
    template <class U>
    void construct(U *p) noexcept(std::is_nothrow_default_constructible<U>::value)
    {
        ::new ((void *)p) U;
    }
    template <class U, class... A>
    void construct(U *p, A &&...args)
    {
        ::new ((void *)p) U(std::forward<A>(args)...);
    }
};
using FieldVec = std::vector<float, DefaultInitAlloc<float>>;


constexpr int HALO = 3;

// Status codes returned through the C ABI (reference abort codes where one
// exists: src/getParams.cpp:100,1001; src/calc_CFL.cpp:344 (110);
// src/pml_deriv.cpp:58 (130); src/modelChecking.cpp:27 (180); alloc 10001).
enum Status : int {
    ST_OK = 0,
    ST_NO_PARAMS = 100,
    ST_CFL = 110,
    ST_PML_SIZE = 130,
    ST_OPTIONS = 180,
    ST_JSON = 1001,
    ST_IO = 1002,
    ST_ALLOC = 10001,
    ST_CUDA = 20001,
    ST_TIMEOUT = 20002,
    ST_ARG = 20003,
    ST_STATE = 20004,
    ST_NONFINITE = 20005,
};

enum Scheme { SCHEME_CGFDM = 0, SCHEME_SCFDM = 1 };

// Fields of the reference's PARAMS (src/struct.h:21-116) that the hot path
// and its inputs use, zero-initialised (the reference leaves missing keys
// uninitialised, src/main.cpp:20), plus run-time switches that replace the
// reference's compile-time ones.
struct Params {
    double TMAX = 0, DT = 0, DH = 0;
    int NX = 0, NY = 0, NZ = 0;
    int PX = 1, PY = 1, PZ = 1;
    int centerX = 0, centerY = 0;
    double centerLatitude = 0, centerLongitude = 0;
    int sourceX = 0, sourceY = 0, sourceZ = 0;
    int IT_SKIP = 0;
    int sliceX = 0, sliceY = 0, sliceZ = 0, sliceFreeSurf = 0;
    int nPML = 0;
    int gauss_hill = 0, useTerrain = 0, useMedium = 0, useMultiSource = 0;
    int useSingleSource_ricker = 0;
    float rickerfc = 0;
    int useSingleSource_double_couple = 0;
    float strike = 0, dip = 0, rake = 0, Mw = 0, duration = 0;
    int ShenModel = 0, Crust_1Model = 0, LayeredModel = 0;
    float MLonStart = 0, MLatStart = 0, MLonEnd = 0, MLatEnd = 0, MLonStep = 0, MLatStep = 0;
    float MVeticalStep = 0, CrustLonStep = 0, CrustLatStep = 0;
    std::string MediumDir, CrustDir;
    int SRTM90 = 0, lonStart = 0, latStart = 0, blockX = 1, blockY = 1;
    std::string TerrainDir;
    std::string LayeredFileName;
    std::string OUT;
    float Depth = 0;
    std::string sourceFile, sourceDir;
    int degree2radian = 0;

    // run-time replacements of the reference's -D switches
    int scheme = SCHEME_CGFDM;       // "scheme": "CGFDM" | "SCFDM" (Makefile_CGFDM / Makefile_SCFDM)
    int pml = 1;                     // PML on 5 faces (CGFDM default build)
    int exp_decay = 0;               // exponential sponge (SCFDM default build)
    int solve_displacement = 0;      // SOLVE_DISPLACEMENT
    int solve_pga = 0;               // SOLVE_PGA: peak ground acceleration beside PGV
    int metric_fp64 = 0;             // "metricPrecision": "fp64" -> metrics computed in FP64
    int adj_fused = 0;               // options "adjointKernel": "two-pass" (default) | "fused"
    int adj_store_max = 0;           // options "adjointStoreSegments": cap on segments kept from the forward (0: memory decides)
    std::string storage = "fp32";    // "storage": "fp32" | "fp16" | "bf16"
    int check_finite = 0;            // "checkFinite": scan the wavefield for NaN/Inf every K steps (0: never)
    int stage_split = 1;             // "stagePipeline": "split" (default) | "ring" (CGFDM FP32 stage kernel)
    int stage_tile = 0;              // "stageTile": 4 | 8 rows of 32 columns (0: 8 for the FP32 split pipeline, else 4)
    // extension inputs (raw arrays the reference has no reader for)
    std::string terrainFile;         // float32 [_ny_][_nx_] surface height (m)
    std::string mediumFile;          // float32 [_nz_][_ny_][_nx_][3] Vs, Vp, rho
};

// Reads params.json with the reference's keys (src/getParams.cpp:58-242).
int read_params(const std::string &path, Params &p, std::string &err);

// Single-rank grid (src/init_grid.cpp:17-106).
struct Grid {
    int NX, NY, NZ;
    int nx, ny, nz;
    int _nx_, _ny_, _nz_;
    int _nx, _ny, _nz;
    int originalX, originalY;
    int nPML;
    float DH, rDH;
    long long npad() const { return (long long)_nx_ * _ny_ * _nz_; }
    long long interior() const { return (long long)nx * ny * nz; }
    long long idx(int i, int j, int k) const { return i + (long long)j * _nx_ + (long long)k * _nx_ * _ny_; }
};
Grid make_grid(const Params &p);

// Finite-fault source after reading, projection, cell location, moment
// tensor, duplicate merge and reordering (src/multiSource.cpp:780-868).
struct FaultSource {
    long long npts = 0;              // distinct grid cells
    int nt = 0;
    float dt = 0;
    std::vector<long long> index;    // padded-grid index per cell, ascending
    std::vector<float> rate;         // [nt][npts][6] Mxx Myy Mzz Mxy Mxz Myz (before mu/(J DH^3))
};

// Single point source (src/singleSource.cpp:25-359).
struct PointSource {
    int kind = 0;                    // 0 none, 1 Ricker (explosive), 2 double couple
    int X = 0, Y = 0, Z = 0;         // padded indices
    bool inside = false;             // reference only injects for interior points
    std::vector<float> amp;          // [7][7][7] Gaussian weights (float, after /0.998...)
    std::vector<float> stf;          // [NT] source-time value at stage-0 time of each step
    float mom[6] = {0, 0, 0, 0, 0, 0};  // double couple: M22 M11 M33 M12 -M23 -M13
    float m0 = 0;
};

struct Model {
    Params p;
    Grid g;
    int NT = 0;
    FieldVec coord;                  // [_nz_][_ny_][_nx_][3] (AoS, reference layout)
    // how coord was made from the grid and the terrain, so the device can
    // make it again instead of receiving it: 0 flat, 1 terrain-following in
    // float (Gauss hill, terrain file; coord_depth_f = Depth * 1000), 2
    // terrain-following in double (useTerrain; coord_depth_d = Depth * 1e3),
    // -1 neither (a part of a decomposed grid: coord is uploaded)
    int coord_mode = 0;
    float coord_depth_f = 0;
    double coord_depth_d = 0;
    // coord not filled: every coordinate follows from the grid, the terrain
    // and coord_mode, and coord_at computes it (the host model build reads
    // only a few columns and layers of it); materialize_coords fills coord
    // for the readers of the whole volume
    bool coord_lazy = false;
    float coord_at(int i, int j, int k, int c) const;
    std::vector<float> terrain;      // [_ny_][_nx_]
    std::vector<double> lon, lat;    // [_ny_][_nx_] column longitude, latitude (SRTM90 runs)
    FieldVec medium;                 // [_nz_][_ny_][_nx_][3] Vs Vp rho
    float H_min = 0, H_max = 0, Vs_min = 0, Vs_max = 0, Vp_min = 0, Vp_max = 0, rho_min = 0, rho_max = 0;
    float dtmax = 0;
    // PML profiles (src/init_pml_para.cpp:97-239): alpha, d/beta, 1/beta per axis
    std::vector<float> pml_alpha_x, pml_beta_x, pml_d_x;
    std::vector<float> pml_alpha_y, pml_beta_y, pml_d_y;
    std::vector<float> pml_alpha_z, pml_beta_z, pml_d_z;
    bool border[6] = {true, true, true, true, true, true};  // x1 x2 y1 y2 z1 z2
    FaultSource fault;
    PointSource point;
    std::vector<int> stations;       // [n][3] padded indices
    std::vector<int> stations_global;// [n][3] global indices as read
    // a sub-domain of a decomposed grid (partition.cpp): interior offset of
    // this part in the global interior, decomposition and this part's place
    // in it, whether it holds the free surface, and the global number of
    // each of its stations
    int part_lo[3] = {0, 0, 0};
    int parts[3] = {1, 1, 1};
    int part_coord[3] = {0, 0, 0};
    // host wall ms of build_model's phases: coordinates and terrain, medium,
    // ranges and PML profiles, sources, stations
    double phase_ms[5] = {0, 0, 0, 0, 0};
    bool fs_top = true;
    std::vector<int> station_ids;
};

// Single point sources (src/singleSource.cpp:42-99, 111-330): the 7 x 7 x 7
// Gaussian weights [dk][dj][di], the Ricker and Gaussian source-time values
// at the stage time of (it, irk), and the moment-tensor components (Mxx,
// Myy, Mzz, Mxy, Mxz, Myz) with m0 of a double couple (degrees).
std::vector<float> point_gauss_weights(int nGauss);
float point_ricker(float rickerfc, int it, int irk, float DT);
float point_gauss_stf(float duration, int it, int irk, float DT);
void point_moment(float strike, float dip, float rake, float Mw, float mom[6], float *m0);

// One part of a PX x PY x PZ decomposition of the global model G (the
// reference's MPI layout, src/init_grid.cpp): interior sizes split as evenly
// as possible, the padded arrays sliced with their 3-cell halos, PML on the
// faces at the global boundary only, the free surface in the top layer of
// parts, sources and stations of the part's interior.  CGFDM only.
int slice_model(const Model &G, const int parts[3], const int coord[3], Model &m, std::string &err);
// fills m.coord if it was left to coord_at (no-op otherwise)
void materialize_coords(Model &m);
// interior offset and size of part c of n along an axis of N points
void part_extent(int N, int n, int c, int *lo, int *len);

// Whole setup from a run directory: params, grid, coordinates, medium, CFL,
// PML profiles, sources and stations.  Metrics are computed on the GPU
// (metrics.cu) from coord and medium.
int build_model(const std::string &run_dir, const std::string &options_json, Model &m, std::string &err);
// As above; medium_ready(m) is called once m.medium is complete (the rest of
// the build only reads it), so a caller can start its upload meanwhile.
int build_model(const std::string &run_dir, const std::string &options_json, Model &m, std::string &err,
                const std::function<void(const Model &)> &medium_ready);

}  // namespace cgfdm
