/*
 * Restated CPU drivers and dump hooks for the oracle's reference CPU build.
 * Test infrastructure only: compiled together with the reference's own
 * src/*.cpp (unmodified, from the read-only reference tree) into the
 * reference oracle binary under oracle/_ref/.
 *
 * What is here:
 *  - definitions for the CPU-branch call sites that do not compile as
 *    shipped (declared in ref_fixups.h); each forwards to the reference's own
 *    kernel function with the arguments its GPU branch passes;
 *  - the SCFDM derivative launcher, whose CPU branch names functions that do
 *    not exist (src/alternative_flux_FD.cpp:1550-1566); this one calls the
 *    reference's six kernels in the order of its GPU branch (:1466-1545);
 *  - the SCFDM metric driver, whose CPU branch runs the CGFDM metric kernel
 *    (src/contravariant.cpp:557-558);
 *  - the double-couple driver (src/singleSource.cpp:320-359), whose CPU
 *    branch calls the Ricker helper;
 *  - SCFDM snapshot conversion (src/data_io.cpp:434-483 for the
 *    conserved->physical map) on top of the non-SCFDM slice writer, because
 *    data_io.cpp's SCFDM branch launches a kernel unconditionally;
 *  - extension-input hooks (raw height map and medium volume, see below);
 *  - dump hooks: the propagate() call in run.cpp is routed through
 *    oracle_hook_propagate (writes CJM and the free-surface matrices), and
 *    freeWave() through oracle_hook_freeWave (writes the final W), so parity
 *    checks can compare whole fields, not only seismograms.
 */
#include "header.h"

#include <string>

static FLOAT *g_oracle_CJM = nullptr;
static GRID g_oracle_grid;
static PARAMS g_oracle_params;

/* ---------------------------------------------------------------- PGV */
void compare_pgv(float *pgv, FLOAT *W, int nx, int ny, int nz, float DT, int it
#ifdef SCFDM
                 , FLOAT *CJM
#endif
);

/* The reference's kernel takes (pgv, W, nx, ny, nz, DT, it [, CJM]); DT and
 * it only matter under SOLVE_PGA (src/PGV.cpp:61-175). */
#ifndef SOLVE_PGA
void compare_pgv(float *pgv, FLOAT *W, int nx, int ny, int nz)
{
    compare_pgv(pgv, W, nx, ny, nz, 0.0f, 0
#ifdef SCFDM
                ,
                g_oracle_CJM
#endif
    );
}
#else
/* Under SOLVE_PGA the kernel also takes W_pre; the shipped CPU branch of
 * comparePGV (src/PGV.cpp:187-229) passes five arguments, so the driver
 * below replaces it (the build renames the shipped one). */
void compare_pgv(float *pgv, FLOAT *W, int nx, int ny, int nz, float DT, int it
#ifdef SCFDM
                 , FLOAT *CJM
#endif
                 , FLOAT *W_pre);
void compare_pgv(float *pgv, FLOAT *W, int nx, int ny, int nz) { (void)pgv, (void)W, (void)nx, (void)ny, (void)nz; }

void comparePGV(GRID grid, MPI_COORDINATE thisMPICoord, FLOAT *W, float *pgv, float DT, int it
#ifdef SCFDM
                , FLOAT *CJM
#endif
                , FLOAT *W_pre)
{
    (void)thisMPICoord;
    compare_pgv(pgv, W, grid.nx, grid.ny, grid.nz, DT, it
#ifdef SCFDM
                , CJM
#endif
                , W_pre);
}

/* src/propagate.cpp:26-58 (cut from the build): one GPU thread per point
 * index copies W_pre[index] = W[index] over _nx_ * _ny_ * _nz_ indices --
 * the first ninth of the nine-field array -- on the CPU the same loop. */
void storage_W_pre(GRID grid, WAVE wave)
{
    const long long n = (long long)grid._nx_ * grid._ny_ * grid._nz_;
    for (long long index = 0; index < n; index++) wave.W_pre[index] = wave.W[index];
}
#endif

/* ---------------------------------------------------------- point sources */
void load_smooth_source_ricker(SOURCE S, FLOAT *h_W, int _nx_, int _ny_, int _nz_,
                               FLOAT *CJM, int it, int iRK, float DT, float DH, int nGauss, float rickerfc);
void load_smooth_source_double_couple(SOURCE S, FLOAT *h_W, int _nx_, int _ny_, int _nz_,
                                      FLOAT *CJM, int it, int iRK, float DT, float DH, int nGauss,
                                      float strike, float dip, float rake, float Mw, float duration);

void load_smooth_source(SOURCE S, FLOAT *h_W, int _nx_, int _ny_, int _nz_,
                        FLOAT *CJM, int it, int irk, float DT, float DH, int nGauss, float rickerfc)
{
    load_smooth_source_ricker(S, h_W, _nx_, _ny_, _nz_, CJM, it, irk, DT, DH, nGauss, rickerfc);
}

void loadPointSource_double_couple(GRID grid, SOURCE S, FLOAT *h_W, FLOAT *CJM, int it, int irk,
                                   float DT, float DH, float strike, float dip, float rake, float Mw,
                                   float duration)
{
    const int nGauss = 3;
    int _nx = grid._nx_ - HALO, _ny = grid._ny_ - HALO, _nz = grid._nz_ - HALO;
    if (S.X >= HALO && S.X < _nx && S.Y >= HALO && S.Y < _ny && S.Z >= HALO && S.Z < _nz)
        load_smooth_source_double_couple(S, h_W, grid._nx_, grid._ny_, grid._nz_, CJM, it, irk, DT, DH,
                                         nGauss, strike, dip, rake, Mw, duration);
}

#ifdef SCFDM
/* ------------------------------------------------ SCFDM CJM-taking kernels */
void addSource1(FLOAT *hW, float *momentRateSlice, long long *srcIndex, int npts, float DT, FLOAT *CJM);
void addSource1(FLOAT *hW, float *momentRateSlice, long long *srcIndex, int npts, float DT)
{
    addSource1(hW, momentRateSlice, srcIndex, npts, DT, g_oracle_CJM);
}

void storage_station(int stationNum, STATION station, FLOAT *W, int _nx_, int _ny_, int _nz_, int NT, int it,
                     FLOAT *CJM);
void storage_station(int stationNum, STATION station, FLOAT *W, int _nx_, int _ny_, int _nz_, int NT, int it)
{
    storage_station(stationNum, station, W, _nx_, _ny_, _nz_, NT, it, g_oracle_CJM);
}

/* ----------------------------------------------- SCFDM derivative launcher */
void wave_deriv_alternative_flux_FD_x(FLOAT *Riemann_flux, FLOAT *h_W, FLOAT *W, FLOAT *CJM,
                                      int _nx_, int _ny_, int _nz_, float rDH, float DT, float alpha);
void wave_deriv_alternative_flux_FD_y(FLOAT *Riemann_flux, FLOAT *h_W, FLOAT *W, FLOAT *CJM,
                                      int _nx_, int _ny_, int _nz_, float rDH, float DT, float alpha);
void wave_deriv_alternative_flux_FD_z(FLOAT *Riemann_flux, FLOAT *h_W, FLOAT *W, FLOAT *CJM,
                                      int _nx_, int _ny_, int _nz_, float rDH, float DT, float alpha);
void cal_du_x(FLOAT *Riemann_flux, FLOAT *h_W, FLOAT *CJM, FLOAT *u,
              int _nx_, int _ny_, int _nz_, float rDH, int FB1, int FB2, int FB3, float DT);
void cal_du_y(FLOAT *Riemann_flux, FLOAT *h_W, FLOAT *CJM, FLOAT *u,
              int _nx_, int _ny_, int _nz_, float rDH, int FB1, int FB2, int FB3, float DT);
void cal_du_z(FLOAT *Riemann_flux, FLOAT *h_W, FLOAT *CJM, FLOAT *u,
              int _nx_, int _ny_, int _nz_, float rDH, int FB1, int FB2, int FB3, float DT);
extern float vp_max_for_SCFDM;

void waveDeriv_alternative_flux_FD(GRID grid, WAVE wave, FLOAT *CJM, int FB1, int FB2, int FB3, float DT,
                                   MPI_COORD, PARAMS)
{
    int _nx_ = grid._nx_, _ny_ = grid._ny_, _nz_ = grid._nz_;
    float rDH = grid.rDH;
    wave_deriv_alternative_flux_FD_x(wave.Riemann_flux, wave.h_W, wave.W, CJM, _nx_, _ny_, _nz_, rDH, DT,
                                     vp_max_for_SCFDM);
    cal_du_x(wave.Riemann_flux, wave.h_W, CJM, wave.W, _nx_, _ny_, _nz_, rDH, FB1, FB2, FB3, DT);
    wave_deriv_alternative_flux_FD_y(wave.Riemann_flux, wave.h_W, wave.W, CJM, _nx_, _ny_, _nz_, rDH, DT,
                                     vp_max_for_SCFDM);
    cal_du_y(wave.Riemann_flux, wave.h_W, CJM, wave.W, _nx_, _ny_, _nz_, rDH, FB1, FB2, FB3, DT);
    wave_deriv_alternative_flux_FD_z(wave.Riemann_flux, wave.h_W, wave.W, CJM, _nx_, _ny_, _nz_, rDH, DT,
                                     vp_max_for_SCFDM);
    cal_du_z(wave.Riemann_flux, wave.h_W, CJM, wave.W, _nx_, _ny_, _nz_, rDH, FB1, FB2, FB3, DT);
}

/* ------------------------------------------------------- SCFDM metrics */
void solve_con_jac_CMM(float *con, float *coord, float *Jac_inv, float *Covariant, int _nx_, int _ny_, int _nz_,
                       float rDH);

/* The GPU branch of src/contravariant.cpp:538-553 (SCFDM): covariant basis
 * by central differences, then cofactors.  The reference's CPU branch calls
 * the CGFDM kernel instead, which leaves CJM[13..18] zero. */
void solveContravariantJac(MPI_Comm, GRID grid, float *con, float *coord, float *Jac, float *, Mat_rDZ)
{
    float DH = grid.DH;
    float rDH = 1.0 / DH;
    long long num = (long long)grid._nx_ * grid._ny_ * grid._nz_;
    float *Cov = (float *)calloc(num * 9, sizeof(float));
    solve_con_jac_CMM(con, coord, Jac, Cov, grid._nx_, grid._ny_, grid._nz_, rDH);
    free(Cov);
}

/* ----------------------------------------------------- SCFDM snapshots */
/* Non-SCFDM slice writer compiled from src/data_io.cpp without -DSCFDM. */
void data2D_XYZ_out(MPI_COORD thisMPICoord, PARAMS params, GRID grid, FLOAT *wave, SLICE slice,
                    SLICE_DATA sliceData, SLICE_DATA sliceDataCpu, char var, int it);

/* Conserved -> physical (src/data_io.cpp:434-483), stored in the CGFDM
 * component order so the non-SCFDM writer picks velocities at 0..2 and
 * stresses at 3..8. */
void data2D_XYZ_out(MPI_COORD thisMPICoord, PARAMS params, GRID grid, FLOAT *wave, SLICE slice,
                    SLICE_DATA sliceData, SLICE_DATA sliceDataCpu, char var, int it, FLOAT *CJM)
{
    long long num = (long long)grid._nx_ * grid._ny_ * grid._nz_;
    FLOAT *phy = (FLOAT *)malloc(sizeof(FLOAT) * WSIZE * num);
    for (long long p = 0; p < num; p++) {
        const FLOAT *u = wave + p * WSIZE;
        float mu = CJM[p * CJMSIZE + 10], lambda = CJM[p * CJMSIZE + 11];
        float buoyancy = CJM[p * CJMSIZE + 12] * Crho;
        FLOAT *o = phy + p * WSIZE;
        o[0] = u[0] * buoyancy;
        o[1] = u[1] * buoyancy;
        o[2] = u[2] * buoyancy;
        o[3] = lambda * u[4] + lambda * u[5] + u[3] * (lambda + 2 * mu);
        o[4] = lambda * u[3] + lambda * u[5] + u[4] * (lambda + 2 * mu);
        o[5] = lambda * u[3] + lambda * u[4] + u[5] * (lambda + 2 * mu);
        o[6] = mu * u[8];
        o[7] = mu * u[7];
        o[8] = mu * u[6];
    }
    data2D_XYZ_out(thisMPICoord, params, grid, phy, slice, sliceData, sliceDataCpu, var, it);
    free(phy);
}
#endif

/* ------------------------------------------------- extension input hooks */
/* The benchmark's curvilinear and heterogeneous configurations need a
 * surface height map and a 3-D (Vs, Vp, rho) volume, which the reference can
 * only build from SRTM/PROJ or Shen/CRUST models.  run.cpp's calls of
 * constructCoord/constructMedium are routed here: after the reference's own
 * construction, a raw float32 height map ("terrainFile", [_ny_][_nx_] in
 * metres) goes through the reference's own terrain-following mapping
 * (construct_terrain_coord, src/coord.cpp:204-255), and a raw float32 volume
 * ("mediumFile", [_nz_][_ny_][_nx_][3]) replaces the medium. */
void construct_terrain_coord(float *coord, float *terrain, int _nx_, int _ny_, int _nz_, int frontNZ, int NZ,
                             float cal_depth);

static std::string oracle_param_string(const char *key)
{
    FILE *fp = fopen("params.json", "r");
    if (!fp) return "";
    fseek(fp, 0, SEEK_END);
    long len = ftell(fp);
    fseek(fp, 0, SEEK_SET);
    std::string text(len, '\0');
    fread(&text[0], 1, len, fp);
    fclose(fp);
    cJSON *root = cJSON_Parse(text.c_str());
    if (!root) return "";
    cJSON *it = cJSON_GetObjectItem(root, key);
    std::string v = (it && it->valuestring) ? it->valuestring : "";
    cJSON_Delete(root);
    return v;
}

static bool oracle_read_raw(const std::string &path, float *dst, size_t n)
{
    FILE *fp = fopen(path.c_str(), "rb");
    if (!fp) {
        fprintf(stderr, "oracle: cannot open %s\n", path.c_str());
        exit(1002 & 0xff);
    }
    size_t got = fread(dst, sizeof(float), n, fp);
    fclose(fp);
    if (got != n) {
        fprintf(stderr, "oracle: %s too short\n", path.c_str());
        exit(1002 & 0xff);
    }
    return true;
}

static void oracle_dump(const char *name, const void *data, size_t bytes);

void oracle_hook_constructCoord(MPI_Comm comm_cart, MPI_COORD thisMPICoord, GRID grid, PARAMS params, float *coord,
                                float *cpu_coord, float *terrain, float *cpu_terrain)
{
    constructCoord(comm_cart, thisMPICoord, grid, params, coord, cpu_coord, terrain, cpu_terrain);
    std::string f = oracle_param_string("terrainFile");
    if (!f.empty() && !params.gauss_hill) {
        oracle_read_raw(f, cpu_terrain, (size_t)grid._nx_ * grid._ny_);
        construct_terrain_coord(cpu_coord, cpu_terrain, grid._nx_, grid._ny_, grid._nz_, grid.frontNZ, grid.NZ,
                                params.Depth * 1000);
    }
    /* the padded coordinates [_nz_][_ny_][_nx_][3] and surface [_ny_][_nx_] */
    g_oracle_params = params;
    oracle_dump("oracle_coord.bin", cpu_coord, sizeof(float) * 3 * (size_t)grid._nx_ * grid._ny_ * grid._nz_);
    oracle_dump("oracle_terrain.bin", cpu_terrain, sizeof(float) * (size_t)grid._nx_ * grid._ny_);
}

void oracle_hook_constructMedium(MPI_COORD thisMPICoord, PARAMS params, GRID grid, float *cpu_coord,
                                 float *cpu_terrain, float *medium, float *cpu_medium)
{
    constructMedium(thisMPICoord, params, grid, cpu_coord, cpu_terrain, medium, cpu_medium);
    std::string f = oracle_param_string("mediumFile");
    if (!f.empty()) oracle_read_raw(f, cpu_medium, (size_t)grid._nx_ * grid._ny_ * grid._nz_ * MSIZE);
}

/* ------------------------------------------------------------- dump hooks */
static void oracle_dump(const char *name, const void *data, size_t bytes)
{
    char path[1024];
    snprintf(path, sizeof(path), "%s/%s", g_oracle_params.OUT, name);
    FILE *fp = fopen(path, "wb");
    if (!fp) {
        fprintf(stderr, "oracle: cannot write %s\n", path);
        return;
    }
    fwrite(data, 1, bytes, fp);
    fclose(fp);
}

void oracle_hook_propagate(MPI_Comm comm_cart, MPI_COORD thisMPICoord, MPI_NEIGHBOR mpiNeighbor, GRID grid,
                           PARAMS params, WAVE wave, Mat_rDZ mat_rDZ, FLOAT *CJM, SOURCE_FILE_INPUT src_in,
                           long long *srcIndex, float *momentRate, float *momentRateSlice, SLICE slice,
                           SLICE_DATA sliceData, SLICE_DATA sliceDataCpu)
{
    g_oracle_CJM = CJM;
    g_oracle_grid = grid;
    g_oracle_params = params;
    long long num = (long long)grid._nx_ * grid._ny_ * grid._nz_;
    oracle_dump("oracle_CJM.bin", CJM, sizeof(FLOAT) * CJMSIZE * num);
#ifndef SCFDM
#ifdef FREE_SURFACE
    oracle_dump("oracle_rDZ.bin", mat_rDZ._rDZ_DX, sizeof(float) * 2 * MATSIZE * grid._nx_ * grid._ny_);
#endif
#endif
    /* scalars of the run as propagate() sees them (src/propagate.cpp:86-90) and,
       for the restated oracle, the finite-fault table before its scaling */
    {
        char path[1024];
        snprintf(path, sizeof(path), "%s/oracle_meta.txt", params.OUT);
        FILE *fp = fopen(path, "w");
        if (fp) {
            float DT = params.DT;
            int NT = params.TMAX / DT;
            fprintf(fp, "nx %d\nny %d\nnz %d\nDT %.9g\nDH %.9g\nrDH %.9g\nNT %d\nnPML %d\n", grid.nx, grid.ny,
                    grid.nz, DT, grid.DH, grid.rDH, NT, params.nPML);
            fprintf(fp, "sourceX %d\nsourceY %d\nsourceZ %d\nrickerfc %.9g\nstrike %.9g\ndip %.9g\nrake %.9g\n"
                        "Mw %.9g\nduration %.9g\n",
                    params.sourceX, params.sourceY, params.sourceZ, params.rickerfc, params.strike, params.dip,
                    params.rake, params.Mw, params.duration);
            int kind = params.useMultiSource ? 3 : params.useSingleSource_ricker ? 1
                                                 : params.useSingleSource_double_couple ? 2 : 0;
            fprintf(fp, "src_kind %d\n", kind);
#ifdef SCFDM
            extern float vp_max_for_SCFDM;
            fprintf(fp, "vp_max %.9g\n", vp_max_for_SCFDM);
#endif
            fclose(fp);
        }
        if (params.useMultiSource) {
            long long npts = src_in.npts, nt = src_in.nt;
            float dt = src_in.dt;
            snprintf(path, sizeof(path), "%s/oracle_src.bin", params.OUT);
            fp = fopen(path, "wb");
            if (fp) {
                fwrite(&npts, 8, 1, fp);
                fwrite(&nt, 8, 1, fp);
                fwrite(&dt, 4, 1, fp);
                fwrite(srcIndex, 8, npts, fp);
                fwrite(momentRate, 4, npts * nt * MOMSIZE, fp);
                fclose(fp);
            }
        }
    }
    propagate(comm_cart, thisMPICoord, mpiNeighbor, grid, params, wave, mat_rDZ, CJM, src_in, srcIndex,
              momentRate, momentRateSlice, slice, sliceData, sliceDataCpu);
}

void oracle_hook_freeWave(WAVE wave)
{
    long long num = (long long)g_oracle_grid._nx_ * g_oracle_grid._ny_ * g_oracle_grid._nz_;
    oracle_dump("oracle_final_W.bin", wave.W, sizeof(FLOAT) * WSIZE * num);
    freeWave(wave);
}

#ifdef SOLVE_DISPLACEMENT
/* ---------------------------------------------------- displacement driver */
/* src/solve_displacement.cpp:65-74 launches its kernel with dim3 on the GPU
 * only; on the CPU the kernel body is the loop nest itself. */
void SolveDisplacementKernel(FLOAT *W, FLOAT *Dis, FLOAT *CJM, int _nx_, int _ny_, int _nz_, FLOAT dt);
void SolveDisplacement(GRID grid, FLOAT *W, FLOAT *Dis, FLOAT *CJM, FLOAT dt)
{
    SolveDisplacementKernel(W, Dis, CJM, grid._nx_, grid._ny_, grid._nz_, dt);
}
#endif
