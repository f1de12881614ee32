/*
 * Force-included (g++ -include) into every reference translation unit of the
 * oracle's reference CPU build.  Test infrastructure only.
 *
 * The reference sources compile unmodified for the CPU (no GPU_CUDA) except
 * for a handful of CPU-branch call sites that do not match their callee
 * (src/PGV.cpp:224, src/singleSource.cpp:210,355, src/station.cpp:409,
 * src/addMoment.cpp:355) and two SCFDM kernels whose CPU
 * branch leaves i/j/k undeclared (src/freeSurface.cpp:57-59,
 * src/exp_decay_absorb.cpp:26-30).  This header supplies declarations that
 * let those call sites resolve, without touching the kernel bodies; the
 * matching definitions are in ref_drivers.cpp.
 */
#ifndef ORACLE_REF_FIXUPS_H
#define ORACLE_REF_FIXUPS_H

#include "header.h"

/* contravariant.cpp:122,145,176 call it unconditionally (SCFDM metrics);
 * on the sequential CPU path it has nothing to wait for. */
static inline int cudaDeviceSynchronize(void) { return 0; }

/* PGV.cpp:224 calls compare_pgv with five arguments on the CPU path. */
void compare_pgv(float *pgv, FLOAT *W, int nx, int ny, int nz);

#ifdef SOLVE_PGA
/* defined in the SOLVE_PGA block that the build cuts from propagate.cpp
 * (GPU-only code); ref_drivers.cpp has the CPU copy. */
void storage_W_pre(GRID grid, WAVE wave);
#endif

/* singleSource.cpp:210,355 call an undefined CPU helper. */
void load_smooth_source(SOURCE S, FLOAT *h_W, int _nx_, int _ny_, int _nz_,
                        FLOAT *CJM, int it, int irk, float DT, float DH, int nGauss, float rickerfc);

#ifdef SCFDM
/* addMoment.cpp:355 and station.cpp:409 drop the CJM argument on the CPU path. */
void addSource1(FLOAT *hW, float *momentRateSlice, long long *srcIndex, int npts, float DT);
void storage_station(int stationNum, STATION station, FLOAT *W, int _nx_, int _ny_, int _nz_, int NT, int it);
#endif

#ifdef ORACLE_GLOBAL_IJK
/* freeSurface.cpp:57-59 and exp_decay_absorb.cpp:26-30: CPU loop indices. */
static int i, j, k;
#endif

#ifdef ORACLE_AFLUX_DUMMIES
/* alternative_flux_FD.cpp:1550-1566: the CPU branch of the SCFDM launcher
 * names helpers that do not exist.  The launcher itself is replaced by the
 * one in ref_drivers.cpp; these only let the file compile. */
static inline void cal_flux(...) {}
static inline void wave_deriv_alternative_flux_FD(...) {}
static inline void cal_du(...) {}
#endif

#ifdef ORACLE_GLOBAL_RICKERFC
/* singleSource.cpp:355 names rickerfc where it is not in scope; the oracle
 * replaces that driver (ref_drivers.cpp), so the value is never used. */
static float rickerfc = 0.0f;
#endif

#endif
