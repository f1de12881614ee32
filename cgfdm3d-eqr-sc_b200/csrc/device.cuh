// Device-side layout shared by all kernels.
//
// Fields are stored structure-of-arrays: field f of a set lives at
// base + f * fstride.  Inside a field, point (i, j, k) of the padded grid
// (i in [0, _nx_), 3 halo cells each side) sits at
//     (k * _ny_ + j) * pitch + xoff + i
// and pitch a multiple of 4 floats.  xoff places the first interior column
// i = HALO = 3: at a 16-byte boundary with xoff = 1 (ME-AWENO), at a
// 128-byte line with xoff = 29 (CGFDM: a warp's 32 points then touch four
// sectors, not five, and its stores write whole sectors; 3.7 % faster).
// The reference stores
// the same points array-of-structures, W[idx * 9 + v] (src/axis.h:237); the
// C ABI converts at its boundary.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace cgfdm {

#ifndef CGFDM_HALO
#define CGFDM_HALO 3
#endif

struct DevGrid {
    int nx, ny, nz;           // interior
    int nxp, nyp, nzp;        // padded (_nx_, _ny_, _nz_)
    int pitch;                // floats per row
    int xoff;                 // column of i = 0
    long long plane;          // floats per k-plane (nyp * pitch)
    long long fstride;        // floats per field (>= nzp * plane, 256-byte multiple)

    __host__ __device__ __forceinline__ long long at(int i, int j, int k) const
    {
        return (long long)k * plane + (long long)j * pitch + xoff + i;
    }
    // 2-D surface arrays use the same row pitch: (j * pitch + xoff + i)
    __host__ __device__ __forceinline__ long long at2(int i, int j) const
    {
        return (long long)j * pitch + xoff + i;
    }
};

inline DevGrid make_devgrid(int nx, int ny, int nz, int xoff = 1)
{
    DevGrid d;
    d.nx = nx, d.ny = ny, d.nz = nz;
    d.nxp = nx + 2 * CGFDM_HALO, d.nyp = ny + 2 * CGFDM_HALO, d.nzp = nz + 2 * CGFDM_HALO;
    d.xoff = xoff;
    d.pitch = (d.nxp + d.xoff + 3) / 4 * 4;
    d.plane = (long long)d.nyp * d.pitch;
    long long n = (long long)d.nzp * d.plane;
    d.fstride = (n + 63) / 64 * 64;
    return d;
}

// CJM field numbers (src/CJM.cpp:118-144)
enum CjmField {
    C_XI_X = 0, C_XI_Y, C_XI_Z, C_ET_X, C_ET_Y, C_ET_Z, C_ZT_X, C_ZT_Y, C_ZT_Z,
    C_JAC = 9, C_MU = 10, C_LAMBDA = 11, C_BUOY = 12,
    C_X_XI = 13, C_Y_XI, C_Z_XI, C_X_ET, C_Y_ET, C_Z_ET  // SCFDM only
};

// MacCormack-type one-sided coefficients (src/macro.h:120-131)
#define CG_AF_1 (-0.30874f)
#define CG_AF0 (-0.6326f)
#define CG_AF1 (1.2330f)
#define CG_AF2 (-0.3334f)
#define CG_AF3 (0.04168f)
// two- and three-point one-sided (src/macro.h:144-146)
#define CG_CF1 (-1.16666667f)
#define CG_CF2 (1.33333333f)
#define CG_CF3 (-0.16666667f)
// classic RK4 (src/macro.h:133-142)
#define RK_ALPHA2 0.5f
#define RK_ALPHA3 0.5f
#define RK_BETA1 0.16666667f
#define RK_BETA2 0.33333333f
#define RK_BETA3 0.33333333f
#define RK_BETA4 0.16666667f

#define CUDA_TRY(x)                                                                           \
    do {                                                                                      \
        cudaError_t e_ = (x);                                                                 \
        if (e_ != cudaSuccess) return e_;                                                     \
    } while (0)

}  // namespace cgfdm
