// Per-function entry points with the reference's names and semantics, on
// the reference's own device arrays: wavefield, CJM, PML auxiliaries and
// free-surface matrices array-of-structures in the XFAST layout
// (point (i, j, k) of the padded grid at i + j _nx_ + k _nx_ _ny_, its
// fields consecutive; src/axis.h:73).  A copy of src/propagate.cpp whose
// drivers forward here runs the reference's time loop on this library's
// kernels, one launch per reference launch, in stream order.
//
// These kernels are the drop-in proof, not the fast path: the fused stage
// (cgfdm_stage.cu) does derivative, free surface, PML and RK update in one
// pass over a structure-of-arrays layout.  One thread per point; the
// arithmetic follows the reference expression by expression (the shared
// point operators of cg_ops.cuh), so the "exact" build rounds as the
// reference's CPU build does.
#include "../../include/cgfdm.h"
#include "../../include/cgfdm_shims.h"

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "cg_ops.cuh"
#include "device.cuh"
#include "sc_ops.cuh"
#include "kernels.cuh"
#include "session.hpp"

namespace cgfdm {

#define HALO_ CGFDM_HALO

struct Aos {
    int nx_, ny_, nz_;
    __device__ __forceinline__ long long at(int i, int j, int k) const
    {
        return (long long)i + (long long)j * nx_ + (long long)k * nx_ * ny_;
    }
};

// the five taps of the L operator along one axis: field f of points q + FB*(m-1)
__device__ __forceinline__ float lop_aos(const float *__restrict__ W, long long q, long long step, int f, int FB,
                                         float rDH)
{
    const long long o = (long long)FB * step;
    return lop(W[(q - o) * 9 + f], W[q * 9 + f], W[(q + o) * 9 + f], W[(q + 2 * o) * 9 + f], W[(q + 3 * o) * 9 + f],
               FB, rDH);
}

// ------------------------------------------------ src/wave_deriv.cpp:76-284
__global__ void k_wave_deriv(float *__restrict__ h_W, const float *__restrict__ W, const float *__restrict__ CJM,
                             const float *bx_, const float *by_, const float *bz_, Aos a, float rDH, int FB1,
                             int FB2, int FB3, float DT)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x + HALO_;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + HALO_;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + HALO_;
    if (i >= a.nx_ - HALO_ || j >= a.ny_ - HALO_ || k >= a.nz_ - HALO_) return;
    const long long q = a.at(i, j, k);
    const float *c = CJM + q * 13;
    const float bx = bx_ ? bx_[i] : 1.0f, by = by_ ? by_[j] : 1.0f, bz = bz_ ? bz_[k] : 1.0f;
    const float mu = c[C_MU], lam = c[C_LAMBDA], buo = c[C_BUOY] * 1.0f;  // buoyancy *= Crho (= 1)
    const long long sy = a.nx_, sz = (long long)a.nx_ * a.ny_;
    float d[9], r[9], h[9];
    for (int f = 0; f < 9; f++) d[f] = lop_aos(W, q, 1, f, FB1, rDH) * bx;
    dir_rhs(c[C_XI_X], c[C_XI_Y], c[C_XI_Z], d, mu, lam, buo, r);
    for (int f = 0; f < 9; f++) h[f] = r[f];
    for (int f = 0; f < 9; f++) d[f] = lop_aos(W, q, sy, f, FB2, rDH) * by;
    dir_rhs(c[C_ET_X], c[C_ET_Y], c[C_ET_Z], d, mu, lam, buo, r);
    for (int f = 0; f < 9; f++) h[f] = h[f] + r[f];
    for (int f = 0; f < 9; f++) d[f] = lop_aos(W, q, sz, f, FB3, rDH) * bz;
    dir_rhs(c[C_ZT_X], c[C_ZT_Y], c[C_ZT_Z], d, mu, lam, buo, r);
    for (int f = 0; f < 9; f++) h_W[q * 9 + f] = (h[f] + r[f]) * DT;
}

// J (metric row . traction) at point p (src/freeSurface.cpp:358-380)
__device__ __forceinline__ void jt_aos(const float *__restrict__ W, const float *__restrict__ CJM, long long p,
                                       int mdir, float out[3])
{
    const float *c = CJM + p * 13 + 3 * mdir;
    const float m0 = c[0], m1 = c[1], m2 = c[2], jac = CJM[p * 13 + C_JAC];
    const float *w = W + p * 9;
    out[0] = ((m0 * w[3] + m1 * w[6]) + m2 * w[7]) * jac;
    out[1] = ((m0 * w[6] + m1 * w[4]) + m2 * w[8]) * jac;
    out[2] = ((m0 * w[7] + m1 * w[8]) + m2 * w[5]) * jac;
}

// ---------------------------------------------- src/freeSurface.cpp:242-492
__global__ void k_free_surface_deriv(float *__restrict__ h_W, const float *__restrict__ W,
                                     const float *__restrict__ CJM, const float *__restrict__ DX,
                                     const float *__restrict__ DY, const float *bx_, const float *by_, Aos a,
                                     float rDH, int FB1, int FB2, int FB3, float DT)
{
    const int _nz = a.nz_ - HALO_;
    const int i = blockIdx.x * blockDim.x + threadIdx.x + HALO_;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + HALO_;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + _nz - HALO_;
    if (i >= a.nx_ - HALO_ || j >= a.ny_ - HALO_ || k >= _nz) return;
    const long long q = a.at(i, j, k);
    const float *c = CJM + q * 13;
    const float mu = c[C_MU], lam = c[C_LAMBDA], buo = c[C_BUOY] * 1.0f;
    const float bx = bx_ ? bx_[i] : 1.0f, by = by_ ? by_[j] : 1.0f;
    const long long sy = a.nx_, sz = (long long)a.nx_ * a.ny_;
    const int ks = (_nz - 1) - k + HALO_;   // relative index of the surface
    // J.T at the five taps along each axis; along z the antisymmetric image
    float Jx[5][3], Jy[5][3], Jz[5][3];
    for (int m = 0; m < 5; m++) {
        jt_aos(W, CJM, q + (long long)(m - 1) * FB1, 0, Jx[m]);
        jt_aos(W, CJM, q + (long long)(m - 1) * FB2 * sy, 1, Jy[m]);
        const int l = 3 + (m - 1) * FB3;
        int src = l;
        float sign = 1.0f;
        if (l > ks) src = 2 * ks - l, sign = -1.0f;
        if (src == ks) {
            Jz[m][0] = Jz[m][1] = Jz[m][2] = 0.0f;
        } else {
            jt_aos(W, CJM, q + (long long)(src - 3) * sz, 2, Jz[m]);
            if (sign < 0.0f) Jz[m][0] = -Jz[m][0], Jz[m][1] = -Jz[m][1], Jz[m][2] = -Jz[m][2];
        }
    }
    const float bj = buo * (1.0f / c[C_JAC]);
    float h[9];
    for (int v = 0; v < 3; v++) {
        const float lx = lop(Jx[0][v], Jx[1][v], Jx[2][v], Jx[3][v], Jx[4][v], FB1, rDH);
        const float ly = lop(Jy[0][v], Jy[1][v], Jy[2][v], Jy[3][v], Jy[4][v], FB2, rDH);
        const float lz = lop(Jz[0][v], Jz[1][v], Jz[2][v], Jz[3][v], Jz[4][v], FB3, rDH);
        h[v] = bj * ((lx * bx + ly * by) + lz);
    }
    float vxi[3], vet[3], vzt[3];
    for (int v = 0; v < 3; v++) vxi[v] = lop_aos(W, q, 1, v, FB1, rDH) * bx;
    for (int v = 0; v < 3; v++) vet[v] = lop_aos(W, q, sy, v, FB2, rDH) * by;
    if (k == _nz - 1) {
        const long long s = (long long)i + (long long)j * a.nx_;
        for (int r = 0; r < 3; r++) {
            const float *dx = DX + s * 9 + r * 3, *dy = DY + s * 9 + r * 3;
            vzt[r] = ((dx[0] * vxi[0] + dx[1] * vxi[1]) + dx[2] * vxi[2]) +
                     ((dy[0] * vet[0] + dy[1] * vet[1]) + dy[2] * vet[2]);
        }
    } else if (k == _nz - 2) {
        for (int v = 0; v < 3; v++) vzt[v] = ((float)FB3 * (W[(q + FB3 * sz) * 9 + v] - W[q * 9 + v])) * rDH;
    } else {
        for (int v = 0; v < 3; v++)
            vzt[v] = ((float)FB3 * ((CG_CF1 * W[q * 9 + v] + CG_CF2 * W[(q + FB3 * sz) * 9 + v]) +
                                    CG_CF3 * W[(q + 2 * FB3 * sz) * 9 + v])) *
                     rDH;
    }
    float s1[9], s2[9], s3[9];
    dir_stress(c[C_XI_X], c[C_XI_Y], c[C_XI_Z], vxi, mu, lam, s1);
    dir_stress(c[C_ET_X], c[C_ET_Y], c[C_ET_Z], vet, mu, lam, s2);
    dir_stress(c[C_ZT_X], c[C_ZT_Y], c[C_ZT_Z], vzt, mu, lam, s3);
    for (int f = 3; f < 9; f++) h[f] = (s1[f] + s2[f]) + s3[f];
    for (int f = 0; f < 9; f++) h_W[q * 9 + f] = h[f] * DT;
}

// ------------------------------------------------ src/pml_deriv.cpp:125-566
// One face: dir 0 x, 1 y, 2 z; far = the face at the high end (FLAG 1).
__global__ void k_pml_deriv(float *__restrict__ h_W, const float *__restrict__ W, float *__restrict__ h_Aux,
                            const float *__restrict__ Aux, const float *__restrict__ CJM,
                            const float *__restrict__ alpha, const float *__restrict__ beta,
                            const float *__restrict__ dd, Aos a, int nPML, int dir, int far, float rDH, int FB,
                            float DT)
{
    const int nx = a.nx_ - 2 * HALO_, ny = a.ny_ - 2 * HALO_, nz = a.nz_ - 2 * HALO_;
    const int n0 = dir == 0 ? nPML : nx, n1 = dir == 1 ? nPML : ny, n2 = dir == 2 ? nPML : nz;
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
    const int j0 = blockIdx.y * blockDim.y + threadIdx.y;
    const int k0 = blockIdx.z * blockDim.z + threadIdx.z;
    if (i0 >= n0 || j0 >= n1 || k0 >= n2) return;
    const int i = i0 + HALO_ + (dir == 0 && far ? nx - nPML : 0);
    const int j = j0 + HALO_ + (dir == 1 && far ? ny - nPML : 0);
    const int k = k0 + HALO_ + (dir == 2 && far ? nz - nPML : 0);
    const long long q = a.at(i, j, k);
    const long long pos = (long long)i0 + (long long)j0 * n0 + (long long)k0 * n0 * n1;
    const float *c = CJM + q * 13;
    const float mu = c[C_MU], lam = c[C_LAMBDA], buo = c[C_BUOY] * 1.0f;
    const int ix = dir == 0 ? i : dir == 1 ? j : k;
    const float b = beta[ix], dv = dd[ix], alpha_d = dv + alpha[ix];
    const long long step = dir == 0 ? 1 : dir == 1 ? (long long)a.nx_ : (long long)a.nx_ * a.ny_;
    float d[9], r[9];
    for (int f = 0; f < 9; f++) d[f] = lop_aos(W, q, step, f, FB, rDH) * dv;
    dir_rhs(c[3 * dir + 0], c[3 * dir + 1], c[3 * dir + 2], d, mu, lam, buo, r);
    for (int f = 0; f < 9; f++) h_Aux[pos * 9 + f] = (r[f] - alpha_d * Aux[pos * 9 + f]) * DT;
    for (int f = 0; f < 9; f++) h_W[q * 9 + f] = h_W[q * 9 + f] + (-b * Aux[pos * 9 + f]) * DT;
}

// ------------------------------------------- src/pml_freeSurface.cpp:16-242
__global__ void k_pml_free_surface(float *__restrict__ h_Aux, const float *__restrict__ W,
                                   const float *__restrict__ CJM, const float *__restrict__ D,
                                   const float *__restrict__ dd, Aos a, int nPML, int dir, int far, float rDH,
                                   int FB, float DT)
{
    const int nx = a.nx_ - 2 * HALO_, ny = a.ny_ - 2 * HALO_, nz = a.nz_ - 2 * HALO_;
    const int n0 = dir == 0 ? nPML : nx, n1 = dir == 1 ? nPML : ny;
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
    const int j0 = blockIdx.y * blockDim.y + threadIdx.y;
    if (i0 >= n0 || j0 >= n1) return;
    const int k0 = nz - 1;
    const int i = i0 + HALO_ + (dir == 0 && far ? nx - nPML : 0);
    const int j = j0 + HALO_ + (dir == 1 && far ? ny - nPML : 0);
    const int k = k0 + HALO_;
    const long long q = a.at(i, j, k);
    const long long s = (long long)i + (long long)j * a.nx_;
    const long long pos = (long long)i0 + (long long)j0 * n0 + (long long)k0 * n0 * n1;
    const float *c = CJM + q * 13;
    const float mu = c[C_MU], lam = c[C_LAMBDA];
    const float dv = dd[dir == 0 ? i : j];
    const long long step = dir == 0 ? 1 : (long long)a.nx_;
    float v[3], vz[3], t3[9];
    for (int f = 0; f < 3; f++) v[f] = lop_aos(W, q, step, f, FB, rDH) * dv;
    for (int r = 0; r < 3; r++) {
        const float *m = D + s * 9 + r * 3;
        vz[r] = (m[0] * v[0] + m[1] * v[1]) + m[2] * v[2];
    }
    dir_stress(c[C_ZT_X], c[C_ZT_Y], c[C_ZT_Z], vz, mu, lam, t3);
    for (int f = 3; f < 9; f++) h_Aux[pos * 9 + f] = h_Aux[pos * 9 + f] + t3[f] * DT;
}

// -------------------------------------------- src/wave_rk.cpp, src/pml_rk.cpp
__global__ void k_rk(float *__restrict__ h_W, float *__restrict__ W, float *__restrict__ t_W, float *__restrict__ m_W,
                     long long n, int irk)
{
    const long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= n) return;
    const float h = h_W[x];
    if (irk == 0) {
        const float m = W[x];
        m_W[x] = m;
        t_W[x] = m + RK_BETA1 * h;
        W[x] = m + RK_ALPHA2 * h;
    } else if (irk == 1) {
        t_W[x] = t_W[x] + RK_BETA2 * h;
        W[x] = m_W[x] + RK_ALPHA3 * h;
    } else if (irk == 2) {
        t_W[x] = t_W[x] + RK_BETA3 * h;
        W[x] = m_W[x] + h;
    } else {
        W[x] = t_W[x] + RK_BETA4 * h;
    }
}

// ------------------------------------------------- src/addMoment.cpp:25-223
__global__ void k_calc_moment_rate(long long npts, long long nt, const float *__restrict__ CJM, int nfield,
                                   float *rate, const long long *__restrict__ idx, float DH)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long t = (long long)blockIdx.y * blockDim.y + threadIdx.y;
    if (i >= npts || t >= nt) return;
    const long long q = idx[i];
    const float jac = CJM[q * nfield + C_JAC], mu = CJM[q * nfield + C_MU];
    float V = jac * DH * DH * DH;
    V = (float)(1.0 / (double)V);
    V = V * 1.0f;   // * Cv (= 1)
    float *r = rate + (i + t * npts) * 6;
    for (int c = 0; c < 6; c++) r[c] = r[c] * (mu * V);
}

__global__ void k_add_moment(float *__restrict__ W, const long long *__restrict__ idx, const float *__restrict__ rate,
                             float *__restrict__ slice, long long npts, int srcIt, float t_weight, float DT,
                             const float *__restrict__ CJM, int nfield, int scfdm)
{
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= npts) return;
    const float *r0 = rate + ((long long)srcIt * npts + i) * 6, *r1 = rate + ((long long)(srcIt + 1) * npts + i) * 6;
    float m[6];
    for (int c = 0; c < 6; c++) {
        m[c] = (r1[c] - r0[c]) * t_weight + r0[c];
        slice[i * 6 + c] = m[c];
    }
    const long long q = idx[i];
    float *w = W + q * 9;
    if (!scfdm) {
        for (int c = 0; c < 6; c++) w[3 + c] = w[3 + c] - m[c] * DT;
        return;
    }
    // stress rate to strain rate (src/addMoment.cpp:205-220)
    const float mu = CJM[q * nfield + C_MU], lam = CJM[q * nfield + C_LAMBDA];
    const float den = 2 * (mu * mu) + 3 * lam * mu;
    float e[6];
    e[0] = (m[0] * (lam + mu)) / den - (lam * m[1]) / (2 * den) - (lam * m[2]) / (2 * den);
    e[1] = (m[1] * (lam + mu)) / den - (lam * m[0]) / (2 * den) - (lam * m[2]) / (2 * den);
    e[2] = (m[2] * (lam + mu)) / den - (lam * m[0]) / (2 * den) - (lam * m[1]) / (2 * den);
    e[3] = m[5] / (mu);
    e[4] = m[4] / (mu);
    e[5] = m[3] / (mu);
    for (int c = 0; c < 6; c++) w[3 + c] = w[3 + c] - e[c] * DT;
}

// ---------------------------------------------------- src/station.cpp:302-380
__global__ void k_storage_station(int n, const int *__restrict__ XYZ, float *__restrict__ wave,
                                  const float *__restrict__ W, const float *__restrict__ CJM, int nfield, Aos a,
                                  int NT, int it, int scfdm)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n) return;
    const long long q = a.at(XYZ[s * 3 + 0], XYZ[s * 3 + 1], XYZ[s * 3 + 2]);
    float *out = wave + ((long long)it + (long long)s * NT) * 9;
    const float *u = W + q * 9;
    if (!scfdm) {
        const float C1 = (float)(1.0 / 1.0), C2 = (float)(1.0 / 1.0);   // 1 / Cv, 1 / Cs
        for (int f = 0; f < 3; f++) out[f] = u[f] * C1;
        for (int f = 3; f < 9; f++) out[f] = u[f] * C2;
        return;
    }
    // conserved to physical (src/station.cpp:336-365)
    const float mu = CJM[q * nfield + C_MU], lam = CJM[q * nfield + C_LAMBDA], buo = CJM[q * nfield + C_BUOY] * 1.0f;
    out[3] = lam * u[4] + lam * u[5] + u[3] * (lam + 2 * mu);
    out[4] = lam * u[3] + lam * u[5] + u[4] * (lam + 2 * mu);
    out[5] = lam * u[3] + lam * u[4] + u[5] * (lam + 2 * mu);
    out[6] = mu * u[8];
    out[7] = mu * u[7];
    out[8] = mu * u[6];
    out[0] = u[0] * buo;
    out[1] = u[1] * buo;
    out[2] = u[2] * buo;
}

// ------------------------------------------------------ src/PGV.cpp:61-171
__global__ void k_compare_pgv(float *__restrict__ pgv, const float *__restrict__ W, const float *__restrict__ W_pre,
                              const float *__restrict__ CJM, int nfield, Aos a, float DT, int it, int scfdm)
{
    const int nx = a.nx_ - 2 * HALO_, ny = a.ny_ - 2 * HALO_;
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x, j0 = blockIdx.y * blockDim.y + threadIdx.y;
    if (i0 >= nx || j0 >= ny) return;
    const long long q = a.at(i0 + HALO_, j0 + HALO_, a.nz_ - HALO_ - 1);
    const long long pos = (long long)i0 + (long long)j0 * nx;
    const int rec = W_pre ? 4 : 2;
    const double cv = 1.0 / 1.0;   // 1 / Cv
    const float buo = scfdm ? CJM[q * nfield + C_BUOY] * 1.0f : 1.0f;
    float Vx, Vy, Vz;
    if (scfdm) {
        Vx = (float)((double)W[q * 9 + 0] * cv * (double)buo);
        Vy = (float)((double)W[q * 9 + 1] * cv * (double)buo);
        Vz = (float)((double)W[q * 9 + 2] * cv * (double)buo);
    } else {
        Vx = (float)((double)W[q * 9 + 0] * cv);
        Vy = (float)((double)W[q * 9 + 1] * cv);
        Vz = (float)((double)W[q * 9 + 2] * cv);
    }
    const float Vh = sqrtf(Vx * Vx + Vy * Vy), V = sqrtf(Vx * Vx + Vy * Vy + Vz * Vz);
    if (pgv[pos * rec + 0] < Vh) pgv[pos * rec + 0] = Vh;
    if (pgv[pos * rec + 1] < V) pgv[pos * rec + 1] = V;
    if (W_pre && it % 10 == 0) {
        float px, py, pz;
        if (scfdm) {
            px = (float)((double)W_pre[q * 9 + 0] * cv * (double)buo);
            py = (float)((double)W_pre[q * 9 + 1] * cv * (double)buo);
            pz = (float)((double)W_pre[q * 9 + 2] * cv * (double)buo);
        } else {
            px = (float)((double)W_pre[q * 9 + 0] * cv);
            py = (float)((double)W_pre[q * 9 + 1] * cv);
            pz = (float)((double)W_pre[q * 9 + 2] * cv);
        }
        const float den = 10 * DT;
        const float Ax = (Vx - px) / den, Ay = (Vy - py) / den, Az = (Vz - pz) / den;
        const float Ah = sqrtf(Ax * Ax + Ay * Ay), A = sqrtf(Ax * Ax + Ay * Ay + Az * Az);
        if (pgv[pos * rec + 2] < Ah) pgv[pos * rec + 2] = Ah;
        if (pgv[pos * rec + 3] < A) pgv[pos * rec + 3] = A;
    }
}

// -------------------------------------------- src/solve_displacement.cpp:25-57
__global__ void k_solve_displacement(const float *__restrict__ W, float *__restrict__ Dis,
                                     const float *__restrict__ CJM, int nfield, long long n, float dt, int scfdm)
{
    const long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n) return;
    const float buo = scfdm ? CJM[q * nfield + C_BUOY] : 1.0f;
    for (int c = 0; c < 3; c++) {
        const float v = scfdm ? W[q * 9 + c] * buo : W[q * 9 + c];
        Dis[q * 3 + c] = Dis[q * 3 + c] + v * dt;
    }
}

// ------------------------------------------------ src/propagate.cpp:26-58
__global__ void k_copy_prefix(float *__restrict__ dst, const float *__restrict__ src, long long n)
{
    const long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (x < n) dst[x] = src[x];
}

// --------------------------------------------- src/singleSource.cpp:111-330
// One 7 x 7 x 7 Gaussian-smoothed point source at the padded point (X, Y,
// Z): kind 1 explosive Ricker (value on the normal stresses), kind 2 double
// couple (moment-rate tensor on the six stresses); SCFDM converts to
// strain rates with the medium of each point.
struct PointArgs {
    float amp[343];
    float mom[6];
    float s, m0;
    int X, Y, Z, kind;
};

__global__ void k_point_source(float *__restrict__ W, const float *__restrict__ CJM, int nfield, Aos a,
                               const PointArgs p, float DT, float DH, int scfdm)
{
    const int t = threadIdx.x;
    if (t >= 343) return;
    const int i = p.X + t % 7 - 3, j = p.Y + (t / 7) % 7 - 3, k = p.Z + t / 49 - 3;
    const long long q = a.at(i, j, k);
    const float jacb = CJM[a.at(p.X, p.Y, p.Z) * nfield + C_JAC];
    const float vol = jacb * (DH * DH * DH);
    float *w = W + q * 9;
    if (p.kind == 1) {
        float value = -1.0f * p.s * p.amp[t] / vol;
        value = (float)((double)value * (1.0 * (double)DT));   // value *= Cs * DT
        if (scfdm) value = value / (3 * CJM[q * nfield + C_LAMBDA] + 2 * CJM[q * nfield + C_MU]);
        for (int c = 0; c < 3; c++) w[3 + c] = w[3 + c] + value;
        return;
    }
    float rate = -1.0f * p.s * p.amp[t] / vol * p.m0;
    rate = (float)((double)rate * (1.0 * (double)DT));
    float mr[6];
    for (int c = 0; c < 6; c++) mr[c] = p.mom[c] * rate;
    if (scfdm) {
        const float mu = CJM[q * nfield + C_MU], lam = CJM[q * nfield + C_LAMBDA];
        const float den = 2 * (mu * mu) + 3 * lam * mu;
        float e[6];
        e[0] = (mr[0] * (lam + mu)) / den - (lam * mr[1]) / (2 * den) - (lam * mr[2]) / (2 * den);
        e[1] = (mr[1] * (lam + mu)) / den - (lam * mr[0]) / (2 * den) - (lam * mr[2]) / (2 * den);
        e[2] = (mr[2] * (lam + mu)) / den - (lam * mr[0]) / (2 * den) - (lam * mr[1]) / (2 * den);
        e[3] = mr[5] / mu;
        e[4] = mr[4] / mu;
        e[5] = mr[3] / mu;
        for (int c = 0; c < 6; c++) mr[c] = e[c];
    }
    for (int c = 0; c < 6; c++) w[3 + c] = w[3 + c] - mr[c];
}

// ====================================================== ME-AWENO (SCFDM)
// CJM has 19 fields per point here (src/macro.h:56-60).
#define SC_NF 19

// --------------------------------- src/alternative_flux_FD.cpp:61-399 (LF)
// Lax-Friedrichs flux of the face between the points q and q + step, stored
// at q; along DIR the faces from index HALO - 1, across it the interior.
__global__ void k_sc_flux(float *__restrict__ RF, const float *__restrict__ W, const float *__restrict__ CJM, Aos a,
                          int dir, float alpha)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x + HALO_ - (dir == 0);
    const int j = blockIdx.y * blockDim.y + threadIdx.y + HALO_ - (dir == 1);
    const int k = blockIdx.z * blockDim.z + threadIdx.z + HALO_ - (dir == 2);
    if (i >= a.nx_ - HALO_ || j >= a.ny_ - HALO_ || k >= a.nz_ - HALO_) return;
    const long long q = a.at(i, j, k);
    const long long s = dir == 0 ? 1 : dir == 1 ? (long long)a.nx_ : (long long)a.nx_ * a.ny_;
    const float *c = CJM + q * SC_NF;
    float uL[9], uR[9], F[9];
    for (int v = 0; v < 9; v++) {
        const float w_2 = W[(q - 2 * s) * 9 + v], w_1 = W[(q - s) * 9 + v], w0 = W[q * 9 + v];
        const float w1 = W[(q + s) * 9 + v], w2 = W[(q + 2 * s) * 9 + v], w3 = W[(q + 3 * s) * 9 + v];
        uL[v] = weno5_ref(w_2, w_1, w0, w1, w2);
        uR[v] = weno5_ref(w3, w2, w1, w0, w_1);
    }
    lf_flux_ref(c[3 * dir + 0], c[3 * dir + 1], c[3 * dir + 2], c[C_LAMBDA], c[C_MU], c[C_BUOY], alpha, uL, uR, F);
    for (int v = 0; v < 9; v++) RF[q * 9 + v] = F[v];
}

// ---------------------------------- src/alternative_flux_FD.cpp:1215-1435
// Flux difference of the interior points along DIR: h_W = (x) or += (y, z)
// DT rDH / J times the corrected difference; in the top three layers the
// corrections come from point fluxes (the surface variant).
__global__ void k_sc_du(float *__restrict__ h_W, const float *__restrict__ RF, const float *__restrict__ W,
                        const float *__restrict__ CJM, Aos a, int dir, float rDH, float DT)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x + HALO_;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + HALO_;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + HALO_;
    const int _nz = a.nz_ - HALO_;
    if (i >= a.nx_ - HALO_ || j >= a.ny_ - HALO_ || k >= _nz) return;
    const long long q = a.at(i, j, k);
    const long long s = dir == 0 ? 1 : dir == 1 ? (long long)a.nx_ : (long long)a.nx_ * a.ny_;
    const float jac = (float)(1.0 / (double)CJM[q * SC_NF + C_JAC]);
    const float coef = DT * rDH * jac;
    float val[9];
    if (k >= _nz - 3) {
        float hu[7][9];
        for (int n = 0; n < 7; n++) {
            const long long qn = q + (n - 3) * s;
            const float *c = CJM + qn * SC_NF;
            point_flux(c[3 * dir + 0], c[3 * dir + 1], c[3 * dir + 2], c[C_LAMBDA], c[C_MU], c[C_BUOY], W + qn * 9,
                       hu[n]);
        }
        auto o2 = [&](int b, int v) {   // -5 u1 + 39 u2 - 34 u3 - 34 u4 + 39 u5 - 5 u6
            return ((((-5.0f * hu[b][v] + 39.0f * hu[b + 1][v]) - 34.0f * hu[b + 2][v]) - 34.0f * hu[b + 3][v]) +
                    39.0f * hu[b + 4][v]) -
                   5.0f * hu[b + 5][v];
        };
        auto o4 = [&](int b, int v) {   // u1 - 3 u2 + 2 u3 + 2 u4 - 3 u5 + u6
            return ((((hu[b][v] - 3.0f * hu[b + 1][v]) + 2.0f * hu[b + 2][v]) + 2.0f * hu[b + 3][v]) -
                    3.0f * hu[b + 4][v]) +
                   hu[b + 5][v];
        };
        const float c24 = 1.0f / 24, c7 = 7.0f / 5760;
        for (int v = 0; v < 9; v++) {
            const float A = RF[q * 9 + v] - c24 * ((1.0f / 48) * o2(1, v)) + c7 * ((1.0f / 2) * o4(1, v));
            const float B = RF[(q - s) * 9 + v] - c24 * ((1.0f / 48) * o2(0, v)) + c7 * ((1.0f / 2) * o4(0, v));
            val[v] = coef * (-(A - B));
        }
    } else {
        for (int v = 0; v < 9; v++) {
            float f[6];
            for (int m = 0; m < 6; m++) f[m] = RF[(q + (m - 3) * s) * 9 + v];
            val[v] = interior_diff_ref(f, coef);
        }
    }
    for (int v = 0; v < 9; v++) h_W[q * 9 + v] = dir == 0 ? val[v] : h_W[q * 9 + v] + val[v];
}

// ------------------------------------------------ src/wave_rk_tvd.cpp:17-78
__global__ void k_tvd(const float *__restrict__ h_W, float *__restrict__ W, float *__restrict__ m_W, long long n,
                      int irk)
{
    const long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= n) return;
    const float h = h_W[x], w = W[x];
    if (irk == 0) {
        m_W[x] = w;
        W[x] = w + h;
    } else if (irk == 1) {
        const double m = m_W[x];
        W[x] = __double2float_rn(
            __dadd_rn(__dadd_rn(__dmul_rn(0.75, m), __dmul_rn(0.25, (double)w)), __dmul_rn(0.25, (double)h)));
    } else {
        const double m = m_W[x];
        W[x] = __double2float_rn(__dadd_rn(__dadd_rn(__dmul_rn(1.0 / 3.0, m), __dmul_rn(2.0 / 3.0, (double)w)),
                                           __dmul_rn(2.0 / 3.0, (double)h)));
    }
}

// ------------------------------------------------ src/freeSurface.cpp:40-194
__global__ void k_char_free_surface(float *__restrict__ W, const float *__restrict__ CJM, Aos a)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x + HALO_;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + HALO_;
    const int _nz = a.nz_ - HALO_;
    if (i >= a.nx_ - HALO_ || j >= a.ny_ - HALO_) return;
    const long long q = a.at(i, j, _nz - 1);
    const float *c = CJM + q * SC_NF;
    float u[9], o[9];
    for (int v = 0; v < 9; v++) u[v] = W[q * 9 + v];
    const float nrm[3] = {c[C_ZT_X], c[C_ZT_Y], c[C_ZT_Z]};
    const float t1[3] = {c[C_X_XI], c[C_Y_XI], c[C_Z_XI]}, t2[3] = {c[C_X_ET], c[C_Y_ET], c[C_Z_ET]};
    char_surface_point(u, c[C_MU], c[C_LAMBDA], c[C_BUOY], c[C_JAC], nrm, t1, t2, o);
    for (int v = 0; v < 9; v++) W[q * 9 + v] = o[v];
    // cubic extrapolation into the halo above: 4 k1 - 6 k2 + 4 k3 - k4
    const long long P = (long long)a.nx_ * a.ny_;
    for (int v = 0; v < 9; v++)
        for (int h = 1; h <= HALO_; h++) {
            const float *b = W + (q + (h - 1) * P) * 9 + v;
            W[(q + h * P) * 9 + v] = 4.0f * b[0] - 6.0f * b[-P * 9] + 4.0f * b[-2 * P * 9] - b[-3 * P * 9];
        }
}

// --------------------------------------------- src/exp_decay_absorb.cpp:19-106
struct DecayTable {
    float G[21];
};

__global__ void k_exp_decay(float *__restrict__ W, Aos a, DecayTable t, int nl, int free_surface)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x + HALO_;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + HALO_;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + HALO_;
    if (i >= a.nx_ - HALO_ || j >= a.ny_ - HALO_ || k >= a.nz_ - HALO_) return;
    const int X = i - HALO_, Y = j - HALO_, Z = k - HALO_;
    const int nx = a.nx_ - 2 * HALO_, ny = a.ny_ - 2 * HALO_, nz = a.nz_ - 2 * HALO_;
    float *w = W + a.at(i, j, k) * 9;
    float G[6];
    int ng = 0;
    if (X <= nl) G[ng++] = t.G[nl - X];
    if (X >= nx - nl) G[ng++] = t.G[nl - (nx - X)];
    if (Y <= nl) G[ng++] = t.G[nl - Y];
    if (Y >= ny - nl) G[ng++] = t.G[nl - (ny - Y)];
    if (Z <= nl) G[ng++] = t.G[nl - Z];
    if (!free_surface && Z >= nz - nl) G[ng++] = t.G[nl - (nz - Z)];
    for (int g = 0; g < ng; g++)
        for (int v = 0; v < 9; v++) w[v] = w[v] * G[g];
}

// ------------------------------------------------------------ model arrays
// The session's arrays in the reference's layouts, for callers that drive
// the entry points above themselves.
int Session::get_array(const char *name, void *out, long long *bytes)
{
    const Grid &G = m.g;
    const std::string n = name ? name : "";
    const long long plane2 = (long long)G._nx_ * G._ny_;
    auto give = [&](const void *src, long long nb) -> int {
        if (bytes && !out) {
            *bytes = nb;
            return ST_OK;
        }
        if (bytes && *bytes < nb) {
            err = "output buffer too small for " + n;
            return ST_ARG;
        }
        if (nb) std::memcpy(out, src, (size_t)nb);
        if (bytes) *bytes = nb;
        return ST_OK;
    };
    if (n == "rDZ_DX" || n == "rDZ_DY") {
        if (m.p.scheme != SCHEME_CGFDM || !rdz_) {
            err = "no free-surface matrices in this session";
            return ST_STATE;
        }
        std::vector<float> planes((size_t)18 * g.plane), aos((size_t)plane2 * 9);
        if (cudaMemcpyAsync(planes.data(), rdz_, sizeof(float) * planes.size(), cudaMemcpyDeviceToHost, stream) !=
                cudaSuccess ||
            cudaStreamSynchronize(stream) != cudaSuccess)
            return ST_CUDA;
        const int o = n == "rDZ_DX" ? 0 : 9;
        for (int j = 0; j < G._ny_; j++)
            for (int i = 0; i < G._nx_; i++)
                for (int r = 0; r < 9; r++)
                    aos[((size_t)i + (size_t)j * G._nx_) * 9 + r] = planes[(size_t)(o + r) * g.plane + g.at2(i, j)];
        return give(aos.data(), (long long)aos.size() * 4);
    }
    static const char *pml_names[9] = {"pml_alpha_x", "pml_beta_x", "pml_d_x", "pml_alpha_y", "pml_beta_y",
                                       "pml_d_y",     "pml_alpha_z", "pml_beta_z", "pml_d_z"};
    const std::vector<float> *pml[9] = {&m.pml_alpha_x, &m.pml_beta_x, &m.pml_d_x, &m.pml_alpha_y, &m.pml_beta_y,
                                        &m.pml_d_y,     &m.pml_alpha_z, &m.pml_beta_z, &m.pml_d_z};
    for (int c = 0; c < 9; c++)
        if (n == pml_names[c]) return give(pml[c]->data(), (long long)pml[c]->size() * 4);
    if (n == "srcIndex") return give(m.fault.index.data(), (long long)m.fault.index.size() * 8);
    if (n == "momentRate") return give(m.fault.rate.data(), (long long)m.fault.rate.size() * 4);
    if (n == "stationXYZ") return give(m.stations.data(), (long long)m.stations.size() * 4);
    err = "unknown array name: " + n;
    return ST_ARG;
}

}  // namespace cgfdm

// ================================================================ C ABI
using namespace cgfdm;

namespace {
thread_local std::string g_shim_error;

int fail(const std::string &e, int code)
{
    g_shim_error = e;
    return code;
}

int launched(const char *what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return fail(std::string(what) + ": " + cudaGetErrorString(e), ST_CUDA);
    return ST_OK;
}

unsigned blocks_for(long long n, int t) { return (unsigned)((n + t - 1) / t); }

bool grid_ok(int nx_, int ny_, int nz_) { return nx_ > 2 * HALO_ && ny_ > 2 * HALO_ && nz_ > 2 * HALO_; }

bool fb_ok(int fb) { return fb == 1 || fb == -1; }
}  // namespace

extern "C" {

const char *cgfdm_shim_last_error(void) { return g_shim_error.c_str(); }

int cgfdm_waveDeriv(int _nx_, int _ny_, int _nz_, float rDH, float *h_W, const float *W, const float *CJM,
                    const float *pml_beta_x, const float *pml_beta_y, const float *pml_beta_z, int FB1, int FB2,
                    int FB3, float DT, void *stream)
{
    if (!h_W || !W || !CJM || !grid_ok(_nx_, _ny_, _nz_) || !fb_ok(FB1) || !fb_ok(FB2) || !fb_ok(FB3))
        return fail("cgfdm_waveDeriv: bad argument", ST_ARG);
    const dim3 t(32, 4, 4);
    const dim3 b(blocks_for(_nx_ - 2 * HALO_, 32), blocks_for(_ny_ - 2 * HALO_, 4), blocks_for(_nz_ - 2 * HALO_, 4));
    k_wave_deriv<<<b, t, 0, (cudaStream_t)stream>>>(h_W, W, CJM, pml_beta_x, pml_beta_y, pml_beta_z,
                                                    Aos{_nx_, _ny_, _nz_}, rDH, FB1, FB2, FB3, DT);
    return launched("cgfdm_waveDeriv");
}

int cgfdm_freeSurfaceDeriv(int _nx_, int _ny_, int _nz_, float rDH, float *h_W, const float *W, const float *CJM,
                           const float *rDZ_DX, const float *rDZ_DY, const float *pml_beta_x, const float *pml_beta_y,
                           int FB1, int FB2, int FB3, float DT, void *stream)
{
    if (!h_W || !W || !CJM || !rDZ_DX || !rDZ_DY || !grid_ok(_nx_, _ny_, _nz_) || _nz_ < 4 * HALO_ ||
        !fb_ok(FB1) || !fb_ok(FB2) || !fb_ok(FB3))
        return fail("cgfdm_freeSurfaceDeriv: bad argument", ST_ARG);
    const dim3 t(32, 4, 1);
    const dim3 b(blocks_for(_nx_ - 2 * HALO_, 32), blocks_for(_ny_ - 2 * HALO_, 4), HALO_);
    k_free_surface_deriv<<<b, t, 0, (cudaStream_t)stream>>>(h_W, W, CJM, rDZ_DX, rDZ_DY, pml_beta_x, pml_beta_y,
                                                            Aos{_nx_, _ny_, _nz_}, rDH, FB1, FB2, FB3, DT);
    return launched("cgfdm_freeSurfaceDeriv");
}

int cgfdm_pmlDeriv(int _nx_, int _ny_, int _nz_, int nPML, float rDH, float *h_W, const float *W, const float *CJM,
                   float *const *aux, const float *const *pml, const int *border, int free_surface, int FB1, int FB2,
                   int FB3, float DT, void *stream)
{
    if (!h_W || !W || !CJM || !aux || !pml || !border || !grid_ok(_nx_, _ny_, _nz_) || nPML < 1 || !fb_ok(FB1) ||
        !fb_ok(FB2) || !fb_ok(FB3))
        return fail("cgfdm_pmlDeriv: bad argument", ST_ARG);
    const int n[3] = {_nx_ - 2 * HALO_, _ny_ - 2 * HALO_, _nz_ - 2 * HALO_};
    const int FB[3] = {FB1, FB2, FB3};
    // launch order x1 y1 z1 x2 y2 z2 (src/pml_deriv.cpp:633-646)
    for (int face = 0; face < 6; face++) {
        if (!border[face] || (face == 5 && free_surface)) continue;
        const int dir = face % 3, far = face / 3;
        if (nPML >= n[dir]) return fail("cgfdm_pmlDeriv: nPML >= grid size", CGFDM_E_PML_SIZE);
        float *hA = aux[face * 4 + 0];
        const float *A = aux[face * 4 + 1];
        const float *al = pml[dir * 3 + 0], *be = pml[dir * 3 + 1], *dd = pml[dir * 3 + 2];
        if (!hA || !A || !al || !be || !dd) return fail("cgfdm_pmlDeriv: missing face array", ST_ARG);
        const int e0 = dir == 0 ? nPML : n[0], e1 = dir == 1 ? nPML : n[1], e2 = dir == 2 ? nPML : n[2];
        const dim3 t(8, 8, 8);
        const dim3 b(blocks_for(e0, 8), blocks_for(e1, 8), blocks_for(e2, 8));
        k_pml_deriv<<<b, t, 0, (cudaStream_t)stream>>>(h_W, W, hA, A, CJM, al, be, dd, Aos{_nx_, _ny_, _nz_}, nPML,
                                                       dir, far, rDH, FB[dir], DT);
        if (int st = launched("cgfdm_pmlDeriv")) return st;
    }
    return ST_OK;
}

int cgfdm_pmlFreeSurfaceDeriv(int _nx_, int _ny_, int _nz_, int nPML, float rDH, const float *W, const float *CJM,
                              float *const *aux, const float *rDZ_DX, const float *rDZ_DY, const float *pml_d_x,
                              const float *pml_d_y, const int *border, int FB1, int FB2, float DT, void *stream)
{
    if (!W || !CJM || !aux || !rDZ_DX || !rDZ_DY || !pml_d_x || !pml_d_y || !border || !grid_ok(_nx_, _ny_, _nz_) ||
        nPML < 1 || !fb_ok(FB1) || !fb_ok(FB2))
        return fail("cgfdm_pmlFreeSurfaceDeriv: bad argument", ST_ARG);
    const int n[2] = {_nx_ - 2 * HALO_, _ny_ - 2 * HALO_};
    // launch order x1 y1 x2 y2 (src/pml_freeSurface.cpp:290-305)
    static const int faces[4] = {0, 1, 3, 4};
    for (int f : faces) {
        if (!border[f]) continue;
        const int dir = f % 3, far = f / 3;
        float *hA = aux[f * 4 + 0];
        if (!hA) return fail("cgfdm_pmlFreeSurfaceDeriv: missing face array", ST_ARG);
        const int e0 = dir == 0 ? nPML : n[0], e1 = dir == 1 ? nPML : n[1];
        const dim3 t(8, 8, 1);
        const dim3 b(blocks_for(e0, 8), blocks_for(e1, 8), 1);
        k_pml_free_surface<<<b, t, 0, (cudaStream_t)stream>>>(hA, W, CJM, dir == 0 ? rDZ_DX : rDZ_DY,
                                                              dir == 0 ? pml_d_x : pml_d_y, Aos{_nx_, _ny_, _nz_},
                                                              nPML, dir, far, rDH, dir == 0 ? FB1 : FB2, DT);
        if (int st = launched("cgfdm_pmlFreeSurfaceDeriv")) return st;
    }
    return ST_OK;
}

int cgfdm_waveRk(int _nx_, int _ny_, int _nz_, int irk, float *h_W, float *W, float *t_W, float *m_W, void *stream)
{
    if (!h_W || !W || !t_W || !m_W || irk < 0 || irk > 3 || _nx_ < 1 || _ny_ < 1 || _nz_ < 1)
        return fail("cgfdm_waveRk: bad argument", ST_ARG);
    const long long n = (long long)_nx_ * _ny_ * _nz_ * 9;
    k_rk<<<blocks_for(n, 1024), 1024, 0, (cudaStream_t)stream>>>(h_W, W, t_W, m_W, n, irk);
    return launched("cgfdm_waveRk");
}

int cgfdm_pmlRk(int nx, int ny, int nz, int nPML, int irk, float *const *aux, const int *border, int free_surface,
                void *stream)
{
    if (!aux || !border || irk < 0 || irk > 3 || nPML < 1) return fail("cgfdm_pmlRk: bad argument", ST_ARG);
    const long long num[3] = {(long long)nPML * ny * nz * 9, (long long)nPML * nx * nz * 9,
                              (long long)nPML * nx * ny * 9};
    for (int face = 0; face < 6; face++) {
        if (!border[face] || (face == 5 && free_surface)) continue;
        float *const *A = aux + face * 4;
        if (!A[0] || !A[1] || !A[2] || !A[3]) return fail("cgfdm_pmlRk: missing face array", ST_ARG);
        const long long n = num[face % 3];
        k_rk<<<blocks_for(n, 1024), 1024, 0, (cudaStream_t)stream>>>(A[0], A[1], A[2], A[3], n, irk);
        if (int st = launched("cgfdm_pmlRk")) return st;
    }
    return ST_OK;
}

int cgfdm_calculateMomentRate(long long npts, long long nt, const float *CJM, float *momentRate,
                              const long long *srcIndex, float DH, int scheme, void *stream)
{
    if (npts == 0) return ST_OK;
    if (npts < 0 || nt < 1 || !CJM || !momentRate || !srcIndex)
        return fail("cgfdm_calculateMomentRate: bad argument", ST_ARG);
    const dim3 t(16, 16, 1), b(blocks_for(npts, 16), blocks_for(nt, 16), 1);
    k_calc_moment_rate<<<b, t, 0, (cudaStream_t)stream>>>(npts, nt, CJM, scheme == SCHEME_SCFDM ? SC_NF : 13,
                                                          momentRate, srcIndex, DH);
    return launched("cgfdm_calculateMomentRate");
}

int cgfdm_addMomenteRate(long long npts, int nt, float dt, float *W, const long long *srcIndex,
                         const float *momentRate, float *momentRateSlice, int it, int irk, float DT, int scheme,
                         const float *CJM, void *stream)
{
    if (npts == 0) return ST_OK;
    if (npts < 0 || nt < 1 || !W || !srcIndex || !momentRate || !momentRateSlice || irk < 0 || irk > 3 ||
        (scheme == SCHEME_SCFDM && !CJM))
        return fail("cgfdm_addMomenteRate: bad argument", ST_ARG);
    // the interpolation weight in float on the host (src/addMoment.cpp:283-303)
    float tmpT;
    if (irk == 0) tmpT = (it + 0.0f) * DT;
    else if (irk == 3) tmpT = (it + 1.0f) * DT;
    else tmpT = (it + 0.5f) * DT;
    const int srcIt = int(tmpT / dt);
    if (srcIt + 1 >= nt) return ST_OK;   // table exhausted: no more injection
    const float t1 = float(srcIt) * dt;
    const float t_weight = (tmpT - t1) / dt;
    k_add_moment<<<blocks_for(npts, 256), 256, 0, (cudaStream_t)stream>>>(
        W, srcIndex, momentRate, momentRateSlice, npts, srcIt, t_weight, DT, CJM, 19, scheme == SCHEME_SCFDM);
    return launched("cgfdm_addMomenteRate");
}

int cgfdm_storageStation(int _nx_, int _ny_, int _nz_, int NT, int stationNum, const int *XYZ, float *wave,
                         const float *W, int it, int scheme, const float *CJM, void *stream)
{
    if (stationNum <= 0) return ST_OK;
    if (!XYZ || !wave || !W || it < 0 || it >= NT || (scheme == SCHEME_SCFDM && !CJM))
        return fail("cgfdm_storageStation: bad argument", ST_ARG);
    k_storage_station<<<blocks_for(stationNum, 32), 32, 0, (cudaStream_t)stream>>>(
        stationNum, XYZ, wave, W, CJM, 19, Aos{_nx_, _ny_, _nz_}, NT, it, scheme == SCHEME_SCFDM);
    return launched("cgfdm_storageStation");
}

int cgfdm_comparePGV(int nx, int ny, int nz, const float *W, float *pgv, float DT, int it, int scheme,
                     const float *CJM, const float *W_pre, void *stream)
{
    if (!W || !pgv || nx < 1 || ny < 1 || nz < 1 || (scheme == SCHEME_SCFDM && !CJM))
        return fail("cgfdm_comparePGV: bad argument", ST_ARG);
    const dim3 t(32, 16, 1), b(blocks_for(nx, 32), blocks_for(ny, 16), 1);
    k_compare_pgv<<<b, t, 0, (cudaStream_t)stream>>>(pgv, W, W_pre, CJM, 19,
                                                     Aos{nx + 2 * HALO_, ny + 2 * HALO_, nz + 2 * HALO_}, DT, it,
                                                     scheme == SCHEME_SCFDM);
    return launched("cgfdm_comparePGV");
}

int cgfdm_SolveDisplacement(int _nx_, int _ny_, int _nz_, const float *W, float *Dis, int scheme, const float *CJM,
                            float DT, void *stream)
{
    if (!W || !Dis || _nx_ < 1 || _ny_ < 1 || _nz_ < 1 || (scheme == SCHEME_SCFDM && !CJM))
        return fail("cgfdm_SolveDisplacement: bad argument", ST_ARG);
    const long long n = (long long)_nx_ * _ny_ * _nz_;
    k_solve_displacement<<<blocks_for(n, 256), 256, 0, (cudaStream_t)stream>>>(W, Dis, CJM, 19, n, DT,
                                                                               scheme == SCHEME_SCFDM);
    return launched("cgfdm_SolveDisplacement");
}

static int point_source(const char *what, int _nx_, int _ny_, int _nz_, int X, int Y, int Z, float *W,
                        const float *CJM, PointArgs &p, float DT, float DH, int scheme, void *stream)
{
    if (!W || !CJM || !grid_ok(_nx_, _ny_, _nz_)) return fail(std::string(what) + ": bad argument", ST_ARG);
    // the reference launches only for a source inside the interior
    if (!(X >= HALO_ && X < _nx_ - HALO_ && Y >= HALO_ && Y < _ny_ - HALO_ && Z >= HALO_ && Z < _nz_ - HALO_))
        return ST_OK;
    p.X = X, p.Y = Y, p.Z = Z;
    const std::vector<float> amp = point_gauss_weights(3);
    for (int t = 0; t < 343; t++) p.amp[t] = amp[t];
    k_point_source<<<1, 352, 0, (cudaStream_t)stream>>>(W, CJM, scheme == SCHEME_SCFDM ? SC_NF : 13,
                                                        Aos{_nx_, _ny_, _nz_}, p, DT, DH, scheme == SCHEME_SCFDM);
    return launched(what);
}

int cgfdm_loadPointSource_ricker(int _nx_, int _ny_, int _nz_, int X, int Y, int Z, float *W, const float *CJM,
                                 int it, int irk, float DT, float DH, float rickerfc, int scheme, void *stream)
{
    if (irk < 0 || irk > 3) return fail("cgfdm_loadPointSource_ricker: bad argument", ST_ARG);
    PointArgs p{};
    p.kind = 1;
    p.s = point_ricker(rickerfc, it, irk, DT);
    return point_source("cgfdm_loadPointSource_ricker", _nx_, _ny_, _nz_, X, Y, Z, W, CJM, p, DT, DH, scheme,
                        stream);
}

int cgfdm_loadPointSource_double_couple(int _nx_, int _ny_, int _nz_, int X, int Y, int Z, float *W,
                                        const float *CJM, int it, int irk, float DT, float DH, float strike,
                                        float dip, float rake, float Mw, float duration, int scheme, void *stream)
{
    if (irk < 0 || irk > 3) return fail("cgfdm_loadPointSource_double_couple: bad argument", ST_ARG);
    PointArgs p{};
    p.kind = 2;
    p.s = point_gauss_stf(duration, it, irk, DT);
    point_moment(strike, dip, rake, Mw, p.mom, &p.m0);
    return point_source("cgfdm_loadPointSource_double_couple", _nx_, _ny_, _nz_, X, Y, Z, W, CJM, p, DT, DH,
                        scheme, stream);
}

int cgfdm_waveDeriv_alternative_flux_FD(int _nx_, int _ny_, int _nz_, float rDH, float *h_W, const float *W,
                                        float *Riemann_flux, const float *CJM, float alpha, float DT, void *stream)
{
    if (!h_W || !W || !Riemann_flux || !CJM || !grid_ok(_nx_, _ny_, _nz_) || _nz_ < 4 * HALO_)
        return fail("cgfdm_waveDeriv_alternative_flux_FD: bad argument", ST_ARG);
    const Aos a{_nx_, _ny_, _nz_};
    const dim3 t(32, 4, 4);
    const int n[3] = {_nx_ - 2 * HALO_, _ny_ - 2 * HALO_, _nz_ - 2 * HALO_};
    // x flux, x difference, y flux, y difference, z flux, z difference
    // (src/alternative_flux_FD.cpp:1477-1537), one flux buffer
    for (int dir = 0; dir < 3; dir++) {
        const dim3 bf(blocks_for(n[0] + (dir == 0), 32), blocks_for(n[1] + (dir == 1), 4),
                      blocks_for(n[2] + (dir == 2), 4));
        k_sc_flux<<<bf, t, 0, (cudaStream_t)stream>>>(Riemann_flux, W, CJM, a, dir, alpha);
        if (int st = launched("cgfdm_waveDeriv_alternative_flux_FD")) return st;
        const dim3 bd(blocks_for(n[0], 32), blocks_for(n[1], 4), blocks_for(n[2], 4));
        k_sc_du<<<bd, t, 0, (cudaStream_t)stream>>>(h_W, Riemann_flux, W, CJM, a, dir, rDH, DT);
        if (int st = launched("cgfdm_waveDeriv_alternative_flux_FD")) return st;
    }
    return ST_OK;
}

int cgfdm_waveRk_tvd(int _nx_, int _ny_, int _nz_, int irk, const float *h_W, float *W, float *m_W, void *stream)
{
    if (!h_W || !W || !m_W || irk < 0 || irk > 2 || _nx_ < 1 || _ny_ < 1 || _nz_ < 1)
        return fail("cgfdm_waveRk_tvd: bad argument", ST_ARG);
    const long long n = (long long)_nx_ * _ny_ * _nz_ * 9;
    k_tvd<<<blocks_for(n, 1024), 1024, 0, (cudaStream_t)stream>>>(h_W, W, m_W, n, irk);
    return launched("cgfdm_waveRk_tvd");
}

int cgfdm_charfreeSurfaceDeriv(int _nx_, int _ny_, int _nz_, float *W, const float *CJM, void *stream)
{
    if (!W || !CJM || !grid_ok(_nx_, _ny_, _nz_) || _nz_ < 4 * HALO_)
        return fail("cgfdm_charfreeSurfaceDeriv: bad argument", ST_ARG);
    const dim3 t(32, 4, 1), b(blocks_for(_nx_ - 2 * HALO_, 32), blocks_for(_ny_ - 2 * HALO_, 4), 1);
    k_char_free_surface<<<b, t, 0, (cudaStream_t)stream>>>(W, CJM, Aos{_nx_, _ny_, _nz_});
    return launched("cgfdm_charfreeSurfaceDeriv");
}

int cgfdm_expDecayLayers(int _nx_, int _ny_, int _nz_, float *W, int free_surface, void *stream)
{
    if (!W || !grid_ok(_nx_, _ny_, _nz_)) return fail("cgfdm_expDecayLayers: bad argument", ST_ARG);
    // 20 layers, alpha 0.015 (src/exp_decay_absorb.cpp:110-111); G[p] =
    // exp(-(alpha p)^2) in float, as the reference's kernel evaluates it
    DecayTable tab;
    const int nl = 20;
    const float alpha = (float)0.015;
    for (int p = 0; p <= nl; p++) {
        const float x = alpha * (float)p;
        tab.G[p] = std::exp(-x * x);
    }
    const dim3 t(32, 4, 1);
    const dim3 b(blocks_for(_nx_ - 2 * HALO_, 32), blocks_for(_ny_ - 2 * HALO_, 4), _nz_ - 2 * HALO_);
    k_exp_decay<<<b, t, 0, (cudaStream_t)stream>>>(W, Aos{_nx_, _ny_, _nz_}, tab, nl, free_surface);
    return launched("cgfdm_expDecayLayers");
}

int cgfdm_storage_W_pre(int _nx_, int _ny_, int _nz_, float *W_pre, const float *W, void *stream)
{
    if (!W_pre || !W || _nx_ < 1 || _ny_ < 1 || _nz_ < 1) return fail("cgfdm_storage_W_pre: bad argument", ST_ARG);
    const long long n = (long long)_nx_ * _ny_ * _nz_;
    k_copy_prefix<<<blocks_for(n, 1024), 1024, 0, (cudaStream_t)stream>>>(W_pre, W, n);
    return launched("cgfdm_storage_W_pre");
}

}  // extern "C"
