// Reference-form time stepping in a chosen precision: the FP64 run.
//
// The session's fused stage kernels compute in FP32, as the reference does.
// This file runs the same time loop (src/propagate.cpp:186-321) with the
// wavefield, PML auxiliaries, station traces and all arithmetic in a type R:
// double gives the FP64 run every FP32 (and reduced-storage) result is
// measured against; float, built with --fmad=false, reproduces the session
// bit for bit and so checks that this restatement is the session's
// algorithm.  The model is the session's own device model (metric and
// medium, free-surface matrices, PML profiles, source tables, stations) in
// FP32, promoted where R is double, as the CPU FP64 oracle promotes the
// reference's FP32 model.
//
// One thread per point and plain loads: this is an accuracy reference, not
// the fast path.  Per step: sources at the stage-0 time; CGFDM: four RK4
// stages, each one launch computing derivative, traction-image free
// surface, CFS-PML and the RK update (src/wave_deriv.cpp:76-284,
// src/freeSurface.cpp:242-494, src/pml_deriv.cpp:125-584,
// src/pml_freeSurface.cpp:16-242, src/wave_rk.cpp:17-104,
// src/pml_rk.cpp:18-73); ME-AWENO: three TVD-RK3 stages of three
// directional flux and flux-difference launches and an update
// (src/alternative_flux_FD.cpp:42-399,1215-1435, src/wave_rk_tvd.cpp:17-78),
// then the characteristic free surface (src/freeSurface.cpp:40-194) and the
// sponge (src/exp_decay_absorb.cpp:19-145); then stations
// (src/station.cpp:302-380) and peak ground velocity (src/PGV.cpp:61-175).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "cg_ops.cuh"
#include "device.cuh"
#include "kernels.cuh"
#include "session.hpp"
#include "session_util.hpp"

namespace cgfdm {

namespace {

template <class R>
__device__ __forceinline__ R r_sqrt(R x)
{
    if constexpr (std::is_same<R, float>::value) return sqrtf(x);
    else return sqrt(x);
}

template <class R>
struct PFace {
    R *A, *B, *T;   // step start / final, stage value, RK accumulator
    long long count;
};

// ------------------------------------------------------------ CGFDM stage
template <class R>
struct PCgArgs {
    DevGrid g;
    const float *cjm, *rdz;
    const float *pa[9];   // alpha, beta, d of x, y, z
    const R *Win, *Wm;
    R *T, *Wout, *pgv;
    PFace<R> face[5];     // x1 y1 z1 x2 y2
    int irk, FB[3], nPML, pml_on, fs_on;
    float rDH, DT;
};

template <class R>
__global__ void __launch_bounds__(128) k_pre_cg_stage(const PCgArgs<R> a)
{
    const DevGrid &g = a.g;
    const int i = blockIdx.x * 32 + threadIdx.x + CGFDM_HALO;
    const int j = blockIdx.y * 4 + threadIdx.y + CGFDM_HALO;
    const int k = blockIdx.z + CGFDM_HALO;
    const int _nx = g.nxp - CGFDM_HALO, _ny = g.nyp - CGFDM_HALO, _nz = g.nzp - CGFDM_HALO;
    if (i >= _nx || j >= _ny) return;
    const long long F = g.fstride, q = g.at(i, j, k);
    const long long st[3] = {1, g.pitch, g.plane};
    const R rDH = (R)a.rDH, DT = (R)a.DT;
    auto C = [&](long long p, int f) -> R { return (R)a.cjm[f * F + p]; };
    auto W = [&](long long p, int f) -> R { return a.Win[f * F + p]; };
    auto L = [&](long long p, int f, long long s, int FB) -> R {
        return lop<R>(W(p - FB * s, f), W(p, f), W(p + FB * s, f), W(p + 2 * FB * s, f), W(p + 3 * FB * s, f), FB, rDH);
    };
    const R mu = C(q, C_MU), lam = C(q, C_LAMBDA), buo = C(q, C_BUOY) * (R)1.0f;
    const R beta[3] = {(R)a.pa[1][i], (R)a.pa[4][j], (R)a.pa[7][k]};
    R h[9];
    if (!(a.fs_on && k >= _nz - 3)) {
        for (int d = 0; d < 3; d++) {
            R dd[9], c[9];
            for (int f = 0; f < 9; f++) dd[f] = L(q, f, st[d], a.FB[d]) * beta[d];
            dir_rhs<R>(C(q, 3 * d), C(q, 3 * d + 1), C(q, 3 * d + 2), dd, mu, lam, buo, c);
            for (int f = 0; f < 9; f++) h[f] = d == 0 ? c[f] : h[f] + c[f];
        }
        for (int f = 0; f < 9; f++) h[f] = h[f] * DT;
    } else {
        // traction image: J (metric row . traction) at the taps, along zeta
        // antisymmetric about the surface
        const int ks = (_nz - 1) - k + CGFDM_HALO;
        R J[3][7][3];
        for (int d = 0; d < 3; d++)
            for (int l = 0; l < 7; l++) {
                if (d == 2 && l >= ks) continue;
                const long long p = q + (long long)(l - CGFDM_HALO) * st[d];
                const R m0 = C(p, 3 * d), m1 = C(p, 3 * d + 1), m2 = C(p, 3 * d + 2), jac = C(p, C_JAC);
                J[d][l][0] = ((m0 * W(p, 3) + m1 * W(p, 6)) + m2 * W(p, 7)) * jac;
                J[d][l][1] = ((m0 * W(p, 6) + m1 * W(p, 4)) + m2 * W(p, 8)) * jac;
                J[d][l][2] = ((m0 * W(p, 7) + m1 * W(p, 8)) + m2 * W(p, 5)) * jac;
            }
        for (int c = 0; c < 3; c++) {
            J[2][ks][c] = (R)0.0f;
            for (int l = ks + 1; l <= 2 * CGFDM_HALO; l++) J[2][l][c] = -J[2][2 * ks - l][c];
        }
        const R jinv = (R)1.0f / C(q, C_JAC);
        R L3[3][3];
        for (int d = 0; d < 3; d++)
            for (int c = 0; c < 3; c++) {
                const int FB = a.FB[d];
                L3[d][c] = lop<R>(J[d][3 - FB][c], J[d][3][c], J[d][3 + FB][c], J[d][3 + 2 * FB][c],
                                  J[d][3 + 3 * FB][c], FB, rDH);
            }
        for (int c = 0; c < 3; c++) h[c] = ((buo * jinv) * ((L3[0][c] * beta[0] + L3[1][c] * beta[1]) + L3[2][c])) * DT;
        R vxi[3], vet[3], vzt[3];
        for (int c = 0; c < 3; c++) {
            vxi[c] = L(q, c, st[0], a.FB[0]) * beta[0];
            vet[c] = L(q, c, st[1], a.FB[1]) * beta[1];
        }
        const int FB3 = a.FB[2];
        if (k == _nz - 1) {
            const long long s = g.at2(i, j);
            for (int r = 0; r < 3; r++) {
                const float *dx = a.rdz + (long long)(r * 3) * g.plane + s;
                const float *dy = a.rdz + (long long)(9 + r * 3) * g.plane + s;
                vzt[r] = (((R)dx[0] * vxi[0] + (R)dx[g.plane] * vxi[1]) + (R)dx[2 * g.plane] * vxi[2]) +
                         (((R)dy[0] * vet[0] + (R)dy[g.plane] * vet[1]) + (R)dy[2 * g.plane] * vet[2]);
            }
        } else if (k == _nz - 2) {
            for (int c = 0; c < 3; c++) vzt[c] = ((R)FB3 * (W(q + FB3 * st[2], c) - W(q, c))) * rDH;
        } else {
            for (int c = 0; c < 3; c++)
                vzt[c] = ((R)FB3 * (((R)CG_CF1 * W(q, c) + (R)CG_CF2 * W(q + FB3 * st[2], c)) +
                                    (R)CG_CF3 * W(q + 2 * FB3 * st[2], c))) *
                         rDH;
        }
        R s1[9], s2[9], s3[9];
        dir_stress<R>(C(q, 0), C(q, 1), C(q, 2), vxi, mu, lam, s1);
        dir_stress<R>(C(q, 3), C(q, 4), C(q, 5), vet, mu, lam, s2);
        dir_stress<R>(C(q, 6), C(q, 7), C(q, 8), vzt, mu, lam, s3);
        for (int f = 3; f < 9; f++) h[f] = ((s1[f] + s2[f]) + s3[f]) * DT;
    }

    // CFS-PML, faces in the reference's launch order x1 y1 z1 x2 y2
    const int nPML = a.nPML;
    const bool sel[5] = {(a.pml_on & 1) && i < CGFDM_HALO + nPML, (a.pml_on & 2) && j < CGFDM_HALO + nPML,
                         (a.pml_on & 4) && k < CGFDM_HALO + nPML, (a.pml_on & 8) && i >= _nx - nPML,
                         (a.pml_on & 16) && j >= _ny - nPML};
    for (int fc = 0; fc < 5; fc++) {
        if (!sel[fc]) continue;
        const int d = fc == 0 || fc == 3 ? 0 : fc == 1 || fc == 4 ? 1 : 2;
        const PFace<R> &P = a.face[fc];
        const int i0 = i - CGFDM_HALO, j0 = j - CGFDM_HALO, k0 = k - CGFDM_HALO;
        long long pos;
        if (d == 0)
            pos = (long long)(i0 - (fc == 3 ? g.nx - nPML : 0)) + (long long)j0 * nPML + (long long)k0 * nPML * g.ny;
        else if (d == 1)
            pos = (long long)i0 + (long long)(j0 - (fc == 4 ? g.ny - nPML : 0)) * g.nx + (long long)k0 * g.nx * nPML;
        else
            pos = (long long)i0 + (long long)j0 * g.nx + (long long)k0 * g.nx * g.ny;
        const int ix = d == 0 ? i : d == 1 ? j : k;
        const R dval = (R)a.pa[d * 3 + 2][ix], be = (R)a.pa[d * 3 + 1][ix];
        const R ad = dval + (R)a.pa[d * 3 + 0][ix];
        R dd[9], rhs[9], aux[9], hA[9];
        for (int f = 0; f < 9; f++) dd[f] = L(q, f, st[d], a.FB[d]) * dval;
        dir_rhs<R>(C(q, 3 * d), C(q, 3 * d + 1), C(q, 3 * d + 2), dd, mu, lam, buo, rhs);
        const R *cur = a.irk == 0 ? P.A : P.B;
        for (int f = 0; f < 9; f++) aux[f] = cur[f * P.count + pos];
        for (int f = 0; f < 9; f++) hA[f] = (rhs[f] - ad * aux[f]) * DT;
        if (a.fs_on && k == _nz - 1 && d < 2) {
            const long long s = g.at2(i, j);
            R vz[3], t3[9];
            for (int r = 0; r < 3; r++) {
                const float *mr = a.rdz + (long long)(d * 9 + r * 3) * g.plane + s;
                vz[r] = ((R)mr[0] * dd[0] + (R)mr[g.plane] * dd[1]) + (R)mr[2 * g.plane] * dd[2];
            }
            dir_stress<R>(C(q, 6), C(q, 7), C(q, 8), vz, mu, lam, t3);
            for (int f = 3; f < 9; f++) hA[f] = hA[f] + t3[f] * DT;
        }
        for (int f = 0; f < 9; f++) h[f] = h[f] + (-be * aux[f]) * DT;
        for (int f = 0; f < 9; f++) {
            const long long x = f * P.count + pos;
            if (a.irk == 0) {
                P.T[x] = aux[f] + (R)RK_BETA1 * hA[f];
                P.B[x] = aux[f] + (R)RK_ALPHA2 * hA[f];
            } else if (a.irk == 1) {
                const R m = P.A[x];
                P.T[x] = P.T[x] + (R)RK_BETA2 * hA[f];
                P.B[x] = m + (R)RK_ALPHA3 * hA[f];
            } else if (a.irk == 2) {
                const R m = P.A[x];
                P.T[x] = P.T[x] + (R)RK_BETA3 * hA[f];
                P.B[x] = m + hA[f];
            } else {
                P.A[x] = P.T[x] + (R)RK_BETA4 * hA[f];
            }
        }
    }

    // RK4 of the wavefield
    R w[9];
    for (int f = 0; f < 9; f++) {
        const long long x = f * F + q;
        if (a.irk == 0) {
            const R m = a.Win[x];
            a.T[x] = m + (R)RK_BETA1 * h[f];
            w[f] = m + (R)RK_ALPHA2 * h[f];
        } else if (a.irk == 1) {
            a.T[x] = a.T[x] + (R)RK_BETA2 * h[f];
            w[f] = a.Wm[x] + (R)RK_ALPHA3 * h[f];
        } else if (a.irk == 2) {
            a.T[x] = a.T[x] + (R)RK_BETA3 * h[f];
            w[f] = a.Wm[x] + h[f];
        } else {
            w[f] = a.T[x] + (R)RK_BETA4 * h[f];
        }
        a.Wout[x] = w[f];
    }
    if (a.pgv && k == _nz - 1) {
        R *p = a.pgv + ((long long)(j - CGFDM_HALO) * g.nx + (i - CGFDM_HALO)) * 2;
        const R Vh = r_sqrt<R>(w[0] * w[0] + w[1] * w[1]), V = r_sqrt<R>(w[0] * w[0] + w[1] * w[1] + w[2] * w[2]);
        if (p[0] < Vh) p[0] = Vh;
        if (p[1] < V) p[1] = V;
    }
}

// ------------------------------------------------------------ ME-AWENO
// WENO5-JS (src/alternative_flux_FD.cpp:42-59): the smoothness indicators in
// R, (beta + 1e-6)^2 and the division by it in double.
template <class R>
__device__ __forceinline__ R weno5(R u1, R u2, R u3, R u4, R u5)
{
    R b1 = (R)0.3333333333f * ((((((R)10 * u3 * u3 - (R)31 * u3 * u4) + (R)25 * u4 * u4) + (R)11 * u3 * u5) -
                               (R)19 * u4 * u5) +
                              (R)4 * u5 * u5);
    R b2 = (R)0.3333333333f * ((((((R)4 * u2 * u2 - (R)13 * u2 * u3) + (R)13 * u3 * u3) + (R)5 * u2 * u4) -
                               (R)13 * u3 * u4) +
                              (R)4 * u4 * u4);
    R b3 = (R)0.3333333333f * ((((((R)4 * u1 * u1 - (R)19 * u1 * u2) + (R)25 * u2 * u2) + (R)11 * u1 * u3) -
                               (R)31 * u2 * u3) +
                              (R)10 * u3 * u3);
    const double e1 = (double)b1 + 1e-6, e2 = (double)b2 + 1e-6, e3 = (double)b3 + 1e-6;
    b1 = (R)(0.3125 / (e1 * e1));
    b2 = (R)(0.625 / (e2 * e2));
    b3 = (R)(0.0625 / (e3 * e3));
    const R tw = (R)1.0f / (b1 + b2 + b3);
    return (b1 * tw) * ((R)0.375f * u3 + (R)0.75f * u4 - (R)0.125f * u5) +
           (b2 * tw) * ((R)-0.125f * u2 + (R)0.75f * u3 + (R)0.375f * u4) +
           (b3 * tw) * ((R)0.375f * u1 - (R)1.25f * u2 + (R)1.875f * u3);
}

// physical flux along a metric row (src/alternative_flux_FD.cpp:146-154)
template <class R>
__device__ __forceinline__ void pflux(R n0, R n1, R n2, R lam, R mu, R b, const R u[9], R f[9])
{
    const R l2m = lam + (R)2 * mu;
    f[0] = -((n0 * ((lam * u[4] + lam * u[5]) + u[3] * l2m) + mu * n1 * u[8]) + mu * n2 * u[7]);
    f[1] = -((n1 * ((lam * u[3] + lam * u[5]) + u[4] * l2m) + mu * n0 * u[8]) + mu * n2 * u[6]);
    f[2] = -((n2 * ((lam * u[3] + lam * u[4]) + u[5] * l2m) + mu * n0 * u[7]) + mu * n1 * u[6]);
    f[3] = -((n0 * u[0]) * b);
    f[4] = -((n1 * u[1]) * b);
    f[5] = -((n2 * u[2]) * b);
    f[6] = -((n1 * u[2]) * b + (n2 * u[1]) * b);
    f[7] = -((n0 * u[2]) * b + (n2 * u[0]) * b);
    f[8] = -((n0 * u[1]) * b + (n1 * u[0]) * b);
}

template <class R>
struct PScArgs {
    DevGrid g;
    const float *cjm;
    const R *W;
    R *RF, *H;
    int dir;
    float alpha, rDH, DT;
};

// Lax-Friedrichs flux of the face between q and q + step along dir, at q
template <class R>
__global__ void __launch_bounds__(128) k_pre_sc_flux(const PScArgs<R> a)
{
    const DevGrid &g = a.g;
    const int d = a.dir;
    const int i = blockIdx.x * 32 + threadIdx.x + CGFDM_HALO - (d == 0);
    const int j = blockIdx.y * 4 + threadIdx.y + CGFDM_HALO - (d == 1);
    const int k = blockIdx.z + CGFDM_HALO - (d == 2);
    if (i >= g.nxp - CGFDM_HALO || j >= g.nyp - CGFDM_HALO) return;
    const long long F = g.fstride, q = g.at(i, j, k);
    const long long s = d == 0 ? 1 : d == 1 ? g.pitch : g.plane;
    auto C = [&](int f) -> R { return (R)a.cjm[f * F + q]; };
    R uL[9], uR[9], fL[9], fR[9];
    for (int v = 0; v < 9; v++) {
        const R *w = a.W + v * F;
        uL[v] = weno5<R>(w[q - 2 * s], w[q - s], w[q], w[q + s], w[q + 2 * s]);
        uR[v] = weno5<R>(w[q + 3 * s], w[q + 2 * s], w[q + s], w[q], w[q - s]);
    }
    pflux<R>(C(3 * d), C(3 * d + 1), C(3 * d + 2), C(C_LAMBDA), C(C_MU), C(C_BUOY), uL, fL);
    pflux<R>(C(3 * d), C(3 * d + 1), C(3 * d + 2), C(C_LAMBDA), C(C_MU), C(C_BUOY), uR, fR);
    for (int v = 0; v < 9; v++) a.RF[v * F + q] = (R)0.5f * (fR[v] + fL[v] - (R)a.alpha * (uR[v] - uL[v]));
}

// flux difference of the interior points along dir (x assigns, y and z add)
template <class R>
__global__ void __launch_bounds__(128) k_pre_sc_du(const PScArgs<R> a)
{
    const DevGrid &g = a.g;
    const int d = a.dir;
    const int i = blockIdx.x * 32 + threadIdx.x + CGFDM_HALO;
    const int j = blockIdx.y * 4 + threadIdx.y + CGFDM_HALO;
    const int k = blockIdx.z + CGFDM_HALO;
    const int _nz = g.nzp - CGFDM_HALO;
    if (i >= g.nxp - CGFDM_HALO || j >= g.nyp - CGFDM_HALO) return;
    const long long F = g.fstride, q = g.at(i, j, k);
    const long long s = d == 0 ? 1 : d == 1 ? g.pitch : g.plane;
    const R jac = (R)(1.0 / (double)a.cjm[C_JAC * F + q]);
    const R coef = (R)a.DT * (R)a.rDH * jac;
    const R c24 = (R)(1.0f / 24), c7 = (R)(7.0f / 5760), c12 = (R)(1.0f / 12), c48 = (R)(1.0f / 48),
            c2 = (R)(1.0f / 2);
    R val[9];
    if (k >= _nz - 3) {
        R hu[7][9];
        for (int n = 0; n < 7; n++) {
            const long long p = q + (n - 3) * s;
            R u[9];
            for (int v = 0; v < 9; v++) u[v] = a.W[v * F + p];
            auto C = [&](int f) -> R { return (R)a.cjm[f * F + p]; };
            pflux<R>(C(3 * d), C(3 * d + 1), C(3 * d + 2), C(C_LAMBDA), C(C_MU), C(C_BUOY), u, hu[n]);
        }
        auto o2 = [&](int b, int v) {
            return c48 * ((((((R)-5 * hu[b][v] + (R)39 * hu[b + 1][v]) - (R)34 * hu[b + 2][v]) - (R)34 * hu[b + 3][v]) +
                           (R)39 * hu[b + 4][v]) -
                          (R)5 * hu[b + 5][v]);
        };
        auto o4 = [&](int b, int v) {
            return c2 * ((((((hu[b][v] - (R)3 * hu[b + 1][v]) + (R)2 * hu[b + 2][v]) + (R)2 * hu[b + 3][v]) -
                           (R)3 * hu[b + 4][v]) +
                          hu[b + 5][v]));
        };
        for (int v = 0; v < 9; v++) {
            const R A = a.RF[v * F + q] - c24 * o2(1, v) + c7 * o4(1, v);
            const R B = a.RF[v * F + q - s] - c24 * o2(0, v) + c7 * o4(0, v);
            val[v] = coef * (-(A - B));
        }
    } else {
        for (int v = 0; v < 9; v++) {
            const R *f = a.RF + v * F + q;
            const R f3 = f[-3 * s], f2 = f[-2 * s], f1 = f[-s], f0 = f[0], g1 = f[s], g2 = f[2 * s];
            const R A = f0 - c24 * (c12 * ((((-f2 + (R)16 * f1) - (R)30 * f0) + (R)16 * g1) - g2)) +
                        c7 * ((((f2 - (R)4 * f1) + (R)6 * f0) - (R)4 * g1) + g2);
            const R B = f1 - c24 * (c12 * ((((-f3 + (R)16 * f2) - (R)30 * f1) + (R)16 * f0) - g1)) +
                        c7 * ((((f3 - (R)4 * f2) + (R)6 * f1) - (R)4 * f0) + g1);
            val[v] = coef * (-(A - B));
        }
    }
    for (int v = 0; v < 9; v++) a.H[v * F + q] = d == 0 ? val[v] : a.H[v * F + q] + val[v];
}

// TVD-RK3 over every stored value (src/wave_rk_tvd.cpp:17-78; halo points
// have a zero right-hand side)
template <class R>
__global__ void k_pre_tvd(R *W, R *Wm, const R *H, long long n, int irk)
{
    const long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= n) return;
    const R h = H[x];
    if (irk == 0) {
        const R w = W[x];
        Wm[x] = w;
        W[x] = w + h;
    } else if (irk == 1) {
        W[x] = (R)(0.75 * (double)Wm[x] + 0.25 * (double)W[x] + 0.25 * (double)h);
    } else {
        W[x] = (R)((1.0 / 3.0) * (double)Wm[x] + (2.0 / 3.0) * (double)W[x] + (2.0 / 3.0) * (double)h);
    }
}

// characteristic free surface of the surface layer, in double with the
// inverse of the basis (n, s, t), then cubic extrapolation into the halo
template <class R>
__global__ void k_pre_char_fs(R *W, const float *__restrict__ cjm, DevGrid g)
{
    const int i = blockIdx.x * 32 + threadIdx.x + CGFDM_HALO;
    const int j = blockIdx.y * 4 + threadIdx.y + CGFDM_HALO;
    if (i >= g.nxp - CGFDM_HALO || j >= g.nyp - CGFDM_HALO) return;
    const long long F = g.fstride, q = g.at(i, j, g.nzp - CGFDM_HALO - 1);
    const float mu = cjm[C_MU * F + q], lam = cjm[C_LAMBDA * F + q], buo = cjm[C_BUOY * F + q];
    const float rho = 1.0f / buo, vs = sqrtf(mu * buo), vp = sqrtf((lam + 2 * mu) * buo);
    const double jac = cjm[C_JAC * F + q];
    double n[3] = {cjm[C_ZT_X * F + q] / jac, cjm[C_ZT_Y * F + q] / jac, cjm[C_ZT_Z * F + q] / jac};
    double sv[3] = {cjm[C_X_XI * F + q], cjm[C_Y_XI * F + q], cjm[C_Z_XI * F + q]};
    double tv[3] = {cjm[C_X_ET * F + q], cjm[C_Y_ET * F + q], cjm[C_Z_ET * F + q]};
    double *bs[3] = {n, sv, tv};
    for (int b = 0; b < 3; b++) {
        const double r = 1.0 / sqrt(bs[b][0] * bs[b][0] + bs[b][1] * bs[b][1] + bs[b][2] * bs[b][2]);
        for (int c = 0; c < 3; c++) bs[b][c] *= r;
    }
    double Rm[3][3];
    for (int b = 0; b < 3; b++) {
        const double *x = bs[(b + 1) % 3], *y = bs[(b + 2) % 3];
        Rm[b][0] = x[1] * y[2] - x[2] * y[1];
        Rm[b][1] = x[2] * y[0] - x[0] * y[2];
        Rm[b][2] = x[0] * y[1] - x[1] * y[0];
    }
    const double det = n[0] * Rm[0][0] + n[1] * Rm[0][1] + n[2] * Rm[0][2];
    for (int b = 0; b < 3; b++)
        for (int c = 0; c < 3; c++) Rm[b][c] /= det;
    double u[9];
    for (int v = 0; v < 9; v++) u[v] = (double)W[v * F + q];
    const double L = lam, M = mu, tr = u[3] + u[4] + u[5];
    const double S[3][3] = {{L * tr + 2 * M * u[3], M * u[8], M * u[7]},
                            {M * u[8], L * tr + 2 * M * u[4], M * u[6]},
                            {M * u[7], M * u[6], L * tr + 2 * M * u[5]}};
    const double vel[3] = {u[0] * buo, u[1] * buo, u[2] * buo};
    double RS[3][3], T[3][3], vb[3];
    for (int b = 0; b < 3; b++)
        for (int c = 0; c < 3; c++) RS[b][c] = Rm[b][0] * S[0][c] + Rm[b][1] * S[1][c] + Rm[b][2] * S[2][c];
    for (int b = 0; b < 3; b++)
        for (int c = 0; c < 3; c++) T[b][c] = RS[b][0] * Rm[c][0] + RS[b][1] * Rm[c][1] + RS[b][2] * Rm[c][2];
    for (int b = 0; b < 3; b++) vb[b] = Rm[b][0] * vel[0] + Rm[b][1] * vel[1] + Rm[b][2] * vel[2];
    const double ratio = L / (L + 2 * M);
    T[1][1] -= T[0][0] * ratio;
    T[2][2] -= T[0][0] * ratio;
    vb[1] -= T[0][1] / ((double)vs * rho);
    vb[2] -= T[0][2] / ((double)vs * rho);
    vb[0] -= T[0][0] / ((double)vp * rho);
    T[0][0] = T[0][1] = T[1][0] = T[0][2] = T[2][0] = 0.0;
    const double B[3][3] = {{n[0], sv[0], tv[0]}, {n[1], sv[1], tv[1]}, {n[2], sv[2], tv[2]}};
    double BT[3][3], Sg[3][3], v2[3];
    for (int b = 0; b < 3; b++)
        for (int c = 0; c < 3; c++) BT[b][c] = B[b][0] * T[0][c] + B[b][1] * T[1][c] + B[b][2] * T[2][c];
    for (int b = 0; b < 3; b++)
        for (int c = 0; c < 3; c++) Sg[b][c] = BT[b][0] * B[c][0] + BT[b][1] * B[c][1] + BT[b][2] * B[c][2];
    for (int b = 0; b < 3; b++) v2[b] = B[b][0] * vb[0] + B[b][1] * vb[1] + B[b][2] * vb[2];
    const double comp = 1.0 / (2 * M * (3 * L + 2 * M)), strace = Sg[0][0] + Sg[1][1] + Sg[2][2];
    double o[9];
    for (int b = 0; b < 3; b++) o[b] = v2[b] * rho;
    for (int b = 0; b < 3; b++) o[3 + b] = (2 * (L + M) * Sg[b][b] - L * (strace - Sg[b][b])) * comp;
    o[6] = Sg[1][2] / M, o[7] = Sg[0][2] / M, o[8] = Sg[0][1] / M;
    for (int v = 0; v < 9; v++) W[v * F + q] = (R)o[v];
    const long long P = g.plane;
    for (int v = 0; v < 9; v++) {
        R *c = W + v * F + q;
        for (int hh = 1; hh <= CGFDM_HALO; hh++)
            c[hh * P] = (R)4.0f * c[(hh - 1) * P] - (R)6.0f * c[(hh - 2) * P] + (R)4.0f * c[(hh - 3) * P] -
                        c[(hh - 4) * P];
    }
}

template <class R>
struct DecayG {
    R G[21];
};

// exponential sponge of the interior (free surface on top: no top layers)
template <class R>
__global__ void k_pre_decay(R *W, DevGrid g, DecayG<R> t)
{
    const int i = blockIdx.x * 32 + threadIdx.x + CGFDM_HALO;
    const int j = blockIdx.y * 4 + threadIdx.y + CGFDM_HALO;
    const int k = blockIdx.z + CGFDM_HALO;
    if (i >= g.nxp - CGFDM_HALO || j >= g.nyp - CGFDM_HALO) return;
    const int nl = 20, X = i - CGFDM_HALO, Y = j - CGFDM_HALO, Z = k - CGFDM_HALO;
    R G[5];
    int ng = 0;
    if (X <= nl) G[ng++] = t.G[nl - X];
    if (X >= g.nx - nl) G[ng++] = t.G[nl - (g.nx - X)];
    if (Y <= nl) G[ng++] = t.G[nl - Y];
    if (Y >= g.ny - nl) G[ng++] = t.G[nl - (g.ny - Y)];
    if (Z <= nl) G[ng++] = t.G[nl - Z];
    const long long q = g.at(i, j, k);
    for (int b = 0; b < ng; b++)
        for (int v = 0; v < 9; v++) W[v * g.fstride + q] = W[v * g.fstride + q] * G[b];
}

// ME-AWENO peak ground velocity of the surface layer
template <class R>
__global__ void k_pre_sc_pgv(const R *W, const float *__restrict__ cjm, DevGrid g, R *pgv)
{
    const int i = blockIdx.x * 32 + threadIdx.x, j = blockIdx.y * 4 + threadIdx.y;
    if (i >= g.nx || j >= g.ny) return;
    const long long F = g.fstride, q = g.at(i + CGFDM_HALO, j + CGFDM_HALO, g.nzp - CGFDM_HALO - 1);
    const R b = (R)cjm[C_BUOY * F + q];
    const R Vx = W[q] * b, Vy = W[F + q] * b, Vz = W[2 * F + q] * b;
    const R Vh = r_sqrt<R>(Vx * Vx + Vy * Vy), V = r_sqrt<R>(Vx * Vx + Vy * Vy + Vz * Vz);
    R *p = pgv + ((long long)j * g.nx + i) * 2;
    if (p[0] < Vh) p[0] = Vh;
    if (p[1] < V) p[1] = V;
}

// ------------------------------------------------------------ sources
// finite fault at the stage-0 time of step it: the table value in float
// (explicitly rounded, as the session computes it), added in R
template <class R>
__global__ void k_pre_fault(R *W, const float *__restrict__ cjm, DevGrid g, FaultDev f, int it, float DT, int scheme)
{
    const float tmpT = __fmul_rn((float)it + 0.0f, DT);
    const int srcIt = (int)__fdiv_rn(tmpT, f.dt);
    if (srcIt + 1 >= f.nt) return;
    const float t1 = __fmul_rn((float)srcIt, f.dt);
    const float tw = __fdiv_rn(__fsub_rn(tmpT, t1), f.dt);
    const long long F = g.fstride;
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < f.npts;
         p += (long long)gridDim.x * blockDim.x) {
        const long long q = f.cell[p];
        const float *r0 = f.rate + ((long long)srcIt * f.npts + p) * 6;
        const float *r1 = f.rate + ((long long)(srcIt + 1) * f.npts + p) * 6;
        R m[6];
        for (int c = 0; c < 6; c++) m[c] = (R)__fadd_rn(__fmul_rn(__fsub_rn(r1[c], r0[c]), tw), r0[c]);
        if (scheme == 1) {
            const R mu = (R)cjm[C_MU * F + q], lam = (R)cjm[C_LAMBDA * F + q];
            const R den = (R)2 * (mu * mu) + (R)3 * lam * mu;
            const R s[6] = {m[0], m[1], m[2], m[3], m[4], m[5]};
            m[0] = ((s[0] * (lam + mu)) / den - (lam * s[1]) / ((R)2 * den)) - (lam * s[2]) / ((R)2 * den);
            m[1] = ((s[1] * (lam + mu)) / den - (lam * s[0]) / ((R)2 * den)) - (lam * s[2]) / ((R)2 * den);
            m[2] = ((s[2] * (lam + mu)) / den - (lam * s[0]) / ((R)2 * den)) - (lam * s[1]) / ((R)2 * den);
            m[3] = s[5] / mu, m[4] = s[4] / mu, m[5] = s[3] / mu;
        }
        for (int c = 0; c < 6; c++) W[(3 + c) * F + q] = W[(3 + c) * F + q] - m[c] * (R)DT;
    }
}

// 7 x 7 x 7 point source (explosive Ricker or double couple) at step it;
// halo cells also receive the value in the stage buffers Wb, Wc, which the
// stages never update there
template <class R>
__global__ void k_pre_point(R *W, R *Wb, R *Wc, const float *__restrict__ cjm, DevGrid g, PointDev p, int it,
                            float DT, float DH, int scheme)
{
    const int t = threadIdx.x;
    if (t >= 343 || !p.inside) return;
    const int i = p.X + t % 7 - 3, j = p.Y + (t / 7) % 7 - 3, k = p.Z + t / 49 - 3;
    const long long F = g.fstride, q = g.at(i, j, k);
    const float jacb = cjm[C_JAC * F + g.at(p.X, p.Y, p.Z)];
    const float s = p.stf[it], amp = p.amp[t];
    const float vol = __fmul_rn(jacb, __fmul_rn(__fmul_rn(DH, DH), DH));
    R add[6] = {0, 0, 0, 0, 0, 0};
    int nc;
    if (p.kind == 1) {
        float value = __fdiv_rn(__fmul_rn(__fmul_rn(-1.0f, s), amp), vol);
        value = (float)__dmul_rn((double)value, __dmul_rn(1.0, (double)DT));
        R v = (R)value;
        if (scheme == 1) v = v / ((R)3 * (R)cjm[C_LAMBDA * F + q] + (R)2 * (R)cjm[C_MU * F + q]);
        add[0] = add[1] = add[2] = v;
        nc = 3;
    } else {
        float rate = __fmul_rn(__fdiv_rn(__fmul_rn(__fmul_rn(-1.0f, s), amp), vol), p.m0);
        rate = (float)__dmul_rn((double)rate, __dmul_rn(1.0, (double)DT));
        R mr[6];
        for (int c = 0; c < 6; c++) mr[c] = (R)__fmul_rn(p.mom[c], rate);
        if (scheme == 1) {
            const R mu = (R)cjm[C_MU * F + q], lam = (R)cjm[C_LAMBDA * F + q];
            const R den = (R)2 * (mu * mu) + (R)3 * lam * mu;
            R e[6];
            e[0] = ((mr[0] * (lam + mu)) / den - (lam * mr[1]) / ((R)2 * den)) - (lam * mr[2]) / ((R)2 * den);
            e[1] = ((mr[1] * (lam + mu)) / den - (lam * mr[0]) / ((R)2 * den)) - (lam * mr[2]) / ((R)2 * den);
            e[2] = ((mr[2] * (lam + mu)) / den - (lam * mr[0]) / ((R)2 * den)) - (lam * mr[1]) / ((R)2 * den);
            e[3] = mr[5] / mu, e[4] = mr[4] / mu, e[5] = mr[3] / mu;
            for (int c = 0; c < 6; c++) mr[c] = e[c];
        }
        for (int c = 0; c < 6; c++) add[c] = -mr[c];
        nc = 6;
    }
    const bool halo = i < CGFDM_HALO || j < CGFDM_HALO || k < CGFDM_HALO || i >= g.nxp - CGFDM_HALO ||
                      j >= g.nyp - CGFDM_HALO || k >= g.nzp - CGFDM_HALO;
    for (int c = 0; c < nc; c++) {
        const R v = W[(3 + c) * F + q] + add[c];
        W[(3 + c) * F + q] = v;
        if (halo) {
            if (Wb) Wb[(3 + c) * F + q] = v;
            if (Wc) Wc[(3 + c) * F + q] = v;
        }
    }
}

// station traces of step n, [station][nsteps][9]
template <class R>
__global__ void k_pre_stations(const R *W, const float *__restrict__ cjm, DevGrid g, const int *__restrict__ idx,
                               int nst, int nsteps, int n, R *out, int scheme)
{
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nst) return;
    const long long F = g.fstride, q = g.at(idx[s * 3], idx[s * 3 + 1], idx[s * 3 + 2]);
    R u[9];
    for (int v = 0; v < 9; v++) u[v] = W[v * F + q];
    R *o = out + ((long long)s * nsteps + n) * 9;
    if (scheme == 1) {
        const R mu = (R)cjm[C_MU * F + q], lam = (R)cjm[C_LAMBDA * F + q], b = (R)cjm[C_BUOY * F + q] * (R)1.0f;
        const R l2m = lam + (R)2 * mu;
        o[0] = u[0] * b, o[1] = u[1] * b, o[2] = u[2] * b;
        o[3] = (lam * u[4] + lam * u[5]) + u[3] * l2m;
        o[4] = (lam * u[3] + lam * u[5]) + u[4] * l2m;
        o[5] = (lam * u[3] + lam * u[4]) + u[5] * l2m;
        o[6] = mu * u[8], o[7] = mu * u[7], o[8] = mu * u[6];
    } else {
        for (int v = 0; v < 9; v++) o[v] = u[v];
    }
}

// SoA (session layout) to the reference's AoS [_nz_][_ny_][_nx_][9], in double
template <class R>
__global__ void k_pre_to_aos(const R *W, DevGrid g, double *out)
{
    const long long n = (long long)g.nxp * g.nyp * g.nzp;
    for (long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(x % g.nxp), j = (int)((x / g.nxp) % g.nyp), k = (int)(x / ((long long)g.nxp * g.nyp));
        const long long q = g.at(i, j, k);
        for (int v = 0; v < 9; v++) out[x * 9 + v] = (double)W[v * g.fstride + q];
    }
}

template <class R>
__global__ void k_pre_to_double(const R *in, long long n, double *out)
{
    for (long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (long long)gridDim.x * blockDim.x)
        out[x] = (double)in[x];
}

}  // namespace

// The run itself.  Buffers are allocated for the call and freed after it;
// the session's own state is not touched.
template <class R>
int Session::run_precise_t(int nsteps, double *st_out, double *pgv_out, double *w_out)
{
    const bool cg = m.p.scheme == SCHEME_CGFDM;
    const long long F = g.fstride;
    // every buffer of the call, freed on every way out
    struct Owned {
        std::vector<void *> p;
        cudaStream_t s;
        ~Owned()
        {
            cudaStreamSynchronize(s);
            for (void *x : p) cudaFree(x);
        }
    } mine{{}, stream};
    auto grab = [&](size_t bytes) -> void * {
        void *p = nullptr;
        if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
        mine.p.push_back(p);
        if (cudaMemsetAsync(p, 0, bytes, stream) != cudaSuccess) return nullptr;
        return p;
    };
    auto fail = [&](int code, const std::string &why) {
        err = why;
        return code;
    };
    R *buf[4] = {nullptr, nullptr, nullptr, nullptr};
    for (int b = 0; b < 4; b++)
        if (!(buf[b] = (R *)grab(sizeof(R) * F * 9))) return fail(ST_ALLOC, "precise run: cannot allocate the wavefield");
    PFace<R> face[5] = {};
    if (cg && m.p.pml)
        for (int fc = 0; fc < 5; fc++) {
            if (!face_[fc].count) continue;
            face[fc].count = face_[fc].count;
            R *p = (R *)grab(sizeof(R) * face_[fc].count * 27);
            if (!p) return fail(ST_ALLOC, "precise run: cannot allocate the PML auxiliaries");
            face[fc].A = p, face[fc].B = p + face_[fc].count * 9, face[fc].T = p + face_[fc].count * 18;
        }
    const long long nst_vals = (long long)nst * nsteps * 9, npgv = (long long)m.g.nx * m.g.ny * 2;
    R *st = nst > 0 ? (R *)grab(sizeof(R) * std::max(nst_vals, 1LL)) : nullptr;
    R *pgv = (R *)grab(sizeof(R) * npgv);
    if ((nst > 0 && !st) || !pgv) return fail(ST_ALLOC, "precise run: cannot allocate the outputs");

    const float DT = (float)m.p.DT;
    const dim3 blk(32, 4, 1), grd((m.g.nx + 31) / 32, (m.g.ny + 3) / 4, m.g.nz);
    DecayG<R> decay{};
    {
        const float alpha = (float)0.015;
        for (int p = 0; p <= 20; p++) {
            const float x = alpha * (float)p;
            const float e = -x * x;
            decay.G[p] = std::is_same<R, float>::value ? (R)std::exp(e) : (R)std::exp((double)e);
        }
    }
    for (int it_ = 0; it_ < nsteps; it_++) {
        R *A = buf[0];
        if (point_.kind && point_.inside) {
            k_pre_point<R><<<1, 352, 0, stream>>>(A, buf[1], cg ? buf[2] : nullptr, cjm_, g, point_, it_, DT, m.g.DH,
                                                   m.p.scheme);
            CU(cudaGetLastError());
        }
        if (fault_.npts > 0) {
            const int nb = (int)std::min<long long>((fault_.npts + 255) / 256, 1024);
            k_pre_fault<R><<<nb, 256, 0, stream>>>(A, cjm_, g, fault_, it_, DT, m.p.scheme);
            CU(cudaGetLastError());
        }
        if (cg) {
            // A -> B -> C -> B -> A with T the accumulator, as the session
            R *B = buf[1], *Cb = buf[2], *T = buf[3];
            R *win[4] = {A, B, Cb, B}, *wout[4] = {B, Cb, B, A};
            int fb[3];
            fb_signs(it_, fb);
            for (int irk = 0; irk < 4; irk++) {
                PCgArgs<R> a{};
                a.g = g;
                a.cjm = cjm_, a.rdz = rdz_;
                for (int c = 0; c < 9; c++) a.pa[c] = pml_[c];
                a.Win = win[irk], a.Wm = A, a.T = T, a.Wout = wout[irk];
                a.pgv = irk == 3 ? pgv : nullptr;
                for (int fc = 0; fc < 5; fc++) a.face[fc] = face[fc];
                a.irk = irk;
                for (int c = 0; c < 3; c++) a.FB[c] = fb[c];
                a.nPML = m.g.nPML, a.pml_on = pml_faces(), a.fs_on = m.fs_top ? 1 : 0;
                a.rDH = m.g.rDH, a.DT = DT;
                k_pre_cg_stage<R><<<grd, blk, 0, stream>>>(a);
                CU(cudaGetLastError());
                for (int c = 0; c < 3; c++) fb[c] = -fb[c];
            }
        } else {
            // TVD-RK3: W (A), step start (B), RHS (C), face fluxes (T)
            R *Wm = buf[1], *H = buf[2], *RF = buf[3];
            for (int irk = 0; irk < 3; irk++) {
                for (int d = 0; d < 3; d++) {
                    PScArgs<R> a{};
                    a.g = g, a.cjm = cjm_, a.W = A, a.RF = RF, a.H = H, a.dir = d;
                    a.alpha = m.Vp_max, a.rDH = m.g.rDH, a.DT = DT;
                    const dim3 gf((m.g.nx + (d == 0) + 31) / 32, (m.g.ny + (d == 1) + 3) / 4, m.g.nz + (d == 2));
                    k_pre_sc_flux<R><<<gf, blk, 0, stream>>>(a);
                    CU(cudaGetLastError());
                    k_pre_sc_du<R><<<grd, blk, 0, stream>>>(a);
                    CU(cudaGetLastError());
                }
                const long long n = F * 9;
                k_pre_tvd<R><<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(A, Wm, H, n, irk);
                CU(cudaGetLastError());
            }
            k_pre_char_fs<R><<<dim3(grd.x, grd.y, 1), blk, 0, stream>>>(A, cjm_, g);
            CU(cudaGetLastError());
            if (m.p.exp_decay) {
                k_pre_decay<R><<<grd, blk, 0, stream>>>(A, g, decay);
                CU(cudaGetLastError());
            }
            k_pre_sc_pgv<R><<<dim3(grd.x, grd.y, 1), blk, 0, stream>>>(A, cjm_, g, pgv);
            CU(cudaGetLastError());
        }
        if (nst > 0) {
            k_pre_stations<R><<<(nst + 63) / 64, 64, 0, stream>>>(A, cjm_, g, st_idx_, nst, nsteps, it_, st,
                                                                  m.p.scheme);
            CU(cudaGetLastError());
        }
    }
    // results in double
    double *dout = (double *)grab(sizeof(double) * std::max({nst_vals, npgv, w_out ? m.g.npad() * 9 : 0LL, 1LL}));
    if (!dout) return fail(ST_ALLOC, "precise run: cannot allocate the read-back buffer");
    auto back = [&](const R *src, long long n, double *host) -> int {
        k_pre_to_double<R><<<1024, 256, 0, stream>>>(src, n, dout);
        CU(cudaGetLastError());
        CU(cudaMemcpyAsync(host, dout, sizeof(double) * n, cudaMemcpyDeviceToHost, stream));
        CU(cudaStreamSynchronize(stream));
        return ST_OK;
    };
    if (st_out && nst > 0)
        if (int s = back(st, nst_vals, st_out)) return s;
    if (pgv_out)
        if (int s = back(pgv, npgv, pgv_out)) return s;
    if (w_out) {
        k_pre_to_aos<R><<<1024, 256, 0, stream>>>(buf[0], g, dout);
        CU(cudaGetLastError());
        CU(cudaMemcpyAsync(w_out, dout, sizeof(double) * m.g.npad() * 9, cudaMemcpyDeviceToHost, stream));
    }
    CU(cudaStreamSynchronize(stream));
    return ST_OK;
}

int Session::run_precise(int nsteps, int bits, double *stations, double *pgv, double *wavefield)
{
    if (is_part_) {
        err = "the precise run applies to a whole grid, not a part";
        return ST_STATE;
    }
    if (nsteps < 0 || nsteps > m.NT || (bits != 32 && bits != 64)) {
        err = "precise run: nsteps must be in [0, NT] and bits 32 or 64";
        return ST_ARG;
    }
    return bits == 64 ? run_precise_t<double>(nsteps, stations, pgv, wavefield)
                      : run_precise_t<float>(nsteps, stations, pgv, wavefield);
}

}  // namespace cgfdm
