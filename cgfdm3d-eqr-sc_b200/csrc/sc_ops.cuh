// Point operators of the ME-AWENO (SCFDM) scheme shared by the tiled passes
// (scfdm_stage.cu) and the per-function entry points (shims.cu): the
// reference's WENO5-JS, physical and Lax-Friedrichs fluxes and flux
// difference term by term, and the characteristic free surface of one
// surface point.
#pragma once

#include "device.cuh"

namespace cgfdm {

// The reference's WENO5_JS term by term (src/alternative_flux_FD.cpp:42-59):
// float polynomials, double (beta + 1e-6)^2 and the division by it.
__device__ __forceinline__ float weno5_ref(float u1, float u2, float u3, float u4, float u5)
{
    float b1 = 10.0f * u3 * u3 - 31.0f * u3 * u4 + 25.0f * u4 * u4 + 11.0f * u3 * u5 - 19.0f * u4 * u5 +
               4.0f * u5 * u5;
    float b2 = 4.0f * u2 * u2 - 13.0f * u2 * u3 + 13.0f * u3 * u3 + 5.0f * u2 * u4 - 13.0f * u3 * u4 +
               4.0f * u4 * u4;
    float b3 = 4.0f * u1 * u1 - 19.0f * u1 * u2 + 25.0f * u2 * u2 + 11.0f * u1 * u3 - 31.0f * u2 * u3 +
               10.0f * u3 * u3;
    b1 = 0.3333333333f * b1;
    b2 = 0.3333333333f * b2;
    b3 = 0.3333333333f * b3;
    double e1 = __dadd_rn((double)b1, 1e-6), e2 = __dadd_rn((double)b2, 1e-6), e3 = __dadd_rn((double)b3, 1e-6);
    b1 = __double2float_rn(__ddiv_rn(0.3125, __dmul_rn(e1, e1)));
    b2 = __double2float_rn(__ddiv_rn(0.625, __dmul_rn(e2, e2)));
    b3 = __double2float_rn(__ddiv_rn(0.0625, __dmul_rn(e3, e3)));
    float tw = __fdiv_rn(1.0f, b1 + b2 + b3);
    return (b1 * tw) * (0.375f * u3 + 0.75f * u4 - 0.125f * u5) +
           (b2 * tw) * (-0.125f * u2 + 0.75f * u3 + 0.375f * u4) +
           (b3 * tw) * (0.375f * u1 - 1.25f * u2 + 1.875f * u3);
}

// Physical flux along the metric row (n0, n1, n2) of the state u
// (src/alternative_flux_FD.cpp:146-154; the same form is hu at 1259-1268).
__device__ __forceinline__ void point_flux(float n0, float n1, float n2, float lam, float mu, float buo,
                                           const float u[9], float f[9])
{
    f[0] = -(n0 * (lam * u[4] + lam * u[5] + u[3] * (lam + 2.0f * mu)) + mu * n1 * u[8] + mu * n2 * u[7]);
    f[1] = -(n1 * (lam * u[3] + lam * u[5] + u[4] * (lam + 2.0f * mu)) + mu * n0 * u[8] + mu * n2 * u[6]);
    f[2] = -(n2 * (lam * u[3] + lam * u[4] + u[5] * (lam + 2.0f * mu)) + mu * n0 * u[7] + mu * n1 * u[6]);
    f[3] = -((n0 * u[0]) * buo);
    f[4] = -((n1 * u[1]) * buo);
    f[5] = -((n2 * u[2]) * buo);
    f[6] = -((n1 * u[2]) * buo + (n2 * u[1]) * buo);
    f[7] = -((n0 * u[2]) * buo + (n2 * u[0]) * buo);
    f[8] = -((n0 * u[1]) * buo + (n1 * u[0]) * buo);
}

// Lax-Friedrichs flux of a face from its left (uL) and right (uR) states,
// as src/alternative_flux_FD.cpp:144-169 forms it.
__device__ __forceinline__ void lf_flux_ref(float n0, float n1, float n2, float lam, float mu, float buo, float alpha,
                                            const float uL[9], const float uR[9], float F[9])
{
    float fL[9], fR[9];
    point_flux(n0, n1, n2, lam, mu, buo, uL, fL);
    point_flux(n0, n1, n2, lam, mu, buo, uR, fR);
#pragma unroll
    for (int v = 0; v < 9; v++) F[v] = 0.5f * (fR[v] + fL[v] - alpha * (uR[v] - uL[v]));
}

// Flux difference of an interior point from the fluxes f[0..5] of the faces
// p-5/2 .. p+5/2 (src/alternative_flux_FD.cpp:1283), coef = DT rDH / J.
__device__ __forceinline__ float interior_diff_ref(const float f[6], float coef)
{
    const float c24 = 1.0f / 24, c7 = 7.0f / 5760;
    const float A = f[3] - c24 * ((1.0f / 12) * ((((-f[1] + 16.0f * f[2]) - 30.0f * f[3]) + 16.0f * f[4]) - f[5])) +
                    c7 * ((((f[1] - 4.0f * f[2]) + 6.0f * f[3]) - 4.0f * f[4]) + f[5]);
    const float B = f[2] - c24 * ((1.0f / 12) * ((((-f[0] + 16.0f * f[1]) - 30.0f * f[2]) + 16.0f * f[3]) - f[4])) +
                    c7 * ((((f[0] - 4.0f * f[1]) + 6.0f * f[2]) - 4.0f * f[3]) + f[4]);
    return coef * (-(A - B));
}

// Characteristic free surface of one surface point (src/freeSurface.cpp:
// 40-176), restated with the inverse of the basis B = [n s t]: T = B^-1
// sigma B^-T and v' = B^-1 v are the stress and velocity in that basis;
// after the condition, sigma = B T B^T, v = B v'.  Evaluated in double from
// the float fields and rounded once.  uin: the conserved variables; nrm: the
// zeta row of the metric (J grad zeta), jacf: J; tan1, tan2: the covariant
// xi and eta vectors; out: the conserved variables after the condition.
__device__ __forceinline__ void char_surface_point(const float uin[9], float mu, float lam, float buo, float jacf,
                                                   const float nrm[3], const float tan1[3], const float tan2[3],
                                                   float out[9])
{
    const float rho = 1.0f / buo;
    const float vs = sqrtf(mu * buo), vp = sqrtf((lam + 2.0f * mu) * buo);
    // orthonormalised surface normal and the two tangent directions
    const double jac = jacf;
    double n[3] = {nrm[0] / jac, nrm[1] / jac, nrm[2] / jac};
    double s[3] = {tan1[0], tan1[1], tan1[2]};
    double t[3] = {tan2[0], tan2[1], tan2[2]};
    auto normalise = [](double *x) {
        double r = 1.0 / sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
        x[0] *= r, x[1] *= r, x[2] *= r;
    };
    normalise(n), normalise(s), normalise(t);
    auto cross = [](const double *x, const double *y, double *o) {
        o[0] = x[1] * y[2] - x[2] * y[1];
        o[1] = x[2] * y[0] - x[0] * y[2];
        o[2] = x[0] * y[1] - x[1] * y[0];
    };
    // rows of B^-1: (s x t, t x n, n x s) / det
    double R[3][3];
    cross(s, t, R[0]), cross(t, n, R[1]), cross(n, s, R[2]);
    const double det = n[0] * R[0][0] + n[1] * R[0][1] + n[2] * R[0][2];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) R[r][c] /= det;

    // conservative -> physical: stress from strain, velocity from momentum
    double u[9];
    for (int v = 0; v < 9; v++) u[v] = uin[v];
    const double L = lam, M = mu, Bu = buo;
    const double tr = u[3] + u[4] + u[5];
    double S[3][3];
    S[0][0] = L * tr + 2.0 * M * u[3];
    S[1][1] = L * tr + 2.0 * M * u[4];
    S[2][2] = L * tr + 2.0 * M * u[5];
    S[0][1] = S[1][0] = M * u[8];
    S[0][2] = S[2][0] = M * u[7];
    S[1][2] = S[2][1] = M * u[6];
    const double vel[3] = {u[0] * Bu, u[1] * Bu, u[2] * Bu};

    // into the (n, s, t) basis
    double RS[3][3], T[3][3], vb[3];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) RS[r][c] = R[r][0] * S[0][c] + R[r][1] * S[1][c] + R[r][2] * S[2][c];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) T[r][c] = RS[r][0] * R[c][0] + RS[r][1] * R[c][1] + RS[r][2] * R[c][2];
    for (int r = 0; r < 3; r++) vb[r] = R[r][0] * vel[0] + R[r][1] * vel[1] + R[r][2] * vel[2];

    // characteristic free-surface condition (src/freeSurface.cpp:142-150)
    const double rho_d = rho, vs_d = vs, vp_d = vp;
    const double ratio = L / (L + 2.0 * M);
    T[1][1] -= T[0][0] * ratio;
    T[2][2] -= T[0][0] * ratio;
    vb[1] -= T[0][1] / (vs_d * rho_d);
    vb[2] -= T[0][2] / (vs_d * rho_d);
    vb[0] -= T[0][0] / (vp_d * rho_d);
    T[0][0] = 0.0, T[0][1] = T[1][0] = 0.0, T[0][2] = T[2][0] = 0.0;

    // back: sigma = B T B^T, v = B v'
    const double Bm[3][3] = {{n[0], s[0], t[0]}, {n[1], s[1], t[1]}, {n[2], s[2], t[2]}};
    double BT[3][3], Sg[3][3], v2[3];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) BT[r][c] = Bm[r][0] * T[0][c] + Bm[r][1] * T[1][c] + Bm[r][2] * T[2][c];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) Sg[r][c] = BT[r][0] * Bm[c][0] + BT[r][1] * Bm[c][1] + BT[r][2] * Bm[c][2];
    for (int r = 0; r < 3; r++) v2[r] = Bm[r][0] * vb[0] + Bm[r][1] * vb[1] + Bm[r][2] * vb[2];

    // physical -> conservative: momentum, and strain by the isotropic compliance
    const double comp = 1.0 / (2.0 * M * (3.0 * L + 2.0 * M));
    const double strace = Sg[0][0] + Sg[1][1] + Sg[2][2];
    double o[9];
    o[0] = v2[0] * rho_d, o[1] = v2[1] * rho_d, o[2] = v2[2] * rho_d;
    for (int d = 0; d < 3; d++) o[3 + d] = (2.0 * (L + M) * Sg[d][d] - L * (strace - Sg[d][d])) * comp;
    o[6] = Sg[1][2] / M, o[7] = Sg[0][2] / M, o[8] = Sg[0][1] / M;
    for (int v = 0; v < 9; v++) out[v] = (float)o[v];
}

}  // namespace cgfdm
