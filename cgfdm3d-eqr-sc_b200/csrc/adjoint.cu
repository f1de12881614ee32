// Discrete adjoint of the CGFDM time step: the exact transpose of the
// forward stage operator of csrc/cgfdm_stage.cu (MacCormack one-sided
// differences with the FB sign sequence, traction-image free surface, CFS
// PML with its auxiliaries and their free-surface term), and the gradient
// of the seismogram misfit with respect to (mu, lambda, buoyancy).
//
// The forward RHS of a stage at an interior point p is, per direction d,
//     h(p) += DT R_d(p) s_d(p) D_d W (p)
// with R_d(p) the 9x9 matrix of dir_rhs (metric row d and medium at p),
// s_d the PML stretch and D_d the one-sided 5-point difference; PML cells
// add DT R_d(p) dval D_d W to their auxiliary RHS.  Its transpose is
//     nu(q) = sum_d D_d^T Phi_d (q),  Phi_d(p) = R_d(p)^T (DT s_d mu(p) + DT dval muA(p)),
// a point-wise product followed by the transposed (reversed) difference.
// k_adj_pre forms Phi_d for every point; k_adj_gather applies D_d^T, adds
// the free-surface terms, the RK4 adjoint combination and the gradient.
//
// In the top three layers (src/freeSurface.cpp:345-492) the velocity rows
// difference J (metric . stress) taken at the tap points, with the
// antisymmetric image about the surface in zeta; their transpose multiplies
// by J and the metric at q after the transposed difference (channels X in
// the surface buffer).  The stress rows use the traction-free zeta
// derivative (rdz combination at the surface, two- and three-point one-sided
// differences below it); their transposes are folded into Phi or applied
// from channel w_z.
//
// Gradient: with mu_s the adjoint of the stored RHS h_s, the medium enters
// h_s at its own point only: h_V = buo (..), h_T = lambda div + mu E, so
//   dJ/dbuo += mu_s,V . h_V / buo,  dJ/dlambda += (mu_s,xx+yy+zz) DT div,
//   dJ/dmu   += (mu_s,T . h_T - lambda DT div (mu_s,xx+yy+zz)) / mu,
// with DT div = (h_xx + h_yy + h_zz) / (3 lambda + 2 mu), plus, at the
// surface, the dependence of rdz on (mu, lambda).  PML cells get none: the
// absorbing layers are not part of the model.
#include "device.cuh"
#include "kernels.cuh"
#include "surface_matrix.cuh"

#ifndef ADJ_TY
#define ADJ_TY 4            // block rows (the block is 32 x ADJ_TY points of one plane)
#endif
// minimum resident blocks per SM (a register cap) of each pass: 4 (no
// spills) and 5; 5 and 5 spilled 156 bytes in the first pass and measured
// 2 % slower in the adjoint steps; the uncapped 4 and 5, 3 % slower
#ifndef ADJ_MINB_PRE
#define ADJ_MINB_PRE 4
#endif
#ifndef ADJ_MINB_GATHER
#define ADJ_MINB_GATHER 5
#endif
#ifdef ADJ_MINB_PRE
#define ADJ_BOUNDS_PRE __launch_bounds__(32 * ADJ_TY, ADJ_MINB_PRE)
#else
#define ADJ_BOUNDS_PRE __launch_bounds__(32 * ADJ_TY)
#endif
#ifdef ADJ_MINB_GATHER
#define ADJ_BOUNDS_GATHER __launch_bounds__(32 * ADJ_TY, ADJ_MINB_GATHER)
#else
#define ADJ_BOUNDS_GATHER __launch_bounds__(32 * ADJ_TY)
#endif

// 1: the two-pass kernels' stores (Phi, the next mu, lambda, the gradient)
// evict-first: each is read back by a later launch, after L2 has turned over
#ifndef ADJ_STREAM_HINTS
#define ADJ_STREAM_HINTS 0
#endif
#if ADJ_STREAM_HINTS
#define AD_ST(p, v) __stcs(&(p), (v))
#else
#define AD_ST(p, v) ((p) = (v))
#endif

namespace cgfdm {

// dir_rhs^T: the 9-vector adjoint of the nine scaled derivatives along one
// direction, given the adjoint nu of that direction's RHS contribution.
__device__ __forceinline__ void dir_rhs_t(float m0, float m1, float m2, const float nu[9], float mu, float lam,
                                          float buo, float phi[9])
{
    const float W = (nu[3] + nu[4]) + nu[5];
    const float m2mu = 2.0f * mu;
    phi[0] = lam * m0 * W + m2mu * m0 * nu[3] + mu * (m1 * nu[6] + m2 * nu[7]);
    phi[1] = lam * m1 * W + m2mu * m1 * nu[4] + mu * (m0 * nu[6] + m2 * nu[8]);
    phi[2] = lam * m2 * W + m2mu * m2 * nu[5] + mu * (m0 * nu[7] + m1 * nu[8]);
    phi[3] = buo * m0 * nu[0];
    phi[4] = buo * m1 * nu[1];
    phi[5] = buo * m2 * nu[2];
    phi[6] = buo * (m1 * nu[0] + m0 * nu[1]);
    phi[7] = buo * (m2 * nu[0] + m0 * nu[2]);
    phi[8] = buo * (m2 * nu[1] + m1 * nu[2]);
}

// dir_stress^T: adjoint of the three velocity derivatives from the stress
// adjoint w[3..8].
__device__ __forceinline__ void dir_stress_t(float m0, float m1, float m2, const float w[9], float mu, float lam,
                                             float out[3])
{
    const float W = (w[3] + w[4]) + w[5];
    const float m2mu = 2.0f * mu;
    out[0] = lam * m0 * W + m2mu * m0 * w[3] + mu * (m1 * w[6] + m2 * w[7]);
    out[1] = lam * m1 * W + m2mu * m1 * w[4] + mu * (m0 * w[6] + m2 * w[8]);
    out[2] = lam * m2 * W + m2mu * m2 * w[5] + mu * (m0 * w[7] + m1 * w[8]);
}

// index of point (i, j, k) in face fc's slab (the forward's layout)
__device__ __forceinline__ long long face_pos(const DevGrid &g, int fc, int n, int i, int j, int k)
{
    const int i0p = i - CGFDM_HALO, j0p = j - CGFDM_HALO, k0p = k - CGFDM_HALO;
    if (fc == 0 || fc == 3)
        return (long long)(i0p - (fc == 3 ? g.nx - n : 0)) + (long long)j0p * n + (long long)k0p * n * g.ny;
    if (fc == 1 || fc == 4)
        return (long long)i0p + (long long)(j0p - (fc == 4 ? g.ny - n : 0)) * g.nx + (long long)k0p * g.nx * n;
    return (long long)i0p + (long long)j0p * g.nx + (long long)k0p * g.nx * g.ny;
}

// --------------------------------------------------------------- pass 1
// Point-wise: Phi_d(p) for the three directions, the surface channels and
// the RK4 adjoint of the PML auxiliaries.
__global__ void ADJ_BOUNDS_PRE k_adj_pre(const __grid_constant__ AdjStageArgs a)
{
    const DevGrid g = a.g;
    const int i = CGFDM_HALO + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = CGFDM_HALO + blockIdx.y * blockDim.y + threadIdx.y;
    const int k = CGFDM_HALO + blockIdx.z;
    const int _nx = g.nxp - CGFDM_HALO, _ny = g.nyp - CGFDM_HALO, _nz = g.nzp - CGFDM_HALO;
    if (i >= _nx || j >= _ny) return;
    const long long F = g.fstride, q = g.at(i, j, k), s = g.at2(i, j), P = g.plane;
    const float DT = a.DT;

    float mu_s[9];
    if (a.irk == 3)
        for (int f = 0; f < 9; f++) mu_s[f] = RK_BETA4 * a.Lp[f * F + q];
    else
        for (int f = 0; f < 9; f++) mu_s[f] = a.M[f * F + q];
    float mt[3][3];
    for (int d = 0; d < 3; d++)
        for (int c = 0; c < 3; c++) mt[d][c] = a.cjm[(3 * d + c) * F + q];
    const float mu = a.cjm[C_MU * F + q], lam = a.cjm[C_LAMBDA * F + q], buo = a.cjm[C_BUOY * F + q];
    const float sd[3] = {a.pml_beta_x[i], a.pml_beta_y[j], a.pml_beta_z[k]};
    const bool fs = a.fs_on && k >= _nz - 3;
    const bool top = a.fs_on && k == _nz - 1;

    // per direction: the adjoint of R_d(p) times the scaled derivatives
    float nu[3][9], extra[3][3];
#pragma unroll
    for (int d = 0; d < 3; d++) {
        for (int f = 0; f < 9; f++) nu[d][f] = (DT * sd[d]) * mu_s[f];
        // free surface: velocity rows are handled at the tap points, and the
        // zeta derivative of the stress rows is not a 5-point difference
        if (fs) {
            for (int f = 0; f < 3; f++) nu[d][f] = 0.0f;
            if (d == 2)
                for (int f = 3; f < 9; f++) nu[d][f] = 0.0f;
        }
        extra[d][0] = extra[d][1] = extra[d][2] = 0.0f;
    }
    float w_top[9];   // DT * the stress adjoint at the surface, for the rdz terms
    if (top) {
        for (int f = 3; f < 9; f++) w_top[f] = DT * mu_s[f];
        float wz[3];
        dir_stress_t(mt[2][0], mt[2][1], mt[2][2], w_top, mu, lam, wz);
#pragma unroll
        for (int d = 0; d < 2; d++)
#pragma unroll
            for (int c = 0; c < 3; c++) {
                const float *r = a.rdz + (long long)(d * 9) * P + s;
                float v = 0.0f;
                for (int rr = 0; rr < 3; rr++) v += r[(rr * 3 + c) * P] * wz[rr];
                extra[d][c] += sd[d] * v;
            }
    }

    // PML faces in the forward's order x1 y1 z1 x2 y2 (src/pml_deriv.cpp:633-646)
    if (a.pml_on) {
        const int n = a.nPML;
        const bool sel[5] = {i < CGFDM_HALO + n, j < CGFDM_HALO + n, k < CGFDM_HALO + n, i >= _nx - n, j >= _ny - n};
        const int i0p = i - CGFDM_HALO, j0p = j - CGFDM_HALO, k0p = k - CGFDM_HALO;
#pragma unroll
        for (int fc = 0; fc < 5; fc++) {
            if (!sel[fc]) continue;
            const int dir = fc == 0 || fc == 3 ? 0 : fc == 1 || fc == 4 ? 1 : 2;
            const PmlFace &Pf = a.face[fc];
            long long pos;
            if (dir == 0)
                pos = (long long)(i0p - (fc == 3 ? g.nx - n : 0)) + (long long)j0p * n + (long long)k0p * n * g.ny;
            else if (dir == 1)
                pos = (long long)i0p + (long long)(j0p - (fc == 4 ? g.ny - n : 0)) * g.nx +
                      (long long)k0p * g.nx * n;
            else
                pos = (long long)i0p + (long long)j0p * g.nx + (long long)k0p * g.nx * g.ny;
            const float *al = dir == 0 ? a.pml_alpha_x : dir == 1 ? a.pml_alpha_y : a.pml_alpha_z;
            const float *be = dir == 0 ? a.pml_beta_x : dir == 1 ? a.pml_beta_y : a.pml_beta_z;
            const float *dd = dir == 0 ? a.pml_d_x : dir == 1 ? a.pml_d_y : a.pml_d_z;
            const int ix = dir == 0 ? i : dir == 1 ? j : k;
            const float dval = dd[ix], beta = be[ix], alpha_d = dval + al[ix];
            // the face's lambda', mu and running sum, all loaded before any store
            float fa[9], muA[9], ft[9];
#pragma unroll
            for (int f = 0; f < 9; f++) {
                const long long e = f * Pf.count + pos;
                fa[f] = a.irk != 0 ? Pf.A[e] : 0.0f;
                muA[f] = a.irk == 3 ? RK_BETA4 * fa[f] : Pf.B[e];
                ft[f] = a.irk != 3 ? Pf.T[e] : 0.0f;
            }
            for (int f = 0; f < 9; f++) nu[dir][f] += (DT * dval) * muA[f];
            if (top && dir < 2) {
                // src/pml_freeSurface.cpp:90-125: the auxiliary's stress rows
                // also take the traction-free zeta derivative
                float w[9], wz[3];
                for (int f = 3; f < 9; f++) w[f] = DT * muA[f];
                dir_stress_t(mt[2][0], mt[2][1], mt[2][2], w, mu, lam, wz);
                for (int c = 0; c < 3; c++) {
                    const float *r = a.rdz + (long long)(dir * 9) * P + s;
                    float v = 0.0f;
                    for (int rr = 0; rr < 3; rr++) v += r[(rr * 3 + c) * P] * wz[rr];
                    extra[dir][c] += dval * v;
                }
            }
            // RK4 adjoint of the auxiliary (src/pml_rk.cpp:18-73)
            const float rb = a.irk == 3 ? RK_BETA3 : a.irk == 2 ? RK_BETA2 : RK_BETA1;
            const float ra = a.irk == 3 ? 1.0f : a.irk == 2 ? RK_ALPHA3 : RK_ALPHA2;
#pragma unroll
            for (int f = 0; f < 9; f++) {
                const float nuA = -DT * (alpha_d * muA[f] + beta * mu_s[f]);
                const long long e = f * Pf.count + pos;
                if (a.irk != 0) Pf.B[e] = rb * fa[f] + ra * nuA;
                Pf.T[e] = (a.irk == 3 ? fa[f] : ft[f]) + nuA;
            }
        }
    }

#pragma unroll
    for (int d = 0; d < 3; d++) {
        float phi[9];
        dir_rhs_t(mt[d][0], mt[d][1], mt[d][2], nu[d], mu, lam, buo, phi);
        for (int c = 0; c < 3; c++) phi[c] += extra[d][c];
        for (int f = 0; f < 9; f++) AD_ST(a.Phi[(d * 9 + f) * F + q], phi[f]);
    }

    if (fs) {
        // velocity rows: DT buo / J mu_V, stretched per direction; stress
        // rows below the surface: the adjoint of their zeta derivative
        const int L = _nz - 1 - k;
        float *sf = a.SF + (long long)(L * 12) * P + s;
        const float bj = buo * (1.0f / a.cjm[C_JAC * F + q]);
        for (int c = 0; c < 3; c++) {
            const float chi = DT * bj * mu_s[c];
            sf[c * P] = sd[0] * chi;
            sf[(3 + c) * P] = sd[1] * chi;
            sf[(6 + c) * P] = chi;
        }
        float w[9], wz[3] = {0.0f, 0.0f, 0.0f};
        if (!top) {
            for (int f = 3; f < 9; f++) w[f] = DT * mu_s[f];
            dir_stress_t(mt[2][0], mt[2][1], mt[2][2], w, mu, lam, wz);
        }
        for (int c = 0; c < 3; c++) sf[(9 + c) * P] = wz[c];
    }
}

// --------------------------------------------------------------- pass 2
__device__ __forceinline__ float tap_sum(const float *__restrict__ f, long long q, long long step, int FB)
{
    // sum_m a_m f(q - (m - 1) FB step): the transposed one-sided difference
    const long long o = (long long)FB * step;
    float s = CG_AF_1 * f[q + o] + CG_AF0 * f[q];
    s = s + CG_AF1 * f[q - o];
    s = s + CG_AF2 * f[q - 2 * o];
    s = s + CG_AF3 * f[q - 3 * o];
    return s;
}

__global__ void ADJ_BOUNDS_GATHER k_adj_gather(const __grid_constant__ AdjStageArgs a)
{
    const DevGrid g = a.g;
    const int i = CGFDM_HALO + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = CGFDM_HALO + blockIdx.y * blockDim.y + threadIdx.y;
    const int k = CGFDM_HALO + blockIdx.z;
    const int _nx = g.nxp - CGFDM_HALO, _ny = g.nyp - CGFDM_HALO, _nz = g.nzp - CGFDM_HALO;
    if (i >= _nx || j >= _ny) return;
    const long long F = g.fstride, q = g.at(i, j, k), s = g.at2(i, j), P = g.plane;
    const float rDH = a.rDH, DT = a.DT;
    const int FB1 = a.FB1, FB2 = a.FB2, FB3 = a.FB3;

    float nu[9];
    for (int f = 0; f < 9; f++) {
        const float sx = tap_sum(a.Phi + (0 * 9 + f) * F, q, 1, FB1);
        const float sy = tap_sum(a.Phi + (1 * 9 + f) * F, q, g.pitch, FB2);
        const float sz = tap_sum(a.Phi + (2 * 9 + f) * F, q, P, FB3);
        nu[f] = (((float)FB1 * sx) * rDH + ((float)FB2 * sy) * rDH) + ((float)FB3 * sz) * rDH;
    }

    if (a.fs_on && k >= _nz - 6) {
        // stress adjoint at q from the surface points' velocity rows
        float px[3] = {0, 0, 0}, py[3] = {0, 0, 0}, pz[3] = {0, 0, 0};
        if (k >= _nz - 3) {
            const float *sf = a.SF + (long long)((_nz - 1 - k) * 12) * P;
            for (int c = 0; c < 3; c++) {
                px[c] = ((float)FB1 * tap_sum(sf + c * P, s, 1, FB1)) * rDH;
                py[c] = ((float)FB2 * tap_sum(sf + (3 + c) * P, s, g.pitch, FB2)) * rDH;
            }
        }
        const float af[5] = {CG_AF_1, CG_AF0, CG_AF1, CG_AF2, CG_AF3};
        for (int L = 0; L < 3; L++) {
            const int kp = _nz - 1 - L, ks_rel = L + 3;
            const float *sf = a.SF + (long long)(L * 12) * P + s;
            for (int m = 0; m < 5; m++) {
                const int l = 3 + (m - 1) * FB3;
                int src = l;
                float sign = 1.0f;
                if (l > ks_rel) src = 2 * ks_rel - l, sign = -1.0f;
                if (src == ks_rel || kp + src - 3 != k) continue;
                const float w = sign * ((float)FB3 * af[m]) * rDH;
                for (int c = 0; c < 3; c++) pz[c] += w * sf[(6 + c) * P];
            }
        }
        const float jac = a.cjm[C_JAC * F + q];
        float mt[3][3];
        for (int d = 0; d < 3; d++)
            for (int c = 0; c < 3; c++) mt[d][c] = a.cjm[(3 * d + c) * F + q];
        const float *ps[3] = {px, py, pz};
        for (int d = 0; d < 3; d++) {
            const float m0 = mt[d][0], m1 = mt[d][1], m2 = mt[d][2], *p = ps[d];
            nu[3] += jac * (m0 * p[0]);
            nu[4] += jac * (m1 * p[1]);
            nu[5] += jac * (m2 * p[2]);
            nu[6] += jac * (m1 * p[0] + m0 * p[1]);
            nu[7] += jac * (m2 * p[0] + m0 * p[2]);
            nu[8] += jac * (m2 * p[1] + m1 * p[2]);
        }
        // velocity adjoint from the two- and three-point zeta derivatives
        {
            const float *w1 = a.SF + (long long)(1 * 12 + 9) * P + s;   // k = _nz - 2
            const int kp = _nz - 2;
            const float c1 = (float)FB3 * rDH;
            if (k == kp + FB3)
                for (int c = 0; c < 3; c++) nu[c] += c1 * w1[c * P];
            if (k == kp)
                for (int c = 0; c < 3; c++) nu[c] -= c1 * w1[c * P];
            const float *w2 = a.SF + (long long)(2 * 12 + 9) * P + s;   // k = _nz - 3
            const int kp2 = _nz - 3;
            const float cf[3] = {CG_CF1, CG_CF2, CG_CF3};
            for (int n = 0; n < 3; n++)
                if (k == kp2 + n * FB3)
                    for (int c = 0; c < 3; c++) nu[c] += (c1 * cf[n]) * w2[c * P];
        }
    }

    // RK4 adjoint (src/wave_rk.cpp:17-104 transposed).  Every operand is
    // loaded before the first store, so the loads issue together.
    const int irk = a.irk;
    const bool grad = a.h && a.hbox.contains(i, j, k);
    const long long hq = grad ? a.hbox.at(i, j, k) : 0;
    float mus[9], lp[9], lm[9], h[9], g3[3], mu = 0.0f, lam = 0.0f, buo = 1.0f;
#pragma unroll
    for (int f = 0; f < 9; f++) {
        lp[f] = irk != 0 ? a.Lp[f * F + q] : 0.0f;
        mus[f] = irk == 3 ? RK_BETA4 * lp[f] : a.M[f * F + q];
        lm[f] = irk != 3 ? a.Lam[f * F + q] : 0.0f;
        h[f] = grad ? a.h[f * a.hbox.fstride + hq] : 0.0f;
    }
    if (grad) {
        for (int c = 0; c < 3; c++) g3[c] = a.grad[c * F + q];
        mu = a.cjm[C_MU * F + q], lam = a.cjm[C_LAMBDA * F + q], buo = a.cjm[C_BUOY * F + q];
    }
    const float beta = irk == 3 ? RK_BETA3 : irk == 2 ? RK_BETA2 : RK_BETA1;
    const float alpha = irk == 3 ? 1.0f : irk == 2 ? RK_ALPHA3 : RK_ALPHA2;
#pragma unroll
    for (int f = 0; f < 9; f++) {
        if (irk != 0) AD_ST(a.M[f * F + q], beta * lp[f] + alpha * nu[f]);
        AD_ST(a.Lam[f * F + q], (irk == 3 ? lp[f] : lm[f]) + nu[f]);
    }

    if (!grad) return;
    const float gb = ((mus[0] * h[0] + mus[1] * h[1]) + mus[2] * h[2]) / buo;
    const float ddiv = ((h[3] + h[4]) + h[5]) / (3.0f * lam + 2.0f * mu);
    float gl = ((mus[3] + mus[4]) + mus[5]) * ddiv;
    float th = 0.0f;
    for (int f = 3; f < 9; f++) th += mus[f] * h[f];
    float gm = (th - lam * gl) / mu;
    if (a.fs_on && k == _nz - 1 && a.vd && a.drdz) {
        float w[9], wz[3];
        for (int f = 3; f < 9; f++) w[f] = DT * mus[f];
        dir_stress_t(a.cjm[C_ZT_X * F + q], a.cjm[C_ZT_Y * F + q], a.cjm[C_ZT_Z * F + q], w, mu, lam, wz);
        float vd[6];
        for (int c = 0; c < 6; c++) vd[c] = a.vd[c * P + s];
        for (int par = 0; par < 2; par++) {
            const float *dx = a.drdz + (long long)(par * 18) * P + s;
            const float *dy = a.drdz + (long long)(par * 18 + 9) * P + s;
            float acc = 0.0f;
            for (int r = 0; r < 3; r++) {
                float dv = 0.0f;
                for (int c = 0; c < 3; c++) dv += dx[(r * 3 + c) * P] * vd[c] + dy[(r * 3 + c) * P] * vd[3 + c];
                acc += wz[r] * dv;
            }
            if (par == 0) gm += acc;
            else gl += acc;
        }
    }
    AD_ST(a.grad[0 * F + q], g3[0] + gm);
    AD_ST(a.grad[1 * F + q], g3[1] + gl);
    AD_ST(a.grad[2 * F + q], g3[2] + gb);
}

cudaError_t launch_adj_stage(const AdjStageArgs &a, cudaStream_t st)
{
    dim3 b(32, ADJ_TY), gr((a.g.nx + 31) / 32, (a.g.ny + ADJ_TY - 1) / ADJ_TY, a.g.nz);
    k_adj_pre<<<gr, b, 0, st>>>(a);
    CUDA_TRY(cudaGetLastError());
    k_adj_gather<<<gr, b, 0, st>>>(a);
    return cudaGetLastError();
}

// ----------------------------------------------------------- fused stage
// One kernel per RK stage.  A block of 32 x ADJF_TY columns walks a chunk
// of planes upward.  Each thread keeps Phi_z of its own column for the last
// five planes (private shared-memory slots); for every output plane the
// block fills Phi_x over its rows with a 3-point halo in x and Phi_y over
// its columns with a 3-point halo in y in shared memory (with the surface
// layers' velocity-row channels), and every thread gathers its transposed
// differences.  Phi never goes to HBM.  Blocks read mu_s (and the faces'
// mu_s) at their neighbours' points while those write mu_{s-1}, so the
// output goes to a second buffer (M2, faceB2) that the host swaps in.
#ifndef ADJF_TY
#define ADJF_TY 8
#endif
#define ADJF_BX (32 + 6)
#define ADJF_BY (ADJF_TY + 6)
#define ADJF_NT (32 * ADJF_TY)
#define ADJF_SMEM_FLOATS (12 * ADJF_TY * ADJF_BX + 12 * ADJF_BY * 32 + 5 * 9 * ADJF_NT + 15 * ADJF_NT)

__device__ __forceinline__ void load_mu_s(const AdjStageArgs &a, long long q, long long F, float m[9])
{
#pragma unroll
    for (int f = 0; f < 9; f++) m[f] = a.irk == 3 ? RK_BETA4 * a.Lp[f * F + q] : a.M[f * F + q];
}

// Phi_d at interior point (i, j, k), as k_adj_pre forms it; with X given,
// also the surface layers' velocity-row channel of direction d
// (DT buo / J mu_V, times the stretch s_d for d < 2).
__device__ void phi_point(const AdjStageArgs &a, int d, int i, int j, int k, float phi[9], float *X)
{
    const DevGrid &g = a.g;
    const int _nx = g.nxp - CGFDM_HALO, _ny = g.nyp - CGFDM_HALO, _nz = g.nzp - CGFDM_HALO;
    const long long F = g.fstride, q = g.at(i, j, k), P = g.plane;
    const float DT = a.DT;
    float m[9];
    load_mu_s(a, q, F, m);
    const float m0 = a.cjm[(3 * d + 0) * F + q], m1 = a.cjm[(3 * d + 1) * F + q], m2 = a.cjm[(3 * d + 2) * F + q];
    const float mu = a.cjm[C_MU * F + q], lam = a.cjm[C_LAMBDA * F + q], buo = a.cjm[C_BUOY * F + q];
    const int ix = d == 0 ? i : d == 1 ? j : k;
    const float sd = (d == 0 ? a.pml_beta_x : d == 1 ? a.pml_beta_y : a.pml_beta_z)[ix];
    const bool fs = a.fs_on && k >= _nz - 3, top = a.fs_on && k == _nz - 1;
    float nu[9];
#pragma unroll
    for (int f = 0; f < 9; f++) nu[f] = (DT * sd) * m[f];
    if (fs) {
        nu[0] = nu[1] = nu[2] = 0.0f;
        if (d == 2)
            for (int f = 3; f < 9; f++) nu[f] = 0.0f;
    }
    float extra[3] = {0.0f, 0.0f, 0.0f};
    const long long s = g.at2(i, j);
    if (top && d < 2) {
        float w[9], wz[3];
        for (int f = 3; f < 9; f++) w[f] = DT * m[f];
        dir_stress_t(a.cjm[C_ZT_X * F + q], a.cjm[C_ZT_Y * F + q], a.cjm[C_ZT_Z * F + q], w, mu, lam, wz);
        const float *r = a.rdz + (long long)(d * 9) * P + s;
        for (int c = 0; c < 3; c++) {
            float v = 0.0f;
            for (int rr = 0; rr < 3; rr++) v += r[(rr * 3 + c) * P] * wz[rr];
            extra[c] += sd * v;
        }
    }
    if (a.pml_on) {
        const int n = a.nPML;
        int fc = -1;
        if (d == 0) fc = i < CGFDM_HALO + n ? 0 : (i >= _nx - n ? 3 : -1);
        else if (d == 1) fc = j < CGFDM_HALO + n ? 1 : (j >= _ny - n ? 4 : -1);
        else fc = k < CGFDM_HALO + n ? 2 : -1;
        if (fc >= 0) {
            const PmlFace &Pf = a.face[fc];
            const long long pos = face_pos(g, fc, n, i, j, k);
            const float dval = (d == 0 ? a.pml_d_x : d == 1 ? a.pml_d_y : a.pml_d_z)[ix];
            float muA[9];
#pragma unroll
            for (int f = 0; f < 9; f++)
                muA[f] = a.irk == 3 ? RK_BETA4 * Pf.A[f * Pf.count + pos] : Pf.B[f * Pf.count + pos];
#pragma unroll
            for (int f = 0; f < 9; f++) nu[f] += (DT * dval) * muA[f];
            if (top && d < 2) {
                float w[9], wz[3];
                for (int f = 3; f < 9; f++) w[f] = DT * muA[f];
                dir_stress_t(a.cjm[C_ZT_X * F + q], a.cjm[C_ZT_Y * F + q], a.cjm[C_ZT_Z * F + q], w, mu, lam, wz);
                const float *r = a.rdz + (long long)(d * 9) * P + s;
                for (int c = 0; c < 3; c++) {
                    float v = 0.0f;
                    for (int rr = 0; rr < 3; rr++) v += r[(rr * 3 + c) * P] * wz[rr];
                    extra[c] += dval * v;
                }
            }
        }
    }
    dir_rhs_t(m0, m1, m2, nu, mu, lam, buo, phi);
    for (int c = 0; c < 3; c++) phi[c] += extra[c];
    if (X) {
        if (fs) {
            const float bj = buo * (1.0f / a.cjm[C_JAC * F + q]);
            for (int c = 0; c < 3; c++) {
                const float chi = DT * bj * m[c];
                X[c] = d < 2 ? sd * chi : chi;
            }
        } else {
            X[0] = X[1] = X[2] = 0.0f;
        }
    }
}

__global__ void __launch_bounds__(ADJF_NT) k_adj_fused(const __grid_constant__ AdjStageArgs a)
{
    extern __shared__ __align__(16) float adj_smem[];
    float(*sx)[ADJF_TY][ADJF_BX] = reinterpret_cast<float(*)[ADJF_TY][ADJF_BX]>(adj_smem);
    float(*sy)[ADJF_BY][32] = reinterpret_cast<float(*)[ADJF_BY][32]>(adj_smem + 12 * ADJF_TY * ADJF_BX);
    float(*zr)[9][ADJF_NT] =
        reinterpret_cast<float(*)[9][ADJF_NT]>(adj_smem + 12 * ADJF_TY * ADJF_BX + 12 * ADJF_BY * 32);
    float(*fz)[ADJF_NT] = reinterpret_cast<float(*)[ADJF_NT]>(adj_smem + 12 * ADJF_TY * ADJF_BX +
                                                             12 * ADJF_BY * 32 + 5 * 9 * ADJF_NT);
    const DevGrid g = a.g;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * 32 + tx;
    const int i0 = CGFDM_HALO + blockIdx.x * 32, j0 = CGFDM_HALO + blockIdx.y * ADJF_TY;
    const int i = i0 + tx, j = j0 + ty;
    const int _nx = g.nxp - CGFDM_HALO, _ny = g.nyp - CGFDM_HALO, _nz = g.nzp - CGFDM_HALO;
    const bool active = i < _nx && j < _ny;
    const int kb = CGFDM_HALO + blockIdx.z * a.kchunk, ke = min(kb + a.kchunk, _nz);
    const long long F = g.fstride, P = g.plane;
    const float rDH = a.rDH, DT = a.DT;
    const int FB1 = a.FB1, FB2 = a.FB2, FB3 = a.FB3;
    const int lag = FB3 > 0 ? 1 : 3, lo = FB3 > 0 ? 3 : 1;
    const long long s = active ? g.at2(i, j) : 0;

    // the own column's surface channels: X_z of the three surface layers
    // and w_z of the two below the surface (k_adj_pre's SF channels 6-11)
    const bool near_top = a.fs_on && ke > _nz - 7;
    if (near_top && active) {
        for (int L = 0; L < 3; L++) {
            const int k = _nz - 1 - L;
            const long long q = g.at(i, j, k);
            float m[9];
            load_mu_s(a, q, F, m);
            const float buo = a.cjm[C_BUOY * F + q];
            const float bj = buo * (1.0f / a.cjm[C_JAC * F + q]);
            for (int c = 0; c < 3; c++) fz[L * 3 + c][tid] = DT * bj * m[c];
            if (L > 0) {
                float w[9], wz[3];
                for (int f = 3; f < 9; f++) w[f] = DT * m[f];
                dir_stress_t(a.cjm[C_ZT_X * F + q], a.cjm[C_ZT_Y * F + q], a.cjm[C_ZT_Z * F + q], w,
                             a.cjm[C_MU * F + q], a.cjm[C_LAMBDA * F + q], wz);
                for (int c = 0; c < 3; c++) fz[9 + (L - 1) * 3 + c][tid] = wz[c];
            }
        }
    }

    const int kfirst = kb - lo;
    auto slot = [&](int kk) { return (kk - kfirst) % 5; };
    for (int kin = kfirst; kin < ke + lag; kin++) {
        if (active) {
            float ph[9];
            if (kin >= CGFDM_HALO && kin < _nz) {
                phi_point(a, 2, i, j, kin, ph, nullptr);
            } else {
#pragma unroll
                for (int f = 0; f < 9; f++) ph[f] = 0.0f;
            }
            const int sl = slot(kin);
#pragma unroll
            for (int f = 0; f < 9; f++) zr[sl][f][tid] = ph[f];
        }
        const int kout = kin - lag;
        if (kout < kb) continue;
        const bool fsl = a.fs_on && kout >= _nz - 3;
        __syncthreads();   // the previous plane's readers of sx, sy are done
        for (int e = tid; e < ADJF_TY * ADJF_BX; e += ADJF_NT) {
            const int r = e / ADJF_BX, c = e - r * ADJF_BX;
            const int pi = i0 - 3 + c, pj = j0 + r;
            float ph[9], X[3] = {0.0f, 0.0f, 0.0f};
            if (pi >= CGFDM_HALO && pi < _nx && pj < _ny) {
                phi_point(a, 0, pi, pj, kout, ph, fsl ? X : nullptr);
            } else {
#pragma unroll
                for (int f = 0; f < 9; f++) ph[f] = 0.0f;
            }
#pragma unroll
            for (int f = 0; f < 9; f++) sx[f][r][c] = ph[f];
            for (int f = 0; f < 3; f++) sx[9 + f][r][c] = X[f];
        }
        for (int e = tid; e < ADJF_BY * 32; e += ADJF_NT) {
            const int r = e / 32, c = e - r * 32;
            const int pi = i0 + c, pj = j0 - 3 + r;
            float ph[9], X[3] = {0.0f, 0.0f, 0.0f};
            if (pi < _nx && pj >= CGFDM_HALO && pj < _ny) {
                phi_point(a, 1, pi, pj, kout, ph, fsl ? X : nullptr);
            } else {
#pragma unroll
                for (int f = 0; f < 9; f++) ph[f] = 0.0f;
            }
#pragma unroll
            for (int f = 0; f < 9; f++) sy[f][r][c] = ph[f];
            for (int f = 0; f < 3; f++) sy[9 + f][r][c] = X[f];
        }
        __syncthreads();
        if (!active) continue;

        // transposed differences: x and y from the planes in shared
        // memory, z from the column's ring
        const int cx = tx + 3, ry = ty + 3;
        const int sp1 = slot(kout + FB3), s0 = slot(kout), sm1 = slot(kout - FB3), sm2 = slot(kout - 2 * FB3),
                  sm3 = slot(kout - 3 * FB3);
        float nu[9];
#pragma unroll
        for (int f = 0; f < 9; f++) {
            float ax = CG_AF_1 * sx[f][ty][cx + FB1] + CG_AF0 * sx[f][ty][cx];
            ax = ax + CG_AF1 * sx[f][ty][cx - FB1];
            ax = ax + CG_AF2 * sx[f][ty][cx - 2 * FB1];
            ax = ax + CG_AF3 * sx[f][ty][cx - 3 * FB1];
            float ay = CG_AF_1 * sy[f][ry + FB2][tx] + CG_AF0 * sy[f][ry][tx];
            ay = ay + CG_AF1 * sy[f][ry - FB2][tx];
            ay = ay + CG_AF2 * sy[f][ry - 2 * FB2][tx];
            ay = ay + CG_AF3 * sy[f][ry - 3 * FB2][tx];
            float az = CG_AF_1 * zr[sp1][f][tid] + CG_AF0 * zr[s0][f][tid];
            az = az + CG_AF1 * zr[sm1][f][tid];
            az = az + CG_AF2 * zr[sm2][f][tid];
            az = az + CG_AF3 * zr[sm3][f][tid];
            nu[f] = (((float)FB1 * ax) * rDH + ((float)FB2 * ay) * rDH) + ((float)FB3 * az) * rDH;
        }
        const long long q = g.at(i, j, kout);

        if (a.fs_on && kout >= _nz - 6) {
            float px[3] = {0, 0, 0}, py[3] = {0, 0, 0}, pz[3] = {0, 0, 0};
            if (fsl) {
                for (int c = 0; c < 3; c++) {
                    float ax = CG_AF_1 * sx[9 + c][ty][cx + FB1] + CG_AF0 * sx[9 + c][ty][cx];
                    ax = ax + CG_AF1 * sx[9 + c][ty][cx - FB1];
                    ax = ax + CG_AF2 * sx[9 + c][ty][cx - 2 * FB1];
                    ax = ax + CG_AF3 * sx[9 + c][ty][cx - 3 * FB1];
                    float ay = CG_AF_1 * sy[9 + c][ry + FB2][tx] + CG_AF0 * sy[9 + c][ry][tx];
                    ay = ay + CG_AF1 * sy[9 + c][ry - FB2][tx];
                    ay = ay + CG_AF2 * sy[9 + c][ry - 2 * FB2][tx];
                    ay = ay + CG_AF3 * sy[9 + c][ry - 3 * FB2][tx];
                    px[c] = ((float)FB1 * ax) * rDH;
                    py[c] = ((float)FB2 * ay) * rDH;
                }
            }
            const float af[5] = {CG_AF_1, CG_AF0, CG_AF1, CG_AF2, CG_AF3};
            for (int L = 0; L < 3; L++) {
                const int kp = _nz - 1 - L, ks_rel = L + 3;
                for (int m = 0; m < 5; m++) {
                    const int l = 3 + (m - 1) * FB3;
                    int src = l;
                    float sign = 1.0f;
                    if (l > ks_rel) src = 2 * ks_rel - l, sign = -1.0f;
                    if (src == ks_rel || kp + src - 3 != kout) continue;
                    const float w = sign * ((float)FB3 * af[m]) * rDH;
                    for (int c = 0; c < 3; c++) pz[c] += w * fz[L * 3 + c][tid];
                }
            }
            const float jac = a.cjm[C_JAC * F + q];
            const float *ps[3] = {px, py, pz};
            for (int d = 0; d < 3; d++) {
                const float m0 = a.cjm[(3 * d) * F + q], m1 = a.cjm[(3 * d + 1) * F + q],
                            m2 = a.cjm[(3 * d + 2) * F + q];
                const float *p = ps[d];
                nu[3] += jac * (m0 * p[0]);
                nu[4] += jac * (m1 * p[1]);
                nu[5] += jac * (m2 * p[2]);
                nu[6] += jac * (m1 * p[0] + m0 * p[1]);
                nu[7] += jac * (m2 * p[0] + m0 * p[2]);
                nu[8] += jac * (m2 * p[1] + m1 * p[2]);
            }
            const float c1 = (float)FB3 * rDH;
            const int kp = _nz - 2;
            if (kout == kp + FB3)
                for (int c = 0; c < 3; c++) nu[c] += c1 * fz[9 + c][tid];
            if (kout == kp)
                for (int c = 0; c < 3; c++) nu[c] -= c1 * fz[9 + c][tid];
            const int kp2 = _nz - 3;
            const float cf[3] = {CG_CF1, CG_CF2, CG_CF3};
            for (int n = 0; n < 3; n++)
                if (kout == kp2 + n * FB3)
                    for (int c = 0; c < 3; c++) nu[c] += (c1 * cf[n]) * fz[12 + c][tid];
        }

        // point-wise: RK4 adjoint of the wavefield and the auxiliaries, gradient
        const int irk = a.irk;
        const bool grad = a.h && a.hbox.contains(i, j, kout);
        const long long hq = grad ? a.hbox.at(i, j, kout) : 0;
        float mus[9], lp[9], lm[9], h[9], g3[3] = {0.0f, 0.0f, 0.0f}, mu = 0.0f, lam = 0.0f, buo = 1.0f;
#pragma unroll
        for (int f = 0; f < 9; f++) {
            lp[f] = irk != 0 ? a.Lp[f * F + q] : 0.0f;
            mus[f] = irk == 3 ? RK_BETA4 * lp[f] : a.M[f * F + q];
            lm[f] = irk != 3 ? a.Lam[f * F + q] : 0.0f;
            h[f] = grad ? a.h[f * a.hbox.fstride + hq] : 0.0f;
        }
        if (grad) {
            for (int c = 0; c < 3; c++) g3[c] = a.grad[c * F + q];
            mu = a.cjm[C_MU * F + q], lam = a.cjm[C_LAMBDA * F + q], buo = a.cjm[C_BUOY * F + q];
        }
        const float beta = irk == 3 ? RK_BETA3 : irk == 2 ? RK_BETA2 : RK_BETA1;
        const float alpha = irk == 3 ? 1.0f : irk == 2 ? RK_ALPHA3 : RK_ALPHA2;
#pragma unroll
        for (int f = 0; f < 9; f++) {
            if (irk != 0) a.M2[f * F + q] = beta * lp[f] + alpha * nu[f];
            a.Lam[f * F + q] = (irk == 3 ? lp[f] : lm[f]) + nu[f];
        }
        if (a.pml_on) {
            const int n = a.nPML;
            const bool sel[5] = {i < CGFDM_HALO + n, j < CGFDM_HALO + n, kout < CGFDM_HALO + n, i >= _nx - n,
                                 j >= _ny - n};
#pragma unroll
            for (int fc = 0; fc < 5; fc++) {
                if (!sel[fc]) continue;
                const int dir = fc == 0 || fc == 3 ? 0 : fc == 1 || fc == 4 ? 1 : 2;
                const PmlFace &Pf = a.face[fc];
                const long long pos = face_pos(g, fc, n, i, j, kout);
                const int ix = dir == 0 ? i : dir == 1 ? j : kout;
                const float *al = dir == 0 ? a.pml_alpha_x : dir == 1 ? a.pml_alpha_y : a.pml_alpha_z;
                const float *be = dir == 0 ? a.pml_beta_x : dir == 1 ? a.pml_beta_y : a.pml_beta_z;
                const float *dd = dir == 0 ? a.pml_d_x : dir == 1 ? a.pml_d_y : a.pml_d_z;
                const float dval = dd[ix], pb = be[ix], alpha_d = dval + al[ix];
                float fa[9], muA[9], ft[9];
#pragma unroll
                for (int f = 0; f < 9; f++) {
                    const long long e = f * Pf.count + pos;
                    fa[f] = irk != 0 ? Pf.A[e] : 0.0f;
                    muA[f] = irk == 3 ? RK_BETA4 * fa[f] : Pf.B[e];
                    ft[f] = irk != 3 ? Pf.T[e] : 0.0f;
                }
                const float rb = irk == 3 ? RK_BETA3 : irk == 2 ? RK_BETA2 : RK_BETA1;
                const float ra = irk == 3 ? 1.0f : irk == 2 ? RK_ALPHA3 : RK_ALPHA2;
                float *B2 = a.faceB2[fc];
#pragma unroll
                for (int f = 0; f < 9; f++) {
                    const float nuA = -DT * (alpha_d * muA[f] + pb * mus[f]);
                    const long long e = f * Pf.count + pos;
                    if (irk != 0) B2[e] = rb * fa[f] + ra * nuA;
                    Pf.T[e] = (irk == 3 ? fa[f] : ft[f]) + nuA;
                }
            }
        }
        if (!grad) continue;
        const float gb = ((mus[0] * h[0] + mus[1] * h[1]) + mus[2] * h[2]) / buo;
        const float ddiv = ((h[3] + h[4]) + h[5]) / (3.0f * lam + 2.0f * mu);
        float gl = ((mus[3] + mus[4]) + mus[5]) * ddiv;
        float th = 0.0f;
        for (int f = 3; f < 9; f++) th += mus[f] * h[f];
        float gm = (th - lam * gl) / mu;
        if (a.fs_on && kout == _nz - 1 && a.vd && a.drdz) {
            float w[9], wz[3];
            for (int f = 3; f < 9; f++) w[f] = DT * mus[f];
            dir_stress_t(a.cjm[C_ZT_X * F + q], a.cjm[C_ZT_Y * F + q], a.cjm[C_ZT_Z * F + q], w, mu, lam, wz);
            float vd[6];
            for (int c = 0; c < 6; c++) vd[c] = a.vd[c * P + s];
            for (int par = 0; par < 2; par++) {
                const float *dx = a.drdz + (long long)(par * 18) * P + s;
                const float *dy = a.drdz + (long long)(par * 18 + 9) * P + s;
                float acc = 0.0f;
                for (int r = 0; r < 3; r++) {
                    float dv = 0.0f;
                    for (int c = 0; c < 3; c++) dv += dx[(r * 3 + c) * P] * vd[c] + dy[(r * 3 + c) * P] * vd[3 + c];
                    acc += wz[r] * dv;
                }
                if (par == 0) gm += acc;
                else gl += acc;
            }
        }
        a.grad[0 * F + q] = g3[0] + gm;
        a.grad[1 * F + q] = g3[1] + gl;
        a.grad[2 * F + q] = g3[2] + gb;
    }
}

cudaError_t launch_adj_stage_fused(const AdjStageArgs &a, cudaStream_t st)
{
    // per device and lost with a device reset: set on every launch
    const size_t smem = sizeof(float) * ADJF_SMEM_FLOATS;
    CUDA_TRY(cudaFuncSetAttribute(k_adj_fused, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 b(32, ADJF_TY), gr((a.g.nx + 31) / 32, (a.g.ny + ADJF_TY - 1) / ADJF_TY, a.nchunk);
    k_adj_fused<<<gr, b, smem, st>>>(a);
    return cudaGetLastError();
}

// ------------------------------------------------------------- residual
__global__ void k_adj_residual(float *Lp, DevGrid g, const int *__restrict__ idx, int nst, int NT, int n,
                               const float *__restrict__ res)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= nst * 3) return;
    const int st = t / 3, c = t - st * 3;
    const long long q = g.at(idx[st * 3 + 0], idx[st * 3 + 1], idx[st * 3 + 2]);
    atomicAdd(&Lp[c * g.fstride + q], res[((long long)st * NT + n) * 3 + c]);
}

cudaError_t launch_adj_residual(float *Lp, DevGrid g, const int *st_idx, int nst, int NT, int n, const float *res,
                                cudaStream_t st)
{
    if (nst <= 0) return cudaSuccess;
    k_adj_residual<<<(nst * 3 + 127) / 128, 128, 0, st>>>(Lp, g, st_idx, nst, NT, n, res);
    return cudaGetLastError();
}

// ------------------------------------------------- surface derivatives
// Forward-mode dual numbers in FP64: value and derivatives with respect to
// mu and lambda.
struct Dual {
    double v, dm, dl;
    __device__ Dual() {}
    __device__ Dual(float x) : v(x), dm(0.0), dl(0.0) {}
    __device__ Dual(double x, double a, double b) : v(x), dm(a), dl(b) {}
    __device__ Dual operator-() const { return Dual(-v, -dm, -dl); }
};
template <>
struct R<Dual> {
    static __device__ __forceinline__ Dual add(Dual a, Dual b) { return Dual(a.v + b.v, a.dm + b.dm, a.dl + b.dl); }
    static __device__ __forceinline__ Dual sub(Dual a, Dual b) { return Dual(a.v - b.v, a.dm - b.dm, a.dl - b.dl); }
    static __device__ __forceinline__ Dual mul(Dual a, Dual b)
    {
        return Dual(a.v * b.v, a.dm * b.v + a.v * b.dm, a.dl * b.v + a.v * b.dl);
    }
    static __device__ __forceinline__ Dual div(Dual a, Dual b)
    {
        const double r = 1.0 / b.v, qv = a.v * r;
        return Dual(qv, (a.dm - qv * b.dm) * r, (a.dl - qv * b.dl) * r);
    }
};

__global__ void k_surface_derivs(const float *__restrict__ cjm, DevGrid g, float *drdz)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x + CGFDM_HALO;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + CGFDM_HALO;
    if (i >= g.nxp - CGFDM_HALO || j >= g.nyp - CGFDM_HALO) return;
    const long long F = g.fstride, P = g.plane;
    const long long q = g.at(i, j, g.nzp - CGFDM_HALO - 1), s = g.at2(i, j);
    Dual m[9];
    for (int c = 0; c < 9; c++) m[c] = Dual(cjm[c * F + q]);
    const Dual mu((double)cjm[C_MU * F + q], 1.0, 0.0), lam((double)cjm[C_LAMBDA * F + q], 0.0, 1.0);
    Dual rx[9], ry[9];
    surface_matrices<Dual>(m, mu, lam, rx, ry);
    for (int e = 0; e < 9; e++) {
        drdz[e * P + s] = (float)rx[e].dm;
        drdz[(9 + e) * P + s] = (float)ry[e].dm;
        drdz[(18 + e) * P + s] = (float)rx[e].dl;
        drdz[(27 + e) * P + s] = (float)ry[e].dl;
    }
}

cudaError_t launch_surface_derivs(const float *cjm, DevGrid g, float *drdz, cudaStream_t st)
{
    dim3 b(32, 4), gr((g.nx + 31) / 32, (g.ny + 3) / 4);
    k_surface_derivs<<<gr, b, 0, st>>>(cjm, g, drdz);
    return cudaGetLastError();
}

// ---------------------------------------------------------- chain rule
// mu = rho Vs^2, lambda = rho (Vp^2 - 2 Vs^2), buoyancy = 1 / rho
// (src/CJM.cpp:52-77).
__global__ void k_grad_chain(const float *__restrict__ grad, const float *__restrict__ med, DevGrid g, float *out)
{
    const int ii = blockIdx.x * blockDim.x + threadIdx.x, jj = blockIdx.y * blockDim.y + threadIdx.y;
    const int kk = blockIdx.z;
    if (ii >= g.nx || jj >= g.ny) return;
    const int i = ii + CGFDM_HALO, j = jj + CGFDM_HALO, k = kk + CGFDM_HALO;
    const long long q = g.at(i, j, k), F = g.fstride;
    const long long n = ((long long)k * g.nyp + j) * g.nxp + i;
    const double vs = med[n * 3 + 0], vp = med[n * 3 + 1], rho = med[n * 3 + 2];
    const double gm = grad[q], gl = grad[F + q], gb = grad[2 * F + q];
    const long long o = ((long long)kk * g.ny + jj) * g.nx + ii, N = (long long)g.nx * g.ny * g.nz;
    out[o] = (float)(gl * 2.0 * rho * vp);
    out[N + o] = (float)(gm * 2.0 * rho * vs - gl * 4.0 * rho * vs);
    out[2 * N + o] = (float)(gm * vs * vs + gl * (vp * vp - 2.0 * vs * vs) - gb / (rho * rho));
}

cudaError_t launch_grad_chain(const float *grad, const float *medium, DevGrid g, float *out, cudaStream_t st)
{
    dim3 b(32, 4), gr((g.nx + 31) / 32, (g.ny + 3) / 4, g.nz);
    k_grad_chain<<<gr, b, 0, st>>>(grad, medium, g, out);
    return cudaGetLastError();
}

}  // namespace cgfdm
