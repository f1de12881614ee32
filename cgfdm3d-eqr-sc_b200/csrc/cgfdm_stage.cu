// Fused CGFDM Runge-Kutta stage for sm_100a.
//
// One launch does, for every interior point, what the reference does in up
// to fifteen launches per stage (src/propagate.cpp:212-251): the one-sided
// MacCormack derivatives with PML stretching (wave_deriv,
// src/wave_deriv.cpp:76-284), the traction-image free surface that
// overwrites the top three layers (free_surface_deriv,
// src/freeSurface.cpp:242-494), the CFS-PML auxiliary update and its
// correction of the RHS (pml_deriv_x/y/z, src/pml_deriv.cpp:125-584), the
// free-surface term of the PML auxiliaries (src/pml_freeSurface.cpp:16-242),
// and the RK4 update of both wavefield and auxiliaries (src/wave_rk.cpp:17-104,
// src/pml_rk.cpp:18-73).  In stage 3 it also updates the peak ground
// velocity (src/PGV.cpp:61-175) and, if enabled, the displacement
// (src/solve_displacement.cpp:27-63).
//
// Tiling: a CTA owns a 32 x 8 column tile and marches up a chunk of z.  The
// nine wavefield components of each z-plane, with the one-sided x/y halo
// the stencil needs (1 cell behind, 3 ahead, per the FB signs), are staged
// once into a six-slot shared-memory ring by cp.async; derivatives along
// x, y and z all read the ring, so each value crosses HBM once per stage.
// Everything else (metric, RK inputs, auxiliaries) is a coalesced
// structure-of-arrays load at the point itself.
//
// Arithmetic follows the reference's expression order term by term; built
// with --fmad=false the stage reproduces the reference's FP32 results bit for
// bit, built normally it differs only by FMA contraction.
#include "device.cuh"
#include "kernels.cuh"

namespace cgfdm {

#define TX 32
#define TY 8
#define HXW (TX + 4)
#define HYW (TY + 4)
#define PLANE_F (HXW * HYW)
#define PLANE (9 * PLANE_F)
#define NSLOT 6

size_t cg_stage_smem_bytes() { return (size_t)NSLOT * PLANE * sizeof(float); }

__device__ __forceinline__ void cp_async4(float *sdst, const float *gsrc, bool valid)
{
    unsigned s = (unsigned)__cvta_generic_to_shared(sdst);
    int n = valid ? 4 : 0;
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(s), "l"(gsrc), "r"(n) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::: "memory"); }

// Stage plane k of the nine components into one ring slot: rows
// j0-hyL .. j0-hyL+HYW-1, columns i0-hxL .. i0-hxL+HXW-1.  Cells beyond the
// padded grid (last tile only) are zero-filled and never used.
__device__ __forceinline__ void load_plane(float *slot, const float *__restrict__ W, const DevGrid &g, int i0,
                                           int j0, int hxL, int hyL, int k, int tid)
{
    const long long kb = (long long)k * g.plane + g.xoff;
    for (int e = tid; e < PLANE; e += TX * TY) {
        int f = e / PLANE_F;
        int r = e - f * PLANE_F;
        int yy = r / HXW;
        int xx = r - yy * HXW;
        int x = i0 - hxL + xx, y = j0 - hyL + yy;
        bool ok = (x < g.nxp) && (y < g.nyp);
        const float *src = ok ? W + f * g.fstride + kb + (long long)y * g.pitch + x : W;
        cp_async4(slot + e, src, ok);
    }
}

// Contribution of one grid direction to the RHS, given the metric row
// (xi, eta or zeta gradient) and the nine scaled derivatives along it
// (src/wave_deriv.cpp:244-272; the same form in pml_deriv and
// pml_free_surface).  out: Vx Vy Vz Txx Tyy Tzz Txy Txz Tyz.
__device__ __forceinline__ void dir_rhs(float m0, float m1, float m2, const float d[9], float mu, float lam,
                                        float buo, float out[9])
{
    out[0] = ((m0 * d[3] + m1 * d[6]) + m2 * d[7]) * buo;
    out[1] = ((m0 * d[6] + m1 * d[4]) + m2 * d[8]) * buo;
    out[2] = ((m0 * d[7] + m1 * d[8]) + m2 * d[5]) * buo;
    float dv = (m0 * d[0] + m1 * d[1]) + m2 * d[2];
    float m2mu = 2.0f * mu;
    out[3] = dv * lam + m2mu * (m0 * d[0]);
    out[4] = dv * lam + m2mu * (m1 * d[1]);
    out[5] = dv * lam + m2mu * (m2 * d[2]);
    out[6] = (m1 * d[0] + m0 * d[1]) * mu;
    out[7] = (m2 * d[0] + m0 * d[2]) * mu;
    out[8] = (m2 * d[1] + m1 * d[2]) * mu;
}

// stress part only (components 3..8) from velocity derivatives v[0..2]
__device__ __forceinline__ void dir_stress(float m0, float m1, float m2, const float v[3], float mu, float lam,
                                           float out[9])
{
    float dv = (m0 * v[0] + m1 * v[1]) + m2 * v[2];
    float m2mu = 2.0f * mu;
    out[3] = dv * lam + m2mu * (m0 * v[0]);
    out[4] = dv * lam + m2mu * (m1 * v[1]);
    out[5] = dv * lam + m2mu * (m2 * v[2]);
    out[6] = (m1 * v[0] + m0 * v[1]) * mu;
    out[7] = (m2 * v[0] + m0 * v[2]) * mu;
    out[8] = (m2 * v[1] + m1 * v[2]) * mu;
}

// One-sided 5-point operator of the L macro (src/axis.h:287):
// FB * (af_1 w[-FB] + af0 w[0] + af1 w[FB] + af2 w[2FB] + af3 w[3FB]) * rDH
__device__ __forceinline__ float lop(float wm, float w0, float w1, float w2, float w3, int FB, float rDH)
{
    float s = CG_AF_1 * wm + CG_AF0 * w0;
    s = s + CG_AF1 * w1;
    s = s + CG_AF2 * w2;
    s = s + CG_AF3 * w3;
    return ((float)FB * s) * rDH;
}

struct Ring {
    const float *ring;
    int base;  // (ty + hyL) * HXW + tx + hxL
    __device__ __forceinline__ float at(int kk, int f, int dx, int dy) const
    {
        return ring[(kk % NSLOT) * PLANE + f * PLANE_F + base + dy * HXW + dx];
    }
};

__device__ __forceinline__ float raw_x(const Ring &R, int k, int f, int FB, float rDH)
{
    return lop(R.at(k, f, -FB, 0), R.at(k, f, 0, 0), R.at(k, f, FB, 0), R.at(k, f, 2 * FB, 0),
               R.at(k, f, 3 * FB, 0), FB, rDH);
}
__device__ __forceinline__ float raw_y(const Ring &R, int k, int f, int FB, float rDH)
{
    return lop(R.at(k, f, 0, -FB), R.at(k, f, 0, 0), R.at(k, f, 0, FB), R.at(k, f, 0, 2 * FB),
               R.at(k, f, 0, 3 * FB), FB, rDH);
}
__device__ __forceinline__ float raw_z(const Ring &R, int k, int f, int FB, float rDH)
{
    return lop(R.at(k - FB, f, 0, 0), R.at(k, f, 0, 0), R.at(k + FB, f, 0, 0), R.at(k + 2 * FB, f, 0, 0),
               R.at(k + 3 * FB, f, 0, 0), FB, rDH);
}
__device__ __forceinline__ float raw_dir(const Ring &R, int dir, int k, int f, int FB, float rDH)
{
    return dir == 0 ? raw_x(R, k, f, FB, rDH) : dir == 1 ? raw_y(R, k, f, FB, rDH) : raw_z(R, k, f, FB, rDH);
}

// J * (metric . traction) at a point, for the traction image
// (src/freeSurface.cpp:358-395).  mdir: 0 xi, 1 eta, 2 zeta.
__device__ __forceinline__ void jt_at(const float *__restrict__ W, const float *__restrict__ cjm, long long F,
                                      long long q, int mdir, float out[3])
{
    float m0 = cjm[(3 * mdir + 0) * F + q], m1 = cjm[(3 * mdir + 1) * F + q], m2 = cjm[(3 * mdir + 2) * F + q];
    float jac = cjm[C_JAC * F + q];
    float Txx = W[3 * F + q], Tyy = W[4 * F + q], Tzz = W[5 * F + q];
    float Txy = W[6 * F + q], Txz = W[7 * F + q], Tyz = W[8 * F + q];
    out[0] = ((m0 * Txx + m1 * Txy) + m2 * Txz) * jac;
    out[1] = ((m0 * Txy + m1 * Tyy) + m2 * Tyz) * jac;
    out[2] = ((m0 * Txz + m1 * Tyz) + m2 * Tzz) * jac;
}

// L_J_T along x or y (src/axis.h:264): taps at offsets FB*(-1..3).
__device__ __forceinline__ void ljt_xy(const float *__restrict__ W, const float *__restrict__ cjm, const DevGrid &g,
                                       int i, int j, int k, int dir, int FB, float rDH, float out[3])
{
    float J[5][3];
    for (int m = 0; m < 5; m++) {
        int o = (m - 1) * FB;
        long long q = dir == 0 ? g.at(i + o, j, k) : g.at(i, j + o, k);
        jt_at(W, cjm, g.fstride, q, dir, J[m]);
    }
    for (int c = 0; c < 3; c++) out[c] = lop(J[0][c], J[1][c], J[2][c], J[3][c], J[4][c], FB, rDH);
}

// L_J_T along zeta with the antisymmetric image about the surface
// (src/freeSurface.cpp:384-405): J[l] for l < k_s from the field,
// J[k_s] = 0, J[l] = -J[2 k_s - l] above.
__device__ __forceinline__ void ljt_z(const float *__restrict__ W, const float *__restrict__ cjm, const DevGrid &g,
                                      int i, int j, int k, int ks_rel, int FB, float rDH, float out[3])
{
    float J[5][3];
    for (int m = 0; m < 5; m++) {
        int l = 3 + (m - 1) * FB;
        int src = l, sign = 1;
        if (l > ks_rel) src = 2 * ks_rel - l, sign = -1;
        if (src == ks_rel) {
            J[m][0] = J[m][1] = J[m][2] = 0.0f;
        } else {
            jt_at(W, cjm, g.fstride, g.at(i, j, k + src - 3), 2, J[m]);
            if (sign < 0) J[m][0] = -J[m][0], J[m][1] = -J[m][1], J[m][2] = -J[m][2];
        }
    }
    for (int c = 0; c < 3; c++) out[c] = lop(J[0][c], J[1][c], J[2][c], J[3][c], J[4][c], FB, rDH);
}

__global__ void __launch_bounds__(TX *TY, 2) k_cg_stage(const CgStageArgs a)
{
    extern __shared__ float ring[];
    const DevGrid g = a.g;
    const long long F = g.fstride;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    const int i0 = CGFDM_HALO + blockIdx.x * TX, j0 = CGFDM_HALO + blockIdx.y * TY;
    const int i = i0 + tx, j = j0 + ty;
    const int _nx = g.nxp - CGFDM_HALO, _ny = g.nyp - CGFDM_HALO, _nz = g.nzp - CGFDM_HALO;
    const bool active = i < _nx && j < _ny;
    const int kb = CGFDM_HALO + blockIdx.z * a.kchunk;
    const int ke = min(kb + a.kchunk, _nz);
    if (kb >= ke) return;
    const int FB1 = a.FB1, FB2 = a.FB2, FB3 = a.FB3;
    const int hxL = FB1 > 0 ? 1 : 3, hyL = FB2 > 0 ? 1 : 3, za = FB3 > 0 ? 1 : 3;
    const float rDH = a.rDH, DT = a.DT;
    const Ring R{ring, (ty + hyL) * HXW + tx + hxL};

    for (int q = 0; q < 5; q++) {
        int kk = kb - za + q;
        load_plane(ring + (kk % NSLOT) * PLANE, a.Win, g, i0, j0, hxL, hyL, kk, tid);
    }
    cp_async_commit();

    const float bx = active ? a.pml_beta_x[i] : 1.0f, by = active ? a.pml_beta_y[j] : 1.0f;
    const int nPML = a.nPML;
    const bool inx1 = a.pml_on && i < CGFDM_HALO + nPML, inx2 = a.pml_on && i >= _nx - nPML;
    const bool iny1 = a.pml_on && j < CGFDM_HALO + nPML, iny2 = a.pml_on && j >= _ny - nPML;

    for (int k = kb; k < ke; k++) {
        cp_async_wait_all();
        __syncthreads();
        if (k + 1 < ke) {
            int kk = k - za + 5;
            load_plane(ring + (kk % NSLOT) * PLANE, a.Win, g, i0, j0, hxL, hyL, kk, tid);
            cp_async_commit();
        }
        if (!active) continue;

        const long long q = g.at(i, j, k);
        const float xi_x = a.cjm[C_XI_X * F + q], xi_y = a.cjm[C_XI_Y * F + q], xi_z = a.cjm[C_XI_Z * F + q];
        const float et_x = a.cjm[C_ET_X * F + q], et_y = a.cjm[C_ET_Y * F + q], et_z = a.cjm[C_ET_Z * F + q];
        const float zt_x = a.cjm[C_ZT_X * F + q], zt_y = a.cjm[C_ZT_Y * F + q], zt_z = a.cjm[C_ZT_Z * F + q];
        const float mu = a.cjm[C_MU * F + q], lam = a.cjm[C_LAMBDA * F + q];
        const float buo = a.cjm[C_BUOY * F + q] * 1.0f;  // buoyancy *= Crho (= 1)
        const float bz = a.pml_beta_z[k];

        float h[9];
        const bool fs = a.fs_on && k >= _nz - 3;
        if (!fs) {
            // src/wave_deriv.cpp:214-282
            float d[9], c[9];
            for (int f = 0; f < 9; f++) d[f] = raw_x(R, k, f, FB1, rDH) * bx;
            dir_rhs(xi_x, xi_y, xi_z, d, mu, lam, buo, c);
            for (int f = 0; f < 9; f++) h[f] = c[f];
            for (int f = 0; f < 9; f++) d[f] = raw_y(R, k, f, FB2, rDH) * by;
            dir_rhs(et_x, et_y, et_z, d, mu, lam, buo, c);
            for (int f = 0; f < 9; f++) h[f] = h[f] + c[f];
            for (int f = 0; f < 9; f++) d[f] = raw_z(R, k, f, FB3, rDH) * bz;
            dir_rhs(zt_x, zt_y, zt_z, d, mu, lam, buo, c);
            for (int f = 0; f < 9; f++) h[f] = (h[f] + c[f]) * DT;
        } else {
            // src/freeSurface.cpp:345-492
            const int ks_rel = (_nz - 1) - k + CGFDM_HALO;
            float jx[3], jy[3], jz[3];
            ljt_xy(a.Win, a.cjm, g, i, j, k, 0, FB1, rDH, jx);
            ljt_xy(a.Win, a.cjm, g, i, j, k, 1, FB2, rDH, jy);
            ljt_z(a.Win, a.cjm, g, i, j, k, ks_rel, FB3, rDH, jz);
            const float jinv = 1.0f / a.cjm[C_JAC * F + q];
            const float bj = buo * jinv;
            for (int c = 0; c < 3; c++) h[c] = (bj * ((jx[c] * bx + jy[c] * by) + jz[c])) * DT;
            float vxi[3], vet[3], vzt[3];
            for (int c = 0; c < 3; c++) vxi[c] = raw_x(R, k, c, FB1, rDH) * bx;
            for (int c = 0; c < 3; c++) vet[c] = raw_y(R, k, c, FB2, rDH) * by;
            if (k == _nz - 1) {
                const long long s = g.at2(i, j);
                for (int r = 0; r < 3; r++) {
                    const float *dx = a.rdz + (long long)(r * 3) * g.plane + s;
                    const float *dy = a.rdz + (long long)(9 + r * 3) * g.plane + s;
                    vzt[r] = ((dx[0] * vxi[0] + dx[g.plane] * vxi[1]) + dx[2 * g.plane] * vxi[2]) +
                             ((dy[0] * vet[0] + dy[g.plane] * vet[1]) + dy[2 * g.plane] * vet[2]);
                }
            } else if (k == _nz - 2) {
                for (int c = 0; c < 3; c++)
                    vzt[c] = ((float)FB3 * (R.at(k + FB3, c, 0, 0) - R.at(k, c, 0, 0))) * rDH;
            } else {
                for (int c = 0; c < 3; c++)
                    vzt[c] = ((float)FB3 * ((CG_CF1 * R.at(k, c, 0, 0) + CG_CF2 * R.at(k + FB3, c, 0, 0)) +
                                            CG_CF3 * R.at(k + 2 * FB3, c, 0, 0))) *
                             rDH;
            }
            float s1[9], s2[9], s3[9];
            dir_stress(xi_x, xi_y, xi_z, vxi, mu, lam, s1);
            dir_stress(et_x, et_y, et_z, vet, mu, lam, s2);
            dir_stress(zt_x, zt_y, zt_z, vzt, mu, lam, s3);
            for (int f = 3; f < 9; f++) h[f] = ((s1[f] + s2[f]) + s3[f]) * DT;
        }

        // ---- PML auxiliaries, faces in the reference's launch order x1 y1 z1 x2 y2
        const bool inz1 = a.pml_on && k < CGFDM_HALO + nPML;
        if (inx1 || iny1 || inz1 || inx2 || iny2) {
            const int i0p = i - CGFDM_HALO, j0p = j - CGFDM_HALO, k0p = k - CGFDM_HALO;
            const int nx = g.nx, ny = g.ny;
            const bool sel[5] = {inx1, iny1, inz1, inx2, iny2};
            for (int fc = 0; fc < 5; fc++) {
                if (!sel[fc]) continue;
                const int dir = fc == 0 || fc == 3 ? 0 : fc == 1 || fc == 4 ? 1 : 2;
                const PmlFace &P = a.face[fc];
                long long pos;
                if (dir == 0) pos = (long long)(i0p - (fc == 3 ? nx - nPML : 0)) + (long long)j0p * nPML + (long long)k0p * nPML * ny;
                else if (dir == 1) pos = (long long)i0p + (long long)(j0p - (fc == 4 ? ny - nPML : 0)) * nx + (long long)k0p * nx * nPML;
                else pos = (long long)i0p + (long long)j0p * nx + (long long)k0p * nx * ny;
                const float *al = dir == 0 ? a.pml_alpha_x : dir == 1 ? a.pml_alpha_y : a.pml_alpha_z;
                const float *be = dir == 0 ? a.pml_beta_x : dir == 1 ? a.pml_beta_y : a.pml_beta_z;
                const float *dd = dir == 0 ? a.pml_d_x : dir == 1 ? a.pml_d_y : a.pml_d_z;
                const int ix = dir == 0 ? i : dir == 1 ? j : k;
                const int FB = dir == 0 ? FB1 : dir == 1 ? FB2 : FB3;
                const float dval = dd[ix], beta = be[ix], alpha_d = dval + al[ix];
                const float m0 = dir == 0 ? xi_x : dir == 1 ? et_x : zt_x;
                const float m1 = dir == 0 ? xi_y : dir == 1 ? et_y : zt_y;
                const float m2 = dir == 0 ? xi_z : dir == 1 ? et_z : zt_z;
                float d[9], rhs[9], aux[9], hA[9];
                for (int f = 0; f < 9; f++) d[f] = raw_dir(R, dir, k, f, FB, rDH) * dval;
                dir_rhs(m0, m1, m2, d, mu, lam, buo, rhs);
                const float *cur = a.irk == 0 ? P.A : P.B;
                for (int f = 0; f < 9; f++) aux[f] = cur[f * P.count + pos];
                for (int f = 0; f < 9; f++) hA[f] = (rhs[f] - alpha_d * aux[f]) * DT;
                if (a.fs_on && k == _nz - 1 && dir < 2) {
                    // src/pml_freeSurface.cpp:90-125
                    const long long s = g.at2(i, j);
                    float vz[3], t3[9];
                    for (int r = 0; r < 3; r++) {
                        const float *mr = a.rdz + (long long)(dir * 9 + r * 3) * g.plane + s;
                        vz[r] = (mr[0] * d[0] + mr[g.plane] * d[1]) + mr[2 * g.plane] * d[2];
                    }
                    dir_stress(zt_x, zt_y, zt_z, vz, mu, lam, t3);
                    for (int f = 3; f < 9; f++) hA[f] = hA[f] + t3[f] * DT;
                }
                for (int f = 0; f < 9; f++) h[f] = h[f] + (-beta * aux[f]) * DT;
                // src/pml_rk.cpp:18-73
                if (a.irk == 0) {
                    for (int f = 0; f < 9; f++) {
                        P.T[f * P.count + pos] = aux[f] + RK_BETA1 * hA[f];
                        P.B[f * P.count + pos] = aux[f] + RK_ALPHA2 * hA[f];
                    }
                } else if (a.irk == 1 || a.irk == 2) {
                    for (int f = 0; f < 9; f++) {
                        float mA = P.A[f * P.count + pos];
                        float t = P.T[f * P.count + pos];
                        P.T[f * P.count + pos] = t + (a.irk == 1 ? RK_BETA2 : RK_BETA3) * hA[f];
                        P.B[f * P.count + pos] = a.irk == 1 ? mA + RK_ALPHA3 * hA[f] : mA + hA[f];
                    }
                } else {
                    for (int f = 0; f < 9; f++) P.A[f * P.count + pos] = P.T[f * P.count + pos] + RK_BETA4 * hA[f];
                }
            }
        }

        // ---- RK4 update of the wavefield (src/wave_rk.cpp:17-104)
        float wout[9];
        if (a.irk == 0) {
            for (int f = 0; f < 9; f++) {
                float m = a.Wm[f * F + q];
                a.T[f * F + q] = m + RK_BETA1 * h[f];
                wout[f] = m + RK_ALPHA2 * h[f];
            }
        } else if (a.irk == 1 || a.irk == 2) {
            for (int f = 0; f < 9; f++) {
                float m = a.Wm[f * F + q];
                float t = a.T[f * F + q];
                a.T[f * F + q] = t + (a.irk == 1 ? RK_BETA2 : RK_BETA3) * h[f];
                wout[f] = a.irk == 1 ? m + RK_ALPHA3 * h[f] : m + h[f];
            }
        } else {
            for (int f = 0; f < 9; f++) wout[f] = a.T[f * F + q] + RK_BETA4 * h[f];
        }
        for (int f = 0; f < 9; f++) a.Wout[f * F + q] = wout[f];

        if (a.irk == 3) {
            if (a.dis)
                for (int c = 0; c < 3; c++) a.dis[c * F + q] = a.dis[c * F + q] + wout[c] * DT;
            if (a.pgv && k == _nz - 1) {
                long long pp = (long long)(i - CGFDM_HALO) + (long long)(j - CGFDM_HALO) * g.nx;
                float Vx = wout[0], Vy = wout[1], Vz = wout[2];
                float Vh = sqrtf(Vx * Vx + Vy * Vy);
                float V = sqrtf(Vx * Vx + Vy * Vy + Vz * Vz);
                if (a.pgv[pp * 2 + 0] < Vh) a.pgv[pp * 2 + 0] = Vh;
                if (a.pgv[pp * 2 + 1] < V) a.pgv[pp * 2 + 1] = V;
            }
        }
    }
}

cudaError_t launch_cg_stage(const CgStageArgs &a, cudaStream_t st)
{
    static bool attr_set = false;
    if (!attr_set) {
        CUDA_TRY(cudaFuncSetAttribute(k_cg_stage, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)cg_stage_smem_bytes()));
        attr_set = true;
    }
    dim3 block(TX, TY, 1);
    dim3 grid((a.g.nx + TX - 1) / TX, (a.g.ny + TY - 1) / TY, (a.g.nz + a.kchunk - 1) / a.kchunk);
    k_cg_stage<<<grid, block, cg_stage_smem_bytes(), st>>>(a);
    return cudaGetLastError();
}

}  // namespace cgfdm
