// GPU setup kernels: medium -> (mu, lambda, buoyancy), curvilinear metrics
// and Jacobian for both schemes, the free-surface matrices of the CGFDM
// traction image, and the moment-rate scaling of the finite-fault table.
//
// Every kernel is templated on the arithmetic type T.  T = float reproduces
// the reference's FP32 setup bit for bit: each operation is an explicitly
// rounded intrinsic in the reference's evaluation order, so no FMA
// contraction can change a result.  T = double is the FP64 setup (metrics
// and Jacobian evaluated in double, rounded once when stored).
#include <cstdio>

#include "device.cuh"
#include "kernels.cuh"
#include "surface_matrix.cuh"

namespace cgfdm {

// ------------------------------------------------------------- medium
// (Vs, Vp, rho) -> mu = rho Vs^2, lambda = rho (Vp^2 - 2 Vs^2), 1/rho
// (src/CJM.cpp:52-77), over the whole padded grid.
template <typename T>
__global__ void k_medium(const float *__restrict__ med, float *cjm, DevGrid g)
{
    long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long npad = (long long)g.nxp * g.nyp * g.nzp;
    if (n >= npad) return;
    int i = (int)(n % g.nxp), j = (int)((n / g.nxp) % g.nyp), k = (int)(n / ((long long)g.nxp * g.nyp));
    T vs = med[n * 3 + 0], vp = med[n * 3 + 1], rho = med[n * 3 + 2];
    using O = R<T>;
    T mu = O::mul(rho, O::mul(vs, vs));
    T lam = O::mul(rho, O::sub(O::mul(vp, vp), O::mul(O::mul((T)2, vs), vs)));
    T b = O::div((T)1, rho);
    long long p = g.at(i, j, k);
    cjm[C_MU * g.fstride + p] = (float)mu;
    cjm[C_LAMBDA * g.fstride + p] = (float)lam;
    cjm[C_BUOY * g.fstride + p] = (float)b;
}

// ------------------------------------------------------- CGFDM metrics
// 4th-order MacCormack pair averaged (LC macro, src/axis.h:272;
// src/contravariant.cpp:181-285), interior points only.
template <typename T>
__device__ __forceinline__ T lc(const float *__restrict__ c, long long p, long long s, int FB, T rDH)
{
    using O = R<T>;
    // taps at p + FB*s*(-1, 0, 1, 2, 3) with af_1, af0, af1, af2, af3
    T a = O::mul((T)CG_AF_1, (T)c[(p - FB * s) * 3]);
    a = O::add(a, O::mul((T)CG_AF0, (T)c[p * 3]));
    a = O::add(a, O::mul((T)CG_AF1, (T)c[(p + FB * s) * 3]));
    a = O::add(a, O::mul((T)CG_AF2, (T)c[(p + 2 * FB * s) * 3]));
    a = O::add(a, O::mul((T)CG_AF3, (T)c[(p + 3 * FB * s) * 3]));
    return O::mul(O::mul((T)FB, a), rDH);
}

template <typename T>
__global__ void k_metric_cgfdm(const float *__restrict__ coord, float *cjm, DevGrid g, float rDHf)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + CGFDM_HALO;
    int j = blockIdx.y * blockDim.y + threadIdx.y + CGFDM_HALO;
    int k = blockIdx.z * blockDim.z + threadIdx.z + CGFDM_HALO;
    if (i >= g.nxp - CGFDM_HALO || j >= g.nyp - CGFDM_HALO || k >= g.nzp - CGFDM_HALO) return;
    using O = R<T>;
    const long long sx = 1, sy = g.nxp, sz = (long long)g.nxp * g.nyp;
    const long long p = i + j * sy + k * sz;  // index into the AoS coordinate array
    const T rDH = (T)rDHf;
    T d[3][3];  // d[comp][dir]: x_xi x_et x_zt / y_.. / z_..
    for (int c = 0; c < 3; c++) {
        const float *cc = coord + c;
        d[c][0] = O::mul((T)0.5f, O::add(lc<T>(cc, p, sx, 1, rDH), lc<T>(cc, p, sx, -1, rDH)));
        d[c][1] = O::mul((T)0.5f, O::add(lc<T>(cc, p, sy, 1, rDH), lc<T>(cc, p, sy, -1, rDH)));
        d[c][2] = O::mul((T)0.5f, O::add(lc<T>(cc, p, sz, 1, rDH), lc<T>(cc, p, sz, -1, rDH)));
    }
    T x_xi = d[0][0], x_et = d[0][1], x_zt = d[0][2];
    T y_xi = d[1][0], y_et = d[1][1], y_zt = d[1][2];
    T z_xi = d[2][0], z_et = d[2][1], z_zt = d[2][2];
    T jac = O::mul(O::mul(x_xi, y_et), z_zt);
    jac = O::add(jac, O::mul(O::mul(x_et, y_zt), z_xi));
    jac = O::add(jac, O::mul(O::mul(x_zt, y_xi), z_et));
    jac = O::sub(jac, O::mul(O::mul(x_zt, y_et), z_xi));
    jac = O::sub(jac, O::mul(O::mul(x_et, y_xi), z_zt));
    jac = O::sub(jac, O::mul(O::mul(x_xi, z_et), y_zt));
    T jinv;
    if (sizeof(T) == 4) jinv = O::div((T)1, (T)(float)jac);  // float: from the stored Jacobian
    else jinv = O::div((T)1, jac);
    auto cof = [&](T a, T b, T c, T e) { return O::mul(O::sub(O::mul(a, b), O::mul(c, e)), jinv); };
    long long q = g.at(i, j, k);
    const long long F = g.fstride;
    cjm[C_XI_X * F + q] = (float)cof(y_et, z_zt, y_zt, z_et);
    cjm[C_XI_Y * F + q] = (float)cof(x_zt, z_et, x_et, z_zt);
    cjm[C_XI_Z * F + q] = (float)cof(x_et, y_zt, x_zt, y_et);
    cjm[C_ET_X * F + q] = (float)cof(y_zt, z_xi, y_xi, z_zt);
    cjm[C_ET_Y * F + q] = (float)cof(x_xi, z_zt, x_zt, z_xi);
    cjm[C_ET_Z * F + q] = (float)cof(x_zt, y_xi, x_xi, y_zt);
    cjm[C_ZT_X * F + q] = (float)cof(y_xi, z_et, y_et, z_xi);
    cjm[C_ZT_Y * F + q] = (float)cof(x_et, z_xi, x_xi, z_et);
    cjm[C_ZT_Z * F + q] = (float)cof(x_xi, y_et, x_et, y_xi);
    cjm[C_JAC * F + q] = (float)jac;
}

// ------------------------------------------- CGFDM free-surface matrices
// At the surface k = _nz - 1: DZ^-1 DX and DZ^-1 DY, negated
// (src/contravariant.cpp:365-461).  Above it, Jacobian and metric are
// mirrored about the surface (:502-516).
template <typename T>
__global__ void k_surface_cgfdm(float *cjm, float *rdz, DevGrid g)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + CGFDM_HALO;
    int j = blockIdx.y * blockDim.y + threadIdx.y + CGFDM_HALO;
    if (i >= g.nxp - CGFDM_HALO || j >= g.nyp - CGFDM_HALO) return;
    const long long F = g.fstride;
    const int ks = g.nzp - CGFDM_HALO - 1;
    long long q = g.at(i, j, ks);
    T m[9];
    for (int c = 0; c < 9; c++) m[c] = cjm[c * F + q];
    T rx[9], ry[9];
    surface_matrices<T>(m, (T)cjm[C_MU * F + q], (T)cjm[C_LAMBDA * F + q], rx, ry);
    long long s = g.at2(i, j);
    const long long P = g.plane;  // rdz fields are [18][nyp][pitch]
    for (int e = 0; e < 9; e++) {
        rdz[e * P + s] = (float)rx[e];
        rdz[(9 + e) * P + s] = (float)ry[e];
    }
}

__global__ void k_mirror_cgfdm(float *cjm, DevGrid g)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x + CGFDM_HALO;
    int j = blockIdx.y * blockDim.y + threadIdx.y + CGFDM_HALO;
    if (i >= g.nxp - CGFDM_HALO || j >= g.nyp - CGFDM_HALO) return;
    const int ks = g.nzp - CGFDM_HALO - 1;
    for (int k = ks + 1; k < g.nzp; k++) {
        long long dst = g.at(i, j, k), src = g.at(i, j, 2 * ks - k);
        for (int f = 0; f <= C_JAC; f++) cjm[f * g.fstride + dst] = cjm[f * g.fstride + src];
    }
}

// ------------------------------------------------------- SCFDM metrics
// Second-order central covariant basis, its determinant and cofactors
// (src/contravariant.cpp:80-177, the GPU branch's intended result).
template <typename T>
__global__ void k_metric_scfdm(const float *__restrict__ coord, float *cjm, DevGrid g, float rDHf)
{
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    int j = blockIdx.y * blockDim.y + threadIdx.y;
    int k = blockIdx.z * blockDim.z + threadIdx.z;
    if (i < 1 || j < 1 || k < 1 || i >= g.nxp - 1 || j >= g.nyp - 1 || k >= g.nzp - 1) return;
    using O = R<T>;
    const long long sy = g.nxp, sz = (long long)g.nxp * g.nyp;
    const long long p = i + j * sy + k * sz;
    const double rdh = rDHf;
    T c[9];
    const long long st[3] = {1, sy, sz};
    for (int d = 0; d < 3; d++)
        for (int comp = 0; comp < 3; comp++) {
            // central_difference2: (0.5 * (u1 - u_1) * rdh), in double, stored float
            float du = __fsub_rn(coord[(p + st[d]) * 3 + comp], coord[(p - st[d]) * 3 + comp]);
            double v = __dmul_rn(__dmul_rn(0.5, (double)du), rdh);
            c[d * 3 + comp] = (T)(float)v;
            if (sizeof(T) == 8) {
                double dd = (double)coord[(p + st[d]) * 3 + comp] - (double)coord[(p - st[d]) * 3 + comp];
                c[d * 3 + comp] = (T)(0.5 * dd * rdh);
            }
        }
    // c = [x_xi y_xi z_xi x_et y_et z_et x_zt y_zt z_zt]
    T jac = O::mul(O::mul(c[0], c[4]), c[8]);
    jac = O::add(jac, O::mul(O::mul(c[1], c[5]), c[6]));
    jac = O::add(jac, O::mul(O::mul(c[2], c[3]), c[7]));
    jac = O::sub(jac, O::mul(O::mul(c[2], c[4]), c[6]));
    jac = O::sub(jac, O::mul(O::mul(c[1], c[3]), c[8]));
    jac = O::sub(jac, O::mul(O::mul(c[0], c[7]), c[5]));
    const long long F = g.fstride;
    long long q = g.at(i, j, k);
    cjm[C_JAC * F + q] = (float)jac;
    for (int m = 0; m < 6; m++) cjm[(C_X_XI + m) * F + q] = (float)c[m];
    if (i < 2 || j < 2 || k < 2 || i >= g.nxp - 2 || j >= g.nyp - 2 || k >= g.nzp - 2) return;
    auto x2 = [&](int a, int b, int e, int f) { return O::sub(O::mul(c[a], c[b]), O::mul(c[e], c[f])); };
    cjm[0 * F + q] = (float)x2(4, 8, 5, 7);
    cjm[1 * F + q] = (float)x2(5, 6, 3, 8);
    cjm[2 * F + q] = (float)x2(3, 7, 4, 6);
    cjm[3 * F + q] = (float)x2(7, 2, 8, 1);
    cjm[4 * F + q] = (float)x2(8, 0, 6, 2);
    cjm[5 * F + q] = (float)x2(6, 1, 7, 0);
    cjm[6 * F + q] = (float)x2(1, 5, 2, 4);
    cjm[7 * F + q] = (float)x2(2, 3, 0, 5);
    cjm[8 * F + q] = (float)x2(0, 4, 1, 3);
}

// ------------------------------------------------- moment-rate scaling
// momentRate *= mu / (J DH^3) at each source cell (src/addMoment.cpp:26-76).
__global__ void k_scale_moment(float *rate, const long long *__restrict__ cell, long long npts, int nt,
                               const float *__restrict__ cjm, DevGrid g, float DH)
{
    long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (n >= npts * nt) return;
    long long p = n % npts;
    long long q = cell[p];  // layout index of the source cell
    float jacb = cjm[C_JAC * g.fstride + q], mu = cjm[C_MU * g.fstride + q];
    float V = __fmul_rn(__fmul_rn(__fmul_rn(jacb, DH), DH), DH);
    V = (float)__ddiv_rn(1.0, (double)V);
    float s = __fmul_rn(mu, V);
    for (int m = 0; m < 6; m++) rate[n * 6 + m] = __fmul_rn(rate[n * 6 + m], s);
}

// ------------------------------------------------------------ launchers
cudaError_t launch_setup(const float *d_coord, const float *d_medium, float *cjm, float *rdz, DevGrid g,
                         float rDH, int scheme, int fp64, cudaStream_t st)
{
    long long npad = (long long)g.nxp * g.nyp * g.nzp;
    int tb = 256;
    unsigned nb = (unsigned)((npad + tb - 1) / tb);
    if (fp64) k_medium<double><<<nb, tb, 0, st>>>(d_medium, cjm, g);
    else k_medium<float><<<nb, tb, 0, st>>>(d_medium, cjm, g);
    CUDA_TRY(cudaGetLastError());
    if (scheme == 0) {
        dim3 b(32, 4, 4), gr((g.nx + 31) / 32, (g.ny + 3) / 4, (g.nz + 3) / 4);
        if (fp64) k_metric_cgfdm<double><<<gr, b, 0, st>>>(d_coord, cjm, g, rDH);
        else k_metric_cgfdm<float><<<gr, b, 0, st>>>(d_coord, cjm, g, rDH);
        CUDA_TRY(cudaGetLastError());
        dim3 b2(32, 8), g2((g.nx + 31) / 32, (g.ny + 7) / 8);
        if (fp64) k_surface_cgfdm<double><<<g2, b2, 0, st>>>(cjm, rdz, g);
        else k_surface_cgfdm<float><<<g2, b2, 0, st>>>(cjm, rdz, g);
        CUDA_TRY(cudaGetLastError());
        k_mirror_cgfdm<<<g2, b2, 0, st>>>(cjm, g);
        CUDA_TRY(cudaGetLastError());
    } else {
        dim3 b(32, 4, 4), gr((g.nxp + 31) / 32, (g.nyp + 3) / 4, (g.nzp + 3) / 4);
        if (fp64) k_metric_scfdm<double><<<gr, b, 0, st>>>(d_coord, cjm, g, rDH);
        else k_metric_scfdm<float><<<gr, b, 0, st>>>(d_coord, cjm, g, rDH);
        CUDA_TRY(cudaGetLastError());
    }
    return cudaSuccess;
}

cudaError_t launch_scale_moment(float *rate, const long long *cell, long long npts, int nt, const float *cjm,
                                DevGrid g, float DH, cudaStream_t st)
{
    if (npts == 0 || nt == 0) return cudaSuccess;
    long long n = npts * nt;
    k_scale_moment<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(rate, cell, npts, nt, cjm, g, DH);
    return cudaGetLastError();
}

}  // namespace cgfdm

namespace cgfdm {

// The coordinates of the padded grid [_nz_][_ny_][_nx_][3] from the grid and
// the surface height map [_ny_][_nx_], with the host model's formulas
// (csrc/model.cpp build_coords, terrain_following_z, terrain_z_double;
// src/coord.cpp:130-132,228-234) in explicitly rounded operations, so they
// equal the host's values in every build.
__global__ void k_build_coords(float *__restrict__ coord, const float *__restrict__ terrain, int nxp, int nyp,
                               int nzp, int mode, float DH, int originalX, int originalY, int NZ, float depth_f,
                               double depth_d)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x, j = blockIdx.y * blockDim.y + threadIdx.y;
    const int k = blockIdx.z;
    if (i >= nxp || j >= nyp) return;
    const long long q = (((long long)k * nyp + j) * nxp + i) * 3;
    coord[q + 0] = __fsub_rn(__fmul_rn((float)(i - CGFDM_HALO), DH), __fmul_rn((float)originalX, DH));
    coord[q + 1] = __fsub_rn(__fmul_rn((float)(j - CGFDM_HALO), DH), __fmul_rn((float)originalY, DH));
    const int K = k - CGFDM_HALO;
    float z;
    if (mode == 0) {
        z = __fsub_rn(__fmul_rn((float)(K + 1), DH), __fmul_rn((float)NZ, DH));
    } else {
        const float h = terrain[(long long)j * nxp + i];
        if (mode == 1) {
            const float a = fabsf(depth_f);
            const float DZ = __double2float_rn(__ddiv_rn((double)__fadd_rn(h, a), (double)(NZ - 1)));
            z = __fadd_rn(-a, __fmul_rn(DZ, (float)K));
        } else {
            const double a = fabs(depth_d);
            const double DZ = __ddiv_rn(__dadd_rn((double)h, a), (double)(NZ - 1));
            z = __double2float_rn(__dadd_rn(-a, __dmul_rn(DZ, (double)K)));
        }
    }
    coord[q + 2] = z;
}

cudaError_t launch_build_coords(float *coord, const float *terrain, int nxp, int nyp, int nzp, int mode, float DH,
                                int originalX, int originalY, int NZ, float depth_f, double depth_d, cudaStream_t st)
{
    const dim3 b(32, 8, 1), gr((nxp + 31) / 32, (nyp + 7) / 8, nzp);
    k_build_coords<<<gr, b, 0, st>>>(coord, terrain, nxp, nyp, nzp, mode, DH, originalX, originalY, NZ, depth_f,
                                     depth_d);
    return cudaGetLastError();
}

}  // namespace cgfdm
