// Explicitly rounded arithmetic R<T> and the CGFDM free-surface matrices.
//
// R<float> rounds every operation separately (no FMA contraction), so the
// setup kernels reproduce the reference's FP32 evaluation bit for bit;
// R<double> is the FP64 setup.  Any other T with R<T> defined (the adjoint
// uses a dual number) runs the same formulas.
#pragma once

#include "device.cuh"

namespace cgfdm {

template <typename T>
struct R;
template <>
struct R<float> {
    static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
    static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
    static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
    static __device__ __forceinline__ float div(float a, float b) { return __fdiv_rn(a, b); }
};
template <>
struct R<double> {
    static __device__ __forceinline__ double add(double a, double b) { return __dadd_rn(a, b); }
    static __device__ __forceinline__ double sub(double a, double b) { return __dsub_rn(a, b); }
    static __device__ __forceinline__ double mul(double a, double b) { return __dmul_rn(a, b); }
    static __device__ __forceinline__ double div(double a, double b) { return __ddiv_rn(a, b); }
};

// Traction-free condition at the surface (src/contravariant.cpp:365-461):
// with DZ, DX, DY the 3x3 blocks that the zeta, xi and eta velocity
// derivatives contribute to the surface traction, the zeta derivative is
// V_zeta = rx V_xi + ry V_eta, rx = -DZ^-1 DX, ry = -DZ^-1 DY (row-major
// 3x3).  m: the nine metric terms xi_x .. zt_z at the surface point.
template <typename T>
__device__ __forceinline__ void surface_matrices(const T m[9], T mu, T lambda, T rx[9], T ry[9])
{
    using O = R<T>;
    const T xi_x = m[0], xi_y = m[1], xi_z = m[2];
    const T et_x = m[3], et_y = m[4], et_z = m[5];
    const T zt_x = m[6], zt_y = m[7], zt_z = m[8];
    T chi = O::add(O::mul((T)2.0f, lambda), mu);
    T lam_mu = O::add(lambda, mu);
    T DZ[9], DX[9], DY[9], rDZ[9];
    DZ[0] = O::add(O::mul(O::mul(chi, zt_x), zt_x), O::mul(mu, O::add(O::mul(zt_y, zt_y), O::mul(zt_z, zt_z))));
    DZ[1] = O::mul(O::mul(lam_mu, zt_x), zt_y);
    DZ[2] = O::mul(O::mul(lam_mu, zt_x), zt_z);
    DZ[3] = DZ[1];
    DZ[4] = O::add(O::mul(O::mul(chi, zt_y), zt_y), O::mul(mu, O::add(O::mul(zt_x, zt_x), O::mul(zt_z, zt_z))));
    DZ[5] = O::mul(O::mul(lam_mu, zt_y), zt_z);
    DZ[6] = DZ[2];
    DZ[7] = DZ[5];
    DZ[8] = O::add(O::mul(O::mul(chi, zt_z), zt_z), O::mul(mu, O::add(O::mul(zt_x, zt_x), O::mul(zt_y, zt_y))));
    T det = O::mul(O::mul(DZ[0], DZ[4]), DZ[8]);
    det = O::add(det, O::mul(O::mul(DZ[1], DZ[5]), DZ[6]));
    det = O::add(det, O::mul(O::mul(DZ[2], DZ[7]), DZ[3]));
    det = O::sub(det, O::mul(O::mul(DZ[2], DZ[4]), DZ[6]));
    det = O::sub(det, O::mul(O::mul(DZ[1], DZ[3]), DZ[8]));
    det = O::sub(det, O::mul(O::mul(DZ[0], DZ[7]), DZ[5]));
    // DX / DY share one pattern with (xi) or (et) in place of a
    auto fill = [&](T *D, T ax, T ay, T az) {
        D[0] = O::add(O::mul(O::mul(chi, zt_x), ax), O::mul(mu, O::add(O::mul(zt_y, ay), O::mul(zt_z, az))));
        D[1] = O::add(O::mul(O::mul(lambda, zt_x), ay), O::mul(O::mul(mu, zt_y), ax));
        D[2] = O::add(O::mul(O::mul(lambda, zt_x), az), O::mul(O::mul(mu, zt_z), ax));
        D[3] = O::add(O::mul(O::mul(lambda, zt_y), ax), O::mul(O::mul(mu, zt_x), ay));
        D[4] = O::add(O::mul(O::mul(chi, zt_y), ay), O::mul(mu, O::add(O::mul(zt_x, ax), O::mul(zt_z, az))));
        D[5] = O::add(O::mul(O::mul(lambda, zt_y), az), O::mul(O::mul(mu, zt_z), ay));
        D[6] = O::add(O::mul(O::mul(lambda, zt_z), ax), O::mul(O::mul(mu, zt_x), az));
        D[7] = O::add(O::mul(O::mul(lambda, zt_z), ay), O::mul(O::mul(mu, zt_y), az));
        D[8] = O::add(O::mul(O::mul(chi, zt_z), az), O::mul(mu, O::add(O::mul(zt_x, ax), O::mul(zt_y, ay))));
    };
    fill(DX, xi_x, xi_y, xi_z);
    fill(DY, et_x, et_y, et_z);
    // adjugate / determinant
    rDZ[0] = O::div(O::sub(O::mul(DZ[4], DZ[8]), O::mul(DZ[5], DZ[7])), det);
    rDZ[1] = O::div(O::add(O::mul(-DZ[3], DZ[8]), O::mul(DZ[5], DZ[6])), det);
    rDZ[2] = O::div(O::sub(O::mul(DZ[3], DZ[7]), O::mul(DZ[4], DZ[6])), det);
    rDZ[3] = O::div(O::add(O::mul(-DZ[1], DZ[8]), O::mul(DZ[2], DZ[7])), det);
    rDZ[4] = O::div(O::sub(O::mul(DZ[0], DZ[8]), O::mul(DZ[2], DZ[6])), det);
    rDZ[5] = O::div(O::add(O::mul(-DZ[0], DZ[7]), O::mul(DZ[1], DZ[6])), det);
    rDZ[6] = O::div(O::sub(O::mul(DZ[1], DZ[5]), O::mul(DZ[2], DZ[4])), det);
    rDZ[7] = O::div(O::add(O::mul(-DZ[0], DZ[5]), O::mul(DZ[2], DZ[3])), det);
    rDZ[8] = O::div(O::sub(O::mul(DZ[0], DZ[4]), O::mul(DZ[1], DZ[3])), det);
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) {
            T vx = O::add(O::add(O::mul(rDZ[r * 3 + 0], DX[0 + c]), O::mul(rDZ[r * 3 + 1], DX[3 + c])),
                          O::mul(rDZ[r * 3 + 2], DX[6 + c]));
            T vy = O::add(O::add(O::mul(rDZ[r * 3 + 0], DY[0 + c]), O::mul(rDZ[r * 3 + 1], DY[3 + c])),
                          O::mul(rDZ[r * 3 + 2], DY[6 + c]));
            rx[r * 3 + c] = -vx;
            ry[r * 3 + c] = -vy;
        }
}

}  // namespace cgfdm
