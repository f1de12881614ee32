// Point operators of the CGFDM right-hand side shared by the fused stage
// kernel (cgfdm_stage.cu), the per-function entry points (shims.cu) and the
// precision-templated reference-form run (precise.cu).  Each keeps the
// reference's evaluation order, so every caller rounds as the reference
// does; R is the arithmetic type (float, or double for the FP64 run, where
// the float constants are promoted as the reference's expressions promote
// them).
#pragma once

#include "device.cuh"

namespace cgfdm {

// Contribution of one grid direction to the RHS, given the metric row
// (xi, eta or zeta gradient) and the nine scaled derivatives along it
// (src/wave_deriv.cpp:244-272; the same form in pml_deriv and
// pml_free_surface).  out: Vx Vy Vz Txx Tyy Tzz Txy Txz Tyz.
template <class R>
__device__ __forceinline__ void dir_rhs(R m0, R m1, R m2, const R d[9], R mu, R lam, R buo, R out[9])
{
    out[0] = ((m0 * d[3] + m1 * d[6]) + m2 * d[7]) * buo;
    out[1] = ((m0 * d[6] + m1 * d[4]) + m2 * d[8]) * buo;
    out[2] = ((m0 * d[7] + m1 * d[8]) + m2 * d[5]) * buo;
    R dv = (m0 * d[0] + m1 * d[1]) + m2 * d[2];
    R m2mu = R(2.0f) * mu;
    out[3] = dv * lam + m2mu * (m0 * d[0]);
    out[4] = dv * lam + m2mu * (m1 * d[1]);
    out[5] = dv * lam + m2mu * (m2 * d[2]);
    out[6] = (m1 * d[0] + m0 * d[1]) * mu;
    out[7] = (m2 * d[0] + m0 * d[2]) * mu;
    out[8] = (m2 * d[1] + m1 * d[2]) * mu;
}

// stress part only (components 3..8) from velocity derivatives v[0..2]
template <class R>
__device__ __forceinline__ void dir_stress(R m0, R m1, R m2, const R v[3], R mu, R lam, R out[9])
{
    R dv = (m0 * v[0] + m1 * v[1]) + m2 * v[2];
    R m2mu = R(2.0f) * mu;
    out[3] = dv * lam + m2mu * (m0 * v[0]);
    out[4] = dv * lam + m2mu * (m1 * v[1]);
    out[5] = dv * lam + m2mu * (m2 * v[2]);
    out[6] = (m1 * v[0] + m0 * v[1]) * mu;
    out[7] = (m2 * v[0] + m0 * v[2]) * mu;
    out[8] = (m2 * v[1] + m1 * v[2]) * mu;
}

// One-sided 5-point operator of the L macro (src/axis.h:287):
// FB * (af_1 w[-FB] + af0 w[0] + af1 w[FB] + af2 w[2FB] + af3 w[3FB]) * rDH
template <class R>
__device__ __forceinline__ R lop(R wm, R w0, R w1, R w2, R w3, int FB, R rDH)
{
    R s = R(CG_AF_1) * wm + R(CG_AF0) * w0;
    s = s + R(CG_AF1) * w1;
    s = s + R(CG_AF2) * w2;
    s = s + R(CG_AF3) * w3;
    return ((R)FB * s) * rDH;
}

}  // namespace cgfdm
