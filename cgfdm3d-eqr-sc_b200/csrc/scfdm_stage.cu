// ME-AWENO (SCFDM) time stepping for sm_100a: alternative-flux WENO5
// finite differences, TVD-RK3, characteristic free surface and
// exponential-decay sponge.
//
// A TVD stage is three pencil kernels, one per grid direction.  Each CTA
// owns a tile of NPOS consecutive positions along its direction (the tile's
// points plus the 3 + 3 neighbours their flux differences reach) times NL
// lanes across it, and runs three phases through shared memory:
//
//   A  every position m computes, per variable, both WENO5-JS states that
//      are upwinded from the cell centred at m: the left state of face m+1/2
//      and the right state of face m-1/2 (src/alternative_flux_FD.cpp:42-59
//      called at 137-141).  The two states share their three smoothness
//      indicators, so they are computed once per position.
//   B  every face m+1/2 combines the left state of position m with the
//      right state of position m+1 into the Lax-Friedrichs flux, with the
//      metric and medium of point m (src/alternative_flux_FD.cpp:144-169).
//   C  every point takes the flux difference with the fourth- and
//      sixth-order corrections (cal_du_x/y/z, src/alternative_flux_FD.cpp:
//      1215-1435), or in the top three layers the variant built from point
//      fluxes (1257-1277).
//
// The x pass stores the RHS, the y pass adds to it and the z pass adds its
// part and applies the TVD-RK3 update (src/wave_rk_tvd.cpp:17-78), so the
// RHS accumulates in the reference's order.  After the third stage one
// kernel per surface column applies the characteristic free surface and
// extrapolates into the halo above it (src/freeSurface.cpp:40-194), the
// sponge factor of the top layers (src/exp_decay_absorb.cpp:19-106; the z
// pass of the last stage applies it below them) and the peak ground velocity
// (src/PGV.cpp:61-175).
//
// Faces the reference never writes -- along each direction those before
// index 2 and from _n on -- have zero flux, exactly as its zero-initialised
// flux buffer gives.  Halo points keep their values through a TVD stage, so
// stage buffers only need the top halo planes copied across.
//
// Built with CGFDM_EXACT (and --fmad=false) every float and double operation
// of phases A-C and of the RK update follows the reference's expression
// order, so the result is bit-identical.  The default build shares the
// smoothness indicators between the two states of a position, combines the
// two fluxes of a face before applying the (linear) flux function, and folds
// the flux-difference corrections into one six-tap filter.
#include "device.cuh"
#include "kernels.cuh"
#include "sc_ops.cuh"

// 1: the passes' RHS and stage-output stores evict-first (each is read back
// by a later pass or stage, long after L2 has turned over)
#ifndef SC_STREAM_HINTS
#define SC_STREAM_HINTS 1
#endif
#if SC_STREAM_HINTS
#define SC_ST(p, v) __stcs(&(p), (v))
#else
#define SC_ST(p, v) ((p) = (v))
#endif
// 2: also the single-use loads of the RHS, the step-start state and DT rDH / J
#if SC_STREAM_HINTS >= 2
#define SC_LD(p) __ldcs(&(p))
#else
#define SC_LD(p) (p)
#endif

namespace cgfdm {

namespace {

constexpr int SC_THREADS = 256;

// ------------------------------------------------------------ WENO5-JS
#ifndef CGFDM_EXACT
__device__ __forceinline__ float rcp_approx(float x)
{
    float r;
    asm("rcp.approx.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
#endif

// Both states upwinded from the cell centred at c, window a b c d e:
// uL at the face c+1/2, uR at the face c-1/2.
__device__ __forceinline__ void weno_pair(float a, float b, float c, float d, float e, float &uL, float &uR)
{
#ifdef CGFDM_EXACT
    uL = weno5_ref(a, b, c, d, e);
    uR = weno5_ref(e, d, c, b, a);
#else
    // Jiang-Shu indicators over the cell of c for the sub-stencils
    // (a,b,c), (b,c,d), (c,d,e): 13/12 (second difference)^2 + 1/4 (slope)^2
    const float k13 = 13.0f / 12.0f;
    const float s0 = (a - 2.0f * b) + c, t0 = (a - 4.0f * b) + 3.0f * c;
    const float s1 = (b - 2.0f * c) + d, t1 = b - d;
    const float s2 = (c - 2.0f * d) + e, t2 = (3.0f * c - 4.0f * d) + e;
    const float B0 = k13 * s0 * s0 + 0.25f * t0 * t0 + 1e-6f;
    const float B1 = k13 * s1 * s1 + 0.25f * t1 * t1 + 1e-6f;
    const float B2 = k13 * s2 * s2 + 0.25f * t2 * t2 + 1e-6f;
    const float r0 = rcp_approx(B0 * B0), r1 = rcp_approx(B1 * B1), r2 = rcp_approx(B2 * B2);
    // linear weights 5/16, 10/16, 1/16 for the sub-stencil on the face side,
    // the centred one and the far one (the common 1/16 cancels)
    {
        const float wa = 5.0f * r2, wb = 10.0f * r1, wc = r0;
        const float qa = 0.375f * c + 0.75f * d - 0.125f * e;
        const float qb = -0.125f * b + 0.75f * c + 0.375f * d;
        const float qc = 0.375f * a - 1.25f * b + 1.875f * c;
        uL = (wa * qa + wb * qb + wc * qc) * rcp_approx(wa + wb + wc);
    }
    {
        const float wa = 5.0f * r0, wb = 10.0f * r1, wc = r2;
        const float qa = 0.375f * c + 0.75f * b - 0.125f * a;
        const float qb = -0.125f * d + 0.75f * c + 0.375f * b;
        const float qc = 0.375f * e - 1.25f * d + 1.875f * c;
        uR = (wa * qa + wb * qb + wc * qc) * rcp_approx(wa + wb + wc);
    }
#endif
}

// Lax-Friedrichs flux of a face from its left (uL) and right (uR) states.
__device__ __forceinline__ void lf_flux(float n0, float n1, float n2, float lam, float mu, float buo, float alpha,
                                        const float uL[9], const float uR[9], float F[9])
{
#ifdef CGFDM_EXACT
    lf_flux_ref(n0, n1, n2, lam, mu, buo, alpha, uL, uR, F);
#else
    // the flux is linear in the state: f(uL) + f(uR) = f(uL + uR)
    float s[9], fs[9];
#pragma unroll
    for (int v = 0; v < 9; v++) s[v] = uL[v] + uR[v];
    const float tr = s[3] + s[4] + s[5], m2 = 2.0f * mu;
    fs[0] = n0 * (lam * tr + m2 * s[3]) + mu * (n1 * s[8] + n2 * s[7]);
    fs[1] = n1 * (lam * tr + m2 * s[4]) + mu * (n0 * s[8] + n2 * s[6]);
    fs[2] = n2 * (lam * tr + m2 * s[5]) + mu * (n0 * s[7] + n1 * s[6]);
    fs[3] = buo * (n0 * s[0]);
    fs[4] = buo * (n1 * s[1]);
    fs[5] = buo * (n2 * s[2]);
    fs[6] = buo * (n1 * s[2] + n2 * s[1]);
    fs[7] = buo * (n0 * s[2] + n2 * s[0]);
    fs[8] = buo * (n0 * s[1] + n1 * s[0]);
    const float ha = 0.5f * alpha;
#pragma unroll
    for (int v = 0; v < 9; v++) F[v] = -0.5f * fs[v] - ha * (uR[v] - uL[v]);
#endif
}

// Exponential-decay factor product of an interior point, in the
// reference's order x-low, x-high, y-low, y-high, z-low
// (src/exp_decay_absorb.cpp:36-92; free surface on, so no z-high layer).
__device__ __forceinline__ float decay_apply(float w, int i, int j, int k, const DevGrid &g, const float *G, int nl)
{
    const int X = i - CGFDM_HALO, Y = j - CGFDM_HALO, Z = k - CGFDM_HALO;
    if (X <= nl) w = w * G[nl - X];
    if (X >= g.nx - nl) w = w * G[nl - (g.nx - X)];
    if (Y <= nl) w = w * G[nl - Y];
    if (Y >= g.ny - nl) w = w * G[nl - (g.ny - Y)];
    if (Z <= nl) w = w * G[nl - Z];
    return w;
}

}  // namespace

// Flux difference of one point in the top three layers: the corrections
// come from point fluxes at p-3 .. p+3 along the direction
// (src/alternative_flux_FD.cpp:1253-1279).  Fp, Fm: fluxes of the faces
// p+1/2 and p-1/2.  Only three layers take this path, so it reads its
// operands from global memory.
__device__ __noinline__ void surface_diff(const ScDirArgs &a, long long q, long long stride, int mc0, float coef,
                                          const float *Fp, const float *Fm, float *val)
{
    const long long F = a.g.fstride;
    const float c24 = 1.0f / 24, c7 = 7.0f / 5760;
    float o2A[9], o4A[9], o2B[9], o4B[9];
    const float c2[6] = {-5.0f, 39.0f, -34.0f, -34.0f, 39.0f, -5.0f};
    const float c4[6] = {1.0f, -3.0f, 2.0f, 2.0f, -3.0f, 1.0f};
    for (int n = 0; n < 7; n++) {
        const long long qn = q + (n - 3) * stride;
        float u[9], hu[9];
#pragma unroll
        for (int v = 0; v < 9; v++) u[v] = a.W[v * F + qn];
        point_flux(a.cjm[(mc0 + 0) * F + qn], a.cjm[(mc0 + 1) * F + qn], a.cjm[(mc0 + 2) * F + qn],
                   a.cjm[C_LAMBDA * F + qn], a.cjm[C_MU * F + qn], a.cjm[C_BUOY * F + qn], u, hu);
#pragma unroll
        for (int v = 0; v < 9; v++) {
            // o2 = -5 u1 + 39 u2 - 34 u3 - 34 u4 + 39 u5 - 5 u6, o4 = u1 - 3 u2 + 2 u3 + 2 u4 - 3 u5 + u6,
            // accumulated left to right: B over hu[0..5], A over hu[1..6]
            if (n <= 5) {
                if (n == 0) o2B[v] = c2[0] * hu[v], o4B[v] = hu[v];
                else {
                    o2B[v] = c2[n] < 0.0f ? o2B[v] - (-c2[n]) * hu[v] : o2B[v] + c2[n] * hu[v];
                    o4B[v] = c4[n] < 0.0f ? o4B[v] - (-c4[n]) * hu[v] : (n == 5 ? o4B[v] + hu[v] : o4B[v] + c4[n] * hu[v]);
                }
            }
            if (n >= 1) {
                const int t = n - 1;
                if (t == 0) o2A[v] = c2[0] * hu[v], o4A[v] = hu[v];
                else {
                    o2A[v] = c2[t] < 0.0f ? o2A[v] - (-c2[t]) * hu[v] : o2A[v] + c2[t] * hu[v];
                    o4A[v] = c4[t] < 0.0f ? o4A[v] - (-c4[t]) * hu[v] : (t == 5 ? o4A[v] + hu[v] : o4A[v] + c4[t] * hu[v]);
                }
            }
        }
    }
#pragma unroll
    for (int v = 0; v < 9; v++) {
        const float A = Fp[v] - c24 * ((1.0f / 48) * o2A[v]) + c7 * ((1.0f / 2) * o4A[v]);
        const float B = Fm[v] - c24 * ((1.0f / 48) * o2B[v]) + c7 * ((1.0f / 2) * o4B[v]);
        val[v] = coef * (-(A - B));
    }
}

// Flux difference of an interior point from the fluxes f[0..5] of the faces
// p-5/2 .. p+5/2 (src/alternative_flux_FD.cpp:1283).
__device__ __forceinline__ float interior_diff(const float f[6], float coef)
{
#ifdef CGFDM_EXACT
    return interior_diff_ref(f, coef);
#else
    // corrected face flux Fh = c2 F-2 + c1 F-1 + c0 F0 + c1 F+1 + c2 F+2 with
    // c0 = 6402/5760, c1 = -348/5760, c2 = 27/5760; val = -coef (Fh[p] - Fh[p-1])
    // = coef (c2 (F[p-3] - F[p+2]) + (c1 - c2) (F[p-2] - F[p+1]) + (c0 - c1) (F[p-1] - F[p]))
    constexpr float e0 = 27.0f / 5760, e1 = (-348.0f - 27.0f) / 5760, e2 = (6402.0f + 348.0f) / 5760;
    return coef * (e0 * (f[0] - f[5]) + e1 * (f[1] - f[4]) + e2 * (f[2] - f[3]));
#endif
}

// The pass's use of the flux difference val of point q = (i, j, k): the x
// pass stores the RHS, the y pass adds to it, the z pass adds its part and
// applies the TVD-RK3 update (src/wave_rk_tvd.cpp:17-78), the sponge below
// the top four layers in the last stage, and carries the halo above the
// surface into the stage buffer in stages 0 and 1 (the reference's update
// runs over every point; halo points have a zero RHS and keep their value).
template <int DIR>
__device__ __forceinline__ void epilogue(const ScDirArgs &a, long long q, int i, int j, int k, const float val[9])
{
    const long long F = a.g.fstride;
    if (DIR == 0) {
#pragma unroll
        for (int v = 0; v < 9; v++) SC_ST(a.H[v * F + q], val[v]);
    } else if (DIR == 1) {
#pragma unroll
        for (int v = 0; v < 9; v++) SC_ST(a.H[v * F + q], SC_LD(a.H[v * F + q]) + val[v]);
    } else {
        const int _nz = a.g.nzp - CGFDM_HALO;
        const bool decay = a.decay != nullptr && k < _nz - 4;
#pragma unroll
        for (int v = 0; v < 9; v++) {
            const float h = SC_LD(a.H[v * F + q]) + val[v];
            const float w = a.W[v * F + q];
            float o;
            if (a.irk == 0) {
                o = w + h;
            } else if (a.irk == 1) {
                const double m = SC_LD(a.Wm[v * F + q]);
                o = __double2float_rn(__dadd_rn(__dadd_rn(__dmul_rn(0.75, m), __dmul_rn(0.25, (double)w)),
                                                __dmul_rn(0.25, (double)h)));
            } else {
                const double m = SC_LD(a.Wm[v * F + q]);
                o = __double2float_rn(__dadd_rn(__dadd_rn(__dmul_rn(1.0 / 3.0, m), __dmul_rn(2.0 / 3.0, (double)w)),
                                                __dmul_rn(2.0 / 3.0, (double)h)));
            }
            if (decay) o = decay_apply(o, i, j, k, a.g, a.decay, a.ndecay);
            SC_ST(a.Wout[v * F + q], o);
        }
        if (a.copy_halo && k == _nz - 1)
            for (int h = 1; h <= CGFDM_HALO; h++)
                for (int v = 0; v < 9; v++) a.Wout[v * F + q + h * a.g.plane] = a.W[v * F + q + h * a.g.plane];
    }
}

// ------------------------------------------------------------ tiled pass
// Tiles of NPOS positions along the pass direction (the tile's NPOS - 6
// points and the neighbours their differences reach) times NL lanes across
// it: rows j for the x pass (grid: x tiles, row groups, k), columns i for
// the y and z passes (grid: column groups, y tiles, k / column groups, j,
// z tiles).  Three phases through shared memory:
//   A  both WENO states upwinded from every position,
//   B  the Lax-Friedrichs flux of every face, written over the left states,
//   C  the flux difference of every point and the pass's epilogue.
constexpr int SCX_NPOS = 64, SCX_NL = 4;
// y and z tiles: 32 positions (26 points) x 16 columns, 37 KB of shared
// memory, five CTAs per SM (register cap 48); on the 512 x 512 x 256 basin
// workload this beat 80 x 16 at two CTAs by 1.4x and a one-warp-per-pencil
// register-streaming variant by 1.7x: the passes are latency-bound and
// occupancy pays (staging the W window in shared memory first, at three to
// five CTAs per SM, was 1.5x slower than reading it through L1, and sliding
// one thread's window over two positions 6 % slower than one position per
// thread).
#ifndef SCY_NPOS
#define SCY_NPOS 32
#endif
#ifndef SCY_NL
#define SCY_NL 16
#endif

#ifndef SC_TILE_MIN_CTAS
#define SC_TILE_MIN_CTAS 5
#endif
// shared memory of a tile: left and right states, 9 + 9 fields per position
constexpr size_t sc_tile_smem(int npos, int nl) { return sizeof(float) * 18 * npos * nl; }

template <int DIR, int NPOS, int NL>
__global__ void __launch_bounds__(SC_THREADS, SC_TILE_MIN_CTAS) k_sc_tile(const ScDirArgs a)
{
    constexpr int P = NPOS - 6;
    extern __shared__ __align__(16) float sm[];
    float *sL = sm, *sR = sm + 9 * NPOS * NL;
    const DevGrid g = a.g;
    const long long F = g.fstride;
    const int _nx = g.nxp - CGFDM_HALO, _ny = g.nyp - CGFDM_HALO, _nz = g.nzp - CGFDM_HALO;
    const int nd = DIR == 0 ? _nx : DIR == 1 ? _ny : _nz;  // points along the pass end before nd
    const long long stride = DIR == 0 ? 1 : DIR == 1 ? (long long)g.pitch : g.plane;
    const int tile = DIR == 0 ? blockIdx.x : DIR == 1 ? blockIdx.y : blockIdx.z;
    const int p0 = CGFDM_HALO + tile * P;
    const int lane0 = CGFDM_HALO + (DIR == 0 ? blockIdx.y : blockIdx.x) * NL;
    const int lane_end = DIR == 0 ? _ny : _nx;
    const int jfix = DIR == 2 ? CGFDM_HALO + (int)blockIdx.y : 0;
    const int kfix = DIR == 2 ? 0 : CGFDM_HALO + (int)blockIdx.z;
    constexpr int mc0 = DIR == 0 ? C_XI_X : DIR == 1 ? C_ET_X : C_ZT_X;  // metric row of this direction

    auto coords = [&](int m, int lane, int &i, int &j, int &k) {
        if (DIR == 0) i = m, j = lane0 + lane, k = kfix;
        else if (DIR == 1) i = lane0 + lane, j = m, k = kfix;
        else i = lane0 + lane, j = jfix, k = m;
    };
    // consecutive threads take consecutive x: positions for the x pass, lanes otherwise
    auto sidx = [](int v, int mi, int lane) {
        return DIR == 0 ? (v * NL + lane) * NPOS + mi : (v * NPOS + mi) * NL + lane;
    };
    auto split = [](int it, int n_along, int &mi, int &lane) {
        if (DIR == 0) mi = it % n_along, lane = it / n_along;
        else lane = it % NL, mi = it / NL;
    };

    // ---- phase A: both WENO states of every position
    for (int it = threadIdx.x; it < NPOS * NL; it += SC_THREADS) {
        int mi, lane;
        split(it, NPOS, mi, lane);
        const int m = p0 - CGFDM_HALO + mi;
        if (lane0 + lane >= lane_end || m < 2 || m > nd) continue;
        int i, j, k;
        coords(m, lane, i, j, k);
        const float *w = a.W + g.at(i, j, k);
#pragma unroll 3
        for (int v = 0; v < 9; v++) {
            const float *wv = w + v * F;
            float uL, uR;
            weno_pair(__ldg(wv - 2 * stride), __ldg(wv - stride), __ldg(wv), __ldg(wv + stride), __ldg(wv + 2 * stride),
                      uL, uR);
            sL[sidx(v, mi, lane)] = uL;
            sR[sidx(v, mi, lane)] = uR;
        }
    }
    __syncthreads();

    // ---- phase B: Lax-Friedrichs flux of face m+1/2, stored over the left state
    for (int it = threadIdx.x; it < NPOS * NL; it += SC_THREADS) {
        int mi, lane;
        split(it, NPOS, mi, lane);
        const int m = p0 - CGFDM_HALO + mi;
        if (lane0 + lane >= lane_end || mi == NPOS - 1) continue;
        float Fv[9];
        if (m >= 2 && m < nd) {
            int i, j, k;
            coords(m, lane, i, j, k);
            const long long q = g.at(i, j, k);
            const float n0 = a.cjm[(mc0 + 0) * F + q], n1 = a.cjm[(mc0 + 1) * F + q], n2 = a.cjm[(mc0 + 2) * F + q];
            const float mu = a.cjm[C_MU * F + q], lam = a.cjm[C_LAMBDA * F + q], buo = a.cjm[C_BUOY * F + q];
            float uL[9], uR[9];
#pragma unroll
            for (int v = 0; v < 9; v++) uL[v] = sL[sidx(v, mi, lane)], uR[v] = sR[sidx(v, mi + 1, lane)];
            lf_flux(n0, n1, n2, lam, mu, buo, a.alpha, uL, uR, Fv);
        } else {
#pragma unroll
            for (int v = 0; v < 9; v++) Fv[v] = 0.0f;
        }
#pragma unroll
        for (int v = 0; v < 9; v++) sL[sidx(v, mi, lane)] = Fv[v];
    }
    __syncthreads();

    // ---- phase C: flux difference at the tile's points
    for (int it = threadIdx.x; it < P * NL; it += SC_THREADS) {
        int pi, lane;
        split(it, P, pi, lane);
        const int p = p0 + pi;
        if (lane0 + lane >= lane_end || p >= nd) continue;
        int i, j, k;
        coords(p, lane, i, j, k);
        const long long q = g.at(i, j, k);
        const float coef = SC_LD(a.sjac[q]);  // DT * rDH / J
        float val[9];
        if (k >= _nz - 3) {
            float Fp[9], Fm[9];
#pragma unroll
            for (int v = 0; v < 9; v++) Fp[v] = sL[sidx(v, pi + 3, lane)], Fm[v] = sL[sidx(v, pi + 2, lane)];
            surface_diff(a, q, stride, mc0, coef, Fp, Fm, val);
        } else {
#pragma unroll
            for (int v = 0; v < 9; v++) {
                float f[6];
#pragma unroll
                for (int t = 0; t < 6; t++) f[t] = sL[sidx(v, pi + t, lane)];  // faces p-5/2 .. p+5/2
                val[v] = interior_diff(f, coef);
            }
        }
        epilogue<DIR>(a, q, i, j, k, val);
    }
}

// --------------------------------------------------------- free surface
// One thread per surface column (src/freeSurface.cpp:40-194).  The
// characteristic condition is restated with the inverse of the basis
// B = [n s t]: T = B^-1 sigma B^-T and v' = B^-1 v are the stress and
// velocity in that basis; after the condition, sigma = B T B^T, v = B v'.
// Evaluated in double from the float fields and rounded once.
__global__ void k_sc_surface(float *W, const float *__restrict__ cjm, DevGrid g, const float *__restrict__ decayG,
                             int ndecay, float *pgv, float *dis, float DT)
{
    const int i = CGFDM_HALO + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = CGFDM_HALO + blockIdx.y * blockDim.y + threadIdx.y;
    const int _nx = g.nxp - CGFDM_HALO, _ny = g.nyp - CGFDM_HALO, _nz = g.nzp - CGFDM_HALO;
    if (i >= _nx || j >= _ny) return;
    const long long F = g.fstride;
    const long long q = g.at(i, j, _nz - 1);
    const float mu = cjm[C_MU * F + q], lam = cjm[C_LAMBDA * F + q], buo = cjm[C_BUOY * F + q];
    float u[9], o[9];
    for (int v = 0; v < 9; v++) u[v] = W[v * F + q];
    const float nrm[3] = {cjm[C_ZT_X * F + q], cjm[C_ZT_Y * F + q], cjm[C_ZT_Z * F + q]};
    const float tan1[3] = {cjm[C_X_XI * F + q], cjm[C_Y_XI * F + q], cjm[C_Z_XI * F + q]};
    const float tan2[3] = {cjm[C_X_ET * F + q], cjm[C_Y_ET * F + q], cjm[C_Z_ET * F + q]};
    char_surface_point(u, mu, lam, buo, cjm[C_JAC * F + q], nrm, tan1, tan2, o);
    for (int v = 0; v < 9; v++) W[v * F + q] = o[v];

    // cubic extrapolation into the three halo layers above
    // (src/freeSurface.cpp:180-190: extrap3 = 4 k1 - 6 k2 + 4 k3 - k4)
    for (int v = 0; v < 9; v++) {
        float *c = W + v * F + q;
        for (int h = 1; h <= CGFDM_HALO; h++) {
            const long long P = g.plane;
            c[h * P] = 4.0f * c[(h - 1) * P] - 6.0f * c[(h - 2) * P] + 4.0f * c[(h - 3) * P] - c[(h - 4) * P];
        }
    }

    // sponge factors of the top four layers (the z pass of the last stage
    // did the layers below; the extrapolation above used values before it)
    if (decayG)
        for (int k = max(CGFDM_HALO, _nz - 4); k < _nz; k++) {
            const long long qk = g.at(i, j, k);
            for (int v = 0; v < 9; v++) W[v * F + qk] = decay_apply(W[v * F + qk], i, j, k, g, decayG, ndecay);
        }

    // displacement, Dis += (momentum * buoyancy) * DT after the sponge
    // (src/solve_displacement.cpp:45-62, called at src/propagate.cpp:264-266).
    // Only the surface layer of Dis is ever read (the FreeSurfU files,
    // src/data_io.cpp:619-633), so only that layer is integrated.
    if (dis)
        for (int c = 0; c < 3; c++)
            dis[c * F + q] = __fadd_rn(dis[c * F + q], __fmul_rn(__fmul_rn(W[c * F + q], buo), DT));

    // peak ground velocity of the surface layer (src/PGV.cpp:115-137)
    if (pgv) {
        const float Vx = __fmul_rn(W[0 * F + q], buo), Vy = __fmul_rn(W[1 * F + q], buo),
                    Vz = __fmul_rn(W[2 * F + q], buo);
        const float Vh = __fsqrt_rn(__fadd_rn(__fmul_rn(Vx, Vx), __fmul_rn(Vy, Vy)));
        const float V = __fsqrt_rn(__fadd_rn(__fadd_rn(__fmul_rn(Vx, Vx), __fmul_rn(Vy, Vy)), __fmul_rn(Vz, Vz)));
        const long long pp = (long long)(i - CGFDM_HALO) + (long long)(j - CGFDM_HALO) * g.nx;
        if (pgv[pp * 2 + 0] < Vh) pgv[pp * 2 + 0] = Vh;
        if (pgv[pp * 2 + 1] < V) pgv[pp * 2 + 1] = V;
    }
}

// DT * rDH / J per interior point, as cal_du forms it (jac = 1.0 / CJM[9]
// in double, stored float; src/alternative_flux_FD.cpp:1251, 1283).
__global__ void k_sc_sjac(const float *__restrict__ cjm, DevGrid g, float DT, float rDH, float *sjac)
{
    const int i = CGFDM_HALO + blockIdx.x * blockDim.x + threadIdx.x;
    const int j = CGFDM_HALO + blockIdx.y * blockDim.y + threadIdx.y;
    const int k = CGFDM_HALO + blockIdx.z;
    if (i >= g.nxp - CGFDM_HALO || j >= g.nyp - CGFDM_HALO) return;
    const long long q = g.at(i, j, k);
    const float jac = __double2float_rn(__ddiv_rn(1.0, (double)cjm[C_JAC * g.fstride + q]));
    sjac[q] = __fmul_rn(__fmul_rn(DT, rDH), jac);
}

// ------------------------------------------------------------ launchers
ScTiling sc_tiling(const DevGrid &g)
{
    ScTiling t;
    t.npos[0] = SCX_NPOS, t.nl[0] = SCX_NL;
    t.ntiles[0] = (g.nx + SCX_NPOS - 7) / (SCX_NPOS - 6);
    t.npos[1] = t.npos[2] = SCY_NPOS, t.nl[1] = t.nl[2] = SCY_NL;
    t.ntiles[1] = (g.ny + SCY_NPOS - 7) / (SCY_NPOS - 6);
    t.ntiles[2] = (g.nz + SCY_NPOS - 7) / (SCY_NPOS - 6);
    return t;
}

template <int DIR, int NPOS, int NL>
static cudaError_t tile_attr()
{
    return cudaFuncSetAttribute(k_sc_tile<DIR, NPOS, NL>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)sc_tile_smem(NPOS, NL));
}

cudaError_t sc_dir_prepare()
{
    CUDA_TRY((tile_attr<0, SCX_NPOS, SCX_NL>()));
    CUDA_TRY((tile_attr<1, SCY_NPOS, SCY_NL>()));
    CUDA_TRY((tile_attr<2, SCY_NPOS, SCY_NL>()));
    return cudaSuccess;
}

cudaError_t launch_sc_dir(int dir, ScDirArgs a, const ScTiling &t, cudaStream_t st)
{
    const DevGrid &g = a.g;
    if (dir == 0) {
        dim3 gr(t.ntiles[0], (g.ny + SCX_NL - 1) / SCX_NL, g.nz);
        k_sc_tile<0, SCX_NPOS, SCX_NL><<<gr, SC_THREADS, sc_tile_smem(SCX_NPOS, SCX_NL), st>>>(a);
    } else {
        const size_t smem = sc_tile_smem(SCY_NPOS, SCY_NL);
        if (dir == 1) {
            dim3 gr((g.nx + SCY_NL - 1) / SCY_NL, t.ntiles[1], g.nz);
            k_sc_tile<1, SCY_NPOS, SCY_NL><<<gr, SC_THREADS, smem, st>>>(a);
        } else {
            dim3 gr((g.nx + SCY_NL - 1) / SCY_NL, g.ny, t.ntiles[2]);
            k_sc_tile<2, SCY_NPOS, SCY_NL><<<gr, SC_THREADS, smem, st>>>(a);
        }
    }
    return cudaGetLastError();
}

cudaError_t launch_sc_surface(float *W, const float *cjm, DevGrid g, const float *decayG, int ndecay, float *pgv,
                              float *dis, float DT, cudaStream_t st)
{
    dim3 b(32, 4), gr((g.nx + 31) / 32, (g.ny + 3) / 4);
    k_sc_surface<<<gr, b, 0, st>>>(W, cjm, g, decayG, ndecay, pgv, dis, DT);
    return cudaGetLastError();
}

cudaError_t launch_sc_sjac(const float *cjm, DevGrid g, float DT, float rDH, float *sjac, cudaStream_t st)
{
    dim3 b(32, 8), gr((g.nx + 31) / 32, (g.ny + 7) / 8, g.nz);
    k_sc_sjac<<<gr, b, 0, st>>>(cjm, g, DT, rDH, sjac);
    return cudaGetLastError();
}

}  // namespace cgfdm
