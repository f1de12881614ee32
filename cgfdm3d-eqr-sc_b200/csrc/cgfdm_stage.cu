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
// Tiling: a CTA owns a 32 x 4 column tile and marches up a chunk of z.  Each
// z-plane of the nine stencil-input components, with the halo the one-sided
// operators need, arrives as one TMA box (40 x 8 x 1 x 9 floats,
// cp.async.bulk.tensor.4d) into a six-slot shared-memory ring, completion
// tracked by one mbarrier per slot; one elected thread issues the copies one
// plane ahead of use.  Derivatives along x, y and z all read the ring, so
// each value crosses HBM once per stage.  The FB signs are template
// parameters, so every stencil tap is a fixed shared-memory offset.  Metric,
// medium and RK inputs are plain coalesced loads issued before the ring wait.
//
// Every wait on an mbarrier is bounded: on timeout the CTA records the fact
// in a device error word, waits (bounded) for its copies in flight and exits.
//
// Arithmetic follows the reference's expression order term by term; built
// with --fmad=false the stage reproduces the reference's FP32 results bit for
// bit, built normally it differs only by FMA contraction.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "cg_ops.cuh"
#include "device.cuh"
#include "kernels.cuh"

// L2 promotion of the plane-ring (halo) and point-operand tensor maps, and
// which point operands are prefetched into L2 ahead of their loads.
#ifndef CG_PROMO_HALO
#define CG_PROMO_HALO CU_TENSOR_MAP_L2_PROMOTION_L2_256B
#endif
#ifndef CG_PROMO_POINT
#define CG_PROMO_POINT CU_TENSOR_MAP_L2_PROMOTION_L2_256B
#endif
#ifndef CG_PREFETCH_C
#define CG_PREFETCH_C 1
#endif
#ifndef CG_PREFETCH_MT
#define CG_PREFETCH_MT 1
#endif
// how many planes ahead the point operands are prefetched
#ifndef CG_PREFETCH_DIST
#define CG_PREFETCH_DIST 1
#endif
// how many planes beyond the newest ring fill the stencil planes are
// prefetched into L2 (0: none)
#ifndef CG_RING_PREFETCH_DIST
#define CG_RING_PREFETCH_DIST 0
#endif
// Cache policy of the point streams (used once per stage): 1 marks the
// stage-output and RK-sum stores evict-first, 2 also the metric, step-start
// and RK-sum loads, so L2 keeps the plane ring the neighbouring tiles share.
#ifndef CG_STREAM_HINTS
#define CG_STREAM_HINTS 1
#endif
// PML points: their auxiliary values prefetched into L2 before the ring wait
// (0: none, 1: this plane's, 2: this and the next plane's, 3: the next
// plane's, the item's first plane in its prologue).  With the face's loads
// issued together (below) the prefetch costs more than it saves: 400x400x200
// ran 7.80 ms per step without it and 8.02 ms with this plane's.
#ifndef CG_PML_PREFETCH
#define CG_PML_PREFETCH 0
#endif
// 1: a PML face's auxiliary, step-start and RK-sum values are all loaded
// before its first store (0: each field's loads after the previous field's
// stores, the order the compiler must keep for possibly aliasing pointers;
// 8.24 ms per step on 400x400x200 against 8.02 with them first)
#ifndef CG_PML_LOADS_FIRST
#define CG_PML_LOADS_FIRST 1
#endif
// 1: the plane-ring TMA loads carry an L2 evict-last policy
#ifndef CG_RING_EVICT_LAST
#define CG_RING_EVICT_LAST 0
#endif
#if CG_STREAM_HINTS >= 1
#define CG_ST(p, v) __stcs(&(p), (v))
#else
#define CG_ST(p, v) ((p) = (v))
#endif
// PML auxiliary stores: 1 evict-first like the stage outputs, 0 plain
// (400x400x200: 7.57 ms per step with 1, 7.51-7.57 with 0; evict-first
// loads as well, CG_STREAM_HINTS 2, took 8.32)
#ifndef CG_PML_STORE_HINT
#define CG_PML_STORE_HINT 0
#endif
#if CG_PML_STORE_HINT
#define CG_PST(p, v) __stcs(&(p), (v))
#else
#define CG_PST(p, v) ((p) = (v))
#endif
#if CG_STREAM_HINTS >= 2
#define CG_LD(p) __ldcs(&(p))
#else
#define CG_LD(p) (p)
#endif

// The file is compiled once per tile height: CG_TILE_Y 4 (this object, an
// inline namespace, so callers name its functions plainly) and 8
// (cgfdm_stage_ty8.cu, namespace cgfdm::ty8); a session picks one.
#ifndef CG_TILE_NS
#define CG_TILE_NS ty4
#define CG_TILE_NS_INLINE inline
#else
#define CG_TILE_NS_INLINE
#endif

namespace cgfdm {
CG_TILE_NS_INLINE namespace CG_TILE_NS {

// 32 x 4 tiles, three CTAs per SM (12 warps, 168 registers): 5 % faster on
// the 400 x 400 x 200 workload than 32 x 8 tiles at two CTAs per SM, the
// three independent per-plane barriers hiding more load latency.  A variant
// that also brought the point operands in by TMA (a second ring) lost
// occupancy and was 9 % slower.
#ifndef CG_TILE_Y
#define CG_TILE_Y 4      // rows per tile (threads per CTA = 32 x CG_TILE_Y)
#endif
#ifndef CG_CTAS_PER_SM
#define CG_CTAS_PER_SM 3
#endif
#define TX 32
#define TY CG_TILE_Y
#define BXW 40           // box width: columns i0-4 .. i0+35 (start 16-byte aligned)
#define BYW (TY + 4)     // box height: one-sided y halo (1 behind, 3 ahead)
#define PF (BXW * BYW)   // floats per field in a slot
#define SLOT_F (9 * PF)  // floats per slot
#define SLOT_BYTES (SLOT_F * 4)
#define NSLOT 6
// split pipeline: the current plane's halo box in a 2-slot ring, the
// z-window's interior column boxes (32 x TY x 9) in a 6-slot ring, and the
// point operands (13 metric/medium + 9 step-start + 9 RK-sum fields) of the
// current plane in one slot
#define CW (TX * TY)
#define CSLOT_F (9 * CW)
#define CSLOT_BYTES (CSLOT_F * 4)
#ifndef CG_SPLIT_HSLOTS
#define CG_SPLIT_HSLOTS 2   // halo ring: the current plane and CG_SPLIT_HSLOTS - 1 ahead
#endif
#ifndef CG_SPLIT_CSLOTS
#define CG_SPLIT_CSLOTS 6   // column ring: the 5-plane window and CG_SPLIT_CSLOTS - 5 ahead
#endif
#ifndef CG_SPLIT_PTS
#define CG_SPLIT_PTS 0      // 1: point operands staged by TMA, 0: plain loads as in the ring pipeline (measured 1 % faster)
#endif
#define NHSLOT CG_SPLIT_HSLOTS
#define NCSLOT CG_SPLIT_CSLOTS
#define PTS_F (CG_SPLIT_PTS ? 31 * CW : 0)
// Split pipeline: the first PML face of each PML point has its operands
// copied into a per-thread shared-memory stash by cp.async before the ring
// wait, so they arrive during the stencil instead of after it: 9 floats a
// thread (the auxiliary values), 18 (and the RK sum) or 27 (and the step
// start); 0: none.  Measured on 400 x 400 x 200: 32 x 8 tiles 7.97 ms per
// step without, 7.57 with 9, 8.30 with 18 (the larger carve-out leaves L1
// too small for the point loads); 32 x 4 tiles 8.03 without, 7.98 with 27.
#ifndef CG_PML_STASH
#define CG_PML_STASH (TY == 8 ? 9 : 27)
#endif
// 1: the first face's operands the stash does not hold are prefetched into
// L2 with the stash copies (32 x 8 tiles: 7.57 -> 7.51 ms per step; loading
// them into registers there instead spilled and took 9.26 ms)
#ifndef CG_PML_REST_PREFETCH
#define CG_PML_REST_PREFETCH 1
#endif
#define STASH_F (CG_PML_STASH * CW)
// the same stash in the ring pipeline (batches, linked parts), FP32 only:
// 9 floats took a 400x400x200 ring session from 8.25 to 8.04 ms per step but
// batch32 from 34.6 to 35.5 ms (its small shots' L1 shrinks with the
// carve-out), and batches are the ring's main users, so none by default
#ifndef CG_PML_STASH_RING
#define CG_PML_STASH_RING 0
#endif
#define STASH_RING_F (CG_PML_STASH_RING * TX * TY)
#define SLOT_HB (9 * PF * 2)  // mixed storage: bytes of a slot's FP16 delta box
// Mixed storage: the ring also holds each plane's FP16 delta box, so a CTA
// needs 104 KB and two fit on an SM.
#ifndef CG_MIX_CTAS_PER_SM
#define CG_MIX_CTAS_PER_SM 2
#endif

// Slot strides: a TMA copy's shared-memory destination must be 128-byte
// aligned, so each slot starts on a 128-byte boundary whatever the box size
// (a 40 x 6 x 9 float box, the 2-row tile's, is 8640 bytes).
#define SLOT_SF ((SLOT_F + 31) / 32 * 32)          // floats between halo-box slots
#define CSLOT_SF ((CSLOT_F + 31) / 32 * 32)        // floats between column-box slots
#define SLOT_HSF ((9 * PF + 63) / 64 * 64)         // halves between FP16 delta-box slots
static_assert(SLOT_SF % 32 == 0 && CSLOT_SF % 32 == 0 && SLOT_HSF % 64 == 0 && CW % 32 == 0,
              "TMA destinations on 128-byte boundaries");

size_t cg_stage_smem_bytes(bool mix)
{
    return (size_t)NSLOT * (SLOT_SF * 4 + (mix ? SLOT_HSF * 2 : 0)) + (mix ? 0 : STASH_RING_F * 4) + NSLOT * 8;
}
size_t cg_stage2_smem_bytes()
{
    return (size_t)(NHSLOT * SLOT_SF + NCSLOT * CSLOT_SF + PTS_F + STASH_F) * 4 + (NHSLOT + NCSLOT + 1) * 8;
}

// ------------------------------------------------------------ TMA helpers
__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }
// one float from global to shared memory, asynchronously (cp.async); this
// thread waits for its own copies with cp_async_wait_all
__device__ __forceinline__ void cp_async4(float *dst, const float *src)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem_u32(dst)), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

__device__ __forceinline__ void mbar_init(unsigned bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(bar), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(bar), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(unsigned bar, unsigned parity)
{
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}
// Bounded wait: gives up after `limit` clock cycles (2^31, about a second,
// unless a test shortens it).
__device__ __forceinline__ bool mbar_wait_bounded(unsigned bar, unsigned parity, long long limit)
{
    if (mbar_try_wait(bar, parity)) return true;
    long long t0 = clock64();
    while (!mbar_try_wait(bar, parity))
        if (clock64() - t0 > limit) return false;
    return true;
}
__device__ __forceinline__ void tma_load_4d(unsigned dst, const void *tmap, int x, int y, int z, int f, unsigned bar)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
        "[%6];\n" ::"r"(dst),
        "l"((unsigned long long)tmap), "r"(x), "r"(y), "r"(z), "r"(f), "r"(bar)
        : "memory");
}

// the same with an L2 cache policy (createpolicy) on the loaded lines
__device__ __forceinline__ void tma_load_4d_hint(unsigned dst, const void *tmap, int x, int y, int z, int f,
                                                 unsigned bar, unsigned long long policy)
{
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint [%0], "
        "[%1, {%2, %3, %4, %5}], [%6], %7;\n" ::"r"(dst),
        "l"((unsigned long long)tmap), "r"(x), "r"(y), "r"(z), "r"(f), "r"(bar), "l"(policy)
        : "memory");
}
__device__ __forceinline__ unsigned long long l2_evict_last_policy()
{
    unsigned long long p;
    asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;\n" : "=l"(p));
    return p;
}
__device__ __forceinline__ void l2_prefetch(const void *p)
{
    asm volatile("prefetch.global.L2 [%0];\n" ::"l"((unsigned long long)p));
}
__device__ __forceinline__ void tma_prefetch_4d(const void *tmap, int x, int y, int z, int f)
{
    asm volatile("cp.async.bulk.prefetch.tensor.4d.L2.global.tile [%0, {%1, %2, %3, %4}];\n" ::"l"(
                     (unsigned long long)tmap),
                 "r"(x), "r"(y), "r"(z), "r"(f)
                 : "memory");
}

// Stencil taps: hc points at this thread's cell of the current plane's halo
// box (x and y derivatives), zp[m] at its cell of plane k + FB3*(m-1) for the
// z derivative, ZS floats a field apart (the halo box itself in the ring
// pipeline, the interior column boxes in the split one).
template <int FB1, int FB2, int FB3, int ZS = PF>
struct Taps {
    const float *hc;
    const float *zp[5];
    __device__ __forceinline__ float rx(int f, float rDH) const
    {
        const float *c = hc + f * PF;
        return lop(c[-FB1], c[0], c[FB1], c[2 * FB1], c[3 * FB1], FB1, rDH);
    }
    __device__ __forceinline__ float ry(int f, float rDH) const
    {
        const float *c = hc + f * PF;
        return lop(c[-FB2 * BXW], c[0], c[FB2 * BXW], c[2 * FB2 * BXW], c[3 * FB2 * BXW], FB2, rDH);
    }
    __device__ __forceinline__ float rz(int f, float rDH) const
    {
        return lop(zp[0][f * ZS], zp[1][f * ZS], zp[2][f * ZS], zp[3][f * ZS], zp[4][f * ZS], FB3, rDH);
    }
    __device__ __forceinline__ float rdir(int dir, int f, float rDH) const
    {
        return dir == 0 ? rx(f, rDH) : dir == 1 ? ry(f, rDH) : rz(f, rDH);
    }
    __device__ __forceinline__ float c(int f) const { return hc[f * PF]; }
    __device__ __forceinline__ float z(int m, int f) const { return zp[m][f * ZS]; }
};

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

// Mixed storage: the stage's stencil input at a point, the FP32 step-start
// state plus the FP16 delta times its inverse scale (stage 0: no delta).
struct MixIn {
    const float *W;
    const __half *S;
    const float *inv;
    DevGrid g, gh;
    __device__ __forceinline__ float operator()(int f, int i, int j, int k) const
    {
        const float v = W[f * g.fstride + g.at(i, j, k)];
        return S ? v + __half2float(S[f * gh.fstride + gh.at(i, j, k)]) * inv[f] : v;
    }
};

// jt_at, ljt_xy and ljt_z of the traction image on the mixed-storage input
__device__ __forceinline__ void jt_at_m(const MixIn &w, const float *__restrict__ cjm, int i, int j, int k, int mdir,
                                        float out[3])
{
    const long long F = w.g.fstride, q = w.g.at(i, j, k);
    const float m0 = cjm[(3 * mdir + 0) * F + q], m1 = cjm[(3 * mdir + 1) * F + q], m2 = cjm[(3 * mdir + 2) * F + q];
    const float jac = cjm[C_JAC * F + q];
    const float Txx = w(3, i, j, k), Tyy = w(4, i, j, k), Tzz = w(5, i, j, k);
    const float Txy = w(6, i, j, k), Txz = w(7, i, j, k), Tyz = w(8, i, j, k);
    out[0] = ((m0 * Txx + m1 * Txy) + m2 * Txz) * jac;
    out[1] = ((m0 * Txy + m1 * Tyy) + m2 * Tyz) * jac;
    out[2] = ((m0 * Txz + m1 * Tyz) + m2 * Tzz) * jac;
}

__device__ __forceinline__ void ljt_xy_m(const MixIn &w, const float *__restrict__ cjm, int i, int j, int k, int dir,
                                         int FB, float rDH, float out[3])
{
    float J[5][3];
    for (int m = 0; m < 5; m++) {
        const int o = (m - 1) * FB;
        jt_at_m(w, cjm, dir == 0 ? i + o : i, dir == 1 ? j + o : j, k, dir, J[m]);
    }
    for (int c = 0; c < 3; c++) out[c] = lop(J[0][c], J[1][c], J[2][c], J[3][c], J[4][c], FB, rDH);
}

__device__ __forceinline__ void ljt_z_m(const MixIn &w, const float *__restrict__ cjm, int i, int j, int k, int ks_rel,
                                        int FB, float rDH, float out[3])
{
    float J[5][3];
    for (int m = 0; m < 5; m++) {
        const int l = 3 + (m - 1) * FB;
        int src = l, sign = 1;
        if (l > ks_rel) src = 2 * ks_rel - l, sign = -1;
        if (src == ks_rel) {
            J[m][0] = J[m][1] = J[m][2] = 0.0f;
        } else {
            jt_at_m(w, cjm, i, j, k + src - 3, 2, J[m]);
            if (sign < 0) J[m][0] = -J[m][0], J[m][1] = -J[m][1], J[m][2] = -J[m][2];
        }
    }
    for (int c = 0; c < 3; c++) out[c] = lop(J[0][c], J[1][c], J[2][c], J[3][c], J[4][c], FB, rDH);
}

// a delta to its stored FP16 value (scaled, saturated)
__device__ __forceinline__ __half to_h16(float x, float sc)
{
    return __float2half_rn(fminf(fmaxf(x * sc, -65504.0f), 65504.0f));
}

// ------------------------------------------------------------- the stage
// Persistent CTAs (three per SM) take work items -- one 32 x 4 column tile
// over one z-chunk -- from an atomic counter, chunks of a tile adjacent in
// the order, so concurrently running items share their halo and chunk-edge
// planes through L2 and no launch ends on a partial wave.
//
// BATCH = false: one session, its descriptor a kernel parameter (arguments
// and tensor maps in parameter space).  BATCH = true: the work items of
// nsess sessions, their descriptors in global memory; a CTA copies the
// arguments of the session its current item belongs to into shared memory.
//
// MIX = true: mixed-precision storage (see CgStageArgs).  Each slot also
// receives the plane's FP16 delta box; when a plane arrives, the CTA adds the
// delta into the FP32 box in place, so the taps read the stage's input as in
// the FP32 kernel.
//
// V2 = true: the split pipeline (see CSLOT_F above).  Only the current plane
// needs its x/y halo; the other planes of the z window need only the tile's
// interior columns, so the shared memory left over holds the current plane's
// point operands, brought in by TMA during the previous plane instead of
// being loaded by every thread at the plane's start.
template <int FB1, int FB2, int FB3, bool BATCH, bool HOUT, bool MIX = false, bool V2 = false>
__global__ void __launch_bounds__(TX *TY, MIX ? CG_MIX_CTAS_PER_SM : CG_CTAS_PER_SM)
    k_cg_stage(const __grid_constant__ CgStageDesc d1, const CgStageDesc *__restrict__ descs,
               const int *__restrict__ item_start, int nsess, int *work)
{
    static_assert(!(V2 && (BATCH || HOUT || MIX)), "the split pipeline is a single-session FP32 variant");
    extern __shared__ __align__(128) unsigned char smem_raw[];
    float *ring = reinterpret_cast<float *>(smem_raw);   // V2: the halo ring (2 slots)
    __half *ring16 = reinterpret_cast<__half *>(smem_raw + NSLOT * SLOT_SF * 4);
    float *col = ring + NHSLOT * SLOT_SF;                 // V2: column ring
    float *pts = col + NCSLOT * CSLOT_SF;                 // V2: point operands
    // PML operands of the first face (split: after the point slot; ring:
    // after the ring)
    float *stash = V2 ? pts + PTS_F : ring + NSLOT * SLOT_SF;
    constexpr int NCS = V2 ? NCSLOT : NSLOT;              // column (V2) or ring slots
    constexpr bool SPTS = V2 && CG_SPLIT_PTS;             // point operands staged in shared memory
    constexpr int NSTASH = V2 ? CG_PML_STASH : MIX ? 0 : CG_PML_STASH_RING;
    constexpr bool STASH = NSTASH > 0;
    unsigned long long *bars = reinterpret_cast<unsigned long long *>(
        V2 ? smem_raw + (NHSLOT * SLOT_SF + NCSLOT * CSLOT_SF + PTS_F + STASH_F) * 4
           : smem_raw + NSLOT * (SLOT_SF * 4 + (MIX ? SLOT_HSF * 2 : 0)) + (MIX ? 0 : STASH_RING_F * 4));
    // barrier of column (V2) or ring slot s
    auto cbar = [&](int s) -> unsigned long long * { return V2 ? &bars[NHSLOT + s] : &bars[s]; };
    __shared__ int s_abort, s_item;
    __shared__ float s_sc[MIX ? 9 : 1], s_inv[MIX ? 9 : 1];
    __shared__ int s_par;
    __shared__ __align__(16) CgStageArgs s_args;
    const CgStageArgs &a = BATCH ? s_args : d1.a;
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * TX + tx;
    constexpr int hyL = FB2 > 0 ? 1 : 3;
    constexpr int za = FB3 > 0 ? 1 : 3;
    const int cell = (ty + hyL) * BXW + tx + 4;
    const int total = BATCH ? item_start[nsess] : d1.a.ntiles_x * d1.a.ntiles_y * d1.a.nchunk;
    int sess = -1;
    // mixed storage (one thread): per-field scales of this step from the
    // bounds of the session's step-start state -- the bound of field f
    // maps below 2^13
    auto mix_scales = [&](const CgStageArgs &A0) {
        const int p = *A0.it_dev & 1;
        s_par = p;
        float M[9], Mv = 0.0f, Ms = 0.0f;
        for (int f = 0; f < 9; f++) {
            M[f] = __uint_as_float(A0.mx[p * 9 + f]);
            if (f < 3 && M[f] > Mv) Mv = M[f];
            if (f >= 3 && M[f] > Ms) Ms = M[f];
        }
        for (int f = 0; f < 9; f++) {
            const float c = f < 3 ? Ms / A0.zs_min : Mv * A0.zp_max;
            const float b = M[f] > c ? M[f] : c;
            int e = 0;
            if (b > 0.0f) frexpf(b, &e);
            s_sc[f] = b > 0.0f ? ldexpf(1.0f, 13 - e) : 1.0f;
            s_inv[f] = b > 0.0f ? ldexpf(1.0f, e - 13) : 1.0f;
        }
    };
    // mixed storage, stage 3 (all threads): this CTA's maxima of the new
    // state raise the bounds of the session's next step
    auto mix_flush = [&](const CgStageArgs &A0, float *r) {
        if (A0.irk != 3) return;
#pragma unroll 1
        for (int f = 0; f < 9; f++) {
            float v = r[f];
            for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
            if ((tid & 31) == 0 && v > 0.0f) atomicMax(&A0.mx[(s_par ^ 1) * 9 + f], __float_as_uint(v));
            r[f] = 0.0f;
        }
    };

    if (tid == 0) {
        s_abort = 0;
        for (int s = 0; s < (V2 ? NHSLOT + NCSLOT + 1 : NSLOT); s++) mbar_init(smem_u32(&bars[s]), 1);
        asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
        if constexpr (MIX && !BATCH) {
            mix_scales(d1.a);
            // the next step's bounds start from zero; stage 3 raises them
            if (d1.a.irk == 0 && blockIdx.x == 0)
                for (int f = 0; f < 9; f++) d1.a.mx[((s_par) ^ 1) * 9 + f] = 0u;
        }
    }
    unsigned seq0 = 0;  // fills issued by this CTA before the current item
    unsigned hseq0 = 0, pseq0 = 0;   // V2: halo-ring and point-slot fills before the current item
    float rm[MIX ? 9 : 1];   // mixed storage, stage 3: running max |new state| per field
#pragma unroll
    for (int f = 0; f < (MIX ? 9 : 1); f++) rm[f] = 0.0f;

    for (;;) {
    __syncthreads();
    if (tid == 0) s_item = atomicAdd(&work[0], 1);
    __syncthreads();
    const int gitem = s_item;
    if (gitem >= total || s_abort) break;
    if (BATCH) {
        // items of one session are consecutive; find this one's session
        int ns = 0;
        while (ns + 1 < nsess && gitem >= item_start[ns + 1]) ns++;
        if (ns != sess) {
            if constexpr (MIX) {
                // the previous session's maxima go to its bounds first
                if (sess >= 0) mix_flush(s_args, rm);
                __syncthreads();
            }
            sess = ns;
            const int *src = reinterpret_cast<const int *>(&descs[sess].a);
            int *dst = reinterpret_cast<int *>(&s_args);
            for (int w = tid; w < (int)(sizeof(CgStageArgs) / 4); w += TX * TY) dst[w] = src[w];
            __syncthreads();
            if constexpr (MIX) {
                if (tid == 0) {
                    mix_scales(s_args);
                    // the CTA with the session's first item resets its next
                    // step's bounds (stage 3, a later launch, raises them)
                    if (s_args.irk == 0 && gitem == item_start[sess])
                        for (int f = 0; f < 9; f++) s_args.mx[(s_par ^ 1) * 9 + f] = 0u;
                }
                __syncthreads();
            }
        }
    } else {
        sess = 0;
    }
    const CgStageDesc &D = BATCH ? descs[sess] : d1;
    const CUtensorMap *tmW = reinterpret_cast<const CUtensorMap *>(D.tmW);
    const CUtensorMap *tmC = reinterpret_cast<const CUtensorMap *>(D.tmC);
    const CUtensorMap *tmM = reinterpret_cast<const CUtensorMap *>(D.tmM);
    const CUtensorMap *tmT = reinterpret_cast<const CUtensorMap *>(D.tmT);
    const CUtensorMap *tmS = reinterpret_cast<const CUtensorMap *>(D.tmS);
    const CUtensorMap *tmWc = reinterpret_cast<const CUtensorMap *>(D.tmWc);
    const DevGrid g = a.g;
    const long long F = g.fstride;
    const int _nx = g.nxp - CGFDM_HALO, _ny = g.nyp - CGFDM_HALO, _nz = g.nzp - CGFDM_HALO;
    const float rDH = a.rDH, DT = a.DT;
    const int nPML = a.nPML;
    // position of point (ii, jj, kk) in the auxiliary arrays of PML face fc
    // (x faces: [z][y][x of the layer]; y faces: [z][y of the layer][x];
    // the z face: [z of the layer][y][x])
    auto pml_pos = [&](int fc, int ii, int jj, int kk) -> long long {
        const int ip = ii - CGFDM_HALO, jp = jj - CGFDM_HALO, kp = kk - CGFDM_HALO;
        if (fc == 0 || fc == 3)
            return (long long)(ip - (fc == 3 ? g.nx - nPML : 0)) + (long long)jp * nPML + (long long)kp * nPML * g.ny;
        if (fc == 1 || fc == 4)
            return (long long)ip + (long long)(jp - (fc == 4 ? g.ny - nPML : 0)) * g.nx +
                   (long long)kp * g.nx * nPML;
        return (long long)ip + (long long)jp * g.nx + (long long)kp * g.nx * g.ny;
    };
    const int item = BATCH ? gitem - item_start[sess] : gitem;
    const int tile = item / a.nchunk, chunk = item - tile * a.nchunk;
    const int by_ = tile / a.ntiles_x, bx_ = tile - by_ * a.ntiles_x;
    const int i0 = CGFDM_HALO + bx_ * TX, j0 = CGFDM_HALO + by_ * TY;
    const int i = i0 + tx, j = j0 + ty;
    const bool active = i < _nx && j < _ny;
    const int kb = CGFDM_HALO + chunk * a.kchunk;
    const int ke = min(kb + a.kchunk, _nz);
    if (kb >= ke) continue;
    const int kf = kb - za;                 // first plane this item loads
    const int tx0 = g.xoff + i0 - 4;        // halo box origin column: a multiple of 4 (16 bytes)
    const int ty0 = j0 - hyL;
    const int px0 = g.xoff + i0;            // point box origin column: a multiple of 4
    const int tx0h = MIX ? a.gh.xoff + i0 - 4 : 0;   // FP16 halo box origin: a multiple of 8 (16 bytes)

    // plane kk of this item is fill number seq0 + (kk - kf) of the CTA
    auto slot_of = [&](int kk) { return (int)((seq0 + (unsigned)(kk - kf)) % NCS); };
    auto parity_of = [&](int kk) { return ((seq0 + (unsigned)(kk - kf)) / NCS) & 1u; };
    // V2: halo box of plane kk (kb <= kk < ke) and point operands of plane kk
    auto hslot_of = [&](int kk) { return (int)((hseq0 + (unsigned)(kk - kb)) % NHSLOT); };
    auto hparity_of = [&](int kk) { return ((hseq0 + (unsigned)(kk - kb)) / NHSLOT) & 1u; };
    auto pparity_of = [&](int kk) { return (pseq0 + (unsigned)(kk - kb)) & 1u; };
    auto issue_halo = [&](int kk) {
        const int hs = hslot_of(kk);
        const unsigned bar = smem_u32(&bars[hs]);
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_expect_tx(bar, SLOT_BYTES);
        tma_load_4d(smem_u32(ring + hs * SLOT_SF), tmW, tx0, ty0, kk, 0, bar);
    };
    auto issue_pts = [&](int kk) {
        const unsigned bar = smem_u32(&bars[NHSLOT + NCSLOT]);
        const bool wm = a.irk == 1 || a.irk == 2, wt = a.irk != 0;
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        mbar_expect_tx(bar, (13 + (wm ? 9 : 0) + (wt ? 9 : 0)) * CW * 4);
        tma_load_4d(smem_u32(pts), tmC, px0, j0, kk, 0, bar);
        if (wm) tma_load_4d(smem_u32(pts + 13 * CW), tmM, px0, j0, kk, 0, bar);
        if (wt) tma_load_4d(smem_u32(pts + 22 * CW), tmT, px0, j0, kk, 0, bar);
    };
    auto issue = [&](int kk) {
        int s = slot_of(kk);
        unsigned bar = smem_u32(cbar(s));
        // test hook: leave this plane's slot without a copy (and without the
        // arrival that would complete its barrier phase), once
        if (a.stall && gitem == a.stall_item && kk - kf == a.stall_fill && atomicExch(a.stall, 0) == 1) return;
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
        if constexpr (MIX) {
            const bool hs = a.irk != 0;
            mbar_expect_tx(bar, SLOT_BYTES + (hs ? SLOT_HB : 0));
            tma_load_4d(smem_u32(ring + s * SLOT_SF), tmW, tx0, ty0, kk, 0, bar);
            if (hs) tma_load_4d(smem_u32(ring16 + s * SLOT_HSF), tmS, tx0h, ty0, kk, 0, bar);
            return;
        }
        if constexpr (V2) {
            mbar_expect_tx(bar, CSLOT_BYTES);
            tma_load_4d(smem_u32(col + s * CSLOT_SF), tmWc, px0, j0, kk, 0, bar);
            return;
        }
        mbar_expect_tx(bar, SLOT_BYTES);
        if (CG_RING_EVICT_LAST)
            tma_load_4d_hint(smem_u32(ring + s * SLOT_SF), tmW, tx0, ty0, kk, 0, bar, l2_evict_last_policy());
        else
            tma_load_4d(smem_u32(ring + s * SLOT_SF), tmW, tx0, ty0, kk, 0, bar);
    };
    // point operands of plane kk into L2 ahead of their plain loads
    auto prefetch_points = [&](int kk) {
        if (CG_PREFETCH_C) tma_prefetch_4d(tmC, px0, j0, kk, 0);
        if constexpr (MIX) {
            // the step-start state in stages 1-3, the FP16 accumulator (halo map) in 2-3
            if (CG_PREFETCH_MT && a.irk != 0) tma_prefetch_4d(tmM, px0, j0, kk, 0);
            if (CG_PREFETCH_MT && a.irk >= 2) tma_prefetch_4d(tmT, tx0h, ty0, kk, 0);
            return;
        }
        if (CG_PREFETCH_MT && (a.irk == 1 || a.irk == 2)) tma_prefetch_4d(tmM, px0, j0, kk, 0);
        if (CG_PREFETCH_MT && a.irk != 0) tma_prefetch_4d(tmT, px0, j0, kk, 0);
    };
    // mixed storage: the delta box of plane kk into its FP32 box, in place,
    // two values at a time (both boxes are [field][row][column], PF values a
    // field, so pair e of one is pair e of the other)
    auto convert = [&](int kk) {
        float2 *r32 = reinterpret_cast<float2 *>(ring + slot_of(kk) * SLOT_SF);
        const __half2 *r16 = reinterpret_cast<const __half2 *>(ring16 + slot_of(kk) * SLOT_HSF);
        for (int e = tid; e < 9 * PF / 2; e += TX * TY) {
            const float inv = s_inv[e / (PF / 2)];
            const float2 d = __half22float2(r16[e]);
            float2 w = r32[e];
            w.x = w.x + d.x * inv;
            w.y = w.y + d.y * inv;
            r32[e] = w;
        }
    };

    const long long wlim = a.wait_limit > 0 ? a.wait_limit : (1LL << 31);
    const int klast = ke - za + 3;          // last plane of the last window
    if (tid == 0) {
        for (int kk = kf; kk <= min(kf + NCS - 1, klast); kk++) issue(kk);
        if constexpr (V2) {
            for (int kk = kb; kk < min(kb + NHSLOT, ke); kk++) issue_halo(kk);
            if (SPTS) {
                issue_pts(kb);
                for (int kk = kb + 1; kk < min(kb + 3, ke); kk++) prefetch_points(kk);
            } else {
                for (int kk = kb; kk < min(kb + CG_PREFETCH_DIST, ke); kk++) prefetch_points(kk);
            }
        } else {
            for (int kk = kb; kk < min(kb + CG_PREFETCH_DIST, ke); kk++) prefetch_points(kk);
        }
    }
    int issued = min(kf + NCS - 1, klast);  // same value in every thread
    int hissued = min(kb + NHSLOT - 1, ke - 1), pissued = kb;  // V2
    // the first window: planes kf .. kf+3 (kf+4 is waited for in the loop)
    bool ok = true;
    for (int kk = kf; kk < kf + 4; kk++) ok = ok && mbar_wait_bounded(smem_u32(cbar(slot_of(kk))), parity_of(kk), wlim);
    if (!ok) {
        s_abort = 1;
        atomicOr(a.err, 1);
    }
    if constexpr (MIX) {
        // (after a failed wait the values are unused: the loop head leaves)
        if (a.irk != 0)
            for (int kk = kf; kk < kf + 4; kk++) convert(kk);
    }

    const float bx = active ? a.pml_beta_x[i] : 1.0f, by = active ? a.pml_beta_y[j] : 1.0f;
    // pml_on: one bit per absorbing face, x1 y1 z1 x2 y2 (bits 0..4)
    const bool inx1 = (a.pml_on & 1) && i < CGFDM_HALO + nPML, inx2 = (a.pml_on & 8) && i >= _nx - nPML;
    const bool iny1 = (a.pml_on & 2) && j < CGFDM_HALO + nPML, iny2 = (a.pml_on & 16) && j >= _ny - nPML;

    for (int k = kb; k < ke; k++) {
        __syncthreads();                    // every thread is done with plane k - za - 1's slot
        if (s_abort) break;
        // issue plane k - za - 1 + NCS into the slot plane k - za - 1 has left
        const int want = k - za - 1 + NCS;
        if (want > issued && want <= klast) {
            if (tid == 0) issue(want);
            issued = want;
        }
        if constexpr (V2) {
            // the halo slot plane k - 1 has left takes plane k - 1 + NHSLOT
            if (k > kb && k - 1 + NHSLOT < ke) {
                if (tid == 0) issue_halo(k - 1 + NHSLOT);
                hissued = k - 1 + NHSLOT;
            }
            if (SPTS) {
                if (tid == 0 && k + 3 < ke) prefetch_points(k + 3);
            } else {
                if (tid == 0 && k + CG_PREFETCH_DIST < ke) prefetch_points(k + CG_PREFETCH_DIST);
            }
        } else if (tid == 0) {
            if (k + CG_PREFETCH_DIST < ke) prefetch_points(k + CG_PREFETCH_DIST);
            if (CG_RING_PREFETCH_DIST > 0 && want + CG_RING_PREFETCH_DIST <= klast)
                tma_prefetch_4d(tmW, tx0, ty0, want + CG_RING_PREFETCH_DIST, 0);
        }
        const long long q = g.at(i, j, k);
        // point-wise operands, loaded before the ring wait
        float xi_x = 0, xi_y = 0, xi_z = 0, et_x = 0, et_y = 0, et_z = 0, zt_x = 0, zt_y = 0, zt_z = 0;
        float mu = 0, lam = 0, buo = 0, bz = 1;
        float mv[9], tv[9];
        if (!SPTS && active) {
            xi_x = CG_LD(a.cjm[C_XI_X * F + q]), xi_y = CG_LD(a.cjm[C_XI_Y * F + q]);
            xi_z = CG_LD(a.cjm[C_XI_Z * F + q]);
            et_x = CG_LD(a.cjm[C_ET_X * F + q]), et_y = CG_LD(a.cjm[C_ET_Y * F + q]);
            et_z = CG_LD(a.cjm[C_ET_Z * F + q]);
            zt_x = CG_LD(a.cjm[C_ZT_X * F + q]), zt_y = CG_LD(a.cjm[C_ZT_Y * F + q]);
            zt_z = CG_LD(a.cjm[C_ZT_Z * F + q]);
            mu = CG_LD(a.cjm[C_MU * F + q]), lam = CG_LD(a.cjm[C_LAMBDA * F + q]);
            buo = CG_LD(a.cjm[C_BUOY * F + q]) * 1.0f;  // buoyancy *= Crho (= 1)
            bz = a.pml_beta_z[k];
            if constexpr (MIX) {
                if (a.irk != 0)
                    for (int f = 0; f < 9; f++) mv[f] = a.Wm[f * F + q];
                if (a.irk >= 2) {
                    const long long qh = a.gh.at(i, j, k);
                    for (int f = 0; f < 9; f++) tv[f] = __half2float(a.T16[f * a.gh.fstride + qh]) * s_inv[f];
                }
            } else {
                if (a.irk == 1 || a.irk == 2)
                    for (int f = 0; f < 9; f++) mv[f] = CG_LD(a.Wm[f * F + q]);
                if (a.irk != 0)
                    for (int f = 0; f < 9; f++) tv[f] = CG_LD(a.T[f * F + q]);
            }
        }
        if (CG_PML_PREFETCH && active && (inx1 || iny1 || inx2 || iny2 || ((a.pml_on & 4) && k < CGFDM_HALO + nPML))) {
            const int i0p = i - CGFDM_HALO, j0p = j - CGFDM_HALO;
            const bool sel[5] = {inx1, iny1, (a.pml_on & 4) && k < CGFDM_HALO + nPML, inx2, iny2};
#pragma unroll 1
            for (int fc = 0; fc < 5; fc++) {
                if (!sel[fc]) continue;
                const PmlFace &P = a.face[fc];
#pragma unroll 1
                for (int dk = (CG_PML_PREFETCH == 3 && k > kb) ? 1 : 0; dk < (CG_PML_PREFETCH == 1 ? 1 : 2); dk++) {
                    const int k0p = k + dk - CGFDM_HALO;
                    if (k0p >= g.nz || (fc == 2 && k0p >= nPML)) break;
                    long long pos;
                    if (fc == 0 || fc == 3)
                        pos = (long long)(i0p - (fc == 3 ? g.nx - nPML : 0)) + (long long)j0p * nPML +
                              (long long)k0p * nPML * g.ny;
                    else if (fc == 1 || fc == 4)
                        pos = (long long)i0p + (long long)(j0p - (fc == 4 ? g.ny - nPML : 0)) * g.nx +
                              (long long)k0p * g.nx * nPML;
                    else
                        pos = (long long)i0p + (long long)j0p * g.nx + (long long)k0p * g.nx * g.ny;
                    // the buffers this stage reads: A (stage 0), B A T (1, 2), B T (3)
                    const float *bufs[3] = {a.irk == 0 ? P.A : P.B, a.irk == 1 || a.irk == 2 ? P.A : nullptr,
                                            a.irk != 0 ? P.T : nullptr};
                    for (int b = 0; b < 3; b++)
                        if (bufs[b])
                            for (int f = 0; f < 9; f++) l2_prefetch(bufs[b] + f * P.count + pos);
                }
            }
        }
        // the first PML face of this point: its operands into the stash
        int fc0 = -1;
        if constexpr (STASH) {
            const bool inz1p = (a.pml_on & 4) && k < CGFDM_HALO + nPML;
            fc0 = !active ? -1 : inx1 ? 0 : iny1 ? 1 : inz1p ? 2 : inx2 ? 3 : iny2 ? 4 : -1;
            if (fc0 >= 0) {
                const PmlFace &P = a.face[fc0];
                const long long pos = pml_pos(fc0, i, j, k);
                float *st = stash + ty * TX + tx;
                const float *cur = a.irk == 0 ? P.A : P.B;
                for (int f = 0; f < 9; f++) cp_async4(st + f * CW, cur + f * P.count + pos);
                if (NSTASH >= 18 && a.irk != 0)
                    for (int f = 0; f < 9; f++) cp_async4(st + (9 + f) * CW, P.T + f * P.count + pos);
                if (NSTASH >= 27 && (a.irk == 1 || a.irk == 2))
                    for (int f = 0; f < 9; f++) cp_async4(st + (18 + f) * CW, P.A + f * P.count + pos);
                cp_async_commit();
                // the face's other operands (RK sum, step start) into L2
                if (CG_PML_REST_PREFETCH) {
                    if (NSTASH < 18 && a.irk != 0)
                        for (int f = 0; f < 9; f++) l2_prefetch(P.T + f * P.count + pos);
                    if (NSTASH < 27 && (a.irk == 1 || a.irk == 2))
                        for (int f = 0; f < 9; f++) l2_prefetch(P.A + f * P.count + pos);
                }
            }
        }
        const int kk_new = k - za + 4;
        bool okw = mbar_wait_bounded(smem_u32(cbar(slot_of(kk_new))), parity_of(kk_new), wlim);
        if constexpr (V2) {
            okw = okw && mbar_wait_bounded(smem_u32(&bars[hslot_of(k)]), hparity_of(k), wlim);
        }
        if constexpr (SPTS) {
            okw = okw && mbar_wait_bounded(smem_u32(&bars[NHSLOT + NCSLOT]), pparity_of(k), wlim);
            if (okw && active) {
                const int cc = ty * TX + tx;
                xi_x = pts[C_XI_X * CW + cc], xi_y = pts[C_XI_Y * CW + cc], xi_z = pts[C_XI_Z * CW + cc];
                et_x = pts[C_ET_X * CW + cc], et_y = pts[C_ET_Y * CW + cc], et_z = pts[C_ET_Z * CW + cc];
                zt_x = pts[C_ZT_X * CW + cc], zt_y = pts[C_ZT_Y * CW + cc], zt_z = pts[C_ZT_Z * CW + cc];
                mu = pts[C_MU * CW + cc], lam = pts[C_LAMBDA * CW + cc];
                buo = pts[C_BUOY * CW + cc] * 1.0f;  // buoyancy *= Crho (= 1)
                bz = a.pml_beta_z[k];
                if (a.irk == 1 || a.irk == 2)
                    for (int f = 0; f < 9; f++) mv[f] = pts[(13 + f) * CW + cc];
                if (a.irk != 0)
                    for (int f = 0; f < 9; f++) tv[f] = pts[(22 + f) * CW + cc];
            }
            if (!okw) {
                s_abort = 1;
                atomicOr(a.err, 1);
            }
            __syncthreads();   // the point slot is free
            if (!s_abort && k + 1 < ke) {
                if (tid == 0) issue_pts(k + 1);
                pissued = k + 1;
            }
        } else if (!okw) {
            s_abort = 1;
            atomicOr(a.err, 1);
        }
        if constexpr (MIX) {
            if (a.irk != 0) {
                convert(kk_new);   // unused if a wait failed: the loop head then leaves
                __syncthreads();
                if (s_abort) continue;
            }
        }
        if (!okw) continue;
        if (!active) continue;

        Taps<FB1, FB2, FB3, V2 ? CW : PF> T;
        for (int m = 0; m < 5; m++) {
            int kk = k + FB3 * (m - 1);
            T.zp[m] = V2 ? col + slot_of(kk) * CSLOT_SF + ty * TX + tx : ring + slot_of(kk) * SLOT_SF + cell;
        }
        T.hc = V2 ? ring + hslot_of(k) * SLOT_SF + cell : T.zp[1];
        if (a.irk == 0)
            for (int f = 0; f < 9; f++) mv[f] = T.c(f);

        float h[9];
        const bool fs = a.fs_on && k >= _nz - 3;
        if (!fs) {
            // src/wave_deriv.cpp:214-282
            float d[9], c[9];
#pragma unroll
            for (int f = 0; f < 9; f++) d[f] = T.rx(f, rDH) * bx;
            dir_rhs(xi_x, xi_y, xi_z, d, mu, lam, buo, c);
#pragma unroll
            for (int f = 0; f < 9; f++) h[f] = c[f];
#pragma unroll
            for (int f = 0; f < 9; f++) d[f] = T.ry(f, rDH) * by;
            dir_rhs(et_x, et_y, et_z, d, mu, lam, buo, c);
#pragma unroll
            for (int f = 0; f < 9; f++) h[f] = h[f] + c[f];
#pragma unroll
            for (int f = 0; f < 9; f++) d[f] = T.rz(f, rDH) * bz;
            dir_rhs(zt_x, zt_y, zt_z, d, mu, lam, buo, c);
#pragma unroll
            for (int f = 0; f < 9; f++) h[f] = (h[f] + c[f]) * DT;
        } else {
            // src/freeSurface.cpp:345-492
            const int ks_rel = (_nz - 1) - k + CGFDM_HALO;
            float jx[3], jy[3], jz[3];
            if constexpr (MIX) {
                const MixIn w{a.Win, a.irk != 0 ? a.Sin : nullptr, s_inv, g, a.gh};
                ljt_xy_m(w, a.cjm, i, j, k, 0, FB1, rDH, jx);
                ljt_xy_m(w, a.cjm, i, j, k, 1, FB2, rDH, jy);
                ljt_z_m(w, a.cjm, i, j, k, ks_rel, FB3, rDH, jz);
            } else {
                ljt_xy(a.Win, a.cjm, g, i, j, k, 0, FB1, rDH, jx);
                ljt_xy(a.Win, a.cjm, g, i, j, k, 1, FB2, rDH, jy);
                ljt_z(a.Win, a.cjm, g, i, j, k, ks_rel, FB3, rDH, jz);
            }
            const float jinv = 1.0f / a.cjm[C_JAC * F + q];
            const float bj = buo * jinv;
            for (int c = 0; c < 3; c++) h[c] = (bj * ((jx[c] * bx + jy[c] * by) + jz[c])) * DT;
            float vxi[3], vet[3], vzt[3];
            for (int c = 0; c < 3; c++) vxi[c] = T.rx(c, rDH) * bx;
            for (int c = 0; c < 3; c++) vet[c] = T.ry(c, rDH) * by;
            if (k == _nz - 1) {
                const long long s = g.at2(i, j);
                if (a.vdstore)
                    for (int c = 0; c < 3; c++) {
                        a.vdstore[c * g.plane + s] = vxi[c];
                        a.vdstore[(3 + c) * g.plane + s] = vet[c];
                    }
                for (int r = 0; r < 3; r++) {
                    const float *dx = a.rdz + (long long)(r * 3) * g.plane + s;
                    const float *dy = a.rdz + (long long)(9 + r * 3) * g.plane + s;
                    vzt[r] = ((dx[0] * vxi[0] + dx[g.plane] * vxi[1]) + dx[2 * g.plane] * vxi[2]) +
                             ((dy[0] * vet[0] + dy[g.plane] * vet[1]) + dy[2 * g.plane] * vet[2]);
                }
            } else if (k == _nz - 2) {
                // L2: plane k + FB3 is tap m = 2
                for (int c = 0; c < 3; c++) vzt[c] = ((float)FB3 * (T.z(2, c) - T.z(1, c))) * rDH;
            } else {
                // L3: planes k, k + FB3, k + 2 FB3 are taps 1, 2, 3
                for (int c = 0; c < 3; c++)
                    vzt[c] = ((float)FB3 * ((CG_CF1 * T.z(1, c) + CG_CF2 * T.z(2, c)) +
                                            CG_CF3 * T.z(3, c))) *
                             rDH;
            }
            float s1[9], s2[9], s3[9];
            dir_stress(xi_x, xi_y, xi_z, vxi, mu, lam, s1);
            dir_stress(et_x, et_y, et_z, vet, mu, lam, s2);
            dir_stress(zt_x, zt_y, zt_z, vzt, mu, lam, s3);
            for (int f = 3; f < 9; f++) h[f] = ((s1[f] + s2[f]) + s3[f]) * DT;
        }

        // ---- PML auxiliaries, faces in the reference's launch order x1 y1 z1 x2 y2
        const bool inz1 = (a.pml_on & 4) && k < CGFDM_HALO + nPML;
        if (inx1 || iny1 || inz1 || inx2 || iny2) {
            const bool sel[5] = {inx1, iny1, inz1, inx2, iny2};
            for (int fc = 0; fc < 5; fc++) {
                if (!sel[fc]) continue;
                const int dir = fc == 0 || fc == 3 ? 0 : fc == 1 || fc == 4 ? 1 : 2;
                const PmlFace &P = a.face[fc];
                const long long pos = pml_pos(fc, i, j, k);
                const float *al = dir == 0 ? a.pml_alpha_x : dir == 1 ? a.pml_alpha_y : a.pml_alpha_z;
                const float *be = dir == 0 ? a.pml_beta_x : dir == 1 ? a.pml_beta_y : a.pml_beta_z;
                const float *dd = dir == 0 ? a.pml_d_x : dir == 1 ? a.pml_d_y : a.pml_d_z;
                const int ix = dir == 0 ? i : dir == 1 ? j : k;
                const float dval = dd[ix], beta = be[ix], alpha_d = dval + al[ix];
                const float m0 = dir == 0 ? xi_x : dir == 1 ? et_x : zt_x;
                const float m1 = dir == 0 ? xi_y : dir == 1 ? et_y : zt_y;
                const float m2 = dir == 0 ? xi_z : dir == 1 ? et_z : zt_z;
                float d[9], rhs[9], aux[9], hA[9];
                for (int f = 0; f < 9; f++) d[f] = T.rdir(dir, f, rDH) * dval;
                dir_rhs(m0, m1, m2, d, mu, lam, buo, rhs);
                const float *cur = a.irk == 0 ? P.A : P.B;
                // every operand of this face loaded before the first store:
                // the stores go through pointers the compiler cannot tell
                // apart from the loads, which would otherwise wait for them
                float xa[9], xt[9];
                if (STASH && fc == fc0) {
                    cp_async_wait_all();
                    const float *st = stash + ty * TX + tx;
                    for (int f = 0; f < 9; f++) aux[f] = st[f * CW];
                    if (a.irk == 1 || a.irk == 2)
                        for (int f = 0; f < 9; f++)
                            xa[f] = NSTASH >= 27 ? st[(18 + f) * CW] : P.A[f * P.count + pos];
                    if (a.irk != 0)
                        for (int f = 0; f < 9; f++)
                            xt[f] = NSTASH >= 18 ? st[(9 + f) * CW] : P.T[f * P.count + pos];
                } else {
                    for (int f = 0; f < 9; f++) aux[f] = cur[f * P.count + pos];
                    if (CG_PML_LOADS_FIRST) {
                        if (a.irk == 1 || a.irk == 2)
                            for (int f = 0; f < 9; f++) xa[f] = P.A[f * P.count + pos];
                        if (a.irk != 0)
                            for (int f = 0; f < 9; f++) xt[f] = P.T[f * P.count + pos];
                    }
                }
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
                        CG_PST(P.T[f * P.count + pos], aux[f] + RK_BETA1 * hA[f]);
                        CG_PST(P.B[f * P.count + pos], aux[f] + RK_ALPHA2 * hA[f]);
                    }
                } else if (a.irk == 1 || a.irk == 2) {
                    for (int f = 0; f < 9; f++) {
                        float mA = CG_PML_LOADS_FIRST || (STASH && fc == fc0) ? xa[f] : P.A[f * P.count + pos];
                        float t = CG_PML_LOADS_FIRST || (STASH && fc == fc0) ? xt[f] : P.T[f * P.count + pos];
                        CG_PST(P.T[f * P.count + pos], t + (a.irk == 1 ? RK_BETA2 : RK_BETA3) * hA[f]);
                        CG_PST(P.B[f * P.count + pos], a.irk == 1 ? mA + RK_ALPHA3 * hA[f] : mA + hA[f]);
                    }
                } else {
                    for (int f = 0; f < 9; f++)
                        CG_PST(P.A[f * P.count + pos],
                               (CG_PML_LOADS_FIRST || (STASH && fc == fc0) ? xt[f] : P.T[f * P.count + pos]) +
                                   RK_BETA4 * hA[f]);
                }
            }
        }

        // the adjoint's gradient reads h outside the PML layers only
        if (a.hstore && a.hbox.contains(i, j, k)) {
            const long long hq = a.hbox.at(i, j, k);
#pragma unroll
            for (int f = 0; f < 9; f++) a.hstore[f * a.hbox.fstride + hq] = h[f];
        }

        // ---- RK4 update of the wavefield (src/wave_rk.cpp:17-104)
        float wout[9];
        if constexpr (MIX) {
            // stage deltas d1 = h0 / 2, d2 = h1 / 2, d3 = h2 and the
            // accumulator delta t - m (b1 h0 = d1 / 3, formed in stage 1)
            const long long qh = a.gh.at(i, j, k), Fh = a.gh.fstride;
            if (a.irk == 0) {
#pragma unroll
                for (int f = 0; f < 9; f++) a.Sout[f * Fh + qh] = to_h16(RK_ALPHA2 * h[f], s_sc[f]);
            } else if (a.irk == 1) {
                const __half *cur16 = ring16 + slot_of(k) * SLOT_HSF + cell;
#pragma unroll
                for (int f = 0; f < 9; f++) {
                    const float d1 = __half2float(cur16[f * PF]) * s_inv[f];
                    a.T16[f * Fh + qh] = to_h16(d1 * 0.33333334f + RK_BETA2 * h[f], s_sc[f]);
                    a.Sout[f * Fh + qh] = to_h16(RK_ALPHA3 * h[f], s_sc[f]);
                }
            } else if (a.irk == 2) {
#pragma unroll
                for (int f = 0; f < 9; f++) {
                    a.T16[f * Fh + qh] = to_h16(tv[f] + RK_BETA3 * h[f], s_sc[f]);
                    a.Sout[f * Fh + qh] = to_h16(h[f], s_sc[f]);
                }
            } else {
#pragma unroll
                for (int f = 0; f < 9; f++) {
                    wout[f] = mv[f] + (tv[f] + RK_BETA4 * h[f]);
                    CG_ST(a.Wout[f * F + q], wout[f]);
                    rm[f] = fmaxf(rm[f], fabsf(wout[f]));
                }
            }
        } else {
        if (a.irk == 0) {
#pragma unroll
            for (int f = 0; f < 9; f++) {
                CG_ST(a.T[f * F + q], mv[f] + RK_BETA1 * h[f]);
                wout[f] = mv[f] + RK_ALPHA2 * h[f];
            }
        } else if (a.irk == 1) {
#pragma unroll
            for (int f = 0; f < 9; f++) {
                CG_ST(a.T[f * F + q], tv[f] + RK_BETA2 * h[f]);
                wout[f] = mv[f] + RK_ALPHA3 * h[f];
            }
        } else if (a.irk == 2) {
#pragma unroll
            for (int f = 0; f < 9; f++) {
                CG_ST(a.T[f * F + q], tv[f] + RK_BETA3 * h[f]);
                wout[f] = mv[f] + h[f];
            }
        } else {
#pragma unroll
            for (int f = 0; f < 9; f++) wout[f] = tv[f] + RK_BETA4 * h[f];
        }
#pragma unroll
        for (int f = 0; f < 9; f++) CG_ST(a.Wout[f * F + q], wout[f]);
        }
        if (HOUT) {
            // a part of a decomposed grid: the interior layers next to a face
            // shared with a neighbour go straight into the neighbour's halo
#pragma unroll 1
            for (int fc = 0; fc < 6; fc++) {
                const HaloOut &h = a.ho[fc];
                if (!h.base) continue;
                const int axis = fc >> 1;
                const int c = axis == 0 ? i : axis == 1 ? j : k;
                const int n = axis == 0 ? g.nx : axis == 1 ? g.ny : g.nz;
                if ((fc & 1) ? c < n : c >= 2 * CGFDM_HALO) continue;
                const long long d = (long long)(k + (axis == 2 ? h.shift : 0)) * h.plane +
                                    (long long)(j + (axis == 1 ? h.shift : 0)) * h.pitch + h.xoff +
                                    (i + (axis == 0 ? h.shift : 0));
#pragma unroll
                for (int f = 0; f < 9; f++) h.base[f * h.fstride + d] = wout[f];
            }
        }

        if (a.irk == 3) {
            // displacement: only the surface layer is ever read (the FreeSurfU
            // files, src/data_io.cpp:619-633), so only it is integrated
            if (a.dis && k == _nz - 1)
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
    __syncthreads();
    if (s_abort) {
        // no copy may still be landing in shared memory when the CTA exits
        if (tid == 0) {
            for (int kk = max(kf, issued - NCS + 1); kk <= issued; kk++)
                if (!mbar_wait_bounded(smem_u32(cbar(slot_of(kk))), parity_of(kk), wlim)) atomicOr(a.err, 2);
            if constexpr (V2) {
                for (int kk = max(kb, hissued - NHSLOT + 1); kk <= hissued; kk++)
                    if (!mbar_wait_bounded(smem_u32(&bars[hslot_of(kk)]), hparity_of(kk), wlim)) atomicOr(a.err, 2);
            }
            if constexpr (SPTS) {
                if (!mbar_wait_bounded(smem_u32(&bars[NHSLOT + NCSLOT]), pparity_of(pissued), wlim)) atomicOr(a.err, 2);
            }
        }
        break;
    }
    // no copy into the stash outlives the item (one may be pending after a
    // failed wait)
    if constexpr (STASH) cp_async_wait_all();
    seq0 += (unsigned)(issued - kf + 1);
    hseq0 += (unsigned)(ke - kb);
    pseq0 += (unsigned)(ke - kb);
    }  // work items

    if constexpr (MIX) {
        // stage 3: raise the bounds of the next step with this CTA's maxima
        if (!BATCH) mix_flush(d1.a, rm);
        else if (sess >= 0) mix_flush(s_args, rm);
    }
    // the last CTA out resets the work counter for the next launch
    __syncthreads();
    if (tid == 0) {
        __threadfence();
        int done = atomicAdd(&work[1], 1);
        if (done == (int)(gridDim.x * gridDim.y * gridDim.z) - 1) {
            atomicExch(&work[0], 0);
            atomicExch(&work[1], 0);
            __threadfence();
        }
    }
}

// ------------------------------------------------------------ host side
int cg_stage_ctas_per_sm() { return CG_CTAS_PER_SM; }
int cg_stage_tile_y() { return TY; }

template <int FB1, int FB2, int FB3, bool BATCH, bool HOUT, bool MIX, bool V2>
static cudaError_t launch_t(const CgStageDesc &d1, const CgStageDesc *descs, const int *item_start, int nsess,
                            int *work, int ctas, cudaStream_t st)
{
    // The shared-memory limit is an attribute of the kernel on the current
    // device (and is lost with a device reset), so it is set on every launch:
    // a host-side call of about a microsecond, legal during stream capture.
    const size_t smem = V2 ? cg_stage2_smem_bytes() : cg_stage_smem_bytes(MIX);
    CUDA_TRY(cudaFuncSetAttribute(k_cg_stage<FB1, FB2, FB3, BATCH, HOUT, MIX, V2>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    k_cg_stage<FB1, FB2, FB3, BATCH, HOUT, MIX, V2>
        <<<ctas, dim3(TX, TY, 1), smem, st>>>(d1, descs, item_start, nsess, work);
    return cudaGetLastError();
}

template <bool BATCH, bool HOUT, bool MIX = false, bool V2 = false>
static cudaError_t launch_b(int FB1, int FB2, int FB3, const CgStageDesc &d1, const CgStageDesc *descs,
                            const int *item_start, int nsess, int *work, int ctas, cudaStream_t st)
{
    const int key = (FB1 > 0) * 4 + (FB2 > 0) * 2 + (FB3 > 0);
    switch (key) {
    case 0: return launch_t<-1, -1, -1, BATCH, HOUT, MIX, V2>(d1, descs, item_start, nsess, work, ctas, st);
    case 1: return launch_t<-1, -1, 1, BATCH, HOUT, MIX, V2>(d1, descs, item_start, nsess, work, ctas, st);
    case 2: return launch_t<-1, 1, -1, BATCH, HOUT, MIX, V2>(d1, descs, item_start, nsess, work, ctas, st);
    case 3: return launch_t<-1, 1, 1, BATCH, HOUT, MIX, V2>(d1, descs, item_start, nsess, work, ctas, st);
    case 4: return launch_t<1, -1, -1, BATCH, HOUT, MIX, V2>(d1, descs, item_start, nsess, work, ctas, st);
    case 5: return launch_t<1, -1, 1, BATCH, HOUT, MIX, V2>(d1, descs, item_start, nsess, work, ctas, st);
    case 6: return launch_t<1, 1, -1, BATCH, HOUT, MIX, V2>(d1, descs, item_start, nsess, work, ctas, st);
    default: return launch_t<1, 1, 1, BATCH, HOUT, MIX, V2>(d1, descs, item_start, nsess, work, ctas, st);
    }
}

int cg_stage_mix_ctas_per_sm() { return CG_MIX_CTAS_PER_SM; }

cudaError_t launch_cg_stage_split(int FB1, int FB2, int FB3, const CgStageDesc &d, int *work, int ctas,
                                  cudaStream_t st)
{
    return launch_b<false, false, false, true>(FB1, FB2, FB3, d, nullptr, nullptr, 1, work, ctas, st);
}

cudaError_t launch_cg_stage_mix(int FB1, int FB2, int FB3, const CgStageDesc &d, int *work, int ctas, cudaStream_t st)
{
    return launch_b<false, false, true>(FB1, FB2, FB3, d, nullptr, nullptr, 1, work, ctas, st);
}

cudaError_t launch_cg_stage_batch_mix(int FB1, int FB2, int FB3, const CgStageDesc *descs, const int *item_start,
                                      int nsess, int *work, int ctas, cudaStream_t st)
{
    static const CgStageDesc unused{};
    return launch_b<true, false, true>(FB1, FB2, FB3, unused, descs, item_start, nsess, work, ctas, st);
}

cudaError_t make_field_tmap16(void *out, const __half *base, const DevGrid &gh, int nf)
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        cudaDriverEntryPointQueryResult q;
        void *fn = nullptr;
        CUDA_TRY(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !fn) return cudaErrorNotSupported;
        encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    cuuint64_t dims[4] = {(cuuint64_t)gh.pitch, (cuuint64_t)gh.nyp, (cuuint64_t)gh.nzp, (cuuint64_t)nf};
    cuuint64_t strides[3] = {(cuuint64_t)gh.pitch * 2, (cuuint64_t)gh.plane * 2, (cuuint64_t)gh.fstride * 2};
    cuuint32_t box[4] = {(cuuint32_t)BXW, (cuuint32_t)BYW, 1, (cuuint32_t)nf};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = encode(reinterpret_cast<CUtensorMap *>(out), CU_TENSOR_MAP_DATA_TYPE_FLOAT16, 4, (void *)base, dims,
                        strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CG_PROMO_HALO,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

// Impedance bounds of the medium over the interior (float bits; the atomics
// order non-negative floats as their bit patterns): min sqrt(mu / b) into
// out[0], max sqrt((lambda + 2 mu) / b) into out[1].
__global__ void k_impedance_bounds(const float *__restrict__ cjm, DevGrid g, unsigned *out)
{
    const int i = blockIdx.x * 32 + threadIdx.x + CGFDM_HALO, j = blockIdx.y * 4 + threadIdx.y + CGFDM_HALO;
    const int k = blockIdx.z + CGFDM_HALO;
    float zs = 3.4e38f, zp = 0.0f;
    if (i < g.nxp - CGFDM_HALO && j < g.nyp - CGFDM_HALO) {
        const long long F = g.fstride, q = g.at(i, j, k);
        const float mu = cjm[C_MU * F + q], lam = cjm[C_LAMBDA * F + q], b = cjm[C_BUOY * F + q];
        zs = __fsqrt_rn(__fdiv_rn(mu, b));
        zp = __fsqrt_rn(__fdiv_rn(__fadd_rn(lam, __fmul_rn(2.0f, mu)), b));
    }
    for (int o = 16; o > 0; o >>= 1) {
        zs = fminf(zs, __shfl_xor_sync(0xffffffffu, zs, o));
        zp = fmaxf(zp, __shfl_xor_sync(0xffffffffu, zp, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(&out[0], __float_as_uint(zs));
        atomicMax(&out[1], __float_as_uint(zp));
    }
}

cudaError_t launch_impedance_bounds(const float *cjm, DevGrid g, unsigned *out, cudaStream_t st)
{
    k_impedance_bounds<<<dim3((g.nx + 31) / 32, (g.ny + 3) / 4, g.nz), dim3(32, 4), 0, st>>>(cjm, g, out);
    return cudaGetLastError();
}

cudaError_t launch_cg_stage(int FB1, int FB2, int FB3, const CgStageDesc &d, int *work, int ctas, cudaStream_t st,
                            bool halo_out)
{
    if (halo_out) return launch_b<false, true>(FB1, FB2, FB3, d, nullptr, nullptr, 1, work, ctas, st);
    return launch_b<false, false>(FB1, FB2, FB3, d, nullptr, nullptr, 1, work, ctas, st);
}

cudaError_t launch_cg_stage_batch(int FB1, int FB2, int FB3, const CgStageDesc *descs, const int *item_start,
                                  int nsess, int *work, int ctas, cudaStream_t st)
{
    static const CgStageDesc unused{};
    return launch_b<true, false>(FB1, FB2, FB3, unused, descs, item_start, nsess, work, ctas, st);
}

cudaError_t make_field_tmap(void *out, const float *base, const DevGrid &g, int nf, bool halo_box)
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
    if (!encode) {
        cudaDriverEntryPointQueryResult q;
        void *fn = nullptr;
        CUDA_TRY(cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q));
        if (q != cudaDriverEntryPointSuccess || !fn) return cudaErrorNotSupported;
        encode = (PFN_cuTensorMapEncodeTiled_v12000)fn;
    }
    cuuint64_t dims[4] = {(cuuint64_t)g.pitch, (cuuint64_t)g.nyp, (cuuint64_t)g.nzp, (cuuint64_t)nf};
    cuuint64_t strides[3] = {(cuuint64_t)g.pitch * 4, (cuuint64_t)g.plane * 4, (cuuint64_t)g.fstride * 4};
    cuuint32_t box[4] = {halo_box ? (cuuint32_t)BXW : (cuuint32_t)TX, halo_box ? (cuuint32_t)BYW : (cuuint32_t)TY, 1,
                         (cuuint32_t)nf};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = encode(reinterpret_cast<CUtensorMap *>(out), CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, (void *)base, dims,
                        strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        halo_box ? CG_PROMO_HALO : CG_PROMO_POINT, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    return r == CUDA_SUCCESS ? cudaSuccess : cudaErrorInvalidValue;
}

}  // namespace CG_TILE_NS
}  // namespace cgfdm
