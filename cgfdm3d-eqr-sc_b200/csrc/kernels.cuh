// Kernel launch interfaces (host side).
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>

#include "device.cuh"

namespace cgfdm {

// ---------------------------------------------------------------- setup
cudaError_t launch_setup(const float *d_coord, const float *d_medium, float *cjm, float *rdz, DevGrid g,
                         float rDH, int scheme, int fp64, cudaStream_t st);
// The padded grid's coordinates from the surface height map (mode: 0 flat,
// 1 terrain-following in float, 2 in double; see Model::coord_mode).
cudaError_t launch_build_coords(float *coord, const float *terrain, int nxp, int nyp, int nzp, int mode, float DH,
                                int originalX, int originalY, int NZ, float depth_f, double depth_d, cudaStream_t st);
cudaError_t launch_scale_moment(float *rate, const long long *cell, long long npts, int nt, const float *cjm,
                                DevGrid g, float DH, cudaStream_t st);

// ------------------------------------------------------------ PML state
// One absorbing face: Aux fields for its slab, three buffers (A holds the
// step-start value and receives the final stage, B the intermediate stage
// values, T the RK accumulator), each 9 fields of `count` floats.
struct PmlFace {
    float *A, *B, *T;
    long long count;     // points in the slab
    int n0, n1;          // slab extent along its two fastest axes (see pml_pos)
};

// The points outside the PML layers, where the adjoint takes a gradient:
// i in [x0, x0 + nx), j in [y0, y0 + ny), k in [z0, z0 + nz) (padded-grid
// indices), stored field by field as [k][j][i] with `fstride` floats a field.
struct HBox {
    int x0, y0, z0, nx, ny, nz;
    long long fstride;
    __host__ __device__ __forceinline__ bool contains(int i, int j, int k) const
    {
        return i >= x0 && i < x0 + nx && j >= y0 && j < y0 + ny && k >= z0 && k < z0 + nz;
    }
    __host__ __device__ __forceinline__ long long at(int i, int j, int k) const
    {
        return ((long long)(k - z0) * ny + (j - y0)) * nx + (i - x0);
    }
};

// --------------------------------------------------------- CGFDM stage
// Where a part's stage kernel stores the interior layers next to one face:
// the neighbour's output buffer of the same stage (its halo on the facing
// side), that buffer's layout, and the shift from this part's padded index
// along the face's axis to the neighbour's.  base null: no neighbour.
struct HaloOut {
    float *base;
    long long plane, fstride;
    int pitch, xoff, shift;
};

struct CgStageArgs {
    DevGrid g;
    HBox hbox;           // layout of hstore
    const float *Win;    // stencil input of this stage
    const float *Wm;     // values at the start of the step (RK "m")
    float *T;            // RK accumulator
    float *Wout;         // stage output
    const float *cjm;    // 13 fields
    const float *rdz;    // 18 surface fields [nyp][pitch]
    const float *pml_alpha_x, *pml_beta_x, *pml_d_x;
    const float *pml_alpha_y, *pml_beta_y, *pml_d_y;
    const float *pml_alpha_z, *pml_beta_z, *pml_d_z;
    PmlFace face[5];     // x1 y1 z1 x2 y2 (order of src/pml_deriv.cpp:633-646)
    float *pgv;          // [ny][nx][2] running max, stage 3 only
    float *dis;          // displacement, 3 fields in the W layout, stage 3 only
    float *hstore;       // or null: receives this stage's RHS h for the adjoint (9 fields, HBox layout)
    float *vdstore;      // or null: receives the surface layer's xi/eta velocity derivatives (6 x plane)
    int *err;            // device error word: bit 0 = a bounded wait gave up, bit 1 = the drain after it did
    // Test hook (null in normal runs): while *stall is 1, the CTA that takes
    // work item stall_item does not issue the copy of its plane number
    // stall_fill (counted from the item's first plane) and clears *stall, so
    // the wait for that plane runs out.  wait_limit: clock cycles a bounded
    // wait spins before it gives up (0: 2^31, about a second).
    int *stall;
    int stall_item, stall_fill;
    long long wait_limit;
    // Mixed-precision storage ("storage": "fp16"; the MIX instantiation).
    // The step-start state stays FP32 and alternates between two buffers
    // with the step's parity (Wm = this step's, Wout in stage 3 = the
    // next's); each stage's delta from it (Sout; the next stage's stencil
    // input is Wm + Sin) and the RK accumulator's delta (T16) are FP16 values
    // times a per-field power-of-two scale, in the FP16 layout gh.  The
    // scales come from mx[parity][9], the bounds of |Wm| at the step start
    // (float bits: stage 3 and the source kernels raise them with atomicMax),
    // coupled between velocity and stress through the medium's impedance
    // bounds zs_min, zp_max.
    DevGrid gh;
    const __half *Sin;
    __half *Sout, *T16;
    unsigned *mx;
    const int *it_dev;
    float zs_min, zp_max;
    int ntiles_x, ntiles_y, nchunk;  // work items: tiles x tiles x z-chunks
    int irk;
    int FB1, FB2, FB3;
    int nPML;
    int pml_on;          // absorbing faces, one bit each: x1 y1 z1 x2 y2 (bits 0..4)
    int fs_on;           // the traction free surface in the top three layers
    int kchunk;
    float rDH, DT;
    HaloOut ho[6];       // faces x-low x-high y-low y-high z-low z-high (halo-out launches only)
};
// TMA descriptors (CUtensorMap, 128 bytes each) used by one stage launch:
// the stencil input with its halo box, and 32x8 point boxes of the metric,
// the step-start state and the RK accumulator for L2 prefetch.
struct CgStageMaps {
    alignas(64) unsigned char winp[128];   // the stencil input, point box (split pipeline)
    alignas(64) unsigned char win[128];
    alignas(64) unsigned char cjm[128];
    alignas(64) unsigned char wm[128];
    alignas(64) unsigned char t[128];
};
// Everything one stage launch needs for one session: the four tensor maps
// (CUtensorMap, 128 bytes each, 64-byte aligned) and the arguments.
// work: the launch's work-counter pair, zero between launches.
struct alignas(64) CgStageDesc {
    unsigned char tmW[128], tmC[128], tmM[128], tmT[128];
    unsigned char tmS[128];   // mixed storage: the FP16 stencil-input delta, halo box
    unsigned char tmWc[128];  // split pipeline: the stencil input, interior column box
    CgStageArgs a;
};
// The stage kernel's host functions, declared once per tile height: the
// 32 x 4 build (inline namespace ty4: these names plainly) and the 32 x 8
// build (cgfdm::ty8, csrc/cgfdm_stage_ty8.cu).
//
// launch_cg_stage: one session's stage (ring pipeline), its descriptor passed
// as a kernel parameter.  launch_cg_stage_batch: session s owns work items
// item_start[s] .. item_start[s+1]-1, its descriptor is descs[s] in device
// memory; all advance with the same FB signs and stage number.
// launch_cg_stage_split: the split pipeline (the current plane's halo box,
// interior column boxes for the z window): one session's FP32 stage.
// launch_cg_stage_mix: mixed-precision storage (the MIX instantiation);
// launch_cg_stage_batch_mix: the same for a batch of such sessions.
// make_field_tmap16: FP16 counterpart of make_field_tmap (halo box), for
// arrays in the layout gh.  launch_impedance_bounds: smallest S and largest
// P impedance, sqrt(mu / b) and sqrt((lambda + 2 mu) / b), over the interior,
// into out[0], out[1] (float bits; the caller sets out[0] to +inf bits and
// out[1] to 0 first).  make_field_tmap: the 4-D tensor map (x, y, z, field)
// of an nf-field buffer, with a halo box (40 x (tile rows + 4) x 1 x nf) or a
// point box (32 x tile rows x 1 x nf); out must hold 128 bytes.
#define CG_STAGE_FUNCTIONS                                                                                         \
    cudaError_t launch_cg_stage(int FB1, int FB2, int FB3, const CgStageDesc &d, int *work, int grid_ctas,      \
                                cudaStream_t st, bool halo_out = false);                                         \
    cudaError_t launch_cg_stage_batch(int FB1, int FB2, int FB3, const CgStageDesc *descs, const int *item_start, \
                                      int nsess, int *work, int grid_ctas, cudaStream_t st);                     \
    size_t cg_stage_smem_bytes(bool mix = false);                                                               \
    size_t cg_stage2_smem_bytes();                                                                              \
    cudaError_t launch_cg_stage_split(int FB1, int FB2, int FB3, const CgStageDesc &d, int *work, int grid_ctas,\
                                      cudaStream_t st);                                                          \
    cudaError_t launch_cg_stage_mix(int FB1, int FB2, int FB3, const CgStageDesc &d, int *work, int grid_ctas,  \
                                    cudaStream_t st);                                                            \
    cudaError_t launch_cg_stage_batch_mix(int FB1, int FB2, int FB3, const CgStageDesc *descs,                  \
                                          const int *item_start, int nsess, int *work, int grid_ctas,           \
                                          cudaStream_t st);                                                      \
    int cg_stage_mix_ctas_per_sm();                                                                             \
    cudaError_t make_field_tmap16(void *out, const __half *base, const DevGrid &gh, int nf);                    \
    cudaError_t launch_impedance_bounds(const float *cjm, DevGrid g, unsigned *out, cudaStream_t st);           \
    cudaError_t make_field_tmap(void *out, const float *base, const DevGrid &g, int nf, bool halo_box);         \
    int cg_stage_ctas_per_sm();                                                                                 \
    int cg_stage_tile_y();
inline namespace ty4 {
CG_STAGE_FUNCTIONS
}
namespace ty8 {
CG_STAGE_FUNCTIONS
}

// ------------------------------------------------ SCFDM (ME-AWENO) stage
// One directional pass of a TVD stage: x stores the RHS in H, y adds to it,
// z adds its part and writes the TVD-RK3 update to Wout.
struct ScDirArgs {
    DevGrid g;
    const float *W;      // stencil input of this stage
    const float *Wm;     // values at the start of the step (stages 1, 2)
    float *Wout;         // stage output (z pass)
    float *H;            // RHS accumulator, 9 fields
    const float *cjm;    // 19 fields
    const float *sjac;   // DT * rDH / J per point
    const float *decay;  // sponge factors G[0..ndecay] (z pass of the last stage), or null
    int ndecay;
    int irk;
    int copy_halo;       // z pass of stages 0 and 1: carry the halo above the surface to Wout
    float alpha;         // Lax-Friedrichs speed (largest Vp)
};
struct ScTiling {
    int npos[3], nl[3], ntiles[3];
};
ScTiling sc_tiling(const DevGrid &g);

cudaError_t sc_dir_prepare();
cudaError_t launch_sc_dir(int dir, ScDirArgs a, const ScTiling &t, cudaStream_t st);
// Characteristic free surface, halo extrapolation, sponge of the top layers,
// peak ground velocity and (dis given) the surface-layer displacement, after
// the third stage of a step.
cudaError_t launch_sc_surface(float *W, const float *cjm, DevGrid g, const float *decayG, int ndecay, float *pgv,
                              float *dis, float DT, cudaStream_t st);
cudaError_t launch_sc_sjac(const float *cjm, DevGrid g, float DT, float rDH, float *sjac, cudaStream_t st);

// ------------------------------------------------------ CGFDM adjoint
// One RK4 stage of the transposed step (csrc/adjoint.cu).  Going back
// through stage s = 3, 2, 1, 0 of step n, with lambda' the adjoint of
// W_{n+1}, mu_s the adjoint of the stage's RHS h_s and nu_s = L_s^T mu_s:
//   mu_3 = b4 lambda'; mu_2 = b3 lambda' + nu_3; mu_1 = b2 lambda' + a3 nu_2;
//   mu_0 = b1 lambda' + a2 nu_1;  lambda_n = lambda' + nu_3 + nu_2 + nu_1 + nu_0,
// for the wavefield and, point-wise, for the PML auxiliaries.
struct AdjStageArgs {
    DevGrid g;
    HBox hbox;           // layout of h
    const float *cjm, *rdz;
    const float *drdz;   // d rdz / d mu (18 fields) then d rdz / d lambda (18), [36][plane], or null
    const float *pml_alpha_x, *pml_beta_x, *pml_d_x;
    const float *pml_alpha_y, *pml_beta_y, *pml_d_y;
    const float *pml_alpha_z, *pml_beta_z, *pml_d_z;
    const float *Lp;     // lambda' (9 fields)
    float *M;            // mu_s in; mu_{s-1} out
    float *Lam;          // running sum; lambda_n after stage 0
    float *Phi;          // 27 fields: per direction, the adjoint of its one-sided differences
    float *SF;           // surface layers L = 0..2 (k = _nz-1-L): 12 channels each, [3][12][plane]
    PmlFace face[5];     // adjoint auxiliaries per face: A = lambda', B = mu, T = running sum
    const float *h;      // stored RHS h_s of the forward stage (9 fields, HBox layout), or null: no gradient
    const float *vd;     // stored surface xi/eta velocity derivatives (6 x plane) of the stage
    float *grad;         // 3 fields: d J / d (mu, lambda, buoyancy), accumulated
    float *M2;           // fused kernel: receives mu_{s-1} (M is read at neighbours meanwhile)
    float *faceB2[5];    // fused kernel: the faces' mu_{s-1}
    int kchunk, nchunk;  // fused kernel: z planes per block, blocks along z
    int irk;
    int FB1, FB2, FB3;
    int nPML, pml_on, fs_on;
    float rDH, DT;
};
cudaError_t launch_adj_stage(const AdjStageArgs &a, cudaStream_t st);        // two passes through Phi in HBM
cudaError_t launch_adj_stage_fused(const AdjStageArgs &a, cudaStream_t st);  // one pass, Phi in shared memory
// Adds the seismogram residual of sample n, res[station][n][3], to the
// velocity of lambda (the misfit is 1/2 sum (v - d)^2).
cudaError_t launch_adj_residual(float *Lp, DevGrid g, const int *st_idx, int nst, int NT, int n, const float *res,
                                cudaStream_t st);
// d rdz / d mu and d rdz / d lambda at the surface, in FP64 dual numbers.
cudaError_t launch_surface_derivs(const float *cjm, DevGrid g, float *drdz, cudaStream_t st);
// (mu, lambda, buoyancy) gradients -> (Vp, Vs, rho) on the interior,
// out [3][nz][ny][nx]; medium [_nz_][_ny_][_nx_][3] as (Vs, Vp, rho).
cudaError_t launch_grad_chain(const float *grad, const float *medium, DevGrid g, float *out, cudaStream_t st);

// --------------------------------------------------- sources / stations
struct FaultDev {
    const float *rate;        // [nt][npts][6], scaled
    const long long *cell;    // layout index per cell
    long long npts;
    int nt;
    float dt;
};
struct PointDev {
    int kind;                 // 1 Ricker, 2 double couple
    int X, Y, Z;
    const float *amp;         // [7][7][7]
    const float *stf;         // [NT]
    float mom[6];
    float m0;
    int inside;
};
// Adds the source terms of step *it_dev to W (stage-0 time), as the
// reference does before the RK stages (src/propagate.cpp:198-210).
// Mixed storage (Walt given): the step-start state of step n is W for even
// n, Walt for odd n, and the injected values raise the bounds mx[n & 1].
cudaError_t launch_sources(float *W, const float *cjm, DevGrid g, const FaultDev &f, const PointDev &p,
                           const int *it_dev, float DT, float DH, int scheme, cudaStream_t st,
                           float *Walt = nullptr, unsigned *mx = nullptr);
cudaError_t launch_point(float *W, float *Wb, float *Wc, const float *cjm, DevGrid g, const PointDev &p,
                         const int *it_dev, float DT, float DH, int scheme, cudaStream_t st, float *Walt = nullptr,
                         unsigned *mx = nullptr);
// Records 9 components per station at step *it_dev, then advances *it_dev.
// Mixed storage (Walt given): the state after step n is in W or Walt by the
// parity of n + 1.
cudaError_t launch_stations(const float *W, const float *cjm, DevGrid g, const int *st_idx, int nst, int NT,
                            float *out, int *it_dev, int scheme, cudaStream_t st, const float *Walt = nullptr);
// Peak ground acceleration [ny][nx][2] (PGAh, PGA) after a step whose index
// *it_dev is a multiple of 10 (the reference's SOLVE_PGA).
cudaError_t launch_pga(const float *W, const float *cjm, DevGrid g, const int *it_dev, float DT, int scheme,
                       float *pga, cudaStream_t st);
// One slice of field `comp` of W for the snapshot files: axis 0/1/2 = the
// plane i/j/k = idx, in the reference's [nz][ny] / [nz][nx] / [ny][nx]
// order; SCFDM (scheme 1, cjm given) converts momentum to velocity.
cudaError_t launch_pack_slice(const float *W, const float *cjm, DevGrid g, int axis, int idx, int comp, int scheme,
                              float *out, cudaStream_t st);
// Gathers W (9 fields) into the reference AoS layout [_nz_][_ny_][_nx_][9].
cudaError_t launch_to_aos(const float *W, int nfield, DevGrid g, float *out, cudaStream_t st);
cudaError_t launch_from_aos(const float *in, int nfield, DevGrid g, float *W, cudaStream_t st);

}  // namespace cgfdm
