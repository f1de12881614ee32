/*
 * C ABI of the B200 velocity-stress time-stepping library (libcgfdm.so).
 *
 * The reference is a C++/CUDA program with no library interface: its hot
 * path is the time loop propagate() (src/propagate.cpp:77-350 of
 * CGFDM3D-EQR-SC) driven from run() (src/run.cpp:28-138), reading a run
 * directory (params.json, station.json, layered-medium and finite-fault
 * files) and writing station and PGV files.  This header is the drop-in
 * boundary for that path: a session replaces run() for one rank on one GPU,
 * with the same inputs and output layouts.
 *
 * Conventions: every function returns 0 on success or a status code
 * (CGFDM_E_*); cgfdm_last_error() describes the last failure.  Pointers are
 * host pointers unless named d_*.  A session is bound to one CUDA device and
 * one stream; it is not thread-safe.  Wavefield arrays cross the boundary in
 * the reference's layout, array-of-structures [_nz_][_ny_][_nx_][9] with the
 * 3-cell halo (src/axis.h:237), components Vx Vy Vz Txx Tyy Tzz Txy Txz Tyz
 * for CGFDM and the conserved variables for SCFDM.
 */
#ifndef CGFDM_H
#define CGFDM_H

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes.  Where the reference aborts, the code is its MPI_Abort code. */
#define CGFDM_OK 0
#define CGFDM_E_NO_PARAMS 100   /* params.json missing (src/getParams.cpp:100) */
#define CGFDM_E_CFL 110         /* DT above the stability bound (src/calc_CFL.cpp:341-345) */
#define CGFDM_E_PML_SIZE 130    /* nPML >= nx/ny/nz (src/pml_deriv.cpp:55-85) */
#define CGFDM_E_OPTIONS 180     /* conflicting or unsupported options (src/modelChecking.cpp:17-61) */
#define CGFDM_E_JSON 1001       /* unparsable json (src/getParams.cpp:123) */
#define CGFDM_E_IO 1002         /* missing or short input file */
#define CGFDM_E_ALLOC 10001     /* allocation failure (src/wave_deriv.cpp:52) */
#define CGFDM_E_CUDA 20001      /* CUDA runtime error */
#define CGFDM_E_TIMEOUT 20002   /* a bounded device wait gave up */
#define CGFDM_E_ARG 20003       /* bad argument */
#define CGFDM_E_STATE 20004     /* call not valid in the session's state */
#define CGFDM_E_NONFINITE 20005 /* NaN or Inf in the wavefield ("checkFinite") */

typedef struct cgfdm_session cgfdm_session;

typedef struct cgfdm_info {
    int scheme;          /* 0 CGFDM (MacCormack + RK4), 1 SCFDM (ME-AWENO + TVD-RK3) */
    int nx, ny, nz;      /* interior points */
    int nxp, nyp, nzp;   /* padded with the 3-cell halo */
    int NT;              /* steps of the run: (int)(TMAX / DT) (src/propagate.cpp:88) */
    int steps_done;
    int n_stations;
    long long n_fault_cells;
    float DT, DH, dtmax; /* dtmax = 1.34 H_min / Vp_max (src/calc_CFL.cpp:325) */
    float H_min, Vp_max;
    double device_bytes; /* device memory held by the session */
    double h2d_bytes;    /* bytes copied host -> device during setup */
    long long kernel_launches; /* kernels of this library launched so far */
    double algo_bytes_per_step; /* bytes a step must move at minimum (see cgfdm_profile_stages) */
    int stage_kernels_per_step; /* fused stage launches per step (4 for RK4, 3 for TVD-RK3) */
    int pgv_fields;      /* floats per point of the PGV record: 2, or 4 with SOLVE_PGA */
} cgfdm_info;

/* Builds the model of a run directory on GPU `device`: reads params.json
 * and the inputs it names, constructs coordinates, medium, metrics (on the
 * GPU), PML profiles, sources and stations, and checks the CFL condition.
 * Replaces src/run.cpp:28-116 up to the call of propagate().
 * `options_json` (may be NULL) overrides run-time switches with the
 * reference's flag names: {"scheme": "CGFDM"|"SCFDM", "PML": 0|1,
 * "EXP_DECAY": 0|1, "SOLVE_DISPLACEMENT": 0|1, "SOLVE_PGA": 0|1, "metricPrecision":
 * "fp32"|"fp64", "OUT": "..."} and this library's own keys ("checkFinite": K,
 * "adjointKernel", "adjointStoreSegments"). */
int cgfdm_create(const char *run_dir, const char *options_json, int device, cgfdm_session **out);

/* ---- Domain decomposition (the reference's MPI layout, src/init_grid.cpp) ----
 * A grid too large for one GPU runs as parts[0] x parts[1] x parts[2]
 * sub-domains, one session per part (one per GPU and process, or several on
 * one GPU).  cgfdm_create_part builds part `coord` (0 <= coord[a] <
 * parts[a]) of the run directory's model: interior sizes split as evenly as
 * possible, the model's padded arrays sliced with 3-cell halos, PML only on
 * the faces at the global boundary, the free surface only in the top parts,
 * the finite-fault cells and stations of the part's interior (a point
 * source's 7x7x7 cube must lie inside one part).  CGFDM only.
 *
 * Stepping: cgfdm_part_advance runs the next of the five phases of a step
 * (0: the source; 1..4: RK stage 0..3, the stations after the last) and
 * returns the phase it ran.  After phases 0..3 every part refreshes its
 * halos: per axis x, y, z in turn, cgfdm_halo_pack(face) the faces it
 * shares with a neighbour into a device buffer of cgfdm_halo_count floats,
 * send each to the neighbour on that side, and cgfdm_halo_unpack(face) what
 * arrives from the neighbour on side `face`.  Faces: 0 x-low, 1 x-high,
 * 2 y-low, 3 y-high, 4 z-low, 5 z-high; which: 0 the wavefield the phase
 * wrote, 1 the 13 metric and medium fields (exchanged once after create).
 * Pack and unpack finish before they return.  cgfdm_run refuses parts. */
int cgfdm_create_part(const char *run_dir, const char *options_json, const int *parts, const int *coord, int device,
                      cgfdm_session **out);
int cgfdm_part_info(const cgfdm_session *s, int *lo, int *n, int *top);
int cgfdm_part_station_ids(const cgfdm_session *s, int *ids, int count);
int cgfdm_part_advance(cgfdm_session *s, int *phase);
/* cgfdm_part_advance in two halves: cgfdm_part_launch enqueues the next
 * phase and returns; cgfdm_part_finish waits for it and checks the device
 * error word.  Parts sharing a GPU launch their phase together and then
 * finish, so their kernels run concurrently. */
int cgfdm_part_launch(cgfdm_session *s, int *phase);
int cgfdm_part_finish(cgfdm_session *s);
/* Folds the exchanges after phases 1..4 into the stage kernel: part s's
 * stages store the interior layers next to `face` straight into the halo of
 * neighbour part nbr (a session in the same process, on the same device or
 * one whose memory s's device can address).  All parts must finish a phase
 * before any starts the next; the exchange after phase 0 stays explicit. */
int cgfdm_part_link(cgfdm_session *s, int face, const cgfdm_session *nbr);
/* The same between processes (one part per GPU): cgfdm_part_handle writes
 * CGFDM_PART_HANDLE_BYTES describing the part's stage buffers (CUDA IPC
 * handles and layout) for its neighbours; cgfdm_part_link_handle(face)
 * opens a neighbour's handle (peer access over NVLink) and links it.  A
 * barrier between phases then replaces the halo exchange of phases 1..4. */
#define CGFDM_PART_HANDLE_BYTES 512
int cgfdm_part_handle(cgfdm_session *s, void *out, long long bytes);
int cgfdm_part_link_handle(cgfdm_session *s, int face, const void *handle, long long bytes);
long long cgfdm_halo_count(const cgfdm_session *s, int face, int which);
int cgfdm_halo_pack(cgfdm_session *s, int face, int which, float *d_buf);
int cgfdm_halo_unpack(cgfdm_session *s, int face, int which, const float *d_buf);

/* Host-only: builds the model of a run directory as cgfdm_create does --
 * parameters, grid, coordinates and the medium from the switches that
 * select it (homogeneous, CRUST1.0, Shen, layered, mediumFile;
 * src/medium.cpp:251-295) -- without touching a GPU, and copies the medium
 * [nzp][nyp][nxp][3] (Vs, Vp, rho) into `out` (NULL: only the dimensions
 * nzp, nyp, nxp go to dims).  Errors as cgfdm_create, message from
 * cgfdm_last_error(NULL). */
int cgfdm_model_medium(const char *run_dir, const char *options_json, float *out, long long count, int *dims);

/* Host-only, as cgfdm_model_medium: the surface height of every column,
 * [nyp][nxp] (gauss_hill, terrainFile or, with useTerrain and SRTM90, the
 * SRTM tiles of src/terrain.cpp:206-770), into `terrain`, and the grid's
 * coordinates [nzp][nyp][nxp][3] (x, y, z) into `coord` (either may be
 * NULL; counts in floats); dims as cgfdm_model_medium. */
int cgfdm_model_coord(const char *run_dir, const char *options_json, float *terrain, long long terrain_count,
                      float *coord, long long coord_count, int *dims);

/* The session's model arrays in the reference's device layouts, for a
 * caller that drives the per-function entry points of cgfdm_shims.h:
 * "rDZ_DX", "rDZ_DY" (float [_ny_][_nx_][9]); "pml_alpha_x", "pml_beta_x",
 * "pml_d_x" and the same for y, z (float [_nx_], [_ny_], [_nz_]);
 * "srcIndex" (int64 [npts], padded-grid point index of each finite-fault
 * cell) and "momentRate" (float [nt][npts][6], before calculateMomentRate);
 * "stationXYZ" (int32 [n][3], padded indices).  Host copies: `out` NULL
 * writes the size in bytes to *bytes; otherwise *bytes is the capacity of
 * `out` on entry and the size on return. */
int cgfdm_get_array(cgfdm_session *s, const char *name, void *out, long long *bytes);

/* Health check: the number of NaN / Inf values in the state at the last step
 * boundary over the interior points (`count`), and the first of them as
 * ((k * ny + j) * nx + i) * 9 + field (`first`, -1 when none).  With the
 * option "checkFinite": K, cgfdm_run scans after every K steps and returns
 * CGFDM_E_NONFINITE, naming the step and point, when one is found. */
int cgfdm_check_finite(cgfdm_session *s, long long *count, long long *first);

/* Advances up to `nsteps` time steps (clamped to NT).  One step is the body
 * of the time loop, src/propagate.cpp:186-321: source term into W, the RK
 * stages with derivative, free surface and PML, station recording and PGV. */
int cgfdm_run(cgfdm_session *s, int nsteps);

/* As cgfdm_run, and returns the device time of those steps in milliseconds,
 * measured with CUDA events on the session's stream. */
int cgfdm_run_timed(cgfdm_session *s, int nsteps, float *ms);

int cgfdm_info_get(const cgfdm_session *s, cgfdm_info *out);

/* Advances `nsteps` steps launching every kernel directly (no graph), with
 * CUDA events around each fused stage kernel, and returns the mean device
 * time of one stage launch in milliseconds.  Divide algo_bytes_per_step by
 * stage_kernels_per_step for the algorithmic bytes of one launch: per
 * interior point and step, the stencil input, metric and medium (12 fields),
 * RK state and accumulator of every stage (192 float fields in all for
 * RK4), plus 144 auxiliary fields per point of each absorbing face. */
int cgfdm_profile_stages(cgfdm_session *s, int nsteps, float *mean_stage_ms);

/* Station traces, [n_stations][NT][9] as the reference stores them
 * (src/station.cpp:334); `count` is the capacity of `out` in floats. */
int cgfdm_get_stations(const cgfdm_session *s, float *out, long long count);

/* Current wavefield, [nzp][nyp][nxp][9]; `count` is the capacity in floats. */
int cgfdm_get_wavefield(const cgfdm_session *s, float *out, long long count);

/* Packed metric/medium array CJM (src/CJM.cpp:106-147), [nzp][nyp][nxp][nfield]
 * with nfield 13 (CGFDM) or 19 (SCFDM); with out == NULL only *nfield is set. */
int cgfdm_get_cjm(const cgfdm_session *s, float *out, long long count, int *nfield);

/* Peak ground velocity at the surface, [ny][nx][2] (PGVh, PGV) (src/PGV.cpp:61-175);
 * with SOLVE_PGA [ny][nx][4] (PGVh, PGV, PGAh, PGA), the peak acceleration as the
 * reference's SOLVE_PGA build evaluates it (|V| / (10 DT) at every tenth step:
 * its previous-velocity copy never reaches the surface points). */
int cgfdm_get_pgv(const cgfdm_session *s, float *out, long long count);

/* Writes OUT/station_mpi_0_0_0.bin and OUT/PGV_Z_mpi_0_0_0.bin in the
 * reference's formats (src/station.cpp:422-443, src/PGV.cpp:177-185). */
int cgfdm_write_outputs(const cgfdm_session *s);

/* Checkpoint of the time-stepping state at the current step boundary: the
 * step counter, the wavefield, the PML auxiliaries, and the running outputs
 * (PGV, displacement, station traces so far), in a host buffer of
 * cgfdm_checkpoint_size bytes.  cgfdm_restore loads one into a session
 * created from the same run directory and options; stepping on from there
 * gives bit-identical results to an uninterrupted run.  The reference keeps
 * no restart files; this replaces re-running it from step 0 (it has no
 * counterpart in src/). */
int cgfdm_checkpoint_size(const cgfdm_session *s, long long *bytes);
int cgfdm_checkpoint(cgfdm_session *s, void *out, long long bytes);
int cgfdm_restore(cgfdm_session *s, const void *in, long long bytes);

/* Overwrites the wavefield, [nzp][nyp][nxp][9] (halo included, held equal
 * in every stage buffer as the point sources keep it); the PML auxiliaries
 * and the step counter are kept.  No counterpart in src/ (an initial
 * condition; the reference always starts from rest). */
int cgfdm_set_wavefield(cgfdm_session *s, const float *in, long long count);

/* Replaces the medium, [nzp][nyp][nxp][3] as (Vs, Vp, rho) in m/s and
 * kg/m^3 -- the layout of a mediumFile -- and rebuilds the packed medium,
 * the free-surface matrices and the finite-fault scaling from it as
 * cgfdm_create does (src/CJM.cpp:52-77, src/contravariant.cpp:365-461); the
 * session returns to step 0 at rest.  CFL is re-checked at the session's DT
 * (CGFDM_E_CFL).  CGFDM only. */
int cgfdm_set_medium(cgfdm_session *s, const float *medium, long long count);

/* Discrete adjoint of the CGFDM time loop (no counterpart in src/).
 *
 * cgfdm_gradient: gradient of the seismogram misfit
 *     J = 1/2 sum over stations, samples n < NT and components x, y, z of
 *         (v - d)^2,
 * v the velocity the run records at the stations (station file
 * components 0..2), d = observed [n_stations][NT][3], with respect to Vp,
 * Vs and rho at every interior grid point: grad [3][nz][ny][nx] (Vp, Vs,
 * rho; zero inside the PML layers), *misfit = J.  The session must stand at
 * step 0 (new, or after cgfdm_set_medium) and have point sources only (it
 * writes no snapshot files; PGV and displacement follow the forward run); it
 * runs the whole forward once keeping the state every `checkpoint_every`
 * steps in device memory, then per segment, last first, re-runs it storing
 * each RK stage's right-hand side and steps the transposed operator back
 * through it.  Device memory: (NT / checkpoint_every + 1) states plus
 * 36 * checkpoint_every wavefield-sized fields per stored segment;
 * CGFDM_E_ALLOC names the amount when one segment does not fit.  The last
 * segments are stored during the first forward run, as many as the free
 * device memory holds (the options key "adjointStoreSegments" caps that
 * number), and need no second run.  This scratch stays allocated on the
 * device after the call, for the next cgfdm_gradient of any session on that
 * device, until the device's last session is destroyed; gradient calls on
 * one device run one at a time.  The session ends at step NT with the forward
 * run's state and station traces.
 *
 * cgfdm_adjoint_apply: applies the transpose of the last `nsteps` steps the
 * session ran (without source and station terms) to `state`,
 * [nzp][nyp][nxp][9] in and out; the PML auxiliaries' adjoints start from
 * zero.  Halo entries are ignored on input and zero on output.  With x and
 * y interior-only states, <A x, y> = <x, A^T y> for A the forward map from
 * cgfdm_set_wavefield to cgfdm_get_wavefield (the dot-product test). */
int cgfdm_gradient(cgfdm_session *s, const float *observed, long long obs_count, int checkpoint_every,
                   double *misfit, float *grad, long long grad_count);
int cgfdm_adjoint_apply(cgfdm_session *s, int nsteps, float *state, long long count);
/* Device time of the phases of the last cgfdm_gradient in ms: ms3[0] the
 * forward run with checkpoints, ms3[1] the segment re-runs that store the
 * stage right-hand sides, ms3[2] the adjoint steps. */
int cgfdm_gradient_profile(const cgfdm_session *s, float *ms3);

/* Autotuner of the CGFDM stage launch (no counterpart in src/).  The stage
 * kernel's persistent CTAs take work items of 32 x `rows` columns by
 * `kchunk` planes; cgfdm_autotune times candidate tile heights (4 and 8
 * rows, where the session's pipeline has both), pencil lengths and CTA
 * counts on `trial_steps` steps each (from a device copy of the state, which
 * is put back: tuning does not advance the run), keeps the fastest and
 * returns its pencil, CTA count and device time per step.  Results are
 * bit-identical for every tiling.  cgfdm_set_tiling / cgfdm_get_tiling set
 * and read the pencil and CTAs directly (ctas is clamped to the resident
 * maximum and the work items); cgfdm_set_stage_tile / cgfdm_get_stage_tile
 * the tile height (8 rows only with FP32 storage on a whole grid, not a
 * part: CGFDM_E_OPTIONS otherwise; the default is 8 on the split pipeline
 * and 4 elsewhere).  cgfdm_batch_autotune does the same for a batch's
 * shared launch, trying both tile heights and one pencil length for all its
 * sessions against their own default ones (*kchunk = 0 when those are
 * kept); cgfdm_batch_set_stage_tile / cgfdm_batch_get_stage_tile set and
 * read the batch's tile height (4 by default).  A candidate replaces the
 * current decomposition only when faster by more than 1 %. */
int cgfdm_autotune(cgfdm_session *s, int trial_steps, int *kchunk, int *ctas, float *ms_per_step);
int cgfdm_set_tiling(cgfdm_session *s, int kchunk, int ctas);
int cgfdm_get_tiling(const cgfdm_session *s, int *kchunk, int *ctas);
int cgfdm_set_stage_tile(cgfdm_session *s, int rows);
int cgfdm_get_stage_tile(const cgfdm_session *s, int *rows);

/* Batches: several CGFDM sessions -- independent shots or media of uneven
 * grid sizes -- advanced together, every RK stage of all of them in one
 * persistent launch of the fused stage kernel, eight steps per replay of a
 * captured CUDA graph.  The sessions must be CGFDM, on one device, at the
 * same step, without snapshots, all with FP32 or all with FP16 storage
 * ("storage": "fp16"; such a batch takes 32 x 4 tiles and no autotuning,
 * CGFDM_E_OPTIONS otherwise); they stay owned by the caller and must
 * outlive the batch, and while batched they are stepped only through it
 * (cgfdm_batch_run advances each by min(nsteps, steps left to the shortest
 * NT)).  Results per session are those of running it alone, bit for bit.
 * The reference runs one model per program; this has no counterpart in src/. */
typedef struct cgfdm_batch cgfdm_batch;
int cgfdm_batch_create(cgfdm_session *const *sessions, int n, cgfdm_batch **out);
int cgfdm_batch_run(cgfdm_batch *b, int nsteps);
/* As cgfdm_batch_run, returning the device time of the steps in ms. */
int cgfdm_batch_run_timed(cgfdm_batch *b, int nsteps, float *ms);
int cgfdm_batch_destroy(cgfdm_batch *b);
int cgfdm_batch_autotune(cgfdm_batch *b, int trial_steps, int *kchunk, int *ctas, float *ms_per_step);
int cgfdm_batch_set_stage_tile(cgfdm_batch *b, int rows);
int cgfdm_batch_get_stage_tile(const cgfdm_batch *b, int *rows);
/* Last failure of b, or of the last failed cgfdm_batch_create in this
 * thread when b is NULL. */
const char *cgfdm_batch_last_error(const cgfdm_batch *b);

int cgfdm_destroy(cgfdm_session *s);

/* Description of the last failure on `s` (or of the last failed
 * cgfdm_create in this thread when s is NULL). */
const char *cgfdm_last_error(const cgfdm_session *s);

/* The session's time loop from step 0 in reference form with the state and
 * all arithmetic in FP64 (bits = 64) or FP32 (bits = 32), on the session's
 * model (metric, medium, free-surface matrices, PML profiles, sources,
 * stations: FP32, promoted in FP64 as the reference's FP32 model is
 * promoted).  No counterpart in the reference, which computes in float
 * throughout (src/propagate.cpp:186-321 with src/wave_deriv.cpp:187-283's
 * float locals): bits = 64 is the FP64 run every FP32 or reduced-storage
 * result states its error against; bits = 32 reproduces cgfdm_run (bit for
 * bit in the "exact" build).  One thread per point, buffers of its own for
 * the call (the session's state, step counter and outputs are untouched).
 * Outputs (each optional, NULL to skip; n_* their lengths in doubles):
 * stations [n_stations][nsteps][9] as cgfdm_get_stations records them, pgv
 * [ny][nx][2], wavefield [_nz_][_ny_][_nx_][9] after the last step. */
int cgfdm_run_precise(cgfdm_session *s, int nsteps, int bits, double *stations, long long n_stations,
                      double *pgv, long long n_pgv, double *wavefield, long long n_wavefield);

/* Host wall milliseconds of the session's set-up: ms[0] the model from the
 * run directory (file reads and host arithmetic, src/run.cpp:28-116's part
 * before the time loop), ms[1] the device set-up (allocation, uploads,
 * metric and CFL kernels), ms[2] all of cgfdm_create, ms[3] the capture of
 * the eight-step CUDA graph (made by the first cgfdm_run of 8 or more steps),
 * ms[4..8] the parts of ms[0]: coordinates and terrain, medium, value ranges
 * and PML profiles, sources, stations; ms[9..11] the parts of ms[1]:
 * allocation, uploads and the CFL check, the rest enqueued, its completion;
 * ms[12], ms[13] the allocation and the upload within ms[9]. */
int cgfdm_create_profile(const cgfdm_session *s, double ms[14]);

/* Test hook of the stage kernel's bounded waits.  No counterpart in the
 * reference, whose CHECK macro prints a CUDA error and carries on
 * (src/macro.h:94-103): here every wait of the CGFDM stage kernel for its
 * plane copies is bounded, and a wait that gives up sets a device error word
 * that the next cgfdm_run reports as CGFDM_E_TIMEOUT.  After this call the
 * next stage launch's work item `item` leaves its plane copy number `fill`
 * (counted from the item's first plane) unissued, once, and every bounded
 * wait gives up after `wait_cycles` clock cycles (0: the default, 2^31).  The
 * kernel then drains the copies it did issue and returns; the session's
 * state is not usable afterwards, the device is.  For tests only. */
int cgfdm_test_stall(cgfdm_session *s, int item, int fill, long long wait_cycles);

/* Allocation-free grid-spacing reduction.  No counterpart in the reference:
 * it offers the smallest and largest point-to-plane distance of the CFL
 * check (the quantity cgfdm_create computes as H_min, after
 * src/calc_CFL.cpp:94-163) to callers that cannot allocate device memory at
 * that point, for example an application whose other streams carry a live
 * simulation (cudaMalloc/cudaFree can synchronize the whole device) or an
 * embedder whose own pool allocator owns the device memory.  It calls no
 * cudaMalloc, cudaFree or allocating library routine.
 *
 * d_coord: device array [nz+6][ny+6][nx+6][3] of float x, y, z (the
 * reference's coordinate layout, halo included).  d_out: device array of two
 * doubles, receiving H_min and H_max.  stream: a cudaStream_t, or NULL for
 * the default stream; the call only enqueues work on it.
 *
 * Scratch lives in a static device array of CGFDM_NOALLOC_MAX_BLOCKS (min,
 * max) pairs, 1 MiB, one pair per block of 32 x 8 x 16 points; grids that
 * need more blocks, or more than 65535 blocks along y or z, are rejected
 * with CGFDM_E_ARG and a message from cgfdm_noalloc_last_error().  The array
 * is shared by every call on a device and keeps the last call's contents, so
 * calls that overlap on the GPU race.  The first call on each device looks
 * up the array's device address with that device current; a later call
 * looks it up again if the device's context has changed (after a
 * cudaDeviceReset). */
#define CGFDM_NOALLOC_MAX_BLOCKS 65536
int cgfdm_hrange_noalloc(const float *d_coord, int nx, int ny, int nz, double *d_out, void *stream);
const char *cgfdm_noalloc_last_error(void);

/* Library build identification: "fast" or "exact" (built with --fmad=false,
 * every float operation rounded separately as on the reference's CPU path). */
const char *cgfdm_build_flavor(void);

#ifdef __cplusplus
}
#endif

#endif
