// A simulation session: one run directory on one GPU.
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <thread>
#include <vector>

#include "device.cuh"
#include "kernels.cuh"
#include "model.hpp"

namespace cgfdm {

// FB signs of the first RK stage of a step (src/propagate.cpp:158-168);
// each later stage flips all three.
void fb_signs(int step, int fb[3]);
// gradient scratch kept per device while sessions live there (csrc/gradient.cu)
void arena_session_add(int device);
void arena_session_remove(int device);

struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
};

class Session {
public:
    ~Session();
    int create(const std::string &run_dir, const std::string &options, int device);
    int run(int nsteps);
    int run_span(int n);                             // n steps with their snapshots
    int run_checked(int n);                          // with the "checkFinite" scans (csrc/health.cu)
    int check_finite(long long *count, long long *first);  // non-finite values in the state
    // a part of a decomposed grid (csrc/partition.cpp, csrc/halo.cu): the
    // step in five phases with a halo exchange after each of the first four
    int create_part(const std::string &run_dir, const std::string &options, const int parts[3], const int coord[3],
                    int device);
    int part_advance(int *phase_done);    // part_launch + part_finish
    int part_launch(int *phase_done);
    int part_finish();
    long long halo_count(int face, int which) const;      // floats; which 0 wavefield, 1 metric (13 fields)
    int halo_copy(int face, int which, float *dev, bool pack);
    // the stage kernel stores the layers next to `face` into the neighbour
    // part's halo directly (same device, or peer memory): the halo exchange
    // of phases 1..4 folded into the stages
    int link_halo(int face, const Session &nbr);
    int link_halo_to(int face, float *const nbr_w[3], const DevGrid &nbr_g);
    // the same across processes: CUDA IPC handles of the stage buffers
    int part_handle(void *out, long long bytes);
    int link_halo_handle(int face, const void *handle, long long bytes);
    int run_timed(int nsteps, float *ms, float *stage_ms);
    int profile_stages(int nsteps, float *mean_stage_ms);
    double algo_bytes_per_step() const;
    int get_wavefield(float *host_aos) const;       // [_nz_][_ny_][_nx_][9]
    int get_cjm(float *host_aos, int *nfield) const;  // [_nz_][_ny_][_nx_][nfield]
    int get_stations(float *host) const;            // [nst][NT][9]
    int get_pgv(float *host) const;                 // [ny][nx][pgv_fields()]
    // model arrays in the reference's layouts, by name (csrc/shims.cu);
    // out NULL: the size in *bytes
    int get_array(const char *name, void *out, long long *bytes);
    int pgv_fields() const { return pga_ ? 4 : 2; } // PGVh, PGV (+ PGAh, PGA)
    int write_outputs() const;
    int sync() const;
    size_t checkpoint_bytes() const;
    int checkpoint(void *host, size_t bytes);       // state at the current step boundary
    int restore(const void *host, size_t bytes);    // from a checkpoint of an identical session
    int set_wavefield(const float *host_aos);       // [_nz_][_ny_][_nx_][9]; PML auxiliaries kept
    // CGFDM adjoint (csrc/gradient.cu)
    int adjoint_apply(int nsteps, float *host_aos);  // transpose of the last nsteps steps, in place
    int gradient(const float *obs, int ckpt_every, double *misfit, float *grad);
    int set_medium(const float *host_medium);       // [_nz_][_ny_][_nx_][3] (Vs, Vp, rho); back to step 0
    float grad_ms[3] = {0, 0, 0};                   // last gradient: forward, re-runs, adjoint steps (device ms)
    // work decomposition of the CGFDM stage kernel (csrc/autotune.cu): z
    // planes per work item and persistent CTAs; autotune times candidates
    // on trial steps and keeps the fastest, the state restored after each
    int set_tiling(int kchunk, int ctas);
    int autotune(int trial_steps, int *kchunk, int *ctas, float *ms_per_step);
    int kchunk() const { return kchunk_; }
    int ctas() const { return grid_ctas_; }
    // device copy of the state a trial step changes (wavefield, PML
    // auxiliaries, PGV, displacement); the step counter goes back to `it`
    size_t tune_bytes() const;
    int tune_save(char *dev);
    int tune_load(const char *dev);
    int time_steps(int nsteps, float *ms);          // direct launches from `it`, `it` unchanged
    // The time loop from step 0 in reference form with state and arithmetic
    // in FP64 (bits 64) or FP32 (bits 32) on the session's model
    // (csrc/precise.cu); buffers of its own, the session's state untouched.
    // stations [nst][nsteps][9], pgv [ny][nx][2], wavefield
    // [_nz_][_ny_][_nx_][9], each optional.
    int run_precise(int nsteps, int bits, double *stations, double *pgv, double *wavefield);

    Model m;
    DevGrid g;
    std::string err;
    std::string run_dir;
    int device = 0;
    int it = 0;  // steps completed
    bool is_part_ = false;  // a part of a decomposition: stepped by part_advance
    int phase_ = 0, cur_ = 0;
    bool halo_out_ = false;
    HaloOut ho_[4][6] = {};  // per stage and face
    std::vector<void *> ipc_open_;  // neighbours' buffers opened from IPC handles
    bool counted_ = false;  // registered with the device's gradient scratch
    int nst = 0;
    cudaStream_t stream = nullptr;
    long long graph_launches = 0, kernel_launches = 0;
    size_t device_bytes = 0;
    double h2d_bytes = 0;
    // host wall ms of cgfdm_create: model from the run directory (files,
    // host arithmetic), device set-up (allocation, uploads, set-up kernels),
    // whole create; and of capturing the eight-step CUDA graph
    double create_ms[3] = {0, 0, 0}, capture_ms = 0;
    double setup_ms[5] = {0, 0, 0, 0, 0};   // parts of create_ms[1] (csrc/session.cu setup_device)

private:
    int cuda_fail(cudaError_t e, const char *what);
    int setup_device();
    int launch_step(int step, bool timed_stages = false);  // one step, direct launches
    double stage_ms_sum_ = 0;
    long long stage_ms_count_ = 0;
    int launch_steps_graph(int n8);      // n8 full FB cycles via the captured graph
    void *alloc(size_t bytes);
    std::vector<void *> allocs_;
    // One device block holds the session's long-lived arrays (sub-allocated
    // on 256-byte boundaries): freeing some 30 separate arrays of an 8 GB
    // session took 50-200 ms, one block 6 ms.  Arrays that do not fit (or
    // that are made after set-up) get their own allocation.
    // the medium volume's upload, started while the host model build goes on
    // (large volumes only): its device buffer, the thread and its status
    float *pre_med_ = nullptr;
    std::thread med_thread_;
    cudaError_t med_err_ = cudaSuccess;
    char *arena_ = nullptr;
    size_t arena_size_ = 0, arena_used_ = 0;
    size_t arena_estimate() const;
    float *W_[4] = {nullptr, nullptr, nullptr, nullptr};  // A B C T
    float *cjm_ = nullptr, *rdz_ = nullptr;
    float *pml_[9] = {};
    PmlFace face_[5] = {};
    float *pgv_ = nullptr, *dis_ = nullptr, *pga_ = nullptr;
    int *st_idx_ = nullptr;
    float *st_out_ = nullptr;
    int *it_dev_ = nullptr;
    FaultDev fault_ = {};
    PointDev point_ = {};
    int kchunk_ = 8;
    cudaGraphExec_t graph8_ = nullptr;
    cudaGraph_t graph8_src_ = nullptr;
    cudaEvent_t ev_[4] = {};
    CgStageMaps maps_[3] = {};                       // TMA descriptors per stencil input A, B, C
    CgStageDesc desc_host_[4] = {};                  // stage descriptors, one per RK stage
    int build_stage_descs();
    int *work_dev_ = nullptr;                        // persistent-CTA work counters
    int ntx_ = 1, nty_ = 1, nchunk_ = 1, grid_ctas_ = 1;
    int *err_dev_ = nullptr;                         // device error word of the stage kernels
    float *h_ = nullptr, *sjac_ = nullptr, *decay_ = nullptr;  // SCFDM RHS, DT*rDH/J, sponge factors
    ScTiling sct_ = {};
    static constexpr int SC_DECAY_LAYERS = 20;       // src/exp_decay_absorb.cpp:109
    int check_device_error();
    template <class R>
    int run_precise_t(int nsteps, double *stations, double *pgv, double *wavefield);
    // mixed-precision storage ("storage": "fp16", CGFDM; see CgStageArgs):
    // step states W_[0] / Walt_ by step parity, stage deltas Sb_ / Sc_ and
    // the accumulator delta T16_ in the FP16 layout gh_, bounds mx_[2][9]
    bool mix_ = false;
    float *Walt_ = nullptr;
    __half *Sb_ = nullptr, *Sc_ = nullptr, *T16_ = nullptr;
    unsigned *mx_ = nullptr;
    DevGrid gh_{};
    float zs_min_ = 0, zp_max_ = 0;
    CgStageDesc desc_mix_[2][4] = {};
    int tile_ = 4;
    int build_maps();                                // tensor maps of the stencil inputs for tile_
    int stage_ctas_per_sm() const;
    int *stall_dev_ = nullptr;                       // test hook of the stage kernel's bounded waits
    int stall_item_ = -1, stall_fill_ = 0;
    long long wait_limit_ = 0;

public:
    // Column-tile height of the CGFDM stage kernel (4 or 8 rows of 32), the
    // tensor maps and work items built for it; set_tile re-encodes them
    // (8 only with FP32 storage on a whole grid)
    int tile() const { return tile_; }
    int set_tile(int rows);
    // one RK stage of this session's CGFDM step, with the pipeline and tile
    // height it uses
    int launch_stage(int FB1, int FB2, int FB3, const CgStageDesc &d);
    bool part_session_ = false;   // made by create_part: ring pipeline, 4-row tiles
    // The wavefield at the current step boundary (mixed storage alternates two buffers).
    float *state() const { return mix_ && (it & 1) ? Walt_ : W_[0]; }
    bool mixed() const { return mix_; }
    // ST_OPTIONS with a message when the session stores FP16 deltas
    int need_fp32_storage(const char *what);
    // Test hook: the next stage launch's work item `item` leaves its plane
    // copy number `fill` unissued, once, and every bounded wait of the stage
    // kernel gives up after `wait_cycles` clocks (0: the default limit).
    int test_stall(int item, int fill, long long wait_cycles);
    // the stage descriptor of RK stage irk (with FP16 storage: for the
    // step-start state of step parity `parity`), and the stage's work items
    // (batches use these)
    void stage_desc(int irk, CgStageDesc &d) const;
    void stage_desc_mix(int parity, int irk, CgStageDesc &d) const;
    int stage_items() const;
    int pml_faces() const;
    int launch_sources_on(cudaStream_t st);
    int launch_stations_on(cudaStream_t st);
    int launch_pga_on(cudaStream_t st);
    int check_errors() { return check_device_error(); }
    bool snapshots_on() const;

private:
    // adjoint state: lambda', mu, running sum (9 fields each), the per-
    // direction difference adjoints (27 fields), the surface channels, the
    // auxiliaries' adjoints per face, the gradient and d rdz / d (mu, lambda)
    struct Adjoint {
        float *Lp = nullptr, *M = nullptr, *Lam = nullptr, *Phi = nullptr, *SF = nullptr;
        float *M2 = nullptr, *B2[5] = {};   // the fused kernel's second mu buffers
        PmlFace face[5] = {};
        float *grad = nullptr, *drdz = nullptr;
    } adj_;
    int adj_prepare();
    HBox hbox() const;                                          // points outside the PML layers
    void adj_args(AdjStageArgs &a, int irk, const int FB[3]) const;
    int adj_step(int n, float *const *h4, float *const *vd4);  // lambda_{n+1} -> lambda_n
    void adj_swap();
    size_t state_bytes() const;                                  // W_A and the faces' A
    int save_state(char *dst);
    int load_state(const char *src);
    void ckpt_parts(std::vector<std::pair<void *, size_t>> &parts) const;
    int run_plain(int n);                 // n steps from `it`, graphs where aligned
    int write_snapshots(int step);        // slices after step `step`
    std::string out_dir() const;
    float *slice_dev_ = nullptr;
};

}  // namespace cgfdm
