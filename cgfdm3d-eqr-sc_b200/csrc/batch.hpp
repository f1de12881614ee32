// A batch of CGFDM sessions advanced together (see batch.cu).
#pragma once

#include <cuda_runtime.h>

#include <string>
#include <vector>

#include "session.hpp"

namespace cgfdm {

class Batch {
public:
    ~Batch();
    int create(const std::vector<Session *> &sessions);
    int run(int nsteps, float *ms = nullptr);   // ms: device time of the steps, if given
    int remaining() const;                      // steps left to the shortest session's NT
    // autotuner of the batched launch (csrc/autotune.cu): z planes per work
    // item (every session) and persistent CTAs
    int set_tiling(int kchunk, int ctas);
    int autotune(int trial_steps, int *kchunk, int *ctas, float *ms_per_step);
    // rows of the column tiles of every session's stage (4 or 8; ring
    // pipeline either way)
    int set_tile(int rows);
    int tile() const { return tile_; }

    std::vector<Session *> s;
    int device = 0;
    int it = 0;
    double points = 0;          // interior points of all sessions
    long long kernel_launches = 0;
    std::string err;
    cudaStream_t stream = nullptr;

private:
    int launch_step(int step);
    int build_tables();                         // descriptor table, item prefix, CTA count
    void drop_graph();
    int want_ctas_ = 0;                         // requested persistent CTAs (0: all resident)
    int tile_ = 4;
    bool mix_ = false;                          // FP16 storage (every session)
    CgStageDesc *descm_[2][4] = {};             // mixed storage: per step parity
    CgStageDesc *desc_[4] = {};
    int *items_ = nullptr;
    int *work_ = nullptr;
    int grid_ctas_ = 1;
    cudaEvent_t ev_[2] = {};
    cudaGraphExec_t graph8_ = nullptr;
    cudaGraph_t graph8_src_ = nullptr;
};

}  // namespace cgfdm
