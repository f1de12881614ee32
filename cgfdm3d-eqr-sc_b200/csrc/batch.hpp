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

    std::vector<Session *> s;
    int device = 0;
    int it = 0;
    double points = 0;          // interior points of all sessions
    long long kernel_launches = 0;
    std::string err;
    cudaStream_t stream = nullptr;

private:
    int launch_step(int step);
    CgStageDesc *desc_[4] = {};
    int *items_ = nullptr;
    int *work_ = nullptr;
    int grid_ctas_ = 1;
    cudaEvent_t ev_[2] = {};
    cudaGraphExec_t graph8_ = nullptr;
    cudaGraph_t graph8_src_ = nullptr;
};

}  // namespace cgfdm
