// Batches: several CGFDM sessions -- independent shots or media of uneven
// grid sizes -- advanced together, each RK stage of all of them in one
// persistent launch of the fused stage kernel.
//
// The stage kernel walks work items from one atomic counter; a batch hands
// it the concatenated descriptor table of its sessions (tensor maps and
// arguments per session) and the prefix offsets of their work items, so
// small grids that could not fill 148 SMs on their own share one launch.
// A step is: the source kernels of every session, four batched stage
// launches, the station kernels of every session; eight steps (one cycle of
// the FB sign table) are captured once as a CUDA graph and replayed.  The
// sessions must be CGFDM, live on one device and stand at the same step;
// each keeps its own buffers, step counter and error word.
#include "batch.hpp"

#include <algorithm>
#include <cstring>

namespace cgfdm {

static const int FB_BATCH[8][3] = {{-1, -1, -1}, {1, 1, -1}, {1, 1, 1},  {-1, -1, 1},
                                   {-1, 1, -1},  {1, -1, -1}, {1, -1, 1}, {-1, 1, 1}};  // src/propagate.cpp:158-168

#define BCU(x)                                                                                                   \
    do {                                                                                                         \
        cudaError_t e__ = (x);                                                                                   \
        if (e__ != cudaSuccess) {                                                                                \
            err = std::string(#x) + ": " + cudaGetErrorString(e__);                                              \
            return ST_CUDA;                                                                                      \
        }                                                                                                        \
    } while (0)

Batch::~Batch()
{
    if (graph8_) cudaGraphExecDestroy(graph8_);
    if (graph8_src_) cudaGraphDestroy(graph8_src_);
    for (int irk = 0; irk < 4; irk++) {
        if (desc_[irk]) cudaFree(desc_[irk]);
        for (int par = 0; par < 2; par++)
            if (descm_[par][irk]) cudaFree(descm_[par][irk]);
    }
    if (items_) cudaFree(items_);
    if (work_) cudaFree(work_);
    if (ev_[0]) cudaEventDestroy(ev_[0]);
    if (ev_[1]) cudaEventDestroy(ev_[1]);
    if (stream) cudaStreamDestroy(stream);
}

int Batch::create(const std::vector<Session *> &sessions)
{
    if (sessions.empty()) {
        err = "empty batch";
        return ST_ARG;
    }
    s = sessions;
    device = s[0]->device;
    it = s[0]->it;
    for (Session *x : s) {
        if (x->m.p.scheme != SCHEME_CGFDM) {
            err = "batches take CGFDM sessions only";
            return ST_ARG;
        }
        if (x->device != device) {
            err = "batch sessions must share one device";
            return ST_ARG;
        }
        if (x->it != it) {
            err = "batch sessions must stand at the same step";
            return ST_ARG;
        }
        if (x->snapshots_on()) {
            err = "batch sessions cannot write snapshots";
            return ST_ARG;
        }
        if (x->mixed() != s[0]->mixed()) {
            err = "batch sessions must share one storage (FP32 or FP16)";
            return ST_OPTIONS;
        }
    }
    mix_ = s[0]->mixed();
    BCU(cudaSetDevice(device));
    for (Session *x : s) BCU(cudaStreamSynchronize(x->stream));
    // the batched launch runs the ring kernel, 32 x 4 tiles unless set_tile
    // chooses 8 rows
    for (Session *x : s)
        if (int st = x->set_tile(tile_)) {
            err = x->err;
            return st;
        }
    BCU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    BCU(cudaEventCreate(&ev_[0]));
    BCU(cudaEventCreate(&ev_[1]));
    const int n = (int)s.size();
    for (int irk = 0; irk < 4; irk++) BCU(cudaMalloc(&desc_[irk], sizeof(CgStageDesc) * n));
    if (mix_)
        for (int par = 0; par < 2; par++)
            for (int irk = 0; irk < 4; irk++) BCU(cudaMalloc(&descm_[par][irk], sizeof(CgStageDesc) * n));
    BCU(cudaMalloc(&items_, sizeof(int) * (n + 1)));
    BCU(cudaMalloc(&work_, sizeof(int) * 2));
    BCU(cudaMemset(work_, 0, sizeof(int) * 2));
    points = 0;
    for (Session *x : s) points += (double)x->m.g.nx * x->m.g.ny * x->m.g.nz;
    return build_tables();
}

// The sessions' stage descriptors and work-item prefix in device memory,
// and the persistent CTA count of the batched launch.
int Batch::build_tables()
{
    const int n = (int)s.size();
    std::vector<int> items(n + 1, 0);
    for (int i = 0; i < n; i++) items[i + 1] = items[i] + s[i]->stage_items();
    std::vector<CgStageDesc> d(n);
    for (int irk = 0; irk < 4; irk++) {
        for (int i = 0; i < n; i++) s[i]->stage_desc(irk, d[i]);
        BCU(cudaMemcpy(desc_[irk], d.data(), sizeof(CgStageDesc) * n, cudaMemcpyHostToDevice));
    }
    if (mix_)
        for (int par = 0; par < 2; par++)
            for (int irk = 0; irk < 4; irk++) {
                for (int i = 0; i < n; i++) s[i]->stage_desc_mix(par, irk, d[i]);
                BCU(cudaMemcpy(descm_[par][irk], d.data(), sizeof(CgStageDesc) * n, cudaMemcpyHostToDevice));
            }
    BCU(cudaMemcpy(items_, items.data(), sizeof(int) * (n + 1), cudaMemcpyHostToDevice));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int full =
        sms * (mix_ ? cg_stage_mix_ctas_per_sm() : tile_ == 8 ? ty8::cg_stage_ctas_per_sm() : cg_stage_ctas_per_sm());
    grid_ctas_ = std::min(want_ctas_ > 0 ? std::min(want_ctas_, full) : full, items[n]);
    return ST_OK;
}

int Batch::set_tile(int rows)
{
    if (rows != 4 && rows != 8) {
        err = "stage tiles have 4 or 8 rows";
        return ST_ARG;
    }
    BCU(cudaSetDevice(device));
    for (Session *x : s) BCU(cudaStreamSynchronize(x->stream));
    BCU(cudaStreamSynchronize(stream));
    for (Session *x : s)
        if (int st = x->set_tile(rows)) {
            err = x->err;
            return st;
        }
    tile_ = rows;
    if (int st = build_tables()) return st;
    drop_graph();
    return ST_OK;
}

void Batch::drop_graph()
{
    if (graph8_) cudaGraphExecDestroy(graph8_);
    if (graph8_src_) cudaGraphDestroy(graph8_src_);
    graph8_ = nullptr;
    graph8_src_ = nullptr;
}

int Batch::remaining() const
{
    int r = 1 << 30;
    for (Session *x : s) r = std::min(r, x->m.NT - x->it);
    return r;
}

int Batch::launch_step(int step)
{
    for (Session *x : s)
        if (int st = x->launch_sources_on(stream)) return st;
    int FB1 = FB_BATCH[step % 8][0], FB2 = FB_BATCH[step % 8][1], FB3 = FB_BATCH[step % 8][2];
    for (int irk = 0; irk < 4; irk++) {
        if (mix_)
            BCU(launch_cg_stage_batch_mix(FB1, FB2, FB3, descm_[step & 1][irk], items_, (int)s.size(), work_,
                                          grid_ctas_, stream));
        else if (tile_ == 8)
            BCU(ty8::launch_cg_stage_batch(FB1, FB2, FB3, desc_[irk], items_, (int)s.size(), work_, grid_ctas_,
                                           stream));
        else
            BCU(launch_cg_stage_batch(FB1, FB2, FB3, desc_[irk], items_, (int)s.size(), work_, grid_ctas_, stream));
        FB1 = -FB1, FB2 = -FB2, FB3 = -FB3;
    }
    for (Session *x : s)
        if (int st = x->launch_pga_on(stream)) return st;
    for (Session *x : s)
        if (int st = x->launch_stations_on(stream)) return st;
    return ST_OK;
}

int Batch::run(int nsteps, float *ms)
{
    if (nsteps < 0) {
        err = "negative step count";
        return ST_ARG;
    }
    BCU(cudaSetDevice(device));
    for (Session *x : s) {
        BCU(cudaStreamSynchronize(x->stream));
        if (x->it != it) {
            err = "a batch session was stepped on its own";
            return ST_STATE;
        }
    }
    const int n = std::min(nsteps, remaining());
    if (ms) BCU(cudaEventRecord(ev_[0], stream));
    int done = 0;
    while (done < n && (it + done) % 8 != 0) {
        if (int st = launch_step(it + done)) return st;
        done++;
    }
    const int n8 = (n - done) / 8;
    if (n8 > 0) {
        if (!graph8_) {
            BCU(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
            int st = ST_OK;
            for (int k = 0; k < 8 && st == ST_OK; k++) st = launch_step(k);
            cudaGraph_t g = nullptr;
            cudaError_t e = cudaStreamEndCapture(stream, &g);
            if (st) return st;
            BCU(e);
            graph8_src_ = g;
            BCU(cudaGraphInstantiate(&graph8_, graph8_src_, 0));
        }
        for (int r = 0; r < n8; r++) BCU(cudaGraphLaunch(graph8_, stream));
        done += n8 * 8;
    }
    while (done < n) {
        if (int st = launch_step(it + done)) return st;
        done++;
    }
    if (ms) BCU(cudaEventRecord(ev_[1], stream));
    BCU(cudaStreamSynchronize(stream));
    if (ms) BCU(cudaEventElapsedTime(ms, ev_[0], ev_[1]));
    it += n;
    int rc = ST_OK;
    kernel_launches += (long long)n * 4;
    for (Session *x : s) {
        x->it += n;
        kernel_launches += (long long)n * (1 + (x->m.fault.npts > 0) + (x->m.point.kind != 0 && x->m.point.inside));
        if (int st = x->check_errors()) {
            err = x->err;
            rc = st;
        }
    }
    return rc;
}

}  // namespace cgfdm
