// Autotuner of the CGFDM stage launch: the work decomposition -- the tile
// height (4 or 8 rows of 32 columns, where the pipeline has both), z planes
// per work item (the pencil a CTA marches through: longer pencils re-read
// fewer chunk-edge planes, shorter ones balance the persistent CTAs better
// on small or uneven grids) and the number of persistent CTAs -- is chosen
// by timing candidates on trial steps.  The tiling changes no arithmetic:
// results are bit-identical for every choice.  Each trial starts from a
// device copy of the state (wavefield, PML auxiliaries, PGV, displacement,
// step counter), which is restored after the last trial, so tuning does
// not advance the run.
#include <algorithm>
#include <vector>

#include "batch.hpp"
#include "session.hpp"
#include "session_util.hpp"

namespace cgfdm {

// pencil lengths tried (clamped to the grid; the current one is added)
static const int KCHUNK_CANDIDATES[] = {8, 12, 16, 20, 24, 32, 48, 64, 96, 128, 192, 256};

static int device_sms(int device)
{
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    return sms;
}

static std::vector<int> kchunk_candidates(int nz_max, int current)
{
    std::vector<int> c;
    for (int k : KCHUNK_CANDIDATES)
        if (k < nz_max) c.push_back(k);
    c.push_back(nz_max);
    if (current > 0) c.push_back(std::min(current, nz_max));
    std::sort(c.begin(), c.end());
    c.erase(std::unique(c.begin(), c.end()), c.end());
    return c;
}

// ------------------------------------------------------------- session
int Session::set_tiling(int kc, int ctas)
{
    if (m.p.scheme != SCHEME_CGFDM) {
        err = "tiling applies to the CGFDM stage kernel";
        return ST_OPTIONS;
    }
    if (kc < 1 || ctas < 1) {
        err = "kchunk and ctas must be >= 1";
        return ST_ARG;
    }
    kchunk_ = std::min(kc, m.g.nz);
    nchunk_ = (m.g.nz + kchunk_ - 1) / kchunk_;
    grid_ctas_ = (int)std::min<long long>(std::min(ctas, device_sms(device) * stage_ctas_per_sm()),
                                          (long long)stage_items());
    if (int st = build_stage_descs()) return st;
    if (graph8_) cudaGraphExecDestroy(graph8_);
    if (graph8_src_) cudaGraphDestroy(graph8_src_);
    graph8_ = nullptr;
    graph8_src_ = nullptr;
    return ST_OK;
}

size_t Session::tune_bytes() const
{
    size_t b = state_bytes() + sizeof(float) * (size_t)m.g.nx * m.g.ny * 2;
    if (dis_) b += sizeof(float) * (size_t)g.fstride * 3;
    if (pga_) b += sizeof(float) * (size_t)m.g.nx * m.g.ny * 2;
    return b;
}

int Session::tune_save(char *dev)
{
    if (int st = save_state(dev)) return st;
    size_t off = state_bytes();
    const size_t pb = sizeof(float) * (size_t)m.g.nx * m.g.ny * 2;
    CU(cudaMemcpyAsync(dev + off, pgv_, pb, cudaMemcpyDeviceToDevice, stream));
    off += pb;
    if (dis_) CU(cudaMemcpyAsync(dev + off, dis_, sizeof(float) * g.fstride * 3, cudaMemcpyDeviceToDevice, stream));
    if (dis_) off += sizeof(float) * g.fstride * 3;
    if (pga_) CU(cudaMemcpyAsync(dev + off, pga_, pb, cudaMemcpyDeviceToDevice, stream));
    return ST_OK;
}

int Session::tune_load(const char *dev)
{
    if (int st = load_state(dev)) return st;
    size_t off = state_bytes();
    const size_t pb = sizeof(float) * (size_t)m.g.nx * m.g.ny * 2;
    CU(cudaMemcpyAsync(pgv_, dev + off, pb, cudaMemcpyDeviceToDevice, stream));
    off += pb;
    if (dis_) CU(cudaMemcpyAsync(dis_, dev + off, sizeof(float) * g.fstride * 3, cudaMemcpyDeviceToDevice, stream));
    if (dis_) off += sizeof(float) * g.fstride * 3;
    if (pga_) CU(cudaMemcpyAsync(pga_, dev + off, pb, cudaMemcpyDeviceToDevice, stream));
    CU(cudaMemcpyAsync(it_dev_, &it, sizeof(int), cudaMemcpyHostToDevice, stream));
    return ST_OK;
}

int Session::time_steps(int nsteps, float *ms)
{
    CU(cudaEventRecord(ev_[0], stream));
    for (int s = 0; s < nsteps; s++)
        if (int st = launch_step(it + s)) return st;
    CU(cudaEventRecord(ev_[1], stream));
    CU(cudaEventSynchronize(ev_[1]));
    CU(cudaEventElapsedTime(ms, ev_[0], ev_[1]));
    return check_device_error();
}

int Session::autotune(int trial, int *best_kc, int *best_ctas, float *best_ms)
{
    if (int st = need_fp32_storage("autotune")) return st;
    if (m.p.scheme != SCHEME_CGFDM) {
        err = "the autotuner tunes the CGFDM stage kernel";
        return ST_OPTIONS;
    }
    trial = std::min(trial, m.NT - it - 1);
    if (trial < 1) {
        err = "too few steps left to tune on";
        return ST_STATE;
    }
    char *buf = nullptr;
    CU(cudaMalloc(&buf, tune_bytes()));
    struct Free {
        char *p;
        ~Free() { cudaFree(p); }
    } fr{buf};
    if (int st = tune_save(buf)) return st;
    // the current decomposition first; another one replaces it only when
    // it is faster by more than the trials' noise (1 %)
    const int t0 = tile_, k0 = kchunk_, c0 = grid_ctas_;
    int bt = t0, bk = k0, bc = c0;
    float bms = 1e30f, ms0 = 1e30f;
    struct Cand {
        int rows, kc, ctas;
    };
    std::vector<Cand> cand{{t0, k0, c0}};
    const bool both = !mix_ && !part_session_;
    for (int rows : {4, 8}) {
        if (rows == 8 && !both) continue;
        if (int st = set_tile(rows)) return st;
        const int full = device_sms(device) * stage_ctas_per_sm();
        for (int kc : kchunk_candidates(m.g.nz, kchunk_))
            for (int ctas : {full, full * 2 / 3}) cand.push_back({rows, kc, ctas});
    }
    for (const Cand &c : cand) {
        if (int st = set_tile(c.rows)) return st;
        if (int st = set_tiling(c.kc, c.ctas)) return st;
        float ms = 0.0f;
        if (int st = tune_load(buf)) return st;
        if (int st = time_steps(1, &ms)) return st;   // first launch of this shape
        if (int st = tune_load(buf)) return st;
        if (int st = time_steps(trial, &ms)) return st;
        if (c.rows == t0 && c.kc == k0 && c.ctas == c0) ms0 = std::min(ms0, ms);
        if (ms < bms) bms = ms, bt = c.rows, bk = c.kc, bc = c.ctas;
    }
    if (bms > 0.99f * ms0) bt = t0, bk = k0, bc = c0, bms = ms0;
    if (int st = set_tile(bt)) return st;
    if (int st = set_tiling(bk, bc)) return st;
    if (int st = tune_load(buf)) return st;
    CU(cudaStreamSynchronize(stream));
    if (best_kc) *best_kc = kchunk_;
    if (best_ctas) *best_ctas = grid_ctas_;
    if (best_ms) *best_ms = bms / trial;
    return ST_OK;
}

// --------------------------------------------------------------- batch
#define BCU(x)                                                                                                   \
    do {                                                                                                         \
        cudaError_t e__ = (x);                                                                                   \
        if (e__ != cudaSuccess) {                                                                                \
            err = std::string(#x) + ": " + cudaGetErrorString(e__);                                              \
            return ST_CUDA;                                                                                      \
        }                                                                                                        \
    } while (0)

int Batch::set_tiling(int kc, int ctas)
{
    if (kc < 1 || ctas < 1) {
        err = "kchunk and ctas must be >= 1";
        return ST_ARG;
    }
    for (Session *x : s)
        if (int st = x->set_tiling(kc, 1 << 30)) {
            err = x->err;
            return st;
        }
    want_ctas_ = ctas;
    if (int st = build_tables()) return st;
    drop_graph();
    return ST_OK;
}

int Batch::autotune(int trial, int *best_kc, int *best_ctas, float *best_ms)
{
    if (mix_) {
        // its trials restore the state from a device copy, which FP16
        // storage does not offer (as for a single session)
        err = "autotune is not available with FP16 storage";
        return ST_OPTIONS;
    }
    trial = std::min(trial, remaining() - 1);
    if (trial < 1) {
        err = "too few steps left to tune on";
        return ST_STATE;
    }
    BCU(cudaSetDevice(device));
    std::vector<char *> bufs(s.size(), nullptr);
    struct Free {
        std::vector<char *> &b;
        ~Free()
        {
            for (char *p : b) cudaFree(p);
        }
    } fr{bufs};
    for (size_t i = 0; i < s.size(); i++) {
        BCU(cudaMalloc(&bufs[i], s[i]->tune_bytes()));
        if (int st = s[i]->tune_save(bufs[i])) {
            err = s[i]->err;
            return st;
        }
    }
    auto load_all = [&]() -> int {
        for (size_t i = 0; i < s.size(); i++)
            if (int st = s[i]->tune_load(bufs[i])) {
                err = s[i]->err;
                return st;
            }
        for (Session *x : s) BCU(cudaStreamSynchronize(x->stream));
        return ST_OK;
    };
    auto time_batch = [&](int n, float *ms) -> int {
        BCU(cudaEventRecord(ev_[0], stream));
        for (int k = 0; k < n; k++)
            if (int st = launch_step(it + k)) return st;
        BCU(cudaEventRecord(ev_[1], stream));
        BCU(cudaEventSynchronize(ev_[1]));
        BCU(cudaEventElapsedTime(ms, ev_[0], ev_[1]));
        return ST_OK;
    };
    int nz_max = 1;
    for (Session *x : s) nz_max = std::max(nz_max, x->m.g.nz);
    // the current decomposition (each session's own pencil) first; a
    // uniform one replaces it only when faster by more than the trials'
    // noise (1 %)
    std::vector<int> k_orig;
    for (Session *x : s) k_orig.push_back(x->kchunk());
    const int want_orig = want_ctas_, t_orig = tile_;
    float ms0 = 0.0f;
    if (int st = load_all()) return st;
    if (int st = time_batch(1, &ms0)) return st;
    if (int st = load_all()) return st;
    if (int st = time_batch(trial, &ms0)) return st;
    int bk = 0, bc = 0, bt = t_orig;
    float bms = 1e30f;
    bool eight = true;   // every session can take 32 x 8 tiles (FP32 storage, whole grid)
    for (Session *x : s) eight = eight && !x->mixed() && !x->part_session_;
    for (int rows : {4, 8}) {
        if (rows == 8 && !eight) continue;
        if (int st = set_tile(rows)) return st;
        const int full = device_sms(device) * (rows == 8 ? ty8::cg_stage_ctas_per_sm() : cg_stage_ctas_per_sm());
        for (int kc : kchunk_candidates(nz_max, 0))
            for (int ctas : {full, full * 2 / 3}) {
                if (int st = set_tiling(kc, ctas)) return st;
                float ms = 0.0f;
                if (int st = load_all()) return st;
                if (int st = time_batch(1, &ms)) return st;
                if (int st = load_all()) return st;
                if (int st = time_batch(trial, &ms)) return st;
                if (ms < bms) bms = ms, bk = kc, bc = ctas, bt = rows;
            }
    }
    if (bms > 0.99f * ms0) {
        if (int st = set_tile(t_orig)) return st;
        for (size_t i = 0; i < s.size(); i++)
            if (int st = s[i]->set_tiling(k_orig[i], 1 << 30)) {
                err = s[i]->err;
                return st;
            }
        want_ctas_ = want_orig;
        if (int st = build_tables()) return st;
        drop_graph();
        bk = 0;   // per-session pencils kept
        bms = ms0;
    } else {
        if (int st = set_tile(bt)) return st;
        if (int st = set_tiling(bk, bc)) return st;
    }
    if (int st = load_all()) return st;
    for (Session *x : s)
        if (int st = x->check_errors()) {
            err = x->err;
            return st;
        }
    if (best_kc) *best_kc = bk;
    if (best_ctas) *best_ctas = grid_ctas_;
    if (best_ms) *best_ms = bms / trial;
    return ST_OK;
}

}  // namespace cgfdm
