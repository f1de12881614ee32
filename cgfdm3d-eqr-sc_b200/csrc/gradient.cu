// Session side of the CGFDM adjoint: the gradient of the seismogram misfit
//     J = 1/2 sum_{station, sample, component} (v - d)^2
// (v the recorded velocity, d the observed one) with respect to Vp, Vs and
// rho, by the discrete adjoint of the whole time loop with checkpointing:
//
//   1. forward run from step 0, the state (W and the PML auxiliaries) kept
//      in device memory every K steps;
//   2. for each segment of K steps, last first: restore its checkpoint, run
//      it forward again storing each stage's RHS h_s (and the surface
//      layer's tangential velocity derivatives), then step the adjoint back
//      through it, adding the residual of each sample at the stations and
//      accumulating the gradient from mu_s . dh_s/dm;
//   3. chain rule from (mu, lambda, buoyancy) to (Vp, Vs, rho).
//
// Point sources do not depend on the medium; a finite-fault table (scaled
// by mu at its cells) is refused.  The gradient is zero in the PML layers.
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>

#include "session.hpp"
#include "session_util.hpp"

#ifndef ADJF_KCHUNK
#define ADJF_KCHUNK 16   // planes per block of the fused adjoint kernel (16 x 8-row tiles measured fastest)
#endif

namespace cgfdm {

__global__ void k_zero_halo(float *W, int nf, DevGrid g)
{
    const long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const long long npad = (long long)g.nxp * g.nyp * g.nzp;
    if (n >= npad) return;
    const int i = (int)(n % g.nxp), j = (int)((n / g.nxp) % g.nyp), k = (int)(n / ((long long)g.nxp * g.nyp));
    if (i >= CGFDM_HALO && i < g.nxp - CGFDM_HALO && j >= CGFDM_HALO && j < g.nyp - CGFDM_HALO && k >= CGFDM_HALO &&
        k < g.nzp - CGFDM_HALO)
        return;
    for (int f = 0; f < nf; f++) W[f * g.fstride + g.at(i, j, k)] = 0.0f;
}

static cudaError_t zero_halo(float *W, int nf, const DevGrid &g, cudaStream_t st)
{
    const long long npad = (long long)g.nxp * g.nyp * g.nzp;
    k_zero_halo<<<(unsigned)((npad + 255) / 256), 256, 0, st>>>(W, nf, g);
    return cudaGetLastError();
}

// ------------------------------------------------------------ state I/O
size_t Session::state_bytes() const
{
    size_t b = sizeof(float) * (size_t)g.fstride * 9;
    for (int fc = 0; fc < 5; fc++) b += sizeof(float) * (size_t)face_[fc].count * 9;
    return b;
}

int Session::save_state(char *dst)
{
    size_t off = 0, w = sizeof(float) * (size_t)g.fstride * 9;
    CU(cudaMemcpyAsync(dst, W_[0], w, cudaMemcpyDeviceToDevice, stream));
    off += w;
    for (int fc = 0; fc < 5; fc++) {
        size_t b = sizeof(float) * (size_t)face_[fc].count * 9;
        if (b) CU(cudaMemcpyAsync(dst + off, face_[fc].A, b, cudaMemcpyDeviceToDevice, stream));
        off += b;
    }
    return ST_OK;
}

int Session::load_state(const char *src)
{
    size_t off = 0, w = sizeof(float) * (size_t)g.fstride * 9;
    CU(cudaMemcpyAsync(W_[0], src, w, cudaMemcpyDeviceToDevice, stream));
    // the halo of the stage buffers mirrors W_A's (point sources write all three)
    CU(cudaMemcpyAsync(W_[1], src, w, cudaMemcpyDeviceToDevice, stream));
    CU(cudaMemcpyAsync(W_[2], src, w, cudaMemcpyDeviceToDevice, stream));
    off += w;
    for (int fc = 0; fc < 5; fc++) {
        size_t b = sizeof(float) * (size_t)face_[fc].count * 9;
        if (b) CU(cudaMemcpyAsync(face_[fc].A, src + off, b, cudaMemcpyDeviceToDevice, stream));
        off += b;
    }
    return ST_OK;
}

int Session::set_wavefield(const float *host)
{
    if (int st = need_fp32_storage("set_wavefield")) return st;
    const long long npad = m.g.npad();
    float *d = nullptr;
    CU(cudaMalloc(&d, sizeof(float) * npad * 9));
    cudaError_t e = cudaMemcpyAsync(d, host, sizeof(float) * npad * 9, cudaMemcpyHostToDevice, stream);
    for (int b = 0; b < 3 && e == cudaSuccess; b++) e = launch_from_aos(d, 9, g, W_[b], stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(e, "set_wavefield");
    return ST_OK;
}

int Session::set_medium(const float *host)
{
    if (int st = need_fp32_storage("set_medium")) return st;
    if (m.p.scheme != SCHEME_CGFDM) {
        err = "set_medium takes CGFDM sessions";
        return ST_OPTIONS;
    }
    const long long npad = m.g.npad();
    FieldVec old = m.medium;
    m.medium.assign(host, host + npad * 3);
    float vpmax = 0.0f;
    for (long long n = 0; n < npad; n++) vpmax = std::max(vpmax, m.medium[n * 3 + 1]);
    if ((float)m.p.DT > (float)(1.34 * m.H_min / vpmax)) {
        m.medium.swap(old);
        err = "the new medium violates the CFL condition at this DT";
        return ST_CFL;
    }
    m.Vp_max = vpmax;
    m.dtmax = (float)(1.34 * m.H_min / m.Vp_max);
    materialize_coords(m);   // the set-up kernels take the coordinate volume
    float *d_coord = nullptr, *d_med = nullptr;
    CU(cudaMalloc(&d_coord, sizeof(float) * npad * 3));
    cudaError_t e = cudaMalloc(&d_med, sizeof(float) * npad * 3);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_coord, m.coord.data(), sizeof(float) * npad * 3, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_med, m.medium.data(), sizeof(float) * npad * 3, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = launch_setup(d_coord, d_med, cjm_, rdz_, g, m.g.rDH, m.p.scheme, m.p.metric_fp64, stream);
    if (e == cudaSuccess && m.fault.npts > 0)
        e = cudaMemcpyAsync((void *)fault_.rate, m.fault.rate.data(), sizeof(float) * m.fault.rate.size(),
                            cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess && m.fault.npts > 0)
        e = launch_scale_moment((float *)fault_.rate, fault_.cell, fault_.npts, fault_.nt, cjm_, g, m.g.DH, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    cudaFree(d_coord);
    cudaFree(d_med);
    if (e != cudaSuccess) return cuda_fail(e, "set_medium");
    // back to step 0
    for (int b = 0; b < 4; b++) CU(cudaMemsetAsync(W_[b], 0, sizeof(float) * g.fstride * 9, stream));
    for (int fc = 0; fc < 5; fc++)
        if (face_[fc].count) {
            const size_t b = sizeof(float) * (size_t)face_[fc].count * 9;
            CU(cudaMemsetAsync(face_[fc].A, 0, b, stream));
            CU(cudaMemsetAsync(face_[fc].B, 0, b, stream));
            CU(cudaMemsetAsync(face_[fc].T, 0, b, stream));
        }
    CU(cudaMemsetAsync(pgv_, 0, sizeof(float) * m.g.nx * m.g.ny * 2, stream));
    if (pga_) CU(cudaMemsetAsync(pga_, 0, sizeof(float) * m.g.nx * m.g.ny * 2, stream));
    if (dis_) CU(cudaMemsetAsync(dis_, 0, sizeof(float) * g.fstride * 3, stream));
    if (st_out_) CU(cudaMemsetAsync(st_out_, 0, sizeof(float) * nst * std::max(m.NT, 1) * 9, stream));
    CU(cudaMemsetAsync(it_dev_, 0, sizeof(int), stream));
    CU(cudaStreamSynchronize(stream));
    it = 0;
    return ST_OK;
}

// ------------------------------------------------------------- adjoint
int Session::adj_prepare()
{
    if (m.p.scheme != SCHEME_CGFDM) {
        err = "the adjoint is built for the CGFDM scheme";
        return ST_OPTIONS;
    }
    if (m.g.nz < m.g.nPML + 8 || m.g.nx < 2 * m.g.nPML + 6 || m.g.ny < 2 * m.g.nPML + 6) {
        err = "the adjoint needs NZ >= nPML + 8 and NX, NY >= 2 nPML + 6";
        return ST_OPTIONS;
    }
    if (adj_.Lp) return ST_OK;
    const long long F = g.fstride;
    ALLOC(adj_.Lp, float, F * 9);
    ALLOC(adj_.M, float, F * 9);
    ALLOC(adj_.Lam, float, F * 9);
    if (!m.p.adj_fused) {
        ALLOC(adj_.Phi, float, F * 27);
        ALLOC(adj_.SF, float, g.plane * 36);
    } else {
        ALLOC(adj_.M2, float, F * 9);
    }
    ALLOC(adj_.grad, float, F * 3);
    ALLOC(adj_.drdz, float, g.plane * 36);
    for (int fc = 0; fc < 5; fc++) {
        adj_.face[fc] = face_[fc];
        if (!face_[fc].count) continue;
        ALLOC(adj_.face[fc].A, float, face_[fc].count * 9);
        ALLOC(adj_.face[fc].B, float, face_[fc].count * 9);
        ALLOC(adj_.face[fc].T, float, face_[fc].count * 9);
        if (m.p.adj_fused) ALLOC(adj_.B2[fc], float, face_[fc].count * 9);
    }
    return ST_OK;
}

HBox Session::hbox() const
{
    const int n = m.p.pml ? m.g.nPML : 0;
    HBox b;
    b.x0 = CGFDM_HALO + n, b.y0 = CGFDM_HALO + n, b.z0 = CGFDM_HALO + n;
    b.nx = m.g.nx - 2 * n, b.ny = m.g.ny - 2 * n, b.nz = m.g.nz - n;   // no PML under the free surface
    b.fstride = ((long long)b.nx * b.ny * b.nz + 63) / 64 * 64;
    return b;
}

void Session::adj_args(AdjStageArgs &a, int irk, const int FB[3]) const
{
    std::memset(&a, 0, sizeof a);
    a.g = g;
    a.hbox = hbox();
    a.cjm = cjm_;
    a.rdz = rdz_;
    a.drdz = adj_.drdz;
    a.pml_alpha_x = pml_[0], a.pml_beta_x = pml_[1], a.pml_d_x = pml_[2];
    a.pml_alpha_y = pml_[3], a.pml_beta_y = pml_[4], a.pml_d_y = pml_[5];
    a.pml_alpha_z = pml_[6], a.pml_beta_z = pml_[7], a.pml_d_z = pml_[8];
    a.Lp = adj_.Lp;
    a.M = adj_.M;
    a.Lam = adj_.Lam;
    a.Phi = adj_.Phi;
    a.SF = adj_.SF;
    for (int fc = 0; fc < 5; fc++) a.face[fc] = adj_.face[fc], a.faceB2[fc] = adj_.B2[fc];
    a.M2 = adj_.M2;
    a.kchunk = std::min(m.g.nz, ADJF_KCHUNK);
    a.nchunk = (m.g.nz + a.kchunk - 1) / a.kchunk;
    a.grad = adj_.grad;
    a.irk = irk;
    const int sgn = (irk & 1) ? -1 : 1;
    a.FB1 = FB[0] * sgn, a.FB2 = FB[1] * sgn, a.FB3 = FB[2] * sgn;
    a.nPML = m.g.nPML;
    a.pml_on = m.p.pml;
    a.fs_on = 1;
    a.rDH = m.g.rDH;
    a.DT = (float)m.p.DT;
}

void Session::adj_swap()
{
    std::swap(adj_.Lp, adj_.Lam);
    for (int fc = 0; fc < 5; fc++) std::swap(adj_.face[fc].A, adj_.face[fc].T);
}

// One step back: lambda_{n+1} (in Lp) -> lambda_n (in Lp after the swap).
int Session::adj_step(int n, float *const *h4, float *const *vd4)
{
    int FB[3];
    fb_signs(n, FB);
    for (int irk = 3; irk >= 0; irk--) {
        AdjStageArgs a;
        adj_args(a, irk, FB);
        a.h = h4 ? h4[irk] : nullptr;
        a.vd = vd4 ? vd4[irk] : nullptr;
        if (!a.h) a.grad = nullptr;
        if (!m.p.adj_fused) {
            CU(launch_adj_stage(a, stream));
        } else {
            CU(launch_adj_stage_fused(a, stream));
            // mu_{s-1} was written beside mu_s
            std::swap(adj_.M, adj_.M2);
            for (int fc = 0; fc < 5; fc++) std::swap(adj_.face[fc].B, adj_.B2[fc]);
        }
    }
    kernel_launches += m.p.adj_fused ? 4 : 8;
    adj_swap();
    return ST_OK;
}

int Session::adjoint_apply(int nsteps, float *host)
{
    if (int st = need_fp32_storage("adjoint_apply")) return st;
    if (nsteps < 0 || nsteps > it) {
        err = "adjoint_apply covers steps the session has run: 0 <= nsteps <= steps completed";
        return ST_ARG;
    }
    if (int st = adj_prepare()) return st;
    const long long npad = m.g.npad();
    float *d = nullptr;
    CU(cudaMalloc(&d, sizeof(float) * npad * 9));
    cudaError_t e = cudaMemcpyAsync(d, host, sizeof(float) * npad * 9, cudaMemcpyHostToDevice, stream);
    if (e == cudaSuccess) e = launch_from_aos(d, 9, g, adj_.Lp, stream);
    if (e == cudaSuccess) e = zero_halo(adj_.Lp, 9, g, stream);
    for (int fc = 0; fc < 5 && e == cudaSuccess; fc++)
        if (adj_.face[fc].count) e = cudaMemsetAsync(adj_.face[fc].A, 0, sizeof(float) * adj_.face[fc].count * 9, stream);
    if (e != cudaSuccess) {
        cudaFree(d);
        return cuda_fail(e, "adjoint_apply");
    }
    int st = ST_OK;
    for (int n = it - 1; n >= it - nsteps && st == ST_OK; n--) st = adj_step(n, nullptr, nullptr);
    if (st == ST_OK) {
        e = launch_to_aos(adj_.Lp, 9, g, d, stream);
        if (e == cudaSuccess) e = cudaMemcpyAsync(host, d, sizeof(float) * npad * 9, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        if (e != cudaSuccess) st = cuda_fail(e, "adjoint_apply");
    }
    cudaFree(d);
    return st;
}

// RAII for the gradient's scratch allocations
// Scratch of the gradient (checkpoints, stage stores, residuals): one
// device block per device, kept while a session exists on that device and
// reused by the next gradient call of any of them, so a run of gradient
// calls maps its tens of GB once.  Gradient calls on one device take turns.
namespace {
struct Arena {
    void *p = nullptr;
    size_t bytes = 0;
    int sessions = 0;
    std::mutex mu;
};
std::mutex g_arenas_mu;
std::map<int, Arena> g_arenas;

Arena &arena_of(int device)
{
    std::lock_guard<std::mutex> lk(g_arenas_mu);
    return g_arenas[device];
}

// carves aligned sub-buffers out of the arena
struct Carve {
    char *base;
    size_t off = 0;
    template <typename T>
    T *take(size_t bytes)
    {
        T *r = reinterpret_cast<T *>(base + off);
        off += (bytes + 255) / 256 * 256;
        return r;
    }
};
}  // namespace

void arena_session_add(int device)
{
    Arena &A = arena_of(device);
    std::lock_guard<std::mutex> lk(A.mu);
    A.sessions++;
}

void arena_session_remove(int device)
{
    Arena &A = arena_of(device);
    std::lock_guard<std::mutex> lk(A.mu);
    if (--A.sessions == 0 && A.p) {
        int cur = 0;
        cudaGetDevice(&cur);
        cudaSetDevice(device);
        cudaFree(A.p);
        cudaSetDevice(cur);
        A.p = nullptr;
        A.bytes = 0;
    }
}

int Session::gradient(const float *obs, int K, double *misfit, float *grad_out)
{
    if (int st = need_fp32_storage("gradient")) return st;
    if (it != 0) {
        err = "gradient starts from step 0 (set_medium returns a session there)";
        return ST_STATE;
    }
    if (K < 1) {
        err = "checkpoint interval must be >= 1";
        return ST_ARG;
    }
    if (m.fault.npts > 0) {
        err = "the gradient takes point sources (a finite-fault table is scaled by mu)";
        return ST_OPTIONS;
    }
    if (int st = adj_prepare()) return st;
    CU(launch_surface_derivs(cjm_, g, adj_.drdz, stream));  // of the current medium
    const int NT = m.NT;
    K = std::min(K, std::max(NT, 1));
    const int nseg = (NT + K - 1) / K;
    const long long F = g.fstride;
    const size_t sb = state_bytes();

    Arena &arena = arena_of(device);
    std::lock_guard<std::mutex> arena_lock(arena.mu);
    char *ckpt = nullptr, *final_state = nullptr;
    float *hstore = nullptr, *vdstore = nullptr, *res = nullptr, *d_med = nullptr, *d_grad = nullptr;
    // stage stores of one segment; the last R segments are stored during the
    // first forward run (as many as device memory holds), the others are
    // re-run from their checkpoints into slot 0
    const HBox hb = hbox();
    const size_t hseg = sizeof(float) * (size_t)hb.fstride * 9 * 4 * K;
    const size_t vseg = sizeof(float) * (size_t)g.plane * 6 * 4 * K;
    const long long nres = (long long)nst * NT * 3;
    const long long npad = m.g.npad();
    auto round256 = [](size_t b) { return (b + 255) / 256 * 256; };
    const size_t other = round256(sb * nseg) + round256(sb) + round256(sizeof(float) * nres) +
                         round256(sizeof(float) * npad * 3) +
                         round256(sizeof(float) * (size_t)m.g.nx * m.g.ny * m.g.nz * 3);
    int R = 1;
    {
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        fr += arena.bytes;   // the arena's block is available to this call
        const size_t reserve = (size_t)768 << 20;
        if (other + round256(hseg) + round256(vseg) + reserve > fr) {
            err = "the gradient needs " + std::to_string((other + hseg + vseg) >> 20) + " MiB of device memory for " +
                  "checkpoints and stage stores at this checkpoint interval; " + std::to_string(fr >> 20) +
                  " MiB are free";
            return ST_ALLOC;
        }
        R = (int)std::min<size_t>((size_t)nseg, (fr - other - reserve) / (round256(hseg) + round256(vseg)));
        if (m.p.adj_store_max > 0) R = std::min(R, m.p.adj_store_max);
    }
    const size_t need = other + R * (round256(hseg) + round256(vseg));
    if (arena.bytes < need) {
        if (arena.p) CU(cudaFree(arena.p));
        arena.p = nullptr;
        arena.bytes = 0;
        CU(cudaMalloc(&arena.p, need));
        arena.bytes = need;
    }
    Carve cv{static_cast<char *>(arena.p)};
    ckpt = cv.take<char>(sb * nseg);
    final_state = cv.take<char>(sb);
    hstore = cv.take<float>(hseg * R);   // R whole segments: round256(hseg) == hseg for 256-byte multiples
    vdstore = cv.take<float>(vseg * R);
    if (nres) res = cv.take<float>(sizeof(float) * nres);
    d_med = cv.take<float>(sizeof(float) * npad * 3);
    d_grad = cv.take<float>(sizeof(float) * (size_t)m.g.nx * m.g.ny * m.g.nz * 3);
    auto slot_of = [&](int s) { return s >= nseg - R ? s - (nseg - R) : 0; };

    cudaEvent_t ev[2];
    CU(cudaEventCreate(&ev[0]));
    CU(cudaEventCreate(&ev[1]));
    struct EvFree {
        cudaEvent_t *e;
        ~EvFree() { cudaEventDestroy(e[0]), cudaEventDestroy(e[1]); }
    } evfree{ev};
    float ms_re = 0.0f, ms_adj = 0.0f;
    auto lap = [&](float *acc) -> int {
        CU(cudaEventRecord(ev[1], stream));
        CU(cudaEventSynchronize(ev[1]));
        float ms = 0.0f;
        CU(cudaEventElapsedTime(&ms, ev[0], ev[1]));
        *acc += ms;
        CU(cudaEventRecord(ev[0], stream));
        return ST_OK;
    };

    // steps n0 .. n1-1 from the current state, storing each stage's RHS
    auto hptr = [&](int slot, int t, int irk) {
        return hstore + (size_t)hb.fstride * 9 * (((size_t)slot * K + t) * 4 + irk);
    };
    auto vdptr = [&](int slot, int t, int irk) {
        return vdstore + (size_t)g.plane * 6 * (((size_t)slot * K + t) * 4 + irk);
    };
    // (first: the forward run itself, which keeps PGV, PGA and displacement;
    // a re-run must not add its displacement a second time)
    auto run_storing = [&](int n0, int n1, int slot, bool first) -> int {
        for (int n = n0; n < n1; n++) {
            if (int st = launch_sources_on(stream)) return st;
            int FB[3];
            fb_signs(n, FB);
            for (int irk = 0; irk < 4; irk++) {
                CgStageDesc d = desc_host_[irk];
                if (!first) {
                    d.a.pgv = nullptr;
                    d.a.dis = nullptr;
                }
                d.a.hstore = hptr(slot, n - n0, irk);
                d.a.hbox = hb;
                d.a.vdstore = vdptr(slot, n - n0, irk);
                const int sgn = (irk & 1) ? -1 : 1;
                if (int st = launch_stage(FB[0] * sgn, FB[1] * sgn, FB[2] * sgn, d)) return st;
            }
            if (first)
                if (int st = launch_pga_on(stream)) return st;
            if (int st = launch_stations_on(stream)) return st;
            kernel_launches += 6;
        }
        return ST_OK;
    };

    // 1. forward with checkpoints; the last R segments store their stage
    //    RHS on the way, so they need no second run
    grad_ms[0] = grad_ms[1] = grad_ms[2] = 0.0f;
    CU(cudaEventRecord(ev[0], stream));
    nvtxRangePushA("gradient: forward with checkpoints");
    struct NvtxPop {
        bool on = true;
        void pop()
        {
            if (on) nvtxRangePop();
            on = false;
        }
        ~NvtxPop() { pop(); }
    } nvtx_fwd;
    for (int s = 0; s < nseg; s++) {
        if (int st = save_state(ckpt + sb * s)) return st;
        const int n = std::min(K, NT - it);
        if (s < nseg - R) {
            if (int st = run_plain(n)) return st;
        } else {
            if (int st = run_storing(it, it + n, slot_of(s), true)) return st;
            it += n;
        }
    }
    if (int st = save_state(final_state)) return st;
    if (int st = lap(&grad_ms[0])) return st;
    nvtx_fwd.pop();
    if (int st = check_device_error()) return st;

    // residuals and misfit
    double J = 0.0;
    if (nres) {
        std::vector<float> rec((size_t)nst * NT * 9), r((size_t)nres);
        CU(cudaMemcpy(rec.data(), st_out_, sizeof(float) * rec.size(), cudaMemcpyDeviceToHost));
        for (long long s = 0; s < nst; s++)
            for (long long n = 0; n < NT; n++)
                for (int c = 0; c < 3; c++) {
                    const long long o = (s * NT + n) * 3 + c;
                    const double d = (double)rec[(s * NT + n) * 9 + c] - (double)obs[o];
                    r[o] = (float)d;
                    J += 0.5 * d * d;
                }
        CU(cudaMemcpyAsync(res, r.data(), sizeof(float) * nres, cudaMemcpyHostToDevice, stream));
    }
    if (misfit) *misfit = J;

    // 2. backward, segment by segment
    CU(cudaEventRecord(ev[0], stream));
    CU(cudaMemsetAsync(adj_.Lp, 0, sizeof(float) * F * 9, stream));
    CU(cudaMemsetAsync(adj_.Lam, 0, sizeof(float) * F * 9, stream));
    CU(cudaMemsetAsync(adj_.grad, 0, sizeof(float) * F * 3, stream));
    for (int fc = 0; fc < 5; fc++)
        if (adj_.face[fc].count) {
            CU(cudaMemsetAsync(adj_.face[fc].A, 0, sizeof(float) * adj_.face[fc].count * 9, stream));
            CU(cudaMemsetAsync(adj_.face[fc].T, 0, sizeof(float) * adj_.face[fc].count * 9, stream));
        }
    for (int s = nseg - 1; s >= 0; s--) {
        const int n0 = s * K, n1 = std::min(NT, n0 + K);
        nvtxRangePushA("gradient: segment");
        NvtxPop nvtx_seg;
        if (s < nseg - R) {
            // forward again from the segment's checkpoint, storing each stage's RHS
            if (int st = load_state(ckpt + sb * s)) return st;
            CU(cudaMemcpyAsync(it_dev_, &n0, sizeof(int), cudaMemcpyHostToDevice, stream));
            if (int st = run_storing(n0, n1, 0, false)) return st;
            if (int st = lap(&ms_re)) return st;
        }
        // and back through it
        for (int n = n1 - 1; n >= n0; n--) {
            CU(launch_adj_residual(adj_.Lp, g, st_idx_, nst, NT, n, res, stream));
            float *h4[4], *vd4[4];
            for (int irk = 0; irk < 4; irk++) {
                h4[irk] = hptr(slot_of(s), n - n0, irk);
                vd4[irk] = vdptr(slot_of(s), n - n0, irk);
            }
            if (int st = adj_step(n, h4, vd4)) return st;
            kernel_launches += 1;
        }
        if (int st = lap(&ms_adj)) return st;
    }
    grad_ms[1] = ms_re;
    grad_ms[2] = ms_adj;

    // 3. chain rule and output; the session returns to its final state
    CU(cudaMemcpyAsync(d_med, m.medium.data(), sizeof(float) * npad * 3, cudaMemcpyHostToDevice, stream));
    CU(launch_grad_chain(adj_.grad, d_med, g, d_grad, stream));
    CU(cudaMemcpyAsync(grad_out, d_grad, sizeof(float) * (size_t)m.g.nx * m.g.ny * m.g.nz * 3, cudaMemcpyDeviceToHost,
                       stream));
    if (int st = load_state(final_state)) return st;
    CU(cudaMemcpyAsync(it_dev_, &NT, sizeof(int), cudaMemcpyHostToDevice, stream));
    CU(cudaStreamSynchronize(stream));
    return check_device_error();
}

}  // namespace cgfdm
