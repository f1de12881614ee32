// Session: device buffers, GPU setup, the per-step launch sequence and its
// CUDA-graph capture, and result readback.
//
// Per step the reference runs, on one rank (src/propagate.cpp:186-321):
// source into W -> 4 RK stages (deriv, free surface, PML, RK) -> stations
// -> PGV.  Here a step is: source kernel, four fused stage kernels (PGV is
// folded into the last), station kernel.  Eight consecutive steps cover
// one cycle of the FB sign table (src/propagate.cpp:158-168) and are
// captured once as a CUDA graph that is replayed.
#include "session.hpp"
#include "session_util.hpp"
#include "upload.hpp"

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <sys/stat.h>

namespace cgfdm {

static const int FB_TABLE[8][3] = {{-1, -1, -1}, {1, 1, -1}, {1, 1, 1}, {-1, -1, 1},
                                   {-1, 1, -1},  {1, -1, -1}, {1, -1, 1}, {-1, 1, 1}};

void fb_signs(int step, int fb[3])
{
    for (int c = 0; c < 3; c++) fb[c] = FB_TABLE[step % 8][c];
}

// ----------------------------------------------------------------- CFL
// Smallest/largest point-to-plane distance through the six diagonal
// neighbour planes (src/calc_CFL.cpp:56-163), in double with each operation
// rounded separately, reduced with integer atomics on the (non-negative)
// bit patterns.
__global__ void k_hrange(const float *__restrict__ coord, int nxp, int nyp, int nzp, unsigned long long *hmin,
                         unsigned long long *hmax)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x + CGFDM_HALO;
    const int j = blockIdx.y * blockDim.y + threadIdx.y + CGFDM_HALO;
    const int k = blockIdx.z * blockDim.z + threadIdx.z + CGFDM_HALO;
    double lo = 1.0e20, hi = 0.0;
    if (i < nxp - CGFDM_HALO && j < nyp - CGFDM_HALO && k < nzp - CGFDM_HALO) {
        auto at = [&](int a, int b, int c) { return ((long long)c * nyp + b) * nxp + a; };
        long long p = at(i, j, k) * 3;
        double P[3] = {coord[p], coord[p + 1], coord[p + 2]};
        for (int ii = -1; ii <= 1; ii += 2)
            for (int jj = -1; jj <= 1; jj += 2)
                for (int kk = -1; kk <= 1; kk += 2) {
                    long long a = at(i - ii, j, k) * 3, b = at(i, j - jj, k) * 3, c = at(i, j, k - kk) * 3;
                    double A[3] = {coord[a], coord[a + 1], coord[a + 2]};
                    double B[3] = {coord[b], coord[b + 1], coord[b + 2]};
                    double C[3] = {coord[c], coord[c + 1], coord[c + 2]};
                    double AB[3], AC[3], PA[3], n[3];
                    for (int t = 0; t < 3; t++) {
                        AB[t] = __dsub_rn(B[t], A[t]);
                        AC[t] = __dsub_rn(C[t], A[t]);
                        PA[t] = __dsub_rn(P[t], A[t]);
                    }
                    n[0] = __dsub_rn(__dmul_rn(AB[1], AC[2]), __dmul_rn(AB[2], AC[1]));
                    n[1] = __dsub_rn(__dmul_rn(AB[2], AC[0]), __dmul_rn(AB[0], AC[2]));
                    n[2] = __dsub_rn(__dmul_rn(AB[0], AC[1]), __dmul_rn(AB[1], AC[0]));
                    double nd = __dsqrt_rn(__dadd_rn(__dadd_rn(__dmul_rn(n[0], n[0]), __dmul_rn(n[1], n[1])),
                                                     __dmul_rn(n[2], n[2])));
                    for (int t = 0; t < 3; t++) n[t] = __ddiv_rn(n[t], nd);
                    double d = fabs(__dadd_rn(__dadd_rn(__dmul_rn(PA[0], n[0]), __dmul_rn(PA[1], n[1])),
                                              __dmul_rn(PA[2], n[2])));
                    lo = lo < d ? lo : d;
                    hi = hi > d ? hi : d;
                }
    }
    // Warp reduction first, then one atomic pair per warp: a per-thread atomic
    // on the same two words serialises the whole grid in L2.
    for (int o = 16; o > 0; o >>= 1) {
        double l2 = __shfl_xor_sync(0xffffffffu, lo, o), h2 = __shfl_xor_sync(0xffffffffu, hi, o);
        lo = lo < l2 ? lo : l2;
        hi = hi > h2 ? hi : h2;
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMin(hmin, (unsigned long long)__double_as_longlong(lo));
        atomicMax(hmax, (unsigned long long)__double_as_longlong(hi));
    }
}

// ----------------------------------------------------------------- util
Session::~Session()
{
    if (med_thread_.joinable()) med_thread_.join();
    if (counted_) arena_session_remove(device);
    if (graph8_) cudaGraphExecDestroy(graph8_);
    if (graph8_src_) cudaGraphDestroy(graph8_src_);
    for (auto &e : ev_)
        if (e) cudaEventDestroy(e);
    for (void *p : ipc_open_) cudaIpcCloseMemHandle(p);
    for (void *p : allocs_) cudaFree(p);
    if (arena_) cudaFree(arena_);
    if (stream) cudaStreamDestroy(stream);
}

int Session::cuda_fail(cudaError_t e, const char *what)
{
    err = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? ST_ALLOC : ST_CUDA;
}

void *Session::alloc(size_t bytes)
{
    void *p = nullptr;
    const size_t rounded = (bytes + 255) / 256 * 256;
    if (arena_ && arena_used_ + rounded <= arena_size_) {
        p = arena_ + arena_used_;
        if (cudaMemsetAsync(p, 0, bytes, stream) != cudaSuccess) return nullptr;
        arena_used_ += rounded;
        device_bytes += bytes;
        return p;
    }
    if (cudaMalloc(&p, bytes) != cudaSuccess) return nullptr;
    if (cudaMemsetAsync(p, 0, bytes, stream) != cudaSuccess) {
        cudaFree(p);
        return nullptr;
    }
    allocs_.push_back(p);
    device_bytes += bytes;
    return p;
}

// --------------------------------------------------------------- create
#ifndef CG_MEDIUM_OVERLAP
#define CG_MEDIUM_OVERLAP 1   // the medium upload overlaps the rest of the host model build
#endif
static double ms_since(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

int Session::create(const std::string &dir, const std::string &options, int dev)
{
    const auto t0 = std::chrono::steady_clock::now();
    run_dir = dir;
    device = dev;
    // a large medium volume starts its way to the device as soon as it is
    // read, while the host model build goes on (ranges, PML profiles,
    // sources, stations)
    auto medium_ready = [&](const Model &mm) {
        if (!CG_MEDIUM_OVERLAP) return;
        const size_t bytes = sizeof(float) * (size_t)mm.g.npad() * 3;
        if (bytes < (size_t(64) << 20) || mm.medium.size() * sizeof(float) < bytes) return;
        float *p = nullptr;
        if (cudaSetDevice(dev) != cudaSuccess || cudaMalloc(&p, bytes) != cudaSuccess) {
            cudaGetLastError();
            return;   // setup_device uploads it then
        }
        pre_med_ = p;
        allocs_.push_back(p);
        device_bytes += bytes;
        const float *src = mm.medium.data();
        med_thread_ = std::thread([this, p, src, bytes, dev] {
            cudaStream_t st = nullptr;
            med_err_ = cudaSetDevice(dev);
            if (med_err_ == cudaSuccess) med_err_ = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
            if (med_err_ == cudaSuccess) med_err_ = upload_h2d(p, src, bytes, dev, st);
            if (st) cudaStreamDestroy(st);
        });
    };
    int st = build_model(dir, options, m, err, medium_ready);
    if (st) return st;
    create_ms[0] = ms_since(t0);
    // the reference builds that exist: CGFDM with PML (Makefile_CGFDM), SCFDM
    // with the exponential sponge (Makefile_SCFDM); exp_decay_absorb.cpp only
    // compiles under SCFDM and the SCFDM flux kernels take no PML terms
    if (m.p.scheme == SCHEME_SCFDM && m.p.pml) {
        err = "PML is not available with the SCFDM scheme (use EXP_DECAY)";
        return ST_OPTIONS;
    }
    if (m.p.scheme == SCHEME_CGFDM && m.p.exp_decay) {
        err = "EXP_DECAY is only available with the SCFDM scheme";
        return ST_OPTIONS;
    }
    if (m.p.storage != "fp32" && m.p.storage != "fp16") {
        err = "storage must be \"fp32\" or \"fp16\"";
        return ST_OPTIONS;
    }
    mix_ = m.p.storage == "fp16";
    if (mix_ && m.p.scheme != SCHEME_CGFDM) {
        err = "FP16 storage is built for the CGFDM scheme";
        return ST_OPTIONS;
    }
    if (mix_ && m.p.solve_pga) {
        err = "SOLVE_PGA is not available with FP16 storage";
        return ST_OPTIONS;
    }
    if (m.p.scheme == SCHEME_SCFDM && m.g.nz < 8) {
        err = "the SCFDM scheme needs NZ >= 8";
        return ST_OPTIONS;
    }
    CU(cudaSetDevice(dev));
    arena_session_add(dev);
    counted_ = true;
    CU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    for (auto &e : ev_) CU(cudaEventCreate(&e));
    const auto t1 = std::chrono::steady_clock::now();
    st = setup_device();
    create_ms[1] = ms_since(t1);
    create_ms[2] = ms_since(t0);
    return st;
}

// Bytes of the arrays setup_device makes after its two upload buffers, each
// rounded to 256 (the same list, in the same order).
size_t Session::arena_estimate() const
{
    const Grid &G = m.g;
    const bool cg = m.p.scheme == SCHEME_CGFDM;
    const size_t F = (size_t)g.fstride;
    size_t b = 0;
    auto add = [&](size_t bytes) { b += (bytes + 255) / 256 * 256; };
    add(sizeof(float) * (size_t)G._nx_ * G._ny_);                  // height map
    add(sizeof(float) * F * (cg ? 13 : 19));                       // metric and medium
    if (cg) add(sizeof(float) * (size_t)g.plane * 18);             // free-surface matrices
    add(16);                                                       // spacing range
    if (mix_) {
        add(sizeof(float) * F * 9), add(sizeof(float) * F * 9);
        for (int x = 0; x < 3; x++) add(2 * (size_t)gh_.fstride * 9);
        add(80);
    } else {
        for (int x = 0; x < (cg ? 4 : 3); x++) add(sizeof(float) * F * 9);
    }
    add(4), add(8);
    if (!cg) add(sizeof(float) * F * 9), add(sizeof(float) * F), add(sizeof(float) * 64);
    if (cg) {
        add(sizeof(float) * G._nx_), add(sizeof(float) * G._nx_), add(sizeof(float) * G._nx_);
        add(sizeof(float) * G._ny_), add(sizeof(float) * G._ny_), add(sizeof(float) * G._ny_);
        add(sizeof(float) * G._nz_), add(sizeof(float) * G._nz_), add(sizeof(float) * G._nz_);
        if (m.p.pml) {
            const size_t nP = (size_t)G.nPML;
            const size_t cnt[5] = {nP * G.ny * G.nz, nP * G.nx * G.nz, nP * G.nx * G.ny, nP * G.ny * G.nz,
                                   nP * G.nx * G.nz};
            for (int fc = 0; fc < 5; fc++)
                if (pml_faces() & (1 << fc))
                    for (int x = 0; x < 3; x++) add(sizeof(float) * cnt[fc] * 9);
        }
    }
    add(sizeof(float) * (size_t)G.nx * G.ny * 2);
    if (m.p.solve_pga) add(sizeof(float) * (size_t)G.nx * G.ny * 2);
    if (m.p.solve_displacement) add(sizeof(float) * F * 3);
    const size_t ns = m.stations.size() / 3;
    if (ns > 0) add(sizeof(int) * ns * 3), add(sizeof(float) * ns * std::max(m.NT, 1) * 9);
    add(4);
    if (m.fault.npts > 0) add(sizeof(long long) * m.fault.npts), add(sizeof(float) * m.fault.rate.size());
    if (m.point.kind) add(sizeof(float) * m.point.amp.size()), add(sizeof(float) * std::max<size_t>(m.point.stf.size(), 1));
    return b + 4096;
}

int Session::setup_device()
{
    const Grid &G = m.g;
    g = make_devgrid(G.nx, G.ny, G.nz, m.p.scheme == SCHEME_CGFDM ? 29 : 1);
    const long long F = g.fstride;
    const long long npad = G.npad();
    const bool cg = m.p.scheme == SCHEME_CGFDM;

    // model arrays -> GPU, metrics on the GPU
    const auto t0 = std::chrono::steady_clock::now();
    float *d_coord, *d_med;
    ALLOC(d_coord, float, npad * 3);
    if (pre_med_)
        d_med = pre_med_;   // already on its way (Session::create)
    else
        ALLOC(d_med, float, npad * 3);
    if (mix_) {
        // FP16 arrays: first interior column on a 16-byte boundary in the TMA
        // halo box (xoff 33: column i0 - 4 = 32 + 32 n), rows of 16 bytes
        gh_ = make_devgrid(G.nx, G.ny, G.nz, 33);
        gh_.pitch = (gh_.pitch + 7) / 8 * 8;
        gh_.plane = (long long)gh_.nyp * gh_.pitch;
        gh_.fstride = ((long long)gh_.nzp * gh_.plane + 63) / 64 * 64;
    }
    if (!part_session_) {
        // the long-lived arrays in one block (falls back to one allocation
        // each if the block cannot be had).  Parts keep one allocation per
        // array: a neighbour in another process maps their stage buffers by
        // CUDA IPC, which maps whole allocations.
        const size_t want = arena_estimate();
        void *p = nullptr;
        if (cudaMalloc(&p, want) == cudaSuccess) {
            arena_ = (char *)p;
            arena_size_ = want;
        } else {
            cudaGetLastError();
        }
    }
    CU(cudaStreamSynchronize(stream));
    setup_ms[3] = ms_since(t0);   // allocation of the two upload buffers and the block
    if (m.coord_mode >= 0) {
        // the coordinates are made again on the device from the height map
        // (0.7 MB) instead of uploaded (12 bytes a point)
        float *d_terrain;
        ALLOC(d_terrain, float, (long long)G._nx_ * G._ny_);
        CU(cudaMemcpyAsync(d_terrain, m.terrain.data(), sizeof(float) * G._nx_ * G._ny_, cudaMemcpyHostToDevice,
                           stream));
        CU(launch_build_coords(d_coord, d_terrain, G._nx_, G._ny_, G._nz_, m.coord_mode, G.DH, G.originalX,
                               G.originalY, G.NZ, m.coord_depth_f, m.coord_depth_d, stream));
        h2d_bytes += sizeof(float) * G._nx_ * G._ny_;
    } else {
        materialize_coords(m);
        CU(upload_h2d(d_coord, m.coord.data(), sizeof(float) * npad * 3, device, stream));
        h2d_bytes += sizeof(float) * npad * 3;
    }
    if (pre_med_) {
        if (med_thread_.joinable()) med_thread_.join();
        if (med_err_ != cudaSuccess) return cuda_fail(med_err_, "medium upload");
    } else {
        CU(upload_h2d(d_med, m.medium.data(), sizeof(float) * npad * 3, device, stream));
    }
    h2d_bytes += sizeof(float) * npad * 3;
    CU(cudaStreamSynchronize(stream));
    setup_ms[4] = ms_since(t0) - setup_ms[3];   // the uploads
    const int ncjm = cg ? 13 : 19;
    ALLOC(cjm_, float, F * ncjm);
    if (cg) ALLOC(rdz_, float, g.plane * 18);
    // CFL (src/calc_CFL.cpp:255-349)
    {
        unsigned long long *d_h;
        ALLOC(d_h, unsigned long long, 2);
        unsigned long long init[2] = {(unsigned long long)0x7ff0000000000000ULL, 0ULL};
        CU(cudaMemcpyAsync(d_h, init, sizeof init, cudaMemcpyHostToDevice, stream));
        dim3 b(32, 4, 4), gr((G.nx + 31) / 32, (G.ny + 3) / 4, (G.nz + 3) / 4);
        k_hrange<<<gr, b, 0, stream>>>(d_coord, G._nx_, G._ny_, G._nz_, d_h, d_h + 1);
        CU(cudaGetLastError());
        unsigned long long hr[2];
        CU(cudaMemcpyAsync(hr, d_h, sizeof hr, cudaMemcpyDeviceToHost, stream));
        CU(cudaStreamSynchronize(stream));
        double lo, hi;
        std::memcpy(&lo, &hr[0], 8);
        std::memcpy(&hi, &hr[1], 8);
        m.H_min = (float)lo;
        m.H_max = (float)hi;
        m.dtmax = (float)(1.34 * m.H_min / m.Vp_max);
        if (m.p.DT > m.dtmax) {
            char buf[160];
            std::snprintf(buf, sizeof buf, "The parameters can't afford the CFL condition: DT = %g > dtmax = %g",
                          m.p.DT, (double)m.dtmax);
            err = buf;
            return ST_CFL;
        }
    }
    setup_ms[0] = ms_since(t0);   // allocation, uploads, CFL check (synchronised)
    CU(launch_setup(d_coord, d_med, cjm_, rdz_, g, G.rDH, m.p.scheme, m.p.metric_fp64, stream));

    // wavefield buffers: A (step start / final), B, C (stage values), T (RK4 sum)
    if (mix_) {
        ALLOC(W_[0], float, F * 9);
        ALLOC(Walt_, float, F * 9);
        ALLOC(Sb_, __half, gh_.fstride * 9);
        ALLOC(Sc_, __half, gh_.fstride * 9);
        ALLOC(T16_, __half, gh_.fstride * 9);
        ALLOC(mx_, unsigned, 20);   // [2][9] bounds, then the two impedance bounds
        const unsigned init[2] = {0x7f800000u, 0u};
        CU(cudaMemcpyAsync(mx_ + 18, init, sizeof init, cudaMemcpyHostToDevice, stream));
        CU(launch_impedance_bounds(cjm_, g, mx_ + 18, stream));
        unsigned zb[2];
        CU(cudaMemcpyAsync(zb, mx_ + 18, sizeof zb, cudaMemcpyDeviceToHost, stream));
        CU(cudaStreamSynchronize(stream));
        std::memcpy(&zs_min_, &zb[0], 4);
        std::memcpy(&zp_max_, &zb[1], 4);
    } else {
        for (int b = 0; b < (cg ? 4 : 3); b++) ALLOC(W_[b], float, F * 9);
    }
    ALLOC(err_dev_, int, 1);
    ALLOC(work_dev_, int, 2);
    // tile height: 32 x 8 for the FP32 split pipeline of a whole grid
    // (measured faster), 32 x 4 for the ring pipeline's users
    if (cg) {
        if (m.p.stage_tile != 0 && m.p.stage_tile != 4 && m.p.stage_tile != 8) {
            err = "\"stageTile\" is 4 or 8 (rows of 32-column stage tiles)";
            return ST_OPTIONS;
        }
        tile_ = m.p.stage_tile ? m.p.stage_tile : (m.p.stage_split && !mix_ && !part_session_ ? 8 : 4);
        if (tile_ == 8 && (mix_ || part_session_)) {
            err = "32 x 8 stage tiles need FP32 storage and a whole grid";
            return ST_OPTIONS;
        }
    }
    if (cg && !mix_)
        if (int st = build_maps()) return st;

    // SCFDM: RHS accumulator, DT * rDH / J, sponge factors, pass tiling
    if (!cg) {
        ALLOC(h_, float, F * 9);
        ALLOC(sjac_, float, F);
        CU(launch_sc_sjac(cjm_, g, (float)m.p.DT, m.g.rDH, sjac_, stream));
        CU(sc_dir_prepare());
        sct_ = sc_tiling(g);
        if (m.p.exp_decay) {
            // G[p] = exp(-(alpha p)^2), p = 0 .. 20, in float as
            // src/exp_decay_absorb.cpp:45,110-111 evaluates it
            const float alpha = (float)0.015;
            float G[SC_DECAY_LAYERS + 1];
            for (int p = 0; p <= SC_DECAY_LAYERS; p++) {
                const float x = alpha * (float)p;
                G[p] = std::exp(-x * x);
            }
            ALLOC(decay_, float, SC_DECAY_LAYERS + 1);
            CU(cudaMemcpyAsync(decay_, G, sizeof G, cudaMemcpyHostToDevice, stream));
        }
    }

    // PML profiles and auxiliaries
    if (cg && m.p.pml) {
        const std::vector<float> *prof[9] = {&m.pml_alpha_x, &m.pml_beta_x, &m.pml_d_x, &m.pml_alpha_y, &m.pml_beta_y,
                                             &m.pml_d_y,     &m.pml_alpha_z, &m.pml_beta_z, &m.pml_d_z};
        for (int a = 0; a < 9; a++) {
            ALLOC(pml_[a], float, prof[a]->size());
            CU(cudaMemcpyAsync(pml_[a], prof[a]->data(), sizeof(float) * prof[a]->size(), cudaMemcpyHostToDevice,
                               stream));
        }
        const long long nP = G.nPML;
        const long long cnt[5] = {nP * G.ny * G.nz, nP * G.nx * G.nz, nP * G.nx * G.ny, nP * G.ny * G.nz,
                                  nP * G.nx * G.nz};
        for (int fc = 0; fc < 5; fc++) {
            if (!(pml_faces() & (1 << fc))) continue;   // a part away from that boundary
            face_[fc].count = cnt[fc];
            ALLOC(face_[fc].A, float, cnt[fc] * 9);
            ALLOC(face_[fc].B, float, cnt[fc] * 9);
            ALLOC(face_[fc].T, float, cnt[fc] * 9);
        }
    } else if (cg) {
        // PML off: unit stretching, zero damping
        std::vector<float> one_x(G._nx_, 1.f), one_y(G._ny_, 1.f), one_z(G._nz_, 1.f);
        std::vector<float> zx(G._nx_, 0.f), zy(G._ny_, 0.f), zz(G._nz_, 0.f);
        const std::vector<float> *prof[9] = {&zx, &one_x, &zx, &zy, &one_y, &zy, &zz, &one_z, &zz};
        for (int a = 0; a < 9; a++) {
            ALLOC(pml_[a], float, prof[a]->size());
            CU(cudaMemcpyAsync(pml_[a], prof[a]->data(), sizeof(float) * prof[a]->size(), cudaMemcpyHostToDevice,
                               stream));
        }
    }

    // PGV, displacement, stations, step counter
    ALLOC(pgv_, float, (long long)G.nx * G.ny * 2);
    if (m.p.solve_pga) ALLOC(pga_, float, (long long)G.nx * G.ny * 2);
    if (m.p.solve_displacement) ALLOC(dis_, float, F * 3);
    nst = (int)m.stations.size() / 3;
    if (nst > 0) {
        ALLOC(st_idx_, int, nst * 3);
        CU(cudaMemcpyAsync(st_idx_, m.stations.data(), sizeof(int) * nst * 3, cudaMemcpyHostToDevice, stream));
        ALLOC(st_out_, float, (long long)nst * std::max(m.NT, 1) * 9);
    }
    ALLOC(it_dev_, int, 1);

    // finite fault: cells in this layout, table scaled by mu / (J DH^3)
    if (m.fault.npts > 0) {
        std::vector<long long> cells(m.fault.npts);
        for (long long p = 0; p < m.fault.npts; p++) {
            long long c = m.fault.index[p];
            int i = (int)(c % G._nx_), j = (int)((c / G._nx_) % G._ny_), k = (int)(c / ((long long)G._nx_ * G._ny_));
            cells[p] = g.at(i, j, k);
        }
        long long *d_cells;
        float *d_rate;
        ALLOC(d_cells, long long, m.fault.npts);
        ALLOC(d_rate, float, m.fault.rate.size());
        CU(cudaMemcpyAsync(d_cells, cells.data(), sizeof(long long) * cells.size(), cudaMemcpyHostToDevice, stream));
        CU(cudaMemcpyAsync(d_rate, m.fault.rate.data(), sizeof(float) * m.fault.rate.size(), cudaMemcpyHostToDevice,
                           stream));
        h2d_bytes += sizeof(float) * m.fault.rate.size();
        CU(launch_scale_moment(d_rate, d_cells, m.fault.npts, m.fault.nt, cjm_, g, G.DH, stream));
        fault_.rate = d_rate;
        fault_.cell = d_cells;
        fault_.npts = m.fault.npts;
        fault_.nt = m.fault.nt;
        fault_.dt = m.fault.dt;
    }
    if (m.point.kind) {
        point_.kind = m.point.kind;
        point_.X = m.point.X, point_.Y = m.point.Y, point_.Z = m.point.Z;
        point_.inside = m.point.inside;
        for (int c = 0; c < 6; c++) point_.mom[c] = m.point.mom[c];
        point_.m0 = m.point.m0;
        float *d_amp, *d_stf;
        ALLOC(d_amp, float, m.point.amp.size());
        ALLOC(d_stf, float, std::max<size_t>(m.point.stf.size(), 1));
        CU(cudaMemcpyAsync(d_amp, m.point.amp.data(), sizeof(float) * m.point.amp.size(), cudaMemcpyHostToDevice,
                           stream));
        if (!m.point.stf.empty())
            CU(cudaMemcpyAsync(d_stf, m.point.stf.data(), sizeof(float) * m.point.stf.size(),
                               cudaMemcpyHostToDevice, stream));
        point_.amp = d_amp;
        point_.stf = d_stf;
    }

    // work items for the persistent stage kernel: 32-column tiles times
    // z-chunks of about 8 planes (measured on 400x400x200: 8 planes 9.66 ms
    // per step, 16 9.80, 29 10.07, 4 9.95), at least four items per
    // resident CTA so the dynamic schedule ends evenly
    int dev_sms = 148;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, device);
    ntx_ = (G.nx + 31) / 32;
    nty_ = (G.ny + tile_ - 1) / tile_;
    const long long tiles = (long long)ntx_ * nty_;
    const int ctas = dev_sms * stage_ctas_per_sm();
    nchunk_ = std::max(1, (G.nz + 7) / 8);
    while (tiles * nchunk_ < 4LL * ctas && G.nz / (nchunk_ + 1) >= 12) nchunk_++;
    kchunk_ = (G.nz + nchunk_ - 1) / nchunk_;
    nchunk_ = (G.nz + kchunk_ - 1) / kchunk_;
    grid_ctas_ = (int)std::min<long long>(ctas, tiles * nchunk_);

    if (cg) {
        int st = build_stage_descs();
        if (st) return st;
    }

    setup_ms[1] = ms_since(t0) - setup_ms[0];   // state buffers, tables, descriptors (enqueued)
    CU(cudaStreamSynchronize(stream));
    setup_ms[2] = ms_since(t0) - setup_ms[0] - setup_ms[1];   // the set-up kernels and copies finishing
    // coordinates and medium are not needed on the device any more
    for (auto it_ = allocs_.begin(); it_ != allocs_.end();) {
        if (*it_ == d_coord || *it_ == d_med) {
            cudaFree(*it_);
            device_bytes -= sizeof(float) * npad * 3;
            it_ = allocs_.erase(it_);
        } else {
            ++it_;
        }
    }
    return ST_OK;
}

// The four stage descriptors (RK4 stage irk reads win[irk] and writes
// wout[irk]: A -> B, B -> C, C -> B, B -> A) with their tensor maps.
void Session::stage_desc(int irk, CgStageDesc &d) const
{
    float *A = W_[0], *B = W_[1], *C = W_[2], *T = W_[3];
    const float *win[4] = {A, B, C, B};
    const int win_map[4] = {0, 1, 2, 1};
    float *wout[4] = {B, C, B, A};
    std::memset(&d, 0, sizeof d);
    CgStageArgs &a = d.a;
    a.g = g;
    a.Win = win[irk];
    a.Wm = A;
    a.T = T;
    a.Wout = wout[irk];
    a.cjm = cjm_;
    a.rdz = rdz_;
    a.pml_alpha_x = pml_[0], a.pml_beta_x = pml_[1], a.pml_d_x = pml_[2];
    a.pml_alpha_y = pml_[3], a.pml_beta_y = pml_[4], a.pml_d_y = pml_[5];
    a.pml_alpha_z = pml_[6], a.pml_beta_z = pml_[7], a.pml_d_z = pml_[8];
    for (int fc = 0; fc < 5; fc++) a.face[fc] = face_[fc];
    a.pgv = irk == 3 ? pgv_ : nullptr;
    a.dis = irk == 3 ? dis_ : nullptr;
    a.irk = irk;
    a.nPML = m.g.nPML;
    a.pml_on = pml_faces();
    a.fs_on = m.fs_top ? 1 : 0;
    a.kchunk = kchunk_;
    a.rDH = m.g.rDH;
    a.DT = (float)m.p.DT;
    a.err = err_dev_;
    a.stall = stall_item_ >= 0 ? stall_dev_ : nullptr;
    a.stall_item = stall_item_;
    a.stall_fill = stall_fill_;
    a.wait_limit = wait_limit_;
    a.ntiles_x = ntx_, a.ntiles_y = nty_, a.nchunk = nchunk_;
    for (int f = 0; f < 6; f++) a.ho[f] = ho_[irk][f];
    std::memcpy(d.tmW, maps_[win_map[irk]].win, 128);
    std::memcpy(d.tmC, maps_[win_map[irk]].cjm, 128);
    std::memcpy(d.tmM, maps_[win_map[irk]].wm, 128);
    std::memcpy(d.tmT, maps_[win_map[irk]].t, 128);
    std::memcpy(d.tmWc, maps_[win_map[irk]].winp, 128);
}

int Session::stage_items() const { return ntx_ * nty_ * nchunk_; }

// Absorbing faces as stage-kernel bits x1 y1 z1 x2 y2 (PML off: none).
int Session::pml_faces() const
{
    if (!m.p.pml) return 0;
    return (m.border[0] ? 1 : 0) | (m.border[2] ? 2 : 0) | (m.border[4] ? 4 : 0) | (m.border[1] ? 8 : 0) |
           (m.border[3] ? 16 : 0);
}

int Session::stage_ctas_per_sm() const
{
    return mix_ ? cg_stage_mix_ctas_per_sm() : tile_ == 8 ? ty8::cg_stage_ctas_per_sm() : cg_stage_ctas_per_sm();
}

int Session::build_maps()
{
    auto tmap = [&](void *out, const float *base, int nf, bool halo) {
        return tile_ == 8 ? ty8::make_field_tmap(out, base, g, nf, halo) : make_field_tmap(out, base, g, nf, halo);
    };
    for (int b = 0; b < 3; b++) {
        CU(tmap(maps_[b].win, W_[b], 9, true));
        CU(tmap(maps_[b].winp, W_[b], 9, false));
        CU(tmap(maps_[b].cjm, cjm_, 13, false));
        CU(tmap(maps_[b].wm, W_[0], 9, false));
        CU(tmap(maps_[b].t, W_[3], 9, false));
    }
    return ST_OK;
}

int Session::set_tile(int rows)
{
    if (rows != 4 && rows != 8) {
        err = "stage tiles have 4 or 8 rows";
        return ST_ARG;
    }
    if (m.p.scheme != SCHEME_CGFDM || rows == tile_) return ST_OK;
    if (rows == 8 && (mix_ || part_session_)) {
        err = "32 x 8 stage tiles need FP32 storage and a whole grid";
        return ST_OPTIONS;
    }
    tile_ = rows;
    nty_ = (m.g.ny + tile_ - 1) / tile_;
    int dev_sms = 148;
    cudaDeviceGetAttribute(&dev_sms, cudaDevAttrMultiProcessorCount, device);
    grid_ctas_ = (int)std::min<long long>((long long)dev_sms * stage_ctas_per_sm(), (long long)stage_items());
    if (int st = build_maps()) return st;
    if (int st = build_stage_descs()) return st;
    if (graph8_) cudaGraphExecDestroy(graph8_);
    if (graph8_src_) cudaGraphDestroy(graph8_src_);
    graph8_ = nullptr;
    graph8_src_ = nullptr;
    return ST_OK;
}

int Session::launch_stage(int FB1, int FB2, int FB3, const CgStageDesc &d)
{
    cudaError_t e;
    if (m.p.stage_split && !mix_)
        e = tile_ == 8 ? ty8::launch_cg_stage_split(FB1, FB2, FB3, d, work_dev_, grid_ctas_, stream)
                       : launch_cg_stage_split(FB1, FB2, FB3, d, work_dev_, grid_ctas_, stream);
    else
        e = tile_ == 8 ? ty8::launch_cg_stage(FB1, FB2, FB3, d, work_dev_, grid_ctas_, stream)
                       : launch_cg_stage(FB1, FB2, FB3, d, work_dev_, grid_ctas_, stream);
    if (e != cudaSuccess) return cuda_fail(e, "stage launch");
    return ST_OK;
}

int Session::build_stage_descs()
{
    if (mix_) {
        for (int p = 0; p < 2; p++)
            for (int irk = 0; irk < 4; irk++) stage_desc_mix(p, irk, desc_mix_[p][irk]);
        return ST_OK;
    }
    for (int irk = 0; irk < 4; irk++) stage_desc(irk, desc_host_[irk]);
    return ST_OK;
}

// Mixed storage: stage irk of a step of the given parity.  The state A is
// read (with the delta of the previous stage as stencil input) and, in
// stage 3, the next state written to the other buffer; deltas go Sb -> Sc -> Sb.
void Session::stage_desc_mix(int parity, int irk, CgStageDesc &d) const
{
    stage_desc(irk, d);   // the common arguments; buffers and maps replaced below
    CgStageArgs &a = d.a;
    float *A = parity ? Walt_ : W_[0], *An = parity ? W_[0] : Walt_;
    a.gh = gh_;
    a.Win = A;
    a.Wm = A;
    a.T = nullptr;
    a.Wout = irk == 3 ? An : nullptr;
    a.Sin = irk == 0 ? nullptr : irk == 2 ? Sc_ : Sb_;
    a.Sout = irk == 0 ? Sb_ : irk == 1 ? Sc_ : irk == 2 ? Sb_ : nullptr;
    a.T16 = T16_;
    a.mx = mx_;
    a.it_dev = it_dev_;
    a.zs_min = zs_min_, a.zp_max = zp_max_;
    make_field_tmap(d.tmW, A, g, 9, true);
    make_field_tmap(d.tmC, cjm_, g, 13, false);
    make_field_tmap(d.tmM, A, g, 9, false);
    make_field_tmap16(d.tmT, T16_, gh_, 9);
    make_field_tmap16(d.tmS, irk == 2 ? Sc_ : Sb_, gh_, 9);
}

int Session::need_fp32_storage(const char *what)
{
    if (!mix_) return ST_OK;
    err = std::string(what) + " is not available with FP16 storage";
    return ST_OPTIONS;
}

// ----------------------------------------------------------------- step
int Session::launch_step(int step, bool timed_stages)
{
    const bool cg = m.p.scheme == SCHEME_CGFDM;
    const float DT = (float)m.p.DT;
    int FB1 = FB_TABLE[step % 8][0], FB2 = FB_TABLE[step % 8][1], FB3 = FB_TABLE[step % 8][2];
    if (int st = launch_sources_on(stream)) return st;
    if (cg) {
        for (int irk = 0; irk < 4; irk++) {
            if (timed_stages) CU(cudaEventRecord(ev_[2], stream));
            if (mix_)
                CU(launch_cg_stage_mix(FB1, FB2, FB3, desc_mix_[step & 1][irk], work_dev_, grid_ctas_, stream));
            else if (int st = launch_stage(FB1, FB2, FB3, desc_host_[irk]))
                return st;
            if (timed_stages) {
                CU(cudaEventRecord(ev_[3], stream));
                CU(cudaEventSynchronize(ev_[3]));
                float ms = 0;
                CU(cudaEventElapsedTime(&ms, ev_[2], ev_[3]));
                stage_ms_sum_ += ms;
                stage_ms_count_++;
            }
            FB1 = -FB1, FB2 = -FB2, FB3 = -FB3;
        }
        kernel_launches += 4;
    } else {
        // TVD-RK3: A -> B, (A, B) -> C, (A, C) -> A (src/propagate.cpp:212-244)
        float *A = W_[0], *B = W_[1], *C = W_[2];
        const float *win[3] = {A, B, C};
        float *wout[3] = {B, C, A};
        for (int irk = 0; irk < 3; irk++) {
            ScDirArgs a{};
            a.g = g;
            a.W = win[irk];
            a.Wm = A;
            a.Wout = wout[irk];
            a.H = h_;
            a.cjm = cjm_;
            a.sjac = sjac_;
            a.decay = irk == 2 ? decay_ : nullptr;
            a.ndecay = SC_DECAY_LAYERS;
            a.irk = irk;
            a.copy_halo = irk < 2;
            a.alpha = m.Vp_max;
            if (timed_stages) CU(cudaEventRecord(ev_[2], stream));
            for (int dir = 0; dir < 3; dir++) CU(launch_sc_dir(dir, a, sct_, stream));
            if (timed_stages) {
                CU(cudaEventRecord(ev_[3], stream));
                CU(cudaEventSynchronize(ev_[3]));
                float ms = 0;
                CU(cudaEventElapsedTime(&ms, ev_[2], ev_[3]));
                stage_ms_sum_ += ms;
                stage_ms_count_++;
            }
        }
        // characteristic free surface, halo, top-layer sponge, PGV (src/propagate.cpp:245-290)
        CU(launch_sc_surface(A, cjm_, g, decay_, SC_DECAY_LAYERS, pgv_, dis_, DT, stream));
        kernel_launches += 10;
    }
    if (int st = launch_pga_on(stream)) return st;
    if (int st = launch_stations_on(stream)) return st;
    kernel_launches += 1 + (fault_.npts > 0) + (point_.kind != 0 && point_.inside);
    return ST_OK;
}

// Sources into W at the stage-0 time of the step *it_dev_ (src/propagate.cpp:198-210).
int Session::launch_sources_on(cudaStream_t st)
{
    const float DT = (float)m.p.DT;
    if (mix_) {
        CU(launch_point(W_[0], nullptr, nullptr, cjm_, g, point_, it_dev_, DT, m.g.DH, m.p.scheme, st, Walt_, mx_));
        CU(launch_sources(W_[0], cjm_, g, fault_, point_, it_dev_, DT, m.g.DH, m.p.scheme, st, Walt_, mx_));
        return ST_OK;
    }
    CU(launch_point(W_[0], W_[1], W_[2], cjm_, g, point_, it_dev_, DT, m.g.DH, m.p.scheme, st));
    CU(launch_sources(W_[0], cjm_, g, fault_, point_, it_dev_, DT, m.g.DH, m.p.scheme, st));
    return ST_OK;
}

// Peak ground acceleration of the step just completed (SOLVE_PGA).
int Session::launch_pga_on(cudaStream_t st)
{
    if (!pga_) return ST_OK;
    CU(launch_pga(W_[0], cjm_, g, it_dev_, (float)m.p.DT, m.p.scheme, pga_, st));
    kernel_launches += 1;
    return ST_OK;
}

// Station traces of the step just completed; advances *it_dev_.
int Session::launch_stations_on(cudaStream_t st)
{
    CU(launch_stations(W_[0], cjm_, g, st_idx_, nst, m.NT, st_out_, it_dev_, m.p.scheme, st, mix_ ? Walt_ : nullptr));
    return ST_OK;
}

int Session::launch_steps_graph(int n8)
{
    if (!graph8_) {
        const auto t0 = std::chrono::steady_clock::now();
        CU(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        long long kl = kernel_launches;
        int st = ST_OK;
        for (int s = 0; s < 8 && st == ST_OK; s++) st = launch_step(s);
        cudaGraph_t gsrc = nullptr;
        cudaError_t e = cudaStreamEndCapture(stream, &gsrc);
        kernel_launches = kl;
        if (st) return st;
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        graph8_src_ = gsrc;
        CU(cudaGraphInstantiate(&graph8_, graph8_src_, 0));
        capture_ms += ms_since(t0);
    }
    const int stage_launches = m.p.scheme == SCHEME_CGFDM ? 4 : 10;
    long long per8 = 8LL * (stage_launches + 1 + (fault_.npts > 0) + (point_.kind != 0 && point_.inside));
    for (int r = 0; r < n8; r++) {
        CU(cudaGraphLaunch(graph8_, stream));
        graph_launches++;
        kernel_launches += per8;
    }
    return ST_OK;
}

// n steps from `it` without synchronizing: direct launches up to the next
// multiple of 8, the captured 8-step graph, direct launches for the rest.
int Session::run_plain(int n)
{
    int done = 0;
    while (done < n && (it + done) % 8 != 0) {
        int st = launch_step(it + done);
        if (st) return st;
        done++;
    }
    int n8 = (n - done) / 8;
    if (n8 > 0) {
        int st = launch_steps_graph(n8);
        if (st) return st;
        done += n8 * 8;
    }
    while (done < n) {
        int st = launch_step(it + done);
        if (st) return st;
        done++;
    }
    it += n;
    return ST_OK;
}

int Session::run(int nsteps)
{
    if (nsteps < 0) {
        err = "negative step count";
        return ST_ARG;
    }
    if (is_part_) {
        err = "a part of a decomposed grid steps with part_advance and halo exchanges";
        return ST_STATE;
    }
    int n = std::min(nsteps, m.NT - it);
    if (int st = run_checked(n)) return st;   // csrc/health.cu
    CU(cudaStreamSynchronize(stream));
    CU(cudaGetLastError());
    return check_device_error();
}

// n steps from `it`, with the snapshots that fall among them.
int Session::run_span(int n)
{
    if (!snapshots_on()) return run_plain(n);
    // snapshots after every step s with s % IT_SKIP == 0 (src/propagate.cpp:289-309)
    const int end = it + n;
    while (it < end) {
        int next = (it + m.p.IT_SKIP - 1) / m.p.IT_SKIP * m.p.IT_SKIP;  // first snapshot step >= it
        int stop = std::min(end, next + 1);
        int st = run_plain(stop - it);
        if (st) return st;
        if (stop == next + 1) {
            st = write_snapshots(next);
            if (st) return st;
        }
    }
    return ST_OK;
}

// A stage kernel whose bounded wait gave up leaves a bit in the error word.
int Session::check_device_error()
{
    int e = 0;
    CU(cudaMemcpy(&e, err_dev_, sizeof e, cudaMemcpyDeviceToHost));
    if (e) {
        err = "a stage kernel's bounded wait for its plane copies gave up (device error word " + std::to_string(e) + ")";
        return ST_TIMEOUT;
    }
    return ST_OK;
}

int Session::test_stall(int item, int fill, long long wait_cycles)
{
    if (m.p.scheme != SCHEME_CGFDM) {
        err = "the stall hook applies to the CGFDM stage kernel";
        return ST_OPTIONS;
    }
    if (item < 0 || item >= stage_items() || fill < 0 || wait_cycles < 0) {
        err = "stall hook: item, fill or wait_cycles out of range";
        return ST_ARG;
    }
    if (!stall_dev_) ALLOC(stall_dev_, int, 1);
    static const int one = 1;
    CU(cudaMemcpyAsync(stall_dev_, &one, sizeof one, cudaMemcpyHostToDevice, stream));
    CU(cudaStreamSynchronize(stream));
    stall_item_ = item, stall_fill_ = fill, wait_limit_ = wait_cycles;
    if (int st = build_stage_descs()) return st;
    // the captured steps hold the old descriptors
    if (graph8_) cudaGraphExecDestroy(graph8_);
    if (graph8_src_) cudaGraphDestroy(graph8_src_);
    graph8_ = nullptr;
    graph8_src_ = nullptr;
    return ST_OK;
}

// Device time of `nsteps` steps (events on the session stream) and, when
// stage_ms is given, the mean device time of one fused stage kernel, taken
// from a separate bracketed launch of each stage of one extra step.
int Session::run_timed(int nsteps, float *ms, float *stage_ms)
{
    int n = std::min(nsteps, m.NT - it);
    CU(cudaEventRecord(ev_[0], stream));
    int st = run(n);
    if (st) return st;
    CU(cudaEventRecord(ev_[1], stream));
    CU(cudaEventSynchronize(ev_[1]));
    CU(cudaEventElapsedTime(ms, ev_[0], ev_[1]));
    if (stage_ms) *stage_ms = 0.0f;
    return ST_OK;
}

int Session::profile_stages(int nsteps, float *mean)
{
    int n = std::min(nsteps, m.NT - it);
    stage_ms_sum_ = 0;
    stage_ms_count_ = 0;
    for (int s = 0; s < n; s++) {
        int st = launch_step(it + s, true);
        if (st) return st;
    }
    it += n;
    CU(cudaStreamSynchronize(stream));
    *mean = stage_ms_count_ ? (float)(stage_ms_sum_ / stage_ms_count_) : 0.0f;
    return check_device_error();
}

// Minimum bytes a step moves (float fields of 4 bytes): RK4 stages read the
// stencil input, 12 metric/medium fields and the RK state and write the stage
// output and accumulator, 39 + 57 + 57 + 39 = 192 fields per interior point;
// each absorbing face adds 27 + 45 + 45 + 27 = 144 auxiliary fields per slab
// point.
double Session::algo_bytes_per_step() const
{
    const Grid &G = m.g;
    double n = (double)G.nx * G.ny * G.nz;
    double faces = 0;
    // SCFDM: W_n + 13 metric/medium fields -> W1 (31 fields), then two stages
    // reading the stage value, the metric and W_n and writing W (40 each)
    if (m.p.scheme == SCHEME_SCFDM) return 4.0 * 111.0 * n;
    // FP16 storage: 4-byte state and metric fields, 2-byte deltas; stage 0
    // reads A and 12 metric fields and writes the delta (84 + 18 B), stage 1
    // adds the delta in and writes the accumulator and the next delta (102 +
    // 36), stages 2-3 also read the accumulator (120 + 36); stage 3 writes
    // the 4-byte state (120 + 36): 552 B per point and step
    if (mix_) {
        if (m.p.pml) faces = (double)G.nPML * (2.0 * G.ny * G.nz + 2.0 * G.nx * G.nz + (double)G.nx * G.ny);
        return 552.0 * n + 4.0 * 144.0 * faces;
    }
    if (m.p.pml && m.p.scheme == SCHEME_CGFDM)
        faces = (double)G.nPML * (2.0 * G.ny * G.nz + 2.0 * G.nx * G.nz + (double)G.nx * G.ny);
    return 4.0 * (192.0 * n + 144.0 * faces);
}

// ------------------------------------------------------------- readback
int Session::sync() const { return cudaStreamSynchronize(stream) == cudaSuccess ? ST_OK : ST_CUDA; }

int Session::get_wavefield(float *host) const
{
    float *d = nullptr;
    long long npad = m.g.npad();
    if (cudaMalloc(&d, sizeof(float) * npad * 9) != cudaSuccess) return ST_ALLOC;
    cudaError_t e = launch_to_aos(state(), 9, g, d, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, d, sizeof(float) * npad * 9, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    cudaFree(d);
    return e == cudaSuccess ? ST_OK : ST_CUDA;
}

int Session::get_cjm(float *host, int *nfield) const
{
    int nf = m.p.scheme == SCHEME_CGFDM ? 13 : 19;
    if (nfield) *nfield = nf;
    if (!host) return ST_OK;
    float *d = nullptr;
    long long npad = m.g.npad();
    if (cudaMalloc(&d, sizeof(float) * npad * nf) != cudaSuccess) return ST_ALLOC;
    cudaError_t e = launch_to_aos(cjm_, nf, g, d, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, d, sizeof(float) * npad * nf, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    cudaFree(d);
    return e == cudaSuccess ? ST_OK : ST_CUDA;
}

int Session::get_stations(float *host) const
{
    if (nst == 0) return ST_OK;
    cudaError_t e = cudaMemcpyAsync(host, st_out_, sizeof(float) * (size_t)nst * m.NT * 9, cudaMemcpyDeviceToHost,
                                    stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    return e == cudaSuccess ? ST_OK : ST_CUDA;
}

int Session::get_pgv(float *host) const
{
    const size_t n = (size_t)m.g.nx * m.g.ny;
    if (!pga_) {
        cudaError_t e = cudaMemcpyAsync(host, pgv_, sizeof(float) * n * 2, cudaMemcpyDeviceToHost, stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
        return e == cudaSuccess ? ST_OK : ST_CUDA;
    }
    // the reference's PGVSIZE = 4 record: PGVh, PGV, PGAh, PGA (src/PGV.cpp:140-171)
    std::vector<float> v(n * 2), a(n * 2);
    cudaError_t e = cudaMemcpyAsync(v.data(), pgv_, sizeof(float) * n * 2, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(a.data(), pga_, sizeof(float) * n * 2, cudaMemcpyDeviceToHost, stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
    if (e != cudaSuccess) return ST_CUDA;
    for (size_t p = 0; p < n; p++) {
        host[p * 4 + 0] = v[p * 2], host[p * 4 + 1] = v[p * 2 + 1];
        host[p * 4 + 2] = a[p * 2], host[p * 4 + 3] = a[p * 2 + 1];
    }
    return ST_OK;
}

// Output files of one rank in the reference's formats: station traces
// (src/station.cpp:422-443) and peak ground velocity (src/PGV.cpp:177-185).
// The directory is created when missing, as the reference creates OUT at
// start-up (src/create_dir.cpp).
std::string Session::out_dir() const
{
    std::string out = m.p.OUT;
    if (out.empty()) out = "./output";
    if (out[0] != '/') out = run_dir + "/" + out;
    for (size_t p = 1; p <= out.size(); p++)
        if (p == out.size() || out[p] == '/') mkdir(out.substr(0, p).c_str(), 0755);
    return out;
}

// "_mpi_X_Y_Z": the rank coordinates in every output file name
// (src/station.cpp:426, src/PGV.cpp:181, src/data_io.cpp:368-424); a part of a
// decomposed grid writes under its own coordinates.
static std::string rank_tag(const Model &m)
{
    return "_mpi_" + std::to_string(m.part_coord[0]) + "_" + std::to_string(m.part_coord[1]) + "_" +
           std::to_string(m.part_coord[2]);
}

// ---------------------------------------------------------------- snapshots
bool Session::snapshots_on() const
{
    if (m.p.IT_SKIP <= 0) return false;
    const int sx = m.p.sliceX + HALO, sy = m.p.sliceY + HALO, sz = m.p.sliceZ + HALO;
    return m.p.sliceFreeSurf || (sx >= HALO && sx < m.g._nx) || (sy >= HALO && sy < m.g._ny) ||
           (sz >= HALO && sz < m.g._nz);
}

// Velocity slices after step `step` (data2D_XYZ_out, src/data_io.cpp:485-560):
// OUT/V{x,y,z}_<step>_{X,Y,Z}_mpi_X_Y_Z.bin at the configured slices and,
// with sliceFreeSurf, OUT/FreeSurfV{x,y,z}_<step>_Z_mpi_X_Y_Z.bin of the top
// layer; with displacement on, OUT/FreeSurfU{x,y,z}_<step>_Z_... as well
// (src/data_io.cpp:613-626).
int Session::write_snapshots(int step)
{
    const Grid &G = m.g;
    const size_t maxn = (size_t)std::max({(long long)G.nx * G.ny, (long long)G.nx * G.nz, (long long)G.ny * G.nz});
    if (!slice_dev_) ALLOC(slice_dev_, float, maxn);
    std::vector<float> host(maxn);
    const std::string out = out_dir();
    auto one = [&](const float *src, int scheme, int axis, int idx, int comp, const std::string &name) -> int {
        const int n0 = axis == 0 ? G.ny : G.nx, n1 = axis == 2 ? G.ny : G.nz;
        CU(launch_pack_slice(src, cjm_, g, axis, idx, comp, scheme, slice_dev_, stream));
        CU(cudaMemcpyAsync(host.data(), slice_dev_, sizeof(float) * n0 * n1, cudaMemcpyDeviceToHost, stream));
        CU(cudaStreamSynchronize(stream));
        const char ax = "XYZ"[axis];
        std::string path = out + "/" + name + "_" + ax + rank_tag(m) + ".bin";
        FILE *fp = std::fopen(path.c_str(), "wb");
        if (!fp) {
            err = "cannot write " + path;
            return ST_IO;
        }
        std::fwrite(host.data(), sizeof(float), (size_t)n0 * n1, fp);
        std::fclose(fp);
        return ST_OK;
    };
    const int idx[3] = {m.p.sliceX + HALO, m.p.sliceY + HALO, m.p.sliceZ + HALO};
    const int lim[3] = {G._nx, G._ny, G._nz};
    const char *comp_name[3] = {"Vx", "Vy", "Vz"};
    const std::string s = std::to_string(step);
    for (int c = 0; c < 3; c++)
        for (int axis = 0; axis < 3; axis++)
            if (idx[axis] >= HALO && idx[axis] < lim[axis]) {
                int st = one(state(), m.p.scheme, axis, idx[axis], c, std::string(comp_name[c]) + "_" + s);
                if (st) return st;
            }
    if (m.p.sliceFreeSurf) {
        for (int c = 0; c < 3; c++) {
            int st = one(state(), m.p.scheme, 2, G._nz - 1, c, std::string("FreeSurf") + comp_name[c] + "_" + s);
            if (st) return st;
        }
        if (dis_) {
            const char *un[3] = {"FreeSurfUx", "FreeSurfUy", "FreeSurfUz"};
            for (int c = 0; c < 3; c++) {
                int st = one(dis_, 0, 2, G._nz - 1, c, std::string(un[c]) + "_" + s);
                if (st) return st;
            }
        }
    }
    return ST_OK;
}

// Model slices (data2D_Model_out, src/data_io.cpp:585-610, written by
// src/run.cpp:70 before the time loop): coordX/Y/Z and Vs/Vp/rho at the
// configured slices, from the host copies of the coordinates and medium.
static int write_model_slices(const Model &m, const std::string &out)
{
    const Grid &G = m.g;
    // global slice index to this part's padded index (src/data_io.cpp:26-60)
    const int idx[3] = {m.p.sliceX + HALO - m.part_lo[0], m.p.sliceY + HALO - m.part_lo[1],
                        m.p.sliceZ + HALO - m.part_lo[2]};
    const int lim[3] = {G._nx, G._ny, G._nz};
    const char *names[6] = {"coordX", "coordY", "coordZ", "Vs", "Vp", "rho"};
    for (int v = 0; v < 6; v++) {
        const FieldVec &src = v < 3 ? m.coord : m.medium;
        if (src.empty() && !(v < 3 && m.coord_lazy)) continue;
        for (int axis = 0; axis < 3; axis++) {
            if (!(idx[axis] >= HALO && idx[axis] < lim[axis])) continue;
            const int n0 = axis == 0 ? G.ny : G.nx, n1 = axis == 2 ? G.ny : G.nz;
            std::vector<float> buf((size_t)n0 * n1);
            for (int a1 = 0; a1 < n1; a1++)
                for (int a0 = 0; a0 < n0; a0++) {
                    int i, j, k;
                    if (axis == 0) i = idx[0], j = a0 + HALO, k = a1 + HALO;
                    else if (axis == 1) i = a0 + HALO, j = idx[1], k = a1 + HALO;
                    else i = a0 + HALO, j = a1 + HALO, k = idx[2];
                    const long long p = ((long long)k * G._ny_ + j) * G._nx_ + i;
                    buf[(size_t)a1 * n0 + a0] = v < 3 ? m.coord_at(i, j, k, v) : src[p * 3 + v % 3];
                }
            std::string path = out + "/" + names[v] + "_" + "XYZ"[axis] + rank_tag(m) + ".bin";
            FILE *fp = std::fopen(path.c_str(), "wb");
            if (!fp) return ST_IO;
            std::fwrite(buf.data(), sizeof(float), buf.size(), fp);
            std::fclose(fp);
        }
    }
    return ST_OK;
}

// The "projection data" of an SRTM90 run (src/terrain.cpp:49-118): longitude,
// latitude and surface height of the interior columns, y outer, as float.
static int write_projection(const Model &m, const std::string &out)
{
    if (!(m.p.useTerrain && m.p.SRTM90 == 1) || m.lon.empty()) return ST_OK;
    const Grid &G = m.g;
    std::vector<float> lon, lat, h;
    for (int j = HALO; j < G._ny; j++)
        for (int i = HALO; i < G._nx; i++) {
            const size_t c = (size_t)i + (size_t)j * G._nx_;
            lon.push_back((float)m.lon[c]);
            lat.push_back((float)m.lat[c]);
            h.push_back(m.terrain[c]);
        }
    const std::pair<const char *, const std::vector<float> *> files[3] = {{"lon", &lon}, {"lat", &lat}, {"terrain", &h}};
    for (auto &f : files) {
        std::string path = out + "/" + f.first + rank_tag(m) + ".bin";
        FILE *fp = std::fopen(path.c_str(), "wb");
        if (!fp) return ST_IO;
        std::fwrite(f.second->data(), sizeof(float), f.second->size(), fp);
        std::fclose(fp);
    }
    return ST_OK;
}

int Session::write_outputs() const
{
    const std::string out = out_dir();
    {
        int st = write_model_slices(m, out);
        if (st) return st;
        if ((st = write_projection(m, out))) return st;
    }
    if (nst > 0) {
        std::vector<float> w((size_t)nst * m.NT * 9);
        int st = get_stations(w.data());
        if (st) return st;
        std::string path = out + "/station" + rank_tag(m) + ".bin";
        FILE *fp = std::fopen(path.c_str(), "wb");
        if (!fp) return ST_IO;
        std::fwrite(m.stations_global.data(), sizeof(int), (size_t)nst * 3, fp);
        std::fwrite(w.data(), sizeof(float), w.size(), fp);
        std::fclose(fp);
    }
    if (m.fs_top) {   // the ranks holding the free surface (src/propagate.cpp:108-118, 347-353)
        std::vector<float> p((size_t)m.g.nx * m.g.ny * pgv_fields());
        int st = get_pgv(p.data());
        if (st) return st;
        std::string path = out + "/PGV_Z" + rank_tag(m) + ".bin";
        FILE *fp = std::fopen(path.c_str(), "wb");
        if (!fp) return ST_IO;
        std::fwrite(p.data(), sizeof(float), p.size(), fp);
        std::fclose(fp);
    }
    return ST_OK;
}

// ------------------------------------------------------ checkpointing
// The state a step depends on: the step counter, the wavefield at the step
// boundary (buffer A; the other buffers are stage temporaries), the PML
// auxiliaries at the step boundary (A of each face), and the running outputs
// (PGV, displacement, station traces recorded so far).  Layout: a header of
// 8 + P int64 (magic, version, scheme, nx, ny, nz, steps done, P, then the
// byte size of each of the P parts listed by ckpt_parts), then the parts.
namespace {
constexpr long long CKPT_MAGIC = 0x314b434d44464743LL;  // "CGFDMCK1"
}

void Session::ckpt_parts(std::vector<std::pair<void *, size_t>> &parts) const
{
    const long long F = g.fstride;
    parts.clear();
    parts.push_back({W_[0], sizeof(float) * F * 9});
    if (m.p.scheme == SCHEME_CGFDM && m.p.pml)
        for (int fc = 0; fc < 5; fc++) parts.push_back({face_[fc].A, sizeof(float) * face_[fc].count * 9});
    parts.push_back({pgv_, sizeof(float) * (size_t)m.g.nx * m.g.ny * 2});
    if (pga_) parts.push_back({pga_, sizeof(float) * (size_t)m.g.nx * m.g.ny * 2});
    if (dis_) parts.push_back({dis_, sizeof(float) * F * 3});
    if (nst > 0) parts.push_back({st_out_, sizeof(float) * (size_t)nst * std::max(m.NT, 1) * 9});
}

size_t Session::checkpoint_bytes() const
{
    std::vector<std::pair<void *, size_t>> parts;
    ckpt_parts(parts);
    size_t n = sizeof(long long) * (8 + parts.size());
    for (auto &p : parts) n += p.second;
    return n;
}

int Session::checkpoint(void *host, size_t bytes)
{
    if (int st = need_fp32_storage("checkpoint")) return st;
    if (bytes < checkpoint_bytes()) {
        err = "checkpoint buffer too small";
        return ST_ARG;
    }
    std::vector<std::pair<void *, size_t>> parts;
    ckpt_parts(parts);
    long long *h = (long long *)host;
    h[0] = CKPT_MAGIC, h[1] = 1, h[2] = m.p.scheme, h[3] = m.g.nx, h[4] = m.g.ny, h[5] = m.g.nz, h[6] = it;
    h[7] = (long long)parts.size();
    for (size_t i = 0; i < parts.size(); i++) h[8 + i] = (long long)parts[i].second;
    char *o = (char *)(h + 8 + parts.size());
    CU(cudaStreamSynchronize(stream));
    for (auto &p : parts) {
        CU(cudaMemcpyAsync(o, p.first, p.second, cudaMemcpyDeviceToHost, stream));
        o += p.second;
    }
    CU(cudaStreamSynchronize(stream));
    return ST_OK;
}

int Session::restore(const void *host, size_t bytes)
{
    if (int st = need_fp32_storage("restore")) return st;
    std::vector<std::pair<void *, size_t>> parts;
    ckpt_parts(parts);
    const long long *h = (const long long *)host;
    if (bytes < sizeof(long long) * 8 || h[0] != CKPT_MAGIC || h[1] != 1) {
        err = "not a checkpoint of this library";
        return ST_ARG;
    }
    if (h[2] != m.p.scheme || h[3] != m.g.nx || h[4] != m.g.ny || h[5] != m.g.nz || h[6] < 0 || h[6] > m.NT ||
        h[7] != (long long)parts.size() || bytes < checkpoint_bytes()) {
        err = "checkpoint does not match this session (scheme, grid, options or NT differ)";
        return ST_ARG;
    }
    for (size_t i = 0; i < parts.size(); i++)
        if (h[8 + i] != (long long)parts[i].second) {
            err = "checkpoint does not match this session (array sizes differ)";
            return ST_ARG;
        }
    const char *o = (const char *)(h + 8 + parts.size());
    CU(cudaStreamSynchronize(stream));
    for (auto &p : parts) {
        CU(cudaMemcpyAsync(p.first, o, p.second, cudaMemcpyHostToDevice, stream));
        o += p.second;
    }
    it = (int)h[6];
    CU(cudaMemcpyAsync(it_dev_, &it, sizeof(int), cudaMemcpyHostToDevice, stream));
    CU(cudaStreamSynchronize(stream));
    return ST_OK;
}

}  // namespace cgfdm
