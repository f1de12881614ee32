// Stepping a part of a decomposed grid (csrc/partition.cpp) and its halo
// exchange.  A step of a part is five phases -- the source into the
// step-start state, then the four RK stages -- and after each of the first
// four the caller refreshes the halos at internal faces: every part packs
// the three interior layers next to each internal face, the neighbours
// exchange them (device copies between parts on one GPU, NCCL send/recv
// between ranks) and unpack them into the three halo layers on that side.
// Faces are exchanged axis by axis, x then y then z, each over the full
// padded extent of the other two axes, so edge and corner halos are filled
// too.  The same exchange refreshes the metric fields after set-up.
#include <nvtx3/nvToolsExt.h>

#include <algorithm>
#include <cstring>

#include "device.cuh"
#include "kernels.cuh"
#include "session.hpp"
#include "session_util.hpp"

namespace cgfdm {

namespace {

// face f: 0 x-low, 1 x-high, 2 y-low, 3 y-high, 4 z-low, 5 z-high.  send:
// the three interior layers next to the face; otherwise the halo layers.
struct Slab {
    int i0, j0, k0, bx, by, bz;
};

Slab face_slab(const DevGrid &g, int face, bool send)
{
    const int axis = face / 2, hi = face % 2;
    const int n = axis == 0 ? g.nx : axis == 1 ? g.ny : g.nz;
    const int start = send ? (hi ? n : CGFDM_HALO) : (hi ? n + CGFDM_HALO : 0);
    Slab s{0, 0, 0, g.nxp, g.nyp, g.nzp};
    if (axis == 0) s.i0 = start, s.bx = CGFDM_HALO;
    if (axis == 1) s.j0 = start, s.by = CGFDM_HALO;
    if (axis == 2) s.k0 = start, s.bz = CGFDM_HALO;
    return s;
}

// buf[f][k][j][i] over the slab <-> field f of the SoA layout
__global__ void k_halo_copy(float *field, long long fstride, DevGrid g, Slab s, int nf, float *buf, int pack)
{
    const long long per = (long long)s.bx * s.by * s.bz;
    const long long n = per * nf;
    for (long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (long long)gridDim.x * blockDim.x) {
        const int f = (int)(x / per);
        long long r = x - (long long)f * per;
        const int k = (int)(r / ((long long)s.bx * s.by));
        r -= (long long)k * s.bx * s.by;
        const int j = (int)(r / s.bx), i = (int)(r - (long long)j * s.bx);
        const long long q = (long long)f * fstride + g.at(s.i0 + i, s.j0 + j, s.k0 + k);
        if (pack) buf[x] = field[q];
        else field[q] = buf[x];
    }
}

}  // namespace

long long Session::halo_count(int face, int which) const
{
    if (face < 0 || face > 5 || which < 0 || which > 1) return -1;
    const Slab s = face_slab(g, face, true);
    return (long long)s.bx * s.by * s.bz * (which == 0 ? 9 : 13);
}

int Session::halo_copy(int face, int which, float *dev, bool pack)
{
    if (m.p.scheme != SCHEME_CGFDM) {
        err = "halo exchange is built for the CGFDM scheme";
        return ST_OPTIONS;
    }
    if (face < 0 || face > 5 || which < 0 || which > 1 || !dev) {
        err = "bad halo face, field set or buffer";
        return ST_ARG;
    }
    const Slab s = face_slab(g, face, pack);
    const int nf = which == 0 ? 9 : 13;
    float *field = which == 0 ? W_[cur_] : cjm_;
    const long long n = (long long)s.bx * s.by * s.bz * nf;
    const int blocks = (int)std::min<long long>((n + 255) / 256, 4096);
    k_halo_copy<<<blocks, 256, 0, stream>>>(field, g.fstride, g, s, nf, dev, pack ? 1 : 0);
    CU(cudaGetLastError());
    CU(cudaStreamSynchronize(stream));
    return ST_OK;
}

int Session::link_halo_to(int face, float *const nw[3], const DevGrid &ng)
{
    if (int st = need_fp32_storage("link_halo_to")) return st;
    if (face < 0 || face > 5 || m.p.scheme != SCHEME_CGFDM || !nw[0] || !nw[1] || !nw[2]) {
        err = "bad face, scheme or buffers for a halo link";
        return ST_ARG;
    }
    const int axis = face / 2;
    const int n_self = axis == 0 ? g.nx : axis == 1 ? g.ny : g.nz;
    const int n_nbr = axis == 0 ? ng.nx : axis == 1 ? ng.ny : ng.nz;
    // the other two axes must match (a tensor-product decomposition)
    const int os[2] = {axis == 0 ? g.nyp : g.nxp, axis == 2 ? g.nyp : g.nzp};
    const int on[2] = {axis == 0 ? ng.nyp : ng.nxp, axis == 2 ? ng.nyp : ng.nzp};
    if (os[0] != on[0] || os[1] != on[1]) {
        err = "the neighbour's grid does not match on the shared face";
        return ST_ARG;
    }
    static const int wout[4] = {1, 2, 1, 0};   // output buffer of RK stage irk
    for (int irk = 0; irk < 4; irk++) {
        HaloOut &h = ho_[irk][face];
        h.base = nw[wout[irk]];
        h.plane = ng.plane, h.fstride = ng.fstride;
        h.pitch = ng.pitch, h.xoff = ng.xoff;
        // high face: interior n_self..n_self+2 -> neighbour halo 0..2;
        // low face: interior 3..5 -> neighbour halo n_nbr+3..n_nbr+5
        h.shift = (face & 1) ? -n_self : n_nbr;
    }
    halo_out_ = true;
    return build_stage_descs();
}

int Session::link_halo(int face, const Session &nbr)
{
    if (nbr.m.p.scheme != SCHEME_CGFDM) {
        err = "the neighbour is not a CGFDM part";
        return ST_ARG;
    }
    float *const nw[3] = {nbr.W_[0], nbr.W_[1], nbr.W_[2]};
    return link_halo_to(face, nw, nbr.g);
}

// A part's stage buffers for a neighbour in another process: CUDA IPC
// handles of buffers A, B, C and their layout.
struct PartHandle {
    cudaIpcMemHandle_t w[3];
    DevGrid g;
    long long magic;
};
static const long long PART_HANDLE_MAGIC = 0x48545241504d4447LL;

int Session::part_handle(void *out, long long bytes)
{
    if (int st = need_fp32_storage("part_handle")) return st;
    static_assert(sizeof(PartHandle) <= 512, "handle size");
    if (!out || bytes < (long long)sizeof(PartHandle) || m.p.scheme != SCHEME_CGFDM) {
        err = "handle buffer too small or not a CGFDM part";
        return ST_ARG;
    }
    PartHandle h;
    std::memset(&h, 0, sizeof h);
    for (int b = 0; b < 3; b++) CU(cudaIpcGetMemHandle(&h.w[b], W_[b]));
    h.g = g;
    h.magic = PART_HANDLE_MAGIC;
    std::memcpy(out, &h, sizeof h);
    return ST_OK;
}

int Session::link_halo_handle(int face, const void *handle, long long bytes)
{
    PartHandle h;
    if (!handle || bytes < (long long)sizeof h) {
        err = "bad part handle";
        return ST_ARG;
    }
    std::memcpy(&h, handle, sizeof h);
    if (h.magic != PART_HANDLE_MAGIC) {
        err = "bad part handle";
        return ST_ARG;
    }
    CU(cudaSetDevice(device));
    float *nw[3];
    for (int b = 0; b < 3; b++) {
        void *p = nullptr;
        CU(cudaIpcOpenMemHandle(&p, h.w[b], cudaIpcMemLazyEnablePeerAccess));
        ipc_open_.push_back(p);
        nw[b] = (float *)p;
    }
    return link_halo_to(face, nw, h.g);
}

int Session::create_part(const std::string &dir, const std::string &options, const int parts[3],
                         const int coord[3], int dev)
{
    run_dir = dir;
    device = dev;
    Model G;
    int st = build_model(dir, options, G, err);
    if (st) return st;
    materialize_coords(G);   // the part receives its slice of the volume
    if ((st = slice_model(G, parts, coord, m, err))) return st;
    if (m.p.storage != "fp32") {
        err = "a part of a decomposed grid stores its wavefield in FP32";
        return ST_OPTIONS;
    }
    is_part_ = parts[0] * parts[1] * parts[2] > 1;
    part_session_ = true;
    CU(cudaSetDevice(dev));
    arena_session_add(dev);
    counted_ = true;
    CU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    for (auto &e : ev_) CU(cudaEventCreate(&e));
    return setup_device();
}

// One phase of a part's step: 0 the source of step `it` into the step-start
// state A, 1..4 RK stage 0..3 (A -> B -> C -> B -> A); after stage 3 the
// stations record and the step is done.  cur_ names the buffer the phase
// wrote, the one the halo exchange refreshes.
int Session::part_advance(int *phase_done)
{
    if (int st = part_launch(phase_done)) return st;
    return part_finish();
}

int Session::part_finish()
{
    CU(cudaStreamSynchronize(stream));
    return check_device_error();
}

// The launches of the next phase, not waited for (part_finish waits): the
// parts of one GPU then run their phases concurrently.
int Session::part_launch(int *phase_done)
{
    if (m.p.scheme != SCHEME_CGFDM) {
        err = "part stepping is built for the CGFDM scheme";
        return ST_OPTIONS;
    }
    if (it >= m.NT) {
        err = "all steps done";
        return ST_STATE;
    }
    const int ph = phase_;
    static const char *names[5] = {"part: source", "part: stage 0", "part: stage 1", "part: stage 2", "part: stage 3"};
    nvtxRangePushA(names[ph]);
    struct Pop {
        ~Pop() { nvtxRangePop(); }
    } pop;
    if (ph == 0) {
        if (int st = launch_sources_on(stream)) return st;
        cur_ = 0;
    } else {
        const int irk = ph - 1;
        int fb[3];
        fb_signs(it, fb);
        const int sgn = (irk & 1) ? -1 : 1;
        CU(launch_cg_stage(fb[0] * sgn, fb[1] * sgn, fb[2] * sgn, desc_host_[irk], work_dev_, grid_ctas_, stream,
                           halo_out_));
        kernel_launches += 1;
        static const int wout[4] = {1, 2, 1, 0};
        cur_ = wout[irk];
        if (irk == 3) {
            if (int st = launch_pga_on(stream)) return st;
            if (int st = launch_stations_on(stream)) return st;
            it++;
        }
    }
    phase_ = (ph + 1) % 5;
    if (phase_done) *phase_done = ph;
    return ST_OK;
}

}  // namespace cgfdm
