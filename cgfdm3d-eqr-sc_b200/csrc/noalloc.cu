// Allocation-free variant of the grid-spacing reduction behind the CFL check.
//
// Some callers cannot call cudaMalloc or cudaFree at the point where they
// need this check.  One example is an application that drives other streams
// of a live simulation, where cudaMalloc and cudaFree can synchronize the
// whole device and stall that work.  Another is an embedder whose own pool
// allocator already holds the device memory, so a library allocation would
// fail.
//
// cgfdm_hrange_noalloc computes the same smallest and largest point-to-plane
// distance as the session set-up (src/calc_CFL.cpp:94-163), without
// allocating anything.  It runs in two passes.  The first writes one (min,
// max) pair per thread block into g_hrange_scratch, a file-scope device
// array of CGFDM_NOALLOC_MAX_BLOCKS pairs (1 MiB).  The second reduces those
// pairs into the caller's output.  Every block overwrites its own pair
// before the second pass reads it, so nothing has to be cleared between
// calls.  The array is shared by all calls on a device and keeps the last
// call's partials: calls that overlap on the GPU (different streams, no
// ordering between them) race on it.
//
// In host code the name g_hrange_scratch only stands for the device
// variable; the device address is looked up with cudaGetSymbolAddress once
// per device, with that device current, on the first call made there, and
// again whenever the device's context has changed since (a cudaDeviceReset
// destroys the context that held the old address).
#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "../../include/cgfdm.h"
#include "device.cuh"

namespace {

constexpr int NOALLOC_MAX_BLOCKS = CGFDM_NOALLOC_MAX_BLOCKS;
constexpr int BX = 32, BY = 8, ZCHUNK = 16;  // one block: 32 x 8 columns, 16 planes

static __device__ __align__(256) double g_hrange_scratch[2 * NOALLOC_MAX_BLOCKS];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;      // guards the per-device address cache
std::mutex g_fn_mu;   // guards the driver entry points
double *g_scratch_addr[MAX_DEVICES] = {};
unsigned long long g_scratch_ctx[MAX_DEVICES] = {};  // context the address belongs to
thread_local std::string g_noalloc_error;

// Point-to-plane distances of one point to the six diagonal-neighbour planes
// (src/calc_CFL.cpp:56-92,123-158), every operation rounded separately.
__device__ void point_range(const float *__restrict__ coord, int nxp, int nyp, int i, int j, int k, double &lo,
                            double &hi)
{
    auto at = [&](int a, int b, int c) { return ((long long)c * nyp + b) * nxp + a; };
    long long p = at(i, j, k) * 3;
    double P[3] = {coord[p], coord[p + 1], coord[p + 2]};
    for (int ii = -1; ii <= 1; ii += 2)
        for (int jj = -1; jj <= 1; jj += 2)
            for (int kk = -1; kk <= 1; kk += 2) {
                long long a = at(i - ii, j, k) * 3, b = at(i, j - jj, k) * 3, c = at(i, j, k - kk) * 3;
                double AB[3], AC[3], PA[3], n[3];
                for (int t = 0; t < 3; t++) {
                    AB[t] = __dsub_rn((double)coord[b + t], (double)coord[a + t]);
                    AC[t] = __dsub_rn((double)coord[c + t], (double)coord[a + t]);
                    PA[t] = __dsub_rn(P[t], (double)coord[a + t]);
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

// Pass 1: block b writes its (min, max) to part[b], part[NOALLOC_MAX_BLOCKS + b].
__global__ void __launch_bounds__(BX *BY) k_hrange_partial(const float *__restrict__ coord, int nx, int ny, int nz,
                                                           double *part)
{
    __shared__ double s_lo[BX * BY], s_hi[BX * BY];
    const int nxp = nx + 2 * CGFDM_HALO, nyp = ny + 2 * CGFDM_HALO;
    const int i = CGFDM_HALO + blockIdx.x * BX + threadIdx.x;
    const int j = CGFDM_HALO + blockIdx.y * BY + threadIdx.y;
    const int k0 = CGFDM_HALO + blockIdx.z * ZCHUNK;
    double lo = 1.0e20, hi = 0.0;
    if (i < nx + CGFDM_HALO && j < ny + CGFDM_HALO)
        for (int k = k0; k < min(k0 + ZCHUNK, nz + CGFDM_HALO); k++) point_range(coord, nxp, nyp, i, j, k, lo, hi);
    const int t = threadIdx.y * BX + threadIdx.x;
    s_lo[t] = lo;
    s_hi[t] = hi;
    __syncthreads();
    for (int w = BX * BY / 2; w > 0; w >>= 1) {
        if (t < w) {
            s_lo[t] = s_lo[t] < s_lo[t + w] ? s_lo[t] : s_lo[t + w];
            s_hi[t] = s_hi[t] > s_hi[t + w] ? s_hi[t] : s_hi[t + w];
        }
        __syncthreads();
    }
    if (t == 0) {
        const int b = (blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x;
        part[b] = s_lo[0];
        part[NOALLOC_MAX_BLOCKS + b] = s_hi[0];
    }
}

// Pass 2: one block reduces nblocks partials into out[0] (min), out[1] (max).
__global__ void __launch_bounds__(1024) k_hrange_final(const double *__restrict__ part, int nblocks, double *out)
{
    __shared__ double s_lo[1024], s_hi[1024];
    double lo = 1.0e20, hi = 0.0;
    for (int b = threadIdx.x; b < nblocks; b += blockDim.x) {
        double l = part[b], h = part[NOALLOC_MAX_BLOCKS + b];
        lo = lo < l ? lo : l;
        hi = hi > h ? hi : h;
    }
    s_lo[threadIdx.x] = lo;
    s_hi[threadIdx.x] = hi;
    __syncthreads();
    for (int w = blockDim.x / 2; w > 0; w >>= 1) {
        if ((int)threadIdx.x < w) {
            s_lo[threadIdx.x] = s_lo[threadIdx.x] < s_lo[threadIdx.x + w] ? s_lo[threadIdx.x] : s_lo[threadIdx.x + w];
            s_hi[threadIdx.x] = s_hi[threadIdx.x] > s_hi[threadIdx.x + w] ? s_hi[threadIdx.x] : s_hi[threadIdx.x + w];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        out[0] = s_lo[0];
        out[1] = s_hi[0];
    }
}

// Unique id of the context current on this thread (cuCtxGetId, through the
// runtime's driver entry points), 0 when none is current yet (the runtime
// binds its primary context on its first real call).  The id of a context
// created after a device reset differs from the old one's.
int current_context_id(unsigned long long *id)
{
    static PFN_cuCtxGetCurrent_v4000 get_current = nullptr;
    static PFN_cuCtxGetId_v12000 get_id = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_fn_mu);
        if (!get_current || !get_id) {
            cudaDriverEntryPointQueryResult q1, q2;
            void *f1 = nullptr, *f2 = nullptr;
            if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f1, cudaEnableDefault, &q1) != cudaSuccess ||
                cudaGetDriverEntryPoint("cuCtxGetId", &f2, cudaEnableDefault, &q2) != cudaSuccess ||
                q1 != cudaDriverEntryPointSuccess || q2 != cudaDriverEntryPointSuccess || !f1 || !f2) {
                g_noalloc_error = "cuCtxGetCurrent / cuCtxGetId not available from the driver";
                return CGFDM_E_CUDA;
            }
            get_current = (PFN_cuCtxGetCurrent_v4000)f1;
            get_id = (PFN_cuCtxGetId_v12000)f2;
        }
    }
    CUcontext c = nullptr;
    unsigned long long v = 0;
    if (get_current(&c) != CUDA_SUCCESS) {
        g_noalloc_error = "cuCtxGetCurrent failed";
        return CGFDM_E_CUDA;
    }
    if (c && get_id(c, &v) != CUDA_SUCCESS) {
        g_noalloc_error = "cuCtxGetId failed";
        return CGFDM_E_CUDA;
    }
    *id = v;
    return CGFDM_OK;
}

// Device address of g_hrange_scratch on the current device, looked up once
// per device and context.
int scratch_for_current_device(double **out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        g_noalloc_error = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
        return CGFDM_E_CUDA;
    }
    if (dev < 0 || dev >= MAX_DEVICES) {
        g_noalloc_error = "device ordinal out of range";
        return CGFDM_E_ARG;
    }
    unsigned long long ctx = 0;
    if (int st = current_context_id(&ctx)) return st;
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_scratch_addr[dev] || ctx == 0 || g_scratch_ctx[dev] != ctx) {
        double *p = nullptr;
        e = cudaGetSymbolAddress((void **)&p, g_hrange_scratch);   // binds the primary context if none is
        if (e != cudaSuccess || !p) {
            g_noalloc_error = std::string("cudaGetSymbolAddress(g_hrange_scratch): ") + cudaGetErrorString(e);
            return CGFDM_E_CUDA;
        }
        if (ctx == 0)
            if (int st = current_context_id(&ctx)) return st;
        g_scratch_addr[dev] = p;
        g_scratch_ctx[dev] = ctx;
    }
    *out = g_scratch_addr[dev];
    return CGFDM_OK;
}

}  // namespace

extern "C" {

int cgfdm_hrange_noalloc(const float *d_coord, int nx, int ny, int nz, double *d_out, void *stream)
{
    if (!d_coord || !d_out || nx <= 0 || ny <= 0 || nz <= 0) {
        g_noalloc_error = "cgfdm_hrange_noalloc: null pointer or non-positive grid size";
        return CGFDM_E_ARG;
    }
    const long long gx = (nx + BX - 1) / BX, gy = (ny + BY - 1) / BY, gz = (nz + ZCHUNK - 1) / ZCHUNK;
    const long long nblocks = gx * gy * gz;
    if (gy > 65535 || gz > 65535) {
        g_noalloc_error = "cgfdm_hrange_noalloc: grid needs " + std::to_string(gy) + " x " + std::to_string(gz) +
                          " thread blocks along y x z; a launch allows at most 65535 each";
        return CGFDM_E_ARG;
    }
    if (nblocks > NOALLOC_MAX_BLOCKS) {
        g_noalloc_error = "cgfdm_hrange_noalloc: grid needs " + std::to_string(nblocks) +
                          " thread blocks of 32x8x16 points; the static scratch holds " +
                          std::to_string(NOALLOC_MAX_BLOCKS) + " (at most " +
                          std::to_string((long long)NOALLOC_MAX_BLOCKS * BX * BY * ZCHUNK) + " points)";
        return CGFDM_E_ARG;
    }
    double *scratch = nullptr;
    int st = scratch_for_current_device(&scratch);
    if (st) return st;
    cudaStream_t s = (cudaStream_t)stream;
    // cudaLaunchKernel returns this launch's own status, not an error an
    // earlier launch of the caller left pending
    int nx_ = nx, ny_ = ny, nz_ = nz, nb = (int)nblocks;
    void *args1[] = {(void *)&d_coord, &nx_, &ny_, &nz_, &scratch};
    cudaError_t e = cudaLaunchKernel((const void *)k_hrange_partial, dim3((unsigned)gx, (unsigned)gy, (unsigned)gz),
                                     dim3(BX, BY, 1), args1, 0, s);
    if (e == cudaSuccess) {
        void *args2[] = {&scratch, &nb, &d_out};
        e = cudaLaunchKernel((const void *)k_hrange_final, dim3(1), dim3(1024), args2, 0, s);
    }
    if (e != cudaSuccess) {
        g_noalloc_error = std::string("cgfdm_hrange_noalloc launch: ") + cudaGetErrorString(e);
        return CGFDM_E_CUDA;
    }
    return CGFDM_OK;
}

const char *cgfdm_noalloc_last_error(void) { return g_noalloc_error.c_str(); }

}  // extern "C"
