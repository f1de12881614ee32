// Wavefield health check: the number of non-finite values (NaN, +-Inf) in
// the step-boundary state over the interior points, and the first of them.
// With the run-time key "checkFinite": K, cgfdm_run scans after every K
// steps and stops with CGFDM_E_NONFINITE, so an unstable run (a DT past the
// stability bound of a modified medium, a bad input volume) is reported at
// the step it blew up instead of as NaN traces at the end.  One pass over
// the wavefield, 36 B per point (about 5 ms on 34 M points).
#include <nvtx3/nvToolsExt.h>

#include <string>

#include "device.cuh"
#include "kernels.cuh"
#include "session.hpp"
#include "session_util.hpp"

namespace cgfdm {

namespace {

__global__ void k_count_nonfinite(const float *__restrict__ W, DevGrid g, unsigned long long *count,
                                  unsigned long long *first)
{
    const long long n = (long long)g.nx * g.ny * g.nz;
    unsigned long long c = 0, f = ~0ULL;
    for (long long x = (long long)blockIdx.x * blockDim.x + threadIdx.x; x < n; x += (long long)gridDim.x * blockDim.x) {
        const int i = (int)(x % g.nx), j = (int)((x / g.nx) % g.ny), k = (int)(x / ((long long)g.nx * g.ny));
        const long long q = g.at(i + CGFDM_HALO, j + CGFDM_HALO, k + CGFDM_HALO);
        for (int v = 0; v < 9; v++)
            if (!isfinite(W[v * g.fstride + q])) {
                c++;
                const unsigned long long code = (unsigned long long)x * 9 + v;
                if (code < f) f = code;
            }
    }
    if (c) {
        atomicAdd(count, c);
        atomicMin(first, f);
    }
}

}  // namespace

int Session::check_finite(long long *count, long long *first)
{
    unsigned long long *d = nullptr;
    CU(cudaMallocAsync((void **)&d, 2 * sizeof(unsigned long long), stream));
    const unsigned long long init[2] = {0ULL, ~0ULL};
    CU(cudaMemcpyAsync(d, init, sizeof init, cudaMemcpyHostToDevice, stream));
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    k_count_nonfinite<<<sms * 4, 256, 0, stream>>>(state(), g, d, d + 1);
    CU(cudaGetLastError());
    unsigned long long h[2];
    CU(cudaMemcpyAsync(h, d, sizeof h, cudaMemcpyDeviceToHost, stream));
    CU(cudaFreeAsync(d, stream));
    CU(cudaStreamSynchronize(stream));
    if (count) *count = (long long)h[0];
    if (first) *first = h[0] ? (long long)h[1] : -1;
    return ST_OK;
}

// The steps of cgfdm_run with the scans that "checkFinite" asks for.
int Session::run_checked(int n)
{
    const int K = m.p.check_finite;
    nvtxRangePushA("cgfdm_run");
    const int end = it + n;
    int st = ST_OK;
    while (it < end && st == ST_OK) {
        const int chunk = K > 0 ? std::min(end - it, K - it % K) : end - it;
        if ((st = run_span(chunk))) break;
        if (K > 0 && it % K == 0) {
            long long c = 0, f = -1;
            if ((st = check_finite(&c, &f))) break;
            if (c) {
                const long long x = f / 9;
                err = "non-finite values in the wavefield after step " + std::to_string(it) + ": " +
                      std::to_string(c) + ", the first at interior point (" + std::to_string(x % m.g.nx) + ", " +
                      std::to_string((x / m.g.nx) % m.g.ny) + ", " + std::to_string(x / ((long long)m.g.nx * m.g.ny)) +
                      ") field " + std::to_string(f % 9);
                st = ST_NONFINITE;
            }
        }
    }
    nvtxRangePop();
    return st;
}

}  // namespace cgfdm
