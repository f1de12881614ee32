// Sparse per-step kernels: source injection (finite fault and single point
// sources) and station recording, plus layout conversion for the C ABI.
// All arithmetic here uses explicitly rounded intrinsics in the reference's
// order, so these kernels are bit-exact in every build.
#include "device.cuh"
#include "kernels.cuh"

namespace cgfdm {

__device__ __forceinline__ void decode_ref(long long c, const DevGrid &g, int &i, int &j, int &k)
{
    i = (int)(c % g.nxp);
    j = (int)((c / g.nxp) % g.nyp);
    k = (int)(c / ((long long)g.nxp * g.nyp));
}

// Finite fault: linear interpolation of the moment-rate table at the
// stage-0 time, W[3..8] -= Mdot * DT (src/addMoment.cpp:100-146,191-260,
// 262-377).  SCFDM stores strain, so the moment rate is converted with the
// local compliance first (:217-238).
__global__ void k_fault(float *W, const float *__restrict__ cjm, DevGrid g, FaultDev f, const int *it_dev, float DT,
                        int scheme, float *Walt, unsigned *mx)
{
    const int it = *it_dev;
    if (Walt && (it & 1)) W = Walt;   // mixed storage: this step's state buffer
    const float tmpT = __fmul_rn((float)it + 0.0f, DT);
    const int srcIt = (int)__fdiv_rn(tmpT, f.dt);
    if (srcIt + 1 >= f.nt) return;  // end of table: the reference stops injecting
    const float t1 = __fmul_rn((float)srcIt, f.dt);
    const float tw = __fdiv_rn(__fsub_rn(tmpT, t1), f.dt);
    for (long long p = (long long)blockIdx.x * blockDim.x + threadIdx.x; p < f.npts;
         p += (long long)gridDim.x * blockDim.x) {
        const long long q = f.cell[p];
        const float *r0 = f.rate + ((long long)srcIt * f.npts + p) * 6;
        const float *r1 = f.rate + ((long long)(srcIt + 1) * f.npts + p) * 6;
        float s[6];
        for (int c = 0; c < 6; c++) s[c] = __fadd_rn(__fmul_rn(__fsub_rn(r1[c], r0[c]), tw), r0[c]);
        const long long F = g.fstride;
        if (scheme == 1) {
            const float mu = cjm[C_MU * F + q], lambda = cjm[C_LAMBDA * F + q];
            const float den = __fadd_rn(__fmul_rn(2.0f, __fmul_rn(mu, mu)), __fmul_rn(__fmul_rn(3.0f, lambda), mu));
            const float lm = __fadd_rn(lambda, mu);
            const float den2 = __fmul_rn(2.0f, den);
            float e[6];
            e[0] = __fsub_rn(__fsub_rn(__fdiv_rn(__fmul_rn(s[0], lm), den), __fdiv_rn(__fmul_rn(lambda, s[1]), den2)),
                             __fdiv_rn(__fmul_rn(lambda, s[2]), den2));
            e[1] = __fsub_rn(__fsub_rn(__fdiv_rn(__fmul_rn(s[1], lm), den), __fdiv_rn(__fmul_rn(lambda, s[0]), den2)),
                             __fdiv_rn(__fmul_rn(lambda, s[2]), den2));
            e[2] = __fsub_rn(__fsub_rn(__fdiv_rn(__fmul_rn(s[2], lm), den), __fdiv_rn(__fmul_rn(lambda, s[0]), den2)),
                             __fdiv_rn(__fmul_rn(lambda, s[1]), den2));
            e[3] = __fdiv_rn(s[5], mu);
            e[4] = __fdiv_rn(s[4], mu);
            e[5] = __fdiv_rn(s[3], mu);
            for (int c = 0; c < 6; c++) W[(3 + c) * F + q] = __fsub_rn(W[(3 + c) * F + q], __fmul_rn(e[c], DT));
        } else {
            for (int c = 0; c < 6; c++) {
                const float v = __fsub_rn(W[(3 + c) * F + q], __fmul_rn(s[c], DT));
                W[(3 + c) * F + q] = v;
                if (mx) atomicMax(&mx[(it & 1) * 9 + 3 + c], __float_as_uint(fabsf(v)));
            }
        }
    }
}

// Single point source, 7x7x7 Gaussian-smoothed (src/singleSource.cpp:111-173
// Ricker, explosive; :216-318 double couple).  Cells inside the halo also
// receive the value in the stage buffers (B, C), because the reference's RK
// update keeps halo cells at their step-start value through all stages.
__global__ void k_point(float *W, float *Wb, float *Wc, const float *__restrict__ cjm, DevGrid g, PointDev p,
                        const int *it_dev, float DT, float DH, int scheme, float *Walt, unsigned *mx)
{
    const int t = threadIdx.x;
    if (t >= 343 || !p.inside) return;
    const int it = *it_dev;
    if (Walt) {
        // mixed storage: the state of this step is one of two buffers; halo
        // cells, which no stage updates, get the value in both
        Wb = (it & 1) ? W : Walt;
        W = (it & 1) ? Walt : W;
        Wc = nullptr;
    }
    const int di = t % 7 - 3, dj = (t / 7) % 7 - 3, dk = t / 49 - 3;
    const int i = p.X + di, j = p.Y + dj, k = p.Z + dk;
    const long long F = g.fstride;
    const long long q = g.at(i, j, k);
    const float amp = p.amp[t];
    const float jacb = cjm[C_JAC * F + g.at(p.X, p.Y, p.Z)];
    const float s = p.stf[it];
    const float vol = __fmul_rn(jacb, __fmul_rn(__fmul_rn(DH, DH), DH));
    float add[6] = {0, 0, 0, 0, 0, 0};
    int nc;
    if (p.kind == 1) {
        float value = __fdiv_rn(__fmul_rn(__fmul_rn(-1.0f, s), amp), vol);
        value = (float)__dmul_rn((double)value, __dmul_rn(1.0, (double)DT));  // value *= Cs * DT
        if (scheme == 1) {
            const float mu = cjm[C_MU * F + q], lambda = cjm[C_LAMBDA * F + q];
            value = __fdiv_rn(value, __fadd_rn(__fmul_rn(3.0f, lambda), __fmul_rn(2.0f, mu)));
        }
        add[0] = add[1] = add[2] = value;
        nc = 3;
    } else {
        float rate = __fmul_rn(__fdiv_rn(__fmul_rn(__fmul_rn(-1.0f, s), amp), vol), p.m0);
        rate = (float)__dmul_rn((double)rate, __dmul_rn(1.0, (double)DT));
        float mr[6];
        for (int c = 0; c < 6; c++) mr[c] = __fmul_rn(p.mom[c], rate);
        if (scheme == 1) {
            const float mu = cjm[C_MU * F + q], lambda = cjm[C_LAMBDA * F + q];
            const float den = __fadd_rn(__fmul_rn(2.0f, __fmul_rn(mu, mu)), __fmul_rn(__fmul_rn(3.0f, lambda), mu));
            const float lm = __fadd_rn(lambda, mu), den2 = __fmul_rn(2.0f, den);
            float e[6];
            e[0] = __fsub_rn(__fsub_rn(__fdiv_rn(__fmul_rn(mr[0], lm), den), __fdiv_rn(__fmul_rn(lambda, mr[1]), den2)),
                             __fdiv_rn(__fmul_rn(lambda, mr[2]), den2));
            e[1] = __fsub_rn(__fsub_rn(__fdiv_rn(__fmul_rn(mr[1], lm), den), __fdiv_rn(__fmul_rn(lambda, mr[0]), den2)),
                             __fdiv_rn(__fmul_rn(lambda, mr[2]), den2));
            e[2] = __fsub_rn(__fsub_rn(__fdiv_rn(__fmul_rn(mr[2], lm), den), __fdiv_rn(__fmul_rn(lambda, mr[0]), den2)),
                             __fdiv_rn(__fmul_rn(lambda, mr[1]), den2));
            e[3] = __fdiv_rn(mr[5], mu);
            e[4] = __fdiv_rn(mr[4], mu);
            e[5] = __fdiv_rn(mr[3], mu);
            for (int c = 0; c < 6; c++) mr[c] = e[c];
        }
        for (int c = 0; c < 6; c++) add[c] = -mr[c];
        nc = 6;
    }
    const bool halo = i < CGFDM_HALO || j < CGFDM_HALO || k < CGFDM_HALO || i >= g.nxp - CGFDM_HALO ||
                      j >= g.nyp - CGFDM_HALO || k >= g.nzp - CGFDM_HALO;
    for (int c = 0; c < nc; c++) {
        float v = __fadd_rn(W[(3 + c) * F + q], add[c]);
        W[(3 + c) * F + q] = v;
        if (halo) {
            if (Wb) Wb[(3 + c) * F + q] = v;
            if (Wc) Wc[(3 + c) * F + q] = v;
        } else if (mx) {
            atomicMax(&mx[(it & 1) * 9 + 3 + c], __float_as_uint(fabsf(v)));
        }
    }
}

cudaError_t launch_sources(float *W, const float *cjm, DevGrid g, const FaultDev &f, const PointDev &p,
                           const int *it_dev, float DT, float DH, int scheme, cudaStream_t st, float *Walt,
                           unsigned *mx)
{
    if (f.npts > 0) {
        int nb = (int)std::min<long long>((f.npts + 255) / 256, 1024);
        k_fault<<<nb, 256, 0, st>>>(W, cjm, g, f, it_dev, DT, scheme, Walt, mx);
        CUDA_TRY(cudaGetLastError());
    }
    return cudaSuccess;
}

cudaError_t launch_point(float *W, float *Wb, float *Wc, const float *cjm, DevGrid g, const PointDev &p,
                         const int *it_dev, float DT, float DH, int scheme, cudaStream_t st, float *Walt, unsigned *mx)
{
    if (p.kind == 0 || !p.inside) return cudaSuccess;
    k_point<<<1, 352, 0, st>>>(W, Wb, Wc, cjm, g, p, it_dev, DT, DH, scheme, Walt, mx);
    return cudaGetLastError();
}

// Station traces [station][NT][9] at position it + s * NT
// (src/station.cpp:302-380).  SCFDM records physical values converted from
// the conserved state (:336-365).  One block; thread 0 then advances the
// step counter for the next step's source term.
__global__ void k_stations(const float *__restrict__ W, const float *__restrict__ cjm, DevGrid g,
                           const int *__restrict__ idx, int nst, int NT, float *out, int *it_dev, int scheme,
                           const float *__restrict__ Walt)
{
    const int it = *it_dev;
    if (Walt && ((it + 1) & 1)) W = Walt;   // mixed storage: the state after step it
    const long long F = g.fstride;
    for (int s = threadIdx.x; s < nst; s += blockDim.x) {
        const long long q = g.at(idx[s * 3 + 0], idx[s * 3 + 1], idx[s * 3 + 2]);
        float *o = out + ((long long)it + (long long)s * NT) * 9;
        if (scheme == 1) {
            const float mu = cjm[C_MU * F + q], lambda = cjm[C_LAMBDA * F + q];
            const float buo = __fmul_rn(cjm[C_BUOY * F + q], 1.0f);
            float u[9];
            for (int c = 0; c < 9; c++) u[c] = W[c * F + q];
            const float l2m = __fadd_rn(lambda, __fmul_rn(2.0f, mu));
            o[0] = __fmul_rn(u[0], buo);
            o[1] = __fmul_rn(u[1], buo);
            o[2] = __fmul_rn(u[2], buo);
            o[3] = __fadd_rn(__fadd_rn(__fmul_rn(lambda, u[4]), __fmul_rn(lambda, u[5])), __fmul_rn(u[3], l2m));
            o[4] = __fadd_rn(__fadd_rn(__fmul_rn(lambda, u[3]), __fmul_rn(lambda, u[5])), __fmul_rn(u[4], l2m));
            o[5] = __fadd_rn(__fadd_rn(__fmul_rn(lambda, u[3]), __fmul_rn(lambda, u[4])), __fmul_rn(u[5], l2m));
            o[6] = __fmul_rn(mu, u[8]);
            o[7] = __fmul_rn(mu, u[7]);
            o[8] = __fmul_rn(mu, u[6]);
        } else {
            for (int c = 0; c < 9; c++) o[c] = W[c * F + q];  // * (1/Cv), * (1/Cs) with Cv = Cs = 1
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) *it_dev = it + 1;
}

cudaError_t launch_stations(const float *W, const float *cjm, DevGrid g, const int *st_idx, int nst, int NT,
                            float *out, int *it_dev, int scheme, cudaStream_t st, const float *Walt)
{
    k_stations<<<1, 256, 0, st>>>(W, cjm, g, st_idx, nst, NT, out, it_dev, scheme, Walt);
    return cudaGetLastError();
}

__global__ void k_to_aos(const float *__restrict__ W, int nf, DevGrid g, float *out)
{
    long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long npad = (long long)g.nxp * g.nyp * g.nzp;
    if (n >= npad) return;
    int i = (int)(n % g.nxp), j = (int)((n / g.nxp) % g.nyp), k = (int)(n / ((long long)g.nxp * g.nyp));
    long long q = g.at(i, j, k);
    for (int f = 0; f < nf; f++) out[n * nf + f] = W[f * g.fstride + q];
}

__global__ void k_from_aos(const float *__restrict__ in, int nf, DevGrid g, float *W)
{
    long long n = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    long long npad = (long long)g.nxp * g.nyp * g.nzp;
    if (n >= npad) return;
    int i = (int)(n % g.nxp), j = (int)((n / g.nxp) % g.nyp), k = (int)(n / ((long long)g.nxp * g.nyp));
    long long q = g.at(i, j, k);
    for (int f = 0; f < nf; f++) W[f * g.fstride + q] = in[n * nf + f];
}

// Peak ground acceleration as the reference's SOLVE_PGA build computes it
// (src/PGV.cpp:140-171 with src/propagate.cpp:26-58,188-192): after every
// step with it % 10 == 0, A = (V - V_pre) / (10 DT) for the surface
// velocity V, maxima of |(Ax, Ay)| and |A| kept.  The reference's V_pre copy
// (stroage_W_pre_gpu) moves W_pre[n] = W[n] for the first _nx_ _ny_ _nz_
// floats of the nine-field array only, which never reaches a surface
// point's velocity (at 9 * index + c), so V_pre reads zero there: the value
// is |V| / (10 DT) at every tenth step, kept here bit for bit.
__global__ void k_pga(const float *__restrict__ W, const float *__restrict__ cjm, DevGrid g, const int *it_dev,
                      float DT, int scheme, float *pga)
{
    if (*it_dev % 10 != 0) return;
    const int ii = blockIdx.x * blockDim.x + threadIdx.x, jj = blockIdx.y * blockDim.y + threadIdx.y;
    if (ii >= g.nx || jj >= g.ny) return;
    const long long F = g.fstride;
    const long long q = g.at(ii + CGFDM_HALO, jj + CGFDM_HALO, g.nzp - CGFDM_HALO - 1);
    float V[3];
    for (int c = 0; c < 3; c++) {
        V[c] = W[c * F + q];
        if (scheme == 1) V[c] = __fmul_rn(V[c], __fmul_rn(cjm[C_BUOY * F + q], 1.0f));
    }
    const float d10 = __fmul_rn(10.0f, DT);
    float A[3];
    for (int c = 0; c < 3; c++) A[c] = __fdiv_rn(__fsub_rn(V[c], 0.0f), d10);
    const float h2 = __fadd_rn(__fmul_rn(A[0], A[0]), __fmul_rn(A[1], A[1]));
    const float Ah = __fsqrt_rn(h2), Am = __fsqrt_rn(__fadd_rn(h2, __fmul_rn(A[2], A[2])));
    float *p = pga + ((long long)jj * g.nx + ii) * 2;
    if (p[0] < Ah) p[0] = Ah;
    if (p[1] < Am) p[1] = Am;
}

cudaError_t launch_pga(const float *W, const float *cjm, DevGrid g, const int *it_dev, float DT, int scheme,
                       float *pga, cudaStream_t st)
{
    dim3 b(32, 8), gr((g.nx + 31) / 32, (g.ny + 7) / 8);
    k_pga<<<gr, b, 0, st>>>(W, cjm, g, it_dev, DT, scheme, pga);
    return cudaGetLastError();
}

// One plane of one field for the snapshot files (pack_iodata_x/y/z,
// src/data_io.cpp:96-250): axis 0 is the plane i = idx laid out [nz][ny],
// axis 1 the plane j = idx as [nz][nx], axis 2 the plane k = idx as [ny][nx].
// SCFDM snapshots hold the velocity, momentum times buoyancy
// (src/data_io.cpp:434-483).
__global__ void k_pack_slice(const float *__restrict__ W, int nf, const float *__restrict__ cjm, DevGrid g,
                             int axis, int idx, int comp, int scheme, float *out)
{
    const int a0 = blockIdx.x * blockDim.x + threadIdx.x, a1 = blockIdx.y * blockDim.y + threadIdx.y;
    const int n0 = axis == 0 ? g.ny : g.nx, n1 = axis == 2 ? g.ny : g.nz;
    if (a0 >= n0 || a1 >= n1) return;
    int i, j, k;
    if (axis == 0) i = idx, j = a0 + CGFDM_HALO, k = a1 + CGFDM_HALO;
    else if (axis == 1) i = a0 + CGFDM_HALO, j = idx, k = a1 + CGFDM_HALO;
    else i = a0 + CGFDM_HALO, j = a1 + CGFDM_HALO, k = idx;
    const long long q = g.at(i, j, k);
    float v = W[comp * g.fstride + q];
    if (scheme == 1 && cjm) v = __fmul_rn(v, cjm[C_BUOY * g.fstride + q]);
    out[(long long)a1 * n0 + a0] = v;
    (void)nf;
}

cudaError_t launch_pack_slice(const float *W, const float *cjm, DevGrid g, int axis, int idx, int comp, int scheme,
                              float *out, cudaStream_t st)
{
    const int n0 = axis == 0 ? g.ny : g.nx, n1 = axis == 2 ? g.ny : g.nz;
    dim3 b(32, 8), gr((n0 + 31) / 32, (n1 + 7) / 8);
    k_pack_slice<<<gr, b, 0, st>>>(W, 9, cjm, g, axis, idx, comp, scheme, out);
    return cudaGetLastError();
}

cudaError_t launch_to_aos(const float *W, int nf, DevGrid g, float *out, cudaStream_t st)
{
    long long npad = (long long)g.nxp * g.nyp * g.nzp;
    k_to_aos<<<(unsigned)((npad + 255) / 256), 256, 0, st>>>(W, nf, g, out);
    return cudaGetLastError();
}

cudaError_t launch_from_aos(const float *in, int nf, DevGrid g, float *W, cudaStream_t st)
{
    long long npad = (long long)g.nxp * g.nyp * g.nzp;
    k_from_aos<<<(unsigned)((npad + 255) / 256), 256, 0, st>>>(in, nf, g, W);
    return cudaGetLastError();
}

}  // namespace cgfdm
