/*
 * CPU restatement of the velocity-stress time-stepping path of
 * CGFDM3D-EQR-SC, both schemes, for use as a test oracle.
 *
 * TEST INFRASTRUCTURE ONLY: the library never links, loads or runs this
 * program; tests, the smoke check and the benchmark's CPU-baseline leg do.
 *
 * Built twice (see Makefile): REAL = float follows the reference's FP32
 * arithmetic operation by operation (including its double-precision
 * promotions), and is checked against the reference's own CPU build; REAL =
 * double runs the same algorithm in FP64 and is the FP64 oracle against
 * which reduced-precision storage is measured.
 *
 * Input: a bundle directory written by oracle/restated.py (see there):
 *   meta.txt        key value lines (grid, DT, DH, NT, scheme, switches, sources)
 *   cjm.bin         metric + medium, float [_nz_][_ny_][_nx_][13 | 19]
 *   rdz.bin         CGFDM free-surface matrices, float [2][_ny_][_nx_][9]
 *   src.bin         finite fault: int64 npts, int64 nt, float dt,
 *                   int64 index[npts], float rate[nt][npts][6] (unscaled)
 *   stations.bin    int32 [n][3] padded-grid indices
 *   perturb.txt     optional, lines "i j k dmu dlambda dbuoyancy": additions
 *                   (in REAL) to the medium of padded-grid point (i, j, k)
 *                   of the CGFDM stencil, the free-surface matrices of a
 *                   perturbed surface point recomputed from it (finite
 *                   differences of the misfit for the adjoint's tests)
 * Output (float32, in the bundle directory):
 *   out_stations.bin [n][NT][9], out_W.bin [_nz_][_ny_][_nx_][9],
 *   out_pgv.bin [ny][nx][2]; the FP64 build also writes
 *   out_stations64.bin [n][NT][9] in float64
 *
 * Layout: the reference's array-of-structures, point (i, j, k) at
 * i + j*_nx_ + k*_nx_*_ny_ (src/axis.h:73), 9 fields per point.
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifndef REAL
#define REAL float
#endif
typedef REAL real;
#define IS_F32 (sizeof(real) == 4)

#define HALO 3
#define REF_PI 3.141592657f /* src/macro.h:72 */

/* float functions where the reference's C++ resolves the float overload */
static real r_sqrt(real x) { return IS_F32 ? (real)sqrtf((float)x) : (real)sqrt((double)x); }
static real r_exp(real x) { return IS_F32 ? (real)expf((float)x) : (real)exp((double)x); }

/* ------------------------------------------------------------ the case */
static int nx, ny, nz, nxp, nyp, nzp, NT, scheme, ncjm;
static int nPML, pml_on, decay_on;
static float DT, DH, rDH;
static int src_kind; /* 0 none, 1 Ricker point, 2 double couple, 3 finite fault */
static int sX, sY, sZ;
static float rickerfc, strike, dip, rake, Mw, duration;
static float vp_max;

static float *CJM;    /* [np][ncjm] */
static float *RDZ;    /* [2][nyp*nxp][9] */
static real *CJMR;    /* CJM in REAL, with the perturbations of perturb.txt */
static real *RDZR;    /* RDZ in REAL, recomputed at perturbed surface cells */
static int nst;
static int *ST;       /* [nst][3] */

static long long np_pad;
#define IDX(i, j, k) ((long long)(i) + (long long)(j) * nxp + (long long)(k) * nxp * nyp)
#define C(idx, f) (CJMR[(idx) * ncjm + (f)])

static real *W, *Wh, *Wt, *Wm; /* state, RHS, RK accumulator, step start */
static real *Ust;              /* stations [nst][NT][9] */
static real *PGV;              /* [ny][nx][2] */

/* ---------------------------------------------------------------- I/O */
static void die(const char *m, const char *a)
{
    fprintf(stderr, "stepper: %s %s\n", m, a ? a : "");
    exit(2);
}

static void *read_file(const char *dir, const char *name, size_t *bytes)
{
    char p[4096];
    snprintf(p, sizeof p, "%s/%s", dir, name);
    FILE *f = fopen(p, "rb");
    if (!f) return NULL;
    fseek(f, 0, SEEK_END);
    long n = ftell(f);
    fseek(f, 0, SEEK_SET);
    void *b = malloc(n > 0 ? n : 1);
    if (n > 0 && fread(b, 1, n, f) != (size_t)n) die("short read", p);
    fclose(f);
    if (bytes) *bytes = n;
    return b;
}

static void write_f32(const char *dir, const char *name, const real *x, long long n)
{
    char p[4096];
    snprintf(p, sizeof p, "%s/%s", dir, name);
    FILE *f = fopen(p, "wb");
    if (!f) die("cannot write", p);
    float buf[4096];
    for (long long o = 0; o < n; o += 4096) {
        long long m = n - o < 4096 ? n - o : 4096;
        for (long long t = 0; t < m; t++) buf[t] = (float)x[o + t];
        fwrite(buf, 4, m, f);
    }
    fclose(f);
}

static void read_meta(const char *dir)
{
    char p[4096], key[128];
    snprintf(p, sizeof p, "%s/meta.txt", dir);
    FILE *f = fopen(p, "r");
    if (!f) die("no meta.txt in", dir);
    double v;
    while (fscanf(f, "%127s %lf", key, &v) == 2) {
#define K(name, var, type) if (!strcmp(key, name)) var = (type)v;
        K("nx", nx, int) K("ny", ny, int) K("nz", nz, int) K("NT", NT, int) K("scheme", scheme, int)
        K("nPML", nPML, int) K("pml", pml_on, int) K("exp_decay", decay_on, int)
        K("DT", DT, float) K("DH", DH, float) K("rDH", rDH, float) K("src_kind", src_kind, int)
        K("sourceX", sX, int) K("sourceY", sY, int) K("sourceZ", sZ, int) K("rickerfc", rickerfc, float)
        K("strike", strike, float) K("dip", dip, float) K("rake", rake, float) K("Mw", Mw, float)
        K("duration", duration, float) K("vp_max", vp_max, float)
#undef K
    }
    fclose(f);
    nxp = nx + 2 * HALO, nyp = ny + 2 * HALO, nzp = nz + 2 * HALO;
    np_pad = (long long)nxp * nyp * nzp;
    ncjm = scheme == 0 ? 13 : 19;
}

/* ===================================================== finite fault
 * src/addMoment.cpp:26-76 (scale by mu / (J DH^3)), 128-142 (linear
 * interpolation in time), 215-262 (addSource1 into W; SCFDM converts the
 * moment rate to a strain rate with the isotropic compliance), 264-321
 * (time of the stage-0 source term and the end of the table).
 */
static long long f_npts, f_nt;
static float f_dt;
static long long *f_idx;
static float *f_rate;

static void fault_scale(void)
{
    for (long long j = 0; j < f_nt; j++)
        for (long long i = 0; i < f_npts; i++) {
            long long idx = f_idx[i];
            float jacb = CJM[idx * ncjm + 9], mu = CJM[idx * ncjm + 10];
            float V = jacb * DH * DH * DH;
            V = (float)(1.0 / V);
            V = (float)(V * 1.0); /* Cv */
            for (int c = 0; c < 6; c++) f_rate[((j * f_npts) + i) * 6 + c] *= mu * V;
        }
}

static void fault_inject(int it)
{
    float tmpT = (it + 0.0f) * DT;
    int srcIt = (int)(tmpT / f_dt);
    if (srcIt + 1 >= f_nt) return;
    float t1 = (float)srcIt * f_dt;
    float tw = (tmpT - t1) / f_dt;
    for (long long i = 0; i < f_npts; i++) {
        long long idx = f_idx[i];
        const float *r0 = f_rate + (srcIt * f_npts + i) * 6, *r1 = f_rate + ((srcIt + 1) * f_npts + i) * 6;
        float s[6];
        for (int c = 0; c < 6; c++) s[c] = (r1[c] - r0[c]) * tw + r0[c];
        real m[6];
        if (scheme == 1) {
            real mu = C(idx, 10), lam = C(idx, 11);
            real den = 2 * (mu * mu) + 3 * lam * mu;
            m[0] = (s[0] * (lam + mu)) / den - (lam * s[1]) / (2 * den) - (lam * s[2]) / (2 * den);
            m[1] = (s[1] * (lam + mu)) / den - (lam * s[0]) / (2 * den) - (lam * s[2]) / (2 * den);
            m[2] = (s[2] * (lam + mu)) / den - (lam * s[0]) / (2 * den) - (lam * s[1]) / (2 * den);
            m[3] = s[5] / mu, m[4] = s[4] / mu, m[5] = s[3] / mu;
        } else {
            for (int c = 0; c < 6; c++) m[c] = s[c];
        }
        for (int c = 0; c < 6; c++) W[idx * 9 + 3 + c] -= m[c] * (real)DT;
    }
}

/* ====================================================== point sources
 * src/singleSource.cpp:25-40 (location), 42-97 (Ricker and Gaussian time
 * functions at the stage-0 time), 111-170 and 195-318 (7x7x7 Gaussian
 * spreading of an explosion or a double couple; SCFDM divides by
 * 3 lambda + 2 mu or applies the compliance), src/macro.h:36-37 (GAUSS_FUN).
 */
static float pt_amp[343];
static float pt_mom[6], pt_m0;

static void point_setup(void)
{
    const int nG = 3;
    float ra = (float)(nG * 0.5);
    int n = 0;
    for (int dk = -nG; dk <= nG; dk++)
        for (int dj = -nG; dj <= nG; dj++)
            for (int di = -nG; di <= nG; di++) {
                int t3[3] = {di, dj, dk};
                float D[3];
                for (int a = 0; a < 3; a++) {
                    double q = (t3[a] - 0.0) / ra;
                    D[a] = (float)(exp(-(q * q)) / (ra * 1.772453850905516));
                }
                float amp = D[0] * D[1] * D[2];
                pt_amp[n++] = (float)(amp / 0.998125703461425);
            }
    if (src_kind == 2) {
        float s = (float)(strike * (3.141592657f / 180.0)), d = (float)(dip * (3.141592657f / 180.0)),
              r = (float)(rake * (3.141592657f / 180.0));
        double sdcr = (double)(sinf(d) * cosf(r));
        float M11 = (float)(-(sdcr * sin(2.0 * s) + sin(2.0 * d) * sinf(r) * sinf(s) * sinf(s)));
        float M22 = (float)(sdcr * sin(2.0 * s) - sin(2.0 * d) * sinf(r) * cosf(s) * cosf(s));
        float M33 = -(M11 + M22);
        float M12 = (float)(sdcr * cos(2.0 * s) + 0.5 * sin(2.0 * d) * sinf(r) * sin(2.0 * s));
        float M13 = (float)(-((double)(cosf(d) * cosf(r) * cosf(s)) + cos(2.0 * d) * sinf(r) * sinf(s)));
        float M23 = (float)(-((double)(cosf(d) * cosf(r) * sinf(s)) - cos(2.0 * d) * sinf(r) * cosf(s)));
        pt_mom[0] = M22, pt_mom[1] = M11, pt_mom[2] = M33, pt_mom[3] = M12, pt_mom[4] = -M23, pt_mom[5] = -M13;
        pt_m0 = (float)(1.5 * powf(10, Mw + 6));
    }
}

static void point_inject(int it)
{
    const int X = sX + HALO, Y = sY + HALO, Z = sZ + HALO;
    if (!(X >= HALO && X < nxp - HALO && Y >= HALO && Y < nyp - HALO && Z >= HALO && Z < nzp - HALO)) return;
    float t = (it + 0.0f) * DT, stf;
    if (src_kind == 1) {
        float tdelay = 1.0f / rickerfc;
        float r = REF_PI * rickerfc * (t - tdelay), rr = r * r;
        stf = (float)(r * (3.0 - 2.0f * rr) * expf(-rr) * sqrtf(REF_PI) * 0.5 * rickerfc * REF_PI);
        stf *= 1e9f;
    } else {
        float tdelay = duration / 2 + 1;
        stf = expf(-(t - tdelay) * (t - tdelay) / (duration * duration)) / (sqrtf(REF_PI) * duration);
    }
    float jacb = CJM[IDX(X, Y, Z) * ncjm + 9];
    int n = 0;
    for (int dk = -3; dk <= 3; dk++)
        for (int dj = -3; dj <= 3; dj++)
            for (int di = -3; di <= 3; di++, n++) {
                long long q = IDX(X + di, Y + dj, Z + dk);
                float vol = jacb * (DH * DH * DH);
                if (src_kind == 1) {
                    float value = -1.0f * stf * pt_amp[n] / vol;
                    value = (float)(value * (1.0 * DT));
                    real v = value;
                    if (scheme == 1) v = v / (3 * C(q, 11) + 2 * C(q, 10));
                    for (int c = 3; c < 6; c++) W[q * 9 + c] = W[q * 9 + c] + v;
                } else {
                    float rate = -1.0f * stf * pt_amp[n] / vol * pt_m0;
                    rate = (float)(rate * (1.0 * DT));
                    real mr[6];
                    for (int c = 0; c < 6; c++) mr[c] = (real)(pt_mom[c] * rate);
                    if (scheme == 1) {
                        real mu = C(q, 10), lam = C(q, 11);
                        real den = 2 * (mu * mu) + 3 * lam * mu, e[6];
                        e[0] = (mr[0] * (lam + mu)) / den - (lam * mr[1]) / (2 * den) - (lam * mr[2]) / (2 * den);
                        e[1] = (mr[1] * (lam + mu)) / den - (lam * mr[0]) / (2 * den) - (lam * mr[2]) / (2 * den);
                        e[2] = (mr[2] * (lam + mu)) / den - (lam * mr[0]) / (2 * den) - (lam * mr[1]) / (2 * den);
                        e[3] = mr[5] / mu, e[4] = mr[4] / mu, e[5] = mr[3] / mu;
                        for (int c = 0; c < 6; c++) mr[c] = e[c];
                    }
                    for (int c = 0; c < 6; c++) W[q * 9 + 3 + c] = W[q * 9 + 3 + c] + (-mr[c]);
                }
            }
}

/* ======================================================== CGFDM pieces */
/* one-sided MacCormack operator (src/macro.h:120-131, src/axis.h:123) */
static const float AF_1 = -0.30874f, AF0 = -0.6326f, AF1 = 1.2330f, AF2 = -0.3334f, AF3 = 0.04168f;
static real Lop(const real *w, long long stride, int FB)
{
    real s = AF_1 * w[-FB * stride] + AF0 * w[0];
    s = s + AF1 * w[FB * stride];
    s = s + AF2 * w[2 * FB * stride];
    s = s + AF3 * w[3 * FB * stride];
    return ((real)FB * s) * (real)rDH;
}

/* contribution of one grid direction with metric row m and the scaled
 * derivatives d (src/wave_deriv.cpp:244-272, src/pml_deriv.cpp:215-227) */
static void dir_rhs(real m0, real m1, real m2, const real d[9], real mu, real lam, real buo, real out[9])
{
    out[0] = ((m0 * d[3] + m1 * d[6]) + m2 * d[7]) * buo;
    out[1] = ((m0 * d[6] + m1 * d[4]) + m2 * d[8]) * buo;
    out[2] = ((m0 * d[7] + m1 * d[8]) + m2 * d[5]) * buo;
    real dv = (m0 * d[0] + m1 * d[1]) + m2 * d[2];
    real m2mu = 2.0f * mu;
    out[3] = dv * lam + m2mu * (m0 * d[0]);
    out[4] = dv * lam + m2mu * (m1 * d[1]);
    out[5] = dv * lam + m2mu * (m2 * d[2]);
    out[6] = (m1 * d[0] + m0 * d[1]) * mu;
    out[7] = (m2 * d[0] + m0 * d[2]) * mu;
    out[8] = (m2 * d[1] + m1 * d[2]) * mu;
}

static real *PA[9];                  /* PML profiles alpha/beta/d for x, y, z */
#define P_ALPHA(a) PA[(a) * 3 + 0]
#define P_BETA(a) PA[(a) * 3 + 1]
#define P_D(a) PA[(a) * 3 + 2]

/* src/init_pml_para.cpp:97-285, single rank (every face is a border) */
static void pml_profiles(void)
{
    const float P_alpha = 1.0f, P_beta = 2.0f, P_d = 2.0f, Cp = 6000.0f, pml_fc = 0.5f;
    float L = DH * (nPML - 1);
    float R = (float)pow(10.0, -(log10((double)nPML) - 1.0) / log10(2.0) - 3.0);
    float d0 = -(P_d + 1.0f) * Cp / (2.0f * L) * logf(R);
    float alpha0 = REF_PI * pml_fc, beta0 = 3.0f;
    const int n_[3] = {nxp, nyp, nzp};
    for (int a = 0; a < 3; a++) {
        const int nn = n_[a], n_in = nn - HALO;
        float *Ls = malloc(sizeof(float) * nn);
        for (int i = 0; i < nn; i++) Ls[i] = -1.0f;
        for (int i = HALO; i < n_in; i++) {
            if (i < HALO + nPML) Ls[i] = (HALO + nPML - 1 - i) * DH;
            if (a < 2 && i >= n_in - nPML) Ls[i] = (i - (n_in - nPML)) * DH;
        }
        for (int q = 0; q < 3; q++) PA[a * 3 + q] = malloc(sizeof(real) * nn);
        for (int i = 0; i < nn; i++) {
            float al = 0.0f, be = 1.0f, dd = 0.0f, l = Ls[i];
            if (i >= HALO && i < n_in && l >= 0.0f) {
                al = alpha0 * (1.0f - powf(l / L, P_alpha));
                be = 1.0f + (beta0 - 1.0f) * powf(l / L, P_beta);
                dd = d0 * powf(l / L, P_d);
            }
            dd /= be;
            be = 1.0f / be;
            P_ALPHA(a)[i] = al, P_BETA(a)[i] = be, P_D(a)[i] = dd;
        }
        free(Ls);
    }
}

/* PML auxiliary state of one face (src/pml_deriv.cpp:44-120): stage value,
 * step start, RK accumulator and RHS for the points of its slab */
typedef struct {
    int dir, hi;                 /* axis; 0 = low face, 1 = high face */
    long long n;
    real *A, *m, *t, *h;
} Face;
static Face FACE[5];             /* x1 y1 z1 x2 y2, the launch order of src/pml_deriv.cpp:633-646 */

static int face_has(const Face *f, int i, int j, int k, long long *pos)
{
    const int c[3] = {i - HALO, j - HALO, k - HALO}, n3[3] = {nx, ny, nz};
    int o = c[f->dir];
    if (!f->hi) {
        if (o >= nPML) return 0;
    } else {
        o -= n3[f->dir] - nPML;
        if (o < 0) return 0;
    }
    int e[3] = {c[0], c[1], c[2]};
    e[f->dir] = o;
    int d[3] = {nx, ny, nz};
    d[f->dir] = nPML;
    *pos = e[0] + (long long)e[1] * d[0] + (long long)e[2] * d[0] * d[1];
    return 1;
}

static void cg_deriv(int FB1, int FB2, int FB3)
{
    const int FB[3] = {FB1, FB2, FB3};
    const long long st[3] = {9, 9LL * nxp, 9LL * nxp * nyp};
    const int _nz = nzp - HALO;
    for (int k = HALO; k < nzp - HALO; k++)
        for (int j = HALO; j < nyp - HALO; j++)
            for (int i = HALO; i < nxp - HALO; i++) {
                const long long q = IDX(i, j, k);
                const real mu = C(q, 10), lam = C(q, 11), buo = C(q, 12) * (real)1.0;
                const real beta[3] = {P_BETA(0)[i], P_BETA(1)[j], P_BETA(2)[k]};
                real h[9];
                if (k < _nz - 3) {
                    /* src/wave_deriv.cpp:214-282 */
                    for (int a = 0; a < 3; a++) {
                        real d[9], c[9];
                        for (int f = 0; f < 9; f++) d[f] = Lop(W + q * 9 + f, st[a], FB[a]) * beta[a];
                        dir_rhs(C(q, 3 * a), C(q, 3 * a + 1), C(q, 3 * a + 2), d, mu, lam, buo, c);
                        for (int f = 0; f < 9; f++) h[f] = a == 0 ? c[f] : h[f] + c[f];
                    }
                    for (int f = 0; f < 9; f++) h[f] = h[f] * (real)DT;
                } else {
                    /* traction image (src/freeSurface.cpp:242-494) */
                    const int ks = (_nz - 1) - k + HALO;
                    real J[3][7][3];
                    for (int a = 0; a < 3; a++)
                        for (int l = 0; l < 7; l++) {
                            long long pos;
                            if (a < 2) pos = q + (long long)(l - HALO) * (st[a] / 9);
                            else if (l < ks) pos = q + (long long)(l - HALO) * (st[2] / 9);
                            else continue;
                            const real m0 = C(pos, 3 * a), m1 = C(pos, 3 * a + 1), m2 = C(pos, 3 * a + 2);
                            const real jac = C(pos, 9);
                            const real *w = W + pos * 9;
                            J[a][l][0] = ((m0 * w[3] + m1 * w[6]) + m2 * w[7]) * jac;
                            J[a][l][1] = ((m0 * w[6] + m1 * w[4]) + m2 * w[8]) * jac;
                            J[a][l][2] = ((m0 * w[7] + m1 * w[8]) + m2 * w[5]) * jac;
                        }
                    for (int c = 0; c < 3; c++) {
                        J[2][ks][c] = 0.0f;
                        for (int l = ks + 1; l <= 2 * HALO; l++) J[2][l][c] = -J[2][2 * ks - l][c];
                    }
                    const real Jinv = 1.0f / C(q, 9);
                    real L3[3][3];
                    for (int a = 0; a < 3; a++)
                        for (int c = 0; c < 3; c++) {
                            real tap[7];
                            for (int l = 0; l < 7; l++) tap[l] = J[a][l][c];
                            L3[a][c] = Lop(tap + 3, 1, FB[a]);
                        }
                    for (int c = 0; c < 3; c++)
                        h[c] = ((buo * Jinv) * ((L3[0][c] * beta[0] + L3[1][c] * beta[1]) + L3[2][c])) * (real)DT;
                    real vxi[3], vet[3], vzt[3];
                    for (int c = 0; c < 3; c++) {
                        vxi[c] = Lop(W + q * 9 + c, st[0], FB1) * beta[0];
                        vet[c] = Lop(W + q * 9 + c, st[1], FB2) * beta[1];
                    }
                    if (k == _nz - 1) {
                        const long long s = (long long)j * nxp + i;
                        const real *dx = RDZR + s * 9, *dy = RDZR + ((long long)nxp * nyp + s) * 9;
                        for (int r = 0; r < 3; r++)
                            vzt[r] = ((dx[r * 3] * vxi[0] + dx[r * 3 + 1] * vxi[1]) + dx[r * 3 + 2] * vxi[2]) +
                                     ((dy[r * 3] * vet[0] + dy[r * 3 + 1] * vet[1]) + dy[r * 3 + 2] * vet[2]);
                    } else if (k == _nz - 2) {
                        for (int c = 0; c < 3; c++)
                            vzt[c] = ((real)FB3 * (W[(q + FB3 * st[2] / 9) * 9 + c] - W[q * 9 + c])) * (real)rDH;
                    } else {
                        for (int c = 0; c < 3; c++)
                            vzt[c] = ((real)FB3 * ((-1.16666667f * W[q * 9 + c] + 1.33333333f * W[(q + FB3 * st[2] / 9) * 9 + c]) +
                                                   -0.16666667f * W[(q + 2 * FB3 * st[2] / 9) * 9 + c])) *
                                     (real)rDH;
                    }
                    real s3[3][9];
                    const real *vv[3] = {vxi, vet, vzt};
                    for (int a = 0; a < 3; a++) {
                        real d[9] = {vv[a][0], vv[a][1], vv[a][2], 0, 0, 0, 0, 0, 0};
                        dir_rhs(C(q, 3 * a), C(q, 3 * a + 1), C(q, 3 * a + 2), d, mu, lam, buo, s3[a]);
                    }
                    for (int f = 3; f < 9; f++) h[f] = ((s3[0][f] + s3[1][f]) + s3[2][f]) * (real)DT;
                }
                /* CFS-PML (src/pml_deriv.cpp:125-584; free-surface term
                 * src/pml_freeSurface.cpp:16-242), faces in launch order */
                if (pml_on)
                    for (int fc = 0; fc < 5; fc++) {
                        Face *F = &FACE[fc];
                        long long pos;
                        if (!face_has(F, i, j, k, &pos)) continue;
                        const int a = F->dir, ix = a == 0 ? i : a == 1 ? j : k;
                        const real dval = P_D(a)[ix], be = P_BETA(a)[ix], ad = dval + P_ALPHA(a)[ix];
                        real d[9], rhs[9];
                        for (int f = 0; f < 9; f++) d[f] = Lop(W + q * 9 + f, st[a], FB[a]) * dval;
                        dir_rhs(C(q, 3 * a), C(q, 3 * a + 1), C(q, 3 * a + 2), d, mu, lam, buo, rhs);
                        real *aux = F->A + pos * 9, *hA = F->h + pos * 9;
                        for (int f = 0; f < 9; f++) hA[f] = (rhs[f] - ad * aux[f]) * (real)DT;
                        if (k == _nz - 1 && a < 2) {
                            const long long s = (long long)j * nxp + i;
                            const real *mr = RDZR + ((long long)a * nxp * nyp + s) * 9;
                            real vz[9] = {0}, t3[9];
                            for (int r = 0; r < 3; r++) vz[r] = (mr[r * 3] * d[0] + mr[r * 3 + 1] * d[1]) + mr[r * 3 + 2] * d[2];
                            dir_rhs(C(q, 6), C(q, 7), C(q, 8), vz, mu, lam, buo, t3);
                            for (int f = 3; f < 9; f++) hA[f] = hA[f] + t3[f] * (real)DT;
                        }
                        for (int f = 0; f < 9; f++) h[f] = h[f] + (-be * aux[f]) * (real)DT;
                    }
                for (int f = 0; f < 9; f++) Wh[q * 9 + f] = h[f];
            }
}

/* RK4 of the wavefield over every point (src/wave_rk.cpp:17-104; halo
 * points have a zero RHS) and of the PML auxiliaries (src/pml_rk.cpp:18-73) */
/* Mixed-precision storage (MIX16, REAL = float): the oracle of the
 * library's "storage": "fp16" CGFDM path.  The step-start state m stays
 * FP32; each stage's delta from it (d1 = a2 h0, d2 = a3 h1, d3 = h2) and the
 * RK accumulator's delta (t - m) are stored as FP16 values times a per-field
 * power-of-two scale, and the next stage's stencil input is m + d as
 * reconstructed from the stored value.  The accumulator after stage 0 is
 * b1 h0 = d1 / 3, formed from the stored d1 in stage 1.  The scale of field
 * f makes the bound M_f of its values at the step start map below 2^13:
 * M_f = max(max |m_f|, coupled) over the interior, where the coupled bound
 * is the stress maximum over the smallest S impedance for a velocity field
 * and the velocity maximum times the largest P impedance for a stress
 * field (a stage's delta can be non-zero where m_f still is, e.g. velocity
 * next to a stress source at step 0).  The PML auxiliaries stay FP32. */
#ifdef MIX16
static float *S16, *T16;            /* stored deltas, as the values they stand for */
static float mscale[9], minv[9];
static float Zs_min, Zp_max;        /* impedance bounds of the medium */
static double Mpre[9];              /* max |m_f| before the step's source term */

static float q16(float x, int f)
{
    float y = x * mscale[f];
    if (y > 65504.0f) y = 65504.0f;
    if (y < -65504.0f) y = -65504.0f;
    return (float)(_Float16)y * minv[f];
}

static void interior_max(double *M)
{
    for (int f = 0; f < 9; f++) M[f] = 0.0;
    for (int k = HALO; k < nzp - HALO; k++)
        for (int j = HALO; j < nyp - HALO; j++)
            for (int i = HALO; i < nxp - HALO; i++)
                for (int f = 0; f < 9; f++) {
                    const double a = fabs((double)W[IDX(i, j, k) * 9 + f]);
                    if (a > M[f]) M[f] = a;
                }
}

static void mix_setup(void)
{
    Zs_min = 3.4e38f, Zp_max = 0.0f;
    for (int k = HALO; k < nzp - HALO; k++)
        for (int j = HALO; j < nyp - HALO; j++)
            for (int i = HALO; i < nxp - HALO; i++) {
                const long long q = IDX(i, j, k);
                const float mu = CJM[q * ncjm + 10], lam = CJM[q * ncjm + 11], b = CJM[q * ncjm + 12];
                const float zs = sqrtf(mu / b), zp = sqrtf((lam + 2.0f * mu) / b);
                if (zs < Zs_min) Zs_min = zs;
                if (zp > Zp_max) Zp_max = zp;
            }
    S16 = calloc(np_pad * 9, sizeof(float));
    T16 = calloc(np_pad * 9, sizeof(float));
}

/* after the source term of a step: the scales of that step */
static void mix_scales(void)
{
    double Mpost[9];
    interior_max(Mpost);
    float M[9], Mv = 0.0f, Ms = 0.0f;
    for (int f = 0; f < 9; f++) {
        M[f] = (float)(Mpre[f] > Mpost[f] ? Mpre[f] : Mpost[f]);
        if (f < 3 && M[f] > Mv) Mv = M[f];
        if (f >= 3 && M[f] > Ms) Ms = M[f];
    }
    for (int f = 0; f < 9; f++) {
        const float c = f < 3 ? Ms / Zs_min : Mv * Zp_max;
        const float b = M[f] > c ? M[f] : c;
        int e = 0;
        if (b > 0.0f) frexpf(b, &e);      /* 2^(e-1) <= b < 2^e */
        mscale[f] = b > 0.0f ? ldexpf(1.0f, 13 - e) : 1.0f;
        minv[f] = b > 0.0f ? ldexpf(1.0f, e - 13) : 1.0f;
    }
}
#endif

static void rk4(int irk)
{
    const float b1 = 0.16666667f, b2 = 0.33333333f, b3 = 0.33333333f, b4 = 0.16666667f, a2 = 0.5f, a3 = 0.5f;
    for (long long n = 0; n < np_pad * 9; n++) {
        real h = Wh[n];
#ifdef MIX16
        const int f = (int)(n % 9);
        if (irk == 0) Wm[n] = W[n], S16[n] = q16(a2 * h, f), W[n] = Wm[n] + S16[n];
        else if (irk == 1) T16[n] = q16(S16[n] * 0.33333334f + b2 * h, f), S16[n] = q16(a3 * h, f), W[n] = Wm[n] + S16[n];
        else if (irk == 2) T16[n] = q16(T16[n] + b3 * h, f), S16[n] = q16(h, f), W[n] = Wm[n] + S16[n];
        else W[n] = Wm[n] + (T16[n] + b4 * h);
#else
        if (irk == 0) Wm[n] = W[n], Wt[n] = Wm[n] + b1 * h, W[n] = Wm[n] + a2 * h;
        else if (irk == 1) Wt[n] = Wt[n] + b2 * h, W[n] = Wm[n] + a3 * h;
        else if (irk == 2) Wt[n] = Wt[n] + b3 * h, W[n] = Wm[n] + h;
        else W[n] = Wt[n] + b4 * h;
#endif
    }
    if (pml_on)
        for (int fc = 0; fc < 5; fc++) {
            Face *F = &FACE[fc];
            for (long long n = 0; n < F->n * 9; n++) {
                real h = F->h[n];
                if (irk == 0) F->m[n] = F->A[n], F->t[n] = F->m[n] + b1 * h, F->A[n] = F->m[n] + a2 * h;
                else if (irk == 1) F->t[n] = F->t[n] + b2 * h, F->A[n] = F->m[n] + a3 * h;
                else if (irk == 2) F->t[n] = F->t[n] + b3 * h, F->A[n] = F->m[n] + h;
                else F->A[n] = F->t[n] + b4 * h;
            }
        }
}

/* ======================================================== SCFDM pieces */
/* WENO5-JS, src/alternative_flux_FD.cpp:42-59 */
static real weno5(real u1, real u2, real u3, real u4, real u5)
{
    real b1 = 0.3333333333f * (10 * u3 * u3 - 31 * u3 * u4 + 25 * u4 * u4 + 11 * u3 * u5 - 19 * u4 * u5 + 4 * u5 * u5);
    real b2 = 0.3333333333f * (4 * u2 * u2 - 13 * u2 * u3 + 13 * u3 * u3 + 5 * u2 * u4 - 13 * u3 * u4 + 4 * u4 * u4);
    real b3 = 0.3333333333f * (4 * u1 * u1 - 19 * u1 * u2 + 25 * u2 * u2 + 11 * u1 * u3 - 31 * u2 * u3 + 10 * u3 * u3);
    b1 = (real)(0.3125f / ((b1 + 1e-6) * (b1 + 1e-6)));
    b2 = (real)(0.625f / ((b2 + 1e-6) * (b2 + 1e-6)));
    b3 = (real)(0.0625f / ((b3 + 1e-6) * (b3 + 1e-6)));
    real tw = 1.0f / (b1 + b2 + b3);
    return (b1 * tw) * (0.375f * u3 + 0.75f * u4 - 0.125f * u5) + (b2 * tw) * (-0.125f * u2 + 0.75f * u3 + 0.375f * u4) +
           (b3 * tw) * (0.375f * u1 - 1.25f * u2 + 1.875f * u3);
}

/* physical flux along a metric row (src/alternative_flux_FD.cpp:146-154) */
static void pflux(real n0, real n1, real n2, real lam, real mu, real b, const real *u, real *f)
{
    f[0] = -(n0 * (lam * u[4] + lam * u[5] + u[3] * (lam + 2 * mu)) + mu * n1 * u[8] + mu * n2 * u[7]);
    f[1] = -(n1 * (lam * u[3] + lam * u[5] + u[4] * (lam + 2 * mu)) + mu * n0 * u[8] + mu * n2 * u[6]);
    f[2] = -(n2 * (lam * u[3] + lam * u[4] + u[5] * (lam + 2 * mu)) + mu * n0 * u[7] + mu * n1 * u[6]);
    f[3] = -((n0 * u[0]) * b);
    f[4] = -((n1 * u[1]) * b);
    f[5] = -((n2 * u[2]) * b);
    f[6] = -((n1 * u[2]) * b + (n2 * u[1]) * b);
    f[7] = -((n0 * u[2]) * b + (n2 * u[0]) * b);
    f[8] = -((n0 * u[1]) * b + (n1 * u[0]) * b);
}

static real *RF; /* Riemann flux, [np][9], zero where never written */

/* flux of direction a at faces i+1/2 stored at i (src/alternative_flux_FD.cpp:61-399) */
static void sc_flux(int a)
{
    const long long s = a == 0 ? 1 : a == 1 ? nxp : (long long)nxp * nyp;
    const int lo[3] = {HALO - (a == 0), HALO - (a == 1), HALO - (a == 2)};
    for (int k = lo[2]; k < nzp - HALO; k++)
        for (int j = lo[1]; j < nyp - HALO; j++)
            for (int i = lo[0]; i < nxp - HALO; i++) {
                const long long q = IDX(i, j, k);
                const real n0 = C(q, 3 * a), n1 = C(q, 3 * a + 1), n2 = C(q, 3 * a + 2);
                const real mu = C(q, 10), lam = C(q, 11), b = C(q, 12);
                real un[9], up[9], fn[9], fp[9];
                for (int v = 0; v < 9; v++) {
                    const real *w = W + v;
                    un[v] = weno5(w[(q - 2 * s) * 9], w[(q - s) * 9], w[q * 9], w[(q + s) * 9], w[(q + 2 * s) * 9]);
                    up[v] = weno5(w[(q + 3 * s) * 9], w[(q + 2 * s) * 9], w[(q + s) * 9], w[q * 9], w[(q - s) * 9]);
                }
                pflux(n0, n1, n2, lam, mu, b, un, fn);
                pflux(n0, n1, n2, lam, mu, b, up, fp);
                for (int v = 0; v < 9; v++) RF[q * 9 + v] = 0.5f * (fp[v] + fn[v] - (real)vp_max * (up[v] - un[v]));
            }
}

#define O2(u1, u2, u3, u4, u5) (1.0f / 12 * (-(u1) + 16 * (u2) - 30 * (u3) + 16 * (u4) - (u5)))
#define O4(u1, u2, u3, u4, u5) (((u1) - 4 * (u2) + 6 * (u3) - 4 * (u4) + (u5)))
#define O2F(u1, u2, u3, u4, u5, u6) (1.0f / 48 * (-5 * (u1) + 39 * (u2) - 34 * (u3) - 34 * (u4) + 39 * (u5) - 5 * (u6)))
#define O4F(u1, u2, u3, u4, u5, u6) (1.0f / 2 * ((u1) - 3 * (u2) + 2 * (u3) + 2 * (u4) - 3 * (u5) + (u6)))

/* flux difference of direction a (src/alternative_flux_FD.cpp:1215-1435) */
static void sc_du(int a)
{
    const long long s = a == 0 ? 1 : a == 1 ? nxp : (long long)nxp * nyp;
    const int _nz = nzp - HALO;
    for (int k = HALO; k < nzp - HALO; k++)
        for (int j = HALO; j < nyp - HALO; j++)
            for (int i = HALO; i < nxp - HALO; i++) {
                const long long q = IDX(i, j, k);
                const real jac = (real)(1.0 / CJM[q * ncjm + 9]);
                const real coef = (real)DT * (real)rDH * jac;
                real hu[7][9];
                const int surf = k >= _nz - 3;
                if (surf)
                    for (int n = 0; n < 7; n++) {
                        long long p = q + (n - 3) * s;
                        pflux(C(p, 3 * a), C(p, 3 * a + 1), C(p, 3 * a + 2), C(p, 11), C(p, 10), C(p, 12), W + p * 9, hu[n]);
                    }
                for (int v = 0; v < 9; v++) {
                    const real *F = RF + v;
                    real val;
                    if (surf) {
                        val = coef * (-((F[q * 9] - 1.0f / 24 * O2F(hu[1][v], hu[2][v], hu[3][v], hu[4][v], hu[5][v], hu[6][v]) +
                                         7.0f / 5760 * O4F(hu[1][v], hu[2][v], hu[3][v], hu[4][v], hu[5][v], hu[6][v])) -
                                        (F[(q - s) * 9] - 1.0f / 24 * O2F(hu[0][v], hu[1][v], hu[2][v], hu[3][v], hu[4][v], hu[5][v]) +
                                         7.0f / 5760 * O4F(hu[0][v], hu[1][v], hu[2][v], hu[3][v], hu[4][v], hu[5][v]))));
                    } else {
                        real f3 = F[(q - 3 * s) * 9], f2 = F[(q - 2 * s) * 9], f1 = F[(q - s) * 9], f0 = F[q * 9],
                             g1 = F[(q + s) * 9], g2 = F[(q + 2 * s) * 9];
                        val = coef * (-((f0 - 1.0f / 24 * O2(f2, f1, f0, g1, g2) + 7.0f / 5760 * O4(f2, f1, f0, g1, g2)) -
                                        (f1 - 1.0f / 24 * O2(f3, f2, f1, f0, g1) + 7.0f / 5760 * O4(f3, f2, f1, f0, g1))));
                    }
                    Wh[q * 9 + v] = a == 0 ? val : Wh[q * 9 + v] + val;
                }
            }
}

/* TVD-RK3 over every point (src/wave_rk_tvd.cpp:17-78) */
static void tvd(int irk)
{
    for (long long n = 0; n < np_pad * 9; n++) {
        real h = Wh[n];
        if (irk == 0) Wm[n] = W[n], W[n] = Wm[n] + h;
        else if (irk == 1) W[n] = (real)(0.75 * Wm[n] + 0.25 * W[n] + 0.25 * h);
        else W[n] = (real)((1.0 / 3.0) * Wm[n] + (2.0 / 3.0) * W[n] + (2.0 / 3.0) * h);
    }
}

/* characteristic free surface (src/freeSurface.cpp:40-194): the stress and
 * velocity in the basin (n, s, t) of the surface normal and the two grid
 * tangents, T = B^-1 sigma B^-T, v' = B^-1 v; the condition; then back,
 * sigma = B T B^T, v = B v'.  Evaluated in double, stored in REAL. */
static void char_fs(void)
{
    const int k = nzp - HALO - 1;
    for (int j = HALO; j < nyp - HALO; j++)
        for (int i = HALO; i < nxp - HALO; i++) {
            const long long q = IDX(i, j, k);
            const float mu = CJM[q * ncjm + 10], lam = CJM[q * ncjm + 11], buo = CJM[q * ncjm + 12];
            const float rho = 1.0f / buo, vs = sqrtf(mu * buo), vp = sqrtf((lam + 2 * mu) * buo);
            const double jac = CJM[q * ncjm + 9];
            double n[3] = {CJM[q * ncjm + 6] / jac, CJM[q * ncjm + 7] / jac, CJM[q * ncjm + 8] / jac};
            double sv[3] = {CJM[q * ncjm + 13], CJM[q * ncjm + 14], CJM[q * ncjm + 15]};
            double tv[3] = {CJM[q * ncjm + 16], CJM[q * ncjm + 17], CJM[q * ncjm + 18]};
            double *bs[3] = {n, sv, tv};
            for (int a = 0; a < 3; a++) {
                double r = 1.0 / sqrt(bs[a][0] * bs[a][0] + bs[a][1] * bs[a][1] + bs[a][2] * bs[a][2]);
                for (int c = 0; c < 3; c++) bs[a][c] *= r;
            }
            double R[3][3];
            const double *x, *y;
            for (int a = 0; a < 3; a++) {
                x = bs[(a + 1) % 3], y = bs[(a + 2) % 3];
                R[a][0] = x[1] * y[2] - x[2] * y[1];
                R[a][1] = x[2] * y[0] - x[0] * y[2];
                R[a][2] = x[0] * y[1] - x[1] * y[0];
            }
            const double det = n[0] * R[0][0] + n[1] * R[0][1] + n[2] * R[0][2];
            for (int a = 0; a < 3; a++)
                for (int c = 0; c < 3; c++) R[a][c] /= det;
            double u[9];
            for (int v = 0; v < 9; v++) u[v] = W[q * 9 + v];
            const double L = lam, M = mu, tr = u[3] + u[4] + u[5];
            double S[3][3] = {{L * tr + 2 * M * u[3], M * u[8], M * u[7]},
                              {M * u[8], L * tr + 2 * M * u[4], M * u[6]},
                              {M * u[7], M * u[6], L * tr + 2 * M * u[5]}};
            double vel[3] = {u[0] * buo, u[1] * buo, u[2] * buo};
            double RS[3][3], T[3][3], vb[3];
            for (int a = 0; a < 3; a++)
                for (int c = 0; c < 3; c++) RS[a][c] = R[a][0] * S[0][c] + R[a][1] * S[1][c] + R[a][2] * S[2][c];
            for (int a = 0; a < 3; a++)
                for (int c = 0; c < 3; c++) T[a][c] = RS[a][0] * R[c][0] + RS[a][1] * R[c][1] + RS[a][2] * R[c][2];
            for (int a = 0; a < 3; a++) vb[a] = R[a][0] * vel[0] + R[a][1] * vel[1] + R[a][2] * vel[2];
            const double ratio = L / (L + 2 * M);
            T[1][1] -= T[0][0] * ratio;
            T[2][2] -= T[0][0] * ratio;
            vb[1] -= T[0][1] / ((double)vs * rho);
            vb[2] -= T[0][2] / ((double)vs * rho);
            vb[0] -= T[0][0] / ((double)vp * rho);
            T[0][0] = T[0][1] = T[1][0] = T[0][2] = T[2][0] = 0.0;
            const double B[3][3] = {{n[0], sv[0], tv[0]}, {n[1], sv[1], tv[1]}, {n[2], sv[2], tv[2]}};
            double BT[3][3], Sg[3][3], v2[3];
            for (int a = 0; a < 3; a++)
                for (int c = 0; c < 3; c++) BT[a][c] = B[a][0] * T[0][c] + B[a][1] * T[1][c] + B[a][2] * T[2][c];
            for (int a = 0; a < 3; a++)
                for (int c = 0; c < 3; c++) Sg[a][c] = BT[a][0] * B[c][0] + BT[a][1] * B[c][1] + BT[a][2] * B[c][2];
            for (int a = 0; a < 3; a++) v2[a] = B[a][0] * vb[0] + B[a][1] * vb[1] + B[a][2] * vb[2];
            const double comp = 1.0 / (2 * M * (3 * L + 2 * M)), strace = Sg[0][0] + Sg[1][1] + Sg[2][2];
            double o[9];
            for (int a = 0; a < 3; a++) o[a] = v2[a] * rho;
            for (int a = 0; a < 3; a++) o[3 + a] = (2 * (L + M) * Sg[a][a] - L * (strace - Sg[a][a])) * comp;
            o[6] = Sg[1][2] / M, o[7] = Sg[0][2] / M, o[8] = Sg[0][1] / M;
            for (int v = 0; v < 9; v++) W[q * 9 + v] = (real)o[v];
            /* cubic extrapolation into the halo, src/freeSurface.cpp:180-190 */
            const long long P = (long long)nxp * nyp * 9;
            for (int v = 0; v < 9; v++)
                for (int hh = 1; hh <= HALO; hh++) {
                    real *c = W + q * 9 + v;
                    c[hh * P] = 4.0f * c[(hh - 1) * P] - 6.0f * c[(hh - 2) * P] + 4.0f * c[(hh - 3) * P] - c[(hh - 4) * P];
                }
        }
}

/* exponential sponge, src/exp_decay_absorb.cpp:19-145 (free surface on) */
static void exp_decay(void)
{
    const int nl = 20;
    const float alpha = (float)0.015;
    real G[21];
    for (int p = 0; p <= nl; p++) {
        float x = alpha * (float)p;
        G[p] = r_exp((real)(-x * x));
    }
    for (int k = HALO; k < nzp - HALO; k++)
        for (int j = HALO; j < nyp - HALO; j++)
            for (int i = HALO; i < nxp - HALO; i++) {
                const int X = i - HALO, Y = j - HALO, Z = k - HALO;
                real g[5];
                int ng = 0;
                if (X <= nl) g[ng++] = G[nl - X];
                if (X >= nx - nl) g[ng++] = G[nl - (nx - X)];
                if (Y <= nl) g[ng++] = G[nl - Y];
                if (Y >= ny - nl) g[ng++] = G[nl - (ny - Y)];
                if (Z <= nl) g[ng++] = G[nl - Z];
                for (int a = 0; a < ng; a++)
                    for (int v = 0; v < 9; v++) W[IDX(i, j, k) * 9 + v] *= g[a];
            }
}

/* ============================================== stations and peak velocity */
/* src/station.cpp:302-380 (SCFDM: physical values from the conserved state) */
static void record(int it)
{
    for (int s = 0; s < nst; s++) {
        const long long q = IDX(ST[s * 3], ST[s * 3 + 1], ST[s * 3 + 2]);
        real *o = Ust + ((long long)s * NT + it) * 9;
        const real *u = W + q * 9;
        if (scheme == 1) {
            const real mu = C(q, 10), lam = C(q, 11), b = C(q, 12) * (real)1.0;
            o[0] = u[0] * b, o[1] = u[1] * b, o[2] = u[2] * b;
            o[3] = lam * u[4] + lam * u[5] + u[3] * (lam + 2 * mu);
            o[4] = lam * u[3] + lam * u[5] + u[4] * (lam + 2 * mu);
            o[5] = lam * u[3] + lam * u[4] + u[5] * (lam + 2 * mu);
            o[6] = mu * u[8], o[7] = mu * u[7], o[8] = mu * u[6];
        } else {
            for (int v = 0; v < 9; v++) o[v] = (real)(u[v] * 1.0);
        }
    }
}

/* src/PGV.cpp:61-175 */
static void pgv_update(void)
{
    const int k = nzp - HALO - 1;
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            const long long q = IDX(i + HALO, j + HALO, k);
            real b = scheme == 1 ? C(q, 12) : (real)1.0;
            real Vx = (real)(W[q * 9] * 1.0 * b), Vy = (real)(W[q * 9 + 1] * 1.0 * b), Vz = (real)(W[q * 9 + 2] * 1.0 * b);
            real Vh = r_sqrt(Vx * Vx + Vy * Vy), V = r_sqrt(Vx * Vx + Vy * Vy + Vz * Vz);
            real *p = PGV + ((long long)j * nx + i) * 2;
            if (p[0] < Vh) p[0] = Vh;
            if (p[1] < V) p[1] = V;
        }
}

/* ======================================================= perturbations
 * The traction-free zeta derivative at the surface (src/contravariant.cpp:
 * 365-461): V_zeta = rx V_xi + ry V_eta with rx = -DZ^-1 DX, ry = -DZ^-1 DY,
 * DZ, DX, DY the 3x3 blocks of the surface traction from the zeta, xi and
 * eta velocity derivatives.  m: xi_x .. zt_z at the point.
 */
static void surface_rdz(const real *m, real mu, real lam, real *rx, real *ry)
{
    const real *xi = m, *et = m + 3, *zt = m + 6;
    const real chi = 2 * lam + mu, lm = lam + mu;
    real DZ[9], DX[9], DY[9], A[9];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++)
            DZ[r * 3 + c] = r == c ? chi * zt[r] * zt[r] + mu * (zt[0] * zt[0] + zt[1] * zt[1] + zt[2] * zt[2] - zt[r] * zt[r])
                                   : lm * zt[r] * zt[c];
    for (int b = 0; b < 2; b++) {
        const real *a = b == 0 ? xi : et;
        real *D = b == 0 ? DX : DY;
        for (int r = 0; r < 3; r++)
            for (int c = 0; c < 3; c++)
                D[r * 3 + c] = r == c ? chi * zt[r] * a[r] + mu * (zt[0] * a[0] + zt[1] * a[1] + zt[2] * a[2] - zt[r] * a[r])
                                      : lam * zt[r] * a[c] + mu * zt[c] * a[r];
    }
    /* inverse of DZ by its adjugate */
    const real det = DZ[0] * (DZ[4] * DZ[8] - DZ[5] * DZ[7]) - DZ[1] * (DZ[3] * DZ[8] - DZ[5] * DZ[6]) +
                     DZ[2] * (DZ[3] * DZ[7] - DZ[4] * DZ[6]);
    A[0] = (DZ[4] * DZ[8] - DZ[5] * DZ[7]) / det, A[1] = (DZ[2] * DZ[7] - DZ[1] * DZ[8]) / det;
    A[2] = (DZ[1] * DZ[5] - DZ[2] * DZ[4]) / det, A[3] = (DZ[5] * DZ[6] - DZ[3] * DZ[8]) / det;
    A[4] = (DZ[0] * DZ[8] - DZ[2] * DZ[6]) / det, A[5] = (DZ[2] * DZ[3] - DZ[0] * DZ[5]) / det;
    A[6] = (DZ[3] * DZ[7] - DZ[4] * DZ[6]) / det, A[7] = (DZ[1] * DZ[6] - DZ[0] * DZ[7]) / det;
    A[8] = (DZ[0] * DZ[4] - DZ[1] * DZ[3]) / det;
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) {
            real vx = 0, vy = 0;
            for (int t = 0; t < 3; t++) vx += A[r * 3 + t] * DX[t * 3 + c], vy += A[r * 3 + t] * DY[t * 3 + c];
            rx[r * 3 + c] = -vx, ry[r * 3 + c] = -vy;
        }
}

static void load_model(const char *dir)
{
    CJMR = malloc(sizeof(real) * np_pad * ncjm);
    for (long long n = 0; n < np_pad * ncjm; n++) CJMR[n] = (real)CJM[n];
    if (scheme != 0) return;
    RDZR = malloc(sizeof(real) * 18 * nxp * nyp);
    for (long long n = 0; n < 18LL * nxp * nyp; n++) RDZR[n] = (real)RDZ[n];
    char p[4096];
    snprintf(p, sizeof p, "%s/perturb.txt", dir);
    FILE *f = fopen(p, "r");
    if (!f) return;
    int i, j, k;
    double dm, dl, db;
    while (fscanf(f, "%d %d %d %lf %lf %lf", &i, &j, &k, &dm, &dl, &db) == 6) {
        if (i < 0 || j < 0 || k < 0 || i >= nxp || j >= nyp || k >= nzp) die("perturbation outside the grid", p);
        const long long q = IDX(i, j, k);
        CJMR[q * ncjm + 10] += (real)dm;
        CJMR[q * ncjm + 11] += (real)dl;
        CJMR[q * ncjm + 12] += (real)db;
        if (k == nzp - HALO - 1) {
            const long long s = (long long)j * nxp + i;
            surface_rdz(CJMR + q * ncjm, CJMR[q * ncjm + 10], CJMR[q * ncjm + 11], RDZR + s * 9,
                        RDZR + ((long long)nxp * nyp + s) * 9);
        }
    }
    fclose(f);
}

static void write_f64(const char *dir, const char *name, const real *x, long long n)
{
    char p[4096];
    snprintf(p, sizeof p, "%s/%s", dir, name);
    FILE *f = fopen(p, "wb");
    if (!f) die("cannot write", p);
    for (long long o = 0; o < n; o++) {
        double v = (double)x[o];
        fwrite(&v, 8, 1, f);
    }
    fclose(f);
}

/* ================================================================ main */
int main(int argc, char **argv)
{
    if (argc < 2) die("usage: stepper BUNDLE_DIR", NULL);
    const char *dir = argv[1];
    read_meta(dir);
    size_t nb;
    CJM = read_file(dir, "cjm.bin", &nb);
    if (!CJM || nb != sizeof(float) * np_pad * ncjm) die("bad cjm.bin in", dir);
    if (scheme == 0) {
        RDZ = read_file(dir, "rdz.bin", &nb);
        if (!RDZ || nb != sizeof(float) * 18 * nxp * nyp) die("bad rdz.bin in", dir);
    }
    load_model(dir);
    ST = read_file(dir, "stations.bin", &nb);
    nst = ST ? (int)(nb / 12) : 0;
    if (src_kind == 3) {
        unsigned char *b = read_file(dir, "src.bin", &nb);
        if (!b) die("no src.bin in", dir);
        memcpy(&f_npts, b, 8), memcpy(&f_nt, b + 8, 8), memcpy(&f_dt, b + 16, 4);
        f_idx = malloc(8 * (f_npts ? f_npts : 1));
        f_rate = malloc(4 * (f_npts * f_nt * 6 + 1));
        memcpy(f_idx, b + 20, 8 * f_npts);
        memcpy(f_rate, b + 20 + 8 * f_npts, 4 * f_npts * f_nt * 6);
        free(b);
        fault_scale();
    } else if (src_kind == 1 || src_kind == 2) {
        point_setup();
    }
    W = calloc(np_pad * 9, sizeof(real));
    Wh = calloc(np_pad * 9, sizeof(real));
    Wm = calloc(np_pad * 9, sizeof(real));
    Wt = scheme == 0 ? calloc(np_pad * 9, sizeof(real)) : NULL;
    RF = scheme == 1 ? calloc(np_pad * 9, sizeof(real)) : NULL;
    Ust = calloc((size_t)(nst ? nst : 1) * NT * 9, sizeof(real));
    PGV = calloc((size_t)nx * ny * 2, sizeof(real));
    if (scheme == 0) {
        pml_profiles();
        if (!pml_on)
            for (int a = 0; a < 3; a++) {
                const int nn = a == 0 ? nxp : a == 1 ? nyp : nzp;
                for (int i = 0; i < nn; i++) P_ALPHA(a)[i] = 0, P_BETA(a)[i] = 1, P_D(a)[i] = 0;
            }
        const int dirs[5] = {0, 1, 2, 0, 1}, his[5] = {0, 0, 0, 1, 1};
        for (int fc = 0; fc < 5; fc++) {
            Face *F = &FACE[fc];
            F->dir = dirs[fc], F->hi = his[fc];
            F->n = (long long)nPML * (F->dir == 0 ? (long long)ny * nz : F->dir == 1 ? (long long)nx * nz : (long long)nx * ny);
            F->A = calloc(F->n * 9, sizeof(real)), F->m = calloc(F->n * 9, sizeof(real));
            F->t = calloc(F->n * 9, sizeof(real)), F->h = calloc(F->n * 9, sizeof(real));
        }
    }
    static const int FBT[8][3] = {{-1, -1, -1}, {1, 1, -1}, {1, 1, 1}, {-1, -1, 1},
                                  {-1, 1, -1},  {1, -1, -1}, {1, -1, 1}, {-1, 1, 1}}; /* src/propagate.cpp:158-168 */
#ifdef MIX16
    if (scheme != 0) die("MIX16 covers the CGFDM scheme", NULL);
    mix_setup();
#endif
    for (int it = 0; it < NT; it++) {
#ifdef MIX16
        interior_max(Mpre);
#endif
        if (src_kind == 1 || src_kind == 2) point_inject(it);
        if (src_kind == 3) fault_inject(it);
#ifdef MIX16
        mix_scales();
#endif
        if (scheme == 0) {
            int FB1 = FBT[it % 8][0], FB2 = FBT[it % 8][1], FB3 = FBT[it % 8][2];
            for (int irk = 0; irk < 4; irk++) {
                cg_deriv(FB1, FB2, FB3);
                rk4(irk);
                FB1 = -FB1, FB2 = -FB2, FB3 = -FB3;
            }
        } else {
            for (int irk = 0; irk < 3; irk++) {
                for (int a = 0; a < 3; a++) sc_flux(a), sc_du(a);
                tvd(irk);
            }
            char_fs();
            if (decay_on) exp_decay();
        }
        record(it);
        pgv_update();
    }
    write_f32(dir, "out_stations.bin", Ust, (long long)nst * NT * 9);
    if (!IS_F32) write_f64(dir, "out_stations64.bin", Ust, (long long)nst * NT * 9);
    write_f32(dir, "out_W.bin", W, np_pad * 9);
    write_f32(dir, "out_pgv.bin", PGV, (long long)nx * ny * 2);
    return 0;
}
