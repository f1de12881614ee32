/*
 * Per-function entry points of libcgfdm.so: the reference's step drivers
 * (called from propagate(), src/propagate.cpp:186-309 of CGFDM3D-EQR-SC)
 * with the same names, argument meanings and effects, on arrays the caller
 * owns.  A copy of propagate.cpp whose drivers forward here (each driver's
 * body replaced by a call of the cgfdm_ entry point of the same name) runs
 * the reference's own time loop on this library's kernels.  The session API
 * (cgfdm.h) is the fast path: it
 * fuses one RK stage into one kernel over its own layout.
 *
 * Arrays are DEVICE pointers in the reference's layouts (XFAST, src/axis.h:73):
 *   W, h_W, t_W, m_W   [_nz_][_ny_][_nx_][9]   (struct WAVE)
 *   CJM                [_nz_][_ny_][_nx_][13]  (CGFDM) or [..][19] (SCFDM)
 *   rDZ_DX, rDZ_DY     [_ny_][_nx_][9]          (struct Mat_rDZ)
 *   pml_{alpha,beta,d}_{x,y,z}  [_nx_], [_ny_], [_nz_]  (PML_ALPHA/BETA/D)
 *   aux                24 pointers: for faces x1 y1 z1 x2 y2 z2 (this
 *                      order), h_Aux, Aux, t_Aux, m_Aux of the face (struct
 *                      AUX6; the x faces [nz][ny][nPML][9], the y faces
 *                      [nz][nPML][nx][9], the z faces [nPML][ny][nx][9])
 *   border             6 ints, the same face order (struct MPI_BORDER)
 *   pml                9 pointers alpha_x beta_x d_x alpha_y beta_y d_y
 *                      alpha_z beta_z d_z
 * _nx_ = nx + 6 etc. (3-cell halo).  `stream` is a cudaStream_t or NULL;
 * calls only enqueue work.  Every call returns 0 or a CGFDM_E_* code
 * (cgfdm.h), with a message from cgfdm_shim_last_error(); the reference's
 * drivers return void.  `scheme` is 0 for the CGFDM build, 1 for the SCFDM
 * build (whose drivers take CJM for the conserved-variable conversions).
 */
#ifndef CGFDM_SHIMS_H
#define CGFDM_SHIMS_H

#ifdef __cplusplus
extern "C" {
#endif

const char *cgfdm_shim_last_error(void);

/* waveDeriv (src/wave_deriv.cpp:286-333): h_W = DT * RHS(W) at the interior
 * points, the derivative along each axis times pml_beta (PML builds; NULL
 * pointers: the build without PML). */
int cgfdm_waveDeriv(int _nx_, int _ny_, int _nz_, float rDH, float *h_W, const float *W, const float *CJM,
                    const float *pml_beta_x, const float *pml_beta_y, const float *pml_beta_z, int FB1, int FB2,
                    int FB3, float DT, void *stream);

/* freeSurfaceDeriv (src/freeSurface.cpp:496-539): h_W of the top three
 * interior layers from the traction image and the surface matrices. */
int cgfdm_freeSurfaceDeriv(int _nx_, int _ny_, int _nz_, float rDH, float *h_W, const float *W, const float *CJM,
                           const float *rDZ_DX, const float *rDZ_DY, const float *pml_beta_x, const float *pml_beta_y,
                           int FB1, int FB2, int FB3, float DT, void *stream);

/* pmlDeriv (src/pml_deriv.cpp:586-670): per face, in the order x1 y1 z1 x2
 * y2 (z2 unless free_surface), h_Aux from W and Aux, and h_W -= beta Aux DT. */
int cgfdm_pmlDeriv(int _nx_, int _ny_, int _nz_, int nPML, float rDH, float *h_W, const float *W, const float *CJM,
                   float *const *aux, const float *const *pml, const int *border, int free_surface, int FB1, int FB2,
                   int FB3, float DT, void *stream);

/* pmlFreeSurfaceDeriv (src/pml_freeSurface.cpp:244-338): the surface-layer
 * correction of the x and y faces' h_Aux. */
int cgfdm_pmlFreeSurfaceDeriv(int _nx_, int _ny_, int _nz_, int nPML, float rDH, const float *W, const float *CJM,
                              float *const *aux, const float *rDZ_DX, const float *rDZ_DY, const float *pml_d_x,
                              const float *pml_d_y, const int *border, int FB1, int FB2, float DT, void *stream);

/* waveRk (src/wave_rk.cpp:106-123): RK4 stage irk over the whole padded grid. */
int cgfdm_waveRk(int _nx_, int _ny_, int _nz_, int irk, float *h_W, float *W, float *t_W, float *m_W, void *stream);

/* pmlRk (src/pml_rk.cpp:75-146): the same stage on every face's auxiliaries. */
int cgfdm_pmlRk(int nx, int ny, int nz, int nPML, int irk, float *const *aux, const int *border, int free_surface,
                void *stream);

/* calculateMomentRate (src/addMoment.cpp:67-87): scales the finite-fault
 * table momentRate [nt][npts][6] by mu / (J DH^3) at each cell srcIndex
 * (int64 padded-grid point index). */
int cgfdm_calculateMomentRate(long long npts, long long nt, const float *CJM, float *momentRate,
                              const long long *srcIndex, float DH, int scheme, void *stream);

/* addMomenteRate (src/addMoment.cpp:262-377, NO_SOURCE_SMOOTH as the
 * reference defines it): interpolates the table at the stage time of (it,
 * irk) into momentRateSlice [npts][6] and subtracts rate * DT from the
 * stresses of W (SCFDM: the strain rates).  Once the table is exhausted the
 * call adds nothing (the reference frees the table). */
int cgfdm_addMomenteRate(long long npts, int nt, float dt, float *W, const long long *srcIndex,
                         const float *momentRate, float *momentRateSlice, int it, int irk, float DT, int scheme,
                         const float *CJM, void *stream);

/* loadPointSource_ricker, loadPointSource_double_couple (src/singleSource.cpp:
 * 175-214, 331-359): a 7 x 7 x 7 Gaussian-smoothed point source at the
 * padded point (X, Y, Z) (struct SOURCE), added to the stresses of W at the
 * stage time of (it, irk); nothing when the point is outside the interior.
 * The weights and source-time values are evaluated on the host in the
 * reference's float/double mix (Ricker M0 = 1e9, double couple m0 = 1.5
 * 10^(Mw + 6)); angles in degrees. */
int cgfdm_loadPointSource_ricker(int _nx_, int _ny_, int _nz_, int X, int Y, int Z, float *W, const float *CJM,
                                 int it, int irk, float DT, float DH, float rickerfc, int scheme, void *stream);
int cgfdm_loadPointSource_double_couple(int _nx_, int _ny_, int _nz_, int X, int Y, int Z, float *W,
                                        const float *CJM, int it, int irk, float DT, float DH, float strike,
                                        float dip, float rake, float Mw, float duration, int scheme, void *stream);

/* storageStation (src/station.cpp:382-411): the nine components at each
 * station XYZ [n][3] (padded indices) into wave [n][NT][9] at step it. */
int cgfdm_storageStation(int _nx_, int _ny_, int _nz_, int NT, int stationNum, const int *XYZ, float *wave,
                         const float *W, int it, int scheme, const float *CJM, void *stream);

/* comparePGV (src/PGV.cpp:187-229): peak horizontal and total surface
 * velocity into pgv [ny][nx][2]; with W_pre (SOLVE_PGA builds) also the
 * peak accelerations every tenth step, pgv [ny][nx][4]. */
int cgfdm_comparePGV(int nx, int ny, int nz, const float *W, float *pgv, float DT, int it, int scheme,
                     const float *CJM, const float *W_pre, void *stream);

/* SolveDisplacement (src/solve_displacement.cpp:65-74): Dis += V DT over the
 * whole padded grid, Dis [_nz_][_ny_][_nx_][3]. */
int cgfdm_SolveDisplacement(int _nx_, int _ny_, int _nz_, const float *W, float *Dis, int scheme, const float *CJM,
                            float DT, void *stream);

/* ---- ME-AWENO (SCFDM build: CJM with 19 fields, conserved variables) ---- */

/* waveDeriv_alternative_flux_FD (src/alternative_flux_FD.cpp:1437-1566, LF
 * flux): per direction x, y, z the WENO5-JS Lax-Friedrichs face fluxes into
 * Riemann_flux (zero-initialised by the caller, [_nz_][_ny_][_nx_][9], faces
 * never written stay zero) and their corrected difference into h_W (x
 * assigns, y and z add).  alpha: the Lax-Friedrichs speed, the reference's
 * vp_max_for_SCFDM. */
int cgfdm_waveDeriv_alternative_flux_FD(int _nx_, int _ny_, int _nz_, float rDH, float *h_W, const float *W,
                                        float *Riemann_flux, const float *CJM, float alpha, float DT, void *stream);

/* waveRk_tvd (src/wave_rk_tvd.cpp:80-97): TVD-RK3 stage irk (0..2). */
int cgfdm_waveRk_tvd(int _nx_, int _ny_, int _nz_, int irk, const float *h_W, float *W, float *m_W, void *stream);

/* charfreeSurfaceDeriv (src/freeSurface.cpp:196-239): the characteristic
 * free-surface condition on the surface layer and the cubic extrapolation
 * into the halo above it.  The condition is evaluated in double through the
 * inverse surface basis (agreeing with the reference's float formulas to
 * about 2e-7 relative). */
int cgfdm_charfreeSurfaceDeriv(int _nx_, int _ny_, int _nz_, float *W, const float *CJM, void *stream);

/* expDecayLayers (src/exp_decay_absorb.cpp:108-145): 20-layer exponential
 * sponge on x1 x2 y1 y2 z1 (and z2 unless free_surface). */
int cgfdm_expDecayLayers(int _nx_, int _ny_, int _nz_, float *W, int free_surface, void *stream);

/* storage_W_pre (src/propagate.cpp:26-58): copies the first _nx_ _ny_ _nz_
 * floats of W into W_pre, as the reference's kernel does. */
int cgfdm_storage_W_pre(int _nx_, int _ny_, int _nz_, float *W_pre, const float *W, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* CGFDM_SHIMS_H */
