/*
 * Minimal stand-in for the PROJ C API (PROJ >= 8.1, not installed here),
 * covering only what the reference calls: proj_context_create/destroy,
 * proj_create("+proj=aeqd +lon_0=.. +lat_0=.. ..."), proj_trans_array with
 * PJ_FWD/PJ_INV, proj_destroy (src/multiSource.cpp:96-171,
 * src/terrain.cpp:120-202,325-347,450-536).  Test infrastructure only.
 *
 * The projection itself is the library's own aeqd implementation
 * (cgfdm3d-eqr-sc_b200/csrc/aeqd.h), so the oracle and the library feed the
 * same x/y into the reference's source-location code.  Agreement with real
 * PROJ is not pinned by any reference test.
 */
#ifndef ORACLE_STUB_PROJ_H
#define ORACLE_STUB_PROJ_H

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include "../../../cgfdm3d-eqr-sc_b200/csrc/aeqd.h"

typedef struct { double x, y; } PJ_XY;
typedef struct { double lam, phi; } PJ_LP;
typedef struct { double x, y, z; } PJ_XYZ;
typedef struct { double lam, phi, z; } PJ_LPZ;
typedef union {
    double v[4];
    PJ_XY xy;
    PJ_LP lp;
    PJ_XYZ xyz;
    PJ_LPZ lpz;
} PJ_COORD;

typedef enum { PJ_FWD = 1, PJ_IDENT = 0, PJ_INV = -1 } PJ_DIRECTION;

typedef struct { int unused; } PJ_CONTEXT;
typedef struct { double lon0, lat0; } PJ; /* radians */

static inline PJ_CONTEXT *proj_context_create(void)
{
    return (PJ_CONTEXT *)calloc(1, sizeof(PJ_CONTEXT));
}
static inline PJ_CONTEXT *proj_context_destroy(PJ_CONTEXT *c)
{
    free(c);
    return NULL;
}

static inline double oracle_proj_param(const char *def, const char *key)
{
    const char *p = strstr(def, key);
    if (!p) return 0.0;
    return atof(p + strlen(key));
}

static inline PJ *proj_create(PJ_CONTEXT *, const char *def)
{
    if (!strstr(def, "+proj=aeqd")) return NULL;
    PJ *P = (PJ *)calloc(1, sizeof(PJ));
    const double d2r = 3.14159265358979323846 / 180.0;
    P->lon0 = oracle_proj_param(def, "+lon_0=") * d2r;
    P->lat0 = oracle_proj_param(def, "+lat_0=") * d2r;
    return P;
}

static inline PJ *proj_destroy(PJ *P)
{
    free(P);
    return NULL;
}

static inline int proj_trans_array(PJ *P, PJ_DIRECTION d, size_t n, PJ_COORD *c)
{
    for (size_t i = 0; i < n; i++) {
        double u, v;
        if (d == PJ_FWD) {
            cgfdm_aeqd_fwd(P->lon0, P->lat0, c[i].lp.lam, c[i].lp.phi, &u, &v);
            c[i].xy.x = u;
            c[i].xy.y = v;
        } else if (d == PJ_INV) {
            cgfdm_aeqd_inv(P->lon0, P->lat0, c[i].xy.x, c[i].xy.y, &u, &v);
            c[i].lp.lam = u;
            c[i].lp.phi = v;
        }
    }
    return 0;
}

#endif
