/*
 * Ellipsoidal (WGS84) azimuthal-equidistant projection centred on
 * (lon0, lat0), written from Vincenty's published geodesic formulas
 * (T. Vincenty, "Direct and inverse solutions of geodesics on the ellipsoid
 * with application of nested equations", Survey Review 23(176), 1975).
 *
 * The reference maps finite-fault sub-fault lon/lat to model x/y with PROJ
 * "+proj=aeqd +lon_0 +lat_0 +x_0=0 +y_0=0 +ellps=WGS84" and
 * proj_trans_array(..., PJ_FWD, ...) (src/multiSource.cpp:122-171).  PROJ is
 * not available here, so this header is the projection used by the library's
 * source reader and by the oracle's PROJ stand-in alike.  Forward: geodesic
 * distance s and initial azimuth a from the centre give x = s sin a,
 * y = s cos a (metres, x east, y north).  Inverse: the direct geodesic
 * problem.  The centre maps to exactly (0, 0).
 *
 * Header-only C, usable from C, C++ and the oracle.
 */
#ifndef CGFDM_AEQD_H
#define CGFDM_AEQD_H

#include <math.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CGFDM_WGS84_A 6378137.0
#define CGFDM_WGS84_F (1.0 / 298.257223563)

/* lon/lat in radians -> x/y in metres.  Returns 0 on success, 1 if the
 * iteration did not converge (near-antipodal points), with x = y = NaN. */
static inline int cgfdm_aeqd_fwd(double lon0, double lat0, double lon, double lat,
                                 double *x, double *y)
{
    const double a = CGFDM_WGS84_A, f = CGFDM_WGS84_F, b = a * (1.0 - f);
    double L = lon - lon0;
    if (L == 0.0 && lat == lat0) {
        *x = 0.0;
        *y = 0.0;
        return 0;
    }
    double U1 = atan((1.0 - f) * tan(lat0));
    double U2 = atan((1.0 - f) * tan(lat));
    double sinU1 = sin(U1), cosU1 = cos(U1);
    double sinU2 = sin(U2), cosU2 = cos(U2);
    double lam = L, lamPrev;
    double sinSig = 0, cosSig = 0, sig = 0, cos2Alpha = 0, cos2SigM = 0;
    int iter = 0;
    do {
        double sinLam = sin(lam), cosLam = cos(lam);
        double t1 = cosU2 * sinLam;
        double t2 = cosU1 * sinU2 - sinU1 * cosU2 * cosLam;
        sinSig = sqrt(t1 * t1 + t2 * t2);
        if (sinSig == 0.0) {
            *x = 0.0;
            *y = 0.0;
            return 0;
        }
        cosSig = sinU1 * sinU2 + cosU1 * cosU2 * cosLam;
        sig = atan2(sinSig, cosSig);
        double sinAlpha = cosU1 * cosU2 * sinLam / sinSig;
        cos2Alpha = 1.0 - sinAlpha * sinAlpha;
        cos2SigM = (cos2Alpha != 0.0) ? cosSig - 2.0 * sinU1 * sinU2 / cos2Alpha : 0.0;
        double C = f / 16.0 * cos2Alpha * (4.0 + f * (4.0 - 3.0 * cos2Alpha));
        lamPrev = lam;
        lam = L + (1.0 - C) * f * sinAlpha *
                      (sig + C * sinSig * (cos2SigM + C * cosSig * (-1.0 + 2.0 * cos2SigM * cos2SigM)));
    } while (fabs(lam - lamPrev) > 1e-13 && ++iter < 200);
    if (iter >= 200) {
        *x = NAN;
        *y = NAN;
        return 1;
    }
    double u2 = cos2Alpha * (a * a - b * b) / (b * b);
    double A = 1.0 + u2 / 16384.0 * (4096.0 + u2 * (-768.0 + u2 * (320.0 - 175.0 * u2)));
    double B = u2 / 1024.0 * (256.0 + u2 * (-128.0 + u2 * (74.0 - 47.0 * u2)));
    double dSig = B * sinSig *
                  (cos2SigM + B / 4.0 *
                                  (cosSig * (-1.0 + 2.0 * cos2SigM * cos2SigM) -
                                   B / 6.0 * cos2SigM * (-3.0 + 4.0 * sinSig * sinSig) *
                                       (-3.0 + 4.0 * cos2SigM * cos2SigM)));
    double s = b * A * (sig - dSig);
    double az = atan2(cosU2 * sin(lam), cosU1 * sinU2 - sinU1 * cosU2 * cos(lam));
    *x = s * sin(az);
    *y = s * cos(az);
    return 0;
}

/* x/y in metres -> lon/lat in radians (direct geodesic problem). */
static inline int cgfdm_aeqd_inv(double lon0, double lat0, double x, double y,
                                 double *lon, double *lat)
{
    const double a = CGFDM_WGS84_A, f = CGFDM_WGS84_F, b = a * (1.0 - f);
    double s = sqrt(x * x + y * y);
    if (s == 0.0) {
        *lon = lon0;
        *lat = lat0;
        return 0;
    }
    double alpha1 = atan2(x, y);
    double sinA1 = sin(alpha1), cosA1 = cos(alpha1);
    double tanU1 = (1.0 - f) * tan(lat0);
    double cosU1 = 1.0 / sqrt(1.0 + tanU1 * tanU1), sinU1 = tanU1 * cosU1;
    double sig1 = atan2(tanU1, cosA1);
    double sinAlpha = cosU1 * sinA1;
    double cos2Alpha = 1.0 - sinAlpha * sinAlpha;
    double u2 = cos2Alpha * (a * a - b * b) / (b * b);
    double A = 1.0 + u2 / 16384.0 * (4096.0 + u2 * (-768.0 + u2 * (320.0 - 175.0 * u2)));
    double B = u2 / 1024.0 * (256.0 + u2 * (-128.0 + u2 * (74.0 - 47.0 * u2)));
    double sig = s / (b * A), sigPrev, cos2SigM, sinSig, cosSig;
    int iter = 0;
    do {
        cos2SigM = cos(2.0 * sig1 + sig);
        sinSig = sin(sig);
        cosSig = cos(sig);
        double dSig = B * sinSig *
                      (cos2SigM + B / 4.0 *
                                      (cosSig * (-1.0 + 2.0 * cos2SigM * cos2SigM) -
                                       B / 6.0 * cos2SigM * (-3.0 + 4.0 * sinSig * sinSig) *
                                           (-3.0 + 4.0 * cos2SigM * cos2SigM)));
        sigPrev = sig;
        sig = s / (b * A) + dSig;
    } while (fabs(sig - sigPrev) > 1e-14 && ++iter < 200);
    cos2SigM = cos(2.0 * sig1 + sig);
    sinSig = sin(sig);
    cosSig = cos(sig);
    double tmp = sinU1 * sinSig - cosU1 * cosSig * cosA1;
    double phi2 = atan2(sinU1 * cosSig + cosU1 * sinSig * cosA1,
                        (1.0 - f) * sqrt(sinAlpha * sinAlpha + tmp * tmp));
    double lamb = atan2(sinSig * sinA1, cosU1 * cosSig - sinU1 * sinSig * cosA1);
    double C = f / 16.0 * cos2Alpha * (4.0 + f * (4.0 - 3.0 * cos2Alpha));
    double L = lamb - (1.0 - C) * f * sinAlpha *
                          (sig + C * sinSig * (cos2SigM + C * cosSig * (-1.0 + 2.0 * cos2SigM * cos2SigM)));
    *lon = lon0 + L;
    *lat = phi2;
    return iter >= 200;
}

#ifdef __cplusplus
}
#endif

#endif
