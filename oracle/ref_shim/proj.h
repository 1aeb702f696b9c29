/*
 * Test infrastructure (oracle harness), not product code.
 *
 * Stand-in for the PROJ API used by the reference's source reader
 * (src-new-FP32-SVE/multiSource.cpp:89-170).  PROJ itself is not installed
 * here.  The stand-in projection is the identity on the values stored in the
 * source file: LonLat2cart multiplies lon/lat by DEGREE2RADIAN and
 * proj_trans_array divides by the same factor, so the file's "lon"/"lat"
 * fields are read as Cartesian metres relative to the grid centre.  This is
 * how the synthetic finite-fault and point-source fixtures are fed to the
 * reference without a real map projection.
 *
 * The inverse direction (PJ_INV) is the terrain reader's (terrain.cpp:
 * grid x/y in metres -> longitude/latitude in radians about the centre of
 * the "+proj=aeqd +lon_0=.. +lat_0=.." string): the azimuthal equidistant
 * projection evaluated on a sphere of radius 6371008.8 m (Snyder 1987, eqs.
 * 20-14 and 20-15), the same stand-in as the library's own DEM reader.
 */
#ifndef CGFDM_ORACLE_PROJ_SHIM_H
#define CGFDM_ORACLE_PROJ_SHIM_H

#include <math.h>
#include <stddef.h>
#include <stdio.h>
#include <string.h>

typedef struct { double lam, phi; } PJ_LP;
typedef struct { double x, y; } PJ_XY;
typedef union { double v[4]; PJ_LP lp; PJ_XY xy; } PJ_COORD;
typedef struct PJ_CONTEXT_S { int unused; } PJ_CONTEXT;
typedef struct PJ_S { double lam0, phi0; } PJ;
typedef enum { PJ_FWD = 1, PJ_IDENT = 0, PJ_INV = -1 } PJ_DIRECTION;

static inline PJ_CONTEXT *proj_context_create(void) {
  static PJ_CONTEXT c;
  return &c;
}
static inline PJ *proj_create(PJ_CONTEXT *c, const char *s) {
  (void)c;
  static PJ p;
  double lo = 0, la = 0;
  const char *a = strstr(s, "+lon_0="), *b = strstr(s, "+lat_0=");
  if (a) sscanf(a + 7, "%lf", &lo);
  if (b) sscanf(b + 7, "%lf", &la);
  p.lam0 = lo * (M_PI / 180.0);
  p.phi0 = la * (M_PI / 180.0);
  return &p;
}
static inline void proj_destroy(PJ *p) { (void)p; }
static inline void proj_context_destroy(PJ_CONTEXT *c) { (void)c; }

/* Undo the degree-to-radian scaling applied by the caller (the same
 * DEGREE2RADIAN expression as macro.h, evaluated in double). */
static inline size_t proj_trans_array(PJ *p, PJ_DIRECTION d, size_t n, PJ_COORD *c) {
  if (d == PJ_INV) {
    const double R = 6371008.8, s0 = sin(p->phi0), c0 = cos(p->phi0);
    for (size_t i = 0; i < n; ++i) {
      const double x = c[i].xy.x, y = c[i].xy.y;
      const double rho = sqrt(x * x + y * y);
      double lam = p->lam0, phi = p->phi0;
      if (rho != 0.0) {
        const double cc = rho / R, sn = sin(cc), cs = cos(cc);
        phi = asin(cs * s0 + y * sn * c0 / rho);
        lam = p->lam0 + atan2(x * sn, rho * c0 * cs - y * s0 * sn);
      }
      c[i].lp.lam = lam;
      c[i].lp.phi = phi;
    }
    return 0;
  }
  const double deg2rad = (double)3.141592657f / 180.0;
  for (size_t i = 0; i < n; ++i) {
    double x = c[i].lp.lam / deg2rad;
    double y = c[i].lp.phi / deg2rad;
    c[i].xy.x = x;
    c[i].xy.y = y;
  }
  return 0;
}

#endif
