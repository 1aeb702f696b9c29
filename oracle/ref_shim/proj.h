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
 */
#ifndef CGFDM_ORACLE_PROJ_SHIM_H
#define CGFDM_ORACLE_PROJ_SHIM_H

#include <stddef.h>

typedef struct { double lam, phi; } PJ_LP;
typedef struct { double x, y; } PJ_XY;
typedef union { double v[4]; PJ_LP lp; PJ_XY xy; } PJ_COORD;
typedef struct PJ_CONTEXT_S { int unused; } PJ_CONTEXT;
typedef struct PJ_S { int unused; } PJ;
typedef enum { PJ_FWD = 1, PJ_IDENT = 0, PJ_INV = -1 } PJ_DIRECTION;

static inline PJ_CONTEXT *proj_context_create(void) {
  static PJ_CONTEXT c;
  return &c;
}
static inline PJ *proj_create(PJ_CONTEXT *c, const char *s) {
  (void)c; (void)s;
  static PJ p;
  return &p;
}
static inline void proj_destroy(PJ *p) { (void)p; }
static inline void proj_context_destroy(PJ_CONTEXT *c) { (void)c; }

/* Undo the degree-to-radian scaling applied by the caller (the same
 * DEGREE2RADIAN expression as macro.h, evaluated in double). */
static inline size_t proj_trans_array(PJ *p, PJ_DIRECTION d, size_t n, PJ_COORD *c) {
  (void)p; (void)d;
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
