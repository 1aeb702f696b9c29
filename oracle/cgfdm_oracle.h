/*
 * CGFDM hot-path ORACLE -- test infrastructure, not product code.
 *
 * A plain-C CPU restatement of the reference's single-rank FP32 time step
 * (src-new-FP32-SVE/propagate.cpp:142-198) used only by tests/, by
 * __graft_entry__.smoke() and by bench.py's cpu_baseline leg, as the checker.
 * The product (the CUDA path behind include/cgfdm_b200.h) never calls it.
 *
 * Pinning: the oracle is checked bit-for-bit against outputs of the reference
 * itself (compiled in place by oracle/Makefile into oracle/_ref/) that are
 * committed as fixtures in tests/golden/ (generator: tests/golden/make_golden.py).
 *
 * Memory layout is the reference's (XFAST, axis.h:61-66): padded dims
 * _nx_ = nx + 6 etc.; field v of a wave buffer at v*num + INDEX(i,j,k);
 * CJM is 13 SoA fields (CJM.cpp:117-131); PML auxiliary slabs are AoS
 * [pos][9] with pos x-fastest inside the slab (pml_deriv.cpp:164,313,464).
 * Every arithmetic expression keeps the reference's evaluation order so the
 * oracle is bit-exact with it (compiled with -ffp-contract=off).
 */
#ifndef CGFDM_ORACLE_H
#define CGFDM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
  int nx, ny, nz;   /* interior points on this (single) rank */
  int nPML;         /* absorbing-layer thickness; slabs x1 y1 z1 x2 y2 */
  float DH, rDH;    /* grid spacing and its reciprocal (grid.rDH) */
} oracle_grid;

/* PML auxiliary state of one slab: 4 buffers of [npos][9] floats. */
typedef struct {
  float *h, *a, *t, *m;
} oracle_aux;

/* Slab order used everywhere: 0=x1 1=y1 2=z1 3=x2 4=y2 (propagate.cpp:159,
 * pml_deriv.cpp:591-599; no top z slab under FREE_SURFACE). */
typedef struct {
  oracle_aux slab[5];
} oracle_aux5;

typedef struct {
  float *alpha_x, *beta_x, *d_x; /* [_nx_] */
  float *alpha_y, *beta_y, *d_y; /* [_ny_] */
  float *alpha_z, *beta_z, *d_z; /* [_nz_] */
} oracle_pml;

long long oracle_num(const oracle_grid *g);
long long oracle_slab_points(const oracle_grid *g, int slab);

/* init_pml_para.cpp:99-234, all six borders present on a single rank, no top
 * z layer (FREE_SURFACE). Arrays sized _nx_, _ny_, _nz_. */
void oracle_pml_params(const oracle_grid *g, oracle_pml *p);

/* One RK stage (propagate.cpp:155-169 minus the halo exchange).
 * W holds the stage input and receives the stage output; hW is scratch. */
void oracle_stage(const oracle_grid *g, int irk, int FB1, int FB2, int FB3, float DT,
                  float *hW, float *W, float *tW, float *mW, const float *CJM,
                  const float *rDZ_DX, const float *rDZ_DY, const oracle_pml *p,
                  oracle_aux5 *aux);

/* The individual pieces, exposed for unit tests. */
void oracle_wave_deriv(const oracle_grid *g, float *hW, const float *W, const float *CJM,
                       const oracle_pml *p, int FB1, int FB2, int FB3, float DT);
void oracle_free_surface_deriv(const oracle_grid *g, float *hW, const float *W,
                               const float *CJM, const float *rDZ_DX, const float *rDZ_DY,
                               const oracle_pml *p, int FB1, int FB2, int FB3, float DT);
void oracle_pml_deriv(const oracle_grid *g, float *hW, const float *W, const float *CJM,
                      const oracle_pml *p, oracle_aux5 *aux, int FB1, int FB2, int FB3,
                      float DT);
void oracle_pml_free_surface(const oracle_grid *g, const float *W, const float *CJM,
                             const float *rDZ_DX, const float *rDZ_DY, const oracle_pml *p,
                             oracle_aux5 *aux, int FB1, int FB2, float DT);
void oracle_wave_rk(int irk, float *hW, float *W, float *tW, float *mW, long long n);

/* Ricker-derivative moment of the single point source at stage 0 of step it
 * (singleSource.cpp:29-56). */
float oracle_ricker_moment(float rickerfc, int it, float DT);
/* 7^3 Gaussian-smoothed explosive source added to W (singleSource.cpp:78-127).
 * (sx,sy,sz) are padded-grid indices of the source cell. */
void oracle_smooth_source(const oracle_grid *g, float *W, const float *CJM, int sx, int sy,
                          int sz, int it, float DT, float rickerfc);

/* Finite-fault moment-rate injection (addMoment.cpp:222-339, NO_SOURCE_SMOOTH):
 * momentRate is [nt][npts][6], already scaled by mu*Cv/(J*DH^3).  Returns 0
 * once the source has run out of samples (srcIt+1 >= nt), 1 otherwise. */
int oracle_add_moment_rate(const oracle_grid *g, float *W, const long long *srcIndex,
                           const float *momentRate, long long npts, int nt, float dt,
                           int it, float DT);
/* calculate_MomentRate (addMoment.cpp:12-65). */
void oracle_scale_moment_rate(const oracle_grid *g, const float *CJM, float *momentRate,
                              const long long *srcIndex, long long npts, int nt);

/* storage_station (station.cpp:310-347): wave[(it + s*NT)*9 + v]. */
void oracle_station(const oracle_grid *g, const float *W, const int *xyz, int nsta, int NT,
                    int it, float *wave);
/* compare_pgv (PGV.cpp:49-101): pgv[ny][nx][2] running max on the top layer. */
void oracle_pgv(const oracle_grid *g, const float *W, float *pgv);

/* The MacCormack sign triple of step it (propagate.cpp:107-117,144). */
void oracle_fb(int it, int fb[3]);

#ifdef __cplusplus
}
#endif
#endif
