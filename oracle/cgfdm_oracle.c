/*
 * CGFDM hot-path ORACLE -- test infrastructure, not product code.
 * See cgfdm_oracle.h for the contract.  Each function names the reference
 * file:line it restates (paths relative to src-new-FP32-SVE/).  Arithmetic is
 * written in the reference's evaluation order, in float, so that results are
 * bit-identical to the reference's scalar FP32 build on x86-64.
 */
#include "cgfdm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define H 3 /* HALO, macro.h:42 */

/* MacCormack one-sided coefficients (macro.h:123-128) and the 2/3-point
 * one-sided surface operators (macro.h:149-151). */
static const float A_M1 = -0.30874f, A_0 = -0.6326f, A_1 = 1.2330f, A_2 = -0.3334f,
                   A_3 = 0.04168f;
static const float CF1 = -1.16666667f, CF2 = 1.33333333f, CF3 = -0.16666667f;
/* RK4 weights (macro.h:138-147). */
static const float RK_B1 = 0.16666667f, RK_B2 = 0.33333333f, RK_B3 = 0.33333333f,
                   RK_B4 = 0.16666667f, RK_A2 = 0.5f, RK_A3 = 0.5f;
static const float PI_F = 3.141592657f; /* macro.h:60 */

typedef struct {
  int nx_, ny_, nz_; /* padded */
  long long num, sx, sy, sz;
} dims;

static dims mkdims(const oracle_grid *g) {
  dims d;
  d.nx_ = g->nx + 2 * H;
  d.ny_ = g->ny + 2 * H;
  d.nz_ = g->nz + 2 * H;
  d.num = (long long)d.nx_ * d.ny_ * d.nz_;
  d.sx = 1;
  d.sy = d.nx_;
  d.sz = (long long)d.nx_ * d.ny_;
  return d;
}

static inline long long IX(const dims *d, int i, int j, int k) {
  return i + (long long)j * d->nx_ + (long long)k * d->nx_ * d->ny_;
}

long long oracle_num(const oracle_grid *g) { return mkdims(g).num; }

long long oracle_slab_points(const oracle_grid *g, int slab) {
  switch (slab) {
    case 0: case 3: return (long long)g->nPML * g->ny * g->nz;
    case 1: case 4: return (long long)g->nx * g->nPML * g->nz;
    default: return (long long)g->nx * g->ny * g->nPML;
  }
}

/* The L operator (axis.h:129-133): FB * (5-point one-sided sum) * rDH. */
static inline float Lop(const float *w, long long c, long long s, int fb, float rDH) {
  long long o = fb * s;
  return (float)fb *
         (A_M1 * w[c - o] + A_0 * w[c] + A_1 * w[c + o] + A_2 * w[c + 2 * o] + A_3 * w[c + 3 * o]) *
         rDH;
}

/* Elastic combination of one direction's derivatives (wave_deriv.cpp:163-191):
 * m = metric row (xi, et or zt), dv = d(Vx,Vy,Vz), dt = d(Txx,Tyy,Tzz,Txy,Txz,Tyz).
 * out[9] in field order Vx Vy Vz Txx Tyy Tzz Txy Txz Tyz. */
static inline void elastic(const float m[3], const float dv[3], const float dt[6], float mu,
                           float lam, float b, float out[9]) {
  const float txx = dt[0], tyy = dt[1], tzz = dt[2], txy = dt[3], txz = dt[4], tyz = dt[5];
  out[0] = (m[0] * txx + m[1] * txy + m[2] * txz) * b;
  out[1] = (m[0] * txy + m[1] * tyy + m[2] * tyz) * b;
  out[2] = (m[0] * txz + m[1] * tyz + m[2] * tzz) * b;
  float div = m[0] * dv[0] + m[1] * dv[1] + m[2] * dv[2];
  out[3] = div * lam + 2.0f * mu * (m[0] * dv[0]);
  out[4] = div * lam + 2.0f * mu * (m[1] * dv[1]);
  out[5] = div * lam + 2.0f * mu * (m[2] * dv[2]);
  out[6] = (m[1] * dv[0] + m[0] * dv[1]) * mu;
  out[7] = (m[2] * dv[0] + m[0] * dv[2]) * mu;
  out[8] = (m[2] * dv[1] + m[1] * dv[2]) * mu;
}

/* Derivatives of all 9 fields along one axis, each times `scale`
 * (pml beta in wave_deriv.cpp:132-160, pml d in pml_deriv.cpp:176-184). */
static inline void deriv9(const float *W, long long num, long long c, long long s, int fb,
                          float rDH, float scale, float dv[3], float dt[6]) {
  for (int v = 0; v < 3; ++v) dv[v] = Lop(W + v * num, c, s, fb, rDH) * scale;
  for (int v = 0; v < 6; ++v) dt[v] = Lop(W + (3 + v) * num, c, s, fb, rDH) * scale;
}

static inline void load_metric(const float *CJM, long long num, long long c, int dir,
                               float m[3]) {
  m[0] = CJM[c + num * (3 * dir + 0)];
  m[1] = CJM[c + num * (3 * dir + 1)];
  m[2] = CJM[c + num * (3 * dir + 2)];
}

/* wave_deriv.cpp:58-203 */
void oracle_wave_deriv(const oracle_grid *g, float *hW, const float *W, const float *CJM,
                       const oracle_pml *p, int FB1, int FB2, int FB3, float DT) {
  dims d = mkdims(g);
  const long long num = d.num;
  for (int k = H; k < d.nz_ - H; ++k)
    for (int j = H; j < d.ny_ - H; ++j)
      for (int i = H; i < d.nx_ - H; ++i) {
        long long c = IX(&d, i, j, k);
        float mu = CJM[c + num * 10], lam = CJM[c + num * 11], b = CJM[c + num * 12];
        float m[3][3], dv[3], dt[6], term[3][9];
        const float beta[3] = {p->beta_x[i], p->beta_y[j], p->beta_z[k]};
        const long long st[3] = {d.sx, d.sy, d.sz};
        const int fb[3] = {FB1, FB2, FB3};
        for (int dir = 0; dir < 3; ++dir) load_metric(CJM, num, c, dir, m[dir]);
        for (int dir = 0; dir < 3; ++dir) {
          deriv9(W, num, c, st[dir], fb[dir], g->rDH, beta[dir], dv, dt);
          elastic(m[dir], dv, dt, mu, lam, b, term[dir]);
        }
        for (int v = 0; v < 9; ++v) hW[c + num * v] = (term[0][v] + term[1][v] + term[2][v]) * DT;
      }
}

/* J-weighted traction row for the free-surface velocity update
 * (freeSurface.cpp:128-153): rows of (m . T) * J at point q. */
static inline void jt_rows(const float *W, const float *CJM, long long num, long long q, int dir,
                           float out[3]) {
  float m0 = CJM[q + num * (3 * dir + 0)], m1 = CJM[q + num * (3 * dir + 1)],
        m2 = CJM[q + num * (3 * dir + 2)], J = CJM[q + num * 9];
  out[0] = (m0 * W[q + num * 3] + m1 * W[q + num * 6] + m2 * W[q + num * 7]) * J;
  out[1] = (m0 * W[q + num * 6] + m1 * W[q + num * 4] + m2 * W[q + num * 8]) * J;
  out[2] = (m0 * W[q + num * 7] + m1 * W[q + num * 8] + m2 * W[q + num * 5]) * J;
}

/* L_J_T (axis.h:71-75) on a 7-entry window centred at index 3. */
static inline float LJT(const float jt[7], int fb, float rDH) {
  return (float)fb *
         (A_M1 * jt[3 - fb] + A_0 * jt[3] + A_1 * jt[3 + fb] + A_2 * jt[3 + 2 * fb] +
          A_3 * jt[3 + 3 * fb]) *
         rDH;
}

/* free_surface_deriv (freeSurface.cpp:22-258): overwrites hW on the top
 * three interior layers. */
void oracle_free_surface_deriv(const oracle_grid *g, float *hW, const float *W,
                               const float *CJM, const float *rDZ_DX, const float *rDZ_DY,
                               const oracle_pml *p, int FB1, int FB2, int FB3, float DT) {
  dims d = mkdims(g);
  const long long num = d.num;
  const int nzt = d.nz_ - H; /* _nz */
  for (int k = nzt - H; k < nzt; ++k)
    for (int j = H; j < d.ny_ - H; ++j)
      for (int i = H; i < d.nx_ - H; ++i) {
        long long c = IX(&d, i, j, k);
        float mu = CJM[c + num * 10], lam = CJM[c + num * 11], b = CJM[c + num * 12];
        float bx = p->beta_x[i], by = p->beta_y[j];
        int ks = (nzt - 1) - k + H;
        float jx[3][7], jy[3][7], jz[3][7], r[3];
        for (int l = 0; l <= 2 * H; ++l) {
          jt_rows(W, CJM, num, IX(&d, i + (l - H), j, k), 0, r);
          for (int a = 0; a < 3; ++a) jx[a][l] = r[a];
          jt_rows(W, CJM, num, IX(&d, i, j + (l - H), k), 1, r);
          for (int a = 0; a < 3; ++a) jy[a][l] = r[a];
        }
        for (int l = 0; l < ks; ++l) {
          jt_rows(W, CJM, num, IX(&d, i, j, k + (l - H)), 2, r);
          for (int a = 0; a < 3; ++a) jz[a][l] = r[a];
        }
        for (int a = 0; a < 3; ++a) jz[a][ks] = 0.0f; /* traction-free surface */
        for (int l = ks + 1; l <= 2 * H; ++l)
          for (int a = 0; a < 3; ++a) jz[a][l] = -jz[a][2 * ks - l]; /* odd image */
        float Jinv = 1.0f / CJM[c + num * 9];
        float hv[3];
        for (int a = 0; a < 3; ++a)
          hv[a] = b * Jinv *
                  (LJT(jx[a], FB1, g->rDH) * bx + LJT(jy[a], FB2, g->rDH) * by +
                   LJT(jz[a], FB3, g->rDH));

        float vxi[3], vet[3], vzt[3];
        for (int v = 0; v < 3; ++v) {
          vxi[v] = Lop(W + v * num, c, d.sx, FB1, g->rDH) * bx;
          vet[v] = Lop(W + v * num, c, d.sy, FB2, g->rDH) * by;
        }
        float m[3][3];
        for (int dir = 0; dir < 3; ++dir) load_metric(CJM, num, c, dir, m[dir]);
        if (k == nzt - 1) { /* velocity z-gradient from the traction condition */
          long long s = (long long)i + (long long)j * d.nx_;
          const float *DX = rDZ_DX + s * 9, *DY = rDZ_DY + s * 9;
          for (int a = 0; a < 3; ++a)
            vzt[a] = (DX[3 * a] * vxi[0] + DX[3 * a + 1] * vxi[1] + DX[3 * a + 2] * vxi[2]) +
                     (DY[3 * a] * vet[0] + DY[3 * a + 1] * vet[1] + DY[3 * a + 2] * vet[2]);
        }
        if (k == nzt - 2) /* L2 (axis.h:92) */
          for (int v = 0; v < 3; ++v)
            vzt[v] = (float)FB3 * (W[c + FB3 * d.sz + num * v] - W[c + num * v]) * g->rDH;
        if (k == nzt - 3) /* L3 (axis.h:93) */
          for (int v = 0; v < 3; ++v)
            vzt[v] = (float)FB3 *
                     (CF1 * W[c + num * v] + CF2 * W[c + FB3 * d.sz + num * v] +
                      CF3 * W[c + 2 * FB3 * d.sz + num * v]) *
                     g->rDH;
        float zero6[6] = {0, 0, 0, 0, 0, 0}, t1[9], t2[9], t3[9];
        elastic(m[0], vxi, zero6, mu, lam, b, t1);
        elastic(m[1], vet, zero6, mu, lam, b, t2);
        elastic(m[2], vzt, zero6, mu, lam, b, t3);
        for (int a = 0; a < 3; ++a) hW[c + num * a] = hv[a] * DT;
        for (int v = 3; v < 9; ++v) hW[c + num * v] = (t1[v] + t2[v] + t3[v]) * DT;
      }
}

/* Slab geometry: loop bounds (slab-local) and the padded-grid offset. */
static void slab_box(const oracle_grid *g, int slab, int n[3], int off[3], int *axis) {
  int flag = slab >= 3;
  int ax = slab % 3;
  n[0] = g->nx; n[1] = g->ny; n[2] = g->nz;
  off[0] = off[1] = off[2] = H;
  n[ax] = g->nPML;
  int full = ax == 0 ? g->nx : ax == 1 ? g->ny : g->nz;
  off[ax] = H + flag * (full - g->nPML);
  *axis = ax;
}

/* pml_deriv_x/y/z (pml_deriv.cpp:90-544) for one slab. */
static void pml_deriv_slab(const oracle_grid *g, const dims *d, float *hW, const float *W,
                           const float *CJM, const oracle_pml *p, oracle_aux *A, int slab,
                           int fb, float DT) {
  int n[3], off[3], ax;
  slab_box(g, slab, n, off, &ax);
  const long long num = d->num;
  const long long st = ax == 0 ? d->sx : ax == 1 ? d->sy : d->sz;
  const float *alpha = ax == 0 ? p->alpha_x : ax == 1 ? p->alpha_y : p->alpha_z;
  const float *beta = ax == 0 ? p->beta_x : ax == 1 ? p->beta_y : p->beta_z;
  const float *dd = ax == 0 ? p->d_x : ax == 1 ? p->d_y : p->d_z;
  for (int k0 = 0; k0 < n[2]; ++k0)
    for (int j0 = 0; j0 < n[1]; ++j0)
      for (int i0 = 0; i0 < n[0]; ++i0) {
        int i = i0 + off[0], j = j0 + off[1], k = k0 + off[2];
        int l = ax == 0 ? i : ax == 1 ? j : k;
        long long c = IX(d, i, j, k);
        long long pos = i0 + (long long)j0 * n[0] + (long long)k0 * n[0] * n[1];
        float mu = CJM[c + num * 10], lam = CJM[c + num * 11], b = CJM[c + num * 12];
        float bt = beta[l], dl = dd[l], ad = dl + alpha[l];
        float m[3], dv[3], dt[6], term[9];
        load_metric(CJM, num, c, ax, m);
        deriv9(W, num, c, st, fb, g->rDH, dl, dv, dt);
        elastic(m, dv, dt, mu, lam, b, term);
        float *ha = A->h + pos * 9;
        const float *aa = A->a + pos * 9;
        for (int v = 0; v < 9; ++v) ha[v] = (term[v] - ad * aa[v]) * DT;
        for (int v = 0; v < 9; ++v) hW[c + num * v] += -bt * aa[v] * DT;
      }
}

void oracle_pml_deriv(const oracle_grid *g, float *hW, const float *W, const float *CJM,
                      const oracle_pml *p, oracle_aux5 *aux, int FB1, int FB2, int FB3,
                      float DT) {
  dims d = mkdims(g);
  const int fb[3] = {FB1, FB2, FB3};
  for (int s = 0; s < 5; ++s) pml_deriv_slab(g, &d, hW, W, CJM, p, &aux->slab[s], s, fb[s % 3], DT);
}

/* pml_free_surface_x/y (pml_freeSurface.cpp:12-235): adds the surface
 * traction correction to the stress auxiliaries of the x and y slabs. */
void oracle_pml_free_surface(const oracle_grid *g, const float *W, const float *CJM,
                             const float *rDZ_DX, const float *rDZ_DY, const oracle_pml *p,
                             oracle_aux5 *aux, int FB1, int FB2, float DT) {
  dims d = mkdims(g);
  const long long num = d.num;
  static const int order[4] = {0, 1, 3, 4}; /* x1 y1 x2 y2 (pml_freeSurface.cpp:278-304) */
  for (int o = 0; o < 4; ++o) {
    int slab = order[o], n[3], off[3], ax;
    slab_box(g, slab, n, off, &ax);
    const int fb = ax == 0 ? FB1 : FB2;
    const long long st = ax == 0 ? d.sx : d.sy;
    const float *dd = ax == 0 ? p->d_x : p->d_y;
    const float *M = ax == 0 ? rDZ_DX : rDZ_DY;
    int k0 = g->nz - 1;
    for (int j0 = 0; j0 < n[1]; ++j0)
      for (int i0 = 0; i0 < n[0]; ++i0) {
        int i = i0 + off[0], j = j0 + off[1], k = k0 + H;
        long long c = IX(&d, i, j, k);
        long long s = (long long)i + (long long)j * d.nx_;
        long long pos = i0 + (long long)j0 * n[0] + (long long)k0 * n[0] * n[1];
        float mu = CJM[c + num * 10], lam = CJM[c + num * 11];
        float dl = dd[ax == 0 ? i : j];
        float zt[3], vd[3], vz[3], zero6[6] = {0, 0, 0, 0, 0, 0}, t[9];
        load_metric(CJM, num, c, 2, zt);
        for (int v = 0; v < 3; ++v) vd[v] = Lop(W + v * num, c, st, fb, g->rDH) * dl;
        const float *R = M + s * 9;
        for (int a = 0; a < 3; ++a) vz[a] = R[3 * a] * vd[0] + R[3 * a + 1] * vd[1] + R[3 * a + 2] * vd[2];
        elastic(zt, vz, zero6, mu, lam, 0.0f, t);
        float *ha = aux->slab[slab].h + pos * 9;
        for (int v = 3; v < 9; ++v) ha[v] += t[v] * DT;
      }
  }
}

/* wave_rk0..3 (wave_rk.cpp:13-99) and wave_pml_rk0..3 (pml_rk.cpp:15-69). */
void oracle_wave_rk(int irk, float *hW, float *W, float *tW, float *mW, long long n) {
  for (long long i = 0; i < n; ++i) {
    float h = hW[i];
    switch (irk) {
      case 0: {
        float m = W[i];
        mW[i] = m;
        tW[i] = m + RK_B1 * h;
        W[i] = m + RK_A2 * h;
      } break;
      case 1:
        tW[i] = tW[i] + RK_B2 * h;
        W[i] = mW[i] + RK_A3 * h;
        break;
      case 2:
        tW[i] = tW[i] + RK_B3 * h;
        W[i] = mW[i] + h;
        break;
      default:
        W[i] = tW[i] + RK_B4 * h;
    }
  }
}

void oracle_stage(const oracle_grid *g, int irk, int FB1, int FB2, int FB3, float DT,
                  float *hW, float *W, float *tW, float *mW, const float *CJM,
                  const float *rDZ_DX, const float *rDZ_DY, const oracle_pml *p,
                  oracle_aux5 *aux) {
  oracle_wave_deriv(g, hW, W, CJM, p, FB1, FB2, FB3, DT);
  oracle_free_surface_deriv(g, hW, W, CJM, rDZ_DX, rDZ_DY, p, FB1, FB2, FB3, DT);
  oracle_pml_deriv(g, hW, W, CJM, p, aux, FB1, FB2, FB3, DT);
  oracle_pml_free_surface(g, W, CJM, rDZ_DX, rDZ_DY, p, aux, FB1, FB2, DT);
  oracle_wave_rk(irk, hW, W, tW, mW, oracle_num(g) * 9);
  for (int s = 0; s < 5; ++s)
    oracle_wave_rk(irk, aux->slab[s].h, aux->slab[s].a, aux->slab[s].t, aux->slab[s].m,
                   oracle_slab_points(g, s) * 9);
}

/* init_pml_para.cpp:99-234 (profiles 13-19; Cp hard-coded to 6000). */
void oracle_pml_params(const oracle_grid *g, oracle_pml *p) {
  const int n_[3] = {g->nx + 2 * H, g->ny + 2 * H, g->nz + 2 * H};
  float *al[3] = {p->alpha_x, p->alpha_y, p->alpha_z};
  float *be[3] = {p->beta_x, p->beta_y, p->beta_z};
  float *dd[3] = {p->d_x, p->d_y, p->d_z};
  const int nPML = g->nPML;
  const float DH = g->DH;
  float Cp = 6000.0f, pml_fc = 0.5f;
  float L = DH * (nPML - 1);
  float R = (float)pow(10.0, -(log10((double)nPML) - 1.0) / log10(2.0) - 3.0);
  float d0 = -(2.0f + 1.0f) * Cp / (2.0f * L) * logf(R);
  float a0 = PI_F * pml_fc, b0 = 3.0f;
  for (int ax = 0; ax < 3; ++ax) {
    int np = n_[ax], ni = np - H; /* _n */
    for (int i = 0; i < np; ++i) {
      float l = -1.0f;
      if (i >= H && i < ni) {
        if (i < H + nPML) l = (H + nPML - 1 - i) * DH;
        if (ax != 2 && i >= ni - nPML) l = (i - (ni - nPML)) * DH;
      }
      float a = 0.0f, b = 1.0f, dv = 0.0f;
      if (i >= H && i < ni) {
        a = l < 0.0f ? 0.0f : a0 * (1.0f - powf(l / L, 1.0f));
        b = l < 0.0f ? 1.0f : 1.0f + (b0 - 1.0f) * powf(l / L, 2.0f);
        dv = l < 0.0f ? 0.0f : d0 * powf(l / L, 2.0f);
      }
      al[ax][i] = a;
      dd[ax][i] = dv / b;
      be[ax][i] = 1.0f / b;
    }
  }
}

/* sourceFunction at irk = 0 (singleSource.cpp:29-56). */
float oracle_ricker_moment(float rickerfc, int it, float DT) {
  float t = (it + 0.0f) * DT;
  float tdelay = 1.2f / rickerfc;
  float f0 = 2;
  float r = PI_F * rickerfc * (t - tdelay);
  float rr = r * r;
  float s = (float)(r * (2.0f * rr - 3.0) * expf(-rr) * f0 * PI_F * rickerfc);
  float M0 = 1e16f;
  s *= M0;
  return s;
}

void oracle_smooth_source(const oracle_grid *g, float *W, const float *CJM, int sx, int sy,
                          int sz, int it, float DT, float rickerfc) {
  dims d = mkdims(g);
  const int nG = 3;
  if (!(sx >= H && sx < d.nx_ - H && sy >= H && sy < d.ny_ - H && sz >= H && sz < d.nz_ - H))
    return; /* singleSource.cpp:168-174 */
  float s = oracle_ricker_moment(rickerfc, it, DT);
  float ra = nG * 0.5f;
  float jacb = CJM[IX(&d, sx, sy, sz) + d.num * 9];
  float DH = g->DH;
  for (int k = sz - nG; k < sz + nG + 1; ++k)
    for (int j = sy - nG; j < sy + nG + 1; ++j)
      for (int i = sx - nG; i < sx + nG + 1; ++i) {
        long long c = IX(&d, i, j, k);
        double di = (i - sx) - 0.0, dj = (j - sy) - 0.0, dk = (k - sz) - 0.0;
        float D1 = (float)(exp(-((di / ra) * (di / ra))) / (ra * 1.772453850905516));
        float D2 = (float)(exp(-((dj / ra) * (dj / ra))) / (ra * 1.772453850905516));
        float D3 = (float)(exp(-((dk / ra) * (dk / ra))) / (ra * 1.772453850905516));
        float amp = D1 * D2 * D3;
        amp = (float)(amp / 0.998125703461425);
        float value = -1.0f * s * amp / (jacb * (DH * DH * DH));
        value = (float)(value * (1.0 * DT));
        for (int v = 3; v < 6; ++v) W[c + d.num * v] = W[c + d.num * v] + value;
      }
}

void oracle_scale_moment_rate(const oracle_grid *g, const float *CJM, float *momentRate,
                              const long long *srcIndex, long long npts, int nt) {
  dims d = mkdims(g);
  float DH = g->DH;
  for (int t = 0; t < nt; ++t)
    for (long long i = 0; i < npts; ++i) {
      long long idx = srcIndex[i];
      float jacb = CJM[idx + d.num * 9], mu = CJM[idx + d.num * 10];
      long long pos = i + (long long)t * npts;
      float V = jacb * DH * DH * DH;
      V = (float)(1.0 / V);
      V = (float)(V * 1.0);
      for (int c = 0; c < 6; ++c) momentRate[pos * 6 + c] *= mu * V;
    }
}

int oracle_add_moment_rate(const oracle_grid *g, float *W, const long long *srcIndex,
                           const float *momentRate, long long npts, int nt, float dt, int it,
                           float DT) {
  dims d = mkdims(g);
  float tmpT = (it + 0.0f) * DT;
  int srcIt = (int)(tmpT / dt);
  if (srcIt + 1 >= nt) return 0;
  float t1 = (float)srcIt * dt;
  float tw = (tmpT - t1) / dt;
  for (long long i = 0; i < npts; ++i) {
    long long idx = srcIndex[i];
    const float *m0 = momentRate + ((long long)srcIt * npts + i) * 6;
    const float *m1 = momentRate + ((long long)(srcIt + 1) * npts + i) * 6;
    for (int c = 0; c < 6; ++c) {
      float slice = (m1[c] - m0[c]) * tw + m0[c];
      W[idx + (3 + c) * d.num] -= slice * DT;
    }
  }
  return 1;
}

void oracle_station(const oracle_grid *g, const float *W, const int *xyz, int nsta, int NT,
                    int it, float *wave) {
  dims d = mkdims(g);
  for (int s = 0; s < nsta; ++s) {
    long long c = IX(&d, xyz[3 * s], xyz[3 * s + 1], xyz[3 * s + 2]);
    long long pos = it + (long long)s * NT;
    for (int v = 0; v < 9; ++v) wave[pos * 9 + v] = W[c + d.num * v] * 1.0f;
  }
}

void oracle_pgv(const oracle_grid *g, const float *W, float *pgv) {
  dims d = mkdims(g);
  int k = d.nz_ - H - 1;
  for (int j0 = 0; j0 < g->ny; ++j0)
    for (int i0 = 0; i0 < g->nx; ++i0) {
      long long c = IX(&d, i0 + H, j0 + H, k);
      long long pos = i0 + (long long)j0 * g->nx;
      float vx = (float)(W[c] * 1.0), vy = (float)(W[c + d.num] * 1.0),
            vz = (float)(W[c + 2 * d.num] * 1.0);
      float vh = sqrtf(vx * vx + vy * vy), v = sqrtf(vx * vx + vy * vy + vz * vz);
      if (pgv[pos * 2] < vh) pgv[pos * 2] = vh;
      if (pgv[pos * 2 + 1] < v) pgv[pos * 2 + 1] = v;
    }
}

void oracle_fb(int it, int fb[3]) {
  static const int T[8][3] = {{-1, -1, -1}, {1, 1, -1}, {1, 1, 1},  {-1, -1, 1},
                              {-1, 1, -1},  {1, -1, -1}, {1, -1, 1}, {-1, 1, 1}};
  for (int a = 0; a < 3; ++a) fb[a] = T[it % 8][a];
}
