/*
 * wloop_oracle.c -- FP64 CPU restatement of the wloop measurement path
 * (bjoern-leder/wloop: modules/smear, modules/lnk, modules/wloop).
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the timed CPU
 * baseline.  The product library never links or calls this file.
 *
 * The functions follow the reference's loop order and operation order
 * (each cites the file:line it restates).  The reference's MPI halo code is
 * the identity at NPROC=1 and is left out; openQCD's su3 products
 * (su3xsu3, su3dagxsu3, su3xsu3dag, _vector_prod_re) are restated from their
 * mathematical definition.  Site order is lexicographic (openQCD's ipt[]
 * argument order); openQCD's internal even/odd site order only changes the
 * order of floating-point sums.
 *
 * Pinned to the reference itself: its modules, compiled unchanged against a
 * one-process openQCD interface (refshim/, `make ref`), agree with this file
 * to 1e-13 function by function and on whole measurements
 * (tests/test_reference.py).
 */
#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#include "wloop_oracle.h"

typedef struct {
  double re, im;
} cplx;

/* row-major 3x3 complex: c[i][j] is openQCD's c(i+1)(j+1) */
typedef struct {
  cplx c[3][3];
} su3;

#define SRT18 4.242640687119285

typedef struct {
  int n[4];
  int vol;
  int *iup; /* [vol][4] */
  int *idn; /* [vol][4] */
} geom;

static void geom_init(geom *g, const int n[4]) {
  int x[4], mu, ix;
  memcpy(g->n, n, 4 * sizeof(int));
  g->vol = n[0] * n[1] * n[2] * n[3];
  g->iup = (int *)malloc(sizeof(int) * 4 * (size_t)g->vol);
  g->idn = (int *)malloc(sizeof(int) * 4 * (size_t)g->vol);
  for (ix = 0; ix < g->vol; ix++) {
    int r = ix;
    x[3] = r % n[3]; r /= n[3];
    x[2] = r % n[2]; r /= n[2];
    x[1] = r % n[1]; r /= n[1];
    x[0] = r;
    for (mu = 0; mu < 4; mu++) {
      int y[4], z[4], k;
      for (k = 0; k < 4; k++) y[k] = z[k] = x[k];
      y[mu] = (x[mu] + 1) % n[mu];
      z[mu] = (x[mu] + n[mu] - 1) % n[mu];
      g->iup[4 * ix + mu] = y[3] + n[3] * (y[2] + n[2] * (y[1] + n[1] * y[0]));
      g->idn[4 * ix + mu] = z[3] + n[3] * (z[2] + n[2] * (z[1] + n[1] * z[0]));
    }
  }
}

static void geom_free(geom *g) {
  free(g->iup);
  free(g->idn);
}

static int site(const geom *g, int x0, int x1, int x2, int x3) {
  return x3 + g->n[3] * (x2 + g->n[2] * (x1 + g->n[1] * x0));
}

int orc_version(void) { return 1; }

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* ---------------------------------------------------------------------------
 * SU(3) algebra (openQCD su3fcts restated from the definitions).
 * w must not alias u or v.
 * ------------------------------------------------------------------------- */

/* w = u*v */
static void su3xsu3(const su3 *u, const su3 *v, su3 *w) {
  int i, j;
  for (i = 0; i < 3; i++)
    for (j = 0; j < 3; j++) {
      w->c[i][j].re = u->c[i][0].re * v->c[0][j].re - u->c[i][0].im * v->c[0][j].im +
                      u->c[i][1].re * v->c[1][j].re - u->c[i][1].im * v->c[1][j].im +
                      u->c[i][2].re * v->c[2][j].re - u->c[i][2].im * v->c[2][j].im;
      w->c[i][j].im = u->c[i][0].re * v->c[0][j].im + u->c[i][0].im * v->c[0][j].re +
                      u->c[i][1].re * v->c[1][j].im + u->c[i][1].im * v->c[1][j].re +
                      u->c[i][2].re * v->c[2][j].im + u->c[i][2].im * v->c[2][j].re;
    }
}

/* w = u^dag * v */
static void su3dagxsu3(const su3 *u, const su3 *v, su3 *w) {
  int i, j;
  for (i = 0; i < 3; i++)
    for (j = 0; j < 3; j++) {
      w->c[i][j].re = u->c[0][i].re * v->c[0][j].re + u->c[0][i].im * v->c[0][j].im +
                      u->c[1][i].re * v->c[1][j].re + u->c[1][i].im * v->c[1][j].im +
                      u->c[2][i].re * v->c[2][j].re + u->c[2][i].im * v->c[2][j].im;
      w->c[i][j].im = u->c[0][i].re * v->c[0][j].im - u->c[0][i].im * v->c[0][j].re +
                      u->c[1][i].re * v->c[1][j].im - u->c[1][i].im * v->c[1][j].re +
                      u->c[2][i].re * v->c[2][j].im - u->c[2][i].im * v->c[2][j].re;
    }
}

/* w = u * v^dag */
static void su3xsu3dag(const su3 *u, const su3 *v, su3 *w) {
  int i, j;
  for (i = 0; i < 3; i++)
    for (j = 0; j < 3; j++) {
      w->c[i][j].re = u->c[i][0].re * v->c[j][0].re + u->c[i][0].im * v->c[j][0].im +
                      u->c[i][1].re * v->c[j][1].re + u->c[i][1].im * v->c[j][1].im +
                      u->c[i][2].re * v->c[j][2].re + u->c[i][2].im * v->c[j][2].im;
      w->c[i][j].im = u->c[i][0].im * v->c[j][0].re - u->c[i][0].re * v->c[j][0].im +
                      u->c[i][1].im * v->c[j][1].re - u->c[i][1].re * v->c[j][1].im +
                      u->c[i][2].im * v->c[j][2].re - u->c[i][2].re * v->c[j][2].im;
    }
}

static void su3_add(su3 *u, const su3 *v) {
  int i, j;
  for (i = 0; i < 3; i++)
    for (j = 0; j < 3; j++) {
      u->c[i][j].re = u->c[i][j].re + v->c[i][j].re;
      u->c[i][j].im = u->c[i][j].im + v->c[i][j].im;
    }
}

static void su3_mulr(su3 *z, double a, const su3 *u) {
  int i, j;
  for (i = 0; i < 3; i++)
    for (j = 0; j < 3; j++) {
      z->c[i][j].re = a * u->c[i][j].re;
      z->c[i][j].im = a * u->c[i][j].im;
    }
}

/* _su3_lcomb (include/smear.h:9-27): z = a*u + b*v */
static void su3_lcomb(su3 *z, double a, const su3 *u, double b, const su3 *v) {
  int i, j;
  for (i = 0; i < 3; i++)
    for (j = 0; j < 3; j++) {
      z->c[i][j].re = (a * u->c[i][j].re + b * v->c[i][j].re);
      z->c[i][j].im = (a * u->c[i][j].im + b * v->c[i][j].im);
    }
}

/* _vector_prod_re summed over the three rows: Re tr(a^dag b) */
static double re_tr_dag(const su3 *a, const su3 *b) {
  int i;
  double s[3];
  for (i = 0; i < 3; i++)
    s[i] = a->c[i][0].re * b->c[i][0].re + a->c[i][0].im * b->c[i][0].im +
           a->c[i][1].re * b->c[i][1].re + a->c[i][1].im * b->c[i][1].im +
           a->c[i][2].re * b->c[i][2].re + a->c[i][2].im * b->c[i][2].im;
  return s[0] + s[1] + s[2];
}

/* ---------------------------------------------------------------------------
 * projection.c:87-154
 * ------------------------------------------------------------------------- */

/* det_im_dble, projection.c:87-117 */
static double det_im(const su3 *u) {
  cplx d1, d2, d3;
  const cplx *c = &u->c[0][0];
  /* c[0]=c11 c[1]=c12 c[2]=c13 c[3]=c21 ... c[8]=c33 */
  d1.re = (c[4].re * c[8].re - c[4].im * c[8].im) - (c[5].re * c[7].re - c[5].im * c[7].im);
  d1.im = (c[4].re * c[8].im + c[4].im * c[8].re) - (c[5].re * c[7].im + c[5].im * c[7].re);
  d2.re = (c[3].re * c[8].re - c[3].im * c[8].im) - (c[5].re * c[6].re - c[5].im * c[6].im);
  d2.im = (c[3].re * c[8].im + c[3].im * c[8].re) - (c[5].re * c[6].im + c[5].im * c[6].re);
  d3.re = (c[3].re * c[7].re - c[3].im * c[7].im) - (c[4].re * c[6].re - c[4].im * c[6].im);
  d3.im = (c[3].re * c[7].im + c[3].im * c[7].re) - (c[4].re * c[6].im + c[4].im * c[6].re);
  return (c[0].re * d1.im + c[0].im * d1.re) - (c[1].re * d2.im + c[1].im * d2.re) +
         (c[2].re * d3.im + c[2].im * d3.re);
}

/* approx_project_to_su3_dble, projection.c:120-154 */
static void project(su3 *u, int iter) {
  int i, j, it;
  double d = 0.0, zim;
  su3 x, y;
  for (i = 0; i < 3; i++)
    for (j = 0; j < 3; j++) d += u->c[i][j].re * u->c[i][j].re + u->c[i][j].im * u->c[i][j].im;
  if (d < SRT18 * DBL_EPSILON) return; /* :136 zero guard */
  d = 1.0 / sqrt(d / 3.0);
  su3_mulr(u, d, u);
  for (it = 0; it < iter; it++) {
    su3dagxsu3(u, u, &x);
    su3_mulr(&x, -0.5, &x);
    x.c[0][0].re += 1.5;
    x.c[1][1].re += 1.5;
    x.c[2][2].re += 1.5;
    su3xsu3(u, &x, &y);
    zim = det_im(&y);
    zim /= -3.0;
    /* _su3_mulc with z = 1 + i*zim */
    for (i = 0; i < 3; i++)
      for (j = 0; j < 3; j++) {
        u->c[i][j].re = 1.0 * y.c[i][j].re - zim * y.c[i][j].im;
        u->c[i][j].im = 1.0 * y.c[i][j].im + zim * y.c[i][j].re;
      }
  }
}

void orc_project(double *u, int iter) { project((su3 *)u, iter); }

/* ---------------------------------------------------------------------------
 * staple_sum.c:53-87, add_up/dn_staple_save lnkstaple.c:318-382.
 * For every x: vb(x,mu) += u1(x,nu) u2(x+nu,mu) u1(x+mu,nu)^dag
 *                        + u1(x-nu,nu)^dag u2(x-nu,mu) u1(x-nu+mu,nu)
 * ------------------------------------------------------------------------- */
static void staple_sum(const geom *g, const su3 *u1, const su3 *u2, int mu, int nu, su3 *vb) {
  int ix;
#pragma omp parallel for schedule(static)
  for (ix = 0; ix < g->vol; ix++) {
    su3 tmp, tmp2;
    su3 *v = vb + 4 * ix + mu;
    int iy, iz;
    /* up staple: su3xsu3dag(u2,u3) then su3xsu3(u1,.) */
    iy = g->iup[4 * ix + nu];
    iz = g->iup[4 * ix + mu];
    su3xsu3dag(u2 + 4 * iy + mu, u1 + 4 * iz + nu, &tmp);
    su3xsu3(u1 + 4 * ix + nu, &tmp, &tmp2);
    su3_add(v, &tmp2);
    /* down staple: su3xsu3(u2,u3) then su3dagxsu3(u1,.) */
    iy = g->idn[4 * ix + nu];
    iz = g->iup[4 * iy + mu];
    su3xsu3(u2 + 4 * iy + mu, u1 + 4 * iz + nu, &tmp);
    su3dagxsu3(u1 + 4 * iy + nu, &tmp, &tmp2);
    su3_add(v, &tmp2);
  }
}

void orc_staple_sum(const int n[4], const double *u1, const double *u2, int mu, int nu,
                    double *vb) {
  geom g;
  geom_init(&g, n);
  staple_sum(&g, (const su3 *)u1, (const su3 *)u2, mu, nu, (su3 *)vb);
  geom_free(&g);
}

static void set_bc(const geom *g, int bc, su3 *ud) {
  /* openQCD set_bc() for open bc: temporal links at x0=N0-1 are zero */
  int ixs, vs;
  if (bc != 0) return;
  vs = g->n[1] * g->n[2] * g->n[3];
  for (ixs = 0; ixs < vs; ixs++) memset(ud + 4 * ((g->n[0] - 1) * vs + ixs), 0, sizeof(su3));
}

/* ---------------------------------------------------------------------------
 * hyp_links.c:128-451
 * ------------------------------------------------------------------------- */
static const int hyp_pair[4][4] = {
    /* dlnks_idx, hyp_links.c:128-139: {01,23}->0, {02,13}->1, {03,12}->2 */
    {0, 0, 1, 2},
    {0, 0, 2, 1},
    {1, 2, 0, 0},
    {2, 1, 0, 0}};

/* decorate / decorate_all, hyp_links.c:154-191 */
static void decorate(const geom *g, const su3 *udb, su3 *vb, double a, double b, int mu0, int mu1,
                     int proj, int iter) {
  int ix;
#pragma omp parallel for schedule(static)
  for (ix = 0; ix < g->vol; ix++) {
    int mu;
    for (mu = mu0; mu < mu1; mu++) {
      su3 *v = vb + 4 * ix + mu;
      su3_lcomb(v, a, udb + 4 * ix + mu, b, v);
      if (proj) project(v, iter);
    }
  }
}

void orc_hyp_links(const int n[4], int bc, double *udp, double a1, double a2, double a3, int proj,
                   int piter, int time, int space) {
  geom g;
  su3 *ud = (su3 *)udp, *dl[6];
  size_t nl;
  double alpha[3], beta[3], a[3];
  int i, mu, nu, rho, eta, mu0, mu1, ix;

  if (a1 == 0.0) return; /* :405 */
  geom_init(&g, n);
  nl = 4 * (size_t)g.vol;
  for (i = 0; i < 6; i++) dl[i] = (su3 *)calloc(nl, sizeof(su3));
  memcpy(dl[3], ud, nl * sizeof(su3)); /* assign_ud2lnk(dlnks[3]) :412 */
  a[0] = a1;
  a[1] = a2;
  a[2] = a3;
  for (i = 0; i < 3; i++) { /* :419-423 */
    alpha[i] = 1.0 - a[i];
    beta[i] = a[i] / (double)(2 * (3 - i));
  }

  /* decorated_links1 (:320-373): level with alpha3 */
  for (i = 0; i < 3; i++) memset(dl[i], 0, nl * sizeof(su3));
  for (mu = 0; mu < 4; mu++)
    for (i = 1; i < 4; i++) {
      eta = (mu + i) & 0x3;
      staple_sum(&g, dl[3], dl[3], mu, eta, dl[hyp_pair[mu][eta]]);
    }
  for (i = 0; i < 3; i++) decorate(&g, ud, dl[i], alpha[2], beta[2], 0, 4, proj, piter);

  /* decorated_links2 (:244-317): level with alpha2 */
  for (i = 0; i < 3; i++) memset(dl[3 + i], 0, nl * sizeof(su3));
  for (mu = 0; mu < 4; mu++)
    for (i = 1; i < 4; i++) {
      int d, nidx;
      nu = (mu + i) & 0x3;
      nidx = hyp_pair[mu][nu];
      d = nu + mu;
      if (d > 3) d = 6 - d;
      for (rho = 0; rho < 4; rho++) {
        if ((rho != mu) && (rho != nu)) {
          int d2 = nu + rho;
          if (d2 > 3) d2 = 6 - d2;
          staple_sum(&g, dl[d - 1], dl[d2 - 1], mu, rho, dl[3 + nidx]);
        }
      }
    }
  for (i = 0; i < 3; i++) decorate(&g, ud, dl[3 + i], alpha[1], beta[1], 0, 4, proj, piter);

  /* decorated_links3 (:194-241): level with alpha1 */
  mu0 = 1 - (time > 0);
  mu1 = 1 + 3 * (space > 0);
  memset(dl[0], 0, nl * sizeof(su3));
  for (mu = mu0; mu < mu1; mu++)
    for (i = 1; i < 4; i++) {
      nu = (mu + i) & 0x3;
      staple_sum(&g, dl[3 + hyp_pair[nu][mu]], dl[3 + hyp_pair[mu][nu]], mu, nu, dl[0]);
    }
  decorate(&g, ud, dl[0], alpha[0], beta[0], mu0, mu1, proj, piter);

  /* copy back (:432-444) and set_bc (:447) */
  for (ix = 0; ix < g.vol; ix++)
    for (mu = mu0; mu < mu1; mu++) ud[4 * ix + mu] = dl[0][4 * ix + mu];
  set_bc(&g, bc, ud);

  for (i = 0; i < 6; i++) free(dl[i]);
  geom_free(&g);
}

/* ---------------------------------------------------------------------------
 * ape_links.c:147-272
 * ------------------------------------------------------------------------- */
static void ape_links(const geom *g, su3 *ub, double alpha, int proj, int piter, int time,
                      su3 *vo, su3 *u) {
  size_t nl = 4 * (size_t)g->vol;
  int mu, eta, ix, mu0 = 1 - (time > 0);
  memcpy(u, ub, nl * sizeof(su3)); /* assign_lnk2lnk(pub,dlnks[1]) :230 */
  memset(vo, 0, nl * sizeof(su3));
  for (mu = mu0; mu < 4; mu++)
    for (eta = mu0; eta < 4; eta++)
      if (eta != mu) staple_sum(g, u, u, mu, eta, vo); /* :162-169 */
#pragma omp parallel for schedule(static)
  for (ix = 0; ix < g->vol; ix++) { /* :239-262 */
    int m;
    for (m = mu0; m < 4; m++) {
      su3 *v = vo + 4 * ix + m, *w = ub + 4 * ix + m;
      su3_mulr(v, alpha, v);
      su3_add(w, v);
      if (proj) project(w, piter);
    }
  }
}

void orc_ape_links(const int n[4], double *ub, double alpha, int proj, int piter, int time) {
  geom g;
  su3 *vo, *u;
  geom_init(&g, n);
  vo = (su3 *)malloc(4 * (size_t)g.vol * sizeof(su3));
  u = (su3 *)malloc(4 * (size_t)g.vol * sizeof(su3));
  ape_links(&g, (su3 *)ub, alpha, proj, piter, time, vo, u);
  free(vo);
  free(u);
  geom_free(&g);
}

/* ---------------------------------------------------------------------------
 * hyp_spatial_links.c:117-344
 * ------------------------------------------------------------------------- */
static const int hyp3_pair[4][4] = {
    /* dlnks_idx, hyp_spatial_links.c:117-125 (note: not symmetric) */
    {0, 0, 0, 0},
    {0, 0, 0, 1},
    {0, 0, 0, 1},
    {0, 0, 1, 0}};

static void hyp_spatial_links(const geom *g, su3 *pub, double a1, double a2, int proj, int piter,
                              su3 *dl[3]) {
  size_t nl = 4 * (size_t)g->vol;
  double alpha[2], beta[2], a[2];
  int i, mu, nu, eta, ix;
  memcpy(dl[2], pub, nl * sizeof(su3)); /* :304 */
  a[0] = a1;
  a[1] = a2;
  for (i = 0; i < 2; i++) { /* :310-314 */
    alpha[i] = 1.0 - a[i];
    beta[i] = a[i] / (double)(2 * (2 - i));
  }
  /* decorated_links1 (:210-265) */
  for (i = 0; i < 2; i++) memset(dl[i], 0, nl * sizeof(su3));
  for (mu = 1; mu < 4; mu++)
    for (i = 0; i < 2; i++) {
      eta = ((mu + i) % 3) + 1;
      staple_sum(g, dl[2], dl[2], mu, eta, dl[hyp3_pair[mu][eta]]);
    }
  for (i = 0; i < 2; i++) decorate(g, pub, dl[i], alpha[1], beta[1], 1, 4, proj, piter);
  /* decorated_links2 (:160-207) */
  memset(dl[2], 0, nl * sizeof(su3));
  for (mu = 1; mu < 4; mu++)
    for (i = 0; i < 2; i++) {
      nu = ((mu + i) % 3) + 1;
      staple_sum(g, dl[hyp3_pair[nu][mu]], dl[hyp3_pair[mu][nu]], mu, nu, dl[2]);
    }
  decorate(g, pub, dl[2], alpha[0], beta[0], 1, 4, proj, piter);
  /* copy back spatial links (:322-334) */
  for (ix = 0; ix < g->vol; ix++)
    for (mu = 1; mu < 4; mu++) pub[4 * ix + mu] = dl[2][4 * ix + mu];
}

void orc_hyp_spatial_links(const int n[4], double *ub, double a1, double a2, int proj, int piter) {
  geom g;
  su3 *dl[3];
  int i;
  geom_init(&g, n);
  for (i = 0; i < 3; i++) dl[i] = (su3 *)malloc(4 * (size_t)g.vol * sizeof(su3));
  hyp_spatial_links(&g, (su3 *)ub, a1, a2, proj, piter, dl);
  for (i = 0; i < 3; i++) free(dl[i]);
  geom_free(&g);
}

/* ---------------------------------------------------------------------------
 * lnkplaq.c:48-128
 * ------------------------------------------------------------------------- */
static double plaq_dble(const geom *g, const su3 *ub, int ix, int mu, int nu) {
  su3 wd1, wd2;
  /* lnk_plaq (lnkcom.c:886-896): u0=U(x,mu) u1=U(x+mu,nu) u2=U(x,nu) u3=U(x+nu,mu) */
  su3xsu3(ub + 4 * ix + mu, ub + 4 * g->iup[4 * ix + mu] + nu, &wd1);
  su3xsu3(ub + 4 * ix + nu, ub + 4 * g->iup[4 * ix + nu] + mu, &wd2);
  return re_tr_dag(&wd1, &wd2);
}

static double plaq_sum(const geom *g, int bc, const su3 *ub) {
  enum { MAX_LEVELS = 8, BLK_LENGTH = 8 };
  int cnt[MAX_LEVELS], ix, mu, nu, k, vs = g->n[1] * g->n[2] * g->n[3];
  double smx[MAX_LEVELS], pa;
  for (k = 0; k < MAX_LEVELS; k++) {
    cnt[k] = 0;
    smx[k] = 0.0;
  }
  for (ix = 0; ix < g->vol; ix++) {
    int t = ix / vs;
    pa = 0.0;
    for (mu = 1; mu < 4; mu++) {
      if ((t < (g->n[0] - 1)) || (bc != 0)) pa += plaq_dble(g, ub, ix, mu, 0);
      for (nu = 1; nu < mu; nu++) pa += plaq_dble(g, ub, ix, mu, nu);
    }
    cnt[0] += 1;
    smx[0] += pa;
    for (k = 1; (cnt[k - 1] >= BLK_LENGTH) && (k < MAX_LEVELS); k++) {
      cnt[k] += 1;
      smx[k] += smx[k - 1];
      cnt[k - 1] = 0;
      smx[k - 1] = 0.0;
    }
  }
  pa = 0.0;
  for (k = 0; k < MAX_LEVELS; k++) pa += smx[k];
  return pa;
}

double orc_plaq_sum(const int n[4], int bc, const double *ub) {
  geom g;
  double p;
  geom_init(&g, n);
  p = plaq_sum(&g, bc, (const su3 *)ub);
  geom_free(&g);
  return p;
}

/* ---------------------------------------------------------------------------
 * smear.c:99-121 and wloop.c:153-608
 * ------------------------------------------------------------------------- */
int orc_wl_idx(int msl, int mwlt, int mwlr, int sl1, int sl2, int t, int r, int x0) {
  return (sl1 + msl * (sl2 + msl * (t + mwlt * (r + mwlr * x0)))); /* wloop_parms.c:433 */
}

int orc_wloop_sum(const int n[4], int bc, const double *udp, int msl, const int *nss, int mwlt,
                  int mwlr, int op_smear, double alpha_ape, const double *alpha_hyp,
                  int proj_iter, double *wl_mat, double *wl_abs, double *plaq, double *levels) {
  geom g;
  const su3 *ud = (const su3 *)udp;
  su3 *plnk, *s1, *s2, *s3, *pus, *u0l, *tmpk;
  int vol, vs, proj, sl, i, R, T, sl1, sl2, ix, k, x0, N0;
  size_t nl;
  double norm;

  /* set_wloop_parms ranges, wloop_parms.c:156-177 (MAX_SM_LEVELS raised) */
  if ((msl < 1) || (msl > ORC_MAX_SM_LEVELS)) return -1;
  if ((mwlt < 1) || (mwlt > n[0] / 2 + 1)) return -1;
  if ((mwlr < 1) || (mwlr > n[1] / 2 + 1) || (mwlr > n[2] / 2 + 1) || (mwlr > n[3] / 2 + 1))
    return -1;
  if ((op_smear != 0) && (op_smear != 1)) return -1;

  geom_init(&g, n);
  vol = g.vol;
  N0 = n[0];
  vs = n[1] * n[2] * n[3];
  nl = 4 * (size_t)vol;
  proj = (proj_iter > 0);
  norm = (double)9 * n[1] * n[2] * n[3]; /* wloop.c:535 */

  plnk = (su3 *)malloc(nl * sizeof(su3));
  s1 = (su3 *)malloc(nl * sizeof(su3));
  s2 = (su3 *)malloc(nl * sizeof(su3));
  s3 = (su3 *)malloc(nl * sizeof(su3));
  /* usb: 3*(2*msl)*VOLUME links, pus[pindx(sl,ix,k)] = pus + k+3*(ix+V*sl) (smear.c:54) */
  pus = (su3 *)malloc((size_t)3 * 2 * msl * vol * sizeof(su3));
  u0l = (su3 *)malloc((size_t)vol * sizeof(su3));
  tmpk = (su3 *)malloc((size_t)3 * vol * sizeof(su3));

  /* smear(), smear.c:99-121 */
  memcpy(plnk, ud, nl * sizeof(su3));
  for (sl = 0; sl < msl; sl++) {
    for (i = 0; i < nss[sl]; i++) {
      if (op_smear == 1) {
        su3 *dl[3];
        dl[0] = s1;
        dl[1] = s2;
        dl[2] = s3;
        hyp_spatial_links(&g, plnk, alpha_hyp[0], alpha_hyp[1], proj, proj_iter, dl);
      } else
        ape_links(&g, plnk, alpha_ape, proj, proj_iter, 0, s1, s2);
    }
    for (ix = 0; ix < vol; ix++) /* copy_lnk2us, smear.c:79-96 */
      for (k = 1; k < 4; k++) pus[k - 1 + 3 * (ix + (size_t)vol * sl)] = plnk[4 * ix + k];
    if (plaq) plaq[sl] = plaq_sum(&g, bc, plnk);
  }
  if (levels) memcpy(levels, pus, (size_t)3 * msl * vol * sizeof(su3));

  /* wloops(), wloop.c:524-604 */
  for (R = 1; R <= mwlr; R++) {
    for (ix = 0; ix < vol; ix++) u0l[ix] = ud[4 * ix]; /* assign_u02lnk(ud_long) :550 */
    for (T = 1; T <= mwlt; T++) {
      if (T > 1) { /* compute_u0_long, wloop.c:153-204: L_T(x) = U0(x) L_{T-1}(x+0) */
        int ixs;
#pragma omp parallel for schedule(static)
        for (ixs = 0; ixs < vs; ixs++) {
          su3 mat0 = u0l[(N0 - 1) * vs + ixs]; /* saved L_{T-1}(N0-1), :171-172 */
          int t0;
          for (t0 = 0; t0 < N0; t0++) {
            /* writes L_T(t0-1) = U0(t0-1) L_{T-1}(t0); the wrap reads the saved copy */
            int tw = (t0 + N0 - 1) % N0;
            const su3 *u2 = (t0 < N0 - 1) ? &u0l[t0 * vs + ixs] : &mat0;
            su3 r;
            su3xsu3(&ud[4 * (tw * vs + ixs)], u2, &r);
            u0l[tw * vs + ixs] = r;
          }
        }
      }
      for (sl1 = 0; sl1 < msl; sl1++) {
        for (sl2 = sl1; sl2 < msl; sl2++) {
          int p1, p2, x1;
          double *res;
          if ((R > 1) && (T == 1) && (sl1 == 0)) {
            /* compute_uk_long(sl2), wloop.c:207-258: Lk_R(x) = U_k(x) Lk_{R-1}(x+k) */
            int sll = (R > 2) ? msl + sl2 : sl2;
#pragma omp parallel for schedule(static)
            for (ix = 0; ix < vol; ix++) {
              int mu;
              for (mu = 1; mu < 4; mu++) {
                int iy = g.iup[4 * ix + mu];
                su3xsu3(&pus[mu - 1 + 3 * (ix + (size_t)vol * sl2)],
                        &pus[mu - 1 + 3 * (iy + (size_t)vol * sll)], &tmpk[3 * ix + mu - 1]);
              }
            }
            memcpy(&pus[3 * (size_t)vol * (msl + sl2)], tmpk, (size_t)3 * vol * sizeof(su3));
          }
          p1 = (R > 1) ? msl + sl1 : sl1;
          p2 = (R > 1) ? msl + sl2 : sl2;
          /* wloop_fixed_t_r_sl, wloop.c:436-508 (get_wloop :261-433) */
          res = (double *)calloc((size_t)4 * N0, sizeof(double));
#pragma omp parallel
          {
            double *lres = (double *)calloc((size_t)4 * N0, sizeof(double));
            int xx;
#pragma omp for schedule(static)
            for (xx = 0; xx < vs; xx++) {
              int x3 = xx % n[3], x2 = (xx / n[3]) % n[2];
              int xs[4];
              x1 = xx / (n[3] * n[2]);
              xs[1] = x1;
              xs[2] = x2;
              xs[3] = x3;
              for (x0 = 0; x0 < N0; x0++) {
                int ixa = site(&g, x0, x1, x2, x3);
                int ixt = site(&g, (x0 + T) % N0, x1, x2, x3);
                const su3 *ub = &u0l[ixa];
                for (k = 0; k < 3; k++) {
                  int xr[4], ixr, c;
                  const su3 *ubR, *ul1, *ul2, *um1, *um2;
                  su3 mat0, mat1;
                  double trc;
                  for (c = 1; c < 4; c++) xr[c] = xs[c];
                  xr[k + 1] = (xs[k + 1] + R) % n[k + 1];
                  ixr = site(&g, x0, xr[1], xr[2], xr[3]);
                  ubR = &u0l[ixr];
                  ul1 = &pus[k + 3 * (ixa + (size_t)vol * p1)];
                  ul2 = &pus[k + 3 * (ixa + (size_t)vol * p2)];
                  um1 = &pus[k + 3 * (ixt + (size_t)vol * p2)];
                  um2 = &pus[k + 3 * (ixt + (size_t)vol * p1)];
                  su3xsu3(ub, um1, &mat0);
                  su3xsu3(ul1, ubR, &mat1);
                  trc = re_tr_dag(&mat0, &mat1);
                  lres[x0] += trc;
                  lres[2 * N0 + x0] += fabs(trc);
                  if (sl1 != sl2) {
                    su3xsu3(ub, um2, &mat0);
                    su3xsu3(ul2, ubR, &mat1);
                    trc = re_tr_dag(&mat0, &mat1);
                    lres[x0 + N0] += trc;
                    lres[3 * N0 + x0] += fabs(trc);
                  }
                }
              }
            }
#pragma omp critical
            {
              int q;
              for (q = 0; q < 4 * N0; q++) res[q] += lres[q];
            }
            free(lres);
          }
          for (i = 0; i < N0; i++) { /* :584-597 */
            int ii = orc_wl_idx(msl, mwlt, mwlr, sl1, sl2, T - 1, R - 1, i);
            wl_mat[ii] = res[i] / norm;
            if (wl_abs) wl_abs[ii] = res[2 * N0 + i] / norm;
          }
          if (sl1 != sl2) {
            for (i = 0; i < N0; i++) {
              int ii = orc_wl_idx(msl, mwlt, mwlr, sl2, sl1, T - 1, R - 1, i);
              wl_mat[ii] = res[i + N0] / norm;
              if (wl_abs) wl_abs[ii] = res[3 * N0 + i] / norm;
            }
          }
          free(res);
        }
      }
    }
  }

  free(plnk);
  free(s1);
  free(s2);
  free(s3);
  free(pus);
  free(u0l);
  free(tmpk);
  geom_free(&g);
  return 0;
}
