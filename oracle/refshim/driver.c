/*
 * driver.c -- ctypes entry points into the reference's own wloop modules
 * (compiled unchanged from their sources against shim.h; oracle/_ref).
 * TEST INFRASTRUCTURE ONLY: the checker for the oracle and the CUDA path,
 * and the reference leg of the CPU timing.  Never linked by the product.
 *
 * Fields cross this boundary in the lexicographic su3_dble layout the
 * product and the oracle use: link (s, mu) at [4*s+mu], s = x3 + N3*(x2 +
 * N2*(x1 + N1*x0)), 18 doubles per link (rows c11..c33, re/im).  The
 * measurement follows ms10's set_data (main/ms10.c:633-646): hyp_links on
 * the gauge field, then wloop_sum, which smears the spatial links level by
 * level and fills wloop_parms().wl_mat.
 */
#include <stdlib.h>
#include <string.h>
#include "shim.h"
#include "lnk.h"
#include "smear.h"
#include "wloop.h"

static int initialised = 0;

static void init(void)
{
  if (!initialised) {
    geometry();
    initialised = 1;
  }
}

/* lattice extents (N0..N3) of this library; returns its MAX_SM_LEVELS */
int wlref_dims(int n[4])
{
  n[0] = N0; n[1] = N1; n[2] = N2; n[3] = N3;
  return MAX_SM_LEVELS;
}

static int lex_of(int ix, int x[4])
{
  /* coordinates of the openQCD site ix, by search over the lexicographic
   * index (ipt is a bijection) */
  static int *inv = NULL;
  int s;
  if (inv == NULL) {
    inv = malloc(VOLUME * sizeof(int));
    for (s = 0; s < VOLUME; s++)
      inv[ipt[s]] = s;
  }
  s = inv[ix];
  x[3] = s % L3;
  x[2] = (s / L3) % L2;
  x[1] = (s / (L3 * L2)) % L1;
  x[0] = s / (L3 * L2 * L1);
  return s;
}

static int lexi4(const int x[4])
{
  return x[3] + L3 * (x[2] + L2 * (x[1] + L1 * x[0]));
}

/* the gauge field from the lexicographic layout, then set_bc() */
void wlref_set_field(int bc, const double *lex)
{
  int ix, mu, s, x[4], y[4], ls[4];
  su3_dble *u;

  init();
  wlref_set_bc_type(bc);
  u = udfld();
  ls[0] = L0; ls[1] = L1; ls[2] = L2; ls[3] = L3;
  for (ix = VOLUME / 2; ix < VOLUME; ix++) {
    s = lex_of(ix, x);
    for (mu = 0; mu < 4; mu++) {
      memcpy(u + 8 * (ix - VOLUME / 2) + 2 * mu, lex + 18 * (4 * (size_t)s + mu),
             sizeof(su3_dble));
      memcpy(y, x, sizeof(y));
      y[mu] = (x[mu] + ls[mu] - 1) % ls[mu];
      memcpy(u + 8 * (ix - VOLUME / 2) + 2 * mu + 1, lex + 18 * (4 * (size_t)lexi4(y) + mu),
             sizeof(su3_dble));
    }
  }
  set_bc();
}

/* the gauge field back into the lexicographic layout */
void wlref_get_field(double *lex)
{
  int ix, mu, s, x[4];
  su3_dble *u;

  init();
  u = udfld();
  for (ix = 0; ix < VOLUME; ix++) {
    s = lex_of(ix, x);
    for (mu = 0; mu < 4; mu++)
      memcpy(lex + 18 * (4 * (size_t)s + mu), lnk(u, ix, mu), sizeof(su3_dble));
  }
}

/* which = 0: hyp_links, 1: hyp_time_links, 2: hyp_space_links */
void wlref_hyp(int which, double a1, double a2, double a3, int proj, int piter)
{
  init();
  if (which == 1)
    hyp_time_links(a1, a2, a3, proj, piter, 0);
  else if (which == 2)
    hyp_space_links(a1, a2, a3, proj, piter, 0);
  else
    hyp_links(a1, a2, a3, proj, piter, 0);
}

/* nsweeps APE sweeps of the gauge field (all four directions when time != 0) */
void wlref_ape(double alpha, int proj, int piter, int time, int nsweeps)
{
  int i;
  init();
  for (i = 0; i < nsweeps; i++) {
    if (time)
      ape_links(udfld(), alpha, proj, piter, 0);
    else
      ape_spatial_links(udfld(), alpha, proj, piter, 0);
  }
}

void wlref_hyp_spatial(double a1, double a2, int proj, int piter, int nsweeps)
{
  int i;
  init();
  for (i = 0; i < nsweeps; i++)
    hyp_spatial_links(udfld(), a1, a2, proj, piter, 0);
}

double wlref_plaq_sum(void)
{
  init();
  return lnk_plaq_sum(udfld());
}

void wlref_project(double *m, int iter)
{
  approx_project_to_su3_dble((su3_dble *)m, iter);
}

static void set_parms(int msl, const int *nss, int mwlt, int mwlr, int op_smear,
                      const double *alpha_action, double alpha_ape, const double *alpha_hyp,
                      int proj_iter)
{
  int k, n[MAX_SM_LEVELS];
  double aa[3], ah[2];
  error(msl < 1 || msl > MAX_SM_LEVELS, 1, "set_parms [driver.c]",
        "msl=%d is outside 1..MAX_SM_LEVELS of this library", msl);
  for (k = 0; k < msl; k++)
    n[k] = nss[k];
  aa[0] = alpha_action[0]; aa[1] = alpha_action[1]; aa[2] = alpha_action[2];
  ah[0] = alpha_hyp[0]; ah[1] = alpha_hyp[1];
  set_wloop_parms(msl, n, mwlt, mwlr, op_smear == 1 ? HYP : APE, aa, alpha_ape, ah, proj_iter);
}

static int copy_out(double *out)
{
  wloop_parms_t wl = wloop_parms();
  memcpy(out, wl.wl_mat, (size_t)wl.wls * sizeof(double));
  return wl.wls;
}

/* wloop_sum on the current gauge field (no action smearing); returns wls */
int wlref_wloop_sum(int msl, const int *nss, int mwlt, int mwlr, int op_smear,
                    const double *alpha_action, double alpha_ape, const double *alpha_hyp,
                    int proj_iter, double *out)
{
  init();
  set_parms(msl, nss, mwlt, mwlr, op_smear, alpha_action, alpha_ape, alpha_hyp, proj_iter);
  wloop_sum(0);
  free_smear();
  return copy_out(out);
}

/* ms10's per-configuration work (set_data): hyp_links with the action
 * parameters, then wloop_sum; returns wls */
int wlref_measure(int msl, const int *nss, int mwlt, int mwlr, int op_smear,
                  const double *alpha_action, double alpha_ape, const double *alpha_hyp,
                  int proj_iter, double *out)
{
  wloop_parms_t wl;
  init();
  set_parms(msl, nss, mwlt, mwlr, op_smear, alpha_action, alpha_ape, alpha_hyp, proj_iter);
  wl = wloop_parms();
  hyp_links(wl.alpha_action[0], wl.alpha_action[1], wl.alpha_action[2], wl.proj, wl.proj_iter,
            0);
  wloop_sum(0);
  free_smear();
  return copy_out(out);
}
