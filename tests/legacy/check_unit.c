/*
 * check_unit.c -- a program written against the reference's C API
 * (hyp_time_links, read_wloop_parms, wloop_sum, wloop_parms, wl_idx), linked
 * with libwloop_b200.so: the unit-field check of devel/wloop/check1.c.
 * Every Wilson loop of the unit field is 1, except loops crossing an open
 * time boundary, which are 0.
 *
 * Usage: check_unit <bc> < input   (input holds a [Wloop] section)
 * A minimal stand-in for openQCD's geometry() and udfld() is defined here.
 */
#include <float.h>
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "wloop_b200_legacy.h"

#define N0 8
#define N1 4
#define N2 4
#define N3 6
#define VOL (N0 * N1 * N2 * N3)

static int ipt[VOL];
static su3_dble* ud;

static su3_dble* udfld(void) { return ud; }

/* even points first, lexicographic within each parity */
static void geometry(void) {
  int s, ne = 0, no = VOL / 2;
  for (s = 0; s < VOL; s++) {
    int x3 = s % N3, x2 = (s / N3) % N2, x1 = (s / (N3 * N2)) % N1, x0 = s / (N3 * N2 * N1);
    if ((x0 + x1 + x2 + x3) % 2 == 0)
      ipt[s] = ne++;
    else
      ipt[s] = no++;
  }
}

int main(int argc, char* argv[]) {
  int bc = (argc > 1) ? atoi(argv[1]) : 3;
  int n[4] = {N0, N1, N2, N3};
  int s, mu, x0, t, r, sl1, sl2, status = 0;
  double eps;
  wloop_parms_t wl;

  geometry();
  ud = calloc(4 * VOL, sizeof(su3_dble));
  wloop_b200_attach(n, bc, ipt, udfld);
  for (s = 0; s < VOL; s++)
    for (mu = 0; mu < 4; mu++) {
      su3_dble* u = lnk(ud, ipt[s], mu);
      memset(u, 0, sizeof(*u));
      if (!(bc == 0 && mu == 0 && s / (N1 * N2 * N3) == N0 - 1))
        u->c11.re = u->c22.re = u->c33.re = 1.0;
    }

  read_wloop_parms();
  wl = wloop_parms();
  print_wloop_parms();

  hyp_time_links(wl.alpha_action[0], wl.alpha_action[1], wl.alpha_action[2], wl.proj,
                 wl.proj_iter, 0);
  wloop_sum(1);
  wl = wloop_parms();

  eps = sqrt(3.0) * ((double)(N0 * N1 / 4)) * DBL_EPSILON; /* devel/wloop/check1.c:108 */
  for (x0 = 0; x0 < N0; x0++)
    for (r = 0; r < wl.mwlr; r++)
      for (t = 0; t < wl.mwlt; t++)
        for (sl2 = 0; sl2 < wl.msl; sl2++)
          for (sl1 = 0; sl1 < wl.msl; sl1++) {
            double w = wl.wl_mat[wl_idx(sl1, sl2, t, r, x0)];
            int crosses = (bc == 0) && (x0 + t + 1 > N0 - 1);
            if (crosses ? (w != 0.0) : (fabs(1.0 - w) > eps)) {
              printf("bad W(sl1=%d,sl2=%d,t=%d,r=%d,x0=%d) = %.17g\n", sl1, sl2, t, r, x0, w);
              status = 1;
            }
          }
  printf("unit field check: %s\n", status ? "FAILED" : "ok");
  free_wloop();
  free(ud);
  return status;
}
