/*
 * wloop_b200_legacy.h -- the reference's own C entry points (include/lnk.h,
 * include/smear.h, include/wloop.h of bjoern-leder/wloop, NPROC = 1) served
 * by libwloop_b200.so.  A program written against the reference (ms10, the
 * devel/ checks) links this library in place of modules/lnk, modules/smear
 * and modules/wloop and adds one call after openQCD's geometry():
 *
 *     wloop_b200_attach(n, bc_type(), ipt, udfld);
 *
 * All smearing and loop arithmetic then runs on the GPU (FP64); the
 * openQCD field udfld() is read and written in its own layout.  Errors are
 * fatal as in the reference (error_root): the message is printed to stderr
 * and the process exits with status 1.
 *
 * When openQCD's su3.h is not included first, layout-compatible su3_dble
 * types are declared here.
 */
#ifndef WLOOP_B200_LEGACY_H
#define WLOOP_B200_LEGACY_H

#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

#ifndef SU3_H
#ifndef WLG_SU3_COMPAT
#define WLG_SU3_COMPAT
typedef struct {
  double re, im;
} complex_dble;
typedef struct {
  complex_dble c1, c2, c3;
} su3_vector_dble;
typedef struct {
  complex_dble c11, c12, c13, c21, c22, c23, c31, c32, c33;
} su3_dble;
#endif
#endif

/* MAX_SM_LEVELS raised from 5 (include/wloop.h:13) to 8. */
#ifndef MAX_SM_LEVELS
#define MAX_SM_LEVELS (8)
#endif

#define wloop_RELEASE "wloop-1.4"

typedef enum { APE, HYP, OP_SMEARS } op_smear_t; /* include/wloop.h:17-21 */

/* include/wloop.h:24-36 (nss sized by the raised level limit) */
typedef struct {
  int msl, nss[MAX_SM_LEVELS];
  int mwlt, mwlr, wls;
  op_smear_t op_smear;
  double alpha_action[3];
  double alpha_ape;
  double alpha_hyp[2];
  int proj;
  int proj_iter;
  double* wl_mat;
} wloop_parms_t;

#ifdef VOLUME
/* include/wloop.h:38-39 */
#define pindx(sl, ix, k) ((k) + 3 * ((ix) + VOLUME * (sl)))
#endif

/* Binds the library to the caller's lattice: global extents n[4] =
 * {N0,N1,N2,N3}, bc (0 open, 3 periodic), openQCD's ipt[] (lexicographic ->
 * openQCD site index) and the function returning the gauge field base
 * address (openQCD udfld()).  Has no counterpart in the reference: openQCD's
 * globals play this role there. */
void wloop_b200_attach(const int n[4], int bc, const int* ipt, su3_dble* (*udfld_fn)(void));
void wloop_b200_detach(void);

/* ---- include/smear.h:49-72 --------------------------------------------- */
void free_hyp(void);                                                     /* hyp_links.c:376 */
void hyp_time_links(double alpha1, double alpha2, double alpha3, int proj_su3, int piter,
                    int keep);                                           /* hyp_links.c:454 */
void hyp_space_links(double alpha1, double alpha2, double alpha3, int proj_su3, int piter,
                     int keep);                                          /* hyp_links.c:461 */
void hyp_links(double alpha1, double alpha2, double alpha3, int proj_su3, int piter,
               int keep);                                                /* hyp_links.c:468 */
void free_hyp_spatial(void);                                             /* hyp_spatial_links.c:268 */
void hyp_spatial_links(su3_dble* ub, double alpha1, double alpha2, int proj_su3, int piter,
                       int keep);                                        /* hyp_spatial_links.c:289 */
void free_ape_links(void);                                               /* ape_links.c:196 */
void ape_links(su3_dble* ub, double a, int proj_su3, int piter, int keep);  /* ape_links.c:275 */
void ape_spatial_links(su3_dble* ub, double a, int proj_su3, int piter,
                       int keep);                                        /* ape_links.c:281 */
void staple_sum(su3_dble* u1, su3_dble* u2, int mu, int nu, su3_dble* vb,
                su3_dble* cbuf);                                         /* staple_sum.c:53 */
void approx_project_to_su3_dble(su3_dble* u, int iter);                  /* projection.c:120 */

/* ---- include/lnk.h:16-53 (NPROC = 1: the copy and send routines have no
 * boundary to exchange and return immediately) ------------------------- */
void copy_bnd(su3_dble* ub);
void copy_u0(su3_dble* ub);
void copyback_u0(su3_dble* ub);
void copy_u0n(su3_dble* ub);
void copyback_u0n(su3_dble* ub);
void copy_uk(su3_dble* ub);
void copyback_uk(su3_dble* ub);
void send_uk(su3_dble* ub, su3_dble* sbuf);
void free_lnk(su3_dble* ub, int cb);                                     /* lnkcom.c:719 */
void free_buf_uk(su3_dble* ub);
su3_dble* alloc_lnk(void);                                               /* lnkcom.c:766 */
su3_dble* alloc_buf_uk(void);
su3_dble* lnk_buf(su3_dble* ub, int ix, int mu, int face);
su3_dble* lnkf(su3_dble* ub, int ix, int mu, int face);                  /* lnkcom.c:862 */
su3_dble* lnk(su3_dble* ub, int ix, int mu);                             /* lnkcom.c:880 */
void lnk_plaq(su3_dble* ub, int ix, int mu, int nu, su3_dble** u);       /* lnkcom.c:886 */
void assign_lnk2lnk(su3_dble* ub1, su3_dble* ub2);                       /* lnkcom.c:899 */
void assign_ud2lnk(su3_dble* ub);                                        /* lnkcom.c:915 */
void assign_lnk2ud(su3_dble* ub);                                        /* lnkcom.c:931 */
int* get_lnk_idx_u0(void);
int* get_lnk_idx_uk(void);
void add_up_staple(su3_dble* u1o, su3_dble* u2o, int ix, int mu, int nu, su3_dble* v);
void add_dn_staple(su3_dble* u1o, su3_dble* u2o, int ix, int mu, int nu, su3_dble* v);
void add_up_staple_lnks(su3_dble* u1, su3_dble* u2, su3_dble* u3, su3_dble* v);
void add_dn_staple_lnks(su3_dble* u1, su3_dble* u2, su3_dble* u3, su3_dble* v);
void add_up_staple_save(su3_dble* u1o, su3_dble* u2o, int ix, int mu, int nu, su3_dble* v);
void add_dn_staple_save(su3_dble* u1o, su3_dble* u2o, int ix, int mu, int nu, su3_dble* v);
void add_up_staple_lnks_save(su3_dble* u1, su3_dble* u2, su3_dble* u3, su3_dble* v);
void add_dn_staple_lnks_save(su3_dble* u1, su3_dble* u2, su3_dble* u3, su3_dble* v);
double lnk_plaq_sum(su3_dble* ub);                                       /* lnkplaq.c:117 */

/* ---- include/wloop.h:45-66 ---------------------------------------------- */
void free_wloop(void);                                                   /* wloop.c:511 */
void wloop_sum(int keep);                                                /* wloop.c:611 */
wloop_parms_t set_wloop_parms(int msl, int nss[], int mwlt, int mwlr, op_smear_t op_smear,
                              double alpha_action[3], double alpha_ape, double alpha_hyp[2],
                              int proj_iter);                            /* wloop_parms.c:96 */
wloop_parms_t wloop_parms(void);                                         /* wloop_parms.c:197 */
/* Reads the [Wloop] section from stdin (wloop_parms.c:203-285). */
void read_wloop_parms(void);
void print_wloop_parms(void);                                            /* wloop_parms.c:288 */
void write_wloop_parms(FILE* fdat);                                      /* wloop_parms.c:343 */
void check_wloop_parms(FILE* fdat);                                      /* wloop_parms.c:385 */
int wl_idx(int sl1, int sl2, int t, int r, int x0);                      /* wloop_parms.c:431 */
void smear(void);                                                        /* smear.c:99 */
su3_dble** get_pus(void);                                                /* smear.c:124 */
void free_smear(void);                                                   /* smear.c:130 */

#ifdef __cplusplus
}
#endif
#endif
