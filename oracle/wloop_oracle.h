/*
 * wloop_oracle.h -- FP64 CPU restatement of the wloop measurement path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker the CUDA path is
 * compared against; only tests/, __graft_entry__.smoke() and the cpu_baseline
 * leg of bench.py may load it.  The product library never links it.
 *
 * Parity status: pinned to the reference (bjoern-leder/wloop) itself.  Its
 * modules compile unchanged against the one-process openQCD-1.4 interface in
 * refshim/ (oracle/Makefile `ref`; openQCD and MPI are not vendored), and
 * tests/test_reference.py holds this oracle to that build at 1e-13, function
 * by function and on whole measurements.  The reference's own property checks
 * (unit field, HYP == APE identity, gauge and translation invariance,
 * unitarity after projection) are restated in tests/ as well.
 *
 * Field layout: lexicographic sites ix = x3 + N3*(x2 + N2*(x1 + N1*x0))
 * (the index openQCD's ipt[] maps from), 4 links per site, link (ix,mu) at
 * u[18*(4*ix+mu)], each link a row-major 3x3 complex matrix c11..c33 stored
 * as (re,im) pairs -- the su3_dble byte layout.
 */
#ifndef WLOOP_ORACLE_H
#define WLOOP_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

#define ORC_MAX_SM_LEVELS 8

int orc_version(void);
void orc_set_threads(int n);

/* projection.c:120-154 */
void orc_project(double *u, int iter);

/* staple_sum.c:53-87 with add_{up,dn}_staple_save (lnkstaple.c:340-382) */
void orc_staple_sum(const int n[4], const double *u1, const double *u2,
                    int mu, int nu, double *vb);

/* hyp_links.c:398-451 (time/space select hyp_time_links/hyp_space_links);
 * bc==0 applies openQCD set_bc() (zero temporal links at x0=N0-1). */
void orc_hyp_links(const int n[4], int bc, double *ud, double a1, double a2,
                   double a3, int proj, int piter, int time, int space);

/* ape_links.c:217-272 (time=1: ape_links, time=0: ape_spatial_links) */
void orc_ape_links(const int n[4], double *ub, double alpha, int proj,
                   int piter, int time);

/* hyp_spatial_links.c:289-344 */
void orc_hyp_spatial_links(const int n[4], double *ub, double a1, double a2,
                           int proj, int piter);

/* lnkplaq.c:48-128 (lnk_plaq_sum) */
double orc_plaq_sum(const int n[4], int bc, const double *ub);

/*
 * smear.c:99-121 + wloop.c:153-608 (wloops, NPROC=1).
 *  ud       HYP-smeared gauge field (read only)
 *  wl_mat   msl*msl*mwlt*mwlr*N0 doubles, index wl_idx (wloop_parms.c:431)
 *  wl_abs   optional (may be NULL): same index, sum of |Re tr| / norm
 *  plaq     optional (may be NULL): msl entries, plaquette sum of the
 *           smeared field after each level (spatial links from the level,
 *           temporal links from ud)
 *  levels   optional (may be NULL): msl*V*3 links, the level store in
 *           [sl][ix][k] order (pindx, wloop.h:38-39)
 * op_smear: 0 = APE (alpha_ape), 1 = HYP (alpha_hyp[2]).
 * Returns 0, or -1 on a parameter error (set_wloop_parms ranges).
 */
int orc_wloop_sum(const int n[4], int bc, const double *ud, int msl,
                  const int *nss, int mwlt, int mwlr, int op_smear,
                  double alpha_ape, const double *alpha_hyp, int proj_iter,
                  double *wl_mat, double *wl_abs, double *plaq,
                  double *levels);

/* wloop_parms.c:431-434 */
int orc_wl_idx(int msl, int mwlt, int mwlr, int sl1, int sl2, int t, int r,
               int x0);

#ifdef __cplusplus
}
#endif
#endif
