/*
 * shim.h -- the part of openQCD-1.4's interface that the wloop modules
 * (modules/smear, modules/lnk, modules/wloop) use, restated for one process
 * (NPROC = 1) so that those modules compile unchanged.
 *
 * TEST INFRASTRUCTURE ONLY: this builds the reference itself (oracle/_ref)
 * as a checker for the oracle and the CUDA path.  Nothing in the product
 * links it.
 *
 * openQCD-1.4 is not vendored with the reference.  Every declaration below
 * is written from what the modules need (call sites cited in each header):
 * the su3 types and products, the lattice geometry (ipt, iup, idn with
 * periodic index wraps on one process), the gauge field udfld() in openQCD's
 * odd-point layout, set_bc() for open (0) and periodic (3) boundary
 * conditions, flags, allocation and error helpers, and an MPI stand-in for
 * one rank.  The lattice size is fixed at compile time (-DL0=.. -DL3=..), as
 * in openQCD's global.h.  ANSI C89, like the reference's own flags.
 */
#ifndef WLREF_SHIM_H
#define WLREF_SHIM_H

#include <stdio.h>
#include <float.h>

/* ---- global.h: compile-time lattice and process grid ------------------- */
#if !(defined L0) || !(defined L1) || !(defined L2) || !(defined L3)
#error "compile with -DL0=.. -DL1=.. -DL2=.. -DL3=.."
#endif
#define NPROC0 1
#define NPROC1 1
#define NPROC2 1
#define NPROC3 1
#define NPROC (NPROC0*NPROC1*NPROC2*NPROC3)
#define N0 (NPROC0*L0)
#define N1 (NPROC1*L1)
#define N2 (NPROC2*L2)
#define N3 (NPROC3*L3)
#define VOLUME (L0*L1*L2*L3)
/* with one process in a direction its faces are wrapped locally */
#define FACE0 0
#define FACE1 0
#define FACE2 0
#define FACE3 0
#define BNDRY (2*(FACE0+FACE1+FACE2+FACE3))
#define ALIGN 6

extern int cpr[4], npr[8];
extern int ipt[VOLUME];
extern int iup[VOLUME][4];
extern int idn[VOLUME][4];
extern int map[BNDRY + NPROC % 2];

/* ---- su3.h: types and the in-line products the modules use ------------- */
typedef struct { float re, im; } complex;
typedef struct { double re, im; } complex_dble;
typedef struct { complex_dble c1, c2, c3; } su3_vector_dble;
typedef struct {
  complex_dble c11, c12, c13, c21, c22, c23, c31, c32, c33;
} su3_dble;

/* r = u s (matrix times vector) */
#define _su3_multiply(r,u,s) \
  (r).c1.re=(u).c11.re*(s).c1.re-(u).c11.im*(s).c1.im \
           +(u).c12.re*(s).c2.re-(u).c12.im*(s).c2.im \
           +(u).c13.re*(s).c3.re-(u).c13.im*(s).c3.im; \
  (r).c1.im=(u).c11.re*(s).c1.im+(u).c11.im*(s).c1.re \
           +(u).c12.re*(s).c2.im+(u).c12.im*(s).c2.re \
           +(u).c13.re*(s).c3.im+(u).c13.im*(s).c3.re; \
  (r).c2.re=(u).c21.re*(s).c1.re-(u).c21.im*(s).c1.im \
           +(u).c22.re*(s).c2.re-(u).c22.im*(s).c2.im \
           +(u).c23.re*(s).c3.re-(u).c23.im*(s).c3.im; \
  (r).c2.im=(u).c21.re*(s).c1.im+(u).c21.im*(s).c1.re \
           +(u).c22.re*(s).c2.im+(u).c22.im*(s).c2.re \
           +(u).c23.re*(s).c3.im+(u).c23.im*(s).c3.re; \
  (r).c3.re=(u).c31.re*(s).c1.re-(u).c31.im*(s).c1.im \
           +(u).c32.re*(s).c2.re-(u).c32.im*(s).c2.im \
           +(u).c33.re*(s).c3.re-(u).c33.im*(s).c3.im; \
  (r).c3.im=(u).c31.re*(s).c1.im+(u).c31.im*(s).c1.re \
           +(u).c32.re*(s).c2.im+(u).c32.im*(s).c2.re \
           +(u).c33.re*(s).c3.im+(u).c33.im*(s).c3.re

/* r = u^dagger s */
#define _su3_inverse_multiply(r,u,s) \
  (r).c1.re=(u).c11.re*(s).c1.re+(u).c11.im*(s).c1.im \
           +(u).c21.re*(s).c2.re+(u).c21.im*(s).c2.im \
           +(u).c31.re*(s).c3.re+(u).c31.im*(s).c3.im; \
  (r).c1.im=(u).c11.re*(s).c1.im-(u).c11.im*(s).c1.re \
           +(u).c21.re*(s).c2.im-(u).c21.im*(s).c2.re \
           +(u).c31.re*(s).c3.im-(u).c31.im*(s).c3.re; \
  (r).c2.re=(u).c12.re*(s).c1.re+(u).c12.im*(s).c1.im \
           +(u).c22.re*(s).c2.re+(u).c22.im*(s).c2.im \
           +(u).c32.re*(s).c3.re+(u).c32.im*(s).c3.im; \
  (r).c2.im=(u).c12.re*(s).c1.im-(u).c12.im*(s).c1.re \
           +(u).c22.re*(s).c2.im-(u).c22.im*(s).c2.re \
           +(u).c32.re*(s).c3.im-(u).c32.im*(s).c3.re; \
  (r).c3.re=(u).c13.re*(s).c1.re+(u).c13.im*(s).c1.im \
           +(u).c23.re*(s).c2.re+(u).c23.im*(s).c2.im \
           +(u).c33.re*(s).c3.re+(u).c33.im*(s).c3.im; \
  (r).c3.im=(u).c13.re*(s).c1.im-(u).c13.im*(s).c1.re \
           +(u).c23.re*(s).c2.im-(u).c23.im*(s).c2.re \
           +(u).c33.re*(s).c3.im-(u).c33.im*(s).c3.re

/* Re(r^dagger s) of two colour vectors */
#define _vector_prod_re(r,s) \
  ((r).c1.re*(s).c1.re+(r).c1.im*(s).c1.im \
  +(r).c2.re*(s).c2.re+(r).c2.im*(s).c2.im \
  +(r).c3.re*(s).c3.re+(r).c3.im*(s).c3.im)

/* u = v w, through the matrix-vector product column by column */
#define _wlref_col(a,m,j) \
  (a).c1=(m).c1##j; (a).c2=(m).c2##j; (a).c3=(m).c3##j
#define _wlref_setcol(m,j,a) \
  (m).c1##j=(a).c1; (m).c2##j=(a).c2; (m).c3##j=(a).c3
#define _su3_times_su3(u,v,w) \
  { su3_vector_dble wlref_p_, wlref_q_; \
    _wlref_col(wlref_p_,w,1); _su3_multiply(wlref_q_,v,wlref_p_); _wlref_setcol(u,1,wlref_q_); \
    _wlref_col(wlref_p_,w,2); _su3_multiply(wlref_q_,v,wlref_p_); _wlref_setcol(u,2,wlref_q_); \
    _wlref_col(wlref_p_,w,3); _su3_multiply(wlref_q_,v,wlref_p_); _wlref_setcol(u,3,wlref_q_); }

/* the SSE prefetch hint is a no-op here (SSE2 is not defined) */
#define _prefetch_su3_dble(addr)

/* ---- su3fcts.h: out-of-line products (w may be the same matrix as v) --- */
void su3xsu3(su3_dble *u, su3_dble *v, su3_dble *w);     /* w = u v */
void su3dagxsu3(su3_dble *u, su3_dble *v, su3_dble *w);  /* w = u^dag v */
void su3xsu3dag(su3_dble *u, su3_dble *v, su3_dble *w);  /* w = u v^dag */

/* ---- lattice.h / uflds.h / flags.h ------------------------------------- */
void geometry(void);
int ipr_global(int *n);
int global_time(int ix);
void set_bc(void);
su3_dble *udfld(void);
void copy_bnd_ud(void);

typedef enum {
  UPDATED_U, UPDATED_UD, ASSIGNED_UD2U, EVENTS
} event_t;
void set_flags(event_t event);
int bc_type(void);

/* ---- utils.h ------------------------------------------------------------ */
#define NAME_SIZE 128
#define IMAX(n,m) (((n)>(m))?(n):(m))
#define UNKNOWN_ENDIAN 0
#define LITTLE_ENDIAN 1
#define BIG_ENDIAN 2
/* 32-bit integer of the binary file formats */
typedef int stdint_t;
void *amalloc(size_t size, int p);
void afree(void *addr);
void error(int test, int no, char *name, char *format, ...);
void error_root(int test, int no, char *name, char *format, ...);
int mpi_tag(void);
int endianness(void);
void bswap_int(int n, void *a);
void bswap_double(int n, void *a);
int fdigits(double x);
int find_section(char *title);
int read_line(char *tag, char *format, ...);
void read_iprms(char *tag, int n, int *iprms);
void read_dprms(char *tag, int n, double *dprms);

/* ---- driver-side controls (not openQCD names) -------------------------- */
void wlref_set_bc_type(int type);

#endif
