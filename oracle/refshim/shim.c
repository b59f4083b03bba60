/*
 * shim.c -- one-process implementation of the openQCD-1.4 interface declared
 * in shim.h, for compiling the reference's wloop modules unchanged
 * (oracle/_ref).  TEST INFRASTRUCTURE ONLY: the checker, never the product.
 *
 * Geometry.  Sites are numbered as openQCD numbers them on one process: the
 * even points (x0+x1+x2+x3 even) first, then the odd points; ipt[] maps the
 * lexicographic index x3 + L3*x2 + L2*L3*x1 + L1*L2*L3*x0 to that number.
 * Within one parity this shim keeps lexicographic order (openQCD orders
 * sites inside its blocks differently; that only changes the order of the
 * floating-point sums over sites).  iup/idn wrap periodically in every
 * direction, as openQCD's do when a direction has one process.
 *
 * Gauge field.  udfld() holds the 4*VOLUME links of the odd points:
 * ud[8*(ix-VOLUME/2)+2*mu] = U(x,mu) and ud[8*(ix-VOLUME/2)+2*mu+1] =
 * U(x-mu,mu) for odd x (the layout the modules address, lnkcom.c:840-859).
 * set_bc() sets the time-like links on the last time slice to zero for open
 * boundary conditions (type 0) and leaves periodic ones (type 3) alone.
 */
#define _POSIX_C_SOURCE 200112L
#include <math.h>
#include <stdarg.h>
#include <stdlib.h>
#include <string.h>
#include "shim.h"
#include "mpi.h"

int cpr[4] = {0, 0, 0, 0};
int npr[8] = {0, 0, 0, 0, 0, 0, 0, 0};
int ipt[VOLUME];
int iup[VOLUME][4];
int idn[VOLUME][4];
int map[BNDRY + NPROC % 2];

static int xtime[VOLUME];       /* x0 of site ix */
static su3_dble *ud = NULL;
static int bctype = 3;
static int geometry_done = 0;

static int lexi(int x0, int x1, int x2, int x3)
{
  return x3 + L3 * (x2 + L2 * (x1 + L1 * x0));
}

void geometry(void)
{
  int x0, x1, x2, x3, s, ne, no, ix, mu;
  int x[4], y[4], ls[4];

  ls[0] = L0; ls[1] = L1; ls[2] = L2; ls[3] = L3;
  ne = 0;
  no = VOLUME / 2;
  for (x0 = 0; x0 < L0; x0++)
    for (x1 = 0; x1 < L1; x1++)
      for (x2 = 0; x2 < L2; x2++)
        for (x3 = 0; x3 < L3; x3++) {
          s = lexi(x0, x1, x2, x3);
          ipt[s] = ((x0 + x1 + x2 + x3) % 2 == 0) ? ne++ : no++;
          xtime[ipt[s]] = x0;
        }
  for (x0 = 0; x0 < L0; x0++)
    for (x1 = 0; x1 < L1; x1++)
      for (x2 = 0; x2 < L2; x2++)
        for (x3 = 0; x3 < L3; x3++) {
          x[0] = x0; x[1] = x1; x[2] = x2; x[3] = x3;
          ix = ipt[lexi(x0, x1, x2, x3)];
          for (mu = 0; mu < 4; mu++) {
            memcpy(y, x, sizeof(x));
            y[mu] = (x[mu] + 1) % ls[mu];
            iup[ix][mu] = ipt[lexi(y[0], y[1], y[2], y[3])];
            y[mu] = (x[mu] + ls[mu] - 1) % ls[mu];
            idn[ix][mu] = ipt[lexi(y[0], y[1], y[2], y[3])];
          }
        }
  map[0] = 0;
  geometry_done = 1;
}

int ipr_global(int *n)
{
  (void)n;
  return 0;
}

int global_time(int ix)
{
  return xtime[ix];
}

su3_dble *udfld(void)
{
  if (ud == NULL) {
    error(geometry_done == 0, 1, "udfld [shim.c]", "geometry() has not been called");
    ud = amalloc((4 * VOLUME + BNDRY / 4) * sizeof(su3_dble), ALIGN);
    error(ud == NULL, 1, "udfld [shim.c]", "Unable to allocate the gauge field");
    memset(ud, 0, (4 * VOLUME + BNDRY / 4) * sizeof(su3_dble));
  }
  return ud;
}

/* the boundary links of the gauge field come from the neighbouring
 * processes; with one process there are none */
void copy_bnd_ud(void)
{
}

void wlref_set_bc_type(int type)
{
  error((type != 0) && (type != 3), 1, "wlref_set_bc_type [shim.c]",
        "only open (0) and periodic (3) boundary conditions");
  bctype = type;
}

int bc_type(void)
{
  return bctype;
}

void set_bc(void)
{
  int ix, x0, x1, x2, x3;
  su3_dble *u = udfld();

  if (bctype != 0)
    return;
  /* U(x,0) with x0 = N0-1 is stored at the odd point of the pair {x, x+0} */
  x0 = L0 - 1;
  for (x1 = 0; x1 < L1; x1++)
    for (x2 = 0; x2 < L2; x2++)
      for (x3 = 0; x3 < L3; x3++) {
        ix = ipt[lexi(x0, x1, x2, x3)];
        if (ix >= VOLUME / 2)
          memset(u + 8 * (ix - VOLUME / 2), 0, sizeof(su3_dble));
        else
          memset(u + 8 * (iup[ix][0] - VOLUME / 2) + 1, 0, sizeof(su3_dble));
      }
}

void set_flags(event_t event)
{
  (void)event;
}

/* ---- su3 products: each result column (or row) from a copy of the inputs,
 * so w may be the same matrix as u or v ------------------------------------ */
void su3xsu3(su3_dble *u, su3_dble *v, su3_dble *w)
{
  su3_dble a = *u, b = *v;
  _su3_times_su3(*w, a, b);
}

void su3dagxsu3(su3_dble *u, su3_dble *v, su3_dble *w)
{
  su3_dble a = *u, b = *v;
  su3_vector_dble p, q;
  _wlref_col(p, b, 1); _su3_inverse_multiply(q, a, p); _wlref_setcol(*w, 1, q);
  _wlref_col(p, b, 2); _su3_inverse_multiply(q, a, p); _wlref_setcol(*w, 2, q);
  _wlref_col(p, b, 3); _su3_inverse_multiply(q, a, p); _wlref_setcol(*w, 3, q);
}

void su3xsu3dag(su3_dble *u, su3_dble *v, su3_dble *w)
{
  /* column j of u v^dag is u times the conjugate of row j of v */
  su3_dble a = *u, b = *v;
  su3_vector_dble p, q;
  p.c1.re = b.c11.re; p.c1.im = -b.c11.im;
  p.c2.re = b.c12.re; p.c2.im = -b.c12.im;
  p.c3.re = b.c13.re; p.c3.im = -b.c13.im;
  _su3_multiply(q, a, p); _wlref_setcol(*w, 1, q);
  p.c1.re = b.c21.re; p.c1.im = -b.c21.im;
  p.c2.re = b.c22.re; p.c2.im = -b.c22.im;
  p.c3.re = b.c23.re; p.c3.im = -b.c23.im;
  _su3_multiply(q, a, p); _wlref_setcol(*w, 2, q);
  p.c1.re = b.c31.re; p.c1.im = -b.c31.im;
  p.c2.re = b.c32.re; p.c2.im = -b.c32.im;
  p.c3.re = b.c33.re; p.c3.im = -b.c33.im;
  _su3_multiply(q, a, p); _wlref_setcol(*w, 3, q);
}

/* ---- utils ---------------------------------------------------------------
 * amalloc/afree keep a registry of the blocks they hand out: afree of an
 * address that is not (or no longer) registered does nothing, which the
 * modules rely on (free_lnk and the free_* routines may release the same
 * field twice, lnkcom.c:719-741). */
struct ablock {
  void *addr;
  struct ablock *next;
};
static struct ablock *blocks = NULL;

void *amalloc(size_t size, int p)
{
  void *a = NULL;
  struct ablock *b;
  size_t al = (size_t)1 << (p < 4 ? 4 : p);
  if (size == 0)
    size = al; /* a zero-sized field still gets a distinct address */
  if (posix_memalign(&a, al, size) != 0)
    return NULL;
  b = malloc(sizeof(struct ablock));
  if (b == NULL) {
    free(a);
    return NULL;
  }
  b->addr = a;
  b->next = blocks;
  blocks = b;
  return a;
}

void afree(void *addr)
{
  struct ablock *b = blocks, *prev = NULL;
  if (addr == NULL)
    return;
  while (b != NULL) {
    if (b->addr == addr) {
      if (prev == NULL)
        blocks = b->next;
      else
        prev->next = b->next;
      free(b->addr);
      free(b);
      return;
    }
    prev = b;
    b = b->next;
  }
}

static void fail(char *name, char *format, va_list args)
{
  fprintf(stderr, "\nError in %s:\n", name);
  vfprintf(stderr, format, args);
  fprintf(stderr, "\nProgram aborted\n\n");
  fflush(stderr);
  exit(1);
}

void error(int test, int no, char *name, char *format, ...)
{
  va_list args;
  (void)no;
  if (test) {
    va_start(args, format);
    fail(name, format, args);
    va_end(args);
  }
}

void error_root(int test, int no, char *name, char *format, ...)
{
  va_list args;
  (void)no;
  if (test) {
    va_start(args, format);
    fail(name, format, args);
    va_end(args);
  }
}

int mpi_tag(void)
{
  return 0;
}

int endianness(void)
{
  unsigned int one = 1;
  return (*(unsigned char *)&one == 1) ? LITTLE_ENDIAN : BIG_ENDIAN;
}

static void bswap(int n, int size, void *a)
{
  unsigned char *c = (unsigned char *)a, t;
  int i, k;
  for (i = 0; i < n; i++, c += size)
    for (k = 0; k < size / 2; k++) {
      t = c[k];
      c[k] = c[size - 1 - k];
      c[size - 1 - k] = t;
    }
}

void bswap_int(int n, void *a)
{
  bswap(n, (int)sizeof(int), a);
}

void bswap_double(int n, void *a)
{
  bswap(n, (int)sizeof(double), a);
}

/* number of decimals needed to print x (at most 16) */
int fdigits(double x)
{
  int k;
  double y = fabs(x);
  for (k = 0; k < 16; k++) {
    if (y == floor(y))
      return k;
    y *= 10.0;
  }
  return 16;
}

/* the input-file readers are not used by the driver; reaching one is an
 * error of the driver */
int find_section(char *title)
{
  error(1, 1, "find_section [shim.c]", "input files are not read by this shim (%s)", title);
  return 0;
}

int read_line(char *tag, char *format, ...)
{
  (void)format;
  error(1, 1, "read_line [shim.c]", "input files are not read by this shim (%s)", tag);
  return 0;
}

void read_iprms(char *tag, int n, int *iprms)
{
  (void)n; (void)iprms;
  error(1, 1, "read_iprms [shim.c]", "input files are not read by this shim (%s)", tag);
}

void read_dprms(char *tag, int n, double *dprms)
{
  (void)n; (void)dprms;
  error(1, 1, "read_dprms [shim.c]", "input files are not read by this shim (%s)", tag);
}

/* ---- MPI on one rank ----------------------------------------------------- */
static int type_size(MPI_Datatype t)
{
  return (t == MPI_DOUBLE) ? (int)sizeof(double) : (int)sizeof(int);
}

int MPI_Comm_rank(MPI_Comm comm, int *rank)
{
  (void)comm;
  *rank = 0;
  return MPI_SUCCESS;
}

int MPI_Comm_size(MPI_Comm comm, int *size)
{
  (void)comm;
  *size = 1;
  return MPI_SUCCESS;
}

int MPI_Bcast(void *buf, int count, MPI_Datatype type, int root, MPI_Comm comm)
{
  (void)buf; (void)count; (void)type; (void)root; (void)comm;
  return MPI_SUCCESS;
}

int MPI_Reduce(void *sbuf, void *rbuf, int count, MPI_Datatype type, MPI_Op op, int root,
               MPI_Comm comm)
{
  (void)op; (void)root; (void)comm;
  if (sbuf != rbuf)
    memmove(rbuf, sbuf, (size_t)count * type_size(type));
  return MPI_SUCCESS;
}

int MPI_Allreduce(void *sbuf, void *rbuf, int count, MPI_Datatype type, MPI_Op op,
                  MPI_Comm comm)
{
  return MPI_Reduce(sbuf, rbuf, count, type, op, 0, comm);
}

int MPI_Barrier(MPI_Comm comm)
{
  (void)comm;
  return MPI_SUCCESS;
}

int MPI_Send(void *buf, int count, MPI_Datatype type, int dest, int tag, MPI_Comm comm)
{
  (void)buf; (void)count; (void)type; (void)dest; (void)tag; (void)comm;
  error(1, 1, "MPI_Send [shim.c]", "point-to-point communication with one rank");
  return 1;
}

int MPI_Recv(void *buf, int count, MPI_Datatype type, int src, int tag, MPI_Comm comm,
             MPI_Status *status)
{
  (void)buf; (void)count; (void)type; (void)src; (void)tag; (void)comm; (void)status;
  error(1, 1, "MPI_Recv [shim.c]", "point-to-point communication with one rank");
  return 1;
}

double MPI_Wtime(void)
{
  return 0.0;
}
