// smear.cu -- link smearing kernels for sm_100a.
//
// All kernels are one-thread-per-output-link, grid-stride over
// (output slot, site) with the site fastest, so every component load of a
// warp is a coalesced SoA request.  Neighbour links are read through the
// read-only path (__ldg): the staple of link (x,mu) touches links within one
// lattice row of x, so the L2 (126 MB) serves the re-reads and HBM sees each
// input field roughly once per kernel.  Staple products run in T (FP64, or
// FP32 in the mixed form); the linear combination and the SU(3) projection
// always run in FP64.
#include <string.h>

#include "internal.h"

namespace wlg {

// unordered pair index used by hyp_links.c:128-139:
// {0,1},{2,3} -> 0; {0,2},{1,3} -> 1; {0,3},{1,2} -> 2
__device__ __forceinline__ int hyp_pair(int a, int b) {
  int d = a + b;
  if (d > 3) d = 6 - d;
  return d - 1;
}

// dlnks_idx of hyp_spatial_links.c:117-125 (not symmetric)
__device__ __forceinline__ int hyp3_slot(int mu, int eta) {
  // [1][2]=0 [1][3]=1 [2][1]=0 [2][3]=1 [3][1]=0 [3][2]=1
  if (mu == 3) return (eta == 1) ? 0 : 1;
  return (eta == 3) ? 1 : 0;
}

static inline int grid_for(long long n, int block) {
  long long g = (n + block - 1) / block;
  long long cap = (long long)num_sms() * 32;
  if (g > cap) g = cap;
  if (g < 1) g = 1;
  return (int)g;
}

template <class T>
__device__ __forceinline__ typename V2<T>::t* fld(typename V2<T>::t* base, int vol, int slot, int mu,
                                                  int ndir) {
  return base + (size_t)(slot * ndir + mu) * link_elems<T>(vol);
}

// v = a*u + b*s (FP64), then optional projection; this is _su3_lcomb +
// approx_project_to_su3_dble of decorate_all (hyp_links.c:154-171).
template <class T>
__device__ __forceinline__ void lcomb_project(M3<double>& v, double a, const M3<T>& u, double b,
                                              const M3<T>& s, int proj, int iter) {
#pragma unroll
  for (int k = 0; k < 9; k++) {
    v.e[k].x = a * (double)u.e[k].x + b * (double)s.e[k].x;
    v.e[k].y = a * (double)u.e[k].y + b * (double)s.e[k].y;
  }
  if (proj) project(v, iter);
}

// ---------------------------------------------------------------------------
// Item functions: one output link each, w = local work index of one lattice
// (site fastest).  The single-lattice kernels below and the batched kernels
// of batch.cu (flattened work lists over many lattices) both call them.
// ---------------------------------------------------------------------------

// HYP level with alpha3 (decorated_links1, hyp_links.c:320-373):
//   vbar[p(mu,eta)](x,mu) = P[(1-a3) U + a3/2 * S_eta(U)];  w in [0, tile_items(V, 12))
template <class T> __device__ __forceinline__ void hyp_l3_item(const SArgs<T>& A, long long w) {
  const Geo& g = A.g;
  int q, s;
  tile_item(w, 12, q, s);
  if (s >= g.vol) return;
  int mu = q / 3, eta = (mu + 1 + q % 3) & 3;
  int x[4];
  coords(g, s, x);
  M3<T> S, u;
  zero(S);
  add_staples(S, g, x, s, A.U.p[eta], A.U.p[mu], mu, eta);
  ld(u, A.U.p[mu], g.vol, s);
  M3<double> v;
  lcomb_project(v, A.a, u, A.b, S, A.proj, A.iter);
  M3<T> o;
  cvt(o, v);
  st(fld<T>(A.aux0, g.vol, hyp_pair(mu, eta), mu, 4), g.vol, s, o);
}

// HYP level with alpha2 (decorated_links2, hyp_links.c:244-317):
//   vtil[p(mu,nu)](x,mu) = P[(1-a2) U + a2/4 * sum_{rho != mu,nu} S_rho]
//   rho-links from vbar[p(mu,nu)], mu-links from vbar[p(nu,rho)];  w in [0, tile_items(V, 12))
template <class T> __device__ __forceinline__ void hyp_l2_item(const SArgs<T>& A, long long w) {
  const Geo& g = A.g;
  int q, s;
  tile_item(w, 12, q, s);
  if (s >= g.vol) return;
  int mu = q / 3, nu = (mu + 1 + q % 3) & 3;
  int x[4];
  coords(g, s, x);
  int pmn = hyp_pair(mu, nu);
  M3<T> S, u;
  zero(S);
#pragma unroll 1  // one staple body in the code: the unrolled planes overflow the instruction cache
  for (int rho = 0; rho < 4; rho++) {
    if (rho == mu || rho == nu) continue;
    add_staples(S, g, x, s, fld<T>(A.aux0, g.vol, pmn, rho, 4),
                fld<T>(A.aux0, g.vol, hyp_pair(nu, rho), mu, 4), mu, rho);
  }
  ld(u, A.U.p[mu], g.vol, s);
  M3<double> v;
  lcomb_project(v, A.a, u, A.b, S, A.proj, A.iter);
  M3<T> o;
  cvt(o, v);
  st(fld<T>(A.aux1, g.vol, pmn, mu, 4), g.vol, s, o);
}

// HYP level with alpha1 (decorated_links3, hyp_links.c:194-241) and the copy
// back into the gauge field (:432-447), in place: each item reads only its
// own U(x,mu) for the linear combination.  w in [0, tile_items(V, nmu))
template <class T> __device__ __forceinline__ void hyp_l1_item(const SArgs<T>& A, long long w) {
  const Geo& g = A.g;
  int q, s;
  tile_item(w, A.nmu, q, s);
  if (s >= g.vol) return;
  int mu = A.mu0 + q;
  int x[4];
  coords(g, s, x);
  M3<T> S, u;
  zero(S);
#pragma unroll 1
  for (int i = 1; i < 4; i++) {
    int nu = (mu + i) & 3, p = hyp_pair(mu, nu);
    add_staples(S, g, x, s, fld<T>(A.aux1, g.vol, p, nu, 4), fld<T>(A.aux1, g.vol, p, mu, 4), mu,
                nu);
  }
  ld(u, A.U.p[mu], g.vol, s);
  M3<double> v;
  lcomb_project(v, A.a, u, A.b, S, A.proj, A.iter);
  M3<T> o;
  cvt(o, v);
  if (A.bc == 0 && mu == 0 && x[0] == g.n[0] - 1) zero(o);  // set_bc(), open bc
  st(A.U.p[mu], g.vol, s, o);
}

// One APE sweep (ape_links_all, ape_links.c:217-272):
//   D(x,mu) = P[U(x,mu) + alpha * sum_{eta != mu} S_eta(U)];
// w in [0, ape_items(vol, mu0)), tile-major: the 4-mu0 directions of one
// 32-site tile are consecutive warps, so the links their staples share are
// re-read from L2 instead of once per direction sweep over the whole field.
template <class T> __device__ __forceinline__ void ape_item(const SArgs<T>& A, long long w) {
  const Geo& g = A.g;
  int q, s;
  tile_item(w, 4 - A.mu0, q, s);
  if (s >= g.vol) return;  // the last tile of a lattice whose volume is not a multiple of 32
  int mu = A.mu0 + q;
  int x[4];
  coords(g, s, x);
  M3<T> S, u;
  zero(S);
  for (int eta = A.mu0; eta < 4; eta++) {
    if (eta == mu) continue;
    add_staples(S, g, x, s, A.U.p[eta], A.U.p[mu], mu, eta);
  }
  ld(u, A.U.p[mu], g.vol, s);
  M3<double> v;
#pragma unroll
  for (int k = 0; k < 9; k++) {  // _su3_mulr then _su3_add (:246-247)
    double sr = A.a * (double)S.e[k].x, si = A.a * (double)S.e[k].y;
    v.e[k].x = (double)u.e[k].x + sr;
    v.e[k].y = (double)u.e[k].y + si;
  }
  if (A.proj) project(v, A.iter);
  M3<T> o;
  cvt(o, v);
  st(A.D.p[mu], g.vol, s, o);
}

// Spatial HYP, level with alpha2 (decorated_links1, hyp_spatial_links.c:210-265)
//   dl[slot(mu,eta)](x,mu) = P[(1-a2) U + a2/2 S_eta(U)];  w in [0, 6V)
template <class T> __device__ __forceinline__ void hyp3_l1_item(const SArgs<T>& A, long long w) {
  const Geo& g = A.g;
  int q = (int)(w / g.vol), s = (int)(w - (long long)q * g.vol);
  int mu = 1 + q / 2, eta = ((mu + q % 2) % 3) + 1;
  int x[4];
  coords(g, s, x);
  M3<T> S, u;
  zero(S);
  add_staples(S, g, x, s, A.U.p[eta], A.U.p[mu], mu, eta);
  ld(u, A.U.p[mu], g.vol, s);
  M3<double> v;
  lcomb_project(v, A.a, u, A.b, S, A.proj, A.iter);
  M3<T> o;
  cvt(o, v);
  st(fld<T>(A.aux0, g.vol, hyp3_slot(mu, eta), mu - 1, 3), g.vol, s, o);
}

// Spatial HYP, level with alpha1 (decorated_links2, hyp_spatial_links.c:160-207),
// in place on D (lcomb with D's own link);  w in [0, 3V)
template <class T> __device__ __forceinline__ void hyp3_l2_item(const SArgs<T>& A, long long w) {
  const Geo& g = A.g;
  int q = (int)(w / g.vol), s = (int)(w - (long long)q * g.vol);
  int mu = 1 + q;
  int x[4];
  coords(g, s, x);
  M3<T> S, u;
  zero(S);
#pragma unroll
  for (int i = 0; i < 2; i++) {
    int nu = ((mu + i) % 3) + 1;
    add_staples(S, g, x, s, fld<T>(A.aux0, g.vol, hyp3_slot(nu, mu), nu - 1, 3),
                fld<T>(A.aux0, g.vol, hyp3_slot(mu, nu), mu - 1, 3), mu, nu);
  }
  ld(u, A.D.p[mu], g.vol, s);
  M3<double> v;
  lcomb_project(v, A.a, u, A.b, S, A.proj, A.iter);
  M3<T> o;
  cvt(o, v);
  st(A.D.p[mu], g.vol, s, o);
}

#define WLG_GRID_STRIDE(n) \
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < (n); \
       w += (long long)gridDim.x * blockDim.x)

// batched: one grid over the flattened work of n lattices
template <class T, int STAGE>
__global__ void __launch_bounds__(128) kb_smear(const SArgs<T>* __restrict__ A,
                                                const long long* __restrict__ pre, int n,
                                                long long total) {
  WLG_GRID_STRIDE(total) {
    const int c = find_item(pre, n, w);
    const long long lw = w - __ldg(pre + c);
    if (STAGE == BATCH_HYP3) hyp_l3_item<T>(A[c], lw);
    if (STAGE == BATCH_HYP2) hyp_l2_item<T>(A[c], lw);
    if (STAGE == BATCH_HYP1) hyp_l1_item<T>(A[c], lw);
    if (STAGE == BATCH_APE) ape_item<T>(A[c], lw);
    if (STAGE == BATCH_HYP3D1) hyp3_l1_item<T>(A[c], lw);
    if (STAGE == BATCH_HYP3D2) hyp3_l2_item<T>(A[c], lw);
  }
}

template <class T> __global__ void __launch_bounds__(128) k_hyp_l3(SArgs<T> A) {
  WLG_GRID_STRIDE(tile_items(A.g.vol, 12)) hyp_l3_item<T>(A, w);
}
template <class T> __global__ void __launch_bounds__(128) k_hyp_l2(SArgs<T> A) {
  WLG_GRID_STRIDE(tile_items(A.g.vol, 12)) hyp_l2_item<T>(A, w);
}
template <class T> __global__ void __launch_bounds__(128) k_hyp_l1(SArgs<T> A) {
  WLG_GRID_STRIDE(tile_items(A.g.vol, A.nmu)) hyp_l1_item<T>(A, w);
}
// minimum resident blocks: FP32 fits 5 blocks of 128 threads per SM in 96
// registers, FP64 3 blocks (the staples' latency needs the extra warps)
template <class T> struct ApeMinBlocks { enum { v = sizeof(T) == 4 ? 5 : 3 }; };

template <class T>
__global__ void __launch_bounds__(128, ApeMinBlocks<T>::v) k_ape(SArgs<T> A) {
  WLG_GRID_STRIDE(ape_items(A.g.vol, A.mu0)) ape_item<T>(A, w);
}
template <class T> __global__ void __launch_bounds__(128) k_hyp3_l1(SArgs<T> A) {
  WLG_GRID_STRIDE(6LL * A.g.vol) hyp3_l1_item<T>(A, w);
}
template <class T> __global__ void __launch_bounds__(128) k_hyp3_l2(SArgs<T> A) {
  WLG_GRID_STRIDE(3LL * A.g.vol) hyp3_l2_item<T>(A, w);
}

// staple_sum: vb(x,mu) += up + down staples in the (mu,nu) plane
template <class T>
__global__ void k_staple_sum(Geo g, Links<T> u1, Links<T> u2, int mu, int nu, Links<T> vb) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < g.vol; s += gridDim.x * blockDim.x) {
    int x[4];
    coords(g, s, x);
    M3<T> v;
    ld(v, vb.p[mu], g.vol, s);
    add_staples(v, g, x, s, u1.p[nu], u2.p[mu], mu, nu);
    st(vb.p[mu], g.vol, s, v);
  }
}

__global__ void k_project_batch(double* m, int n, int iter) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    M3<double> u;
    const double2* p = reinterpret_cast<const double2*>(m + 18 * (size_t)i);
#pragma unroll
    for (int c = 0; c < 9; c++) u.e[c] = p[c];
    project(u, iter);
    double2* q = reinterpret_cast<double2*>(m + 18 * (size_t)i);
#pragma unroll
    for (int c = 0; c < 9; c++) q[c] = u.e[c];
  }
}

// ---------------------------------------------------------------------------
// Plaquette sum (local_plaq_sum_dble, lnkplaq.c:68-114): per site the (mu,0)
// plaquettes (skipped at x0=N0-1 for open bc) and the (mu,nu) spatial ones,
// products in T, sums in FP64; warp shuffle + block reduction into one
// partial per block, then a fixed-order final pass (deterministic).
// ---------------------------------------------------------------------------
constexpr int kPlaqBlocks = 1184;  // 8 x 148 SMs
constexpr int kPlaqThreads = 256;
int plaq_partials() { return kPlaqBlocks; }

template <class T>
__device__ __forceinline__ double plaq_at(const Geo& g, const Links<T>& U, const int x[4], int s,
                                          int mu, int nu) {
  M3<T> a, b, w1, w2;
  ld(a, U.p[mu], g.vol, s);
  ld(b, U.p[nu], g.vol, up(g, s, x[mu], mu));
  mul(w1, a, b);
  ld(a, U.p[nu], g.vol, s);
  ld(b, U.p[mu], g.vol, up(g, s, x[nu], nu));
  mul(w2, a, b);
  return (double)retr_dag(w1, w2);
}

__device__ __forceinline__ double block_sum(double v) {
  __shared__ double red[32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if (lane == 0) red[wid] = v;
  __syncthreads();
  double r = 0.0;
  if (wid == 0) {
    r = (lane < (int)(blockDim.x >> 5)) ? red[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
  }
  __syncthreads();
  return r;
}

template <class T>
__global__ void __launch_bounds__(kPlaqThreads) k_plaq(Geo g, int bc, Links<T> U, double* partial) {
  double acc = 0.0;
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < g.vol; s += gridDim.x * blockDim.x) {
    int x[4];
    coords(g, s, x);
    double pa = 0.0;
    for (int mu = 1; mu < 4; mu++) {
      if (x[0] < g.n[0] - 1 || bc != 0) pa += plaq_at(g, U, x, s, mu, 0);
      for (int nu = 1; nu < mu; nu++) pa += plaq_at(g, U, x, s, mu, nu);
    }
    acc += pa;
  }
  double r = block_sum(acc);
  if (threadIdx.x == 0) partial[blockIdx.x] = r;
}

__global__ void k_sum_partials(const double* partial, int n, double* out) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) acc += partial[i];
  double r = block_sum(acc);
  if (threadIdx.x == 0) *out = r;
}

// ---------------------------------------------------------------------------
// Single staples on explicit link triples (add_*_staple_lnks[_save],
// lnkstaple.c:145-410).  save = 1: general 3x3 form v += u1 u2 u3^dag (up)
// or u1^dag u2 u3 (down).  save = 0: the SU(3) form of up_staple/dn_staple
// (:145-256): only the first two columns of the product are formed and the
// third is added as conj(col1 x col2) (add_to_v, :108-142).
// Matrices are packed su3_dble (18 doubles), FP64.
// ---------------------------------------------------------------------------
__global__ void k_staples_lnks(int n, const double2* u1, const double2* u2, const double2* u3,
                               double2* v, int dn, int save) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    M3<double> a, b, c, t, r;
#pragma unroll
    for (int k = 0; k < 9; k++) {
      a.e[k] = u1[9 * (size_t)i + k];
      b.e[k] = u2[9 * (size_t)i + k];
      c.e[k] = u3[9 * (size_t)i + k];
    }
    if (dn) {
      mul(t, b, c);
      mul_da(r, a, t);
    } else {
      mul_ad(t, b, c);
      mul(r, a, t);
    }
    if (!save) {
      // third column from the first two: c_i3 = conj(c1 x c2)_i
#pragma unroll
      for (int row = 0; row < 3; row++) {
        int p = (row + 1) % 3, q = (row + 2) % 3;
        double2 x1 = r.e[3 * p], y2 = r.e[3 * q + 1], x2 = r.e[3 * q], y1 = r.e[3 * p + 1];
        double re = (x1.x * y2.x - x1.y * y2.y) - (x2.x * y1.x - x2.y * y1.y);
        double im = (x1.x * y2.y + x1.y * y2.x) - (x2.x * y1.y + x2.y * y1.x);
        r.e[3 * row + 2] = make_double2(re, -im);
      }
    }
#pragma unroll
    for (int k = 0; k < 9; k++) {
      double2 o = v[9 * (size_t)i + k];
      o.x += r.e[k].x;
      o.y += r.e[k].y;
      v[9 * (size_t)i + k] = o;
    }
  }
}

void staples_lnks(int n, const double* u1, const double* u2, const double* u3, double* v, int dn,
                  int save, cudaStream_t st) {
  if (n <= 0) return;
  k_staples_lnks<<<grid_for(n, 128), 128, 0, st>>>(
      n, reinterpret_cast<const double2*>(u1), reinterpret_cast<const double2*>(u2),
      reinterpret_cast<const double2*>(u3), reinterpret_cast<double2*>(v), dn, save);
  WLG_LAUNCH_CHECK("staples_lnks");
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
template <class T> static SArgs<T> sargs(const Geo& g) {
  SArgs<T> A;
  memset(&A, 0, sizeof(A));
  A.g = g;
  return A;
}

template <class T>
void hyp_level3(const Geo& g, Links<T> U, typename V2<T>::t* vbar, double a3, int proj, int iter,
                cudaStream_t st) {
  SArgs<T> A = sargs<T>(g);
  A.U = U;
  A.aux0 = vbar;
  A.a = 1.0 - a3;
  A.b = a3 / 2.0;
  A.proj = proj;
  A.iter = iter;
  k_hyp_l3<T><<<grid_for(tile_items(g.vol, 12), 128), 128, 0, st>>>(A);
  WLG_LAUNCH_CHECK("hyp_level3");
}
template <class T>
void hyp_level2(const Geo& g, Links<T> U, const typename V2<T>::t* vbar, typename V2<T>::t* vtil,
                double a2, int proj, int iter, cudaStream_t st) {
  SArgs<T> A = sargs<T>(g);
  A.U = U;
  A.aux0 = const_cast<typename V2<T>::t*>(vbar);
  A.aux1 = vtil;
  A.a = 1.0 - a2;
  A.b = a2 / 4.0;
  A.proj = proj;
  A.iter = iter;
  k_hyp_l2<T><<<grid_for(tile_items(g.vol, 12), 128), 128, 0, st>>>(A);
  WLG_LAUNCH_CHECK("hyp_level2");
}
template <class T>
void hyp_level1(const Geo& g, Links<T> U, const typename V2<T>::t* vtil, double a1, int proj,
                int iter, int mu0, int mu1, int bc, cudaStream_t st) {
  int nmu = mu1 - mu0;
  if (nmu <= 0) return;
  SArgs<T> A = sargs<T>(g);
  A.U = U;
  A.aux1 = const_cast<typename V2<T>::t*>(vtil);
  A.a = 1.0 - a1;
  A.b = a1 / 6.0;
  A.proj = proj;
  A.iter = iter;
  A.mu0 = mu0;
  A.nmu = nmu;
  A.bc = bc;
  k_hyp_l1<T><<<grid_for(tile_items(g.vol, nmu), 128), 128, 0, st>>>(A);
  WLG_LAUNCH_CHECK("hyp_level1");
}
template <class T>
void ape_sweep(const Geo& g, Links<T> src, Links<T> dst, double alpha, int proj, int iter, int mu0,
               cudaStream_t st) {
  SArgs<T> A = sargs<T>(g);
  A.U = src;
  A.D = dst;
  A.a = alpha;
  A.proj = proj;
  A.iter = iter;
  A.mu0 = mu0;
  k_ape<T><<<grid_for(ape_items(g.vol, mu0), 128), 128, 0, st>>>(A);
  WLG_LAUNCH_CHECK("ape_sweep");
}
template <class T>
void hyp3d_level1(const Geo& g, Links<T> U, typename V2<T>::t* dl, double a2, int proj, int iter,
                  cudaStream_t st) {
  SArgs<T> A = sargs<T>(g);
  A.U = U;
  A.aux0 = dl;
  A.a = 1.0 - a2;
  A.b = a2 / 2.0;
  A.proj = proj;
  A.iter = iter;
  k_hyp3_l1<T><<<grid_for(6LL * g.vol, 128), 128, 0, st>>>(A);
  WLG_LAUNCH_CHECK("hyp3d_level1");
}
template <class T>
void hyp3d_level2(const Geo& g, Links<T> U, const typename V2<T>::t* dl, double a1, int proj,
                  int iter, cudaStream_t st) {
  SArgs<T> A = sargs<T>(g);
  A.D = U;
  A.aux0 = const_cast<typename V2<T>::t*>(dl);
  A.a = 1.0 - a1;
  A.b = a1 / 4.0;
  A.proj = proj;
  A.iter = iter;
  k_hyp3_l2<T><<<grid_for(3LL * g.vol, 128), 128, 0, st>>>(A);
  WLG_LAUNCH_CHECK("hyp3d_level2");
}
template <class T>
void smear_batch(int stage, const SArgs<T>* A, const long long* pre, int n, long long total,
                 cudaStream_t st) {
  if (n <= 0 || total <= 0) return;
  const int grid = grid_for(total, 128);
  switch (stage) {
    case BATCH_HYP3: kb_smear<T, BATCH_HYP3><<<grid, 128, 0, st>>>(A, pre, n, total); break;
    case BATCH_HYP2: kb_smear<T, BATCH_HYP2><<<grid, 128, 0, st>>>(A, pre, n, total); break;
    case BATCH_HYP1: kb_smear<T, BATCH_HYP1><<<grid, 128, 0, st>>>(A, pre, n, total); break;
    case BATCH_APE: kb_smear<T, BATCH_APE><<<grid, 128, 0, st>>>(A, pre, n, total); break;
    case BATCH_HYP3D1: kb_smear<T, BATCH_HYP3D1><<<grid, 128, 0, st>>>(A, pre, n, total); break;
    case BATCH_HYP3D2: kb_smear<T, BATCH_HYP3D2><<<grid, 128, 0, st>>>(A, pre, n, total); break;
    default: set_error("smear_batch: unknown stage %d", stage); return;
  }
  WLG_LAUNCH_CHECK("smear_batch");
}

template <class T>
void staple_sum(const Geo& g, Links<T> u1, Links<T> u2, int mu, int nu, Links<T> vb,
                cudaStream_t st) {
  k_staple_sum<T><<<grid_for(g.vol, 128), 128, 0, st>>>(g, u1, u2, mu, nu, vb);
  WLG_LAUNCH_CHECK("staple_sum");
}
void project_batch(double* m, int n, int iter, cudaStream_t st) {
  if (n <= 0) return;
  k_project_batch<<<grid_for(n, 128), 128, 0, st>>>(m, n, iter);
  WLG_LAUNCH_CHECK("project_batch");
}
template <class T>
void plaq_sum(const Geo& g, int bc, Links<T> U, double* partial, double* out, cudaStream_t st) {
  k_plaq<T><<<kPlaqBlocks, kPlaqThreads, 0, st>>>(g, bc, U, partial);
  WLG_LAUNCH_CHECK("plaq_sum");
  k_sum_partials<<<1, 1024, 0, st>>>(partial, kPlaqBlocks, out);
  WLG_LAUNCH_CHECK("plaq_sum_final");
}

#define WLG_INST(T)                                                                               \
  template void hyp_level3<T>(const Geo&, Links<T>, V2<T>::t*, double, int, int, cudaStream_t);   \
  template void hyp_level2<T>(const Geo&, Links<T>, const V2<T>::t*, V2<T>::t*, double, int, int, \
                              cudaStream_t);                                                      \
  template void hyp_level1<T>(const Geo&, Links<T>, const V2<T>::t*, double, int, int, int, int,  \
                              int, cudaStream_t);                                                 \
  template void ape_sweep<T>(const Geo&, Links<T>, Links<T>, double, int, int, int, cudaStream_t); \
  template void hyp3d_level1<T>(const Geo&, Links<T>, V2<T>::t*, double, int, int, cudaStream_t); \
  template void hyp3d_level2<T>(const Geo&, Links<T>, const V2<T>::t*, double, int, int,          \
                                cudaStream_t);                                                    \
  template void staple_sum<T>(const Geo&, Links<T>, Links<T>, int, int, Links<T>, cudaStream_t);  \
  template void plaq_sum<T>(const Geo&, int, Links<T>, double*, double*, cudaStream_t);    \
  template void smear_batch<T>(int, const SArgs<T>*, const long long*, int, long long, cudaStream_t);

WLG_INST(double)
WLG_INST(float)

}  // namespace wlg
