// gram.cu -- the Wilson-loop stage in the temporal gauge: the contraction as
// a banded Gram product of gauge-transformed spatial lines.
//
// Every term of the loop sum (wloop.c:436-508, get_wloop :261-433)
//     Re tr[ S_s1(x) L_T(x+R k) S_s2(x+T)^dag L_T(x)^dag ]
// is the trace of a closed loop.  With g(x0,xs) = U0(0,xs) U0(1,xs) ...
// U0(x0-1,xs) the temporal line is exactly L_T(x) = g(x0)^-1 g(x0+T) (the
// smeared links need not be exactly unitary: the approximate projection
// leaves them unitary only approximately), and the term becomes
//     Re tr[ A_s1(x0,xs) B_s2(x0+T,xs)^dag ],
//     B(x) = g(x) S(x) g(x+Rk)^dag,   A(x) = H(x)^-1 B(x) H(x+Rk)^-1,   H = g g^dag
// (A = B for unitary links): a real dot product of the 18 numbers of two
// matrices.  The lines obey B(x,R+1) = B(x,R) Uh(x+Rk) with the transformed
// links Uh(y) = H(y)^-1 g(y) U_k(y) g(y+k)^dag and B(x,1) = H(x) Uh(x).  For
// periodic time the time axis is unrolled to Nu = N0 + mwlt slices with
// g(N0+y) = P g(y) (P the time-line product through the lattice), so a loop
// from x0 to x0+T past the last slice reads the wrapped temporal links
// through g; for open time (Nu = N0) the loops that cross the last slice
// contain its zero temporal link and are exact zeros.  Per extent R the
// stage is therefore
//     W_{s1 s2}(x0,T) = sum_{xs,k,c} VA[x0,s1][xs,k,c] VB[x0+T,s2][xs,k,c] / (9 N1 N2 N3)
// with VA, VB the matrices whose rows are (slice, level) and whose columns
// are (site, direction, component): 36 msl^2 flops per site and (T,R)
// instead of the 2 msl M + 36 msl^2 of carrying the temporal lines (M = 198).
// If g is far from unitary (max |H - 1| > 1/4: no projection, or one that
// has not converged on a rough field) the form is not used, since H^-1 would
// amplify rounding; the caller checks.
//
// Slab layout (this file only): a field over the unrolled volume Nu x vs,
// one array per (level, direction), of element type E (float, double):
//     component c (= 2 e + {0: re, 1: im} of entry e, row-major) of site
//     (y0, j), j the lexicographic spatial index, at
//         ((y0 * ntile + j / 32) * 18 + c) * 32 + j % 32,   ntile = ceil(vs / 32),
// so one slice of one array is contiguous, a warp reads or writes one
// component of 32 sites as one 128-byte line, and a run of 32 (FP32) or 16
// (FP64) consecutive elements is one column chunk of the Gram product.  Sites
// j >= vs of the last tile are zeros (they add nothing to any sum).  The A
// lines have N0 slices (start slices only), the others Nu.
//
// g, H^-1 and the transformed links are computed in FP64 in both forms (the
// mixed form stores the links and lines rounded to FP32, as it stores the
// smeared links); the line products are in the stored type; the Gram product accumulates
// in the form's type over a bounded run of columns per block (FP32: a few
// thousand products) and the per-block partial sums are added in FP64 in a
// fixed order.
#include <algorithm>
#include <cmath>
#include <mutex>
#include <set>
#include <utility>

#include "internal.h"

namespace wlg {
namespace {

constexpr int kSlabTile = 576;  // elements per 32-site tile of one slab array

__host__ __device__ __forceinline__ size_t slab_tile(int y0, int ntile, int jt) {
  return (size_t)y0 * ntile + jt;
}

template <class E>
__device__ __forceinline__ void ld_slab(M3<double>& m, const E* __restrict__ base, size_t tile,
                                        int lane) {
  const E* p = base + tile * kSlabTile + lane;
#pragma unroll
  for (int e = 0; e < 9; e++) {
    m.e[e].x = (double)__ldg(p + (2 * e) * 32);
    m.e[e].y = (double)__ldg(p + (2 * e + 1) * 32);
  }
}

template <class E>
__device__ __forceinline__ void st_slab(E* __restrict__ base, size_t tile, int lane,
                                        const M3<double>& m) {
  E* p = base + tile * kSlabTile + lane;
#pragma unroll
  for (int e = 0; e < 9; e++) {
    p[(2 * e) * 32] = (E)m.e[e].x;
    p[(2 * e + 1) * 32] = (E)m.e[e].y;
  }
}

// the same in arithmetic type A (loads convert from the stored type S)
template <class A, class S>
__device__ __forceinline__ void ld_slab_as(M3<A>& m, const S* __restrict__ base, size_t tile,
                                           int lane) {
  const S* p = base + tile * kSlabTile + lane;
#pragma unroll
  for (int e = 0; e < 9; e++) {
    m.e[e].x = (A)__ldg(p + (2 * e) * 32);
    m.e[e].y = (A)__ldg(p + (2 * e + 1) * 32);
  }
}

template <class E, class A>
__device__ __forceinline__ void st_slab_from(E* __restrict__ base, size_t tile, int lane,
                                             const M3<A>& m) {
  E* p = base + tile * kSlabTile + lane;
#pragma unroll
  for (int e = 0; e < 9; e++) {
    p[(2 * e) * 32] = (E)m.e[e].x;
    p[(2 * e + 1) * 32] = (E)m.e[e].y;
  }
}

template <class E> __device__ __forceinline__ void zero_slab(E* __restrict__ base, size_t tile, int lane) {
  E* p = base + tile * kSlabTile + lane;
#pragma unroll
  for (int c = 0; c < 18; c++) p[c * 32] = E(0);
}

__device__ __forceinline__ void unit(M3<double>& m) {
  zero(m);
  m.e[0].x = m.e[4].x = m.e[8].x = 1.0;
}

// 3x3 complex inverse by cofactors, inv = adj(h) / det(h)
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ void inverse3(M3<double>& inv, const M3<double>& h) {
  const double2* e = h.e;
  // cofactor matrix transposed: inv_ij = C_ji
  double2 c00 = csub(cmul(e[4], e[8]), cmul(e[5], e[7]));
  double2 c01 = csub(cmul(e[2], e[7]), cmul(e[1], e[8]));
  double2 c02 = csub(cmul(e[1], e[5]), cmul(e[2], e[4]));
  double2 c10 = csub(cmul(e[5], e[6]), cmul(e[3], e[8]));
  double2 c11 = csub(cmul(e[0], e[8]), cmul(e[2], e[6]));
  double2 c12 = csub(cmul(e[2], e[3]), cmul(e[0], e[5]));
  double2 c20 = csub(cmul(e[3], e[7]), cmul(e[4], e[6]));
  double2 c21 = csub(cmul(e[1], e[6]), cmul(e[0], e[7]));
  double2 c22 = csub(cmul(e[0], e[4]), cmul(e[1], e[3]));
  double2 det = cmul(e[0], c00);
  double2 t = cmul(e[1], c10);
  det.x += t.x;
  det.y += t.y;
  t = cmul(e[2], c20);
  det.x += t.x;
  det.y += t.y;
  const double n = det.x * det.x + det.y * det.y;
  const double2 r = make_double2(det.x / n, -det.y / n);  // 1 / det
  inv.e[0] = cmul(c00, r);
  inv.e[1] = cmul(c01, r);
  inv.e[2] = cmul(c02, r);
  inv.e[3] = cmul(c10, r);
  inv.e[4] = cmul(c11, r);
  inv.e[5] = cmul(c12, r);
  inv.e[6] = cmul(c20, r);
  inv.e[7] = cmul(c21, r);
  inv.e[8] = cmul(c22, r);
}

// ---------------------------------------------------------------------------
// g(y0, j) and H^-1(y0, j) = (g g^dag)^-1 for y0 in [0, Nu): g(0) = 1,
// g(y0+1) = g(y0) U0(y0 mod N0, j); FP64 slabs.  One thread per spatial site
// (the chain is sequential in time).  *dev receives max |H - 1| over the
// sites (as the bits of a non-negative double, atomicMax).
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(128) k_gauge_chain(Geo g, int Nu, int ntile,
                                                     const typename V2<T>::t* __restrict__ u0,
                                                     double* __restrict__ G,
                                                     double* __restrict__ Hinv,
                                                     unsigned long long* __restrict__ dev) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  double worst = 0.0;
  if (j < ntile * 32) {
    const int jt = j >> 5, lane = j & 31;
    if (j >= g.vs) {
      for (int y0 = 0; y0 < Nu; y0++) {
        zero_slab(G, slab_tile(y0, ntile, jt), lane);
        zero_slab(Hinv, slab_tile(y0, ntile, jt), lane);
      }
    } else {
      M3<double> m, t, ud;
      unit(m);
      for (int y0 = 0; y0 < Nu; y0++) {
        const size_t tile = slab_tile(y0, ntile, jt);
        st_slab(G, tile, lane, m);
        mul_ad(t, m, m);  // H = g g^dag
#pragma unroll
        for (int e = 0; e < 9; e++) {
          const double dr = fabs(t.e[e].x - ((e % 4 == 0) ? 1.0 : 0.0)), di = fabs(t.e[e].y);
          if (!(dr <= worst)) worst = dr;  // a NaN sticks
          if (!(di <= worst)) worst = di;
        }
        inverse3(ud, t);
        st_slab(Hinv, tile, lane, ud);
        if (y0 + 1 < Nu) {
          M3<T> u;
          ld<T>(u, u0, g.vol, (y0 % g.n[0]) * g.vs + j);
          cvt(ud, u);
          mul(t, m, ud);
          m = t;
        }
      }
    }
  }
  // NaN (a singular chain) compares as the largest value
  if (worst != worst) worst = 1e300;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) worst = fmax(worst, __shfl_xor_sync(0xffffffffu, worst, o));
  if ((threadIdx.x & 31) == 0) atomicMax(dev, (unsigned long long)__double_as_longlong(worst));
}

// ---------------------------------------------------------------------------
// Lines of length 1 and the recursion links, per (k, y0, tile, lane), all
// levels per item:
//     B1 = g(y) U_k(y mod N0) g(y+k)^dag      -> B lines   (all Nu slices)
//     Uh = H^-1(y) B1                        -> recursion (all Nu slices)
//     A1 = Uh H^-1(y+k)                      -> A lines   (y0 < N0; unless
//                                           alines is null, when a line step
//                                           with R = 1 writes them)
// FP64 products, stored as E.
// ---------------------------------------------------------------------------
template <class T, class E>
__global__ void __launch_bounds__(128) k_gauge_first(Geo g, int Nu, int ntile, int msl,
                                                     const typename V2<T>::t* __restrict__ lev,
                                                     size_t lev_stride,
                                                     const double* __restrict__ G,
                                                     const double* __restrict__ Hinv,
                                                     E* __restrict__ uh, E* __restrict__ blines,
                                                     E* __restrict__ alines, size_t A, size_t Aa) {
  const long long n = (long long)3 * Nu * ntile * 32;
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < n;
       w += (long long)gridDim.x * blockDim.x) {
    const int lane = (int)(w & 31);
    long long rest = w >> 5;
    const int jt = (int)(rest % ntile);
    rest /= ntile;
    const int y0 = (int)(rest % Nu);
    const int k = (int)(rest / Nu);
    const int j = jt * 32 + lane;
    const size_t tile = slab_tile(y0, ntile, jt);
    const bool start = y0 < g.n[0];
    if (j >= g.vs) {
      for (int sl = 0; sl < msl; sl++) {
        zero_slab(uh + (size_t)(sl * 3 + k) * A, tile, lane);
        zero_slab(blines + (size_t)(sl * 3 + k) * A, tile, lane);
        if (start && alines) zero_slab(alines + (size_t)(sl * 3 + k) * Aa, tile, lane);
      }
      continue;
    }
    const int x0 = y0 % g.n[0];
    const int s = x0 * g.vs + j;
    int x[4];
    coords(g, s, x);
    const int jr = up(g, s, x[k + 1], k + 1) - x0 * g.vs;
    const size_t tr = slab_tile(y0, ntile, jr >> 5);
    for (int sl = 0; sl < msl; sl++) {
      // the four g / H^-1 factors are re-read per level (L1 hits) rather
      // than held, which would exceed the register file
      const size_t q = (size_t)(sl * 3 + k);
      M3<double> f, ud, t1, t2;
      M3<T> u;
      ld<T>(u, lev + q * lev_stride, g.vol, s);
      cvt(ud, u);
      ld_slab(f, G, tile, lane);
      mul(t1, f, ud);
      ld_slab(f, G, tr, jr & 31);
      mul_ad(t2, t1, f);
      st_slab(blines + q * A, tile, lane, t2);
      ld_slab(f, Hinv, tile, lane);
      mul(t1, f, t2);
      st_slab(uh + q * A, tile, lane, t1);
      if (start && alines) {
        ld_slab(f, Hinv, tr, jr & 31);
        mul(t2, t1, f);
        st_slab(alines + q * Aa, tile, lane, t2);
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Line step: B(y, j) <- B(y, j) Uh(y, j + (R-1) k) in place (compute_uk_long,
// wloop.c:207-258, multiplied at the far end), and for the start slices
// A(y, j) = H^-1(y, j) B(y, j) H^-1(y, j + R k); products in the stored type
// (the mixed form's as packed two-lane FP32 FMAs: each line is rounded to
// FP32 at every step anyway, and FP64 products here cost FP64-pipe time and
// registers that limited this HBM-bound kernel).  With R = 1 only A, from
// the lines of length 1.
// ---------------------------------------------------------------------------
template <class E>
__global__ void __launch_bounds__(128) k_gauge_line_step(Geo g, int Nu, int ntile, int msl, int R,
                                                         const E* __restrict__ uh,
                                                         const double* __restrict__ Hinv,
                                                         E* __restrict__ blines,
                                                         E* __restrict__ alines, size_t A,
                                                         size_t Aa) {
  // item order (y0, tile, level x direction, lane): the 3 msl arrays of one
  // tile run in neighbouring warps, so the two H^-1 tiles they share come
  // from L2 rather than once per array from DRAM
  const int nq = msl * 3;
  const long long n = (long long)nq * Nu * ntile * 32;
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < n;
       w += (long long)gridDim.x * blockDim.x) {
    const int lane = (int)(w & 31);
    long long rest = w >> 5;
    const int q = (int)(rest % nq);  // sl * 3 + k
    rest /= nq;
    const int jt = (int)(rest % ntile);
    const int y0 = (int)(rest / ntile);
    const int k = q % 3;
    const int j = jt * 32 + lane;
    const size_t tile = slab_tile(y0, ntile, jt);
    const bool start = y0 < g.n[0];
    if (j >= g.vs) {  // B: zeros since the first lines; A: zeros written here
      if (R == 1 && start) zero_slab(alines + (size_t)q * Aa, tile, lane);
      continue;
    }
    if (R == 1 && !start) continue;
    int x[4];
    coords(g, j, x);  // slice 0: the spatial coordinates of j
    const int n_k = g.n[k + 1];
    M3<E> a, b, c;
    if (R >= 2) {
      const int jr = shift(g, j, x[k + 1], k + 1, (R - 1) % n_k);
      ld_slab_as(a, blines + (size_t)q * A, tile, lane);
      ld_slab_as(b, uh + (size_t)q * A, slab_tile(y0, ntile, jr >> 5), jr & 31);
      mul(c, a, b);
      st_slab_from(blines + (size_t)q * A, tile, lane, c);
    } else {
      ld_slab_as(c, blines + (size_t)q * A, tile, lane);
    }
    if (start) {
      const int je = shift(g, j, x[k + 1], k + 1, R % n_k);
      ld_slab_as(a, Hinv, tile, lane);
      mul(b, a, c);
      ld_slab_as(a, Hinv, slab_tile(y0, ntile, je >> 5), je & 31);
      mul(c, b, a);
      st_slab_from(alines + (size_t)q * Aa, tile, lane, c);
    }
  }
}

// ---------------------------------------------------------------------------
// The banded Gram product.  Block (blk, split) owns the start slices
// x0 in [blk*BX, blk*BX + BX) and every extent T in [1, mwlt], over the
// column chunks [split*cpc, split*cpc + cpc).  A chunk is a run of KW
// consecutive slab elements of one direction (32 sites x 1 component in FP32,
// 16 in FP64, 128 bytes).  Per chunk the block stages its A rows (sl, x0) and
// its B rows (sl, y0), y0 in [blk*BX + 1, blk*BX + BX + mwlt), into shared
// memory with cp.async, `stages` chunks ahead of the arithmetic.  A staged
// row is 128 bytes, its 16-byte slot q stored at q ^ (row & 7) so that eight
// consecutive rows read at one slot fall on distinct banks; each level's rows
// start at a multiple of 8 (A rows BXp apart, B rows NYBp apart), so a
// thread's swizzle is fixed.  Thread (i, gq) owns start slice x0 = blk*BX + i
// and the TQ extents T = gq + 1 + NG j (j < TQ): per 16-byte column group it
// reads the L A-vectors of its slice and, one at a time, the L B-vectors of
// each partner slice, and advances the L sums of a B vector (the order of
// the FMAs and the occupancy -- one block of 256, two of 192 or one of 384
// threads per SM -- are kernel variants; the plan picks one per precision).
// Lanes of a warp share start slices (broadcast reads), and the partner rows
// one read of a warp touches span at most 32/NG + NG - 1 consecutive slices.
// ---------------------------------------------------------------------------
template <class E> struct GVec;
template <> struct GVec<float> {
  typedef float4 t;
  enum { N = 4 };
};
template <> struct GVec<double> {
  typedef double2 t;
  enum { N = 2 };
};
__device__ __forceinline__ float comp(const float4& v, int c) {
  return c == 0 ? v.x : (c == 1 ? v.y : (c == 2 ? v.z : v.w));
}
__device__ __forceinline__ double comp(const double2& v, int c) { return c == 0 ? v.x : v.y; }

__device__ __forceinline__ void gcp_async16(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void gcp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
// wait until at most n of this thread's newest copy groups are in flight
__device__ __forceinline__ void gcp_wait(int n) {
  if (n >= 2)
    asm volatile("cp.async.wait_group 2;\n" ::: "memory");
  else if (n == 1)
    asm volatile("cp.async.wait_group 1;\n" ::: "memory");
  else
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
}

constexpr int kRowBytes = 128;
// occupancy variants: OCC 1 = one block of up to 256 threads per SM (255
// registers a thread), OCC 2 = two blocks of up to 192 threads (170
// registers), OCC 3 = one block of up to 384 threads (170 registers)
__host__ __device__ constexpr int gram_threads(int occ) {
  return occ == 2 ? 192 : (occ == 3 ? 384 : 256);
}
__host__ __device__ constexpr int gram_blocks_per_sm(int occ) { return occ == 2 ? 2 : 1; }
constexpr int kMaxGramThreads = 384;
constexpr unsigned kNoRow = 0xffffffffu;

struct GramArgs {
  const void* alines;  // [msl][3] slab arrays of Aa elements (N0 slices)
  const void* blines;  // [msl][3] slab arrays of A elements (Nu slices)
  void* partial;       // [nsplit][N0][mwlt][L][L] partial sums (element type of the form)
  size_t A, Aa;
  int Nu, ntile, N0, mwlt, BX, BXp, NG, NYB, NYBp, nblk, nchunks, cpc, stages, nrows;
};

__host__ __device__ __forceinline__ int gram_tab_bytes(int nrows) { return (nrows * 4 + 127) & ~127; }
__host__ __device__ __forceinline__ int round8(int v) { return (v + 7) & ~7; }

// ORD 0: each B vector's dot products as chains of VN dependent FMAs (the L
// chains of one B vector interleave); ORD 1: one component at a time over
// the L sums of a B vector
template <class E, int L, int TQ, int OCC, int ORD>
__global__ void __launch_bounds__(gram_threads(OCC), gram_blocks_per_sm(OCC)) k_gram(GramArgs P) {
  constexpr int KW = 128 / (int)sizeof(E);
  constexpr int VN = GVec<E>::N;
  typedef typename GVec<E>::t V;
  extern __shared__ __align__(128) unsigned char gsm[];
  // row table: offset of row r's slice in 16-byte units from the A (r < nA)
  // or the B lines, kNoRow for rows not loaded
  unsigned* rowtab = reinterpret_cast<unsigned*>(gsm);
  unsigned char* stage0 = gsm + gram_tab_bytes(P.nrows);
  const int blk = blockIdx.x % P.nblk, split = blockIdx.x / P.nblk;
  const int c0 = split * P.cpc;
  const int nk = min(P.nchunks, c0 + P.cpc) - c0;
  const size_t stage_bytes = (size_t)P.nrows * kRowBytes;
  const int nA = L * P.BXp;  // rows [0, nA): A rows (sl, x0); then B rows (sl, y0)
  const size_t tile_bytes = (size_t)P.ntile * kSlabTile * sizeof(E);
  for (int r = threadIdx.x; r < P.nrows; r += blockDim.x) {
    unsigned off = kNoRow;  // padding rows and rows past the lattice stay unloaded
    if (r < nA) {
      const int sl = r / P.BXp, ii = r - sl * P.BXp, y0 = blk * P.BX + ii;
      if (ii < P.BX && y0 < P.N0)
        off = (unsigned)(((size_t)(sl * 3) * P.Aa * sizeof(E) + (size_t)y0 * tile_bytes) >> 4);
    } else {
      const int rr = r - nA, sl = rr / P.NYBp, yy = rr - sl * P.NYBp, y0 = blk * P.BX + 1 + yy;
      if (yy < P.NYB && y0 < P.Nu)
        off = (unsigned)(((size_t)(sl * 3) * P.A * sizeof(E) + (size_t)y0 * tile_bytes) >> 4);
    }
    rowtab[r] = off;
  }
  __syncthreads();
  const int per_dir = P.ntile * 18 * (32 / KW);
  const int npieces = P.nrows * 8;
  auto issue = [&](int cidx, int buf) {
    const int k = cidx / per_dir;
    const size_t within = (size_t)(cidx - k * per_dir) * KW;
    const char* baseA = static_cast<const char*>(P.alines) + ((size_t)k * P.Aa + within) * sizeof(E);
    const char* baseB = static_cast<const char*>(P.blines) + ((size_t)k * P.A + within) * sizeof(E);
    unsigned char* dst = stage0 + (size_t)buf * stage_bytes;
    for (int p = threadIdx.x; p < npieces; p += blockDim.x) {
      const int r = p >> 3, q = p & 7;
      const unsigned ro = rowtab[r];
      if (ro != kNoRow)
        gcp_async16(dst + r * kRowBytes + ((q ^ (r & 7)) << 4),
                    (r < nA ? baseA : baseB) + ((size_t)ro << 4) + q * 16);
    }
  };

  int i = threadIdx.x / P.NG;
  const int gq = threadIdx.x - i * P.NG;
  const int x0 = blk * P.BX + i;
  const bool live = (i < P.BX) && (x0 < P.N0);
  if (i >= P.BX) i = P.BX - 1;  // idle threads read in-range rows and store nothing
  const int sa = i & 7;         // swizzle of this thread's A rows
  int brow[TQ], sb[TQ];
#pragma unroll
  for (int j = 0; j < TQ; j++) {
    int T = gq + 1 + P.NG * j;
    if (T > P.mwlt) T = P.mwlt;
    brow[j] = nA + i + T - 1;
    sb[j] = (i + T - 1) & 7;
  }
  E acc[TQ][L][L];
#pragma unroll
  for (int j = 0; j < TQ; j++)
#pragma unroll
    for (int a = 0; a < L; a++)
#pragma unroll
      for (int b = 0; b < L; b++) acc[j][a][b] = E(0);

  for (int s = 0; s < P.stages - 1; s++) {
    if (s < nk) issue(c0 + s, s);
    gcp_commit();
  }
  const size_t astride = (size_t)P.BXp * kRowBytes, bstride = (size_t)P.NYBp * kRowBytes;
  for (int it = 0; it < nk; it++) {
    gcp_wait(P.stages - 2);
    __syncthreads();
    {
      const int nx = it + P.stages - 1;
      if (nx < nk) issue(c0 + nx, nx % P.stages);
      gcp_commit();
    }
    const unsigned char* st = stage0 + (size_t)(it % P.stages) * stage_bytes;
    const unsigned char* arow = st + (size_t)i * kRowBytes;
#pragma unroll 1
    for (int qk = 0; qk < 8; qk++) {  // 16-byte column groups of the chunk
      V a[L];
#pragma unroll
      for (int s1 = 0; s1 < L; s1++)
        a[s1] = *reinterpret_cast<const V*>(arow + s1 * astride + ((qk ^ sa) << 4));
#pragma unroll
      for (int j = 0; j < TQ; j++) {
        const unsigned char* bp = st + (size_t)brow[j] * kRowBytes + ((qk ^ sb[j]) << 4);
#pragma unroll
        for (int s2 = 0; s2 < L; s2++) {
          const V b = *reinterpret_cast<const V*>(bp + s2 * bstride);
          if constexpr (ORD == 0) {
#pragma unroll
            for (int s1 = 0; s1 < L; s1++)
#pragma unroll
              for (int c = 0; c < VN; c++)
                acc[j][s1][s2] = fma(comp(a[s1], c), comp(b, c), acc[j][s1][s2]);
          } else {
#pragma unroll
            for (int c = 0; c < VN; c++)
#pragma unroll
              for (int s1 = 0; s1 < L; s1++)
                acc[j][s1][s2] = fma(comp(a[s1], c), comp(b, c), acc[j][s1][s2]);
          }
        }
      }
    }
  }
  gcp_wait(0);
  if (live) {
    E* out = static_cast<E*>(P.partial) + ((size_t)split * P.N0 + x0) * P.mwlt * L * L;
#pragma unroll
    for (int j = 0; j < TQ; j++) {
      const int T = gq + 1 + P.NG * j;
      if (T <= P.mwlt) {
        E* o = out + (size_t)(T - 1) * L * L;
#pragma unroll
        for (int s2 = 0; s2 < L; s2++)
#pragma unroll
          for (int s1 = 0; s1 < L; s1++) o[s2 * L + s1] = acc[j][s1][s2];
      }
    }
  }
}

// wl[wl_idx(s1,s2,t,r,x0)] = sum over the splits (FP64, fixed order) / norm;
// open time: the loops through the last slice are exact zeros
template <class E>
__global__ void __launch_bounds__(256) k_gram_reduce(const E* __restrict__ partial, int nsplit,
                                                     int N0, int mwlt, int L, int mwlr, int r,
                                                     int open, double norm, double* __restrict__ wl) {
  const int LL = L * L, nout = N0 * mwlt * LL;
  for (int o = blockIdx.x * blockDim.x + threadIdx.x; o < nout; o += gridDim.x * blockDim.x) {
    const int x0 = o / (mwlt * LL);
    int rem = o - x0 * mwlt * LL;
    const int t = rem / LL;
    rem -= t * LL;
    const int s2 = rem / L, s1 = rem - s2 * L;
    double v = 0.0;
    if (!open || x0 + t + 1 < N0) {
      for (int sp = 0; sp < nsplit; sp++) v += (double)__ldg(partial + (size_t)sp * nout + o);
      v = v / norm;
    }
    wl[s1 + L * (s2 + L * (t + mwlt * (r + mwlr * x0)))] = v;
  }
}

// ---------------------------------------------------------------------------
// Instantiations (element, levels L, extents per thread TQ, occupancy OCC,
// FMA order ORD).  The first entry of a (type, L) pair is its default; the
// others are tuning candidates or serve where the default's rows do not fit
// its shared memory.  FP32 keeps at most 128 sums per thread
// (72 in OCC 3), FP64 at most 64 doubles in OCC 2 (170 registers) and 72 in
// OCC 1.
// ---------------------------------------------------------------------------
#define WLG_GRAM_VARIANTS(X)                                                                   \
  X(float, 1, 8, 1, 0) X(float, 2, 8, 1, 0) X(float, 3, 6, 1, 0) X(float, 4, 6, 1, 0)           \
  X(float, 4, 4, 1, 0) X(float, 5, 4, 1, 0) X(float, 6, 3, 1, 0) X(float, 6, 3, 1, 1)           \
  X(float, 6, 3, 2, 0) X(float, 6, 3, 2, 1) X(float, 6, 2, 3, 0) X(float, 4, 4, 3, 0)           \
  X(float, 7, 2, 1, 0) X(float, 8, 2, 1, 0)                                                     \
  X(double, 1, 8, 2, 1) X(double, 2, 6, 2, 1) X(double, 3, 4, 2, 1) X(double, 4, 3, 2, 1)       \
  X(double, 4, 2, 2, 1) X(double, 5, 2, 2, 1) X(double, 6, 1, 2, 1) X(double, 6, 1, 2, 0)       \
  X(double, 6, 2, 1, 0) X(double, 6, 2, 1, 1) X(double, 7, 1, 2, 1) X(double, 8, 1, 2, 1)       \
  X(double, 7, 1, 1, 1) X(double, 8, 1, 1, 1)

void* gram_kernel(int esize, int L, int TQ, int occ, int ord) {
#define WLG_GRAM_PICK(ET, LL, TT, OO, RR)                                                     \
  if (esize == (int)sizeof(ET) && L == LL && TQ == TT && occ == OO && ord == RR)              \
    return (void*)k_gram<ET, LL, TT, OO, RR>;
  WLG_GRAM_VARIANTS(WLG_GRAM_PICK)
#undef WLG_GRAM_PICK
  return nullptr;
}

struct GramVariant {
  int TQ, occ, ord;
};
// the variants for (esize, L) that match the requested occupancy / order
// (0: any), in table order
static int gram_variants(int esize, int L, int occ, int ord, GramVariant* out, int max) {
  int n = 0;
#define WLG_GRAM_LIST(ET, LL, TT, OO, RR)                                                     \
  if (esize == (int)sizeof(ET) && L == LL && (occ == 0 || occ == OO) &&                      \
      (ord == 0 || ord - 1 == RR) && n < max)                                                 \
    out[n++] = GramVariant{TT, OO, RR};
  WLG_GRAM_VARIANTS(WLG_GRAM_LIST)
#undef WLG_GRAM_LIST
  return n;
}

}  // namespace

bool gram_plan(GramPlan& p, const Geo& g, int bc, int msl, int mwlt, bool fp64,
               const GramTuning* tune) {
  GramTuning none;
  if (!tune) tune = &none;
  p = GramPlan();
  if (msl < 1 || msl > 8 || mwlt < 1 || g.n[0] < 1 || g.vs < 1) return false;
  const int esz = fp64 ? 8 : 4;
  p.esize = esz;
  p.L = msl;
  p.Nu = g.n[0] + (bc == 0 ? 0 : mwlt);
  p.ntile = (g.vs + 31) / 32;
  p.A = (size_t)p.Nu * p.ntile * kSlabTile;
  p.Aa = (size_t)g.n[0] * p.ntile * kSlabTile;
  GramVariant cand[16];
  const int nc = gram_variants(esz, msl, tune->occ, tune->ord, cand, 16);
  const int N0 = g.n[0];
  // the (occupancy, order) groups in table order: the first is the level
  // count's default, a later one serves where the default's rows do not fit
  // its shared memory (two blocks per SM on a long time extent)
  for (int grp = 0; grp < nc && p.BX == 0; grp++) {
    bool seen = false;
    for (int c = 0; c < grp; c++)
      seen = seen || (cand[c].occ == cand[grp].occ && cand[c].ord == cand[grp].ord);
    if (seen) continue;
    // the group's variant with the extents per thread that waste the fewest
    // (ties: the first listed)
    int best = -1, bw = 1 << 30;
    for (int c = grp; c < nc; c++) {
      if (cand[c].occ != cand[grp].occ || cand[c].ord != cand[grp].ord) continue;
      const int ng = (mwlt + cand[c].TQ - 1) / cand[c].TQ;
      const int waste = ng * cand[c].TQ - mwlt;
      if (waste < bw) {
        bw = waste;
        best = c;
      }
    }
    const int TQ = cand[best].TQ, occ = cand[best].occ;
    const int NG = (mwlt + TQ - 1) / TQ;
    const int cap = gram_threads(occ);
    if (NG > cap) continue;
    const int bxmax = std::min(cap / NG, tune->bx > 0 ? tune->bx : N0);
    // the fewest start-slice blocks whose rows fit two stages in the shared
    // memory of one block (half an SM's for two blocks per SM)
    const size_t lim = gram_blocks_per_sm(occ) == 2 ? 113 * 1024 : 227 * 1024;
    for (int nblk = (N0 + bxmax - 1) / bxmax; nblk <= N0; nblk++) {
      const int BX = (N0 + nblk - 1) / nblk;
      const int nrows = msl * (round8(BX) + round8(BX + mwlt - 1));
      const size_t tab = (size_t)gram_tab_bytes(nrows), per = (size_t)nrows * kRowBytes;
      if (tab + 2 * per > lim) continue;
      p.TQ = TQ;
      p.occ = occ;
      p.ord = cand[best].ord;
      p.NG = NG;
      p.BX = BX;
      p.BXp = round8(BX);
      p.nblk = (N0 + BX - 1) / BX;
      p.NYB = BX + mwlt - 1;
      p.NYBp = round8(p.NYB);
      p.nrows = nrows;
      p.stages = (int)std::min<size_t>(4, (lim - tab) / per);
      if (tune->stages >= 2 && tune->stages < p.stages) p.stages = tune->stages;
      p.smem = tab + (size_t)p.stages * per;
      break;
    }
  }
  if (p.BX == 0) return false;
  // row offsets are kept as 32-bit multiples of 16 bytes
  if ((size_t)3 * msl * p.A * esz / 16 >= (size_t)kNoRow) return false;
  p.block = ((p.BX * p.NG + 31) / 32) * 32;
  p.nchunks = 3 * p.ntile * 18 * (32 * esz / 128);
  // column chunks per block: as many as the precision allows (at most 512;
  // FP32 at most 2 sqrt(nchunks / 32): the rounding error of one FP32
  // partial grows with its run of n = cpc x 32 products and the relative
  // error of W after the FP64 sum of the partials as n / sqrt(all
  // products), so this keeps it at one level, about 1e-7 of W, on small and
  // large lattices); then the splits rounded so that the blocks fill whole
  // waves of the SMs
  long long cmax = 512;
  if (!fp64) cmax = std::min(cmax, (long long)(2.0 * std::sqrt((double)p.nchunks / 32.0)));
  if (tune->cpc > 0) cmax = tune->cpc;
  if (cmax < 1) cmax = 1;
  const long long slots = (long long)num_sms() * gram_blocks_per_sm(p.occ);
  const long long total = (long long)p.nchunks * p.nblk;
  long long waves = (total + cmax * slots - 1) / (cmax * slots);
  long long nsplit = std::max(1LL, (waves * slots) / p.nblk);
  long long cpc = (p.nchunks + nsplit - 1) / nsplit;
  if (tune->cpc > 0) cpc = tune->cpc;
  p.cpc = (int)std::max(1LL, std::min(cpc, cmax));
  p.nsplit = (p.nchunks + p.cpc - 1) / p.cpc;
  p.partial_elems = (size_t)p.nsplit * N0 * mwlt * msl * msl;
  return true;
}

template <class T>
void gauge_chain(const Geo& g, const GramPlan& p, const typename V2<T>::t* u0, double* G,
                 double* Hinv, unsigned long long* dev, cudaStream_t st) {
  const int nthr = p.ntile * 32;
  cudaMemsetAsync(dev, 0, sizeof(unsigned long long), st);
  k_gauge_chain<T><<<(nthr + 127) / 128, 128, 0, st>>>(g, p.Nu, p.ntile, u0, G, Hinv, dev);
  WLG_LAUNCH_CHECK("gauge_chain");
}

template <class T>
void gauge_first(const Geo& g, const GramPlan& p, int msl, const typename V2<T>::t* levels,
                 const double* G, const double* Hinv, T* uh, T* blines, T* alines,
                 cudaStream_t st) {
  const long long n = (long long)3 * p.Nu * p.ntile * 32;
  long long grid = (n + 127) / 128;
  if (grid > num_sms() * 16) grid = num_sms() * 16;
  k_gauge_first<T, T><<<(int)grid, 128, 0, st>>>(g, p.Nu, p.ntile, msl, levels,
                                                 link_elems<T>(g.vol), G, Hinv, uh, blines,
                                                 alines, p.A, p.Aa);
  WLG_LAUNCH_CHECK("gauge_first");
}

template <class T>
void gram_line_step(const Geo& g, const GramPlan& p, int msl, int R, const T* uh,
                    const double* Hinv, T* blines, T* alines, cudaStream_t st) {
  const long long n = (long long)msl * 3 * p.Nu * p.ntile * 32;
  long long grid = (n + 127) / 128;
  if (grid > num_sms() * 16) grid = num_sms() * 16;
  k_gauge_line_step<T><<<(int)grid, 128, 0, st>>>(g, p.Nu, p.ntile, msl, R, uh, Hinv, blines,
                                                  alines, p.A, p.Aa);
  WLG_LAUNCH_CHECK("gauge_line_step");
}

template <class T>
void gram_contract(const Geo& g, const GramPlan& p, int mwlt, const T* alines, const T* blines,
                   T* partial, cudaStream_t st) {
  GramArgs a;
  a.alines = alines;
  a.blines = blines;
  a.partial = partial;
  a.A = p.A;
  a.Aa = p.Aa;
  a.Nu = p.Nu;
  a.ntile = p.ntile;
  a.N0 = g.n[0];
  a.mwlt = mwlt;
  a.BX = p.BX;
  a.BXp = p.BXp;
  a.NG = p.NG;
  a.NYB = p.NYB;
  a.NYBp = p.NYBp;
  a.nblk = p.nblk;
  a.nchunks = p.nchunks;
  a.cpc = p.cpc;
  a.stages = p.stages;
  a.nrows = p.nrows;
  void* fn = gram_kernel((int)sizeof(T), p.L, p.TQ, p.occ, p.ord);
  if (!fn) {
    set_error("kernel gram: none for %d levels and %d extents per thread", p.L, p.TQ);
    return;
  }
  void* args[] = {&a};
  cudaLaunchKernel(fn, dim3(p.nblk * p.nsplit), dim3(p.block), args, p.smem, st);
  WLG_LAUNCH_CHECK("gram");
}

int gram_prepare(const GramPlan& p) {
  void* fn = gram_kernel(p.esize, p.L, p.TQ, p.occ, p.ord);
  if (!fn) {
    set_error("gram: no kernel for %d levels and %d extents per thread", p.L, p.TQ);
    return -1;
  }
  // the limit is per kernel, not per plan: the largest any plan may use, so
  // that plans of other lattices keep launching; set once per kernel and device
  static std::mutex mu;
  static std::set<std::pair<int, void*>> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  if (done.count({dev, fn})) return 0;
  if (cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024) !=
      cudaSuccess) {
    set_error("gram: %zu bytes of shared memory per block: %s", p.smem,
              cudaGetErrorString(cudaGetLastError()));
    return -1;
  }
  done.insert({dev, fn});
  return 0;
}

template <class T>
void gram_reduce(const Geo& g, const GramPlan& p, int bc, int mwlt, int mwlr, int r,
                 const T* partial, double* wl, cudaStream_t st) {
  const int nout = g.n[0] * mwlt * p.L * p.L;
  const double norm = 9.0 * g.n[1] * g.n[2] * g.n[3];  // wloop.c:535
  const int grid = (nout + 255) / 256;
  k_gram_reduce<T><<<grid, 256, 0, st>>>(partial, p.nsplit, g.n[0], mwlt, p.L, mwlr, r,
                                          bc == 0 ? 1 : 0, norm, wl);
  WLG_LAUNCH_CHECK("gram_reduce");
}

#define WLG_GRAM_INST(T)                                                                       \
  template void gauge_chain<T>(const Geo&, const GramPlan&, const V2<T>::t*, double*, double*, \
                               unsigned long long*, cudaStream_t);                             \
  template void gauge_first<T>(const Geo&, const GramPlan&, int, const V2<T>::t*,              \
                               const double*, const double*, T*, T*, T*, cudaStream_t);        \
  template void gram_line_step<T>(const Geo&, const GramPlan&, int, int, const T*,             \
                                  const double*, T*, T*, cudaStream_t);                        \
  template void gram_contract<T>(const Geo&, const GramPlan&, int, const T*, const T*, T*,     \
                                 cudaStream_t);                                                \
  template void gram_reduce<T>(const Geo&, const GramPlan&, int, int, int, int, const T*,      \
                               double*, cudaStream_t);
WLG_GRAM_INST(float)
WLG_GRAM_INST(double)
#undef WLG_GRAM_INST

}  // namespace wlg
