// common.cuh -- device types shared by every wloop_b200 kernel.
//
// Link fields live in HBM in a tiled structure-of-arrays layout: each
// direction of a field is an array of 32-site tiles (lexicographic site
// s = x3 + N3*(x2 + N2*(x1 + N1*x0)), the argument order of openQCD's
// ipt[]); a tile holds the 9 complex entries (row-major c11..c33) of its 32
// links component-major, so a warp reading one component of 32 consecutive
// sites issues one fully coalesced request and the 9 components of a link
// sit at compile-time offsets from one base address.
//   FP64: component c of site s at double2 index  (s/32)*288 + c*32 + s%32
//   FP32: entries paired into float4 (c = 2p, 2p+1; p = 0..4, the 10th slot
//         is padding) at float4 index  (s/32)*160 + p*32 + s%32
// so FP64 links load as 9 and FP32 links as 5 128-bit transactions.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#define WLG_MAX_LEVELS 8

namespace wlg {

template <class T> struct V2;
template <> struct V2<double> { typedef double2 t; };
template <> struct V2<float> { typedef float2 t; };

// A 3x3 complex matrix held in registers, row-major.
template <class T> struct M3 {
  typename V2<T>::t e[9];
};

// ---------------------------------------------------------------------------
// Geometry
// ---------------------------------------------------------------------------
struct Geo {
  int n[4];    // N0 (time), N1, N2, N3
  int st[4];   // strides: st[0]=N1*N2*N3, st[1]=N2*N3, st[2]=N3, st[3]=1
  int vol;     // N0*N1*N2*N3
  int vs;      // N1*N2*N3 (one time slice)
};

static inline Geo make_geo(const int n[4]) {
  Geo g;
  for (int i = 0; i < 4; i++) g.n[i] = n[i];
  g.st[3] = 1;
  g.st[2] = n[3];
  g.st[1] = n[2] * n[3];
  g.st[0] = n[1] * n[2] * n[3];
  g.vs = g.st[0];
  g.vol = n[0] * g.st[0];
  return g;
}

__device__ __forceinline__ void coords(const Geo& g, int s, int x[4]) {
  x[0] = s / g.st[0];
  int r = s - x[0] * g.st[0];
  x[1] = r / g.st[1];
  r -= x[1] * g.st[1];
  x[2] = r / g.st[2];
  x[3] = r - x[2] * g.st[2];
}

// neighbour of site s (coordinate xm along mu) shifted by +1 / -1, periodic
__device__ __forceinline__ int up(const Geo& g, int s, int xm, int mu) {
  return (xm == g.n[mu] - 1) ? s - (g.n[mu] - 1) * g.st[mu] : s + g.st[mu];
}
__device__ __forceinline__ int dn(const Geo& g, int s, int xm, int mu) {
  return (xm == 0) ? s + (g.n[mu] - 1) * g.st[mu] : s - g.st[mu];
}
// shift by +d (0 <= d < N_mu), periodic
__device__ __forceinline__ int shift(const Geo& g, int s, int xm, int mu, int d) {
  int y = xm + d;
  if (y >= g.n[mu]) y -= g.n[mu];
  return s + (y - xm) * g.st[mu];
}

// ---------------------------------------------------------------------------
// Field views: one base pointer per direction (any may be null when a kernel
// never touches that direction).  Component c of link (s,mu) is at
// p[mu][c*vol + s].
// ---------------------------------------------------------------------------
template <class T> struct Links {
  typename V2<T>::t* p[4];
};

// largest c in [0,n) with pre[c] <= w: the lattice that owns flattened work
// item w of a batched launch (pre is the prefix of per-lattice work)
__device__ __forceinline__ int find_item(const long long* __restrict__ pre, int n, long long w) {
  int lo = 0, hi = n - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (__ldg(pre + mid) <= w)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// Arguments of one smearing launch on one lattice (see the item functions of
// smear.cu); the batched kernels take an array of these.
template <class T> struct SArgs {
  Geo g;
  Links<T> U;               // links read (staples / linear combination)
  Links<T> D;               // links written (APE destination, spatial-HYP level 2)
  typename V2<T>::t* aux0;  // HYP first-level / spatial-HYP level-1 scratch
  typename V2<T>::t* aux1;  // HYP second-level scratch
  double a, b;              // linear combination a U + b S (APE: a = alpha)
  int proj, iter, mu0, nmu, bc;
};

// Arguments of one spatial-line step (loops.cu): dst = src(x) level(x+(R-1)k)
template <class T> struct LArgs {
  Geo g;
  int msl, R;
  const typename V2<T>::t* level;
  const typename V2<T>::t* src;
  typename V2<T>::t* dst;
};

// Arguments of one contraction launch on one lattice (loops.cu)
template <class T> struct CArgs {
  Geo g;
  const typename V2<T>::t* u0;     // temporal links
  const typename V2<T>::t* lines;  // [msl][3] spatial lines of length R
  int msl, mwlt, R, ngrp, nCB;
  double* partial;
  // optional, fourth form only: next[sl][k](x) = lines[sl][k](x) * level[sl][k](x + R k),
  // the lines of length R+1 (null: not computed)
  const typename V2<T>::t* level;
  typename V2<T>::t* next;
};

// Arguments of one partial-sum reduction (loops.cu): wl for spatial extent r
struct RArgs {
  int msl, mwlt, mwlr, r, G, ngrp, nCB, nout;
  double norm;
  const double* partial;
  double* wl;
};

// elements (of V2<T>::t) per 32-site tile and per direction array
template <class T> struct Tile;
template <> struct Tile<double> { enum { TS = 288 }; };  // 9 x 32 double2
template <> struct Tile<float> { enum { TS = 320 }; };   // 5 x 32 float4 = 320 float2
template <class T> __host__ __device__ __forceinline__ size_t link_elems(int vol) {
  return (size_t)((vol + 31) >> 5) * Tile<T>::TS;
}

template <class T>
__device__ __forceinline__ void ld(M3<T>& m, const typename V2<T>::t* __restrict__ base, int vol,
                                   int s);
template <class T>
__device__ __forceinline__ void st(typename V2<T>::t* __restrict__ base, int vol, int s,
                                   const M3<T>& m);

template <>
__device__ __forceinline__ void ld<double>(M3<double>& m, const double2* __restrict__ base, int,
                                           int s) {
  const double2* p = base + (size_t)(s >> 5) * 288 + (s & 31);
#pragma unroll
  for (int c = 0; c < 9; c++) m.e[c] = __ldg(p + c * 32);
}
template <>
__device__ __forceinline__ void st<double>(double2* __restrict__ base, int, int s,
                                           const M3<double>& m) {
  double2* p = base + (size_t)(s >> 5) * 288 + (s & 31);
#pragma unroll
  for (int c = 0; c < 9; c++) p[c * 32] = m.e[c];
}
template <>
__device__ __forceinline__ void ld<float>(M3<float>& m, const float2* __restrict__ base, int,
                                          int s) {
  const float4* p = reinterpret_cast<const float4*>(base) + (size_t)(s >> 5) * 160 + (s & 31);
#pragma unroll
  for (int q = 0; q < 5; q++) {
    float4 v = __ldg(p + q * 32);
    m.e[2 * q] = make_float2(v.x, v.y);
    if (q < 4) m.e[2 * q + 1] = make_float2(v.z, v.w);
  }
}
template <>
__device__ __forceinline__ void st<float>(float2* __restrict__ base, int, int s,
                                          const M3<float>& m) {
  float4* p = reinterpret_cast<float4*>(base) + (size_t)(s >> 5) * 160 + (s & 31);
#pragma unroll
  for (int q = 0; q < 5; q++) {
    float4 v;
    v.x = m.e[2 * q].x;
    v.y = m.e[2 * q].y;
    v.z = (q < 4) ? m.e[2 * q + 1].x : 0.f;
    v.w = (q < 4) ? m.e[2 * q + 1].y : 0.f;
    p[q * 32] = v;
  }
}

// ---------------------------------------------------------------------------
// SU(3) algebra (definitions of openQCD's su3xsu3, su3dagxsu3, su3xsu3dag).
// ---------------------------------------------------------------------------
template <class T> __device__ __forceinline__ void zero(M3<T>& a) {
#pragma unroll
  for (int c = 0; c < 9; c++) {
    a.e[c].x = T(0);
    a.e[c].y = T(0);
  }
}

// c = a*b
template <class T> __device__ __forceinline__ void mul(M3<T>& c, const M3<T>& a, const M3<T>& b) {
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      T re = a.e[3 * i].x * b.e[j].x - a.e[3 * i].y * b.e[j].y;
      T im = a.e[3 * i].x * b.e[j].y + a.e[3 * i].y * b.e[j].x;
#pragma unroll
      for (int k = 1; k < 3; k++) {
        re = fma(a.e[3 * i + k].x, b.e[3 * k + j].x, re);
        re = fma(-a.e[3 * i + k].y, b.e[3 * k + j].y, re);
        im = fma(a.e[3 * i + k].x, b.e[3 * k + j].y, im);
        im = fma(a.e[3 * i + k].y, b.e[3 * k + j].x, im);
      }
      c.e[3 * i + j].x = re;
      c.e[3 * i + j].y = im;
    }
}

// c = a^dag * b
template <class T> __device__ __forceinline__ void mul_da(M3<T>& c, const M3<T>& a, const M3<T>& b) {
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      T re = a.e[i].x * b.e[j].x + a.e[i].y * b.e[j].y;
      T im = a.e[i].x * b.e[j].y - a.e[i].y * b.e[j].x;
#pragma unroll
      for (int k = 1; k < 3; k++) {
        re = fma(a.e[3 * k + i].x, b.e[3 * k + j].x, re);
        re = fma(a.e[3 * k + i].y, b.e[3 * k + j].y, re);
        im = fma(a.e[3 * k + i].x, b.e[3 * k + j].y, im);
        im = fma(-a.e[3 * k + i].y, b.e[3 * k + j].x, im);
      }
      c.e[3 * i + j].x = re;
      c.e[3 * i + j].y = im;
    }
}

// c = a * b^dag
template <class T> __device__ __forceinline__ void mul_ad(M3<T>& c, const M3<T>& a, const M3<T>& b) {
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      T re = a.e[3 * i].x * b.e[3 * j].x + a.e[3 * i].y * b.e[3 * j].y;
      T im = a.e[3 * i].y * b.e[3 * j].x - a.e[3 * i].x * b.e[3 * j].y;
#pragma unroll
      for (int k = 1; k < 3; k++) {
        re = fma(a.e[3 * i + k].x, b.e[3 * j + k].x, re);
        re = fma(a.e[3 * i + k].y, b.e[3 * j + k].y, re);
        im = fma(a.e[3 * i + k].y, b.e[3 * j + k].x, im);
        im = fma(-a.e[3 * i + k].x, b.e[3 * j + k].y, im);
      }
      c.e[3 * i + j].x = re;
      c.e[3 * i + j].y = im;
    }
}

// FP32 single products as packed two-lane FMAs (fma.rn.f32x2): a complex
// multiply-add c += p q runs as {c.re, c.im} += P1 * {p.re, p.re} + P2 *
// {p.im, p.im}, with p's entries broadcast into pairs once per product and
// the pairs P1, P2 of the other factor formed once per entry (q itself and
// q turned by a quarter, conjugated as the product needs).  The products of
// the scalar forms above in the same k order.
__device__ __forceinline__ float2 f2bc(float v) { return make_float2(v, v); }

// c = a*b: a_ik b_kj = {b.re, b.im} a.re + {-b.im, b.re} a.im
template <> __device__ __forceinline__ void mul<float>(M3<float>& c, const M3<float>& a,
                                                       const M3<float>& b) {
  float2 rb[9];
#pragma unroll
  for (int k = 0; k < 9; k++) rb[k] = make_float2(-b.e[k].y, b.e[k].x);
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const float2 ar0 = f2bc(a.e[3 * i].x), ai0 = f2bc(a.e[3 * i].y);
    const float2 ar1 = f2bc(a.e[3 * i + 1].x), ai1 = f2bc(a.e[3 * i + 1].y);
    const float2 ar2 = f2bc(a.e[3 * i + 2].x), ai2 = f2bc(a.e[3 * i + 2].y);
#pragma unroll
    for (int j = 0; j < 3; j++) {
      float2 o = __fmul2_rn(b.e[j], ar0);
      o = __ffma2_rn(rb[j], ai0, o);
      o = __ffma2_rn(b.e[3 + j], ar1, o);
      o = __ffma2_rn(rb[3 + j], ai1, o);
      o = __ffma2_rn(b.e[6 + j], ar2, o);
      o = __ffma2_rn(rb[6 + j], ai2, o);
      c.e[3 * i + j] = o;
    }
  }
}

// c = a^dag*b: conj(a_ki) b_kj = {b.re, b.im} a.re + {b.im, -b.re} a.im
template <> __device__ __forceinline__ void mul_da<float>(M3<float>& c, const M3<float>& a,
                                                          const M3<float>& b) {
  float2 rb[9];
#pragma unroll
  for (int k = 0; k < 9; k++) rb[k] = make_float2(b.e[k].y, -b.e[k].x);
#pragma unroll
  for (int i = 0; i < 3; i++) {
    const float2 ar0 = f2bc(a.e[i].x), ai0 = f2bc(a.e[i].y);
    const float2 ar1 = f2bc(a.e[3 + i].x), ai1 = f2bc(a.e[3 + i].y);
    const float2 ar2 = f2bc(a.e[6 + i].x), ai2 = f2bc(a.e[6 + i].y);
#pragma unroll
    for (int j = 0; j < 3; j++) {
      float2 o = __fmul2_rn(b.e[j], ar0);
      o = __ffma2_rn(rb[j], ai0, o);
      o = __ffma2_rn(b.e[3 + j], ar1, o);
      o = __ffma2_rn(rb[3 + j], ai1, o);
      o = __ffma2_rn(b.e[6 + j], ar2, o);
      o = __ffma2_rn(rb[6 + j], ai2, o);
      c.e[3 * i + j] = o;
    }
  }
}

// c = a*b^dag: a_ik conj(b_jk) = {a.re, a.im} b.re + {a.im, -a.re} b.im
template <> __device__ __forceinline__ void mul_ad<float>(M3<float>& c, const M3<float>& a,
                                                          const M3<float>& b) {
  float2 ra[9];
#pragma unroll
  for (int k = 0; k < 9; k++) ra[k] = make_float2(a.e[k].y, -a.e[k].x);
#pragma unroll
  for (int j = 0; j < 3; j++) {
    const float2 br0 = f2bc(b.e[3 * j].x), bi0 = f2bc(b.e[3 * j].y);
    const float2 br1 = f2bc(b.e[3 * j + 1].x), bi1 = f2bc(b.e[3 * j + 1].y);
    const float2 br2 = f2bc(b.e[3 * j + 2].x), bi2 = f2bc(b.e[3 * j + 2].y);
#pragma unroll
    for (int i = 0; i < 3; i++) {
      float2 o = __fmul2_rn(a.e[3 * i], br0);
      o = __ffma2_rn(ra[3 * i], bi0, o);
      o = __ffma2_rn(a.e[3 * i + 1], br1, o);
      o = __ffma2_rn(ra[3 * i + 1], bi1, o);
      o = __ffma2_rn(a.e[3 * i + 2], br2, o);
      o = __ffma2_rn(ra[3 * i + 2], bi2, o);
      c.e[3 * i + j] = o;
    }
  }
}

// In-place products with 6 temporaries: c <- a^dag c (column by column) and
// c <- c b (row by row).  Same arithmetic as mul_da / mul.
template <class T> __device__ __forceinline__ void lmul_dag_inplace(M3<T>& c, const M3<T>& a) {
#pragma unroll
  for (int j = 0; j < 3; j++) {
    typename V2<T>::t x0 = c.e[j], x1 = c.e[3 + j], x2 = c.e[6 + j];
#pragma unroll
    for (int i = 0; i < 3; i++) {
      T re = a.e[i].x * x0.x + a.e[i].y * x0.y;
      T im = a.e[i].x * x0.y - a.e[i].y * x0.x;
      re = fma(a.e[3 + i].x, x1.x, re);
      re = fma(a.e[3 + i].y, x1.y, re);
      im = fma(a.e[3 + i].x, x1.y, im);
      im = fma(-a.e[3 + i].y, x1.x, im);
      re = fma(a.e[6 + i].x, x2.x, re);
      re = fma(a.e[6 + i].y, x2.y, re);
      im = fma(a.e[6 + i].x, x2.y, im);
      im = fma(-a.e[6 + i].y, x2.x, im);
      c.e[3 * i + j].x = re;
      c.e[3 * i + j].y = im;
    }
  }
}

template <class T> __device__ __forceinline__ void rmul_inplace(M3<T>& c, const M3<T>& b) {
#pragma unroll
  for (int i = 0; i < 3; i++) {
    typename V2<T>::t x0 = c.e[3 * i], x1 = c.e[3 * i + 1], x2 = c.e[3 * i + 2];
#pragma unroll
    for (int j = 0; j < 3; j++) {
      T re = x0.x * b.e[j].x - x0.y * b.e[j].y;
      T im = x0.x * b.e[j].y + x0.y * b.e[j].x;
      re = fma(x1.x, b.e[3 + j].x, re);
      re = fma(-x1.y, b.e[3 + j].y, re);
      im = fma(x1.x, b.e[3 + j].y, im);
      im = fma(x1.y, b.e[3 + j].x, im);
      re = fma(x2.x, b.e[6 + j].x, re);
      re = fma(-x2.y, b.e[6 + j].y, re);
      im = fma(x2.x, b.e[6 + j].y, im);
      im = fma(x2.y, b.e[6 + j].x, im);
      c.e[3 * i + j].x = re;
      c.e[3 * i + j].y = im;
    }
  }
}

template <class T> __device__ __forceinline__ void acc(M3<T>& c, const M3<T>& a) {
#pragma unroll
  for (int k = 0; k < 9; k++) {
    c.e[k].x += a.e[k].x;
    c.e[k].y += a.e[k].y;
  }
}

// Re tr(a^dag b) = sum_ij Re(conj(a_ij) b_ij)  (openQCD _vector_prod_re over rows),
// accumulated as two independent partial sums (real and imaginary parts).
template <class T> __device__ __forceinline__ T retr_dag(const M3<T>& a, const M3<T>& b) {
  T s = a.e[0].x * b.e[0].x;
  T t = a.e[0].y * b.e[0].y;
#pragma unroll
  for (int k = 1; k < 9; k++) {
    s = fma(a.e[k].x, b.e[k].x, s);
    t = fma(a.e[k].y, b.e[k].y, t);
  }
  return s + t;
}

// FP32: the real and the imaginary chain advance together as one packed
// two-lane FMA (fma.rn.f32x2 of sm_100a, each lane rounded as fmaf); the same
// products in the same order as the generic form, so the same result.
template <> __device__ __forceinline__ float retr_dag<float>(const M3<float>& a, const M3<float>& b) {
  float2 p = __fmul2_rn(a.e[0], b.e[0]);
#pragma unroll
  for (int k = 1; k < 9; k++) p = __ffma2_rn(a.e[k], b.e[k], p);
  return p.x + p.y;
}

// ---------------------------------------------------------------------------
// FP32 in-place products of G matrices by one shared matrix, as packed
// two-lane FMAs: a complex multiply-add c += p q is
//   {c.re, c.im} += {q.re, q.im} * {p.re, p.re} + {-q.im, q.re} * {p.im, p.im}
// with the shared factor p in broadcast pairs (formed once per call, used by
// all G matrices and all three rows or columns) and the per-matrix factor q
// rotated once per entry.  The products of the scalar forms above, summed in
// the same k order; within one k the two products of an imaginary part may be
// added in the other order (FP32 rounding differences only).
// ---------------------------------------------------------------------------
// SW (the tenth form's variant): the sign of the second term moves from the
// per-matrix turned pair into the shared broadcast pair, {c.im, c.re} *
// {a.im, -a.im} instead of {c.im, -c.re} * {a.im, a.im}: the same products
// (a sign is exact), so the same result, with 9 sign flips per product
// instead of 9 per matrix and product.
// c[g] <- a^dag c[g]   (conj(a_ki) c_kj = {c.re, c.im} a.re + {c.im, -c.re} a.im)
template <int G, bool SW = false>
__device__ __forceinline__ void lmul_dag_inplace_x2(M3<float> (&c)[G], const M3<float>& a) {
  float2 ar[9], ai[9];
#pragma unroll
  for (int k = 0; k < 9; k++) {
    ar[k] = make_float2(a.e[k].x, a.e[k].x);
    ai[k] = SW ? make_float2(a.e[k].y, -a.e[k].y) : make_float2(a.e[k].y, a.e[k].y);
  }
#pragma unroll
  for (int g = 0; g < G; g++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      const float2 x0 = c[g].e[j], x1 = c[g].e[3 + j], x2 = c[g].e[6 + j];
      const float2 r0 = SW ? make_float2(x0.y, x0.x) : make_float2(x0.y, -x0.x),
                   r1 = SW ? make_float2(x1.y, x1.x) : make_float2(x1.y, -x1.x),
                   r2 = SW ? make_float2(x2.y, x2.x) : make_float2(x2.y, -x2.x);
#pragma unroll
      for (int i = 0; i < 3; i++) {
        float2 o = __fmul2_rn(x0, ar[i]);
        o = __ffma2_rn(r0, ai[i], o);
        o = __ffma2_rn(x1, ar[3 + i], o);
        o = __ffma2_rn(r1, ai[3 + i], o);
        o = __ffma2_rn(x2, ar[6 + i], o);
        o = __ffma2_rn(r2, ai[6 + i], o);
        c[g].e[3 * i + j] = o;
      }
    }
}

// c[g] <- c[g] b   (c_ik b_kj = {c.re, c.im} b.re + {-c.im, c.re} b.im;
// SW: {c.im, c.re} * {-b.im, b.im})
template <int G, bool SW = false>
__device__ __forceinline__ void rmul_inplace_x2(M3<float> (&c)[G], const M3<float>& b) {
  float2 br[9], bi[9];
#pragma unroll
  for (int k = 0; k < 9; k++) {
    br[k] = make_float2(b.e[k].x, b.e[k].x);
    bi[k] = SW ? make_float2(-b.e[k].y, b.e[k].y) : make_float2(b.e[k].y, b.e[k].y);
  }
#pragma unroll
  for (int g = 0; g < G; g++)
#pragma unroll
    for (int i = 0; i < 3; i++) {
      const float2 x0 = c[g].e[3 * i], x1 = c[g].e[3 * i + 1], x2 = c[g].e[3 * i + 2];
      const float2 r0 = SW ? make_float2(x0.y, x0.x) : make_float2(-x0.y, x0.x),
                   r1 = SW ? make_float2(x1.y, x1.x) : make_float2(-x1.y, x1.x),
                   r2 = SW ? make_float2(x2.y, x2.x) : make_float2(-x2.y, x2.x);
#pragma unroll
      for (int j = 0; j < 3; j++) {
        float2 o = __fmul2_rn(x0, br[j]);
        o = __ffma2_rn(r0, bi[j], o);
        o = __ffma2_rn(x1, br[3 + j], o);
        o = __ffma2_rn(r1, bi[3 + j], o);
        o = __ffma2_rn(x2, br[6 + j], o);
        o = __ffma2_rn(r2, bi[6 + j], o);
        c[g].e[3 * i + j] = o;
      }
    }
}

template <class D, class S> __device__ __forceinline__ void cvt(M3<D>& d, const M3<S>& s) {
#pragma unroll
  for (int k = 0; k < 9; k++) {
    d.e[k].x = (D)s.e[k].x;
    d.e[k].y = (D)s.e[k].y;
  }
}

// ---------------------------------------------------------------------------
// Approximate SU(3) projection of hep-lat/0506008 as implemented by
// approx_project_to_su3_dble (modules/smear/projection.c:120-154).  Always FP64.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double det_im(const M3<double>& u) {
  const double2* c = u.e;
  double d1re = (c[4].x * c[8].x - c[4].y * c[8].y) - (c[5].x * c[7].x - c[5].y * c[7].y);
  double d1im = (c[4].x * c[8].y + c[4].y * c[8].x) - (c[5].x * c[7].y + c[5].y * c[7].x);
  double d2re = (c[3].x * c[8].x - c[3].y * c[8].y) - (c[5].x * c[6].x - c[5].y * c[6].y);
  double d2im = (c[3].x * c[8].y + c[3].y * c[8].x) - (c[5].x * c[6].y + c[5].y * c[6].x);
  double d3re = (c[3].x * c[7].x - c[3].y * c[7].y) - (c[4].x * c[6].x - c[4].y * c[6].y);
  double d3im = (c[3].x * c[7].y + c[3].y * c[7].x) - (c[4].x * c[6].y + c[4].y * c[6].x);
  return (c[0].x * d1im + c[0].y * d1re) - (c[1].x * d2im + c[1].y * d2re) +
         (c[2].x * d3im + c[2].y * d3re);
}

// c = a*b for a right factor b whose diagonal is real (b.e[0], b.e[4], b.e[8]
// have zero imaginary parts, as in the projection's X): mul() without the
// products of those zeros.  Dropping them leaves every sum unchanged (adding
// a product with an exact zero changes at most the sign of a zero result).
__device__ __forceinline__ void mul_rdiag(M3<double>& c, const M3<double>& a, const M3<double>& b) {
#pragma unroll
  for (int i = 0; i < 3; i++)
#pragma unroll
    for (int j = 0; j < 3; j++) {
      double re, im;
      if (j == 0) {
        re = a.e[3 * i].x * b.e[0].x;
        im = a.e[3 * i].y * b.e[0].x;
      } else {
        re = a.e[3 * i].x * b.e[j].x - a.e[3 * i].y * b.e[j].y;
        im = a.e[3 * i].x * b.e[j].y + a.e[3 * i].y * b.e[j].x;
      }
#pragma unroll
      for (int k = 1; k < 3; k++) {
        re = fma(a.e[3 * i + k].x, b.e[3 * k + j].x, re);
        if (k != j) re = fma(-a.e[3 * i + k].y, b.e[3 * k + j].y, re);
        if (k != j) im = fma(a.e[3 * i + k].x, b.e[3 * k + j].y, im);
        im = fma(a.e[3 * i + k].y, b.e[3 * k + j].x, im);
      }
      c.e[3 * i + j].x = re;
      c.e[3 * i + j].y = im;
    }
}

#define WLG_SRT18_EPS (4.242640687119285 * 2.220446049250313080847e-16)

__device__ __forceinline__ void project(M3<double>& u, int iter) {
  double d = 0.0;
#pragma unroll
  for (int k = 0; k < 9; k++) d += u.e[k].x * u.e[k].x + u.e[k].y * u.e[k].y;
  if (d < WLG_SRT18_EPS) return;  // zero guard, projection.c:136
  d = 1.0 / sqrt(d / 3.0);
#pragma unroll
  for (int k = 0; k < 9; k++) {
    u.e[k].x *= d;
    u.e[k].y *= d;
  }
  for (int it = 0; it < iter; it++) {
    // X = 3/2 - U^dag U / 2 (projection.c:144-146).  U^dag U is Hermitian:
    // its real diagonal and upper triangle are formed, the lower triangle is
    // their conjugate (the full product gives the same numbers up to the
    // rounding of an exactly vanishing diagonal imaginary part).
    M3<double> x, y;
#pragma unroll
    for (int i = 0; i < 3; i++) {
      double dg = 0.0;
#pragma unroll
      for (int k = 0; k < 3; k++) {
        dg = fma(u.e[3 * k + i].x, u.e[3 * k + i].x, dg);
        dg = fma(u.e[3 * k + i].y, u.e[3 * k + i].y, dg);
      }
      x.e[4 * i].x = fma(-0.5, dg, 1.5);
      x.e[4 * i].y = 0.0;
#pragma unroll
      for (int j = i + 1; j < 3; j++) {
        double re = 0.0, im = 0.0;
#pragma unroll
        for (int k = 0; k < 3; k++) {
          re = fma(u.e[3 * k + i].x, u.e[3 * k + j].x, re);
          re = fma(u.e[3 * k + i].y, u.e[3 * k + j].y, re);
          im = fma(u.e[3 * k + i].x, u.e[3 * k + j].y, im);
          im = fma(-u.e[3 * k + i].y, u.e[3 * k + j].x, im);
        }
        x.e[3 * i + j].x = -0.5 * re;
        x.e[3 * i + j].y = -0.5 * im;
        x.e[3 * j + i].x = -0.5 * re;
        x.e[3 * j + i].y = 0.5 * im;
      }
    }
    mul_rdiag(y, u, x);
    // z = 1 - i Im det(Y) / 3 (projection.c:150-152)
    double zim = det_im(y) * (-1.0 / 3.0);
#pragma unroll
    for (int k = 0; k < 9; k++) {
      u.e[k].x = y.e[k].x - zim * y.e[k].y;
      u.e[k].y = y.e[k].y + zim * y.e[k].x;
    }
  }
}

// ---------------------------------------------------------------------------
// Up and down staples of link (x,mu) in the (mu,nu) plane, general 3x3 form
// (add_up_staple_save / add_dn_staple_save, modules/lnk/lnkstaple.c:318-382):
//   up = u1(x,nu) u2(x+nu,mu) u1(x+mu,nu)^dag
//   dn = u1(x-nu,nu)^dag u2(x-nu,mu) u1(x-nu+mu,nu)
// nu-links come from a, mu-links from b; the sum is added to v.
// ---------------------------------------------------------------------------
template <class T>
__device__ __forceinline__ void add_staples(M3<T>& v, const Geo& g, const int x[4], int s,
                                            const typename V2<T>::t* __restrict__ a_nu,
                                            const typename V2<T>::t* __restrict__ b_mu, int mu,
                                            int nu) {
  const int vol = g.vol;
  M3<T> p, q, r;
  int s_pn = up(g, s, x[nu], nu);
  int s_pm = up(g, s, x[mu], mu);
  ld(p, b_mu, vol, s_pn);
  ld(q, a_nu, vol, s_pm);
  mul_ad(r, p, q);
  ld(p, a_nu, vol, s);
  mul(q, p, r);
  acc(v, q);
  int s_mn = dn(g, s, x[nu], nu);
  int xm = x[mu];  // x-nu has the same mu coordinate
  int s_mn_pm = up(g, s_mn, xm, mu);
  ld(p, b_mu, vol, s_mn);
  ld(q, a_nu, vol, s_mn_pm);
  mul(r, p, q);
  ld(p, a_nu, vol, s_mn);
  mul_da(q, p, r);
  acc(v, q);
}

}  // namespace wlg
