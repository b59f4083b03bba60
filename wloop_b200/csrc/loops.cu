// loops.cu -- Wilson-loop stage: spatial lines, the fused temporal-line /
// contraction kernel and its deterministic reduction.
//
// The reference (wloop.c:436-508) rebuilds the temporal lines L_T for every
// T and, for every level pair (sl1,sl2), multiplies two full products per
// site: msl^2 (2M+36) flops per site and direction.  Here the quantity
//     W_{s1 s2}(x0,T) = sum_{xs,k} Re tr[ line_s2(x0+T)^dag  C_s1(x0,T) ]
//     C_s1(x0,T)      = U0(x0+T-1)^dag C_s1(x0,T-1) U0'(x0+T-1),  C_s1(x0,0) = line_s1(x0)
// (U0 at xs, U0' at xs+R k) is the same trace, Re tr[(ub um)^dag (ul ubR)],
// with C carried in registers along T: 2 msl M + 36 msl^2 flops.  One thread
// owns one column (xs,k) at one start slice x0 and G bottom levels; the
// msl*G traces of each T are summed over the warp (through shared memory in
// the default fourth form, by shuffles in the earlier forms) and accumulated
// in a per-warp shared-memory row, so no atomics and a fixed summation order.
// Every stage also has a batched kernel that covers many lattices in one
// launch (flattened work list, find_item).
#include "internal.h"

namespace wlg {

// lines_dst[sl][k](x) = lines_src[sl][k](x) * level[sl][k](x + (R-1) k)
// (compute_uk_long, wloop.c:207-258, multiplied from the other end so the
// update is in place).
// w in [0, msl*3*V)
template <class T> __device__ __forceinline__ void line_step_item(const LArgs<T>& A, long long w) {
  const Geo& g = A.g;
  int q = (int)(w / g.vol), s = (int)(w - (long long)q * g.vol);
  int k = q % 3;
  int x[4];
  coords(g, s, x);
  int y = shift(g, s, x[k + 1], k + 1, (A.R - 1) % g.n[k + 1]);
  M3<T> a, b, c;
  const size_t off = (size_t)q * link_elems<T>(g.vol);
  ld(a, A.src + off, g.vol, s);
  ld(b, A.level + off, g.vol, y);
  mul(c, a, b);
  st(A.dst + off, g.vol, s, c);
}

template <class T> __global__ void __launch_bounds__(128) k_line_step(LArgs<T> A) {
  const long long n = (long long)A.msl * 3 * A.g.vol;
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < n;
       w += (long long)gridDim.x * blockDim.x)
    line_step_item<T>(A, w);
}

// batched: pre[c] = first work item of lattice c
template <class T>
__global__ void __launch_bounds__(128) kb_line_step(const LArgs<T>* __restrict__ A,
                                                    const long long* __restrict__ pre, int n,
                                                    long long total) {
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < total;
       w += (long long)gridDim.x * blockDim.x) {
    const int c = find_item(pre, n, w);
    line_step_item<T>(A[c], w - pre[c]);
  }
}

template <class T>
void line_step(const Geo& g, int msl, int R, const typename V2<T>::t* level,
               const typename V2<T>::t* src, typename V2<T>::t* dst, cudaStream_t st) {
  long long n = (long long)msl * 3 * g.vol;
  long long grid = (n + 127) / 128;
  if (grid > num_sms() * 32) grid = num_sms() * 32;
  LArgs<T> A;
  A.g = g;
  A.msl = msl;
  A.R = R;
  A.level = level;
  A.src = src;
  A.dst = const_cast<typename V2<T>::t*>(dst);
  k_line_step<T><<<(int)grid, 128, 0, st>>>(A);
  WLG_LAUNCH_CHECK("line_step");
}

// ---------------------------------------------------------------------------
// warp transposing reduction: every lane holds KP values; afterwards lane l
// holds the warp sum of value index (l >> (5 - log2 KP)).
// ---------------------------------------------------------------------------
template <int KP> struct Log2;
template <> struct Log2<1> { enum { v = 0 }; };
template <> struct Log2<2> { enum { v = 1 }; };
template <> struct Log2<4> { enum { v = 2 }; };
template <> struct Log2<8> { enum { v = 3 }; };
template <> struct Log2<16> { enum { v = 4 }; };
template <> struct Log2<32> { enum { v = 5 }; };

template <int KP>
__device__ __forceinline__ double wt_reduce(double (&v)[KP], int lane) {
  constexpr int L = Log2<KP>::v;
#pragma unroll
  for (int st = 0; st < 5; st++) {
    const int off = 16 >> st;
    if (st < L) {
      const int h = KP >> (st + 1);
      const bool upper = (lane & off) != 0;
#pragma unroll
      for (int i = 0; i < h; i++) {
        double send = upper ? v[i] : v[i + h];
        double keep = upper ? v[i + h] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, off);
      }
    } else {
      v[0] += __shfl_xor_sync(0xffffffffu, v[0], off);
    }
  }
  return v[0];
}

template <int K> struct Pow2 { enum { v = (K <= 1) ? 1 : (K <= 2) ? 2 : (K <= 4) ? 4 : (K <= 8) ? 8 : (K <= 16) ? 16 : 32 }; };

// ---------------------------------------------------------------------------
// contraction kernel, second form.  One thread owns one column (xs,k) at
// one start slice x0 and G bottom levels; grid.x = N0 * ngrp * nCB with x0
// fastest (concurrent blocks share columns through L2); the block writes
// partial[((x0*ngrp + grp)*nCB + cb)][T][g][s2].  Per T-step:
//  * C updated in place (6 temporaries per product instead of a full matrix),
//  * the next T-step's temporal links loaded right after they are consumed,
//    so their latency overlaps the traces and the reduction,
//  * the top levels taken SB at a time in a rolled loop with a K=G*SB shuffle
//    reduction (small register footprint, compact code),
//  * __launch_bounds__ minimum-blocks hint so three or more blocks fit an SM.
// ---------------------------------------------------------------------------
template <class T, int G, int SB, int MINB>
__global__ void __launch_bounds__(128, MINB) k_contract2(Geo g,
                                                         const typename V2<T>::t* __restrict__ u0,
                                                         const typename V2<T>::t* __restrict__ lines,
                                                         int msl, int mwlt, int R, int ngrp,
                                                         int nCB, double* __restrict__ partial) {
  extern __shared__ double acc[];  // [nwarps][mwlt][G][msl]
  constexpr int K = G * SB;
  constexpr int KP = Pow2<K>::v;
  static_assert(K <= 32, "G*SB must not exceed 32");

  const int N0 = g.n[0], vs = g.vs, vol = g.vol;
  int b = blockIdx.x;
  const int x0 = b % N0;
  b /= N0;
  const int grp = b % ngrp;
  const int cb = b / ngrp;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int rowlen = mwlt * G * msl;
  double* wacc = acc + (size_t)warp * rowlen;
  for (int i = lane; i < rowlen; i += 32) wacc[i] = 0.0;
  __syncwarp();

  const int s1_0 = grp * G;
  const int ncol = 3 * vs;
  const int per = (ncol + nCB - 1) / nCB;
  const int c_begin = cb * per;
  const int c_end = min(ncol, c_begin + per);
  const size_t fstride = link_elems<T>(vol);
  const int idx = lane >> (5 - Log2<KP>::v);
  const bool writer = (lane & ((32 / KP) - 1)) == 0 && idx < K;
  const int wg = idx / SB, wj = idx % SB;

  for (int cbase = c_begin; cbase < c_end; cbase += blockDim.x) {
    const int col = cbase + threadIdx.x;
    const bool active = col < c_end;
    const int cc = active ? col : c_begin;
    const int k = cc / vs, xs = cc - k * vs;
    int xsR;
    {
      // xs + R k inside the time slice (selects, no local-memory array)
      const int x1 = xs / g.st[1], r = xs - x1 * g.st[1];
      const int x2 = r / g.st[2], x3 = r - x2 * g.st[2];
      const int xk = (k == 0) ? x1 : ((k == 1) ? x2 : x3);
      const int nk = g.n[k + 1];
      int y = xk + (R % nk);
      if (y >= nk) y -= nk;
      xsR = xs + (y - xk) * g.st[k + 1];
    }
    const typename V2<T>::t* lk = lines + (size_t)k * fstride;  // level s stride 3*fstride
    M3<T> C[G];
#pragma unroll
    for (int gi = 0; gi < G; gi++) {
      int s1 = min(s1_0 + gi, msl - 1);
      ld(C[gi], lk + (size_t)s1 * 3 * fstride, vol, x0 * vs + xs);
    }
    M3<T> ua, ub;
    ld(ua, u0, vol, x0 * vs + xs);
    ld(ub, u0, vol, x0 * vs + xsR);
    int t0 = x0;
    for (int tt = 1; tt <= mwlt; tt++) {
#pragma unroll
      for (int gi = 0; gi < G; gi++) lmul_dag_inplace(C[gi], ua);
#pragma unroll
      for (int gi = 0; gi < G; gi++) rmul_inplace(C[gi], ub);
      t0 = (t0 + 1 == N0) ? 0 : t0 + 1;  // x0+T mod N0: top slice, next bottom link slice
      if (tt < mwlt) {
        ld(ua, u0, vol, t0 * vs + xs);
        ld(ub, u0, vol, t0 * vs + xsR);
      }
      const int stop = t0 * vs + xs;
      double* arow = wacc + (size_t)(tt - 1) * G * msl;
#pragma unroll 1
      for (int sb = 0; sb < msl; sb += SB) {
        double v[KP];
#pragma unroll
        for (int i = 0; i < KP; i++) v[i] = 0.0;
#pragma unroll
        for (int j = 0; j < SB; j++) {
          const int s2 = sb + j;
          if (s2 < msl) {
            M3<T> l;
            ld(l, lk + (size_t)s2 * 3 * fstride, vol, stop);
#pragma unroll
            for (int gi = 0; gi < G; gi++)
              v[gi * SB + j] = active ? (double)retr_dag(l, C[gi]) : 0.0;
          }
        }
        double sum = wt_reduce<KP>(v, lane);
        if (writer && sb + wj < msl) arow[wg * msl + sb + wj] += sum;
      }
    }
  }
  __syncthreads();
  double* out = partial + ((size_t)(x0 * ngrp + grp) * nCB + cb) * rowlen;
  for (int i = threadIdx.x; i < rowlen; i += blockDim.x) {
    double s = 0.0;
    for (int w = 0; w < nwarps; w++) s += acc[(size_t)w * rowlen + i];
    out[i] = s;
  }
}

ContractPlan contract_plan(const Geo& g, int msl, int mwlt, bool fp64, int G_hint, int nCB_hint,
                           int block_hint) {
  ContractPlan p;
  int G = G_hint;
  if (G <= 0) {
    // two level groups for msl >= 4 (C of G levels stays in registers), one below
    G = (msl <= 3) ? msl : (msl + 1) / 2;
    if (fp64 && G > 3) G = 3;
  }
  if (G > msl) G = msl;
  if (G < 1) G = 1;
  if (G == 5) G = 6;
  p.G = G;
  p.SB = (msl >= 2 && G <= 4 && !(fp64 && G >= 3)) ? 2 : 1;
  // fourth form (staged top lines, shared-memory reduction) unless G = 6,
  // which only the second form has: in FP32 with its level loops unrolled,
  // packed two-lane FMA products and the next level's line read ahead (form
  // 8; 4.6 % faster than form 5 at 32^3x64) with the products' signs in the
  // shared broadcast pairs (form 10; the same result, 1.9 % faster than form
  // 8), in FP64 with the top lines staged by
  // bulk copies (form 7; 5 % faster there, 2 % slower in FP32; the unrolled
  // FP64 kernel spills registers)
  p.variant = (G <= 4) ? (fp64 ? 7 : 10) : 2;
  p.ngrp = (msl + G - 1) / G;
  // FP64 stages twice the bytes per thread: 64-thread blocks keep 3 blocks per SM
  p.block = block_hint > 0 ? block_hint : ((fp64 && p.variant >= 4) ? 64 : 128);
  int ncol = 3 * g.vs;
  int nCB = nCB_hint;
  if (nCB <= 0) {
    // At least 8 blocks per SM, and at most 4 column passes per block: the
    // blocks of neighbouring x0 read the same lines one step apart, and they
    // only share them through L2 while they stay in step.  Long column loops
    // let them drift apart (at 32^3x64 with 77 passes per block the launch
    // read its lines from DRAM 5-7 times over and ran 20-25 % slower).
    long long want = (long long)num_sms() * 8;
    long long base = (long long)g.n[0] * p.ngrp;
    nCB = (int)((want + base - 1) / base);
    const int passes = 4;
    const int lockstep = (ncol + passes * p.block - 1) / (passes * p.block);
    if (nCB < lockstep) nCB = lockstep;
    int maxcb = (ncol + p.block - 1) / p.block;
    if (nCB > maxcb) nCB = maxcb;
    if (nCB < 1) nCB = 1;
  }
  p.nCB = nCB;
  // per-warp rows; rounded to 16 bytes, where the line stage starts
  p.smem = (((size_t)(p.block / 32) * mwlt * G * msl + 1) & ~(size_t)1) * sizeof(double);
  p.partial_doubles = (size_t)g.n[0] * p.ngrp * nCB * mwlt * G * msl;
  return p;
}

template <class T, int G, int SB>
static void launch_contract2(const Geo& g, const ContractPlan& p, const typename V2<T>::t* u0,
                             const typename V2<T>::t* lines, int msl, int mwlt, int R,
                             double* partial, cudaStream_t st) {
  constexpr int MINB = (sizeof(T) == 4) ? ((G <= 3) ? 3 : 2) : ((G <= 1) ? 3 : 2);
  auto kern = k_contract2<T, G, SB, MINB>;
  static size_t smem_set = 48 * 1024;
  if (p.smem > smem_set) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)p.smem);
    smem_set = p.smem;
  }
  int grid = g.n[0] * p.ngrp * p.nCB;
  kern<<<grid, p.block, p.smem, st>>>(g, u0, lines, msl, mwlt, R, p.ngrp, p.nCB, partial);
  WLG_LAUNCH_CHECK("contract");
}

template <class T, int G>
static void launch_contract2_sb(const Geo& g, const ContractPlan& p, const typename V2<T>::t* u0,
                                const typename V2<T>::t* lines, int msl, int mwlt, int R,
                                double* partial, cudaStream_t st) {
  if (p.SB == 2)
    launch_contract2<T, G, 2>(g, p, u0, lines, msl, mwlt, R, partial, st);
  else
    launch_contract2<T, G, 1>(g, p, u0, lines, msl, mwlt, R, partial, st);
}

// ---------------------------------------------------------------------------
// contraction kernel, third form: the second form plus asynchronous staging
// of the top-level lines.  At the start of every T-step each thread issues
// cp.async copies of its msl top lines (slice x0+T) into its own
// shared-memory slots, then runs the 2G matrix products of the recursion
// while the copies are in flight, and reads the lines back from shared
// memory for the traces.  Slots are laid out [level][16-byte chunk][thread]
// so the copies and the reads of a warp are bank-conflict free.
// ---------------------------------------------------------------------------
template <class T> struct Chunks;
template <> struct Chunks<double> { enum { N = 9 }; };  // 9 x double2 per link
template <> struct Chunks<float> { enum { N = 5 }; };   // 5 x float4 per link (tiled pairs)

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;\n" ::); }

// ---- bulk (TMA) copies of whole 32-site tiles into shared memory ----------
// One-dimensional cp.async.bulk from this GPU's global memory into this
// CTA's own shared memory only, completing on an mbarrier (no tensor map).
// Every wait is bounded: a wait that runs out sets g_stage_timeout,
// which the host reads after the measurement.
__device__ int g_stage_timeout;

__device__ __forceinline__ unsigned smem_addr(const void* p) {
  return (unsigned)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_addr(bar)), "r"(count)
               : "memory");
}
// before the barrier's shared memory goes back to other uses
__device__ __forceinline__ void mbar_inval(uint64_t* bar) {
  asm volatile("mbarrier.inval.shared::cta.b64 [%0];\n" ::"r"(smem_addr(bar)) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_addr(bar)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned phase) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      " selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_addr(bar)), "r"(phase)
      : "memory");
  return ok != 0;
}
__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %globaltimer;\n" : "=l"(t));
  return t;
}
// waits at most limit_ns of wall time (the global nanosecond timer bounds it,
// whatever each try_wait's own suspension); false if the phase did not complete
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned phase,
                                                  uint64_t limit_ns = 2000000000ull) {
  if (mbar_try_wait(bar, phase)) return true;
  const uint64_t t0 = global_ns();
  while (!mbar_try_wait(bar, phase))
    if (global_ns() - t0 > limit_ns) return false;
  return true;
}
// orders this thread's earlier shared-memory accesses before later
// async-proxy (bulk copy) writes to the same memory
__device__ __forceinline__ void fence_proxy_async_smem() {
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
}
// dst, src and bytes multiples of 16
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, unsigned bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::
          "r"(smem_addr(dst)),
      "l"(src), "r"(bytes), "r"(smem_addr(bar))
      : "memory");
}

// 16-byte chunk q of link s in a tiled direction array (common.cuh layout)
template <class T> __device__ __forceinline__ const char* chunk_ptr(const typename V2<T>::t* base, int s, int q);
template <> __device__ __forceinline__ const char* chunk_ptr<double>(const double2* base, int s, int q) {
  return reinterpret_cast<const char*>(base + (size_t)(s >> 5) * 288 + q * 32 + (s & 31));
}
template <> __device__ __forceinline__ const char* chunk_ptr<float>(const float2* base, int s, int q) {
  return reinterpret_cast<const char*>(reinterpret_cast<const float4*>(base) + (size_t)(s >> 5) * 160 +
                                       q * 32 + (s & 31));
}
template <class T> __device__ __forceinline__ void ld_stage(M3<T>& m, const char* slot, int stride);
template <> __device__ __forceinline__ void ld_stage<double>(M3<double>& m, const char* slot, int stride) {
#pragma unroll
  for (int q = 0; q < 9; q++) m.e[q] = *reinterpret_cast<const double2*>(slot + q * stride);
}
template <> __device__ __forceinline__ void ld_stage<float>(M3<float>& m, const char* slot, int stride) {
#pragma unroll
  for (int q = 0; q < 5; q++) {
    float4 v = *reinterpret_cast<const float4*>(slot + q * stride);
    m.e[2 * q] = make_float2(v.x, v.y);
    if (q < 4) m.e[2 * q + 1] = make_float2(v.z, v.w);
  }
}

template <class T, int G, int SB>
__device__ __forceinline__ void contract3_body(const CArgs<T>& A, int bid) {
  extern __shared__ double acc[];  // [nwarps][mwlt][G][msl] doubles, then the line stage
  constexpr int K = G * SB;
  constexpr int KP = Pow2<K>::v;
  constexpr int NQ = Chunks<T>::N;
  static_assert(K <= 32, "G*SB must not exceed 32");

  const Geo& g = A.g;
  const typename V2<T>::t* __restrict__ u0 = A.u0;
  const typename V2<T>::t* __restrict__ lines = A.lines;
  const int msl = A.msl, mwlt = A.mwlt, R = A.R, ngrp = A.ngrp, nCB = A.nCB;
  double* __restrict__ partial = A.partial;
  const int N0 = g.n[0], vs = g.vs, vol = g.vol;
  int b = bid;
  const int x0 = b % N0;
  b /= N0;
  const int grp = b % ngrp;
  const int cb = b / ngrp;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int rowlen = mwlt * G * msl;
  double* wacc = acc + (size_t)warp * rowlen;
  // line stage: [msl][NQ][blockDim] 16-byte chunks; this thread's slot of chunk (s2,q)
  // 16-byte aligned for the 16-byte copies (an even number of doubles)
  char* stage = reinterpret_cast<char*>(acc + (((size_t)nwarps * rowlen + 1) & ~(size_t)1));
  const int qstride = blockDim.x * 16;
  char* myslot = stage + threadIdx.x * 16;
  for (int i = lane; i < rowlen; i += 32) wacc[i] = 0.0;
  __syncwarp();

  const int s1_0 = grp * G;
  const int ncol = 3 * vs;
  const int per = (ncol + nCB - 1) / nCB;
  const int c_begin = cb * per;
  const int c_end = min(ncol, c_begin + per);
  const size_t fstride = link_elems<T>(vol);
  const int idx = lane >> (5 - Log2<KP>::v);
  const bool writer = (lane & ((32 / KP) - 1)) == 0 && idx < K;
  const int wg = idx / SB, wj = idx % SB;

  for (int cbase = c_begin; cbase < c_end; cbase += blockDim.x) {
    const int col = cbase + threadIdx.x;
    const bool active = col < c_end;
    const int cc = active ? col : c_begin;
    const int k = cc / vs, xs = cc - k * vs;
    int xsR;
    {
      const int x1 = xs / g.st[1], r = xs - x1 * g.st[1];
      const int x2 = r / g.st[2], x3 = r - x2 * g.st[2];
      const int xk = (k == 0) ? x1 : ((k == 1) ? x2 : x3);
      const int nk = g.n[k + 1];
      int y = xk + (R % nk);
      if (y >= nk) y -= nk;
      xsR = xs + (y - xk) * g.st[k + 1];
    }
    const typename V2<T>::t* lk = lines + (size_t)k * fstride;
    const size_t lvl = 3 * fstride;
    M3<T> C[G];
#pragma unroll
    for (int gi = 0; gi < G; gi++) {
      int s1 = min(s1_0 + gi, msl - 1);
      ld(C[gi], lk + (size_t)s1 * lvl, vol, x0 * vs + xs);
    }
    M3<T> ua, ub;
    ld(ua, u0, vol, x0 * vs + xs);
    ld(ub, u0, vol, x0 * vs + xsR);
    int t0 = x0;
    for (int tt = 1; tt <= mwlt; tt++) {
      const int t1 = (t0 + 1 == N0) ? 0 : t0 + 1;  // x0+T mod N0: the top slice
      const int stop = t1 * vs + xs;
      // stage the msl top lines of this step (own slots: no block barrier needed)
      for (int s2 = 0; s2 < msl; s2++) {
        const typename V2<T>::t* src = lk + (size_t)s2 * lvl;
#pragma unroll
        for (int q = 0; q < NQ; q++)
          cp_async16(myslot + (s2 * NQ + q) * qstride, chunk_ptr<T>(src, stop, q));
      }
      cp_async_commit();
#pragma unroll
      for (int gi = 0; gi < G; gi++) lmul_dag_inplace(C[gi], ua);
#pragma unroll
      for (int gi = 0; gi < G; gi++) rmul_inplace(C[gi], ub);
      t0 = t1;
      if (tt < mwlt) {
        ld(ua, u0, vol, t0 * vs + xs);
        ld(ub, u0, vol, t0 * vs + xsR);
      }
      cp_async_wait_all();
      double* arow = wacc + (size_t)(tt - 1) * G * msl;
#pragma unroll 1
      for (int sb = 0; sb < msl; sb += SB) {
        double v[KP];
#pragma unroll
        for (int i = 0; i < KP; i++) v[i] = 0.0;
#pragma unroll
        for (int j = 0; j < SB; j++) {
          const int s2 = sb + j;
          if (s2 < msl) {
            M3<T> l;
            ld_stage<T>(l, myslot + s2 * NQ * qstride, qstride);
#pragma unroll
            for (int gi = 0; gi < G; gi++)
              v[gi * SB + j] = active ? (double)retr_dag(l, C[gi]) : 0.0;
          }
        }
        double sum = wt_reduce<KP>(v, lane);
        if (writer && sb + wj < msl) arow[wg * msl + sb + wj] += sum;
      }
    }
  }
  __syncthreads();
  double* out = partial + ((size_t)(x0 * ngrp + grp) * nCB + cb) * rowlen;
  for (int i = threadIdx.x; i < rowlen; i += blockDim.x) {
    double s = 0.0;
    for (int w = 0; w < nwarps; w++) s += acc[(size_t)w * rowlen + i];
    out[i] = s;
  }
}

// rows, the line stage, and one mbarrier per warp (bulk-staged forms)
template <class T> size_t contract3_smem(const ContractPlan& p, int msl) {
  return p.smem + (size_t)msl * Chunks<T>::N * p.block * 16 + (size_t)(p.block / 32) * 8;
}

template <class T, int G, int SB, int MINB>
__global__ void __launch_bounds__(128, MINB) k_contract3(CArgs<T> A) {
  contract3_body<T, G, SB>(A, blockIdx.x);
}

// batched: the blocks of all lattices in one grid; pre[c] = first block of lattice c
template <class T, int G, int SB, int MINB>
__global__ void __launch_bounds__(128, MINB) kb_contract3(const CArgs<T>* __restrict__ A,
                                                          const long long* __restrict__ pre, int n) {
  const int c = find_item(pre, n, (long long)blockIdx.x);
  contract3_body<T, G, SB>(A[c], (int)(blockIdx.x - pre[c]));
}

template <class T, int G, int SB>
static void launch_contract3(const Geo& g, const ContractPlan& p, const typename V2<T>::t* u0,
                             const typename V2<T>::t* lines, int msl, int mwlt, int R,
                             double* partial, cudaStream_t st) {
  constexpr int MINB = (sizeof(T) == 4) ? ((G <= 3) ? 3 : 2) : ((G <= 1) ? 3 : 2);
  auto kern = k_contract3<T, G, SB, MINB>;
  size_t smem = contract3_smem<T>(p, msl);
  static size_t smem_set = 48 * 1024;  // attribute is raised only when needed (never under capture)
  if (smem > smem_set) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    smem_set = smem;
  }
  int grid = g.n[0] * p.ngrp * p.nCB;
  CArgs<T> A{};
  A.g = g;
  A.u0 = u0;
  A.lines = lines;
  A.msl = msl;
  A.mwlt = mwlt;
  A.R = R;
  A.ngrp = p.ngrp;
  A.nCB = p.nCB;
  A.partial = partial;
  kern<<<grid, p.block, smem, st>>>(A);
  WLG_LAUNCH_CHECK("contract");
}

template <class T, int G>
static void launch_contract3_sb(const Geo& g, const ContractPlan& p, const typename V2<T>::t* u0,
                                const typename V2<T>::t* lines, int msl, int mwlt, int R,
                                double* partial, cudaStream_t st) {
  if (p.SB == 2)
    launch_contract3<T, G, 2>(g, p, u0, lines, msl, mwlt, R, partial, st);
  else
    launch_contract3<T, G, 1>(g, p, u0, lines, msl, mwlt, R, partial, st);
}

// ---------------------------------------------------------------------------
// contraction kernel, fourth form: the third form with the warp reduction
// done through shared memory instead of shuffles.  After the recursion a lane
// forms its G*msl traces one top level at a time; once a level's staged
// lines are in registers (warp barrier), the lanes write their traces into
// that level's stage chunks (row (g,s2): 32 doubles, one per lane, in chunk
// (s2, q=g) shifted by (row & 7) * 16 bytes so that eight consecutive rows
// fall on distinct banks); after a second barrier lane r adds up row r in FP64
// and accumulates it.  No shuffles, no dependent reduction chains, and no
// extra shared memory: the rows reuse the stage of the current step.
// ---------------------------------------------------------------------------
// BULK: the msl top-line tiles of a warp's 32 columns arrive as msl bulk
// copies of one tile each (one lane per level) on a per-warp mbarrier,
// instead of 16-byte cp.async per thread and chunk.  Needs 32-aligned column
// ranges inside one direction: N1 N2 N3 a multiple of 32 (the launcher
// checks), column blocks rounded to 32 columns (below).
// PK (FP32 only), the eighth form: the recursion's products as packed
// two-lane FMAs (lmul_dag_inplace_x2 / rmul_inplace_x2), and each top level's
// staged line read from shared memory one level ahead.
template <class T, int G, int MSL, bool BULK, int PK = 0>
__device__ __forceinline__ void contract4_body(const CArgs<T>& A, int bid) {
  extern __shared__ double acc[];  // [nwarps][mwlt][G][msl] doubles, the line stage, mbarriers
  constexpr int NQ = Chunks<T>::N;
  constexpr int UNR = MSL > 0 ? MSL : 1;  // level loops unrolled when msl is a constant
  constexpr unsigned TILE_BYTES = NQ * 32 * 16;  // one direction tile of 32 links
  static_assert(G <= NQ, "one stage chunk per bottom level");

  const Geo& g = A.g;
  const typename V2<T>::t* __restrict__ u0 = A.u0;
  const typename V2<T>::t* __restrict__ lines = A.lines;
  const int msl = MSL > 0 ? MSL : A.msl;
  const int mwlt = A.mwlt, R = A.R, ngrp = A.ngrp, nCB = A.nCB;
  double* __restrict__ partial = A.partial;
  const int N0 = g.n[0], vs = g.vs, vol = g.vol;
  int b = bid;
  const int x0 = b % N0;
  b /= N0;
  const int grp = b % ngrp;
  const int cb = b / ngrp;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int rowlen = mwlt * G * msl;
  double* wacc = acc + (size_t)warp * rowlen;
  // 16-byte aligned for the 16-byte copies (an even number of doubles)
  char* stage = reinterpret_cast<char*>(acc + (((size_t)nwarps * rowlen + 1) & ~(size_t)1));
  // the warp's stage: chunk (s2, q) of its 32 lanes at wchunks + (s2*NQ + q)*512,
  // lane l's 16 bytes at + 16 l (the layout of a tile in global memory)
  constexpr int qstride = 512;
  char* wchunks = stage + (size_t)warp * msl * NQ * 512;
  char* myslot = wchunks + lane * 16;
  uint64_t* bar = reinterpret_cast<uint64_t*>(stage + (size_t)nwarps * msl * NQ * 512) + warp;
  unsigned phase = 0;
  bool stage_ok = true;
  for (int i = lane; i < rowlen; i += 32) wacc[i] = 0.0;
  if (BULK) {
    if (lane == 0) {
      mbar_init(bar, 1);
      mbar_init_fence();
    }
  }
  __syncwarp();

  const int s1_0 = grp * G;
  const int ncol = 3 * vs;
  // whole 32-column tiles per warp (needed by the bulk copies; kept for both
  // staging paths so that they split the columns, and sum, identically)
  const int per = (((ncol + nCB - 1) / nCB) + 31) & ~31;
  const int c_begin = cb * per;
  const int c_end = min(ncol, c_begin + per);
  const size_t fstride = link_elems<T>(vol);
  const int nrows = G * msl;

  for (int cbase = c_begin; cbase < c_end; cbase += blockDim.x) {
    const int col = cbase + threadIdx.x;
    const bool active = col < c_end;
    const int cc = active ? col : c_begin;
    const int k = cc / vs, xs = cc - k * vs;
    int xsR;
    {
      const int x1 = xs / g.st[1], r = xs - x1 * g.st[1];
      const int x2 = r / g.st[2], x3 = r - x2 * g.st[2];
      const int xk = (k == 0) ? x1 : ((k == 1) ? x2 : x3);
      const int nk = g.n[k + 1];
      int y = xk + (R % nk);
      if (y >= nk) y -= nk;
      xsR = xs + (y - xk) * g.st[k + 1];
    }
    const typename V2<T>::t* lk = lines + (size_t)k * fstride;
    const size_t lvl = 3 * fstride;
    M3<T> C[G];
#pragma unroll
    for (int gi = 0; gi < G; gi++) {
      int s1 = min(s1_0 + gi, msl - 1);
      ld(C[gi], lk + (size_t)s1 * lvl, vol, x0 * vs + xs);
      if (!active) zero(C[gi]);  // idle lanes contribute exact zeros
    }
    if (A.next) {
      // the spatial line step of the next R (compute_uk_long, wloop.c:207-258)
      // for this thread's own bottom lines: every (x0, column, level) has
      // exactly one owner, and the product is line_step_item's
      const size_t kof = (size_t)k * fstride;
#pragma unroll
      for (int gi = 0; gi < G; gi++) {
        const int s1 = s1_0 + gi;
        if (active && s1 < msl) {
          M3<T> lv, nx;
          ld(lv, A.level + kof + (size_t)s1 * lvl, vol, x0 * vs + xsR);
          mul(nx, C[gi], lv);
          st(A.next + kof + (size_t)s1 * lvl, vol, x0 * vs + xs, nx);
        }
      }
    }
    M3<T> ua, ub;
    ld(ua, u0, vol, x0 * vs + xs);
    ld(ub, u0, vol, x0 * vs + xsR);
    int t0 = x0;
    for (int tt = 1; tt <= mwlt; tt++) {
      const int t1 = (t0 + 1 == N0) ? 0 : t0 + 1;  // x0+T mod N0: the top slice
      const int stop = t1 * vs + xs;
      if (BULK) {
        // every lane's reads and writes of the stage come before the copies
        fence_proxy_async_smem();
        __syncwarp();
        if (stage_ok) {
          if (lane == 0) mbar_expect_tx(bar, (unsigned)msl * TILE_BYTES);
          __syncwarp();
          if (lane < msl) {
            // the warp's 32 columns are one tile: site stop - lane of lane 0
            const typename V2<T>::t* src = lk + (size_t)lane * lvl + (size_t)(stop >> 5) * Tile<T>::TS;
            bulk_g2s(wchunks + (size_t)lane * NQ * 512, src, TILE_BYTES, bar);
          }
        }
      } else {
        __syncwarp();  // previous step's rows are read before the stage is refilled
#pragma unroll UNR
        for (int s2 = 0; s2 < msl; s2++) {
          const typename V2<T>::t* src = lk + (size_t)s2 * lvl;
#pragma unroll
          for (int q = 0; q < NQ; q++)
            cp_async16(myslot + (s2 * NQ + q) * qstride, chunk_ptr<T>(src, stop, q));
        }
        cp_async_commit();
      }
      if constexpr (PK != 0 && sizeof(T) == 4) {
        lmul_dag_inplace_x2<G, PK == 2>(C, ua);
        rmul_inplace_x2<G, PK == 2>(C, ub);
      } else {
#pragma unroll
        for (int gi = 0; gi < G; gi++) lmul_dag_inplace(C[gi], ua);
#pragma unroll
        for (int gi = 0; gi < G; gi++) rmul_inplace(C[gi], ub);
      }
      t0 = t1;
      if (tt < mwlt) {
        ld(ua, u0, vol, t0 * vs + xs);
        ld(ub, u0, vol, t0 * vs + xsR);
      }
      if (BULK) {
        if (stage_ok) {
          const bool done = mbar_wait_bounded(bar, phase);
          if (__all_sync(0xffffffffu, done)) {
            phase ^= 1u;
          } else {
            // the copies did not arrive: flag it, stop staging, finish with
            // what is in the stage (the host discards the result)
            stage_ok = false;
            if (lane == 0) atomicExch(&g_stage_timeout, 1);
          }
        }
      } else {
        cp_async_wait_all();
      }
      if constexpr (PK != 0 && sizeof(T) == 4) {
        // the next level's staged line is read before this level's barrier
        // (its chunks are overwritten only after its own barrier), so the
        // shared-memory latency overlaps this level's traces
        M3<T> ln;
        ld_stage<T>(ln, myslot, qstride);
#pragma unroll UNR
        for (int s2 = 0; s2 < msl; s2++) {
          const M3<T> l = ln;
          if (s2 + 1 < msl) ld_stage<T>(ln, myslot + (s2 + 1) * NQ * qstride, qstride);
          __syncwarp();  // every lane holds level s2 before its chunks are overwritten
#pragma unroll
          for (int gi = 0; gi < G; gi++) {
            const int row = gi * msl + s2;
            double* dst = reinterpret_cast<double*>(wchunks + (s2 * NQ + gi) * qstride + (row & 7) * 16);
            dst[lane] = (double)retr_dag(l, C[gi]);
          }
        }
      } else {
#pragma unroll UNR
        for (int s2 = 0; s2 < msl; s2++) {
          M3<T> l;
          ld_stage<T>(l, myslot + s2 * NQ * qstride, qstride);
          __syncwarp();  // every lane holds level s2 before its chunks are overwritten
#pragma unroll
          for (int gi = 0; gi < G; gi++) {
            const int row = gi * msl + s2;
            double* dst = reinterpret_cast<double*>(wchunks + (s2 * NQ + gi) * qstride + (row & 7) * 16);
            dst[lane] = (double)retr_dag(l, C[gi]);
          }
        }
      }
      __syncwarp();
      double* arow = wacc + (size_t)(tt - 1) * nrows;
      for (int row = lane; row < nrows; row += 32) {
        const int gi = row / msl, s2 = row - gi * msl;
        const double2* src =
            reinterpret_cast<const double2*>(wchunks + (s2 * NQ + gi) * qstride + (row & 7) * 16);
        double s0 = 0.0, s1 = 0.0;
#pragma unroll
        for (int j = 0; j < 16; j++) {
          double2 v = src[j];
          s0 += v.x;
          s1 += v.y;
        }
        arow[row] += s0 + s1;
      }
    }
  }
  if (BULK && !stage_ok) mbar_wait_bounded(bar, phase);  // copies still in flight, bounded
  if (BULK && stage_ok) {  // every phase completed: nothing pending on the barrier
    __syncwarp();
    if (lane == 0) mbar_inval(bar);
  }
  __syncthreads();
  double* out = partial + ((size_t)(x0 * ngrp + grp) * nCB + cb) * rowlen;
  for (int i = threadIdx.x; i < rowlen; i += blockDim.x) {
    double s = 0.0;
    for (int w = 0; w < nwarps; w++) s += acc[(size_t)w * rowlen + i];
    out[i] = s;
  }
}

template <class T, int G, int MSL, int MINB, bool BULK, int PK>
__global__ void __launch_bounds__(128, MINB) k_contract4(CArgs<T> A) {
  contract4_body<T, G, MSL, BULK, PK>(A, blockIdx.x);
}

template <class T, int G, int MSL, int MINB, bool BULK, int PK>
__global__ void __launch_bounds__(128, MINB) kb_contract4(const CArgs<T>* __restrict__ A,
                                                          const long long* __restrict__ pre, int n) {
  const int c = find_item(pre, n, (long long)blockIdx.x);
  contract4_body<T, G, MSL, BULK, PK>(A[c], (int)(blockIdx.x - pre[c]));
}

// ---------------------------------------------------------------------------
// contraction kernel, ninth form (FP32 only): the eighth form reshaped for
// four blocks per SM.  Each warp owns one 32-column chunk (no column passes),
// so it needs no accumulator rows: after every step the lanes that sum a row
// write it straight into the warp's own partial record in global memory,
// [x0][group][chunk][T][G][msl] (the reduction kernel sums the records of
// all chunks).  A staged line takes 72 bytes (four 16-byte copies and one
// 8-byte copy of its first 36 floats; the 80-byte tile slot ends in 8 bytes
// of padding) instead of 80, so a 128-thread block holds 55 KB of shared
// memory instead of 75, and the launch bounds cap the registers at 128.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem));
}

constexpr int kLv9 = 4 * 512 + 256;  // stage bytes per level and warp

__device__ __forceinline__ void ld_stage9(M3<float>& m, const char* slot, const char* tail) {
#pragma unroll
  for (int q = 0; q < 4; q++) {
    float4 v = *reinterpret_cast<const float4*>(slot + q * 512);
    m.e[2 * q] = make_float2(v.x, v.y);
    m.e[2 * q + 1] = make_float2(v.z, v.w);
  }
  m.e[8] = *reinterpret_cast<const float2*>(tail);
}

template <int G, int MSL>
__device__ __forceinline__ void contract9_body(const CArgs<float>& A, int bid) {
  extern __shared__ double stage9[];  // [nwarps][msl][4 x 512 B + 256 B]
  static_assert(G >= 1 && G <= 4, "trace rows go to the level's first G chunks");
  constexpr int msl = MSL;
  const Geo& g = A.g;
  const float2* __restrict__ u0 = A.u0;
  const float2* __restrict__ lines = A.lines;
  const int mwlt = A.mwlt, R = A.R, ngrp = A.ngrp, nchunk = A.nCB;
  const int N0 = g.n[0], vs = g.vs, vol = g.vol;
  int b = bid;
  const int x0 = b % N0;
  b /= N0;
  const int grp = b % ngrp;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
  const int chunk = (b / ngrp) * nwarps + warp;
  if (chunk >= nchunk) return;  // the whole warp; the kernel has no block barrier
  char* wst = reinterpret_cast<char*>(stage9) + (size_t)warp * msl * kLv9;
  char* myslot = wst + lane * 16;
  char* mytail = wst + 4 * 512 + lane * 8;
  constexpr int nrows = G * msl;
  double* __restrict__ out = A.partial + ((size_t)(x0 * ngrp + grp) * nchunk + chunk) * mwlt * nrows;

  const int s1_0 = grp * G;
  const int ncol = 3 * vs;
  const int col = chunk * 32 + lane;
  const bool active = col < ncol;
  const int cc = active ? col : chunk * 32;
  const int k = cc / vs, xs = cc - k * vs;
  int xsR;
  {
    const int x1 = xs / g.st[1], r = xs - x1 * g.st[1];
    const int x2 = r / g.st[2], x3 = r - x2 * g.st[2];
    const int xk = (k == 0) ? x1 : ((k == 1) ? x2 : x3);
    const int nk = g.n[k + 1];
    int y = xk + (R % nk);
    if (y >= nk) y -= nk;
    xsR = xs + (y - xk) * g.st[k + 1];
  }
  const size_t fstride = link_elems<float>(vol);
  const float2* lk = lines + (size_t)k * fstride;
  const size_t lvl = 3 * fstride;
  M3<float> C[G];
#pragma unroll
  for (int gi = 0; gi < G; gi++) {
    const int s1 = min(s1_0 + gi, msl - 1);
    ld(C[gi], lk + (size_t)s1 * lvl, vol, x0 * vs + xs);
    if (!active) zero(C[gi]);  // idle lanes contribute exact zeros
  }
  if (A.next) {
    // the spatial line step of the next R for this thread's own bottom lines
    // (compute_uk_long, wloop.c:207-258), as in the fourth form
    const size_t kof = (size_t)k * fstride;
#pragma unroll
    for (int gi = 0; gi < G; gi++) {
      const int s1 = s1_0 + gi;
      if (active && s1 < msl) {
        M3<float> lv, nx;
        ld(lv, A.level + kof + (size_t)s1 * lvl, vol, x0 * vs + xsR);
        mul(nx, C[gi], lv);
        st(A.next + kof + (size_t)s1 * lvl, vol, x0 * vs + xs, nx);
      }
    }
  }
  M3<float> ua, ub;
  ld(ua, u0, vol, x0 * vs + xs);
  ld(ub, u0, vol, x0 * vs + xsR);
  int t0 = x0;
  for (int tt = 1; tt <= mwlt; tt++) {
    const int t1 = (t0 + 1 == N0) ? 0 : t0 + 1;  // x0+T mod N0: the top slice
    const int stop = t1 * vs + xs;
    __syncwarp();  // the previous step's rows are read before the stage is refilled
#pragma unroll
    for (int s2 = 0; s2 < msl; s2++) {
      const float2* src = lk + (size_t)s2 * lvl;
#pragma unroll
      for (int q = 0; q < 4; q++)
        cp_async16(myslot + s2 * kLv9 + q * 512, chunk_ptr<float>(src, stop, q));
      cp_async8(mytail + s2 * kLv9, chunk_ptr<float>(src, stop, 4));
    }
    cp_async_commit();
    lmul_dag_inplace_x2<G>(C, ua);
    rmul_inplace_x2<G>(C, ub);
    t0 = t1;
    if (tt < mwlt) {
      ld(ua, u0, vol, t0 * vs + xs);
      ld(ub, u0, vol, t0 * vs + xsR);
    }
    cp_async_wait_all();
#pragma unroll
    for (int s2 = 0; s2 < msl; s2++) {
      M3<float> l;
      ld_stage9(l, myslot + s2 * kLv9, mytail + s2 * kLv9);
      __syncwarp();  // every lane holds level s2 before its chunks are overwritten
#pragma unroll
      for (int gi = 0; gi < G; gi++) {
        const int row = gi * msl + s2;
        double* dst = reinterpret_cast<double*>(wst + s2 * kLv9 + gi * 512 + (row & 7) * 16);
        dst[lane] = (double)retr_dag(l, C[gi]);
      }
    }
    __syncwarp();
    if (lane < nrows) {
      const int row = lane, gi = row / msl, s2 = row - gi * msl;
      const double2* src =
          reinterpret_cast<const double2*>(wst + s2 * kLv9 + gi * 512 + (row & 7) * 16);
      double a0 = 0.0, a1 = 0.0;
#pragma unroll
      for (int j = 0; j < 16; j++) {
        const double2 v = src[j];
        a0 += v.x;
        a1 += v.y;
      }
      out[(size_t)(tt - 1) * nrows + row] = a0 + a1;
    }
  }
}

template <int G, int MSL>
__global__ void __launch_bounds__(128, 4) k_contract9(CArgs<float> A) {
  contract9_body<G, MSL>(A, blockIdx.x);
}

size_t contract9_smem(int block, int msl) { return (size_t)(block / 32) * msl * kLv9; }

template <int G, int MSL>
static void launch_contract9_m(const Geo& g, const ContractPlan& p, const float2* u0,
                               const float2* lines, int mwlt, int R, double* partial,
                               const float2* level, float2* next, cudaStream_t st) {
  auto kern = k_contract9<G, MSL>;
  const size_t smem = contract9_smem(p.block, MSL);
  static size_t smem_set = 48 * 1024;
  if (smem > smem_set) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    smem_set = smem;
  }
  CArgs<float> A{};
  A.g = g;
  A.u0 = u0;
  A.lines = lines;
  A.msl = MSL;
  A.mwlt = mwlt;
  A.R = R;
  A.ngrp = p.ngrp;
  A.nCB = p.nCB;
  A.partial = partial;
  A.level = level;
  A.next = next;
  const int per_block = p.block / 32;
  kern<<<g.n[0] * p.ngrp * ((p.nCB + per_block - 1) / per_block), p.block, smem, st>>>(A);
  WLG_LAUNCH_CHECK("contract9");
}

bool contract9_available(int msl, int G, bool fp64) {
  return !fp64 && msl >= 4 && msl <= 6 && G == (msl + 1) / 2;
}

void contract9_plan(ContractPlan& p, const Geo& g, int msl, int mwlt) {
  p.variant = 9;
  p.block = 128;
  p.nCB = (3 * g.vs + 31) / 32;  // one 32-column chunk per warp
  p.smem = contract9_smem(p.block, msl);
  p.partial_doubles = (size_t)g.n[0] * p.ngrp * p.nCB * mwlt * p.G * msl;
}

static void launch_contract9(const Geo& g, const ContractPlan& p, const float2* u0,
                             const float2* lines, int msl, int mwlt, int R, double* partial,
                             const float2* level, float2* next, cudaStream_t st) {
  switch (msl) {
    case 4: launch_contract9_m<2, 4>(g, p, u0, lines, mwlt, R, partial, level, next, st); return;
    case 5: launch_contract9_m<3, 5>(g, p, u0, lines, mwlt, R, partial, level, next, st); return;
    case 6: launch_contract9_m<3, 6>(g, p, u0, lines, mwlt, R, partial, level, next, st); return;
    default: set_error("contract: the ninth form needs msl 4-6");
  }
}

// level counts with their own fully unrolled kernels (the usual 4-6); others
// run the generic kernel (MSL = 0)
static inline int msl_variant(int msl) { return (msl >= 4 && msl <= 6) ? msl : 0; }

template <class T, int G, int MSL, bool BULK, int PK>
static void launch_contract4_m(const Geo& g, const ContractPlan& p, const typename V2<T>::t* u0,
                               const typename V2<T>::t* lines, int msl, int mwlt, int R,
                               double* partial, const typename V2<T>::t* level,
                               typename V2<T>::t* next, cudaStream_t st) {
  constexpr int MINB = (sizeof(T) == 4) ? ((G <= 3) ? 3 : 2) : ((G <= 1) ? 3 : 2);
  auto kern = k_contract4<T, G, MSL, MINB, BULK, PK>;
  size_t smem = contract3_smem<T>(p, msl);
  static size_t smem_set = 48 * 1024;
  if (smem > smem_set) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    smem_set = smem;
  }
  CArgs<T> A{};
  A.g = g;
  A.u0 = u0;
  A.lines = lines;
  A.msl = msl;
  A.mwlt = mwlt;
  A.R = R;
  A.ngrp = p.ngrp;
  A.nCB = p.nCB;
  A.partial = partial;
  A.level = level;
  A.next = next;
  kern<<<g.n[0] * p.ngrp * p.nCB, p.block, smem, st>>>(A);
  WLG_LAUNCH_CHECK("contract");
}

// unroll_msl: msl to unroll the level loops for, 0 for the generic kernel
template <class T, int G, bool BULK, int PK = 0>
static void launch_contract4_b(const Geo& g, const ContractPlan& p, const typename V2<T>::t* u0,
                               const typename V2<T>::t* lines, int msl, int unroll_msl, int mwlt,
                               int R, double* partial, const typename V2<T>::t* level,
                               typename V2<T>::t* next, cudaStream_t st) {
  switch (msl_variant(unroll_msl)) {
    case 4: launch_contract4_m<T, G, 4, BULK, PK>(g, p, u0, lines, msl, mwlt, R, partial, level, next, st); break;
    case 5: launch_contract4_m<T, G, 5, BULK, PK>(g, p, u0, lines, msl, mwlt, R, partial, level, next, st); break;
    case 6: launch_contract4_m<T, G, 6, BULK, PK>(g, p, u0, lines, msl, mwlt, R, partial, level, next, st); break;
    default: launch_contract4_m<T, G, 0, BULK, PK>(g, p, u0, lines, msl, mwlt, R, partial, level, next, st); break;
  }
}

// pk: packed FP32 products (eighth form; FP32 with cp.async staging only)
// pk 1: packed FP32 products (form 8); 2: the same with the signs in the
// shared broadcast pairs (form 10)
template <class T, int G>
static void launch_contract4(const Geo& g, const ContractPlan& p, const typename V2<T>::t* u0,
                             const typename V2<T>::t* lines, int msl, int unroll_msl, bool bulk,
                             int pk, int mwlt, int R, double* partial,
                             const typename V2<T>::t* level, typename V2<T>::t* next,
                             cudaStream_t st) {
  if constexpr (sizeof(T) == 4) {
    if (pk == 1) {
      launch_contract4_b<T, G, false, 1>(g, p, u0, lines, msl, unroll_msl, mwlt, R, partial, level, next, st);
      return;
    }
    if (pk == 2) {
      launch_contract4_b<T, G, false, 2>(g, p, u0, lines, msl, unroll_msl, mwlt, R, partial, level, next, st);
      return;
    }
  }
  if (bulk)
    launch_contract4_b<T, G, true>(g, p, u0, lines, msl, unroll_msl, mwlt, R, partial, level, next, st);
  else
    launch_contract4_b<T, G, false>(g, p, u0, lines, msl, unroll_msl, mwlt, R, partial, level, next, st);
}

template <class T, int G, int MSL, bool BULK, int PK = 0>
static void launch_contract4_batch_m(const CArgs<T>* A, const long long* pre, int n,
                                     long long nblocks, int block, size_t smem, cudaStream_t st) {
  constexpr int MINB = (sizeof(T) == 4) ? ((G <= 3) ? 3 : 2) : ((G <= 1) ? 3 : 2);
  auto kern = kb_contract4<T, G, MSL, MINB, BULK, PK>;
  static size_t smem_set = 48 * 1024;
  if (smem > smem_set) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    smem_set = smem;
  }
  kern<<<(unsigned)nblocks, block, smem, st>>>(A, pre, n);
  WLG_LAUNCH_CHECK("contract_batch");
}

// msl: the level count shared by every lattice of the launch, or 0
// pk: packed FP32 products with the signs in the shared broadcast pairs (tenth
// form, cp.async staging; FP32 only)
template <class T, int G>
static void launch_contract4_batch(const CArgs<T>* A, const long long* pre, int n, long long nblocks,
                                   int block, size_t smem, int msl, bool bulk, bool pk,
                                   cudaStream_t st) {
  if constexpr (sizeof(T) == 4) {
    if (pk && !bulk) {
      switch (msl_variant(msl)) {
        case 4: launch_contract4_batch_m<T, G, 4, false, 2>(A, pre, n, nblocks, block, smem, st); return;
        case 5: launch_contract4_batch_m<T, G, 5, false, 2>(A, pre, n, nblocks, block, smem, st); return;
        case 6: launch_contract4_batch_m<T, G, 6, false, 2>(A, pre, n, nblocks, block, smem, st); return;
        default: launch_contract4_batch_m<T, G, 0, false, 2>(A, pre, n, nblocks, block, smem, st); return;
      }
    }
  }
  switch (bulk ? 0 : msl_variant(msl)) {
    case 4: launch_contract4_batch_m<T, G, 4, false>(A, pre, n, nblocks, block, smem, st); break;
    case 5: launch_contract4_batch_m<T, G, 5, false>(A, pre, n, nblocks, block, smem, st); break;
    case 6: launch_contract4_batch_m<T, G, 6, false>(A, pre, n, nblocks, block, smem, st); break;
    default:
      if (bulk)
        launch_contract4_batch_m<T, G, 0, true>(A, pre, n, nblocks, block, smem, st);
      else
        launch_contract4_batch_m<T, G, 0, false>(A, pre, n, nblocks, block, smem, st);
      break;
  }
}

template <class T>
void contract(const Geo& g, const ContractPlan& p, const typename V2<T>::t* u0,
              const typename V2<T>::t* lines, int msl, int mwlt, int R, double* partial,
              const typename V2<T>::t* level, typename V2<T>::t* next, cudaStream_t st) {
  if (next && !contract_fuses_lines(p)) {
    set_error("contract: this form does not compute the next lines");
    return;
  }
  if (p.variant == 9) {
    if constexpr (sizeof(T) == 4) {
      if (!contract9_available(msl, p.G, false)) {
        set_error("contract: the ninth form needs FP32, msl 4-6 and G = (msl+1)/2");
        return;
      }
      launch_contract9(g, p, u0, lines, msl, mwlt, R, partial, level, next, st);
    } else {
      set_error("contract: the ninth form is FP32 only");
    }
    return;
  }
  if ((p.variant >= 4 && p.variant <= 8) || p.variant == 10) {
    // form 5: form 4 with the level loops unrolled for msl 4-6; forms 6 / 7:
    // forms 5 / 4 with the top lines staged by bulk copies, where a time
    // slice is whole 32-site tiles (else they run as forms 5 / 4); form 8:
    // form 5 with packed FP32 products (the FP64 form runs form 5)
    const int m = (p.variant == 5 || p.variant == 6 || p.variant == 8 || p.variant == 10) ? msl : 0;
    const bool bulk = (p.variant == 6 || p.variant == 7) && contract_can_bulk(g);
    const int pk = p.variant == 8 ? 1 : (p.variant == 10 ? 2 : 0);
    switch (p.G) {
      case 1: launch_contract4<T, 1>(g, p, u0, lines, msl, m, bulk, pk, mwlt, R, partial, level, next, st); return;
      case 2: launch_contract4<T, 2>(g, p, u0, lines, msl, m, bulk, pk, mwlt, R, partial, level, next, st); return;
      case 3: launch_contract4<T, 3>(g, p, u0, lines, msl, m, bulk, pk, mwlt, R, partial, level, next, st); return;
      case 4: launch_contract4<T, 4>(g, p, u0, lines, msl, m, bulk, pk, mwlt, R, partial, level, next, st); return;
      default: break;
    }
  }
  if (p.variant == 3) {
    switch (p.G) {
      case 1: launch_contract3_sb<T, 1>(g, p, u0, lines, msl, mwlt, R, partial, st); return;
      case 2: launch_contract3_sb<T, 2>(g, p, u0, lines, msl, mwlt, R, partial, st); return;
      case 3: launch_contract3_sb<T, 3>(g, p, u0, lines, msl, mwlt, R, partial, st); return;
      case 4: launch_contract3_sb<T, 4>(g, p, u0, lines, msl, mwlt, R, partial, st); return;
      default: break;  // G=6 falls through to the second form
    }
  }
  switch (p.G) {
    case 1: launch_contract2_sb<T, 1>(g, p, u0, lines, msl, mwlt, R, partial, st); break;
    case 2: launch_contract2_sb<T, 2>(g, p, u0, lines, msl, mwlt, R, partial, st); break;
    case 3: launch_contract2_sb<T, 3>(g, p, u0, lines, msl, mwlt, R, partial, st); break;
    case 4: launch_contract2_sb<T, 4>(g, p, u0, lines, msl, mwlt, R, partial, st); break;
    case 6: launch_contract2<T, 6, 1>(g, p, u0, lines, msl, mwlt, R, partial, st); break;
    default: set_error("contract: unsupported G=%d", p.G);
  }
}

// wl_mat[sl1 + msl*(sl2 + msl*(t + mwlt*(r + mwlr*x0)))] (wloop_parms.c:431-434)
__device__ __forceinline__ void reduce_item(const RArgs& A, int i) {
  const int msl = A.msl, mwlt = A.mwlt;
  const int rowlen = mwlt * A.G * msl;
  int s1 = i % msl, q = i / msl;
  int s2 = q % msl;
  q /= msl;
  int t = q % mwlt, x0 = q / mwlt;
  int grp = s1 / A.G, gi = s1 - grp * A.G;
  const double* p =
      A.partial + (size_t)((x0 * A.ngrp + grp) * A.nCB) * rowlen + (t * A.G + gi) * msl + s2;
  double s = 0.0;
  for (int cb = 0; cb < A.nCB; cb++) s += p[(size_t)cb * rowlen];
  A.wl[s1 + msl * (s2 + msl * (t + mwlt * (A.r + A.mwlr * x0)))] = s / A.norm;
}

__global__ void k_contract_reduce(RArgs A, int nout) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < nout; i += gridDim.x * blockDim.x)
    reduce_item(A, i);
}

__global__ void kb_contract_reduce(const RArgs* __restrict__ A, const long long* __restrict__ pre,
                                   int n, long long total) {
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < total;
       w += (long long)gridDim.x * blockDim.x) {
    const int c = find_item(pre, n, w);
    reduce_item(A[c], (int)(w - pre[c]));
  }
}

RArgs reduce_args(const Geo& g, const ContractPlan& p, int msl, int mwlt, int mwlr, int r,
                  const double* partial, double* wl_mat) {
  RArgs A;
  A.msl = msl;
  A.mwlt = mwlt;
  A.mwlr = mwlr;
  A.r = r;
  A.G = p.G;
  A.ngrp = p.ngrp;
  A.nCB = p.nCB;
  A.norm = 9.0 * (double)g.n[1] * (double)g.n[2] * (double)g.n[3];  // wloop.c:535
  A.partial = partial;
  A.wl = wl_mat;
  A.nout = g.n[0] * mwlt * msl * msl;
  return A;
}

void contract_reduce(const Geo& g, const ContractPlan& p, int msl, int mwlt, int mwlr, int r,
                     const double* partial, double* wl_mat, cudaStream_t st) {
  RArgs A = reduce_args(g, p, msl, mwlt, mwlr, r, partial, wl_mat);
  int grid = (A.nout + 255) / 256;
  k_contract_reduce<<<grid, 256, 0, st>>>(A, A.nout);
  WLG_LAUNCH_CHECK("contract_reduce");
}

// ---- batched launchers ----------------------------------------------------
static int bgrid(long long total, int block) {
  long long gsz = (total + block - 1) / block;
  long long cap = (long long)num_sms() * 32;
  return (int)(gsz < 1 ? 1 : (gsz > cap ? cap : gsz));
}

template <class T>
void line_step_batch(const LArgs<T>* A, const long long* pre, int n, long long total,
                     cudaStream_t st) {
  if (n <= 0 || total <= 0) return;
  kb_line_step<T><<<bgrid(total, 128), 128, 0, st>>>(A, pre, n, total);
  WLG_LAUNCH_CHECK("line_step_batch");
}

void contract_reduce_batch(const RArgs* A, const long long* pre, int n, long long total,
                           cudaStream_t st) {
  if (n <= 0 || total <= 0) return;
  kb_contract_reduce<<<bgrid(total, 256), 256, 0, st>>>(A, pre, n, total);
  WLG_LAUNCH_CHECK("contract_reduce_batch");
}

template <class T, int G, int SB>
static void launch_contract3_batch(const CArgs<T>* A, const long long* pre, int n,
                                   long long nblocks, int block, size_t smem, cudaStream_t st) {
  constexpr int MINB = (sizeof(T) == 4) ? ((G <= 3) ? 3 : 2) : ((G <= 1) ? 3 : 2);
  auto kern = kb_contract3<T, G, SB, MINB>;
  static size_t smem_set = 48 * 1024;  // raised only when needed (never under capture)
  if (smem > smem_set) {
    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    smem_set = smem;
  }
  kern<<<(unsigned)nblocks, block, smem, st>>>(A, pre, n);
  WLG_LAUNCH_CHECK("contract_batch");
}

template <class T>
void contract_batch(int G, int SB, const CArgs<T>* A, const long long* pre, int n, long long nblocks,
                    int block, size_t smem, int msl, cudaStream_t st) {
  if (n <= 0 || nblocks <= 0) return;
  // SB 0: fourth form (shared-memory reduction); SB 3: the same with its level
  // loops unrolled, where msl (shared by the launch) is 4-6; SB 4: the fourth
  // form with bulk-copy staging (every lattice's time slice whole tiles);
  // SB 5: SB 3 with packed FP32 products (the eighth form; FP64 runs SB 3)
  if (SB == 0 || SB == 3 || SB == 4 || SB == 5) {
    if (SB != 3 && SB != 5) msl = 0;
    const bool bulk = SB == 4, pk = SB == 5;
    switch (G) {
      case 1: launch_contract4_batch<T, 1>(A, pre, n, nblocks, block, smem, msl, bulk, pk, st); return;
      case 2: launch_contract4_batch<T, 2>(A, pre, n, nblocks, block, smem, msl, bulk, pk, st); return;
      case 3: launch_contract4_batch<T, 3>(A, pre, n, nblocks, block, smem, msl, bulk, pk, st); return;
      case 4: launch_contract4_batch<T, 4>(A, pre, n, nblocks, block, smem, msl, bulk, pk, st); return;
    }
  }
  if (SB == 2) {
    switch (G) {
      case 1: launch_contract3_batch<T, 1, 2>(A, pre, n, nblocks, block, smem, st); return;
      case 2: launch_contract3_batch<T, 2, 2>(A, pre, n, nblocks, block, smem, st); return;
      case 3: launch_contract3_batch<T, 3, 2>(A, pre, n, nblocks, block, smem, st); return;
      case 4: launch_contract3_batch<T, 4, 2>(A, pre, n, nblocks, block, smem, st); return;
    }
  } else {
    switch (G) {
      case 1: launch_contract3_batch<T, 1, 1>(A, pre, n, nblocks, block, smem, st); return;
      case 2: launch_contract3_batch<T, 2, 1>(A, pre, n, nblocks, block, smem, st); return;
      case 3: launch_contract3_batch<T, 3, 1>(A, pre, n, nblocks, block, smem, st); return;
      case 4: launch_contract3_batch<T, 4, 1>(A, pre, n, nblocks, block, smem, st); return;
    }
  }
  set_error("contract_batch: unsupported G=%d SB=%d", G, SB);
}

template void line_step<double>(const Geo&, int, int, const double2*, const double2*, double2*,
                                cudaStream_t);
template void line_step<float>(const Geo&, int, int, const float2*, const float2*, float2*,
                               cudaStream_t);
// Self-test of the bounded wait: one warp arms an mbarrier for bytes that no
// copy ever delivers and waits with the given limit, as the contraction
// waits for its staged lines; the outcome goes to out[0] (1: the wait ran
// out) and out[1] (elapsed ns).  Nothing faults or hangs: the wait ends at
// the limit and the barrier is left in shared memory that the block frees.
__global__ void k_wait_selftest(uint64_t limit_ns, unsigned long long* out) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    mbar_init_fence();
  }
  __syncwarp();
  if (threadIdx.x == 0) mbar_expect_tx(&bar, 512);  // no copy follows
  __syncwarp();
  const uint64_t t0 = global_ns();
  const bool done = mbar_wait_bounded(&bar, 0, limit_ns);
  const uint64_t t1 = global_ns();
  if (!__all_sync(0xffffffffu, done) && threadIdx.x == 0) {
    out[0] = 1;
    out[1] = t1 - t0;
  } else if (threadIdx.x == 0) {
    out[0] = 0;
    out[1] = t1 - t0;
  }
}

int wait_selftest(double limit_s, int* timed_out, double* elapsed_s) {
  unsigned long long* d = nullptr;
  unsigned long long h[2] = {0, 0};
  if (cudaMalloc(&d, sizeof(h)) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  k_wait_selftest<<<1, 32>>>((uint64_t)(limit_s * 1e9), d);
  cudaError_t e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
  cudaFree(d);
  if (e != cudaSuccess) return -1;
  *timed_out = (int)h[0];
  *elapsed_s = h[1] * 1e-9;
  return 0;
}

int contract_stage_failed() {
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, g_stage_timeout, sizeof(int)) != cudaSuccess) {
    cudaGetLastError();
    return -1;
  }
  if (v) {
    const int zero = 0;
    cudaMemcpyToSymbol(g_stage_timeout, &zero, sizeof(int));
  }
  return v;
}

template void contract<double>(const Geo&, const ContractPlan&, const double2*, const double2*, int,
                               int, int, double*, const double2*, double2*, cudaStream_t);
template void contract<float>(const Geo&, const ContractPlan&, const float2*, const float2*, int,
                              int, int, double*, const float2*, float2*, cudaStream_t);

}  // namespace wlg

namespace wlg {
template void line_step_batch<double>(const LArgs<double>*, const long long*, int, long long,
                                      cudaStream_t);
template void line_step_batch<float>(const LArgs<float>*, const long long*, int, long long,
                                     cudaStream_t);
template void contract_batch<double>(int, int, const CArgs<double>*, const long long*, int,
                                     long long, int, size_t, int, cudaStream_t);
template void contract_batch<float>(int, int, const CArgs<float>*, const long long*, int, long long,
                                    int, size_t, int, cudaStream_t);
template size_t contract3_smem<double>(const ContractPlan&, int);
template size_t contract3_smem<float>(const ContractPlan&, int);
}  // namespace wlg
