// internal.h -- launchers shared between the wloop_b200 translation units.
// Nothing here is exported; the C-ABI lives in include/wloop_b200.h.
#pragma once
#include <cuda_runtime.h>
#include <string>
#include "common.cuh"

namespace wlg {

// Launch shape for the site-parallel kernels (picked by the autotuner).
struct Shape {
  int block;  // threads per block
  int waves;  // grid = waves * SMs * blocks-per-SM (grid-stride loops)
};

int num_sms();

// ---- smearing (smear.cu) --------------------------------------------------
// HYP in three levels (hyp_links.c:194-451).  vbar/vtil hold 3 pair slots x 4
// directions; U is updated in place for the directions in [mu0,mu1).
template <class T>
void hyp_level3(const Geo& g, Links<T> U, typename V2<T>::t* vbar, double a3, int proj, int iter,
                cudaStream_t st);
template <class T>
void hyp_level2(const Geo& g, Links<T> U, const typename V2<T>::t* vbar, typename V2<T>::t* vtil,
                double a2, int proj, int iter, cudaStream_t st);
template <class T>
void hyp_level1(const Geo& g, Links<T> U, const typename V2<T>::t* vtil, double a1, int proj,
                int iter, int mu0, int mu1, int bc, cudaStream_t st);
// Work items of a smearing pass with nq outputs per site, ordered
// tile-major: item w is output q of site s with the nq outputs of one 32-site
// tile in consecutive warps, so the neighbour links their staples share are
// re-read from L2 rather than once per output over the whole field.  The
// volume is rounded up to whole tiles; items past the volume do nothing.
__host__ __device__ inline long long tile_items(int vol, int nq) {
  return (long long)nq * ((vol + 31) & ~31);
}
__host__ __device__ inline void tile_item(long long w, int nq, int& q, int& s) {
  const long long tile = w / (32 * nq);
  const int rem = (int)(w - tile * 32 * nq);
  q = rem >> 5;
  s = (int)(tile * 32) + (rem & 31);
}
// APE sweep over directions [mu0,4)
__host__ __device__ inline long long ape_items(int vol, int mu0) { return tile_items(vol, 4 - mu0); }
// One APE sweep dst = P[src + alpha * staples] over directions [mu0,4)
// (ape_links.c:147-272).  dst must not alias src.
template <class T>
void ape_sweep(const Geo& g, Links<T> src, Links<T> dst, double alpha, int proj, int iter,
               int mu0, cudaStream_t st);
// Two-level spatial HYP (hyp_spatial_links.c:160-344); dl holds 2 slots x 3
// spatial directions; U's spatial links are updated in place.
template <class T>
void hyp3d_level1(const Geo& g, Links<T> U, typename V2<T>::t* dl, double a2, int proj, int iter,
                  cudaStream_t st);
template <class T>
void hyp3d_level2(const Geo& g, Links<T> U, const typename V2<T>::t* dl, double a1, int proj,
                  int iter, cudaStream_t st);
// staple_sum (staple_sum.c:53-87): vb(x,mu) += staples in the (mu,nu) plane.
template <class T>
void staple_sum(const Geo& g, Links<T> u1, Links<T> u2, int mu, int nu, Links<T> vb,
                cudaStream_t st);
// v[i] += staple(u1[i],u2[i],u3[i]) for n packed FP64 matrices (dn: down
// staple; save: general form, else SU(3) third-column form).
void staples_lnks(int n, const double* u1, const double* u2, const double* u3, double* v, int dn,
                  int save, cudaStream_t st);
// In-place projection of n packed FP64 matrices (18 doubles each).
void project_batch(double* m, int n, int iter, cudaStream_t st);
// Plaquette sum (lnkplaq.c:48-128) into *out (device double); partial holds
// at least plaq_partials() doubles.
template <class T>
void plaq_sum(const Geo& g, int bc, Links<T> U, double* partial, double* out, cudaStream_t st);
int plaq_partials();
// FP64 plaquette sum of a field in device memory in the AoS lexicographic
// su3_dble layout of the host (noalloc.cu); partials must hold
// plaq_aos_partials(vol) doubles, out one double (both device memory).
void plaq_sum_aos(const Geo& g, int bc, const double* links, double* partials, double* out,
                  cudaStream_t st);
int plaq_aos_partials(long long vol);

// ---- loops (loops.cu) -----------------------------------------------------
// lines_dst[sl][k] = lines_src[sl][k](x) * level[sl][k](x + (R-1) k)
template <class T>
void line_step(const Geo& g, int msl, int R, const typename V2<T>::t* level,
               const typename V2<T>::t* src, typename V2<T>::t* dst, cudaStream_t st);
// Contraction for one spatial extent R: partial sums of
// Re tr(line_s2(x0+T)^dag  U0^dag...  line_s1(x0) ...U0') over columns.
struct ContractPlan {
  int variant;  // 1: first form, 2: in-place / prefetching form
  int SB;       // top levels per shuffle reduction (form 2)
  int G;        // bottom levels per thread
  int ngrp;     // ceil(msl/G)
  int nCB;      // column blocks per (x0, group)
  int block;    // threads per block
  size_t smem;  // dynamic shared memory bytes
  size_t partial_doubles;
};
ContractPlan contract_plan(const Geo& g, int msl, int mwlt, bool fp64, int G_hint, int nCB_hint,
                           int block_hint);
// With next non-null (forms 4 and 5 only) the launch also writes the lines of
// length R+1: next[sl][k](x) = lines[sl][k](x) level[sl][k](x + R k); next
// must not alias lines or level.
template <class T>
void contract(const Geo& g, const ContractPlan& p, const typename V2<T>::t* u0,
              const typename V2<T>::t* lines, int msl, int mwlt, int R, double* partial,
              const typename V2<T>::t* level, typename V2<T>::t* next, cudaStream_t st);
inline bool contract_fuses_lines(const ContractPlan& p) { return p.variant >= 4 && p.variant <= 10; }
// the ninth form (FP32, msl 4-6, G = (msl+1)/2): one 32-column chunk per warp,
// row sums written to per-warp partial records; contract9_plan turns a plan
// into one (nCB then counts 32-column chunks)
bool contract9_available(int msl, int G, bool fp64);
void contract9_plan(ContractPlan& p, const Geo& g, int msl, int mwlt);
// the bulk-staged forms need time slices of whole 32-site tiles
inline bool contract_can_bulk(const Geo& g) { return g.vs % 32 == 0; }
// 1 if a bulk-staged contraction gave up waiting for its copies since the
// last call (the flag is cleared), 0 if not, -1 if the flag cannot be read
int contract_stage_failed();
// runs the bounded-wait self-test on the current device (0 or -1)
int wait_selftest(double limit_s, int* timed_out, double* elapsed_s);
// Sums the partials and writes wl_mat[wl_idx(s1,s2,t,r,x0)] / norm.
void contract_reduce(const Geo& g, const ContractPlan& p, int msl, int mwlt, int mwlr, int r,
                     const double* partial, double* wl_mat, cudaStream_t st);

// ---- the temporal-gauge Gram form (gram.cu) -----------------------------------
// Shapes of one lattice's Gram stage; gram_plan returns false when the level
// count or mwlt do not fit the kernel (the other forms then apply).
struct GramPlan {
  int esize = 0;    // element bytes (4: mixed, 8: FP64)
  int L = 0;        // levels
  int Nu = 0;       // unrolled time extent (N0 + mwlt periodic, N0 open)
  int ntile = 0;    // 32-site tiles per time slice
  size_t A = 0;     // elements of one slab array over Nu slices
  size_t Aa = 0;    // elements of one slab array over N0 slices (the A lines)
  int TQ = 0, occ = 0, ord = 0;  // kernel variant: extents per thread, blocks per SM, FMA order
  int NG = 0, BX = 0, BXp = 0, NYB = 0, NYBp = 0, nblk = 0, nrows = 0, stages = 0;
  int block = 0;
  size_t smem = 0;  // dynamic shared memory per block
  int nchunks = 0, cpc = 0, nsplit = 0;
  size_t partial_elems = 0;
};
// Tuning of the Gram stage (0: automatic): blocks per SM (1, 2), FMA order
// (1: dot-product chains, 2: component-major), start slices per block (an
// upper bound), pipeline stages, column chunks per block.
struct GramTuning {
  int occ = 0, ord = 0, bx = 0, stages = 0, cpc = 0;
};
bool gram_plan(GramPlan& p, const Geo& g, int bc, int msl, int mwlt, bool fp64,
               const GramTuning* tune = nullptr);
// largest |g g^dag - 1| along time for which the form is used: beyond it
// (links smeared without a converged projection) H^-1 would amplify rounding
// and the carried-line form measures
constexpr double kGramMaxDeviation = 0.25;
// smallest lattice (sites) on which the form is the default: below it its
// fixed costs per measurement (the deviation read-back, the gauge chain, two
// more launches per R) outweigh the arithmetic it saves (8^4: 0.65 against
// 0.49 ms per measurement); it can still be asked for explicitly
constexpr long long kGramMinSites = 32768;
// The gauge field g and H^-1 = (g g^dag)^-1 (FP64 slabs of A doubles each)
// from the temporal links u0; *dev (device) receives max |g g^dag - 1| as the
// bits of a non-negative double (the form is not used when it exceeds 1/4).
template <class T>
void gauge_chain(const Geo& g, const GramPlan& p, const typename V2<T>::t* u0, double* G,
                 double* Hinv, unsigned long long* dev, cudaStream_t st);
// The recursion links uh and the lines of length 1 (blines, alines; [msl][3]
// slab arrays of A resp. Aa elements) from the level store; with alines
// null the A lines are left to gram_line_step with R = 1 (so that they may
// overwrite the level store, which this call reads).
template <class T>
void gauge_first(const Geo& g, const GramPlan& p, int msl, const typename V2<T>::t* levels,
                 const double* G, const double* Hinv, T* uh, T* blines, T* alines,
                 cudaStream_t st);
// blines of length R from those of length R-1 (in place), alines of length R
// (R = 1: alines only)
template <class T>
void gram_line_step(const Geo& g, const GramPlan& p, int msl, int R, const T* uh,
                    const double* Hinv, T* blines, T* alines, cudaStream_t st);
// sets the kernel's shared-memory limit for the plan (before any launch,
// outside stream capture); 0 or -1
int gram_prepare(const GramPlan& p);
// partial[nsplit][N0][mwlt][L][L] of the lines of one R
template <class T>
void gram_contract(const Geo& g, const GramPlan& p, int mwlt, const T* alines, const T* blines,
                   T* partial, cudaStream_t st);
// wl_mat entries of spatial extent index r from the partials
template <class T>
void gram_reduce(const Geo& g, const GramPlan& p, int bc, int mwlt, int mwlr, int r,
                 const T* partial, double* wl, cudaStream_t st);

// ---- batched stages (one launch over many lattices) ------------------------
// A: device array of n per-lattice argument records; pre: device array of
// n+1 prefix sums of the per-lattice work items (blocks for the contraction).
template <class T>
void smear_batch(int stage, const SArgs<T>* A, const long long* pre, int n, long long total,
                 cudaStream_t st);
enum { BATCH_HYP3 = 0, BATCH_HYP2, BATCH_HYP1, BATCH_APE, BATCH_HYP3D1, BATCH_HYP3D2 };
template <class T>
void line_step_batch(const LArgs<T>* A, const long long* pre, int n, long long total,
                     cudaStream_t st);
// msl: level count shared by all lattices of the launch (0 if they differ)
template <class T>
void contract_batch(int G, int SB, const CArgs<T>* A, const long long* pre, int n, long long nblocks,
                    int block, size_t smem, int msl, cudaStream_t st);
template <class T> size_t contract3_smem(const ContractPlan& p, int msl);
RArgs reduce_args(const Geo& g, const ContractPlan& p, int msl, int mwlt, int mwlr, int r,
                  const double* partial, double* wl_mat);
void contract_reduce_batch(const RArgs* A, const long long* pre, int n, long long total,
                           cudaStream_t st);

// ---- batch memory pool (batch.cu) -------------------------------------------
// gives the idle memory the batch pool of device dev keeps back to the device
void batch_pool_trim(int dev);

// ---- layout (layout.cu) ---------------------------------------------------
// AoS lexicographic FP64 [V][4][18] <-> SoA field of type T (directions [mu0,mu1)).
template <class T>
void aos_to_soa(const Geo& g, const double* aos, Links<T> U, int mu0, int mu1, cudaStream_t st);
template <class T>
void soa_to_aos(const Geo& g, Links<T> U, double* aos, int mu0, int mu1, cudaStream_t st);
// openQCD layout (8 links per odd point, lnkcom.c:840-859) <-> SoA; ipt maps
// lexicographic to openQCD site index.
template <class T>
void openqcd_to_soa(const Geo& g, const double* ud, const int* ipt, Links<T> U, int mu0, int mu1,
                    cudaStream_t st);
template <class T>
void soa_to_openqcd(const Geo& g, Links<T> U, const int* ipt, double* ud, int mu0, int mu1,
                    cudaStream_t st);

// ---- symmetry transformations (symm.cu) ------------------------------------
// U_mu(x) <- g(x) U_mu(x) g(x+mu)^dag with g a synthetic SU(3) field keyed by
// seed (written to G, one direction array); dst(x) = src(x - s), periodic.
template <class T>
void gauge_transform(const Geo& g, Links<T> U, typename V2<T>::t* G, uint64_t seed, double eps,
                     cudaStream_t st);
template <class T>
void shift_links(const Geo& g, Links<T> src, Links<T> dst, const int s[4], cudaStream_t st);

// ---- synthetic fields (gen_dev.cu) -----------------------------------------
// Writes the synthetic link field of the given seed/eps straight into SoA.
template <class T>
void generate_soa(const Geo& g, int bc, uint64_t seed, double eps, Links<T> U, cudaStream_t st);

// ---- error handling and launch accounting ---------------------------------
void set_error(const char* fmt, ...);
const char* get_error();
void count_launch();

}  // namespace wlg

#define WLG_CUDA(call)                                                                    \
  do {                                                                                    \
    cudaError_t e_ = (call);                                                              \
    if (e_ != cudaSuccess) {                                                              \
      wlg::set_error("%s failed at %s:%d: %s", #call, __FILE__, __LINE__,                 \
                     cudaGetErrorString(e_));                                             \
      return -1;                                                                          \
    }                                                                                     \
  } while (0)

#define WLG_LAUNCH_CHECK(name)                                                            \
  do {                                                                                    \
    wlg::count_launch();                                                                  \
    cudaError_t e_ = cudaGetLastError();                                                  \
    if (e_ != cudaSuccess) {                                                              \
      wlg::set_error("kernel %s: %s", name, cudaGetErrorString(e_));                      \
    }                                                                                     \
  } while (0)
