// ctx.cu -- the C ABI (include/wloop_b200.h): a context owns one lattice on
// one GPU, its scratch buffers and its stream, and sequences the kernels of
// smear.cu / loops.cu / layout.cu.
#include <float.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>
#include <algorithm>
#include <atomic>
#include <map>
#include <string>
#include <vector>
#include <nvtx3/nvToolsExt.h>
#include "internal.h"
#include "../../include/wloop_b200.h"

namespace wlg {

static thread_local char g_err[1024] = "";

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}
const char* get_error() { return g_err; }

static std::atomic<long long> g_launches{0};
void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

int num_sms() {
  static int cached[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  if (cached[dev] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
      n = 148;
      cudaGetLastError();  // no GPU (host-only planning): drop the failed query's error
    }
    cached[dev] = n;
  }
  return cached[dev];
}

}  // namespace wlg

using namespace wlg;

struct DevBuf {
  void* p = nullptr;
  size_t cap = 0;
};

struct ProfStat {
  double ms = 0.0;
  long long n = 0;
};

struct wlg_ctx {
  int dev = 0, prec = WLG_FP64, bc = 3;
  Geo g;
  cudaStream_t st = nullptr;
  DevBuf U, U0, bar, til, apeA, apeB, dl, levels, lines, lines2, partial, wl, plaq_part, plaq_out,
      staging, ipt;
  // the temporal-gauge form: g, H^-1, recursion links, B and A lines, the
  // unitarity deviation of g
  DevBuf gG, gH, gUh, gB, gA, gDev;
  void* lines_at = nullptr;  // buffer holding the lines of length lines_len
  // after a temporal-gauge measurement the lines of length lines_lazy are
  // rebuilt from the level store when they are asked for
  int lines_lazy = 0;
  // prefetch: the next field's host-to-device copy on its own stream
  DevBuf prefetch_buf;
  cudaStream_t cst = nullptr;
  cudaEvent_t copied = nullptr, consumed = nullptr;
  bool prefetched = false;
  int cG = 0, cNCB = 0, cBlock = 0, cVariant = 0, cSB = 0;
  GramTuning gtune;  // the temporal-gauge form's kernel variant and shape
  bool prof = false;
  std::map<std::string, ProfStat> stats;
  struct Pending {
    std::string name;
    cudaEvent_t a, b;
  };
  std::vector<Pending> pending;
  std::vector<cudaEvent_t> evpool;
  int last_msl = 0;
  int lines_len = 0;
  int used_variant = 0;  // contraction form of the last measurement
};

static int ensure(DevBuf& b, size_t bytes) {
  if (b.cap >= bytes && b.p) return 0;
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
  if (bytes == 0) return 0;
  cudaError_t e = cudaMalloc(&b.p, bytes);
  if (e != cudaSuccess) {
    // memory kept idle by the batch pool counts as free: return it, retry
    cudaGetLastError();
    int dev = 0;
    cudaGetDevice(&dev);
    batch_pool_trim(dev);
    e = cudaMalloc(&b.p, bytes);
  }
  if (e != cudaSuccess) {
    set_error("cudaMalloc(%zu bytes) failed: %s", bytes, cudaGetErrorString(e));
    cudaGetLastError();
    return -1;
  }
  b.cap = bytes;
  return 0;
}

static void release(DevBuf& b) {
  if (b.p) cudaFree(b.p);
  b.p = nullptr;
  b.cap = 0;
}

// bytes of one direction array (tiled layout, common.cuh) and of ndir of them
static size_t dir_bytes(const wlg_ctx* c) {
  return c->prec == WLG_FP64 ? link_elems<double>(c->g.vol) * sizeof(double2)
                             : link_elems<float>(c->g.vol) * sizeof(float2);
}
static size_t field_bytes(const wlg_ctx* c, int ndir) { return (size_t)ndir * dir_bytes(c); }

template <class T> static Links<T> view4(void* base, int vol) {
  Links<T> L;
  typename V2<T>::t* b = (typename V2<T>::t*)base;
  for (int mu = 0; mu < 4; mu++) L.p[mu] = b ? b + (size_t)mu * link_elems<T>(vol) : nullptr;
  return L;
}
// spatial-only field stored as 3 directions: p[0] is null
template <class T> static Links<T> view3(void* base, int vol) {
  Links<T> L;
  typename V2<T>::t* b = (typename V2<T>::t*)base;
  L.p[0] = nullptr;
  for (int k = 1; k < 4; k++) L.p[k] = b + (size_t)(k - 1) * link_elems<T>(vol);
  return L;
}

static cudaEvent_t get_event(wlg_ctx* c) {
  if (!c->evpool.empty()) {
    cudaEvent_t e = c->evpool.back();
    c->evpool.pop_back();
    return e;
  }
  cudaEvent_t e;
  cudaEventCreate(&e);
  return e;
}

// One stage of a measurement: an NVTX range of the stage's name around its
// launches (profilers select kernels by stage, e.g. ncu --nvtx --nvtx-include
// "contract/"; without a tool attached the range calls return at once) and,
// with profiling on, CUDA events on the context's stream around them.
struct ProfScope {
  wlg_ctx* c;
  const char* name;
  cudaEvent_t a = nullptr;
  ProfScope(wlg_ctx* c_, const char* n) : c(c_), name(n) {
    nvtxRangePushA(n);
    if (c->prof) {
      a = get_event(c);
      cudaEventRecord(a, c->st);
    }
  }
  ~ProfScope() {
    if (c->prof) {
      cudaEvent_t b = get_event(c);
      cudaEventRecord(b, c->st);
      c->pending.push_back({name, a, b});
    }
    nvtxRangePop();
  }
};

static void harvest(wlg_ctx* c) {
  if (c->pending.empty()) return;
  cudaStreamSynchronize(c->st);
  for (auto& p : c->pending) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, p.a, p.b);
    ProfStat& s = c->stats[p.name];
    s.ms += ms;
    s.n += 1;
    c->evpool.push_back(p.a);
    c->evpool.push_back(p.b);
  }
  c->pending.clear();
}

static int finish(const char* what) {
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("%s: %s", what, cudaGetErrorString(e));
    return -1;
  }
  if (get_error()[0] && strncmp(get_error(), "kernel ", 7) == 0) return -1;
  return 0;
}

#define CTX_BEGIN(c)                                  \
  do {                                                \
    if (!(c)) {                                       \
      set_error("null context");                      \
      return -1;                                      \
    }                                                 \
    set_error("%s", "");                              \
    WLG_CUDA(cudaSetDevice((c)->dev));                \
  } while (0)

// ---------------------------------------------------------------------------
// typed implementations
// ---------------------------------------------------------------------------
template <class T> static int do_hyp(wlg_ctx* c, double a1, double a2, double a3, int proj,
                                     int piter, int mu0, int mu1, int keep) {
  if (a1 == 0.0) return 0;  // hyp_links.c:405
  size_t fb = field_bytes(c, 12);
  if (ensure(c->bar, fb) || ensure(c->til, fb)) return -1;
  Links<T> U = view4<T>(c->U.p, c->g.vol);
  {
    ProfScope ps(c, "hyp");
    hyp_level3<T>(c->g, U, (typename V2<T>::t*)c->bar.p, a3, proj, piter, c->st);
    hyp_level2<T>(c->g, U, (const typename V2<T>::t*)c->bar.p, (typename V2<T>::t*)c->til.p, a2,
                  proj, piter, c->st);
    hyp_level1<T>(c->g, U, (const typename V2<T>::t*)c->til.p, a1, proj, piter, mu0, mu1, c->bc,
                  c->st);
  }
  if (!keep) {
    WLG_CUDA(cudaStreamSynchronize(c->st));
    release(c->bar);
    release(c->til);
  }
  return finish("hyp");
}

template <class T> static int do_ape(wlg_ctx* c, double alpha, int proj, int piter, int time,
                                     int nsweeps, int keep) {
  if (nsweeps <= 0) return 0;
  int mu0 = time ? 0 : 1;
  if (ensure(c->apeA, field_bytes(c, 4))) return -1;
  Links<T> U = view4<T>(c->U.p, c->g.vol), A = view4<T>(c->apeA.p, c->g.vol);
  {
    ProfScope ps(c, "ape");
    for (int i = 0; i < nsweeps; i++) {
      if (i % 2 == 0)
        ape_sweep<T>(c->g, U, A, alpha, proj, piter, mu0, c->st);
      else
        ape_sweep<T>(c->g, A, U, alpha, proj, piter, mu0, c->st);
    }
  }
  if (nsweeps % 2 == 1) {
    size_t off = (size_t)mu0 * dir_bytes(c);
    WLG_CUDA(cudaMemcpyAsync((char*)c->U.p + off, (char*)c->apeA.p + off,
                             field_bytes(c, 4 - mu0), cudaMemcpyDeviceToDevice, c->st));
  }
  if (!keep) {
    WLG_CUDA(cudaStreamSynchronize(c->st));
    release(c->apeA);
  }
  return finish("ape");
}


// one spatial-HYP sweep src -> dst (dst may equal src)
template <class T> static int hyp3_sweep(wlg_ctx* c, Links<T> src, Links<T> dst, double a1,
                                         double a2, int proj, int piter) {
  if (ensure(c->dl, field_bytes(c, 6))) return -1;
  hyp3d_level1<T>(c->g, src, (typename V2<T>::t*)c->dl.p, a2, proj, piter, c->st);
  if (src.p[1] != dst.p[1]) {
    // level 2 reads only its own src link for the linear combination
    for (int k = 1; k < 4; k++)
      WLG_CUDA(cudaMemcpyAsync(dst.p[k], src.p[k], dir_bytes(c),
                               cudaMemcpyDeviceToDevice, c->st));
  }
  hyp3d_level2<T>(c->g, dst, (const typename V2<T>::t*)c->dl.p, a1, proj, piter, c->st);
  return 0;
}

template <class T> static int do_hyp_spatial(wlg_ctx* c, double a1, double a2, int proj, int piter,
                                             int nsweeps, int keep) {
  Links<T> U = view4<T>(c->U.p, c->g.vol);
  {
    ProfScope ps(c, "hyp3");
    for (int i = 0; i < nsweeps; i++)
      if (hyp3_sweep<T>(c, U, U, a1, a2, proj, piter)) return -1;
  }
  if (!keep) {
    WLG_CUDA(cudaStreamSynchronize(c->st));
    release(c->dl);
  }
  return finish("hyp_spatial");
}

template <class T> static int do_plaq(wlg_ctx* c, Links<T> L, double* dev_out) {
  if (ensure(c->plaq_part, sizeof(double) * plaq_partials())) return -1;
  ProfScope ps(c, "plaq");
  plaq_sum<T>(c->g, c->bc, L, (double*)c->plaq_part.p, dev_out, c->st);
  return 0;
}

static int check_parms(const wlg_ctx* c, const wlg_wloop_parms* p) {
  const int* n = c->g.n;
  if (!p) {
    set_error("null parameters");
    return -1;
  }
  if (p->msl < 1 || p->msl > WLG_MAX_SM_LEVELS) {  // wloop_parms.c:156-157
    set_error("max smearing level out of range (msl=%d)", p->msl);
    return -1;
  }
  if (p->mwlt < 1 || p->mwlt > n[0] / 2 + 1) {  // :174-175
    set_error("max wloop time extension out of range (mwlt=%d)", p->mwlt);
    return -1;
  }
  if (p->mwlr < 1 || p->mwlr > n[1] / 2 + 1 || p->mwlr > n[2] / 2 + 1 || p->mwlr > n[3] / 2 + 1) {
    set_error("max wloop spatial extension out of range (mwlr=%d)", p->mwlr);  // :176-177
    return -1;
  }
  if (p->op_smear != WLG_OP_APE && p->op_smear != WLG_OP_HYP) {  // :104-105
    set_error("Unknown type of operator smearing");
    return -1;
  }
  for (int i = 0; i < p->msl; i++)
    if (p->nss[i] < 0) {
      set_error("negative number of smearing steps");
      return -1;
    }
  return 0;
}

// smear(): spatial smearing levels into the level store (smear.c:99-121)
template <class T>
static int do_smear(wlg_ctx* c, const wlg_wloop_parms* p, double* plaq) {
  if (check_parms(c, p)) return -1;
  const Geo& g = c->g;
  const int msl = p->msl, proj = p->proj_iter > 0;
  const size_t f3 = field_bytes(c, 3);
  if (ensure(c->levels, f3 * msl) || ensure(c->apeA, f3) || ensure(c->apeB, f3)) return -1;
  if (ensure(c->plaq_out, sizeof(double) * WLG_MAX_SM_LEVELS)) return -1;
  c->last_msl = msl;
  c->lines_lazy = 0;  // lines of an earlier measurement no longer match the levels
  Links<T> U = view4<T>(c->U.p, g.vol);
  Links<T> A = view3<T>(c->apeA.p, g.vol), B = view3<T>(c->apeB.p, g.vol);
  Links<T> cur = U;
  for (int sl = 0; sl < msl; sl++) {
    Links<T> lv = view3<T>((char*)c->levels.p + f3 * sl, g.vol);
    int ns = p->nss[sl];
    if (ns == 0) {
      for (int k = 1; k < 4; k++)
        WLG_CUDA(cudaMemcpyAsync(lv.p[k], cur.p[k], dir_bytes(c),
                                 cudaMemcpyDeviceToDevice, c->st));
    }
    for (int i = 0; i < ns; i++) {
      Links<T> dst = (i == ns - 1) ? lv : ((cur.p[1] == A.p[1]) ? B : A);
      ProfScope ps(c, p->op_smear == WLG_OP_APE ? "ape" : "hyp3");
      if (p->op_smear == WLG_OP_APE)
        ape_sweep<T>(g, cur, dst, p->alpha_ape, proj, p->proj_iter, 1, c->st);
      else if (hyp3_sweep<T>(c, cur, dst, p->alpha_hyp[0], p->alpha_hyp[1], proj, p->proj_iter))
        return -1;
      cur = dst;
    }
    cur = lv;
    if (plaq) {
      Links<T> pl = lv;
      pl.p[0] = U.p[0];
      if (do_plaq<T>(c, pl, (double*)c->plaq_out.p + sl)) return -1;
    }
  }
  if (plaq)
    WLG_CUDA(cudaMemcpyAsync(plaq, c->plaq_out.p, sizeof(double) * msl, cudaMemcpyDeviceToHost, c->st));
  return 0;
}

// The smearing and upload scratch (HYP levels, APE ping-pong, spatial-HYP
// level, host staging) is idle during the loop stage and allocated again by
// the next measurement that needs it: it is returned to the device when the
// loop stage's buffers do not fit beside it (FP64 at 48^3x96 holds 58 GB of
// it).  cudaFree waits for the device, so no copy or kernel still uses it.
static void release_idle_scratch(wlg_ctx* c) {
  release(c->bar);
  release(c->til);
  release(c->apeA);
  release(c->apeB);
  release(c->dl);
  release(c->staging);
  set_error("%s", "");
}

// wloops() in the temporal gauge (gram.cu): the gauge field and H^-1 once,
// then the first lines; per R the line step, the banded Gram product and its
// reduction.  Returns 1 (nothing done) when the form does not apply: shapes
// that do not fit, or a gauge field too far from unitary (links smeared
// without projection), which the other forms then measure.
template <class T>
static int do_loops_gram(wlg_ctx* c, const wlg_wloop_parms* p, double* wl_mat) {
  typedef typename V2<T>::t T2;
  const Geo& g = c->g;
  const int msl = p->msl;
  GramPlan gp;
  // the form needs projected smearing (the projection keeps the temporal
  // links near SU(3), so g stays well conditioned)
  if (p->proj_iter < 3) return 1;
  if (!gram_plan(gp, g, c->bc, msl, p->mwlt, c->prec == WLG_FP64, &c->gtune)) return 1;
  if (gram_prepare(gp)) return -1;
  const size_t nb = gp.A * sizeof(T) * 3 * msl, na = gp.Aa * sizeof(T) * 3 * msl;
  const size_t nwl = (size_t)msl * msl * p->mwlt * p->mwlr * g.n[0];
  if (ensure(c->gG, gp.A * sizeof(double)) || ensure(c->gH, gp.A * sizeof(double)) ||
      ensure(c->gDev, sizeof(unsigned long long)))
    return -1;
  Links<T> U = view4<T>(c->U.p, g.vol);
  double dev = 0.0;
  {
    ProfScope ps(c, "gauge");
    gauge_chain<T>(g, gp, U.p[0], (double*)c->gG.p, (double*)c->gH.p,
                   (unsigned long long*)c->gDev.p, c->st);
    unsigned long long bits = 0;
    WLG_CUDA(cudaMemcpyAsync(&bits, c->gDev.p, sizeof(bits), cudaMemcpyDeviceToHost, c->st));
    WLG_CUDA(cudaStreamSynchronize(c->st));
    memcpy(&dev, &bits, sizeof(dev));
  }
  if (!(dev <= kGramMaxDeviation)) return 1;
  auto alloc = [&]() {
    return ensure(c->gUh, nb) || ensure(c->gB, nb) || ensure(c->gA, na) ||
           ensure(c->partial, gp.partial_elems * sizeof(T)) || ensure(c->wl, sizeof(double) * nwl);
  };
  if (alloc()) {
    release_idle_scratch(c);
    if (alloc()) {
      // no room for the transformed lines: the carried-line form measures
      set_error("%s", "");
      release(c->gUh);
      release(c->gB);
      release(c->gA);
      release(c->gG);
      release(c->gH);
      return 1;
    }
  }
  c->used_variant = 11;
  c->lines_len = 0;
  c->lines_at = nullptr;
  c->lines_lazy = p->mwlr >= 2 ? p->mwlr : 0;
  T* uh = (T*)c->gUh.p;
  T* bl = (T*)c->gB.p;
  T* al = (T*)c->gA.p;
  const double* hinv = (const double*)c->gH.p;
  {
    ProfScope ps(c, "gauge");
    // the A lines of length 1 from the stored B lines, as a batch makes them
    gauge_first<T>(g, gp, msl, (const T2*)c->levels.p, (const double*)c->gG.p, hinv, uh, bl,
                   nullptr, c->st);
    gram_line_step<T>(g, gp, msl, 1, uh, hinv, bl, al, c->st);
  }
  for (int r = 0; r < p->mwlr; r++) {
    const int R = r + 1;
    if (R >= 2) {
      ProfScope ps(c, "lines");
      gram_line_step<T>(g, gp, msl, R, uh, hinv, bl, al, c->st);
    }
    {
      ProfScope ps(c, "contract");
      gram_contract<T>(g, gp, p->mwlt, al, bl, (T*)c->partial.p, c->st);
    }
    {
      ProfScope ps(c, "reduce");
      gram_reduce<T>(g, gp, c->bc, p->mwlt, p->mwlr, r, (const T*)c->partial.p, (double*)c->wl.p,
                     c->st);
    }
  }
  if (get_error()[0]) return -1;
  if (wl_mat)
    WLG_CUDA(cudaMemcpyAsync(wl_mat, c->wl.p, sizeof(double) * nwl, cudaMemcpyDeviceToHost, c->st));
  return 0;
}

// wloops(): spatial lines, fused temporal lines + contraction, reduction
// (wloop.c:524-608); needs the level store of do_smear.
template <class T>
static int do_loops(wlg_ctx* c, const wlg_wloop_parms* p, double* wl_mat) {
  typedef typename V2<T>::t T2;
  const Geo& g = c->g;
  const int msl = p->msl;
  const size_t f3 = field_bytes(c, 3);
  Links<T> U = view4<T>(c->U.p, g.vol);
  ContractPlan cp = contract_plan(g, msl, p->mwlt, c->prec == WLG_FP64, c->cG, c->cNCB, c->cBlock);
  if (c->cVariant) cp.variant = c->cVariant;
  if (c->cSB) cp.SB = c->cSB;
  if (cp.variant == 9) {
    if (!contract9_available(msl, cp.G, c->prec == WLG_FP64)) {
      set_error("contract: the ninth form needs FP32, msl 4-6 and G = (msl+1)/2");
      return -1;
    }
    contract9_plan(cp, g, msl, p->mwlt);
  }
  // the temporal-gauge form when asked for, or by default on lattices of at
  // least kGramMinSites sites
  if (c->cVariant == 11 || (c->cVariant == 0 && (long long)g.vol >= kGramMinSites)) {
    const int rc = do_loops_gram<T>(c, p, wl_mat);
    if (rc != 1) return rc;
    if (cp.variant == 11) cp = contract_plan(g, msl, p->mwlt, c->prec == WLG_FP64, c->cG, c->cNCB,
                                             c->cBlock);
  }
  c->lines_lazy = 0;
  c->used_variant = cp.variant;
  size_t nwl = (size_t)msl * msl * p->mwlt * p->mwlr * g.n[0];
  // forms 4 and 5 compute the lines of the next R inside the contraction
  // (ping-pong between two line buffers); other forms run the line step
  const bool fuse = contract_fuses_lines(cp);
  auto alloc = [&]() {
    return ensure(c->partial, sizeof(double) * cp.partial_doubles) ||
           ensure(c->wl, sizeof(double) * nwl) || (p->mwlr > 1 && ensure(c->lines, f3 * msl)) ||
           (fuse && p->mwlr > 2 && ensure(c->lines2, f3 * msl));
  };
  if (alloc()) {
    release_idle_scratch(c);
    if (alloc()) return -1;
  }
  c->lines_len = 0;
  c->lines_at = nullptr;
  const T2* lev = (const T2*)c->levels.p;
  T2* lines = (T2*)c->lines.p;
  T2* buf[2] = {(T2*)c->lines.p, (T2*)c->lines2.p};
  const T2* L = lev;
  for (int r = 0; r < p->mwlr; r++) {
    const int R = r + 1;
    if (!fuse && R >= 2) {
      ProfScope ps(c, "lines");
      line_step<T>(g, msl, R, lev, R == 2 ? lev : lines, lines, c->st);
      L = lines;
      c->lines_len = R;
      c->lines_at = lines;
    }
    T2* next = (fuse && R < p->mwlr) ? buf[r & 1] : nullptr;
    {
      ProfScope ps(c, "contract");
      contract<T>(g, cp, U.p[0], L, msl, p->mwlt, R, (double*)c->partial.p, lev, next, c->st);
    }
    if (next) {
      L = next;
      c->lines_len = R + 1;
      c->lines_at = next;
    }
    {
      ProfScope ps(c, "reduce");
      contract_reduce(g, cp, msl, p->mwlt, p->mwlr, r, (const double*)c->partial.p,
                      (double*)c->wl.p, c->st);
    }
  }
  if (wl_mat)
    WLG_CUDA(cudaMemcpyAsync(wl_mat, c->wl.p, sizeof(double) * nwl, cudaMemcpyDeviceToHost, c->st));
  return 0;
}

template <class T>
static int do_wloop_sum(wlg_ctx* c, const wlg_wloop_parms* p, double* wl_mat, double* plaq) {
  if (do_smear<T>(c, p, plaq) || do_loops<T>(c, p, wl_mat)) return -1;
  WLG_CUDA(cudaStreamSynchronize(c->st));
  if ((c->used_variant == 6 || c->used_variant == 7) && contract_stage_failed() != 0) {
    set_error("wloop_sum: the contraction's staged-line copies did not arrive in time");
    return -1;
  }
  return finish("wloop_sum");
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------
extern "C" {

const char* wlg_last_error(void) { return get_error(); }

int wlg_version(void) { return 100; }

int wlg_device_count(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

int wlg_create(const int n[4], int bc, int precision, int device, wlg_ctx** out) {
  set_error("%s", "");
  if (!n || !out) {
    set_error("null argument");
    return -1;
  }
  for (int i = 0; i < 4; i++)
    if (n[i] < 2) {
      set_error("lattice extent N%d=%d < 2", i, n[i]);
      return -1;
    }
  if ((long long)n[0] * n[1] * n[2] * n[3] > (1LL << 30)) {
    set_error("lattice volume too large");
    return -1;
  }
  if (bc != 0 && bc != 3) {
    set_error("only open (0) and periodic (3) boundary conditions are supported");
    return -1;
  }
  if (precision != WLG_FP64 && precision != WLG_MIXED) {
    set_error("unknown precision %d", precision);
    return -1;
  }
  int nd = wlg_device_count();
  if (nd <= 0) {
    set_error("no CUDA device available (the wloop_b200 path has no CPU fallback)");
    return -1;
  }
  if (device < 0 || device >= nd) {
    set_error("device %d out of range (%d devices)", device, nd);
    return -1;
  }
  WLG_CUDA(cudaSetDevice(device));
  wlg_ctx* c = new wlg_ctx();
  c->dev = device;
  c->prec = precision;
  c->bc = bc;
  c->g = make_geo(n);
  if (cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking) != cudaSuccess) {
    set_error("cudaStreamCreate failed");
    delete c;
    return -1;
  }
  if (ensure(c->U, field_bytes(c, 4))) {
    cudaStreamDestroy(c->st);
    delete c;
    return -1;
  }
  WLG_CUDA(cudaMemsetAsync(c->U.p, 0, field_bytes(c, 4), c->st));
  *out = c;
  return 0;
}

int wlg_free_scratch(wlg_ctx* c) {
  CTX_BEGIN(c);
  WLG_CUDA(cudaStreamSynchronize(c->st));
  if (c->cst) WLG_CUDA(cudaStreamSynchronize(c->cst));
  if (!c->prefetched) release(c->prefetch_buf);
  release(c->bar);
  release(c->til);
  release(c->apeA);
  release(c->apeB);
  release(c->dl);
  release(c->levels);
  release(c->lines);
  release(c->lines2);
  release(c->gG);
  release(c->gH);
  release(c->gUh);
  release(c->gB);
  release(c->gA);
  release(c->gDev);
  c->lines_at = nullptr;
  c->lines_len = 0;
  c->lines_lazy = 0;
  release(c->partial);
  release(c->staging);
  return 0;
}

int wlg_destroy(wlg_ctx* c) {
  if (!c) return 0;
  cudaSetDevice(c->dev);
  cudaStreamSynchronize(c->st);
  if (c->cst) cudaStreamSynchronize(c->cst);
  harvest(c);
  DevBuf* all[] = {&c->U, &c->U0, &c->bar, &c->til, &c->apeA, &c->apeB, &c->dl, &c->levels, &c->lines, &c->lines2,
                   &c->gG, &c->gH, &c->gUh, &c->gB, &c->gA, &c->gDev, &c->partial, &c->wl, &c->plaq_part, &c->plaq_out, &c->staging, &c->ipt,
                   &c->prefetch_buf};
  for (DevBuf* b : all) release(*b);
  for (cudaEvent_t e : c->evpool) cudaEventDestroy(e);
  if (c->cst) {
    cudaEventDestroy(c->copied);
    cudaEventDestroy(c->consumed);
    cudaStreamDestroy(c->cst);
  }
  cudaStreamDestroy(c->st);
  delete c;
  return 0;
}

int wlg_sync(wlg_ctx* c) {
  CTX_BEGIN(c);
  WLG_CUDA(cudaStreamSynchronize(c->st));
  return finish("sync");
}

int wlg_upload_links(wlg_ctx* c, const double* aos) {
  CTX_BEGIN(c);
  size_t bytes = (size_t)4 * 144 * c->g.vol;
  if (ensure(c->staging, bytes)) return -1;
  WLG_CUDA(cudaMemcpyAsync(c->staging.p, aos, bytes, cudaMemcpyHostToDevice, c->st));
  if (c->prec == WLG_FP64)
    aos_to_soa<double>(c->g, (const double*)c->staging.p, view4<double>(c->U.p, c->g.vol), 0, 4, c->st);
  else
    aos_to_soa<float>(c->g, (const double*)c->staging.p, view4<float>(c->U.p, c->g.vol), 0, 4, c->st);
  WLG_CUDA(cudaStreamSynchronize(c->st));
  return finish("upload_links");
}

// The host-to-device copy of the next field on a copy stream, so that it
// overlaps the measurement running on the context's stream.
int wlg_prefetch_links(wlg_ctx* c, const double* aos) {
  CTX_BEGIN(c);
  if (!aos) {
    set_error("prefetch_links: null field");
    return -1;
  }
  const size_t bytes = (size_t)4 * 144 * c->g.vol;
  if (!c->cst) {
    if (cudaStreamCreateWithFlags(&c->cst, cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->copied, cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&c->consumed, cudaEventDisableTiming) != cudaSuccess) {
      cudaGetLastError();
      set_error("prefetch_links: stream or event creation failed");
      return -1;
    }
    WLG_CUDA(cudaEventRecord(c->consumed, c->st));
  }
  if (c->prefetched) {
    set_error("prefetch_links: the previous prefetched field has not been uploaded");
    return -1;
  }
  if (c->prefetch_buf.cap < bytes) {
    WLG_CUDA(cudaStreamSynchronize(c->cst));
    if (ensure(c->prefetch_buf, bytes)) return -1;
  }
  // the buffer's previous contents have been transposed into U
  WLG_CUDA(cudaStreamWaitEvent(c->cst, c->consumed, 0));
  WLG_CUDA(cudaMemcpyAsync(c->prefetch_buf.p, aos, bytes, cudaMemcpyHostToDevice, c->cst));
  WLG_CUDA(cudaEventRecord(c->copied, c->cst));
  c->prefetched = true;
  return finish("prefetch_links");
}

int wlg_upload_prefetched(wlg_ctx* c) {
  CTX_BEGIN(c);
  if (!c->prefetched) {
    set_error("upload_prefetched: no field was prefetched");
    return -1;
  }
  WLG_CUDA(cudaStreamWaitEvent(c->st, c->copied, 0));
  if (c->prec == WLG_FP64)
    aos_to_soa<double>(c->g, (const double*)c->prefetch_buf.p, view4<double>(c->U.p, c->g.vol), 0, 4, c->st);
  else
    aos_to_soa<float>(c->g, (const double*)c->prefetch_buf.p, view4<float>(c->U.p, c->g.vol), 0, 4, c->st);
  WLG_CUDA(cudaEventRecord(c->consumed, c->st));
  c->prefetched = false;
  return finish("upload_prefetched");
}

int wlg_download_links(wlg_ctx* c, double* aos) {
  CTX_BEGIN(c);
  size_t bytes = (size_t)4 * 144 * c->g.vol;
  if (ensure(c->staging, bytes)) return -1;
  if (c->prec == WLG_FP64)
    soa_to_aos<double>(c->g, view4<double>(c->U.p, c->g.vol), (double*)c->staging.p, 0, 4, c->st);
  else
    soa_to_aos<float>(c->g, view4<float>(c->U.p, c->g.vol), (double*)c->staging.p, 0, 4, c->st);
  WLG_CUDA(cudaMemcpyAsync(aos, c->staging.p, bytes, cudaMemcpyDeviceToHost, c->st));
  WLG_CUDA(cudaStreamSynchronize(c->st));
  return finish("download_links");
}

// ipt must be a permutation of [0,V) that puts even sites first: it is used
// as an index on the device, so it is checked here.
static int check_ipt(const wlg_ctx* c, const int* ipt) {
  if (!ipt) {
    set_error("null ipt");
    return -1;
  }
  const Geo& g = c->g;
  std::vector<char> seen(g.vol, 0);
  for (int s = 0; s < g.vol; s++) {
    int iq = ipt[s];
    int x0 = s / g.st[0], r = s % g.st[0];
    int x1 = r / g.st[1], x2 = (r % g.st[1]) / g.st[2], x3 = r % g.st[2];
    int even = ((x0 + x1 + x2 + x3) & 1) == 0;
    if (iq < 0 || iq >= g.vol || seen[iq] || (even != (iq < g.vol / 2))) {
      set_error("ipt[%d]=%d is not an even-first permutation of the %d sites", s, iq, g.vol);
      return -1;
    }
    seen[iq] = 1;
  }
  return 0;
}

int wlg_upload_openqcd(wlg_ctx* c, const double* ud, const int* ipt) {
  CTX_BEGIN(c);
  if (check_ipt(c, ipt)) return -1;
  size_t bytes = (size_t)4 * 144 * c->g.vol;
  if (ensure(c->staging, bytes) || ensure(c->ipt, sizeof(int) * c->g.vol)) return -1;
  WLG_CUDA(cudaMemcpyAsync(c->staging.p, ud, bytes, cudaMemcpyHostToDevice, c->st));
  WLG_CUDA(cudaMemcpyAsync(c->ipt.p, ipt, sizeof(int) * c->g.vol, cudaMemcpyHostToDevice, c->st));
  if (c->prec == WLG_FP64)
    openqcd_to_soa<double>(c->g, (const double*)c->staging.p, (const int*)c->ipt.p,
                           view4<double>(c->U.p, c->g.vol), 0, 4, c->st);
  else
    openqcd_to_soa<float>(c->g, (const double*)c->staging.p, (const int*)c->ipt.p,
                          view4<float>(c->U.p, c->g.vol), 0, 4, c->st);
  WLG_CUDA(cudaStreamSynchronize(c->st));
  return finish("upload_openqcd");
}

int wlg_download_openqcd(wlg_ctx* c, double* ud, const int* ipt) {
  CTX_BEGIN(c);
  if (check_ipt(c, ipt)) return -1;
  size_t bytes = (size_t)4 * 144 * c->g.vol;
  if (ensure(c->staging, bytes) || ensure(c->ipt, sizeof(int) * c->g.vol)) return -1;
  WLG_CUDA(cudaMemcpyAsync(c->ipt.p, ipt, sizeof(int) * c->g.vol, cudaMemcpyHostToDevice, c->st));
  if (c->prec == WLG_FP64)
    soa_to_openqcd<double>(c->g, view4<double>(c->U.p, c->g.vol), (const int*)c->ipt.p,
                           (double*)c->staging.p, 0, 4, c->st);
  else
    soa_to_openqcd<float>(c->g, view4<float>(c->U.p, c->g.vol), (const int*)c->ipt.p,
                          (double*)c->staging.p, 0, 4, c->st);
  WLG_CUDA(cudaMemcpyAsync(ud, c->staging.p, bytes, cudaMemcpyDeviceToHost, c->st));
  WLG_CUDA(cudaStreamSynchronize(c->st));
  return finish("download_openqcd");
}

int wlg_generate(wlg_ctx* c, uint64_t seed, double eps) {
  CTX_BEGIN(c);
  if (c->prec == WLG_FP64)
    generate_soa<double>(c->g, c->bc, seed, eps, view4<double>(c->U.p, c->g.vol), c->st);
  else
    generate_soa<float>(c->g, c->bc, seed, eps, view4<float>(c->U.p, c->g.vol), c->st);
  WLG_CUDA(cudaStreamSynchronize(c->st));
  return finish("generate");
}

int wlg_hyp(wlg_ctx* c, double a1, double a2, double a3, int proj, int piter, int mu0, int mu1,
            int keep) {
  CTX_BEGIN(c);
  if (mu0 < 0 || mu1 > 4 || mu0 >= mu1) {
    set_error("hyp: bad direction range [%d,%d)", mu0, mu1);
    return -1;
  }
  int rc = c->prec == WLG_FP64 ? do_hyp<double>(c, a1, a2, a3, proj, piter, mu0, mu1, keep)
                               : do_hyp<float>(c, a1, a2, a3, proj, piter, mu0, mu1, keep);
  return rc;
}

int wlg_ape(wlg_ctx* c, double alpha, int proj, int piter, int time, int nsweeps, int keep) {
  CTX_BEGIN(c);
  return c->prec == WLG_FP64 ? do_ape<double>(c, alpha, proj, piter, time, nsweeps, keep)
                             : do_ape<float>(c, alpha, proj, piter, time, nsweeps, keep);
}

int wlg_hyp_spatial(wlg_ctx* c, double a1, double a2, int proj, int piter, int nsweeps, int keep) {
  CTX_BEGIN(c);
  return c->prec == WLG_FP64 ? do_hyp_spatial<double>(c, a1, a2, proj, piter, nsweeps, keep)
                             : do_hyp_spatial<float>(c, a1, a2, proj, piter, nsweeps, keep);
}

int wlg_plaq_sum(wlg_ctx* c, double* out) {
  CTX_BEGIN(c);
  if (ensure(c->plaq_out, sizeof(double) * WLG_MAX_SM_LEVELS)) return -1;
  int rc = c->prec == WLG_FP64
               ? do_plaq<double>(c, view4<double>(c->U.p, c->g.vol), (double*)c->plaq_out.p)
               : do_plaq<float>(c, view4<float>(c->U.p, c->g.vol), (double*)c->plaq_out.p);
  if (rc) return rc;
  WLG_CUDA(cudaMemcpyAsync(out, c->plaq_out.p, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  WLG_CUDA(cudaStreamSynchronize(c->st));
  return finish("plaq_sum");
}

// Number of plaquettes the sum runs over: 6 V, or (6 N0 - 3) N1 N2 N3 with
// open boundary conditions (the time plaquettes of the last slice are
// absent; lnkplaq.c:88).
static double plaquette_count(const wlg_ctx* c) {
  const double vs = (double)c->g.n[1] * c->g.n[2] * c->g.n[3];
  return (c->bc == 0 ? 6.0 * c->g.n[0] - 3.0 : 6.0 * c->g.n[0]) * vs;
}

// FP64 average plaquette of the su3_dble field in the staging buffer (the
// field as uploaded, before any rounding to the context's precision).
static int staged_average_plaquette(wlg_ctx* c, double* avg) {
  if (ensure(c->plaq_part, sizeof(double) * std::max(plaq_partials(),
                                                     plaq_aos_partials(c->g.vol))) ||
      ensure(c->plaq_out, sizeof(double) * WLG_MAX_SM_LEVELS))
    return -1;
  plaq_sum_aos(c->g, c->bc, (const double*)c->staging.p, (double*)c->plaq_part.p,
               (double*)c->plaq_out.p, c->st);
  double sum = 0.0;
  WLG_CUDA(cudaMemcpyAsync(&sum, c->plaq_out.p, sizeof(double), cudaMemcpyDeviceToHost, c->st));
  WLG_CUDA(cudaStreamSynchronize(c->st));
  *avg = sum / plaquette_count(c);
  return 0;
}

int wlg_import_cnfg(wlg_ctx* c, const char* path, double* plaq) {
  CTX_BEGIN(c);
  if (!path) {
    set_error("import_cnfg: null path");
    return -1;
  }
  std::vector<double> host((size_t)4 * 18 * c->g.vol);
  double stored = 0.0;
  if (wlg_cnfg_import(path, c->g.n, host.data(), &stored)) {
    set_error("%s", wlg_cnfg_error());
    return -1;
  }
  if (c->bc == 0) {
    // set_bc(): the time links of the last slice are zero with open bc
    const long long vs = (long long)c->g.n[1] * c->g.n[2] * c->g.n[3];
    for (long long s = (long long)(c->g.n[0] - 1) * vs; s < (long long)c->g.n[0] * vs; s++)
      memset(host.data() + 18 * (4 * s), 0, 18 * sizeof(double));
  }
  if (wlg_upload_links(c, host.data())) return -1;
  double avg = 0.0;
  if (staged_average_plaquette(c, &avg)) return -1;
  // openQCD's import check: |plaq(field) - plaq(head)| <= sqrt(nplaq) DBL_EPSILON
  const double tol = sqrt(plaquette_count(c)) * DBL_EPSILON;
  if (plaq) *plaq = avg;
  if (!(fabs(avg - stored) <= tol)) {
    set_error("import_cnfg: Incorrect average plaquette in %s (head %.16e, field %.16e)", path,
              stored, avg);
    return -1;
  }
  return finish("import_cnfg");
}

int wlg_export_cnfg(wlg_ctx* c, const char* path, double* plaq) {
  CTX_BEGIN(c);
  if (!path) {
    set_error("export_cnfg: null path");
    return -1;
  }
  std::vector<double> host((size_t)4 * 18 * c->g.vol);
  if (wlg_download_links(c, host.data())) return -1;
  // the plaquette of exactly the links written, in FP64
  size_t bytes = host.size() * sizeof(double);
  if (ensure(c->staging, bytes)) return -1;
  WLG_CUDA(cudaMemcpyAsync(c->staging.p, host.data(), bytes, cudaMemcpyHostToDevice, c->st));
  double avg = 0.0;
  if (staged_average_plaquette(c, &avg)) return -1;
  if (plaq) *plaq = avg;
  if (wlg_cnfg_export(path, c->g.n, host.data(), avg)) {
    set_error("%s", wlg_cnfg_error());
    return -1;
  }
  return finish("export_cnfg");
}

int wlg_wloop_sum(wlg_ctx* c, const wlg_wloop_parms* p, double* wl_mat, double* plaq) {
  CTX_BEGIN(c);
  return c->prec == WLG_FP64 ? do_wloop_sum<double>(c, p, wl_mat, plaq)
                             : do_wloop_sum<float>(c, p, wl_mat, plaq);
}

int wlg_smear_levels(wlg_ctx* c, const wlg_wloop_parms* p, double* plaq) {
  CTX_BEGIN(c);
  int rc = c->prec == WLG_FP64 ? do_smear<double>(c, p, plaq) : do_smear<float>(c, p, plaq);
  if (rc) return rc;
  WLG_CUDA(cudaStreamSynchronize(c->st));
  return finish("smear_levels");
}

int wlg_measure(wlg_ctx* c, const wlg_wloop_parms* p, double* wl_mat, double* plaq) {
  CTX_BEGIN(c);
  if (check_parms(c, p)) return -1;
  int proj = p->proj_iter > 0;
  if (wlg_hyp(c, p->alpha_action[0], p->alpha_action[1], p->alpha_action[2], proj, p->proj_iter, 0,
              4, 1))
    return -1;
  return wlg_wloop_sum(c, p, wl_mat, plaq);
}

static int download_spatial(wlg_ctx* c, void* base, double* aos3);

int wlg_download_level(wlg_ctx* c, int sl, double* aos3) {
  CTX_BEGIN(c);
  if (!c->levels.p || sl < 0 || sl >= c->last_msl) {
    set_error("level %d not available", sl);
    return -1;
  }
  return download_spatial(c, (char*)c->levels.p + field_bytes(c, 3) * sl, aos3);
}

}  // extern "C"

// the untransformed lines of length lines_lazy, rebuilt from the level store
// (the temporal-gauge form keeps only gauge-transformed lines)
template <class T> static int rebuild_lines(wlg_ctx* c) {
  typedef typename V2<T>::t T2;
  if (ensure(c->lines, field_bytes(c, 3) * c->last_msl)) return -1;
  const T2* lev = (const T2*)c->levels.p;
  T2* lines = (T2*)c->lines.p;
  for (int R = 2; R <= c->lines_lazy; R++)
    line_step<T>(c->g, c->last_msl, R, lev, R == 2 ? lev : lines, lines, c->st);
  c->lines_at = lines;
  c->lines_len = c->lines_lazy;
  c->lines_lazy = 0;
  return finish("download_lines");
}

extern "C" {

int wlg_download_lines(wlg_ctx* c, int sl, double* aos3, int* length) {
  CTX_BEGIN(c);
  if (!c->lines_at && c->lines_lazy >= 2 && c->levels.p) {
    if ((c->prec == WLG_FP64 ? rebuild_lines<double>(c) : rebuild_lines<float>(c)) != 0) return -1;
  }
  if (length) *length = c->lines_len;
  if (!c->lines_at || c->lines_len < 2 || sl < 0 || sl >= c->last_msl) {
    set_error("no spatial lines of level %d", sl);
    return -1;
  }
  return download_spatial(c, (char*)c->lines_at + field_bytes(c, 3) * sl, aos3);
}

static int download_spatial(wlg_ctx* c, void* base, double* aos3) {
  size_t bytes = (size_t)4 * 144 * c->g.vol;
  if (ensure(c->staging, bytes)) return -1;
  // convert to a 4-direction AoS with the temporal slot unused, then compact
  if (c->prec == WLG_FP64) {
    Links<double> L = view3<double>(base, c->g.vol);
    soa_to_aos<double>(c->g, L, (double*)c->staging.p, 1, 4, c->st);
  } else {
    Links<float> L = view3<float>(base, c->g.vol);
    soa_to_aos<float>(c->g, L, (double*)c->staging.p, 1, 4, c->st);
  }
  // AoS [V][4][18] -> [V][3][18]: strided copy of the spatial links
  WLG_CUDA(cudaMemcpy2DAsync(aos3, 3 * 144, (char*)c->staging.p + 144, 4 * 144, 3 * 144,
                             c->g.vol, cudaMemcpyDeviceToHost, c->st));
  WLG_CUDA(cudaStreamSynchronize(c->st));
  return finish("download_level");
}

int wlg_staple_sum(const int n[4], const double* u1, const double* u2, int mu, int nu, double* vb) {
  set_error("%s", "");
  if (mu < 0 || mu > 3 || nu < 0 || nu > 3 || mu == nu) {
    set_error("staple_sum: need 0<=mu,nu<4 and mu!=nu");
    return -1;
  }
  wlg_ctx* c = nullptr;
  if (wlg_create(n, 3, WLG_FP64, 0, &c)) return -1;
  int rc = -1;
  size_t fb = field_bytes(c, 4);
  DevBuf b1, b2;
  do {
    if (ensure(b1, fb) || ensure(b2, fb)) break;
    if (wlg_upload_links(c, u1)) break;
    WLG_CUDA(cudaMemcpyAsync(b1.p, c->U.p, fb, cudaMemcpyDeviceToDevice, c->st));
    if (wlg_upload_links(c, u2)) break;
    WLG_CUDA(cudaMemcpyAsync(b2.p, c->U.p, fb, cudaMemcpyDeviceToDevice, c->st));
    if (wlg_upload_links(c, vb)) break;
    staple_sum<double>(c->g, view4<double>(b1.p, c->g.vol), view4<double>(b2.p, c->g.vol), mu, nu,
                       view4<double>(c->U.p, c->g.vol), c->st);
    if (wlg_download_links(c, vb)) break;
    rc = 0;
  } while (0);
  release(b1);
  release(b2);
  wlg_destroy(c);
  return rc;
}

int wlg_project(double* mats, int nmat, int iter) {
  set_error("%s", "");
  if (nmat <= 0) return 0;
  if (wlg_device_count() <= 0) {
    set_error("no CUDA device available (the wloop_b200 path has no CPU fallback)");
    return -1;
  }
  DevBuf b;
  if (ensure(b, sizeof(double) * 18 * (size_t)nmat)) return -1;
  WLG_CUDA(cudaMemcpy(b.p, mats, sizeof(double) * 18 * (size_t)nmat, cudaMemcpyHostToDevice));
  project_batch((double*)b.p, nmat, iter, 0);
  WLG_CUDA(cudaMemcpy(mats, b.p, sizeof(double) * 18 * (size_t)nmat, cudaMemcpyDeviceToHost));
  release(b);
  return finish("project");
}

int wlg_staples(int nmat, const double* u1, const double* u2, const double* u3, double* v, int dn,
                int save) {
  set_error("%s", "");
  if (nmat <= 0) return 0;
  if (wlg_device_count() <= 0) {
    set_error("no CUDA device available (the wloop_b200 path has no CPU fallback)");
    return -1;
  }
  size_t bytes = sizeof(double) * 18 * (size_t)nmat;
  DevBuf b;
  if (ensure(b, 4 * bytes)) return -1;
  char* p = (char*)b.p;
  WLG_CUDA(cudaMemcpy(p, u1, bytes, cudaMemcpyHostToDevice));
  WLG_CUDA(cudaMemcpy(p + bytes, u2, bytes, cudaMemcpyHostToDevice));
  WLG_CUDA(cudaMemcpy(p + 2 * bytes, u3, bytes, cudaMemcpyHostToDevice));
  WLG_CUDA(cudaMemcpy(p + 3 * bytes, v, bytes, cudaMemcpyHostToDevice));
  staples_lnks(nmat, (const double*)p, (const double*)(p + bytes), (const double*)(p + 2 * bytes),
               (double*)(p + 3 * bytes), dn, save, 0);
  WLG_CUDA(cudaMemcpy(v, p + 3 * bytes, bytes, cudaMemcpyDeviceToHost));
  release(b);
  return finish("staples");
}

int wlg_set_profiling(wlg_ctx* c, int on) {
  CTX_BEGIN(c);
  harvest(c);
  c->prof = on != 0;
  return 0;
}

int wlg_kernel_time(wlg_ctx* c, const char* name, double* total_ms, long long* launches) {
  CTX_BEGIN(c);
  harvest(c);
  auto it = c->stats.find(name ? name : "");
  double ms = 0.0;
  long long n = 0;
  if (it != c->stats.end()) {
    ms = it->second.ms;
    n = it->second.n;
  }
  if (total_ms) *total_ms = ms;
  if (launches) *launches = n;
  return 0;
}

int wlg_reset_kernel_times(wlg_ctx* c) {
  CTX_BEGIN(c);
  harvest(c);
  c->stats.clear();
  return 0;
}

int wlg_set_contract_tuning(wlg_ctx* c, int variant, int G, int SB, int nCB, int block) {
  CTX_BEGIN(c);
  if (variant == 1 || variant < 0 || variant > 11 || G < 0 || G == 5 || G > 6 || SB < 0 || SB > 2 ||
      nCB < 0 || (block != 0 && (block % 32 != 0 || block > 128)) ||
      (variant == 2 && G == 6 && SB == 2) || (variant >= 3 && G > 4)) {
    set_error("bad contraction tuning (variant %d, G %d, SB %d, nCB %d, block %d)", variant, G,
              SB, nCB, block);
    return -1;
  }
  c->cVariant = variant;
  c->cG = G;
  c->cSB = SB;
  c->cNCB = nCB;
  c->cBlock = block;
  return 0;
}

int wlg_set_contract_shape(wlg_ctx* c, int G, int nCB, int block) {
  CTX_BEGIN(c);
  if (G < 0 || G == 5 || G > 6 || nCB < 0 || (block != 0 && (block % 32 != 0 || block > 128))) {
    set_error("bad contraction shape");
    return -1;
  }
  c->cG = G;
  c->cNCB = nCB;
  c->cBlock = block;
  return 0;
}

void* wlg_stream(wlg_ctx* c) { return c ? (void*)c->st : nullptr; }

int wlg_set_gram_tuning(wlg_ctx* c, int occ, int ord, int bx, int stages, int cpc) {
  CTX_BEGIN(c);
  if (occ < 0 || occ > 3 || ord < 0 || ord > 2 || bx < 0 || stages < 0 || stages > 4 ||
      stages == 1 || cpc < 0) {
    set_error("bad temporal-gauge tuning (occ %d, ord %d, bx %d, stages %d, cpc %d)", occ, ord,
              bx, stages, cpc);
    return -1;
  }
  c->gtune.occ = occ;
  c->gtune.ord = ord;
  c->gtune.bx = bx;
  c->gtune.stages = stages;
  c->gtune.cpc = cpc;
  return 0;
}

int wlg_gram_shape(wlg_ctx* c, int msl, int mwlt, int* shape) {
  CTX_BEGIN(c);
  GramPlan gp;
  if (!shape || !gram_plan(gp, c->g, c->bc, msl, mwlt, c->prec == WLG_FP64, &c->gtune)) {
    set_error("no temporal-gauge plan for msl %d, mwlt %d", msl, mwlt);
    return -1;
  }
  const int v[10] = {gp.TQ, gp.occ, gp.ord + 1, gp.BX, gp.nblk, gp.stages, gp.cpc, gp.nsplit,
                     gp.block, (int)(gp.smem / 1024)};
  for (int i = 0; i < 10; i++) shape[i] = v[i];
  return 0;
}

int wlg_gram_plan_shape(const int n[4], int bc, int msl, int mwlt, int precision,
                        const int tune[5], long long shape[16]) {
  set_error("%s", "");
  if (!n || !shape || (precision != WLG_FP64 && precision != WLG_MIXED) ||
      (bc != 0 && bc != 3)) {
    set_error("gram_plan_shape: bad arguments");
    return -1;
  }
  // the lattices wlg_create accepts
  for (int i = 0; i < 4; i++)
    if (n[i] < 2) {
      set_error("gram_plan_shape: lattice extent N%d=%d < 2", i, n[i]);
      return -1;
    }
  if ((long long)n[0] * n[1] * n[2] * n[3] > (1LL << 30)) {
    set_error("gram_plan_shape: lattice volume too large");
    return -1;
  }
  GramTuning t;
  if (tune) {
    t.occ = tune[0];
    t.ord = tune[1];
    t.bx = tune[2];
    t.stages = tune[3];
    t.cpc = tune[4];
  }
  GramPlan gp;
  if (!gram_plan(gp, make_geo(n), bc, msl, mwlt, precision == WLG_FP64, &t)) {
    set_error("no temporal-gauge plan for msl %d, mwlt %d", msl, mwlt);
    return -1;
  }
  const long long v[16] = {gp.TQ, gp.occ, gp.ord + 1, gp.BX, gp.BXp, gp.NG, gp.NYB, gp.NYBp,
                           gp.nblk, gp.nrows, gp.stages, gp.block, (long long)gp.smem,
                           gp.nchunks, gp.cpc, gp.nsplit};
  for (int i = 0; i < 16; i++) shape[i] = v[i];
  return 0;
}

int wlg_contract_form(wlg_ctx* c, int* form) {
  CTX_BEGIN(c);
  if (!form) {
    set_error("null argument");
    return -1;
  }
  *form = c->used_variant;
  return 0;
}

long long wlg_launch_count(void) { return g_launches.load(); }

int wlg_gauge_transform(wlg_ctx* c, uint64_t seed, double eps) {
  CTX_BEGIN(c);
  if (!(eps > 0.0)) {
    set_error("gauge_transform: eps must be positive");
    return -1;
  }
  if (ensure(c->apeB, dir_bytes(c))) return -1;
  if (c->prec == WLG_FP64)
    gauge_transform<double>(c->g, view4<double>(c->U.p, c->g.vol), (double2*)c->apeB.p, seed, eps,
                            c->st);
  else
    gauge_transform<float>(c->g, view4<float>(c->U.p, c->g.vol), (float2*)c->apeB.p, seed, eps,
                           c->st);
  return finish("gauge_transform");
}

int wlg_shift_links(wlg_ctx* c, const int s[4]) {
  CTX_BEGIN(c);
  if (!s) {
    set_error("shift_links: null shift");
    return -1;
  }
  if (c->bc == 0 && s[0] % c->g.n[0] != 0) {
    // the zero time links at x0 = N0-1 would move into the bulk
    set_error("shift_links: open boundary conditions allow spatial shifts only");
    return -1;
  }
  if (ensure(c->apeA, field_bytes(c, 4))) return -1;
  const size_t fb = field_bytes(c, 4);
  WLG_CUDA(cudaMemcpyAsync(c->apeA.p, c->U.p, fb, cudaMemcpyDeviceToDevice, c->st));
  if (c->prec == WLG_FP64)
    shift_links<double>(c->g, view4<double>(c->apeA.p, c->g.vol), view4<double>(c->U.p, c->g.vol),
                        s, c->st);
  else
    shift_links<float>(c->g, view4<float>(c->apeA.p, c->g.vol), view4<float>(c->U.p, c->g.vol), s,
                       c->st);
  return finish("shift_links");
}

int wlg_selftest_wait(int device, double limit_s, int* timed_out, double* elapsed_s) {
  set_error("%s", "");
  if (!timed_out || !elapsed_s || !(limit_s > 0.0) || limit_s > 10.0) {
    set_error("selftest_wait: bad arguments (limit 0 < s <= 10)");
    return -1;
  }
  if (device < 0 || device >= wlg_device_count() || cudaSetDevice(device) != cudaSuccess) {
    cudaGetLastError();
    set_error("selftest_wait: no device %d", device);
    return -1;
  }
  if (wait_selftest(limit_s, timed_out, elapsed_s)) {
    set_error("selftest_wait: %s", cudaGetErrorString(cudaGetLastError()));
    return -1;
  }
  return 0;
}

int wlg_snapshot(wlg_ctx* c) {
  CTX_BEGIN(c);
  if (ensure(c->U0, field_bytes(c, 4))) return -1;
  WLG_CUDA(cudaMemcpyAsync(c->U0.p, c->U.p, field_bytes(c, 4), cudaMemcpyDeviceToDevice, c->st));
  return finish("snapshot");
}

int wlg_restore(wlg_ctx* c) {
  CTX_BEGIN(c);
  if (!c->U0.p) {
    set_error("restore: no snapshot");
    return -1;
  }
  WLG_CUDA(cudaMemcpyAsync(c->U.p, c->U0.p, field_bytes(c, 4), cudaMemcpyDeviceToDevice, c->st));
  return finish("restore");
}

}  // extern "C"

// ---------------------------------------------------------------------------
// vector FMA throughput probe: 8 independent FMA chains per thread
// ---------------------------------------------------------------------------
template <class T>
__global__ void __launch_bounds__(256) k_peak(T* out, int iters, T a, T b) {
  T x[8];
#pragma unroll
  for (int j = 0; j < 8; j++) x[j] = (T)(threadIdx.x + j) * (T)1e-3;
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int j = 0; j < 8; j++) x[j] = fma(x[j], a, b);
  }
  T s = 0;
#pragma unroll
  for (int j = 0; j < 8; j++) s += x[j];
  if (s == (T)-12345.0) out[threadIdx.x] = s;  // keeps the chains live
}

// the same with packed two-lane FP32 FMAs (fma.rn.f32x2): 8 chains of
// float2, 16 FMAs per iteration and thread
__global__ void __launch_bounds__(256) k_peak_x2(float* out, int iters, float a, float b) {
  float2 x[8];
  const float2 a2 = make_float2(a, a), b2 = make_float2(b, b);
#pragma unroll
  for (int j = 0; j < 8; j++) x[j] = make_float2((threadIdx.x + j) * 1e-3f, (threadIdx.x - j) * 1e-3f);
  for (int i = 0; i < iters; i++) {
#pragma unroll
    for (int j = 0; j < 8; j++) x[j] = __ffma2_rn(x[j], a2, b2);
  }
  float s = 0.f;
#pragma unroll
  for (int j = 0; j < 8; j++) s += x[j].x + x[j].y;
  if (s == -12345.0f) out[threadIdx.x] = s;  // keeps the chains live
}

template <class T> static int peak_impl(int device, double* tflops, bool packed = false) {
  WLG_CUDA(cudaSetDevice(device));
  T* out = nullptr;
  WLG_CUDA(cudaMalloc(&out, 256 * sizeof(T)));
  int blocks = num_sms() * 8, iters = 1 << 15;
  cudaEvent_t a, b;
  cudaEventCreate(&a);
  cudaEventCreate(&b);
  float best = 1e30f;
  for (int rep = 0; rep < 4; rep++) {
    cudaEventRecord(a);
    if (packed)
      k_peak_x2<<<blocks, 256>>>((float*)out, iters, 0.999f, 1e-4f);
    else
      k_peak<T><<<blocks, 256>>>(out, iters, (T)0.999, (T)1e-4);
    cudaEventRecord(b);
    cudaEventSynchronize(b);
    float ms = 0;
    cudaEventElapsedTime(&ms, a, b);
    if (rep > 0 && ms < best) best = ms;
  }
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  cudaFree(out);
  double flops = 2.0 * (packed ? 16.0 : 8.0) * iters * 256.0 * blocks;
  *tflops = flops / (best * 1e-3) / 1e12;
  return finish("peak_flops");
}

extern "C" int wlg_peak_flops(int precision, int device, double* tflops) {
  set_error("%s", "");
  if (wlg_device_count() <= 0) {
    set_error("no CUDA device");
    return -1;
  }
  if (precision == WLG_PEAK_F32X2) return peak_impl<float>(device, tflops, true);
  return precision == WLG_FP64 ? peak_impl<double>(device, tflops) : peak_impl<float>(device, tflops);
}
