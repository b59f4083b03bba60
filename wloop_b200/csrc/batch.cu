// batch.cu -- many configurations, of possibly different lattices, measured
// together: every stage is one kernel over the flattened work of all
// lattices (the batched kernels of smear.cu / loops.cu), and the whole
// pipeline -- HYP, the spatial smearing levels, and for every spatial extent
// the line step, the contraction and its reduction, then the result copies --
// is captured once into a CUDA graph and replayed per batch.
//
// Memory: one arena per batch.  Per lattice: the gauge field, its snapshot,
// and one region that holds the HYP scratch while HYP runs and afterwards the
// APE ping-pong buffers, the level store and two spatial-line buffers (HYP
// has finished for every lattice before the first sweep writes there).  The
// contraction forms 4-7 write the next R's lines themselves, alternating
// between the two line buffers; the third form runs a line-step stage.
// Configurations of at least kGramMinSites sites whose smearing projects
// (proj_iter >= 3) run the temporal-gauge form (gram.cu) instead, one launch
// per lattice and stage
// inside the same graph: its g and H^-1 take the APE ping-pong slots, its A
// lines the level store (dead once the first lines exist), its recursion
// links and B lines start at the first line buffer, the region grown where
// they need more; the carried-line shapes of wlg_batch_set_contract_shape
// switch it off.  A run fails if g g^dag of such a lattice is far from 1.
#include <string.h>

#include <algorithm>
#include <mutex>
#include <vector>

#include "internal.h"
#include "../../include/wloop_b200.h"

using namespace wlg;

namespace {

struct Cfg {
  Geo g;
  int bc;
  wlg_wloop_parms p;
  ContractPlan cp;
  size_t D;  // elements per direction array
  size_t U, U0, region, wl;  // byte offsets in the arena
  size_t partial;            // byte offset in the partial-sum buffer
  size_t nwl;
  size_t wl_host;  // offset (doubles) in the pinned result block
  // temporal-gauge form: eligible (layout) and in use (plan), its plan and
  // the byte offsets of its buffers in the arena
  bool gram_ok, gram;
  GramPlan gp;
  size_t gG, gH, gUh, gB, gA, gDev;
  size_t gpartial;  // byte offset of its partial sums in the partial-sum buffer
};

enum OpKind {
  OP_SMEAR, OP_COPY, OP_LINES, OP_CONTRACT, OP_REDUCE, OP_D2H,
  OP_GRAM_CHAIN, OP_GRAM_PREP, OP_GRAM_R
};

struct Op {
  int kind;
  int stage;           // OP_SMEAR
  size_t tab, pre;     // byte offsets of the argument table and prefix in the table buffer
  int n;               // lattices in the launch
  long long total;     // work items (blocks for OP_CONTRACT)
  int G, SB, block;    // OP_CONTRACT
  int msl;             // OP_CONTRACT: level count of every lattice in the launch, 0 if mixed
  size_t smem;
  void* dst;
  const void* src;
  size_t bytes;
  int cfg, R;  // OP_GRAM_*: the lattice and the spatial extent
};

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace

struct wlg_batch {
  int dev = 0, prec = WLG_FP64;
  cudaStream_t st = nullptr;
  std::vector<Cfg> cfg;
  char* arena = nullptr;
  size_t arena_bytes = 0;
  char* pbuf = nullptr;  // contraction partial sums (depends on the contraction plan)
  size_t pbuf_bytes = 0, pbuf_cap = 0;
  double* wl_host = nullptr;  // pinned
  size_t wl_host_doubles = 0;
  unsigned long long* dev_host = nullptr;  // pinned: |g g^dag - 1| per lattice (bits)
  char* staging = nullptr;    // device AoS staging for uploads
  size_t staging_bytes = 0;
  // phase 0: smearing and the gauge chains; phase 1: the loops, per lattice
  // in the form phase 0's deviations allow (use_gram)
  struct Phase {
    std::vector<Op> ops;
    std::vector<char> host_tables;
    char* tables = nullptr;
    bool built = false;  // argument tables on the device
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    int kernels = 0;  // kernels one run of the phase launches
  } ph[2];
  std::vector<char> use_gram;  // per lattice: the temporal-gauge form runs in phase 1
  bool use_graph = true;       // capture each phase after its first run and replay it
  int tG = 0, tSB = 0, tBlock = 0, tNCB = 0;  // contraction shape override (tuning)
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // the temporal-gauge lattices of phase 1 run on these streams, lattice c
  // on side[c % kSide], forked from and joined back into st (inside the
  // captured graph, parallel branches), so the small per-lattice kernels of
  // different lattices overlap
  static constexpr int kSide = 4;
  cudaStream_t side[kSide] = {nullptr, nullptr, nullptr, nullptr};
  cudaEvent_t fork = nullptr, join[kSide] = {nullptr, nullptr, nullptr, nullptr};
  float last_ms = 0.f;
  int kernels = 0;
};

namespace {

// Device memory of batches comes from one stream-ordered pool per device
// that keeps freed memory (release threshold: never): a serving loop creates
// and destroys a batch per group of requests, and cudaMalloc / cudaFree would
// cost an allocation round trip and a device-wide synchronisation each time,
// stalling the batches of other workers in flight.
constexpr int kMaxPoolDevices = 64;
std::mutex g_pool_mutex;
cudaMemPool_t g_pool[kMaxPoolDevices] = {nullptr};

cudaMemPool_t batch_pool(int dev) {
  if (dev < 0 || dev >= kMaxPoolDevices) return nullptr;
  std::lock_guard<std::mutex> lock(g_pool_mutex);
  if (!g_pool[dev]) {
    cudaMemPoolProps props;
    memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t p = nullptr;
    if (cudaMemPoolCreate(&p, &props) != cudaSuccess) {
      cudaGetLastError();
      return nullptr;
    }
    uint64_t keep = ~0ull;
    cudaMemPoolSetAttribute(p, cudaMemPoolAttrReleaseThreshold, &keep);
    g_pool[dev] = p;
  }
  return g_pool[dev];
}

// stream-ordered allocation on the batch's stream; on failure the pool's
// idle memory is given back to the device and the allocation tried once more
template <class P>
int pool_alloc(wlg_batch* b, P** ptr, size_t bytes);

template <class P>
void pool_free(wlg_batch* b, P*& ptr);

}  // namespace

namespace {

size_t elem_bytes(const wlg_batch* b) { return b->prec == WLG_FP64 ? sizeof(double2) : sizeof(float2); }

template <class T> Links<T> lview(char* base, size_t D, int ndir, int first_mu) {
  Links<T> L;
  typename V2<T>::t* p = (typename V2<T>::t*)base;
  for (int mu = 0; mu < 4; mu++) L.p[mu] = nullptr;
  for (int k = 0; k < ndir; k++) L.p[first_mu + k] = p + (size_t)k * D;
  return L;
}

// the lattices a context accepts (wlg_create): extents of at least 2, at
// most 2^30 sites, open or periodic time; 0 or -1
static int check_lattice(const int* n, int bc) {
  for (int i = 0; i < 4; i++)
    if (n[i] < 2) return -1;
  if ((long long)n[0] * n[1] * n[2] * n[3] > (1LL << 30)) return -1;
  return (bc == 0 || bc == 3) ? 0 : -1;
}

int check_parms(const Geo& g, const wlg_wloop_parms& p) {
  if (p.msl < 1 || p.msl > WLG_MAX_SM_LEVELS) return -1;
  if (p.mwlt < 1 || p.mwlt > g.n[0] / 2 + 1) return -1;
  if (p.mwlr < 1 || p.mwlr > g.n[1] / 2 + 1 || p.mwlr > g.n[2] / 2 + 1 || p.mwlr > g.n[3] / 2 + 1)
    return -1;
  if (p.op_smear != WLG_OP_APE && p.op_smear != WLG_OP_HYP) return -1;
  for (int i = 0; i < p.msl; i++)
    if (p.nss[i] < 0) return -1;
  return 0;
}

// ---- table builder ----------------------------------------------------------
struct Tables {
  std::vector<char> bytes;
  template <class R> size_t add(const std::vector<R>& recs) {
    size_t off = align256(bytes.size());
    bytes.resize(off + recs.size() * sizeof(R));
    memcpy(bytes.data() + off, recs.data(), recs.size() * sizeof(R));
    return off;
  }
  size_t add_prefix(const std::vector<long long>& units) {
    std::vector<long long> pre(units.size() + 1, 0);
    for (size_t i = 0; i < units.size(); i++) pre[i + 1] = pre[i] + units[i];
    return add(pre);
  }
};

template <class T> void build_ops(wlg_batch* b, int phase) {
  typedef typename V2<T>::t T2;
  Tables tb;
  std::vector<Op> all;  // ops are generated for both phases; this phase's are kept
  int cur_phase = 0;    // phase of the ops generated next
  std::vector<int> phase_of;
  struct OpSink {
    std::vector<Op>* v;
    std::vector<int>* ph;
    int* cur;
    void push_back(const Op& o) {
      v->push_back(o);
      ph->push_back(*cur);
    }
  } sink{&all, &phase_of, &cur_phase};
  const int n = (int)b->cfg.size();
  auto base = [&](size_t off) { return b->arena + off; };
  auto push_smear = [&](int stage, const std::vector<SArgs<T>>& A, const std::vector<long long>& u) {
    if (A.empty()) return;
    Op op{};
    op.kind = OP_SMEAR;
    op.stage = stage;
    op.tab = tb.add(A);
    op.pre = tb.add_prefix(u);
    op.n = (int)A.size();
    op.total = 0;
    for (long long x : u) op.total += x;
    sink.push_back(op);
  };
  auto push_copy = [&](void* dst, const void* src, size_t bytes) {
    Op op{};
    op.kind = OP_COPY;
    op.dst = dst;
    op.src = src;
    op.bytes = bytes;
    sink.push_back(op);
  };

  // ---- HYP (hyp_links, all directions) ----
  {
    std::vector<SArgs<T>> a3, a2, a1;
    std::vector<long long> u12, u4;
    for (int c = 0; c < n; c++) {
      const Cfg& f = b->cfg[c];
      if (f.p.alpha_action[0] == 0.0) continue;  // hyp_links.c:405
      SArgs<T> A;
      memset(&A, 0, sizeof(A));
      A.g = f.g;
      A.U = lview<T>(base(f.U), f.D, 4, 0);
      A.aux0 = (T2*)base(f.region);
      A.aux1 = (T2*)base(f.region) + 12 * f.D;
      A.proj = f.p.proj_iter > 0;
      A.iter = f.p.proj_iter;
      A.bc = f.bc;
      A.mu0 = 0;
      A.nmu = 4;
      SArgs<T> x = A;
      x.a = 1.0 - f.p.alpha_action[2];
      x.b = f.p.alpha_action[2] / 2.0;
      a3.push_back(x);
      x.a = 1.0 - f.p.alpha_action[1];
      x.b = f.p.alpha_action[1] / 4.0;
      a2.push_back(x);
      x.a = 1.0 - f.p.alpha_action[0];
      x.b = f.p.alpha_action[0] / 6.0;
      a1.push_back(x);
      u12.push_back(tile_items(f.g.vol, 12));
      u4.push_back(tile_items(f.g.vol, 4));
    }
    push_smear(BATCH_HYP3, a3, u12);
    push_smear(BATCH_HYP2, a2, u12);
    push_smear(BATCH_HYP1, a1, u4);
  }

  // ---- spatial smearing levels (smear.c:99-121) ----
  // per lattice: cur = spatial links of U; sweep i of level sl writes the
  // level slot on its last sweep, else the ping-pong buffer not holding cur
  std::vector<Links<T>> cur(n), A(n), B(n);
  std::vector<char*> levels(n), lines(n), lines2(n), dl(n);
  int maxmsl = 0, maxr = 0;
  for (int c = 0; c < n; c++) {
    const Cfg& f = b->cfg[c];
    char* r = base(f.region);
    size_t es = elem_bytes(b);
    A[c] = lview<T>(r, f.D, 3, 1);
    B[c] = lview<T>(r + 3 * f.D * es, f.D, 3, 1);
    levels[c] = r + 6 * f.D * es;
    lines[c] = r + (6 + 3 * (size_t)f.p.msl) * f.D * es;
    dl[c] = r + (6 + 6 * (size_t)f.p.msl) * f.D * es;
    lines2[c] = r + (12 + 6 * (size_t)f.p.msl) * f.D * es;
    cur[c] = lview<T>(base(f.U) + f.D * es, f.D, 3, 1);
    maxmsl = std::max(maxmsl, f.p.msl);
    maxr = std::max(maxr, f.p.mwlr);
  }
  for (int sl = 0; sl < maxmsl; sl++) {
    int maxns = 0;
    for (int c = 0; c < n; c++) {
      const Cfg& f = b->cfg[c];
      if (sl >= f.p.msl) continue;
      maxns = std::max(maxns, f.p.nss[sl]);
      if (f.p.nss[sl] == 0) {
        Links<T> lv = lview<T>(levels[c] + (size_t)sl * 3 * f.D * elem_bytes(b), f.D, 3, 1);
        for (int k = 1; k < 4; k++) push_copy(lv.p[k], cur[c].p[k], f.D * elem_bytes(b));
        cur[c] = lv;
      }
    }
    for (int i = 0; i < maxns; i++) {
      std::vector<SArgs<T>> ape, h1, h2;
      std::vector<long long> u3, u6;
      for (int c = 0; c < n; c++) {
        const Cfg& f = b->cfg[c];
        if (sl >= f.p.msl || i >= f.p.nss[sl]) continue;
        Links<T> lv = lview<T>(levels[c] + (size_t)sl * 3 * f.D * elem_bytes(b), f.D, 3, 1);
        Links<T> dst = (i == f.p.nss[sl] - 1) ? lv : ((cur[c].p[1] == A[c].p[1]) ? B[c] : A[c]);
        SArgs<T> x;
        memset(&x, 0, sizeof(x));
        x.g = f.g;
        x.proj = f.p.proj_iter > 0;
        x.iter = f.p.proj_iter;
        if (f.p.op_smear == WLG_OP_APE) {
          x.U = cur[c];
          x.D = dst;
          x.a = f.p.alpha_ape;
          x.mu0 = 1;
          ape.push_back(x);
          u3.push_back(ape_items(f.g.vol, 1));
        } else {
          // spatial HYP: level 1 from cur into dl, copy cur -> dst, level 2 in place on dst
          x.U = cur[c];
          x.aux0 = (T2*)dl[c];
          x.a = 1.0 - f.p.alpha_hyp[1];
          x.b = f.p.alpha_hyp[1] / 2.0;
          h1.push_back(x);
          u6.push_back(6LL * f.g.vol);
          x.D = dst;
          x.a = 1.0 - f.p.alpha_hyp[0];
          x.b = f.p.alpha_hyp[0] / 4.0;
          h2.push_back(x);
        }
        cur[c] = dst;
      }
      push_smear(BATCH_APE, ape, u3);
      if (!h1.empty()) {
        push_smear(BATCH_HYP3D1, h1, u6);
        std::vector<long long> u3h;
        for (auto& x : h2) {
          u3h.push_back(3LL * x.g.vol);
          // the source of this sweep is h1's U for the same lattice
        }
        for (size_t j = 0; j < h2.size(); j++)
          for (int k = 1; k < 4; k++)
            if (h1[j].U.p[k] != h2[j].D.p[k])
              push_copy(h2[j].D.p[k], h1[j].U.p[k], link_elems<T>(h2[j].g.vol) * elem_bytes(b));
        push_smear(BATCH_HYP3D2, h2, u3h);
      }
    }
  }

  // ---- phase 0 ends with the gauge chains of the temporal-gauge lattices
  // and the read-back of their deviations from unitarity ----
  for (int c = 0; c < n; c++) {
    if (!b->cfg[c].gram) continue;
    Op op{};
    op.kind = OP_GRAM_CHAIN;
    op.cfg = c;
    sink.push_back(op);
    op.kind = OP_D2H;
    op.dst = b->dev_host + c;
    op.src = base(b->cfg[c].gDev);
    op.bytes = sizeof(unsigned long long);
    sink.push_back(op);
  }
  cur_phase = 1;
  auto gram_on = [&](int c) { return c < (int)b->use_gram.size() && b->use_gram[c]; };

  // ---- loops (wloop.c:524-608) ----
  // temporal-gauge lattices: the first lines, then per R their line step,
  // Gram product and reduction (one launch per lattice)
  for (int c = 0; c < n; c++) {
    if (!gram_on(c)) continue;
    Op op{};
    op.kind = OP_GRAM_PREP;
    op.cfg = c;
    sink.push_back(op);
  }
  for (int r = 0; r < maxr; r++)
    for (int c = 0; c < n; c++) {
      if (!gram_on(c) || r >= b->cfg[c].p.mwlr) continue;
      Op op{};
      op.kind = OP_GRAM_R;
      op.cfg = c;
      op.R = r + 1;
      sink.push_back(op);
    }
  for (int r = 0; r < maxr; r++) {
    const int R = r + 1;
    std::vector<LArgs<T>> la;
    std::vector<long long> lu;
    std::vector<RArgs> ra;
    std::vector<long long> ru;
    struct Group {
      int G, SB, block, msl;
      size_t smem;
      std::vector<CArgs<T>> a;
      std::vector<long long> blocks;
    };
    std::vector<Group> groups;
    for (int c = 0; c < n; c++) {
      const Cfg& f = b->cfg[c];
      if (r >= f.p.mwlr || gram_on(c)) continue;
      const T2* lev = (const T2*)levels[c];
      const T2* L = lev;
      const bool fuse = contract_fuses_lines(f.cp);
      T2* buf[2] = {(T2*)lines[c], (T2*)lines2[c]};
      if (fuse && R >= 2) L = buf[(R - 2) & 1];
      if (!fuse && R >= 2) {
        LArgs<T> x;
        x.g = f.g;
        x.msl = f.p.msl;
        x.R = R;
        x.level = lev;
        x.src = (R == 2) ? lev : (const T2*)lines[c];
        x.dst = (T2*)lines[c];
        la.push_back(x);
        lu.push_back((long long)f.p.msl * 3 * f.g.vol);
        L = (const T2*)lines[c];
      }
      CArgs<T> ca{};
      ca.g = f.g;
      ca.u0 = (const T2*)base(f.U);
      ca.lines = L;
      ca.msl = f.p.msl;
      ca.mwlt = f.p.mwlt;
      ca.R = R;
      ca.ngrp = f.cp.ngrp;
      ca.nCB = f.cp.nCB;
      ca.partial = (double*)(b->pbuf + f.partial);
      ca.level = lev;
      ca.next = (fuse && R < f.p.mwlr) ? buf[(R - 1) & 1] : nullptr;
      Group* gp = nullptr;
      for (auto& gr : groups)
        if (gr.G == f.cp.G && gr.SB == f.cp.SB && gr.block == f.cp.block) gp = &gr;
      if (!gp) {
        groups.push_back(Group{f.cp.G, f.cp.SB, f.cp.block, f.p.msl, 0, {}, {}});
        gp = &groups.back();
      }
      // unrolled kernels need one level count for the whole launch
      if (gp->msl != f.p.msl || (f.cp.variant != 5 && f.cp.variant != 8)) gp->msl = 0;
      gp->smem = std::max(gp->smem, contract3_smem<T>(f.cp, f.p.msl));
      gp->a.push_back(ca);
      gp->blocks.push_back((long long)f.g.n[0] * f.cp.ngrp * f.cp.nCB);
      RArgs rr = reduce_args(f.g, f.cp, f.p.msl, f.p.mwlt, f.p.mwlr, r,
                             (const double*)(b->pbuf + f.partial), (double*)base(f.wl));
      ra.push_back(rr);
      ru.push_back(rr.nout);
    }
    if (!la.empty()) {
      Op op{};
      op.kind = OP_LINES;
      op.tab = tb.add(la);
      op.pre = tb.add_prefix(lu);
      op.n = (int)la.size();
      for (long long x : lu) op.total += x;
      sink.push_back(op);
    }
    for (auto& gr : groups) {
      Op op{};
      op.kind = OP_CONTRACT;
      op.tab = tb.add(gr.a);
      op.pre = tb.add_prefix(gr.blocks);
      op.n = (int)gr.a.size();
      for (long long x : gr.blocks) op.total += x;
      op.G = gr.G;
      op.SB = gr.SB;
      op.block = gr.block;
      op.msl = gr.msl;
      op.smem = gr.smem;
      sink.push_back(op);
    }
    if (!ra.empty()) {
      Op op{};
      op.kind = OP_REDUCE;
      op.tab = tb.add(ra);
      op.pre = tb.add_prefix(ru);
      op.n = (int)ra.size();
      for (long long x : ru) op.total += x;
      sink.push_back(op);
    }
  }
  for (int c = 0; c < n; c++) {
    const Cfg& f = b->cfg[c];
    Op op{};
    op.kind = OP_D2H;
    op.dst = b->wl_host + f.wl_host;
    op.src = base(f.wl);
    op.bytes = f.nwl * sizeof(double);
    sink.push_back(op);
  }
  b->ph[phase].ops.clear();
  for (size_t k = 0; k < all.size(); k++)
    if (phase_of[k] == phase) b->ph[phase].ops.push_back(all[k]);
  b->ph[phase].host_tables.swap(tb.bytes);
}

template <class T> int issue(wlg_batch* b, int phase) {
  int kernels = 0;
  const char* tables = b->ph[phase].tables;
  bool forked = false;
  auto lattice_stream = [&](int c) -> cudaStream_t {
    return b->side[0] ? b->side[c % wlg_batch::kSide] : b->st;
  };
  for (const Op& op : b->ph[phase].ops) {
    const bool gram_op = op.kind == OP_GRAM_PREP || op.kind == OP_GRAM_R;
    if (gram_op && !forked && b->side[0]) {
      WLG_CUDA(cudaEventRecord(b->fork, b->st));
      for (int k = 0; k < wlg_batch::kSide; k++) WLG_CUDA(cudaStreamWaitEvent(b->side[k], b->fork, 0));
      forked = true;
    }
    if (op.kind == OP_D2H && forked) {
      for (int k = 0; k < wlg_batch::kSide; k++) {
        WLG_CUDA(cudaEventRecord(b->join[k], b->side[k]));
        WLG_CUDA(cudaStreamWaitEvent(b->st, b->join[k], 0));
      }
      forked = false;
    }
    switch (op.kind) {
      case OP_SMEAR:
        smear_batch<T>(op.stage, (const SArgs<T>*)(tables + op.tab),
                       (const long long*)(tables + op.pre), op.n, op.total, b->st);
        kernels++;
        break;
      case OP_COPY:
        WLG_CUDA(cudaMemcpyAsync(op.dst, op.src, op.bytes, cudaMemcpyDeviceToDevice, b->st));
        break;
      case OP_LINES:
        line_step_batch<T>((const LArgs<T>*)(tables + op.tab),
                           (const long long*)(tables + op.pre), op.n, op.total, b->st);
        kernels++;
        break;
      case OP_CONTRACT:
        contract_batch<T>(op.G, op.SB, (const CArgs<T>*)(tables + op.tab),
                          (const long long*)(tables + op.pre), op.n, op.total, op.block,
                          op.smem, op.msl, b->st);
        kernels++;
        break;
      case OP_REDUCE:
        contract_reduce_batch((const RArgs*)(tables + op.tab),
                              (const long long*)(tables + op.pre), op.n, op.total, b->st);
        kernels++;
        break;
      case OP_D2H:
        WLG_CUDA(cudaMemcpyAsync(op.dst, op.src, op.bytes, cudaMemcpyDeviceToHost, b->st));
        break;
      case OP_GRAM_CHAIN: {
        const Cfg& f = b->cfg[op.cfg];
        gauge_chain<T>(f.g, f.gp, lview<T>(b->arena + f.U, f.D, 4, 0).p[0],
                       (double*)(b->arena + f.gG), (double*)(b->arena + f.gH),
                       (unsigned long long*)(b->arena + f.gDev), b->st);
        kernels++;
        break;
      }
      case OP_GRAM_PREP: {
        const Cfg& f = b->cfg[op.cfg];
        typedef typename V2<T>::t T2;
        char* r = b->arena + f.region;
        const size_t es = elem_bytes(b);
        cudaStream_t ls = lattice_stream(op.cfg);
        gauge_first<T>(f.g, f.gp, f.p.msl, (const T2*)(r + 6 * f.D * es),
                       (const double*)(b->arena + f.gG), (const double*)(b->arena + f.gH),
                       (T*)(b->arena + f.gUh), (T*)(b->arena + f.gB), nullptr, ls);
        // the A lines of length 1 (they may overwrite the level store)
        gram_line_step<T>(f.g, f.gp, f.p.msl, 1, (const T*)(b->arena + f.gUh),
                          (const double*)(b->arena + f.gH), (T*)(b->arena + f.gB),
                          (T*)(b->arena + f.gA), ls);
        kernels += 2;
        break;
      }
      case OP_GRAM_R: {
        const Cfg& f = b->cfg[op.cfg];
        T* bl = (T*)(b->arena + f.gB);
        T* al = (T*)(b->arena + f.gA);
        cudaStream_t ls = lattice_stream(op.cfg);
        if (op.R >= 2) {
          gram_line_step<T>(f.g, f.gp, f.p.msl, op.R, (const T*)(b->arena + f.gUh),
                            (const double*)(b->arena + f.gH), bl, al, ls);
          kernels++;
        }
        gram_contract<T>(f.g, f.gp, f.p.mwlt, al, bl, (T*)(b->pbuf + f.gpartial), ls);
        gram_reduce<T>(f.g, f.gp, f.bc, f.p.mwlt, f.p.mwlr, op.R - 1,
                       (const T*)(b->pbuf + f.gpartial), (double*)(b->arena + f.wl), ls);
        kernels += 2;
        break;
      }
    }
  }
  return get_error()[0] ? -1 : kernels;
}

// contraction plans and partial-sum offsets (may change with the shape)
int plan(wlg_batch* b) {
  size_t poff = 0;
  const bool fp64 = b->prec == WLG_FP64;
  for (Cfg& f : b->cfg) {
    f.cp = contract_plan(f.g, f.p.msl, f.p.mwlt, fp64, b->tG, b->tNCB, b->tBlock);
    // batched forms: SB = 1 or 2 selects the third form, SB = 0 the fourth,
    // SB = 3 the fourth with its level loops unrolled (msl 4-6; the unrolled
    // FP64 kernel spills), SB = 4 the fourth with bulk-copy staging (the FP64
    // default where a time slice is whole 32-site tiles; lattices that are not
    // run the fourth form), SB 5 the unrolled fourth form with packed FP32
    // products, their signs in the shared broadcast pairs (the tenth form;
    // the FP32 default, as for a single lattice; an FP64 batch runs SB 3)
    f.cp.SB = b->tG ? b->tSB : (fp64 ? 4 : 5);
    if (f.cp.SB == 4 && !contract_can_bulk(f.g)) f.cp.SB = 0;
    if (f.cp.SB == 5 && fp64) f.cp.SB = 3;
    f.cp.variant = (f.cp.SB == 1 || f.cp.SB == 2) ? 3
                 : (f.cp.SB == 3 ? 5 : (f.cp.SB == 4 ? 7 : (f.cp.SB == 5 ? 10 : 4)));
    // the temporal-gauge form where it applies (phase 1 falls back to the
    // carried lines per lattice, so those get their partial sums too)
    f.gram = f.gram_ok && b->tG == 0;
    if (f.gram) {
      f.gpartial = poff;
      poff = align256(poff + f.gp.partial_elems * (fp64 ? 8 : 4));
    }
    if (f.cp.G > 4) {
      set_error("batch: contraction shape G=%d is not available in batched form", f.cp.G);
      return -1;
    }
    f.partial = poff;
    poff = align256(poff + f.cp.partial_doubles * sizeof(double));
  }
  b->pbuf_bytes = poff;
  return 0;
}

// field offsets in the arena (fixed for the life of the batch)
void layout(wlg_batch* b) {
  size_t off = 0, host = 0, maxv = 0;
  const bool fp64 = b->prec == WLG_FP64;
  for (Cfg& f : b->cfg) {
    f.D = fp64 ? link_elems<double>(f.g.vol) : link_elems<float>(f.g.vol);
    size_t es = elem_bytes(b);
    f.U = off;
    off = align256(off + 4 * f.D * es);
    f.U0 = off;
    off = align256(off + 4 * f.D * es);
    f.region = off;
    // APE ping-pong 6 + levels 3 msl + lines 3 msl + spatial-HYP scratch 6 +
    // second lines 3 msl, or the HYP scratch (24), whichever is larger
    size_t rdirs = std::max<size_t>(24, 12 + 9 * (size_t)f.p.msl);
    size_t rbytes = rdirs * f.D * es;
    f.gram_ok = f.p.proj_iter >= 3 && (long long)f.g.vol >= kGramMinSites &&
                gram_plan(f.gp, f.g, f.bc, f.p.msl, f.p.mwlt, fp64);
    if (f.gram_ok) {
      // after the smearing: g and H^-1 in the APE ping-pong slots (6 D),
      // Uh, B and A lines from the first line buffer on
      const size_t esz = fp64 ? 8 : 4, nb = 3 * (size_t)f.p.msl * f.gp.A * esz;
      const size_t gh = align256(f.gp.A * sizeof(double));
      const size_t lines_at = (6 + 3 * (size_t)f.p.msl) * f.D * es;
      size_t o = align256(lines_at);
      f.gUh = f.region + o;
      o = align256(o + nb);
      f.gB = f.region + o;
      o = align256(o + nb);
      // the A lines take the level store, dead once the first lines exist,
      // where they fit in it (they are written after it is read)
      const size_t na = 3 * (size_t)f.p.msl * f.gp.Aa * esz;
      if (na <= 3 * (size_t)f.p.msl * f.D * es) {
        f.gA = f.region + 6 * f.D * es;
      } else {
        f.gA = f.region + o;
        o = align256(o + na);
      }
      f.gDev = f.region + o;
      o = align256(o + 8);
      if (2 * gh <= 6 * f.D * es) {
        f.gG = f.region;
        f.gH = f.region + gh;
      } else {
        f.gG = f.region + o;
        o = align256(o + gh);
        f.gH = f.region + o;
        o = align256(o + gh);
      }
      rbytes = std::max(rbytes, o);
    }
    off = align256(off + rbytes);
    f.nwl = (size_t)f.p.msl * f.p.msl * f.p.mwlt * f.p.mwlr * f.g.n[0];
    f.wl = off;
    off = align256(off + f.nwl * sizeof(double));
    f.wl_host = host;
    host += f.nwl;
    maxv = std::max(maxv, (size_t)f.g.vol);
  }
  b->arena_bytes = off;
  b->wl_host_doubles = host;
  b->staging_bytes = maxv * 4 * 144;
}

template <class P>
int pool_alloc(wlg_batch* b, P** ptr, size_t bytes) {
  *ptr = nullptr;
  cudaMemPool_t pool = batch_pool(b->dev);
  if (!pool) return -1;
  void* p = nullptr;
  cudaError_t e = cudaMallocFromPoolAsync(&p, bytes, pool, b->st);
  if (e != cudaSuccess) {
    cudaGetLastError();
    cudaStreamSynchronize(b->st);
    cudaMemPoolTrimTo(pool, 0);
    e = cudaMallocFromPoolAsync(&p, bytes, pool, b->st);
    if (e != cudaSuccess) {
      cudaGetLastError();
      return -1;
    }
  }
  *ptr = static_cast<P*>(p);
  return 0;
}

template <class P>
void pool_free(wlg_batch* b, P*& ptr) {
  if (ptr) cudaFreeAsync(ptr, b->st);
  ptr = nullptr;
}

int ensure_pbuf(wlg_batch* b) {
  if (b->pbuf && b->pbuf_cap >= b->pbuf_bytes) return 0;
  pool_free(b, b->pbuf);
  b->pbuf_cap = 0;
  if (pool_alloc(b, &b->pbuf, std::max<size_t>(256, b->pbuf_bytes))) {
    set_error("batch: cannot allocate %zu bytes of partial sums", b->pbuf_bytes);
    return -1;
  }
  b->pbuf_cap = std::max<size_t>(256, b->pbuf_bytes);
  return 0;
}

int build(wlg_batch* b, int phase) {
  wlg_batch::Phase& P = b->ph[phase];
  if (P.built) return 0;
  if (phase == 1)
    for (size_t c = 0; c < b->cfg.size(); c++)
      if (c < b->use_gram.size() && b->use_gram[c] && gram_prepare(b->cfg[c].gp)) return -1;
  if (b->prec == WLG_FP64)
    build_ops<double>(b, phase);
  else
    build_ops<float>(b, phase);
  pool_free(b, P.tables);
  if (pool_alloc(b, &P.tables, std::max<size_t>(256, P.host_tables.size()))) {
    set_error("batch: cannot allocate the argument tables");
    return -1;
  }
  WLG_CUDA(cudaMemcpyAsync(P.tables, P.host_tables.data(), P.host_tables.size(),
                           cudaMemcpyHostToDevice, b->st));
  WLG_CUDA(cudaStreamSynchronize(b->st));  // host_tables may change after this
  P.built = true;
  return 0;
}

// capture one phase into a graph (nothing executes during capture)
int capture(wlg_batch* b, int phase) {
  wlg_batch::Phase& P = b->ph[phase];
  WLG_CUDA(cudaStreamBeginCapture(b->st, cudaStreamCaptureModeThreadLocal));
  int rc = b->prec == WLG_FP64 ? issue<double>(b, phase) : issue<float>(b, phase);
  cudaGraph_t g = nullptr;
  cudaError_t e = cudaStreamEndCapture(b->st, &g);
  if (rc < 0 || e != cudaSuccess) {
    if (g) cudaGraphDestroy(g);
    set_error("batch: graph capture failed: %s", cudaGetErrorString(e));
    cudaGetLastError();
    return -1;
  }
  P.graph = g;
  WLG_CUDA(cudaGraphInstantiate(&P.exec, g, 0));
  return 0;
}

void unbuild_phase(wlg_batch* b, int phase) {
  wlg_batch::Phase& P = b->ph[phase];
  if (P.exec) cudaGraphExecDestroy(P.exec);
  if (P.graph) cudaGraphDestroy(P.graph);
  pool_free(b, P.tables);
  P.exec = nullptr;
  P.graph = nullptr;
  P.built = false;
}

void unbuild(wlg_batch* b) {
  unbuild_phase(b, 0);
  unbuild_phase(b, 1);
}

// runs one phase: its graph, or its ops directly the first time (then
// captured); returns the kernels launched or -1
int run_phase(wlg_batch* b, int phase) {
  wlg_batch::Phase& P = b->ph[phase];
  if (build(b, phase)) return -1;
  if (P.exec) {
    WLG_CUDA(cudaGraphLaunch(P.exec, b->st));
  } else {
    const int k = b->prec == WLG_FP64 ? issue<double>(b, phase) : issue<float>(b, phase);
    if (k < 0) return -1;
    P.kernels = k;
  }
  return P.kernels;
}

}  // namespace

extern "C" {

int wlg_batch_create(int nconf, const int* dims, const int* bcs, const wlg_wloop_parms* parms,
                     int precision, int device, wlg_batch** out) {
  set_error("%s", "");
  if (nconf < 1 || !dims || !bcs || !parms || !out) {
    set_error("batch_create: bad arguments");
    return -1;
  }
  if (precision != WLG_FP64 && precision != WLG_MIXED) {
    set_error("batch_create: unknown precision");
    return -1;
  }
  if (wlg_device_count() <= device || device < 0) {
    set_error("batch_create: no CUDA device %d (no CPU fallback)", device);
    return -1;
  }
  WLG_CUDA(cudaSetDevice(device));
  wlg_batch* b = new wlg_batch();
  b->dev = device;
  b->prec = precision;
  for (int c = 0; c < nconf; c++) {
    Cfg f;
    memset(&f, 0, sizeof(f));
    if (check_lattice(dims + 4 * c, bcs[c])) {
      set_error("batch_create: lattice %d: an extent < 2, more than 2^30 sites, or a boundary "
                "condition other than 0 and 3", c);
      delete b;
      return -1;
    }
    f.g = make_geo(dims + 4 * c);
    f.bc = bcs[c];
    f.p = parms[c];
    if (check_parms(f.g, f.p)) {
      set_error("batch_create: configuration %d: bad boundary condition or parameters", c);
      delete b;
      return -1;
    }
    b->cfg.push_back(f);
  }
  layout(b);
  if (plan(b)) {
    delete b;
    return -1;
  }
  if (cudaStreamCreateWithFlags(&b->st, cudaStreamNonBlocking) != cudaSuccess || ensure_pbuf(b) ||
      pool_alloc(b, &b->arena, b->arena_bytes) || pool_alloc(b, &b->staging, b->staging_bytes) ||
      cudaMallocHost(&b->wl_host, b->wl_host_doubles * sizeof(double)) != cudaSuccess ||
      cudaMallocHost(&b->dev_host, nconf * sizeof(unsigned long long)) != cudaSuccess) {
    set_error("batch_create: cannot allocate %.2f GB arena: %s", b->arena_bytes / 1e9,
              cudaGetErrorString(cudaGetLastError()));
    wlg_batch_destroy(b);
    return -1;
  }
  // the allocations are ordered on the batch's stream; complete them before
  // the host hands the buffers to copies on other streams
  WLG_CUDA(cudaStreamSynchronize(b->st));
  for (int k = 0; k < wlg_batch::kSide; k++) {
    if (cudaStreamCreateWithFlags(&b->side[k], cudaStreamNonBlocking) != cudaSuccess ||
        cudaEventCreateWithFlags(&b->join[k], cudaEventDisableTiming) != cudaSuccess) {
      set_error("batch_create: cannot create the lattice streams");
      wlg_batch_destroy(b);
      return -1;
    }
  }
  if (cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess) {
    set_error("batch_create: cannot create the lattice streams");
    wlg_batch_destroy(b);
    return -1;
  }
  cudaEventCreate(&b->ev0);
  cudaEventCreate(&b->ev1);
  *out = b;
  return 0;
}

int wlg_batch_destroy(wlg_batch* b) {
  if (!b) return 0;
  cudaSetDevice(b->dev);
  if (b->st) {
    cudaStreamSynchronize(b->st);
    unbuild(b);
    pool_free(b, b->arena);
    pool_free(b, b->pbuf);
    pool_free(b, b->staging);
    cudaStreamSynchronize(b->st);  // the frees are ordered on the stream
  }
  if (b->wl_host) cudaFreeHost(b->wl_host);
  if (b->dev_host) cudaFreeHost(b->dev_host);
  if (b->ev0) cudaEventDestroy(b->ev0);
  if (b->ev1) cudaEventDestroy(b->ev1);
  for (int k = 0; k < wlg_batch::kSide; k++) {
    if (b->side[k]) {
      cudaStreamSynchronize(b->side[k]);
      cudaStreamDestroy(b->side[k]);
    }
    if (b->join[k]) cudaEventDestroy(b->join[k]);
  }
  if (b->fork) cudaEventDestroy(b->fork);
  if (b->st) cudaStreamDestroy(b->st);
  delete b;
  return 0;
}

}  // extern "C"

namespace wlg {
void batch_pool_trim(int dev) {
  if (dev < 0 || dev >= kMaxPoolDevices) return;
  cudaMemPool_t pool = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    pool = g_pool[dev];
  }
  if (pool) cudaMemPoolTrimTo(pool, 0);
}
}  // namespace wlg

extern "C" {

long long wlg_batch_pool_idle_bytes(int device) {
  cudaMemPool_t pool = batch_pool(device);
  if (!pool) return 0;
  uint64_t reserved = 0, used = 0;
  if (cudaMemPoolGetAttribute(pool, cudaMemPoolAttrReservedMemCurrent, &reserved) != cudaSuccess ||
      cudaMemPoolGetAttribute(pool, cudaMemPoolAttrUsedMemCurrent, &used) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return reserved > used ? (long long)(reserved - used) : 0;
}

int wlg_batch_size(wlg_batch* b) { return b ? (int)b->cfg.size() : 0; }

long long wlg_batch_bytes(wlg_batch* b) { return b ? (long long)b->arena_bytes : 0; }

int wlg_batch_upload(wlg_batch* b, int i, const double* aos) {
  set_error("%s", "");
  if (!b || i < 0 || i >= (int)b->cfg.size() || !aos) {
    set_error("batch_upload: bad arguments");
    return -1;
  }
  WLG_CUDA(cudaSetDevice(b->dev));
  const Cfg& f = b->cfg[i];
  size_t bytes = (size_t)4 * 144 * f.g.vol;
  WLG_CUDA(cudaMemcpyAsync(b->staging, aos, bytes, cudaMemcpyHostToDevice, b->st));
  if (b->prec == WLG_FP64)
    aos_to_soa<double>(f.g, (const double*)b->staging, lview<double>(b->arena + f.U, f.D, 4, 0), 0, 4,
                       b->st);
  else
    aos_to_soa<float>(f.g, (const double*)b->staging, lview<float>(b->arena + f.U, f.D, 4, 0), 0, 4,
                      b->st);
  WLG_CUDA(cudaStreamSynchronize(b->st));
  return get_error()[0] ? -1 : 0;
}

int wlg_batch_generate(wlg_batch* b, const uint64_t* seeds, const double* eps) {
  set_error("%s", "");
  if (!b || !seeds || !eps) {
    set_error("batch_generate: bad arguments");
    return -1;
  }
  WLG_CUDA(cudaSetDevice(b->dev));
  for (size_t c = 0; c < b->cfg.size(); c++) {
    const Cfg& f = b->cfg[c];
    if (b->prec == WLG_FP64)
      generate_soa<double>(f.g, f.bc, seeds[c], eps[c], lview<double>(b->arena + f.U, f.D, 4, 0),
                           b->st);
    else
      generate_soa<float>(f.g, f.bc, seeds[c], eps[c], lview<float>(b->arena + f.U, f.D, 4, 0),
                          b->st);
  }
  WLG_CUDA(cudaStreamSynchronize(b->st));
  return get_error()[0] ? -1 : 0;
}

int wlg_batch_snapshot(wlg_batch* b) {
  set_error("%s", "");
  WLG_CUDA(cudaSetDevice(b->dev));
  for (const Cfg& f : b->cfg)
    WLG_CUDA(cudaMemcpyAsync(b->arena + f.U0, b->arena + f.U, 4 * f.D * elem_bytes(b),
                             cudaMemcpyDeviceToDevice, b->st));
  WLG_CUDA(cudaStreamSynchronize(b->st));
  return 0;
}

int wlg_batch_restore(wlg_batch* b) {
  set_error("%s", "");
  WLG_CUDA(cudaSetDevice(b->dev));
  for (const Cfg& f : b->cfg)
    WLG_CUDA(cudaMemcpyAsync(b->arena + f.U, b->arena + f.U0, 4 * f.D * elem_bytes(b),
                             cudaMemcpyDeviceToDevice, b->st));
  return 0;
}

int wlg_batch_run(wlg_batch* b) {
  set_error("%s", "");
  if (!b) {
    set_error("batch_run: null batch");
    return -1;
  }
  WLG_CUDA(cudaSetDevice(b->dev));
  const size_t n = b->cfg.size();
  WLG_CUDA(cudaEventRecord(b->ev0, b->st));
  // phase 0: smearing and the gauge chains
  const int k0 = run_phase(b, 0);
  if (k0 < 0) return -1;
  const bool captured0 = b->ph[0].exec != nullptr;
  WLG_CUDA(cudaStreamSynchronize(b->st));
  // the temporal-gauge form for the lattices whose g is near unitary, the
  // carried lines for the others (the rule of a single context)
  std::vector<char> use(n, 0);
  for (size_t c = 0; c < n; c++) {
    if (!b->cfg[c].gram) continue;
    double dev;
    memcpy(&dev, b->dev_host + c, sizeof(dev));
    use[c] = dev <= kGramMaxDeviation;
  }
  if (use != b->use_gram) {
    unbuild_phase(b, 1);
    b->use_gram = use;
  }
  const int k1 = run_phase(b, 1);
  if (k1 < 0) return -1;
  const bool captured1 = b->ph[1].exec != nullptr;
  WLG_CUDA(cudaEventRecord(b->ev1, b->st));
  WLG_CUDA(cudaStreamSynchronize(b->st));
  cudaEventElapsedTime(&b->last_ms, b->ev0, b->ev1);
  b->kernels = k0 + k1;
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("batch_run: %s", cudaGetErrorString(e));
    return -1;
  }
  bool bulk = false;
  for (size_t c = 0; c < n; c++) bulk = bulk || (!b->use_gram[c] && b->cfg[c].cp.variant == 7);
  if (bulk && contract_stage_failed() != 0) {
    set_error("batch_run: the contraction's staged-line copies did not arrive in time");
    return -1;
  }
  // a phase that ran its ops directly is captured for the next runs
  if (b->use_graph && !captured0 && capture(b, 0)) return -1;
  if (b->use_graph && !captured1 && capture(b, 1)) return -1;
  return 0;
}

int wlg_batch_use_graph(wlg_batch* b, int on) {
  if (!b) return -1;
  b->use_graph = on != 0;
  return 0;
}

// device bytes a batch of these configurations would hold (no allocation)
long long wlg_batch_estimate_bytes(int nconf, const int* dims, const int* bcs,
                                   const wlg_wloop_parms* parms, int precision) {
  if (nconf < 1 || !dims || !bcs || !parms) return -1;
  if (precision != WLG_FP64 && precision != WLG_MIXED) return -1;
  wlg_batch tmp;
  tmp.prec = precision;
  for (int c = 0; c < nconf; c++) {
    Cfg f;
    memset(&f, 0, sizeof(f));
    if (check_lattice(dims + 4 * c, bcs[c])) return -1;
    f.g = make_geo(dims + 4 * c);
    f.bc = bcs[c];
    f.p = parms[c];
    if (check_parms(f.g, f.p)) return -1;
    tmp.cfg.push_back(f);
  }
  layout(&tmp);
  if (plan(&tmp)) return -1;
  return (long long)(tmp.arena_bytes + tmp.pbuf_bytes + tmp.staging_bytes + (1 << 20));
}

int wlg_batch_result(wlg_batch* b, int i, double* wl_mat) {
  set_error("%s", "");
  if (!b || i < 0 || i >= (int)b->cfg.size() || !wl_mat) {
    set_error("batch_result: bad arguments");
    return -1;
  }
  const Cfg& f = b->cfg[i];
  memcpy(wl_mat, b->wl_host + f.wl_host, f.nwl * sizeof(double));
  return 0;
}

int wlg_batch_stats(wlg_batch* b, double* last_ms, int* kernels_per_run) {
  if (!b) return -1;
  if (last_ms) *last_ms = b->last_ms;
  if (kernels_per_run) *kernels_per_run = b->kernels;
  return 0;
}

void* wlg_batch_stream(wlg_batch* b) { return b ? (void*)b->st : nullptr; }

int wlg_batch_set_contract_shape(wlg_batch* b, int G, int SB, int nCB, int block) {
  set_error("%s", "");
  if (!b || G < 0 || G > 4 || SB < 0 || SB > 5 || nCB < 0 ||
      (block != 0 && (block % 32 != 0 || block > 128))) {
    set_error("batch_set_contract_shape: bad shape");
    return -1;
  }
  WLG_CUDA(cudaSetDevice(b->dev));
  WLG_CUDA(cudaStreamSynchronize(b->st));
  b->tG = G;
  b->tSB = SB;
  b->tNCB = nCB;
  b->tBlock = block;
  unbuild(b);
  if (plan(b) || ensure_pbuf(b)) return -1;
  return 0;
}

}  // extern "C"
