// legacy.cpp -- the reference's C entry points (include/lnk.h, include/smear.h,
// include/wloop.h of bjoern-leder/wloop at NPROC = 1) over the wlg_* C ABI.
//
// State that the reference keeps file-static in each module (hyp_links.c:68-73,
// ape_links.c, smear.c:40-42, wloop.c:62-67, wloop_parms.c:91-93) lives in one
// process-global record here; the caller's geometry and gauge field arrive
// through wloop_b200_attach().  Every smearing and loop computation runs on
// the GPU in FP64; host code here only moves links between the openQCD layout
// and the device, resolves link addresses (lnk, lnkf, lnk_plaq) and handles
// parameters and files.  Errors end the process with a message on stderr, as
// error_root() does in the reference.
#include <float.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <set>
#include <string>
#include <vector>

#include "../../include/wloop_b200.h"
#include "../../include/wloop_b200_legacy.h"

namespace {

struct State {
  bool attached = false;
  int n[4] = {0, 0, 0, 0};
  int vol = 0;
  int bc = 3;
  std::vector<int> ipt;  // lexicographic -> openQCD index
  std::vector<int> iup;  // [openQCD index][mu] -> openQCD index of x+mu
  std::vector<int> idn;
  su3_dble* (*udfld)(void) = nullptr;
  wlg_ctx* ctx = nullptr;
  wloop_parms_t wl;
  bool have_parms = false;
  std::vector<double> wlm;
  std::vector<su3_dble> usb;  // host copy of the level store for get_pus()
  std::vector<su3_dble*> pus;
  bool pus_valid = false;
  std::set<su3_dble*> lnks;
};

State S;

[[noreturn]] void fatal(const char* program, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  fprintf(stderr, "\nError in %s:\n", program);
  vfprintf(stderr, fmt, ap);
  fprintf(stderr, "\nProgram aborted\n\n");
  va_end(ap);
  fflush(stderr);
  exit(1);
}

void need_attach(const char* who) {
  if (!S.attached) fatal(who, "wloop_b200_attach() has not been called");
}

wlg_ctx* ctx(const char* who) {
  need_attach(who);
  if (!S.ctx && wlg_create(S.n, S.bc, WLG_FP64, 0, &S.ctx)) fatal(who, "%s", wlg_last_error());
  return S.ctx;
}

void check(int rc, const char* who) {
  if (rc) fatal(who, "%s", wlg_last_error());
}

// offset of U(ix,mu) in an openQCD link field (ofs_lnk, lnkcom.c:840-859, NPROC = 1)
int ofs_lnk(int ix, int mu) {
  const int h = S.vol / 2;
  if (ix < h) return 8 * (S.iup[4 * ix + mu] - h) + 2 * mu + 1;
  return 8 * (ix - h) + 2 * mu;
}

void upload(su3_dble* ub, const char* who) {
  check(wlg_upload_openqcd(ctx(who), reinterpret_cast<double*>(ub), S.ipt.data()), who);
}

void download(su3_dble* ub, const char* who) {
  check(wlg_download_openqcd(ctx(who), reinterpret_cast<double*>(ub), S.ipt.data()), who);
}

// openQCD layout <-> AoS lexicographic [V][4] (host index shuffles only)
void to_aos(const su3_dble* ub, std::vector<su3_dble>& aos) {
  aos.resize(4 * (size_t)S.vol);
  for (int s = 0; s < S.vol; s++)
    for (int mu = 0; mu < 4; mu++) aos[4 * (size_t)s + mu] = ub[ofs_lnk(S.ipt[s], mu)];
}

void from_aos(const std::vector<su3_dble>& aos, su3_dble* ub) {
  for (int s = 0; s < S.vol; s++)
    for (int mu = 0; mu < 4; mu++) ub[ofs_lnk(S.ipt[s], mu)] = aos[4 * (size_t)s + mu];
}

wlg_wloop_parms to_c(const wloop_parms_t& w) {
  wlg_wloop_parms p;
  memset(&p, 0, sizeof(p));
  p.msl = w.msl;
  for (int i = 0; i < w.msl && i < WLG_MAX_SM_LEVELS; i++) p.nss[i] = w.nss[i];
  p.mwlt = w.mwlt;
  p.mwlr = w.mwlr;
  p.op_smear = (w.op_smear == HYP) ? WLG_OP_HYP : WLG_OP_APE;
  for (int i = 0; i < 3; i++) p.alpha_action[i] = w.alpha_action[i];
  p.alpha_ape = w.alpha_ape;
  p.alpha_hyp[0] = w.alpha_hyp[0];
  p.alpha_hyp[1] = w.alpha_hyp[1];
  p.proj_iter = w.proj_iter;
  return p;
}

void need_parms(const char* who) {
  if (!S.have_parms) fatal(who, "wloop parameters are not set (set_wloop_parms / read_wloop_parms)");
}

// number of decimals that print x exactly enough (openQCD fdigits semantics)
int fdigits(double x) {
  for (int n = 0; n < 16; n++) {
    double p = pow(10.0, n);
    if (fabs(round(x * p) / p - x) <= DBL_EPSILON * fabs(x)) return n;
  }
  return 16;
}

// ---- [Wloop] input section (openQCD find_section / read_line semantics) ----
struct Input {
  std::vector<std::string> lines;
  size_t begin = 0, end = 0;
};

Input read_stdin_section(const char* title) {
  Input in;
  std::string all;
  if (fseek(stdin, 0L, SEEK_SET) != 0) clearerr(stdin);
  char buf[4096];
  size_t k;
  while ((k = fread(buf, 1, sizeof(buf), stdin)) > 0) all.append(buf, k);
  size_t pos = 0;
  while (pos <= all.size()) {
    size_t e = all.find('\n', pos);
    if (e == std::string::npos) e = all.size();
    in.lines.push_back(all.substr(pos, e - pos));
    pos = e + 1;
  }
  std::string want = std::string("[") + title + "]";
  int found = 0;
  for (size_t i = 0; i < in.lines.size(); i++) {
    const char* l = in.lines[i].c_str();
    while (*l == ' ' || *l == '\t') l++;
    if (strncmp(l, want.c_str(), want.size()) == 0) {
      found++;
      in.begin = i + 1;
    }
  }
  if (found != 1)
    fatal("find_section [wloop_b200]", "Section [%s] not found or not unique", title);
  in.end = in.begin;
  while (in.end < in.lines.size()) {
    const char* l = in.lines[in.end].c_str();
    while (*l == ' ' || *l == '\t') l++;
    if (*l == '[') break;
    in.end++;
  }
  return in;
}

// values after `tag` in the section; empty if the tag is absent
std::vector<std::string> find_tag(const Input& in, const char* tag) {
  std::vector<std::string> out;
  for (size_t i = in.begin; i < in.end; i++) {
    char line[4096];
    snprintf(line, sizeof(line), "%s", in.lines[i].c_str());
    char* save = nullptr;
    char* tok = strtok_r(line, " \t\r", &save);
    if (!tok || tok[0] == '#' || strcmp(tok, tag) != 0) continue;
    while ((tok = strtok_r(nullptr, " \t\r", &save)) != nullptr) {
      if (tok[0] == '#') break;
      out.push_back(tok);
    }
    return out;
  }
  return out;
}

std::vector<std::string> need_tag(const Input& in, const char* tag, size_t n) {
  std::vector<std::string> v = find_tag(in, tag);
  if (v.size() < n) fatal("read_line [wloop_b200]", "Missing or incomplete data line \"%s\"", tag);
  return v;
}

void invalidate_levels() { S.pus_valid = false; }

}  // namespace

extern "C" {

// ---------------------------------------------------------------------------
// attach
// ---------------------------------------------------------------------------
void wloop_b200_attach(const int n[4], int bc, const int* ipt, su3_dble* (*udfld_fn)(void)) {
  const char* who = "wloop_b200_attach";
  if (!n || !ipt || !udfld_fn) fatal(who, "null argument");
  for (int i = 0; i < 4; i++)
    if (n[i] < 2 || (n[i] & 1)) fatal(who, "lattice extents must be even and >= 2");
  if (bc != 0 && bc != 3) fatal(who, "only open (0) and periodic (3) boundary conditions");
  if (S.ctx) {
    wlg_destroy(S.ctx);
    S.ctx = nullptr;
  }
  memcpy(S.n, n, sizeof(S.n));
  S.vol = n[0] * n[1] * n[2] * n[3];
  S.bc = bc;
  S.ipt.assign(ipt, ipt + S.vol);
  std::vector<int> seen(S.vol, 0);
  for (int s = 0; s < S.vol; s++) {
    if (ipt[s] < 0 || ipt[s] >= S.vol || seen[ipt[s]]) fatal(who, "ipt is not a permutation");
    seen[ipt[s]] = 1;
  }
  S.iup.assign(4 * (size_t)S.vol, 0);
  S.idn.assign(4 * (size_t)S.vol, 0);
  const int st[4] = {n[1] * n[2] * n[3], n[2] * n[3], n[3], 1};
  for (int s = 0; s < S.vol; s++) {
    int x[4], r = s;
    for (int mu = 0; mu < 4; mu++) {
      x[mu] = r / st[mu];
      r -= x[mu] * st[mu];
    }
    for (int mu = 0; mu < 4; mu++) {
      int up = s + ((x[mu] == n[mu] - 1) ? -(n[mu] - 1) * st[mu] : st[mu]);
      int dn = s + ((x[mu] == 0) ? (n[mu] - 1) * st[mu] : -st[mu]);
      S.iup[4 * (size_t)ipt[s] + mu] = ipt[up];
      S.idn[4 * (size_t)ipt[s] + mu] = ipt[dn];
    }
  }
  S.udfld = udfld_fn;
  S.attached = true;
  invalidate_levels();
}

void wloop_b200_detach(void) {
  if (S.ctx) wlg_destroy(S.ctx);
  S.ctx = nullptr;
  S.attached = false;
  S.pus.clear();
  S.usb.clear();
}

// ---------------------------------------------------------------------------
// include/smear.h
// ---------------------------------------------------------------------------
static void hyp_dirs(double a1, double a2, double a3, int proj, int piter, int mu0, int mu1,
                     int keep, const char* who) {
  need_attach(who);
  if (a1 == 0.0) return;  // hyp_links.c:405
  su3_dble* ud = S.udfld();
  upload(ud, who);
  check(wlg_hyp(ctx(who), a1, a2, a3, proj, piter, mu0, mu1, keep), who);
  download(ud, who);
}

void hyp_links(double a1, double a2, double a3, int proj_su3, int piter, int keep) {
  hyp_dirs(a1, a2, a3, proj_su3, piter, 0, 4, keep, "hyp_links [hyp_links.c]");
}
void hyp_time_links(double a1, double a2, double a3, int proj_su3, int piter, int keep) {
  hyp_dirs(a1, a2, a3, proj_su3, piter, 0, 1, keep, "hyp_time_links [hyp_links.c]");
}
void hyp_space_links(double a1, double a2, double a3, int proj_su3, int piter, int keep) {
  hyp_dirs(a1, a2, a3, proj_su3, piter, 1, 4, keep, "hyp_space_links [hyp_links.c]");
}

void free_hyp(void) {
  if (S.ctx) wlg_free_scratch(S.ctx);
}
void free_ape_links(void) {
  if (S.ctx) wlg_free_scratch(S.ctx);
}
void free_hyp_spatial(void) {
  if (S.ctx) wlg_free_scratch(S.ctx);
}

static void ape_any(su3_dble* ub, double a, int proj, int piter, int time, int keep,
                    const char* who) {
  upload(ub, who);
  check(wlg_ape(ctx(who), a, proj, piter, time, 1, keep), who);
  download(ub, who);
}

void ape_links(su3_dble* ub, double a, int proj_su3, int piter, int keep) {
  ape_any(ub, a, proj_su3, piter, 1, keep, "ape_links [ape_links.c]");
}
void ape_spatial_links(su3_dble* ub, double a, int proj_su3, int piter, int keep) {
  ape_any(ub, a, proj_su3, piter, 0, keep, "ape_spatial_links [ape_links.c]");
}

void hyp_spatial_links(su3_dble* ub, double a1, double a2, int proj_su3, int piter, int keep) {
  const char* who = "hyp_spatial_links [hyp_spatial_links.c]";
  upload(ub, who);
  check(wlg_hyp_spatial(ctx(who), a1, a2, proj_su3, piter, 1, keep), who);
  download(ub, who);
}

void staple_sum(su3_dble* u1, su3_dble* u2, int mu, int nu, su3_dble* vb, su3_dble* cbuf) {
  const char* who = "staple_sum [staple_sum.c]";
  (void)cbuf;  // boundary buffer: empty at NPROC = 1
  need_attach(who);
  std::vector<su3_dble> a1, a2, av;
  to_aos(u1, a1);
  to_aos(u2, a2);
  to_aos(vb, av);
  check(wlg_staple_sum(S.n, reinterpret_cast<const double*>(a1.data()),
                       reinterpret_cast<const double*>(a2.data()), mu, nu,
                       reinterpret_cast<double*>(av.data())),
        who);
  from_aos(av, vb);
}

void approx_project_to_su3_dble(su3_dble* u, int iter) {
  check(wlg_project(reinterpret_cast<double*>(u), 1, iter),
        "approx_project_to_su3_dble [projection.c]");
}

// ---------------------------------------------------------------------------
// include/lnk.h
// ---------------------------------------------------------------------------
void copy_bnd(su3_dble*) {}
void copy_u0(su3_dble*) {}
void copyback_u0(su3_dble*) {}
void copy_u0n(su3_dble*) {}
void copyback_u0n(su3_dble*) {}
void copy_uk(su3_dble*) {}
void copyback_uk(su3_dble*) {}
void send_uk(su3_dble*, su3_dble*) {}

su3_dble* alloc_lnk(void) {
  need_attach("alloc_lnk [lnkcom.c]");
  void* p = nullptr;
  if (posix_memalign(&p, 64, 4 * (size_t)S.vol * sizeof(su3_dble)) != 0 || !p)
    fatal("alloc_lnk [lnkcom.c]", "Unable to allocate memory for link field");
  memset(p, 0, 4 * (size_t)S.vol * sizeof(su3_dble));
  S.lnks.insert((su3_dble*)p);
  return (su3_dble*)p;
}

void free_lnk(su3_dble* ub, int cb) {
  (void)cb;
  auto it = S.lnks.find(ub);
  if (it != S.lnks.end()) {
    free(ub);
    S.lnks.erase(it);
  }
}

su3_dble* alloc_buf_uk(void) { return nullptr; }  // lnkcom.c:785-802: NULL at NPROC = 1
void free_buf_uk(su3_dble*) {}
su3_dble* lnk_buf(su3_dble*, int, int, int) { return nullptr; }

su3_dble* lnk(su3_dble* ub, int ix, int mu) {
  need_attach("lnk [lnkcom.c]");
  return ub + ofs_lnk(ix, mu);
}

su3_dble* lnkf(su3_dble* ub, int ix, int mu, int face) {
  (void)face;  // ix < VOLUME always at NPROC = 1
  return lnk(ub, ix, mu);
}

void lnk_plaq(su3_dble* ub, int ix, int mu, int nu, su3_dble** u) {
  need_attach("lnk_plaq [lnkcom.c]");
  u[0] = lnk(ub, ix, mu);
  u[1] = lnkf(ub, S.iup[4 * (size_t)ix + mu], nu, mu);
  u[2] = lnk(ub, ix, nu);
  u[3] = lnkf(ub, S.iup[4 * (size_t)ix + nu], mu, nu);
}

void assign_lnk2lnk(su3_dble* ub1, su3_dble* ub2) {
  need_attach("assign_lnk2lnk [lnkcom.c]");
  memcpy(ub2, ub1, 4 * (size_t)S.vol * sizeof(su3_dble));
}
void assign_ud2lnk(su3_dble* ub) {
  need_attach("assign_ud2lnk [lnkcom.c]");
  memcpy(ub, S.udfld(), 4 * (size_t)S.vol * sizeof(su3_dble));
}
void assign_lnk2ud(su3_dble* ub) {
  need_attach("assign_lnk2ud [lnkcom.c]");
  memcpy(S.udfld(), ub, 4 * (size_t)S.vol * sizeof(su3_dble));
}

int* get_lnk_idx_u0(void) { return nullptr; }
int* get_lnk_idx_uk(void) { return nullptr; }

static void one_staple(su3_dble* u1, su3_dble* u2, su3_dble* u3, su3_dble* v, int dn, int save,
                       const char* who) {
  check(wlg_staples(1, reinterpret_cast<const double*>(u1), reinterpret_cast<const double*>(u2),
                    reinterpret_cast<const double*>(u3), reinterpret_cast<double*>(v), dn, save),
        who);
}

// link triples of lnkstaple.c:259-293 / :340-382
static void up_links(su3_dble* u1o, su3_dble* u2o, int ix, int mu, int nu, su3_dble** u) {
  u[0] = lnk(u1o, ix, nu);
  u[1] = lnkf(u2o, S.iup[4 * (size_t)ix + nu], mu, nu);
  u[2] = lnkf(u1o, S.iup[4 * (size_t)ix + mu], nu, mu);
}
static void dn_links(su3_dble* u1o, su3_dble* u2o, int ix, int mu, int nu, su3_dble** u) {
  int iy = S.idn[4 * (size_t)ix + nu];
  u[0] = lnk(u1o, iy, nu);
  u[1] = lnk(u2o, iy, mu);
  u[2] = lnkf(u1o, S.iup[4 * (size_t)iy + mu], nu, mu);
}

void add_up_staple(su3_dble* u1o, su3_dble* u2o, int ix, int mu, int nu, su3_dble* v) {
  su3_dble* u[3];
  need_attach("add_up_staple [lnkstaple.c]");
  up_links(u1o, u2o, ix, mu, nu, u);
  one_staple(u[0], u[1], u[2], v, 0, 0, "add_up_staple [lnkstaple.c]");
}
void add_dn_staple(su3_dble* u1o, su3_dble* u2o, int ix, int mu, int nu, su3_dble* v) {
  su3_dble* u[3];
  need_attach("add_dn_staple [lnkstaple.c]");
  dn_links(u1o, u2o, ix, mu, nu, u);
  one_staple(u[0], u[1], u[2], v, 1, 0, "add_dn_staple [lnkstaple.c]");
}
void add_up_staple_save(su3_dble* u1o, su3_dble* u2o, int ix, int mu, int nu, su3_dble* v) {
  su3_dble* u[3];
  need_attach("add_up_staple_save [lnkstaple.c]");
  up_links(u1o, u2o, ix, mu, nu, u);
  one_staple(u[0], u[1], u[2], v, 0, 1, "add_up_staple_save [lnkstaple.c]");
}
void add_dn_staple_save(su3_dble* u1o, su3_dble* u2o, int ix, int mu, int nu, su3_dble* v) {
  su3_dble* u[3];
  need_attach("add_dn_staple_save [lnkstaple.c]");
  dn_links(u1o, u2o, ix, mu, nu, u);
  one_staple(u[0], u[1], u[2], v, 1, 1, "add_dn_staple_save [lnkstaple.c]");
}
void add_up_staple_lnks(su3_dble* u1, su3_dble* u2, su3_dble* u3, su3_dble* v) {
  one_staple(u1, u2, u3, v, 0, 0, "add_up_staple_lnks [lnkstaple.c]");
}
void add_dn_staple_lnks(su3_dble* u1, su3_dble* u2, su3_dble* u3, su3_dble* v) {
  one_staple(u1, u2, u3, v, 1, 0, "add_dn_staple_lnks [lnkstaple.c]");
}
void add_up_staple_lnks_save(su3_dble* u1, su3_dble* u2, su3_dble* u3, su3_dble* v) {
  one_staple(u1, u2, u3, v, 0, 1, "add_up_staple_lnks_save [lnkstaple.c]");
}
void add_dn_staple_lnks_save(su3_dble* u1, su3_dble* u2, su3_dble* u3, su3_dble* v) {
  one_staple(u1, u2, u3, v, 1, 1, "add_dn_staple_lnks_save [lnkstaple.c]");
}

double lnk_plaq_sum(su3_dble* ub) {
  const char* who = "lnk_plaq_sum [lnkplaq.c]";
  double p = 0.0;
  upload(ub, who);
  check(wlg_plaq_sum(ctx(who), &p), who);
  return p;
}

// ---------------------------------------------------------------------------
// include/wloop.h
// ---------------------------------------------------------------------------
wloop_parms_t set_wloop_parms(int msl, int nss[], int mwlt, int mwlr, op_smear_t op_smear,
                              double alpha_action[3], double alpha_ape, double alpha_hyp[2],
                              int proj_iter) {
  const char* who = "set_wloop_parms [wloop_parms.c]";
  need_attach(who);
  if (op_smear != APE && op_smear != HYP) fatal(who, "Unknown type of operator smearing");
  if (msl < 1 || msl > MAX_SM_LEVELS) fatal(who, "max smearing level out of range");
  wloop_parms_t w;
  memset(&w, 0, sizeof(w));
  w.msl = msl;
  for (int k = 0; k < msl; k++) w.nss[k] = nss[k];
  w.alpha_ape = alpha_ape;
  w.alpha_hyp[0] = alpha_hyp[0];
  w.alpha_hyp[1] = alpha_hyp[1];
  for (int k = 0; k < 3; k++) w.alpha_action[k] = alpha_action[k];
  w.proj = (proj_iter > 0);
  w.proj_iter = proj_iter;
  if (mwlt < 1 || mwlt > S.n[0] / 2 + 1) fatal(who, "max wloop time extension out of range");
  if (mwlr < 1 || mwlr > S.n[1] / 2 + 1 || mwlr > S.n[2] / 2 + 1 || mwlr > S.n[3] / 2 + 1)
    fatal(who, "max wloop spatial extension out of range");
  w.mwlt = mwlt;
  w.mwlr = mwlr;
  w.op_smear = op_smear;
  w.wls = w.msl * w.msl * w.mwlt * w.mwlr * S.n[0];
  S.wlm.assign(w.wls, 1.0);  // wloop_parms.c:188-189
  w.wl_mat = S.wlm.data();
  S.wl = w;
  S.have_parms = true;
  invalidate_levels();
  return S.wl;
}

wloop_parms_t wloop_parms(void) { return S.wl; }

int wl_idx(int sl1, int sl2, int t, int r, int x0) {
  return sl1 + S.wl.msl * (sl2 + S.wl.msl * (t + S.wl.mwlt * (r + S.wl.mwlr * x0)));
}

void read_wloop_parms(void) {
  Input in = read_stdin_section("Wloop");
  std::vector<std::string> v = need_tag(in, "op_smear", 1);
  op_smear_t op = OP_SMEARS;
  if (v[0] == "APE")
    op = APE;
  else if (v[0] == "HYP")
    op = HYP;
  else
    fatal("read_wloop_parms [wloop_parms.c]", "Unknown operator smearing %s", v[0].c_str());
  int mwlt = atoi(need_tag(in, "mwlt", 1)[0].c_str());
  int mwlr = atoi(need_tag(in, "mwlr", 1)[0].c_str());
  int proj_iter = atoi(need_tag(in, "proj_iter", 1)[0].c_str());
  std::vector<std::string> aa = need_tag(in, "alpha_action", 3);
  double alpha_action[3] = {atof(aa[0].c_str()), atof(aa[1].c_str()), atof(aa[2].c_str())};
  int msl = atoi(need_tag(in, "msl", 1)[0].c_str());
  if (msl < 1 || msl > MAX_SM_LEVELS)
    fatal("read_wloop_parms [wloop_parms.c]", "max smearing level out of range");
  std::vector<std::string> ns = need_tag(in, "nss", (size_t)msl);
  int nss[MAX_SM_LEVELS] = {0};
  for (int i = 0; i < msl; i++) nss[i] = atoi(ns[i].c_str());
  double alpha_ape = 0.0, alpha_hyp[2] = {0.0, 0.0};
  if (op == APE) alpha_ape = atof(need_tag(in, "alpha", 1)[0].c_str());
  if (op == HYP) {
    std::vector<std::string> ah = need_tag(in, "alpha", 2);
    alpha_hyp[0] = atof(ah[0].c_str());
    alpha_hyp[1] = atof(ah[1].c_str());
  }
  set_wloop_parms(msl, nss, mwlt, mwlr, op, alpha_action, alpha_ape, alpha_hyp, proj_iter);
}

void print_wloop_parms(void) {
  const wloop_parms_t& w = S.wl;
  printf("Wloop parameters:\n");
  printf("msl = %d\n", w.msl);
  printf("nss =");
  for (int i = 0; i < w.msl; i++) printf(" %d", w.nss[i]);
  printf("\n");
  printf("mwlt = %d\n", w.mwlt);
  printf("mwlr = %d\n", w.mwlr);
  printf("alpha_action =");
  for (int i = 0; i < 3; i++) {
    int n = fdigits(w.alpha_action[i]);
    printf(" %.*f", n > 1 ? n : 1, w.alpha_action[i]);
  }
  printf("\n");
  printf("proj_iter = %d\n", w.proj_iter);
  printf("operator smearing = ");
  if (w.op_smear == APE) {
    int n = fdigits(w.alpha_ape);
    printf("APE\n");
    printf("alpha = %.*f\n", n > 1 ? n : 1, w.alpha_ape);
  } else if (w.op_smear == HYP) {
    printf("HYP\n");
    printf("alpha =");
    for (int i = 0; i < 2; i++) {
      int n = fdigits(w.alpha_hyp[i]);
      printf(" %.*f", n > 1 ? n : 1, w.alpha_hyp[i]);
    }
    printf("\n");
  }
  printf("\n");
}

// int32 little-endian record of wloop_parms.c:343-382
void write_wloop_parms(FILE* fdat) {
  const char* who = "write_wloop_parms [wloop_parms.c]";
  need_parms(who);
  const wloop_parms_t& w = S.wl;
  int32_t istd[MAX_SM_LEVELS + 4];
  double dstd[6];
  for (int i = 0; i < w.msl; i++) istd[i] = (int32_t)w.nss[i];
  istd[w.msl + 0] = w.mwlt;
  istd[w.msl + 1] = w.mwlr;
  istd[w.msl + 2] = (int32_t)w.op_smear;
  istd[w.msl + 3] = w.proj_iter;
  dstd[0] = w.alpha_ape;
  dstd[1] = w.alpha_hyp[0];
  dstd[2] = w.alpha_hyp[1];
  dstd[3] = w.alpha_action[0];
  dstd[4] = w.alpha_action[1];
  dstd[5] = w.alpha_action[2];
  size_t iw = fwrite(istd, sizeof(int32_t), w.msl + 4, fdat);
  iw += fwrite(dstd, sizeof(double), 6, fdat);
  if (iw != (size_t)(w.msl + 10)) fatal(who, "Incorrect write count");
}

void check_wloop_parms(FILE* fdat) {
  const char* who = "check_wloop_parms [wloop_parms.c]";
  need_parms(who);
  const wloop_parms_t& w = S.wl;
  int32_t istd[MAX_SM_LEVELS + 4];
  double dstd[6];
  size_t ir = fread(istd, sizeof(int32_t), w.msl + 4, fdat);
  ir += fread(dstd, sizeof(double), 6, fdat);
  if (ir != (size_t)(w.msl + 10)) fatal(who, "Incorrect read count");
  int ie = 0;
  for (int i = 0; i < w.msl; i++) ie |= (istd[i] != w.nss[i]);
  ie |= (istd[w.msl + 0] != w.mwlt);
  ie |= (istd[w.msl + 1] != w.mwlr);
  ie |= (istd[w.msl + 2] != (int32_t)w.op_smear);
  ie |= (istd[w.msl + 3] != w.proj_iter);
  ie |= (dstd[0] != w.alpha_ape);
  ie |= (dstd[1] != w.alpha_hyp[0]);
  ie |= (dstd[2] != w.alpha_hyp[1]);
  ie |= (dstd[3] != w.alpha_action[0]);
  ie |= (dstd[4] != w.alpha_action[1]);
  ie |= (dstd[5] != w.alpha_action[2]);
  if (ie) fatal(who, "Parameters do not match");
}

void smear(void) {
  const char* who = "smear [smear.c]";
  need_parms(who);
  wlg_wloop_parms p = to_c(S.wl);
  upload(S.udfld(), who);
  check(wlg_smear_levels(ctx(who), &p, nullptr), who);
  invalidate_levels();
}

su3_dble** get_pus(void) {
  const char* who = "get_pus [smear.c]";
  need_parms(who);
  if (!S.ctx) return nullptr;
  if (!S.pus_valid) {
    const int msl = S.wl.msl, V = S.vol;
    // usb: [slot][lexicographic site][k], 2 msl slots (smear.c:45-76)
    S.usb.assign((size_t)2 * msl * V * 3, su3_dble());
    S.pus.assign((size_t)2 * msl * V * 3, nullptr);
    std::vector<su3_dble> tmp((size_t)V * 3);
    for (int sl = 0; sl < msl; sl++) {
      check(wlg_download_level(S.ctx, sl, reinterpret_cast<double*>(tmp.data())), who);
      memcpy(&S.usb[(size_t)sl * V * 3], tmp.data(), tmp.size() * sizeof(su3_dble));
      int len = 0;
      if (wlg_download_lines(S.ctx, sl, reinterpret_cast<double*>(tmp.data()), &len) == 0)
        memcpy(&S.usb[(size_t)(msl + sl) * V * 3], tmp.data(), tmp.size() * sizeof(su3_dble));
    }
    for (int sl = 0; sl < 2 * msl; sl++)
      for (int s = 0; s < V; s++)
        for (int k = 0; k < 3; k++)  // pindx(sl,ix,k) = k + 3*(ix + VOLUME*sl), ix = ipt[s]
          S.pus[k + 3 * ((size_t)S.ipt[s] + (size_t)V * sl)] = &S.usb[((size_t)sl * V + s) * 3 + k];
    S.pus_valid = true;
  }
  return S.pus.data();
}

void free_smear(void) {
  S.usb.clear();
  S.pus.clear();
  S.pus_valid = false;
  if (S.ctx) wlg_free_scratch(S.ctx);
}

void wloop_sum(int keep) {
  const char* who = "wloop_sum [wloop.c]";
  need_parms(who);
  wlg_wloop_parms p = to_c(S.wl);
  upload(S.udfld(), who);
  check(wlg_wloop_sum(ctx(who), &p, S.wlm.data(), nullptr), who);
  invalidate_levels();
  // keep: as in the reference, the level store stays readable through
  // get_pus() either way (free_wloop does not free it, wloop.c:511-521);
  // device scratch is released by free_wloop / free_smear.
  (void)keep;
}

void free_wloop(void) {
  if (S.ctx) wlg_free_scratch(S.ctx);
}

}  // extern "C"
