// datfile.cpp -- the measurement program's binary output files.
//
// .dat (main/ms10.c:86-190): a head of 5 int32 {wls, msl, mwlt, mwlr, tmax}
// followed by one record per configuration, int32 nc and wls doubles (the
// wl_mat of that configuration, index wl_idx), all little-endian whatever the
// host byte order (ms10 swaps on big-endian hosts).
// .par, wloop part (wloop_parms.c:343-382): msl+4 int32 {nss[0..msl-1], mwlt,
// mwlr, op_smear, proj_iter} then 6 doubles {alpha_ape, alpha_hyp[0..1],
// alpha_action[0..2]}.
// .par, boundary-condition part, which precedes the wloop part (ms10 calls
// openQCD-1.4's write_bc_parms / check_bc_parms first, main/ms10.c:290-295):
// one int32 bc type then 10 doubles {cG, cG', cF, cF', phi[0..2],
// phi'[0..2]}.  ms10 passes cG = cG' = cF = cF' = 1 (ms10.c:290), and the
// phi angles are zero for open (0) and periodic (3) boundary conditions, the
// two types this library measures.  openQCD's flags/lat_parms.c is not
// vendored with the reference: the record is restated from openQCD-1.4's
// published parameter-file format and is not pinned by any file here.
#include <stdarg.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

#include "../../include/wloop_b200.h"

namespace {

thread_local std::string g_err;

int fail(const char* fmt, ...) {
  char buf[512];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_err = buf;
  return -1;
}

bool big_endian() {
  const uint16_t one = 1;
  unsigned char c;
  memcpy(&c, &one, 1);
  return c == 0;
}

template <class T>
void to_le(T* v, size_t n) {
  if (!big_endian()) return;
  for (size_t i = 0; i < n; i++) {
    unsigned char b[sizeof(T)];
    memcpy(b, &v[i], sizeof(T));
    for (size_t k = 0; k < sizeof(T) / 2; k++) {
      unsigned char t = b[k];
      b[k] = b[sizeof(T) - 1 - k];
      b[sizeof(T) - 1 - k] = t;
    }
    memcpy(&v[i], b, sizeof(T));
  }
}

struct File {
  FILE* f = nullptr;
  File(const char* path, const char* mode) { f = fopen(path, mode); }
  ~File() {
    if (f) fclose(f);
  }
};

int valid_head(const int h[5]) {
  // wls = msl^2 mwlt mwlr tmax (wloop_parms.c:182)
  if (h[1] < 1 || h[1] > WLG_MAX_SM_LEVELS || h[2] < 1 || h[3] < 1 || h[4] < 1)
    return fail("dat head: msl, mwlt, mwlr, tmax out of range");
  long long wls = (long long)h[1] * h[1] * h[2] * h[3] * h[4];
  if (wls != h[0]) return fail("dat head: wls %d is not msl^2 mwlt mwlr tmax", h[0]);
  return 0;
}

long long file_size(FILE* f) {
  if (fseek(f, 0, SEEK_END) != 0) return -1;
  long long n = ftell(f);
  fseek(f, 0, SEEK_SET);
  return n;
}

}  // namespace

extern "C" {

const char* wlg_dat_error(void) { return g_err.c_str(); }

int wlg_dat_head(const wlg_wloop_parms* p, int n0, int head[5]) {
  if (!p || !head || n0 < 1) return fail("wlg_dat_head: null argument");
  const long long wls = (long long)p->msl * p->msl * p->mwlt * p->mwlr * n0;
  if (wls > INT32_MAX) return fail("wlg_dat_head: %lld entries do not fit the int32 head", wls);
  head[0] = (int)wls;
  head[1] = p->msl;
  head[2] = p->mwlt;
  head[3] = p->mwlr;
  head[4] = n0;
  return valid_head(head);
}

int wlg_dat_write_head(const char* path, const int head[5]) {
  if (!path || !head) return fail("wlg_dat_write_head: null argument");
  if (valid_head(head)) return -1;
  File f(path, "wb");
  if (!f.f) return fail("write_file_head: unable to open %s", path);
  int32_t istd[5];
  for (int i = 0; i < 5; i++) istd[i] = head[i];
  to_le(istd, 5);
  if (fwrite(istd, sizeof(int32_t), 5, f.f) != 5) return fail("write_file_head: Incorrect write count");
  return 0;
}

int wlg_dat_check_head(const char* path, const int head[5]) {
  if (!path || !head) return fail("wlg_dat_check_head: null argument");
  File f(path, "rb");
  if (!f.f) return fail("check_file_head: unable to open %s", path);
  int32_t istd[5];
  if (fread(istd, sizeof(int32_t), 5, f.f) != 5) return fail("check_file_head: Incorrect read count");
  to_le(istd, 5);
  for (int i = 0; i < 5; i++)
    if (istd[i] != head[i]) return fail("check_file_head: Unexpected value of wls, msl, mwlt, mwlr or tmax");
  return 0;
}

int wlg_dat_append(const char* path, int nc, const double* wl_mat, int wls) {
  if (!path || !wl_mat || wls < 1) return fail("wlg_dat_append: null argument");
  File f(path, "ab");
  if (!f.f) return fail("save_data: unable to open %s", path);
  int32_t istd = nc;
  to_le(&istd, 1);
  std::vector<double> d(wl_mat, wl_mat + wls);
  to_le(d.data(), d.size());
  size_t iw = fwrite(&istd, sizeof(int32_t), 1, f.f);
  iw += fwrite(d.data(), sizeof(double), d.size(), f.f);
  if (iw != (size_t)wls + 1) return fail("write_data: Incorrect write count");
  return 0;
}

long long wlg_dat_count(const char* path, int head[5]) {
  if (!path || !head) return fail("wlg_dat_count: null argument");
  File f(path, "rb");
  if (!f.f) return fail("wlg_dat_count: unable to open %s", path);
  long long size = file_size(f.f);
  int32_t istd[5];
  if (size < 20 || fread(istd, sizeof(int32_t), 5, f.f) != 5) return fail("wlg_dat_count: no head in %s", path);
  to_le(istd, 5);
  for (int i = 0; i < 5; i++) head[i] = istd[i];
  if (valid_head(head)) return -1;
  const long long rec = 4 + 8LL * head[0];
  if ((size - 20) % rec != 0)
    return fail("read_data: Read error or incomplete data record in %s (%lld trailing bytes)", path,
                (size - 20) % rec);
  return (size - 20) / rec;
}

int wlg_dat_read(const char* path, long long rec, int* nc, double* wl_mat, int wls) {
  if (!path || !nc || !wl_mat || rec < 0) return fail("wlg_dat_read: null argument");
  int head[5];
  long long n = wlg_dat_count(path, head);
  if (n < 0) return -1;
  if (rec >= n) return fail("wlg_dat_read: record %lld does not exist", rec);
  if (wls != head[0]) return fail("wlg_dat_read: buffer holds %d doubles, records have %d", wls, head[0]);
  File f(path, "rb");
  if (!f.f) return fail("wlg_dat_read: unable to open %s", path);
  if (fseek(f.f, 20 + rec * (4 + 8LL * wls), SEEK_SET) != 0) return fail("wlg_dat_read: seek failed");
  int32_t istd;
  size_t ir = fread(&istd, sizeof(int32_t), 1, f.f);
  ir += fread(wl_mat, sizeof(double), wls, f.f);
  if (ir != (size_t)wls + 1) return fail("read_data: Read error or incomplete data record");
  to_le(&istd, 1);
  to_le(wl_mat, wls);
  *nc = istd;
  return 0;
}

int wlg_par_write_wloop(const char* path, const wlg_wloop_parms* p) {
  if (!path || !p) return fail("wlg_par_write_wloop: null argument");
  if (p->msl < 1 || p->msl > WLG_MAX_SM_LEVELS) return fail("write_wloop_parms: msl out of range");
  int32_t istd[WLG_MAX_SM_LEVELS + 4];
  double dstd[6] = {p->alpha_ape, p->alpha_hyp[0], p->alpha_hyp[1],
                    p->alpha_action[0], p->alpha_action[1], p->alpha_action[2]};
  for (int i = 0; i < p->msl; i++) istd[i] = p->nss[i];
  istd[p->msl + 0] = p->mwlt;
  istd[p->msl + 1] = p->mwlr;
  istd[p->msl + 2] = p->op_smear;
  istd[p->msl + 3] = p->proj_iter;
  to_le(istd, p->msl + 4);
  to_le(dstd, 6);
  File f(path, "ab");
  if (!f.f) return fail("write_wloop_parms: unable to open %s", path);
  size_t iw = fwrite(istd, sizeof(int32_t), p->msl + 4, f.f);
  iw += fwrite(dstd, sizeof(double), 6, f.f);
  if (iw != (size_t)p->msl + 10) return fail("write_wloop_parms: Incorrect write count");
  return 0;
}

namespace {
// the bc record's values for open / periodic boundary conditions
void bc_record(int bc, int32_t* istd, double dstd[10]) {
  *istd = bc;
  const double v[10] = {1.0, 1.0, 1.0, 1.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
  memcpy(dstd, v, sizeof(v));
}
}  // namespace

int wlg_par_write_bc(const char* path, int bc) {
  if (!path) return fail("wlg_par_write_bc: null argument");
  if (bc != 0 && bc != 3) return fail("write_bc_parms: only open (0) and periodic (3) boundary conditions");
  int32_t istd;
  double dstd[10];
  bc_record(bc, &istd, dstd);
  to_le(&istd, 1);
  to_le(dstd, 10);
  File f(path, "ab");
  if (!f.f) return fail("write_bc_parms: unable to open %s", path);
  size_t iw = fwrite(&istd, sizeof(int32_t), 1, f.f);
  iw += fwrite(dstd, sizeof(double), 10, f.f);
  if (iw != 11) return fail("write_bc_parms: Incorrect write count");
  return 0;
}

int wlg_par_check_bc(const char* path, long long offset, int bc) {
  if (!path || offset < 0) return fail("wlg_par_check_bc: null argument");
  if (bc != 0 && bc != 3) return fail("check_bc_parms: only open (0) and periodic (3) boundary conditions");
  File f(path, "rb");
  if (!f.f) return fail("check_bc_parms: unable to open %s", path);
  if (fseek(f.f, offset, SEEK_SET) != 0) return fail("check_bc_parms: seek failed");
  int32_t istd, want_i;
  double dstd[10], want_d[10];
  size_t ir = fread(&istd, sizeof(int32_t), 1, f.f);
  ir += fread(dstd, sizeof(double), 10, f.f);
  if (ir != 11) return fail("check_bc_parms: Incorrect read count");
  to_le(&istd, 1);
  to_le(dstd, 10);
  bc_record(bc, &want_i, want_d);
  int ie = istd != want_i;
  for (int i = 0; i < 10; i++) ie |= dstd[i] != want_d[i];
  if (ie) return fail("check_bc_parms: Parameters do not match");
  return 0;
}

int wlg_par_check_wloop(const char* path, long long offset, const wlg_wloop_parms* p) {
  if (!path || !p || offset < 0) return fail("wlg_par_check_wloop: null argument");
  if (p->msl < 1 || p->msl > WLG_MAX_SM_LEVELS) return fail("check_wloop_parms: msl out of range");
  File f(path, "rb");
  if (!f.f) return fail("check_wloop_parms: unable to open %s", path);
  if (fseek(f.f, offset, SEEK_SET) != 0) return fail("check_wloop_parms: seek failed");
  int32_t istd[WLG_MAX_SM_LEVELS + 4];
  double dstd[6];
  size_t ir = fread(istd, sizeof(int32_t), p->msl + 4, f.f);
  ir += fread(dstd, sizeof(double), 6, f.f);
  if (ir != (size_t)p->msl + 10) return fail("check_wloop_parms: Incorrect read count");
  to_le(istd, p->msl + 4);
  to_le(dstd, 6);
  int ie = 0;
  for (int i = 0; i < p->msl; i++) ie |= istd[i] != p->nss[i];
  ie |= istd[p->msl + 0] != p->mwlt;
  ie |= istd[p->msl + 1] != p->mwlr;
  ie |= istd[p->msl + 2] != p->op_smear;
  ie |= istd[p->msl + 3] != p->proj_iter;
  ie |= dstd[0] != p->alpha_ape;
  ie |= dstd[1] != p->alpha_hyp[0];
  ie |= dstd[2] != p->alpha_hyp[1];
  ie |= dstd[3] != p->alpha_action[0];
  ie |= dstd[4] != p->alpha_action[1];
  ie |= dstd[5] != p->alpha_action[2];
  if (ie) return fail("check_wloop_parms: Parameters do not match");
  return 0;
}

}  // extern "C"
