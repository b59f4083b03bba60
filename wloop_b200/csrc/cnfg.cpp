// cnfg.cpp -- gauge configurations in openQCD's exported file format.
//
// ms10 reads the configurations it measures with openQCD's import_cnfg
// (main/ms10.c:709-718).  openQCD is not part of the reference, and the
// format below is restated from openQCD's documentation of its export
// format; no real exported file was available to check it against.
//
// Layout (little-endian): 4 int32 lattice extents N0..N3, one double (the
// average plaquette as the writer computed it), then for every odd point x
// (x0+x1+x2+x3 odd) in lexicographic order, x3 fastest, the 8 links
// U(x,0), U(x-0,0), U(x,1), U(x-1,1), U(x,2), U(x-2,2), U(x,3), U(x-3,3),
// each 18 doubles (su3_dble: 9 complex entries, row-major, re/im).  Every link
// of the lattice appears exactly once: (y,mu) has exactly one odd endpoint,
// y or y+mu.  The links are delivered here in the library's host layout
// [V][4][18], lexicographic sites s = x3 + N3 (x2 + N2 (x1 + N1 x0)).
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
void swap_if_big(T* v, size_t n) {
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

// lexicographic index of x - mu (periodic)
long long site_minus(const int n[4], const int x[4], int mu) {
  int y[4] = {x[0], x[1], x[2], x[3]};
  y[mu] = (y[mu] == 0) ? n[mu] - 1 : y[mu] - 1;
  return y[3] + (long long)n[3] * (y[2] + (long long)n[2] * (y[1] + (long long)n[1] * y[0]));
}

// calls f(record index of the point, site of U(x,mu) / U(x-mu,mu), mu) for
// the 8 links of every odd point, in file order
template <class F>
void for_file_links(const int n[4], F f) {
  long long rec = 0;
  int x[4];
  for (x[0] = 0; x[0] < n[0]; x[0]++)
    for (x[1] = 0; x[1] < n[1]; x[1]++)
      for (x[2] = 0; x[2] < n[2]; x[2]++)
        for (x[3] = 0; x[3] < n[3]; x[3]++) {
          if (((x[0] + x[1] + x[2] + x[3]) & 1) == 0) continue;
          const long long s = x[3] + (long long)n[3] * (x[2] + (long long)n[2] * (x[1] + (long long)n[1] * x[0]));
          for (int mu = 0; mu < 4; mu++) {
            f(8 * rec + 2 * mu, s, mu);
            f(8 * rec + 2 * mu + 1, site_minus(n, x, mu), mu);
          }
          rec++;
        }
}

int check_dims(const int n[4], const char* who) {
  long long v = 1;
  for (int i = 0; i < 4; i++) {
    if (n[i] < 2 || (n[i] & 1)) return fail("%s: lattice extent N%d = %d (openQCD extents are even and >= 2)", who, i, n[i]);
    v *= n[i];
  }
  if (v > (1LL << 31)) return fail("%s: lattice too large", who);
  return 0;
}

}  // namespace

extern "C" {

const char* wlg_cnfg_error(void) { return g_err.c_str(); }

int wlg_cnfg_read_head(const char* path, int n[4], double* plaq) {
  if (!path || !n) return fail("wlg_cnfg_read_head: null argument");
  File f(path, "rb");
  if (!f.f) return fail("import_cnfg: unable to open %s", path);
  int32_t istd[4];
  double d;
  if (fread(istd, sizeof(int32_t), 4, f.f) != 4 || fread(&d, sizeof(double), 1, f.f) != 1)
    return fail("import_cnfg: %s is too short for a head", path);
  swap_if_big(istd, 4);
  swap_if_big(&d, 1);
  for (int i = 0; i < 4; i++) n[i] = istd[i];
  if (plaq) *plaq = d;
  return check_dims(n, "import_cnfg");
}

int wlg_cnfg_import(const char* path, const int n[4], double* links, double* plaq) {
  if (!path || !n || !links) return fail("wlg_cnfg_import: null argument");
  int m[4];
  double p = 0.0;
  if (wlg_cnfg_read_head(path, m, &p)) return -1;
  for (int i = 0; i < 4; i++)
    if (m[i] != n[i])
      return fail("import_cnfg: %s holds a %dx%dx%dx%d lattice, expected %dx%dx%dx%d", path, m[0],
                  m[1], m[2], m[3], n[0], n[1], n[2], n[3]);
  const long long vol = (long long)n[0] * n[1] * n[2] * n[3];
  const long long nlinks = 4 * vol;  // = 8 links x V/2 odd points
  File f(path, "rb");
  if (!f.f) return fail("import_cnfg: unable to open %s", path);
  if (fseek(f.f, 0, SEEK_END) != 0) return fail("import_cnfg: seek failed");
  const long long size = ftell(f.f);
  const long long want = 16 + 8 + nlinks * 144;
  if (size != want) return fail("import_cnfg: %s has %lld bytes, the format needs %lld", path, size, want);
  if (fseek(f.f, 24, SEEK_SET) != 0) return fail("import_cnfg: seek failed");
  std::vector<double> buf((size_t)nlinks * 18);
  if (fread(buf.data(), sizeof(double), buf.size(), f.f) != buf.size())
    return fail("import_cnfg: read error in %s", path);
  swap_if_big(buf.data(), buf.size());
  std::vector<char> seen((size_t)nlinks, 0);
  long long dup = 0;
  for_file_links(n, [&](long long r, long long s, int mu) {
    const size_t dst = (size_t)(4 * s + mu);
    dup += seen[dst];
    seen[dst] = 1;
    memcpy(links + dst * 18, buf.data() + (size_t)r * 18, 18 * sizeof(double));
  });
  if (dup) return fail("import_cnfg: internal error, %lld links placed twice", dup);
  if (plaq) *plaq = p;
  return 0;
}

int wlg_cnfg_export(const char* path, const int n[4], const double* links, double plaq) {
  if (!path || !n || !links) return fail("wlg_cnfg_export: null argument");
  if (check_dims(n, "export_cnfg")) return -1;
  const long long vol = (long long)n[0] * n[1] * n[2] * n[3];
  std::vector<double> buf((size_t)(4 * vol) * 18);
  for_file_links(n, [&](long long r, long long s, int mu) {
    memcpy(buf.data() + (size_t)r * 18, links + (size_t)(4 * s + mu) * 18, 18 * sizeof(double));
  });
  int32_t istd[4] = {n[0], n[1], n[2], n[3]};
  double d = plaq;
  swap_if_big(istd, 4);
  swap_if_big(&d, 1);
  swap_if_big(buf.data(), buf.size());
  File f(path, "wb");
  if (!f.f) return fail("export_cnfg: unable to open %s", path);
  size_t w = fwrite(istd, sizeof(int32_t), 4, f.f);
  w += fwrite(&d, sizeof(double), 1, f.f);
  w += fwrite(buf.data(), sizeof(double), buf.size(), f.f);
  if (w != 5 + buf.size()) return fail("export_cnfg: write error in %s", path);
  return 0;
}

}  // extern "C"
