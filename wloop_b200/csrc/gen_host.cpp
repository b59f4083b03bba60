// gen_host.cpp -- host generator of the synthetic gauge field (same bytes as
// the device kernel in gen_dev.cu; compiled with -ffp-contract=off).
#include <stdint.h>
#include <string.h>
#include <math.h>
#include "gen.h"
#include "../../include/wloop_b200.h"

extern "C" int wlg_generate_links(const int n[4], int bc, uint64_t seed, double eps,
                                  double* aos) {
  if (!n || !aos) return -1;
  for (int i = 0; i < 4; i++)
    if (n[i] < 1) return -1;
  const long long vs = (long long)n[1] * n[2] * n[3];
  const long long nl = 4LL * n[0] * vs;
#pragma omp parallel for schedule(static)
  for (long long w = 0; w < nl; w++) {
    long long s = w >> 2;
    int mu = (int)(w & 3);
    double* out = aos + 18 * w;
    if (bc == 0 && mu == 0 && s / vs == n[0] - 1)
      memset(out, 0, 18 * sizeof(double));
    else
      wlg_gen::make_link(seed, (uint64_t)w, eps, out);
  }
  return 0;
}

extern "C" double wlg_aux_uniform(uint64_t seed, uint64_t index, uint32_t tag) {
  return wlg_gen::aux_uniform(seed, index, tag);
}
