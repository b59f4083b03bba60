// gen.h -- synthetic SU(3) gauge links, shared by the host and device builds.
//
// Per link (s,mu): h_a ~ N(0,1) (a=1..8), H = sum_a h_a lambda_a (Gell-Mann),
// U = exp(i eps H) by scaling and squaring of a Taylor series, then
// reunitarised (Gram-Schmidt on rows 1,2; row 3 = conj(row1 x row2)).
// Randomness: Philox4x32-10 (Salmon et al., SC'11) keyed by the seed, counter
// (link lo, link hi, draw, tag); normals by Marsaglia's polar method with a
// logarithm evaluated here from its atanh series.  Only IEEE +,-,*,/ and
// sqrt are used, and both builds disable FMA contraction (host
// -ffp-contract=off, device --fmad=false), so the host and the device write
// identical bytes.
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define WLG_HD __host__ __device__ __forceinline__
#else
#define WLG_HD static inline
#endif

namespace wlg_gen {

struct u4 {
  uint32_t x, y, z, w;
};

WLG_HD void mulhilo(uint32_t a, uint32_t b, uint32_t* hi, uint32_t* lo) {
  uint64_t p = (uint64_t)a * (uint64_t)b;
  *hi = (uint32_t)(p >> 32);
  *lo = (uint32_t)p;
}

// Philox4x32 with 10 rounds
WLG_HD u4 philox(u4 c, uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; r++) {
    uint32_t hi0, lo0, hi1, lo1;
    mulhilo(0xD2511F53u, c.x, &hi0, &lo0);
    mulhilo(0xCD9E8D57u, c.z, &hi1, &lo1);
    u4 o;
    o.x = hi1 ^ c.y ^ k0;
    o.y = lo1;
    o.z = hi0 ^ c.w ^ k1;
    o.w = lo0;
    c = o;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

// 53-bit uniform in [0,1) from two 32-bit words
WLG_HD double u01(uint32_t a, uint32_t b) {
  return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

// natural logarithm of a positive normal double:
// x = m 2^e with m in [sqrt(1/2), sqrt(2)), log m = 2 atanh((m-1)/(m+1))
WLG_HD double log_pos(double x) {
  union {
    double d;
    uint64_t u;
  } v;
  v.d = x;
  int e = (int)((v.u >> 52) & 0x7ff) - 1023;
  v.u = (v.u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL;  // m in [1,2)
  double m = v.d;
  if (m > 1.4142135623730951) {
    m = m * 0.5;
    e += 1;
  }
  double z = (m - 1.0) / (m + 1.0);
  double z2 = z * z;
  double p = 1.0 / 27.0;
  for (int k = 12; k >= 0; k--) p = p * z2 + 1.0 / (double)(2 * k + 1);
  return (double)e * 0.6931471805599453094 + 2.0 * z * p;
}

// 8 standard normals for link id `link`
WLG_HD void normals8(uint64_t seed, uint64_t link, double h[8]) {
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  for (int p = 0; p < 4; p++) {
    double z1 = 0.0, z2 = 0.0;
    for (int a = 0; a < 64; a++) {
      u4 c;
      c.x = (uint32_t)link;
      c.y = (uint32_t)(link >> 32);
      c.z = (uint32_t)(p * 64 + a);
      c.w = 0x57A7u;
      u4 r = philox(c, k0, k1);
      double v1 = 2.0 * u01(r.x, r.y) - 1.0;
      double v2 = 2.0 * u01(r.z, r.w) - 1.0;
      double s = v1 * v1 + v2 * v2;
      if (s >= 1.0 || s == 0.0) continue;
      double f = sqrt(-2.0 * log_pos(s) / s);
      z1 = v1 * f;
      z2 = v2 * f;
      break;
    }
    h[2 * p] = z1;
    h[2 * p + 1] = z2;
  }
}

// uniform double in [0,1) for auxiliary per-config draws (eps, arrivals, ...)
WLG_HD double aux_uniform(uint64_t seed, uint64_t index, uint32_t tag) {
  u4 c;
  c.x = (uint32_t)index;
  c.y = (uint32_t)(index >> 32);
  c.z = 0xA0000000u;
  c.w = tag;
  u4 r = philox(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  return u01(r.x, r.y);
}

// complex 3x3 helpers on arrays re[9], im[9]
WLG_HD void cmul3(const double* ar, const double* ai, const double* br, const double* bi,
                  double* cr, double* ci) {
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      double sr = 0.0, si = 0.0;
      for (int k = 0; k < 3; k++) {
        double xr = ar[3 * i + k], xi = ai[3 * i + k], yr = br[3 * k + j], yi = bi[3 * k + j];
        sr = sr + (xr * yr - xi * yi);
        si = si + (xr * yi + xi * yr);
      }
      cr[3 * i + j] = sr;
      ci[3 * i + j] = si;
    }
}

// link value in su3_dble order (re,im interleaved, row-major)
WLG_HD void make_link(uint64_t seed, uint64_t link, double eps, double out[18]) {
  double h[8];
  normals8(seed, link, h);
  const double r3 = 1.0 / sqrt(3.0);
  double Hr[9], Hi[9];
  Hr[0] = h[2] + h[7] * r3;  Hi[0] = 0.0;
  Hr[4] = -h[2] + h[7] * r3; Hi[4] = 0.0;
  Hr[8] = -2.0 * h[7] * r3;  Hi[8] = 0.0;
  Hr[1] = h[0];  Hi[1] = -h[1];
  Hr[3] = h[0];  Hi[3] = h[1];
  Hr[2] = h[3];  Hi[2] = -h[4];
  Hr[6] = h[3];  Hi[6] = h[4];
  Hr[5] = h[5];  Hi[5] = -h[6];
  Hr[7] = h[5];  Hi[7] = h[6];
  // A = i eps H
  double Ar[9], Ai[9], nrm = 0.0;
  for (int k = 0; k < 9; k++) {
    Ar[k] = -eps * Hi[k];
    Ai[k] = eps * Hr[k];
    nrm = nrm + (Ar[k] * Ar[k] + Ai[k] * Ai[k]);
  }
  nrm = sqrt(nrm);
  int sq = 0;
  double scale = 1.0;
  while (nrm * scale > 0.25 && sq < 30) {
    scale = scale * 0.5;
    sq++;
  }
  for (int k = 0; k < 9; k++) {
    Ar[k] = Ar[k] * scale;
    Ai[k] = Ai[k] * scale;
  }
  // Taylor: E = sum_{n=0}^{14} A^n / n!
  double Er[9], Ei[9], Tr[9], Ti[9], Wr[9], Wi[9];
  for (int k = 0; k < 9; k++) {
    Er[k] = (k % 4 == 0) ? 1.0 : 0.0;
    Ei[k] = 0.0;
    Tr[k] = Er[k];
    Ti[k] = 0.0;
  }
  for (int n = 1; n <= 14; n++) {
    cmul3(Tr, Ti, Ar, Ai, Wr, Wi);
    double inv = 1.0 / (double)n;
    for (int k = 0; k < 9; k++) {
      Tr[k] = Wr[k] * inv;
      Ti[k] = Wi[k] * inv;
      Er[k] = Er[k] + Tr[k];
      Ei[k] = Ei[k] + Ti[k];
    }
  }
  for (int q = 0; q < sq; q++) {
    cmul3(Er, Ei, Er, Ei, Wr, Wi);
    for (int k = 0; k < 9; k++) {
      Er[k] = Wr[k];
      Ei[k] = Wi[k];
    }
  }
  // reunitarise
  double n1 = 0.0;
  for (int j = 0; j < 3; j++) n1 = n1 + (Er[j] * Er[j] + Ei[j] * Ei[j]);
  n1 = 1.0 / sqrt(n1);
  for (int j = 0; j < 3; j++) {
    Er[j] = Er[j] * n1;
    Ei[j] = Ei[j] * n1;
  }
  double dr = 0.0, di = 0.0;  // <row1,row2> = sum conj(r1) r2
  for (int j = 0; j < 3; j++) {
    dr = dr + (Er[j] * Er[3 + j] + Ei[j] * Ei[3 + j]);
    di = di + (Er[j] * Ei[3 + j] - Ei[j] * Er[3 + j]);
  }
  for (int j = 0; j < 3; j++) {
    Er[3 + j] = Er[3 + j] - (dr * Er[j] - di * Ei[j]);
    Ei[3 + j] = Ei[3 + j] - (dr * Ei[j] + di * Er[j]);
  }
  double n2 = 0.0;
  for (int j = 0; j < 3; j++) n2 = n2 + (Er[3 + j] * Er[3 + j] + Ei[3 + j] * Ei[3 + j]);
  n2 = 1.0 / sqrt(n2);
  for (int j = 0; j < 3; j++) {
    Er[3 + j] = Er[3 + j] * n2;
    Ei[3 + j] = Ei[3 + j] * n2;
  }
  // row3 = conj(row1 x row2)
  for (int j = 0; j < 3; j++) {
    int a = (j + 1) % 3, b = (j + 2) % 3;
    double cr = (Er[a] * Er[3 + b] - Ei[a] * Ei[3 + b]) - (Er[b] * Er[3 + a] - Ei[b] * Ei[3 + a]);
    double ci = (Er[a] * Ei[3 + b] + Ei[a] * Er[3 + b]) - (Er[b] * Ei[3 + a] + Ei[b] * Er[3 + a]);
    Er[6 + j] = cr;
    Ei[6 + j] = -ci;
  }
  for (int k = 0; k < 9; k++) {
    out[2 * k] = Er[k];
    out[2 * k + 1] = Ei[k];
  }
}

}  // namespace wlg_gen
