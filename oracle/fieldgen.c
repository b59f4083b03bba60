/*
 * fieldgen.c -- test-side copy of the synthetic gauge-field generator.
 * TEST INFRASTRUCTURE ONLY: lets the CPU baseline and the reference leg
 * build their inputs without loading the product library.  A CPU test
 * checks that it writes the same bytes as the product's generator.
 *
 * Per link (s, mu) of the lexicographic su3_dble field: eight N(0,1)
 * coefficients h_a from Philox4x32-10 (Salmon et al., SC'11) keyed by the
 * seed, counter (link low word, link high word, draw, 0x57A7), normals by
 * Marsaglia's polar method (logarithm from its atanh series); H = sum_a
 * h_a lambda_a; U = exp(i eps H) by scaling and squaring of a 14-term
 * Taylor series; Gram-Schmidt on rows 1, 2 and row 3 = conj(row1 x row2).
 * With open boundary conditions the time links of the last slice are zero.
 * Only +, -, *, / and sqrt, with contraction off (-ffp-contract=off), so
 * the bytes do not depend on the compiler's choices.
 */
#include <math.h>
#include <stdint.h>
#include <string.h>

typedef struct {
  uint32_t v[4];
} ctr4;

static ctr4 philox10(ctr4 c, uint32_t k0, uint32_t k1)
{
  int r;
  for (r = 0; r < 10; r++) {
    uint64_t p0 = (uint64_t)0xD2511F53u * c.v[0];
    uint64_t p1 = (uint64_t)0xCD9E8D57u * c.v[2];
    ctr4 o;
    o.v[0] = (uint32_t)(p1 >> 32) ^ c.v[1] ^ k0;
    o.v[1] = (uint32_t)p1;
    o.v[2] = (uint32_t)(p0 >> 32) ^ c.v[3] ^ k1;
    o.v[3] = (uint32_t)p0;
    c = o;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

static double unit53(uint32_t a, uint32_t b)
{
  return ((double)(a >> 5) * 67108864.0 + (double)(b >> 6)) * (1.0 / 9007199254740992.0);
}

/* log x for normal x > 0: x = m 2^e, m in [sqrt(1/2), sqrt(2)),
 * log m = 2 atanh(z), z = (m-1)/(m+1), by the series sum z^(2k+1)/(2k+1) */
static double series_log(double x)
{
  union {
    double d;
    uint64_t u;
  } b;
  int e, k;
  double m, z, z2, acc;
  b.d = x;
  e = (int)((b.u >> 52) & 0x7ff) - 1023;
  b.u = (b.u & 0x000fffffffffffffULL) | 0x3ff0000000000000ULL;
  m = b.d;
  if (m > 1.4142135623730951) {
    m = m * 0.5;
    e += 1;
  }
  z = (m - 1.0) / (m + 1.0);
  z2 = z * z;
  acc = 1.0 / 27.0;
  for (k = 12; k >= 0; k--)
    acc = acc * z2 + 1.0 / (double)(2 * k + 1);
  return (double)e * 0.6931471805599453094 + 2.0 * z * acc;
}

static void gaussians8(uint64_t seed, uint64_t link, double h[8])
{
  uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
  int pair, a;
  for (pair = 0; pair < 4; pair++) {
    double g1 = 0.0, g2 = 0.0;
    for (a = 0; a < 64; a++) {
      ctr4 c, r;
      double v1, v2, s, f;
      c.v[0] = (uint32_t)link;
      c.v[1] = (uint32_t)(link >> 32);
      c.v[2] = (uint32_t)(pair * 64 + a);
      c.v[3] = 0x57A7u;
      r = philox10(c, k0, k1);
      v1 = 2.0 * unit53(r.v[0], r.v[1]) - 1.0;
      v2 = 2.0 * unit53(r.v[2], r.v[3]) - 1.0;
      s = v1 * v1 + v2 * v2;
      if (s >= 1.0 || s == 0.0)
        continue;
      f = sqrt(-2.0 * series_log(s) / s);
      g1 = v1 * f;
      g2 = v2 * f;
      break;
    }
    h[2 * pair] = g1;
    h[2 * pair + 1] = g2;
  }
}

/* C = A B for 3x3 complex matrices held as separate real and imaginary parts */
static void mat_mul(const double *ar, const double *ai, const double *br, const double *bi,
                    double *cr, double *ci)
{
  int i, j, k;
  for (i = 0; i < 3; i++)
    for (j = 0; j < 3; j++) {
      double sr = 0.0, si = 0.0;
      for (k = 0; k < 3; k++) {
        double xr = ar[3 * i + k], xi = ai[3 * i + k], yr = br[3 * k + j], yi = bi[3 * k + j];
        sr = sr + (xr * yr - xi * yi);
        si = si + (xr * yi + xi * yr);
      }
      cr[3 * i + j] = sr;
      ci[3 * i + j] = si;
    }
}

static void one_link(uint64_t seed, uint64_t link, double eps, double out[18])
{
  double h[8], Hr[9], Hi[9], Ar[9], Ai[9], Er[9], Ei[9], Tr[9], Ti[9], Wr[9], Wi[9];
  const double r3 = 1.0 / sqrt(3.0);
  double nrm = 0.0, scale = 1.0, n1, n2, dr, di;
  int k, sq = 0, n, q, j;

  gaussians8(seed, link, h);
  /* H = sum_a h_a lambda_a (Gell-Mann) */
  Hr[0] = h[2] + h[7] * r3;  Hi[0] = 0.0;
  Hr[4] = -h[2] + h[7] * r3; Hi[4] = 0.0;
  Hr[8] = -2.0 * h[7] * r3;  Hi[8] = 0.0;
  Hr[1] = h[0]; Hi[1] = -h[1];
  Hr[3] = h[0]; Hi[3] = h[1];
  Hr[2] = h[3]; Hi[2] = -h[4];
  Hr[6] = h[3]; Hi[6] = h[4];
  Hr[5] = h[5]; Hi[5] = -h[6];
  Hr[7] = h[5]; Hi[7] = h[6];
  for (k = 0; k < 9; k++) { /* A = i eps H */
    Ar[k] = -eps * Hi[k];
    Ai[k] = eps * Hr[k];
    nrm = nrm + (Ar[k] * Ar[k] + Ai[k] * Ai[k]);
  }
  nrm = sqrt(nrm);
  while (nrm * scale > 0.25 && sq < 30) {
    scale = scale * 0.5;
    sq++;
  }
  for (k = 0; k < 9; k++) {
    Ar[k] = Ar[k] * scale;
    Ai[k] = Ai[k] * scale;
    Er[k] = (k % 4 == 0) ? 1.0 : 0.0;
    Ei[k] = 0.0;
    Tr[k] = Er[k];
    Ti[k] = 0.0;
  }
  for (n = 1; n <= 14; n++) {
    double inv = 1.0 / (double)n;
    mat_mul(Tr, Ti, Ar, Ai, Wr, Wi);
    for (k = 0; k < 9; k++) {
      Tr[k] = Wr[k] * inv;
      Ti[k] = Wi[k] * inv;
      Er[k] = Er[k] + Tr[k];
      Ei[k] = Ei[k] + Ti[k];
    }
  }
  for (q = 0; q < sq; q++) {
    mat_mul(Er, Ei, Er, Ei, Wr, Wi);
    memcpy(Er, Wr, sizeof(Er));
    memcpy(Ei, Wi, sizeof(Ei));
  }
  n1 = 0.0;
  for (j = 0; j < 3; j++)
    n1 = n1 + (Er[j] * Er[j] + Ei[j] * Ei[j]);
  n1 = 1.0 / sqrt(n1);
  for (j = 0; j < 3; j++) {
    Er[j] = Er[j] * n1;
    Ei[j] = Ei[j] * n1;
  }
  dr = 0.0;
  di = 0.0;
  for (j = 0; j < 3; j++) {
    dr = dr + (Er[j] * Er[3 + j] + Ei[j] * Ei[3 + j]);
    di = di + (Er[j] * Ei[3 + j] - Ei[j] * Er[3 + j]);
  }
  for (j = 0; j < 3; j++) {
    Er[3 + j] = Er[3 + j] - (dr * Er[j] - di * Ei[j]);
    Ei[3 + j] = Ei[3 + j] - (dr * Ei[j] + di * Er[j]);
  }
  n2 = 0.0;
  for (j = 0; j < 3; j++)
    n2 = n2 + (Er[3 + j] * Er[3 + j] + Ei[3 + j] * Ei[3 + j]);
  n2 = 1.0 / sqrt(n2);
  for (j = 0; j < 3; j++) {
    Er[3 + j] = Er[3 + j] * n2;
    Ei[3 + j] = Ei[3 + j] * n2;
  }
  for (j = 0; j < 3; j++) {
    int a = (j + 1) % 3, b = (j + 2) % 3;
    double cr = (Er[a] * Er[3 + b] - Ei[a] * Ei[3 + b]) - (Er[b] * Er[3 + a] - Ei[b] * Ei[3 + a]);
    double ci = (Er[a] * Ei[3 + b] + Ei[a] * Er[3 + b]) - (Er[b] * Ei[3 + a] + Ei[b] * Er[3 + a]);
    Er[6 + j] = cr;
    Ei[6 + j] = -ci;
  }
  for (k = 0; k < 9; k++) {
    out[2 * k] = Er[k];
    out[2 * k + 1] = Ei[k];
  }
}

void orc_generate_links(const int n[4], int bc, uint64_t seed, double eps, double *aos)
{
  const long long vs = (long long)n[1] * n[2] * n[3];
  const long long nl = 4LL * n[0] * vs;
  long long w;
#pragma omp parallel for schedule(static)
  for (w = 0; w < nl; w++) {
    long long s = w >> 2;
    int mu = (int)(w & 3);
    if (bc == 0 && mu == 0 && s / vs == n[0] - 1)
      memset(aos + 18 * w, 0, 18 * sizeof(double));
    else
      one_link(seed, (uint64_t)w, eps, aos + 18 * w);
  }
}

double orc_aux_uniform(uint64_t seed, uint64_t index, uint32_t tag)
{
  ctr4 c, r;
  c.v[0] = (uint32_t)index;
  c.v[1] = (uint32_t)(index >> 32);
  c.v[2] = 0xA0000000u;
  c.v[3] = tag;
  r = philox10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  return unit53(r.v[0], r.v[1]);
}
