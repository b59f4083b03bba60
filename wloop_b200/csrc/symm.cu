// symm.cu -- symmetry transformations of a gauge field on the device.
//
// The reference checks its loop code with two exact symmetries of the
// measurement: a random gauge transformation U_mu(x) -> g(x) U_mu(x)
// g(x+mu)^dag leaves every Wilson loop unchanged (devel/wloop/check2.c:316-363,
// openQCD's random_g / transform_ud), and a translation of the field by a
// lattice vector s, U(x) -> U(x - s), permutes the time slices of the result,
// W'(x0) = W(x0 - s0) (devel/wloop/check3.c:106-145, openQCD's shift_ud).  The
// kernels below do both on the device so the checks run at full lattice
// sizes.  g(x) is a synthetic SU(3) matrix from the link generator (gen.h)
// keyed by (seed, x); any SU(3) field serves, Haar measure is not needed.
#include "gen.h"
#include "internal.h"

namespace wlg {

template <class T>
__global__ void k_gauge_field(Geo g, uint64_t seed, double eps, typename V2<T>::t* G) {
  for (int s = blockIdx.x * blockDim.x + threadIdx.x; s < g.vol; s += gridDim.x * blockDim.x) {
    double v[18];
    wlg_gen::make_link(seed, (uint64_t)s, eps, v);
    M3<T> m;
#pragma unroll
    for (int c = 0; c < 9; c++) {
      m.e[c].x = (T)v[2 * c];
      m.e[c].y = (T)v[2 * c + 1];
    }
    st(G, g.vol, s, m);
  }
}

// U_mu(x) <- g(x) U_mu(x) g(x+mu)^dag for every link; a zero link (open
// boundary) stays zero
template <class T>
__global__ void k_gauge_apply(Geo g, Links<T> U, const typename V2<T>::t* __restrict__ G) {
  const long long n = 4LL * g.vol;
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < n;
       w += (long long)gridDim.x * blockDim.x) {
    const int mu = (int)(w / g.vol), s = (int)(w - (long long)mu * g.vol);
    int x[4];
    coords(g, s, x);
    M3<T> u, gx, gy, t;
    ld(u, U.p[mu], g.vol, s);
    ld(gx, G, g.vol, s);
    ld(gy, G, g.vol, up(g, s, x[mu], mu));
    mul(t, gx, u);
    mul_ad(u, t, gy);
    st(U.p[mu], g.vol, s, u);
  }
}

// dst_mu(x) = src_mu(x - s) (periodic in every direction)
template <class T>
__global__ void k_shift(Geo g, Links<T> src, Links<T> dst, int4 sh) {
  const long long n = 4LL * g.vol;
  const int shv[4] = {sh.x, sh.y, sh.z, sh.w};
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < n;
       w += (long long)gridDim.x * blockDim.x) {
    const int mu = (int)(w / g.vol), s = (int)(w - (long long)mu * g.vol);
    int x[4];
    coords(g, s, x);
    int y = 0;
#pragma unroll
    for (int d = 0; d < 4; d++) {
      int v = x[d] - shv[d];  // shv[d] in [0, N_d)
      if (v < 0) v += g.n[d];
      y += v * g.st[d];
    }
    M3<T> u;
    ld(u, src.p[mu], g.vol, y);
    st(dst.p[mu], g.vol, s, u);
  }
}

static int grid_for(long long n) {
  long long grid = (n + 255) / 256;
  const long long cap = (long long)num_sms() * 8;
  return (int)(grid < cap ? grid : cap);
}

template <class T>
void gauge_transform(const Geo& g, Links<T> U, typename V2<T>::t* G, uint64_t seed, double eps,
                     cudaStream_t st) {
  k_gauge_field<T><<<grid_for(g.vol), 256, 0, st>>>(g, seed, eps, G);
  WLG_LAUNCH_CHECK("gauge_field");
  k_gauge_apply<T><<<grid_for(4LL * g.vol), 256, 0, st>>>(g, U, G);
  WLG_LAUNCH_CHECK("gauge_apply");
}

template <class T>
void shift_links(const Geo& g, Links<T> src, Links<T> dst, const int s[4], cudaStream_t st) {
  int4 sh;
  int r[4];
  for (int d = 0; d < 4; d++) r[d] = ((s[d] % g.n[d]) + g.n[d]) % g.n[d];
  sh.x = r[0];
  sh.y = r[1];
  sh.z = r[2];
  sh.w = r[3];
  k_shift<T><<<grid_for(4LL * g.vol), 256, 0, st>>>(g, src, dst, sh);
  WLG_LAUNCH_CHECK("shift");
}

template void gauge_transform<double>(const Geo&, Links<double>, double2*, uint64_t, double,
                                      cudaStream_t);
template void gauge_transform<float>(const Geo&, Links<float>, float2*, uint64_t, double,
                                     cudaStream_t);
template void shift_links<double>(const Geo&, Links<double>, Links<double>, const int*, cudaStream_t);
template void shift_links<float>(const Geo&, Links<float>, Links<float>, const int*, cudaStream_t);

}  // namespace wlg
