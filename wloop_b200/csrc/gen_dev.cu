// gen_dev.cu -- device generator of the synthetic gauge field.
// Compiled with --fmad=false so it writes the same bytes as gen_host.cpp.
#include "internal.h"
#include "gen.h"

namespace wlg {

template <class T>
__global__ void k_generate(Geo g, int bc, uint64_t seed, double eps, Links<T> U) {
  const long long n = 4LL * g.vol;
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < n;
       w += (long long)gridDim.x * blockDim.x) {
    int s = (int)(w >> 2), mu = (int)(w & 3);
    double v[18];
    if (bc == 0 && mu == 0 && s / g.vs == g.n[0] - 1) {
      for (int k = 0; k < 18; k++) v[k] = 0.0;
    } else {
      wlg_gen::make_link(seed, (uint64_t)w, eps, v);
    }
    M3<T> m;
    for (int c = 0; c < 9; c++) {
      m.e[c].x = (T)v[2 * c];
      m.e[c].y = (T)v[2 * c + 1];
    }
    st(U.p[mu], g.vol, s, m);
  }
}

template <class T>
void generate_soa(const Geo& g, int bc, uint64_t seed, double eps, Links<T> U, cudaStream_t st) {
  long long n = 4LL * g.vol;
  long long grid = (n + 127) / 128;
  if (grid > num_sms() * 16) grid = num_sms() * 16;
  k_generate<T><<<(int)grid, 128, 0, st>>>(g, bc, seed, eps, U);
  WLG_LAUNCH_CHECK("generate");
}

template void generate_soa<double>(const Geo&, int, uint64_t, double, Links<double>, cudaStream_t);
template void generate_soa<float>(const Geo&, int, uint64_t, double, Links<float>, cudaStream_t);

}  // namespace wlg
