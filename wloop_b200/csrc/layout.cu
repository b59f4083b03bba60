// layout.cu -- conversions between host link layouts and the device SoA field.
//
// Host layouts:
//  * AoS lexicographic FP64: link (s,mu) at aos[18*(4*s+mu)] (su3_dble bytes)
//  * openQCD (NPROC=1): 8 links per odd point iq >= V/2 (lnkcom.c:840-859):
//      ud[8*(iq-V/2)+2mu]   = U(x_iq, mu)
//      ud[8*(iq-V/2)+2mu+1] = U(x_iq - mu, mu)
//    ipt[s] gives the openQCD index of lexicographic site s.
// The host buffer is copied to the device as is; these kernels do the
// transposition on the device (one thread per link, coalesced SoA side).
#include "internal.h"

namespace wlg {

template <class T>
__global__ void k_aos_to_soa(Geo g, const double2* __restrict__ aos, Links<T> U, int mu0, int nmu) {
  const long long n = (long long)nmu * g.vol;
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < n;
       w += (long long)gridDim.x * blockDim.x) {
    int q = (int)(w / g.vol), s = (int)(w - (long long)q * g.vol);
    int mu = mu0 + q;
    const double2* src = aos + 9 * ((size_t)4 * s + mu);
    M3<T> m;
#pragma unroll
    for (int c = 0; c < 9; c++) {
      double2 v = src[c];
      m.e[c].x = (T)v.x;
      m.e[c].y = (T)v.y;
    }
    st(U.p[mu], g.vol, s, m);
  }
}

// SoA -> AoS through shared memory, one block of 128 threads per 32-site
// tile: warp q reads direction mu0+q of the tile component by component (one
// coalesced 512-byte request per component), the block then writes the
// tile's links in AoS order, consecutive threads on consecutive 16 bytes.
// Per site the stage holds 4 links (36 double2) plus one double2 of padding,
// so that eight consecutive lanes writing their sites' entries hit distinct
// banks.
constexpr int kSiteStride = 37;  // double2 per site in the stage
template <class T>
__global__ void __launch_bounds__(128) k_soa_to_aos(Geo g, Links<T> U, double2* __restrict__ aos,
                                                    int mu0, int nmu) {
  __shared__ double2 tile[32 * kSiteStride];
  const int s0 = blockIdx.x * 32;
  const int q = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int s = s0 + lane;
  if (q < nmu && s < g.vol) {
    M3<T> m;
    ld(m, U.p[mu0 + q], g.vol, s);
    double2* t = tile + lane * kSiteStride + 9 * q;
#pragma unroll
    for (int c = 0; c < 9; c++) t[c] = make_double2((double)m.e[c].x, (double)m.e[c].y);
  }
  __syncthreads();
  const int nsite = min(32, g.vol - s0);
  const int per = 9 * nmu;  // double2 per site written
  for (int e = threadIdx.x; e < nsite * per; e += blockDim.x) {
    const int site = e / per, r = e - site * per;
    const int mu = r / 9, c = r - mu * 9;
    aos[9 * ((size_t)4 * (s0 + site) + mu0 + mu) + c] = tile[site * kSiteStride + r];
  }
}

// offset (in links) of U(s,mu) inside an openQCD field (ofs_lnk, lnkcom.c:840-859)
__device__ __forceinline__ size_t openqcd_ofs(const Geo& g, const int* ipt, int s, int mu) {
  int iq = ipt[s];
  int h = g.vol / 2;
  if (iq >= h) return (size_t)8 * (iq - h) + 2 * mu;
  int x[4];
  coords(g, s, x);
  int iy = ipt[up(g, s, x[mu], mu)];
  return (size_t)8 * (iy - h) + 2 * mu + 1;
}

template <class T>
__global__ void k_openqcd_to_soa(Geo g, const double2* __restrict__ ud, const int* __restrict__ ipt,
                                 Links<T> U, int mu0, int nmu) {
  const long long n = (long long)nmu * g.vol;
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < n;
       w += (long long)gridDim.x * blockDim.x) {
    int q = (int)(w / g.vol), s = (int)(w - (long long)q * g.vol);
    int mu = mu0 + q;
    const double2* src = ud + 9 * openqcd_ofs(g, ipt, s, mu);
    M3<T> m;
#pragma unroll
    for (int c = 0; c < 9; c++) {
      double2 v = src[c];
      m.e[c].x = (T)v.x;
      m.e[c].y = (T)v.y;
    }
    st(U.p[mu], g.vol, s, m);
  }
}

template <class T>
__global__ void k_soa_to_openqcd(Geo g, Links<T> U, const int* __restrict__ ipt,
                                 double2* __restrict__ ud, int mu0, int nmu) {
  const long long n = (long long)nmu * g.vol;
  for (long long w = blockIdx.x * (long long)blockDim.x + threadIdx.x; w < n;
       w += (long long)gridDim.x * blockDim.x) {
    int q = (int)(w / g.vol), s = (int)(w - (long long)q * g.vol);
    int mu = mu0 + q;
    double2* dst = ud + 9 * openqcd_ofs(g, ipt, s, mu);
    M3<T> m;
    ld(m, U.p[mu], g.vol, s);
#pragma unroll
    for (int c = 0; c < 9; c++) dst[c] = make_double2((double)m.e[c].x, (double)m.e[c].y);
  }
}

static int grid_n(long long n) {
  long long gsz = (n + 255) / 256;
  long long cap = (long long)num_sms() * 16;
  return (int)(gsz < 1 ? 1 : (gsz > cap ? cap : gsz));
}

template <class T>
void aos_to_soa(const Geo& g, const double* aos, Links<T> U, int mu0, int mu1, cudaStream_t st) {
  int nmu = mu1 - mu0;
  k_aos_to_soa<T><<<grid_n((long long)nmu * g.vol), 256, 0, st>>>(
      g, reinterpret_cast<const double2*>(aos), U, mu0, nmu);
  WLG_LAUNCH_CHECK("aos_to_soa");
}
template <class T>
void soa_to_aos(const Geo& g, Links<T> U, double* aos, int mu0, int mu1, cudaStream_t st) {
  int nmu = mu1 - mu0;
  if (nmu < 1 || nmu > 4) return;
  k_soa_to_aos<T><<<(g.vol + 31) / 32, 128, 0, st>>>(g, U, reinterpret_cast<double2*>(aos), mu0,
                                                     nmu);
  WLG_LAUNCH_CHECK("soa_to_aos");
}
template <class T>
void openqcd_to_soa(const Geo& g, const double* ud, const int* ipt, Links<T> U, int mu0, int mu1,
                    cudaStream_t st) {
  int nmu = mu1 - mu0;
  k_openqcd_to_soa<T><<<grid_n((long long)nmu * g.vol), 256, 0, st>>>(
      g, reinterpret_cast<const double2*>(ud), ipt, U, mu0, nmu);
  WLG_LAUNCH_CHECK("openqcd_to_soa");
}
template <class T>
void soa_to_openqcd(const Geo& g, Links<T> U, const int* ipt, double* ud, int mu0, int mu1,
                    cudaStream_t st) {
  int nmu = mu1 - mu0;
  k_soa_to_openqcd<T><<<grid_n((long long)nmu * g.vol), 256, 0, st>>>(
      g, U, ipt, reinterpret_cast<double2*>(ud), mu0, nmu);
  WLG_LAUNCH_CHECK("soa_to_openqcd");
}
#define WLG_INST_L(T)                                                                       \
  template void aos_to_soa<T>(const Geo&, const double*, Links<T>, int, int, cudaStream_t); \
  template void soa_to_aos<T>(const Geo&, Links<T>, double*, int, int, cudaStream_t);       \
  template void openqcd_to_soa<T>(const Geo&, const double*, const int*, Links<T>, int, int, \
                                  cudaStream_t);                                            \
  template void soa_to_openqcd<T>(const Geo&, Links<T>, const int*, double*, int, int,      \
                                  cudaStream_t);
WLG_INST_L(double)
WLG_INST_L(float)

}  // namespace wlg
