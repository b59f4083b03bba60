// noalloc.cu -- plaquette sum that allocates no device memory.
//
// Some callers cannot allocate device memory when they need this sum: codes
// whose device memory is owned by another allocator (a framework's caching
// pool, or a preallocated arena that leaves nothing for cudaMalloc), and code
// on a latency-critical path where cudaMalloc / cudaFree would synchronise
// the device and stall other streams.  wlg_plaq_sum_noalloc serves them: the
// caller passes the gauge field and the result slot in device memory it
// already owns, and the only scratch the computation needs -- one FP64
// partial sum per chunk of sites -- lives in the file-scope array below,
// which the driver allocates when this module is loaded on a GPU and which
// every GPU that loads the library holds until the process exits.  With
// CUDA's lazy module loading (the default) the module, and with it the
// array, is loaded on a device by the first call here on that device (its
// cudaGetSymbolAddress), so that first call can itself need device memory:
// make it at start-up, before a preallocated arena claims the memory and
// before any stream capture.
//
// The array is shared by all calls on a device and keeps the last call's
// contents.  Every partial a call reads is written by that same call first,
// so nothing has to start at zero; calls that overlap on the GPU (different
// streams, or host threads, without ordering between them) race on the array
// and must not be issued.
#include <mutex>

#include "internal.h"
#include "../../include/wloop_b200.h"

namespace wlg {
namespace {

constexpr int kThreads = 256;
constexpr int kChunk = 2048;  // sites summed by one block into one partial
constexpr int kMaxPartials = WLG_NOALLOC_MAX_SITES / kChunk;
static_assert(WLG_NOALLOC_MAX_SITES % kChunk == 0, "site limit must be a multiple of the chunk");

// the scratch: kMaxPartials doubles (128 KiB)
static __device__ __align__(256) double g_noalloc_partials[kMaxPartials];

constexpr int kMaxDevices = 64;
std::mutex g_setup_mutex;
double* g_partials_addr[kMaxDevices] = {nullptr};  // device address of the array, per GPU

// link (s,mu) of an AoS lexicographic su3_dble field in device memory
__device__ __forceinline__ void ld_aos(M3<double>& m, const double2* __restrict__ u, int s, int mu) {
  const double2* p = u + 9 * ((size_t)4 * s + mu);
#pragma unroll
  for (int c = 0; c < 9; c++) m.e[c] = __ldg(p + c);
}

__device__ __forceinline__ double plaq_aos(const Geo& g, const double2* __restrict__ u,
                                           const int x[4], int s, int mu, int nu) {
  M3<double> a, b, w1, w2;
  ld_aos(a, u, s, mu);
  ld_aos(b, u, up(g, s, x[mu], mu), nu);
  mul(w1, a, b);
  ld_aos(a, u, s, nu);
  ld_aos(b, u, up(g, s, x[nu], nu), mu);
  mul(w2, a, b);
  return retr_dag(w1, w2);
}

__device__ __forceinline__ double block_sum256(double v) {
  __shared__ double red[kThreads / 32];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = v;
  __syncthreads();
  double r = 0.0;
  if (threadIdx.x < 32) {
    r = (threadIdx.x < kThreads / 32) ? red[threadIdx.x] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) r += __shfl_xor_sync(0xffffffffu, r, o);
  }
  return r;
}

// one block per chunk of kChunk sites: same per-site sum as k_plaq
// (lnkplaq.c:68-114), reading the su3_dble field directly
__global__ void __launch_bounds__(kThreads) k_plaq_chunks(Geo g, int bc, const double2* __restrict__ u,
                                                          double* partials) {
  const int s0 = blockIdx.x * kChunk;
  const int s1 = min(g.vol, s0 + kChunk);
  double acc = 0.0;
  for (int s = s0 + threadIdx.x; s < s1; s += kThreads) {
    int x[4];
    coords(g, s, x);
    double pa = 0.0;
    for (int mu = 1; mu < 4; mu++) {
      if (x[0] < g.n[0] - 1 || bc != 0) pa += plaq_aos(g, u, x, s, mu, 0);
      for (int nu = 1; nu < mu; nu++) pa += plaq_aos(g, u, x, s, mu, nu);
    }
    acc += pa;
  }
  double r = block_sum256(acc);
  if (threadIdx.x == 0) partials[blockIdx.x] = r;
}

// fixed-order sum of the chunk partials into the caller's result slot
__global__ void __launch_bounds__(kThreads) k_plaq_chunks_total(const double* partials, int n,
                                                                double* out) {
  double acc = 0.0;
  for (int i = threadIdx.x; i < n; i += kThreads) acc += partials[i];
  double r = block_sum256(acc);
  if (threadIdx.x == 0) *out = r;
}

// device pointer check without touching the memory: a host pointer handed to
// the kernel would fault or silently read the wrong memory, and so would
// device memory of another GPU (no peer access is set up for it)
int device_accessible(const void* p, const char* what, int dev) {
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    set_error("wlg_plaq_sum_noalloc: %s is not a CUDA pointer", what);
    return 0;
  }
  if (a.type != cudaMemoryTypeDevice && a.type != cudaMemoryTypeManaged) {
    set_error("wlg_plaq_sum_noalloc: %s must point to device (or managed) memory", what);
    return 0;
  }
  if (a.type == cudaMemoryTypeDevice && a.device != dev) {
    set_error("wlg_plaq_sum_noalloc: %s lives on device %d, but device %d is current", what,
              a.device, dev);
    return 0;
  }
  return 1;
}

}  // namespace

int plaq_aos_partials(long long vol) { return (int)((vol + kChunk - 1) / kChunk); }

void plaq_sum_aos(const Geo& g, int bc, const double* links, double* partials, double* out,
                  cudaStream_t st) {
  const int nchunks = plaq_aos_partials(g.vol);
  k_plaq_chunks<<<nchunks, kThreads, 0, st>>>(g, bc, reinterpret_cast<const double2*>(links),
                                               partials);
  WLG_LAUNCH_CHECK("plaq_chunks");
  k_plaq_chunks_total<<<1, kThreads, 0, st>>>(partials, nchunks, out);
  WLG_LAUNCH_CHECK("plaq_chunks_total");
}

}  // namespace wlg

using namespace wlg;

extern "C" int wlg_plaq_sum_noalloc(const double* links, const int n[4], int bc, double* out,
                                    void* stream) {
  set_error("%s", "");
  if (!links || !n || !out) {
    set_error("wlg_plaq_sum_noalloc: null argument");
    return -1;
  }
  for (int i = 0; i < 4; i++)
    if (n[i] < 2) {
      set_error("wlg_plaq_sum_noalloc: lattice extent N%d=%d < 2", i, n[i]);
      return -1;
    }
  if (bc != 0 && bc != 3) {
    set_error("wlg_plaq_sum_noalloc: only open (0) and periodic (3) boundary conditions");
    return -1;
  }
  const long long vol = (long long)n[0] * n[1] * n[2] * n[3];
  if (vol > WLG_NOALLOC_MAX_SITES) {
    set_error("wlg_plaq_sum_noalloc: %lld sites exceed the maximum of %d this entry point's "
              "fixed scratch supports (use wlg_plaq_sum)",
              vol, WLG_NOALLOC_MAX_SITES);
    return -1;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    set_error("wlg_plaq_sum_noalloc: no usable current CUDA device");
    return -1;
  }
  if (!device_accessible(links, "links", dev) || !device_accessible(out, "out", dev)) return -1;
  double* partials = nullptr;
  {
    // set-up once per device, with that device current: the device address of
    // the scratch array (its name in host code is only a host-side stand-in)
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_partials_addr[dev]) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
      if (e != cudaSuccess || !p) {
        cudaGetLastError();
        set_error("wlg_plaq_sum_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
        return -1;
      }
      g_partials_addr[dev] = static_cast<double*>(p);
    }
    partials = g_partials_addr[dev];
  }
  plaq_sum_aos(make_geo(n), bc, links, partials, out, static_cast<cudaStream_t>(stream));
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    set_error("wlg_plaq_sum_noalloc: %s", cudaGetErrorString(e));
    return -1;
  }
  return get_error()[0] ? -1 : 0;
}
