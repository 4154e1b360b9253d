// ws_run_algorithm_noalloc: the MBS loop with its scratch in a fixed,
// statically allocated device array.
//
// Who needs this: code that must not allocate GPU memory while it runs -
// for example a host application that has handed the whole device to its own
// memory pool or arena, a real-time or embedded loop that forbids allocation
// after start-up, or a plug-in that runs inside another framework's allocator
// and may only use the buffers it is given.  Such a caller passes device
// buffers for every input and output; the loop's working arrays (the field
// increment dE, the transform buffer, twiddle tables and the loop state) live
// in g_ws_scratch below instead of cudaMalloc'd memory.
//
// Limits and rules:
//  * The scratch array is kScratchBytes (40 MiB).  Each GPU that loads this
//    part of the library holds it until the process exits.  A grid needs
//    16 bytes per field element (Ny*Nx*Nz*Nc) plus its twiddle tables; larger
//    grids are rejected with WS_ERR_INVALID_ARGUMENT before any launch.
//  * Every call shares the one array and leaves its contents behind; each call
//    clears what must start at zero.  Calls that overlap on the GPU (several
//    host threads, or several streams) race on the array: serialise them.
//  * The first call on a device looks up the array's device address
//    (cudaGetSymbolAddress, with that device current).  Make that first call
//    before any stream capture is active.
//  * No cudaMalloc, cudaFree, graph instantiation or other allocating call is
//    made; the loop is driven from the host, one wiggle cycle at a time.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>

#include "wavesim_b200.h"
#include "ws_fast.cuh"
#include "ws_kernels.cuh"

namespace ws {
namespace noalloc {

constexpr size_t kScratchBytes = 40ull << 20;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_ws_scratch[kScratchBytes];

static void* g_scratch_addr[kMaxDevices] = {};  // device address of g_ws_scratch per device
static bool g_attrs_set[kMaxDevices] = {};
static std::mutex g_setup_mutex;  // guards the two tables above

thread_local std::string t_error;
static int fail(int code, const std::string& m) {
  t_error = m;
  return code;
}

#define NA_CUDA(call)                                                                  \
  do {                                                                                 \
    cudaError_t e__ = (call);                                                          \
    if (e__ != cudaSuccess) return fail(WS_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e__)); \
  } while (0)

static bool pow2(int n) { return n > 0 && (n & (n - 1)) == 0; }

// Radix schedule of the generic kernels (largest radices first).
static bool plan(int n, FftPlan& p) {
  static const int pref[] = {16, 12, 13, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2};
  p.n = n;
  p.nst = 0;
  while (n > 1) {
    int r = 0;
    for (int c : pref)
      if (n % c == 0) {
        r = c;
        break;
      }
    if (!r || p.nst == kMaxStages) return false;
    p.radix[p.nst++] = r;
    n /= r;
  }
  for (int i = p.nst; i < kMaxStages; ++i) p.radix[i] = 1;
  return true;
}

// exp(-2 pi i k / n) for k < n, in double precision on the device.
__global__ void k_twiddles(float2* tw, int n) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
    double s, c;
    sincospi(-2.0 * (double)k / (double)n, &s, &c);
    tw[k] = make_float2((float)c, (float)s);
  }
}

// Shapes of this entry point: power-of-two 2-D grids (columns of 64..2048,
// pencils of 32..1024) and 3-D grids with 64^2 or 128^2 planes use the fast
// kernels; every other supported size uses the generic kernels.
struct Shape {
  int mode3d = 0, fast = 0, n = 0, csize = 1, ncols = 1, ty = 16, th = 256, rset = kPow2;
  size_t smem_inner = 0, smem_outer = 0;
  long long grid_inner = 0, grid_outer = 0;
  int fast_pencil = 0;
};

template <int N, int C, bool DX>
static void attrs_fast(int optin) {
  cudaFuncSetAttribute((const void*)fast::kf_plane_fwd<N, C, DX>, cudaFuncAttributeMaxDynamicSharedMemorySize, optin);
  cudaFuncSetAttribute((const void*)fast::kf_plane_inv<N, C, DX>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                       optin - 256);
}

static int set_attributes(int dev) {
  if (g_attrs_set[dev]) return WS_OK;
  int optin = 0;
  NA_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  const int lim = optin - 1024;
  NA_CUDA(cudaFuncSetAttribute(k_fwd_inner<16, kPow2>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
  NA_CUDA(cudaFuncSetAttribute(k_inv_inner<16, kPow2>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
  NA_CUDA(cudaFuncSetAttribute(k_outer<16, kPow2>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
  NA_CUDA(cudaFuncSetAttribute(k_fwd_inner<16, kMixed>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
  NA_CUDA(cudaFuncSetAttribute(k_inv_inner<16, kMixed>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
  NA_CUDA(cudaFuncSetAttribute(k_outer<16, kMixed>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim));
  NA_CUDA(cudaFuncSetAttribute(k_fwd_inner<16, kPow2>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  NA_CUDA(cudaFuncSetAttribute(k_inv_inner<16, kPow2>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  NA_CUDA(cudaFuncSetAttribute(k_fwd_inner<16, kMixed>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  NA_CUDA(cudaFuncSetAttribute(k_inv_inner<16, kMixed>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
  attrs_fast<64, 1, true>(lim);
  attrs_fast<128, 2, true>(lim);
  attrs_fast<64, 1, false>(lim);
  attrs_fast<128, 1, false>(lim);
  attrs_fast<256, 1, false>(lim);
  attrs_fast<512, 1, false>(lim);
  attrs_fast<1024, 1, false>(lim);
  attrs_fast<2048, 1, false>(lim);
  NA_CUDA(cudaGetLastError());
  g_attrs_set[dev] = true;
  return WS_OK;
}

static int shape_for(const Geom& g, Shape& s) {
  s.mode3d = g.nz > 1;
  const int lim_threads = 512, emax = 16;
  const size_t budget = 150 * 1024;
  bool all_pow2 = pow2(g.ny) && pow2(g.nx) && pow2(g.nz);
  s.rset = all_pow2 ? kPow2 : kMixed;
  auto threads_for = [&](long long e) {
    long long t = ((e + emax - 1) / emax + 31) / 32 * 32;
    return (int)std::max(32LL, std::min((long long)lim_threads, t));
  };
  const size_t colb = (size_t)padded(g.ny) * sizeof(float2);
  // fast kernels
  if (s.mode3d && g.nc == 1 && g.ny == g.nx && (g.ny == 64 || g.ny == 128)) {
    s.fast = 1;
    s.n = g.ny;
    s.csize = g.ny == 64 ? 1 : 2;
    s.grid_inner = (long long)g.nz * g.nc * s.csize;
    s.smem_inner = g.ny == 64 ? fast::PlaneGeom<64, 1, true>::smem : fast::PlaneGeom<128, 2, true>::smem;
  } else if (!s.mode3d && pow2(g.ny) && g.ny >= 64 && g.ny <= 2048) {
    s.fast = 1;
    s.n = g.ny;
    s.ncols = std::max(1, 4096 / g.ny);
    s.grid_inner = ((long long)g.nx * g.nc + s.ncols - 1) / s.ncols;
    s.smem_inner = (size_t)(s.ncols + 1) * (g.ny + g.ny / 16 + 1) * sizeof(float2);
  } else if (s.mode3d) {
    int best = 0;
    for (int c = 1; c <= 16; ++c) {
      if (g.nx % c) continue;
      const long long cols = g.nx / c;
      if (cols * g.ny > (long long)lim_threads * emax || cols * colb > budget) continue;
      FftPlan tmp{};
      if (c > 1 && !plan((int)cols, tmp)) continue;  // the x-local length must have a radix schedule
      best = c;
      break;
    }
    if (!best) return WS_ERR_UNSUPPORTED;
    s.csize = best;
    const long long cols = g.nx / best;
    s.th = threads_for(cols * g.ny);
    s.smem_inner = cols * colb;
    s.grid_inner = (long long)g.nz * g.nc * best;
  } else {
    if ((long long)g.ny > (long long)lim_threads * emax || colb > budget) return WS_ERR_UNSUPPORTED;
    const long long total = (long long)g.nx * g.nc;
    // a block holds at most lim_threads x emax elements: the FFT stages of the
    // generic kernels cover no more butterflies than that
    const long long max_cols_fit =
        std::max(1LL, std::min((long long)(budget / colb), (long long)lim_threads * emax / (long long)g.ny));
    long long want = std::max(1LL, std::min(max_cols_fit, (8192LL + g.ny - 1) / g.ny));
    while (want > 1 && (total + want - 1) / want < 296) want /= 2;
    s.ncols = (int)want;
    s.th = threads_for(want * g.ny);
    s.smem_inner = want * colb;
    s.grid_inner = (total + want - 1) / want;
  }
  // outer pass (generic kernel, or the fast pencil kernel for scalar power-of-two 2-D / 3-D)
  const int no = s.mode3d ? g.nz : g.nx;
  const long long mids = s.mode3d ? g.nx : 1;
  if (g.nc == 1 && pow2(no) && no >= 32 && no <= 256 && g.ny % 16 == 0) {
    s.fast_pencil = 1;
    s.ty = 16;
    s.grid_outer = (long long)(g.ny / 16) * mids;
    s.smem_outer = (size_t)17 * no * sizeof(float2);
    return WS_OK;
  }
  int ty = 16;
  while (ty > 1 && ((long long)padded(g.nc * ty) * no * 8 > (long long)budget || (long long)g.nc * ty * no > 8192)) ty /= 2;
  if (ty > g.ny) ty = std::max(1, g.ny);
  if ((long long)padded(g.nc * ty) * no * 8 > (long long)budget || (long long)g.nc * ty * no > 8192)
    return WS_ERR_UNSUPPORTED;
  s.ty = ty;
  s.smem_outer = (size_t)padded(g.nc * ty) * no * sizeof(float2);
  s.grid_outer = (long long)((g.ny + ty - 1) / ty) * mids;
  s.th = std::max(s.th, 32);
  return WS_OK;
}

struct Run {
  Geom g;
  Shape sh;
  InnerArgs ia;
  OuterArgs oa;
  float2 *dE, *T, *E, *src;
  const float2* gamma;
  DevState* st;
  double* partials;
  cudaStream_t stream;
};

static cudaError_t launch_inner(const Run& r, bool inverse, void** args, const void* fast_fn, const void* gen_fn,
                                int threads) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)r.sh.grid_inner);
  cfg.blockDim = dim3(threads);
  cfg.dynamicSmemBytes = r.sh.smem_inner;
  cfg.stream = r.stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = r.sh.mode3d ? r.sh.csize : 1;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  (void)inverse;
  return cudaLaunchKernelExC(&cfg, r.sh.fast ? fast_fn : gen_fn, args);
}

static const void* fast_fwd(const Shape& s) {
  if (s.mode3d) return s.n == 64 ? (const void*)fast::kf_plane_fwd<64, 1, true> : (const void*)fast::kf_plane_fwd<128, 2, true>;
  switch (s.n) {
    case 64: return (const void*)fast::kf_plane_fwd<64, 1, false>;
    case 128: return (const void*)fast::kf_plane_fwd<128, 1, false>;
    case 256: return (const void*)fast::kf_plane_fwd<256, 1, false>;
    case 512: return (const void*)fast::kf_plane_fwd<512, 1, false>;
    case 1024: return (const void*)fast::kf_plane_fwd<1024, 1, false>;
    default: return (const void*)fast::kf_plane_fwd<2048, 1, false>;
  }
}
static const void* fast_inv(const Shape& s) {
  if (s.mode3d) return s.n == 64 ? (const void*)fast::kf_plane_inv<64, 1, true> : (const void*)fast::kf_plane_inv<128, 2, true>;
  switch (s.n) {
    case 64: return (const void*)fast::kf_plane_inv<64, 1, false>;
    case 128: return (const void*)fast::kf_plane_inv<128, 1, false>;
    case 256: return (const void*)fast::kf_plane_inv<256, 1, false>;
    case 512: return (const void*)fast::kf_plane_inv<512, 1, false>;
    case 1024: return (const void*)fast::kf_plane_inv<1024, 1, false>;
    default: return (const void*)fast::kf_plane_inv<2048, 1, false>;
  }
}
static const void* fast_pencil(int no) {
  switch (no) {
    case 32: return (const void*)fast::kf_pencil<32, 16>;
    case 64: return (const void*)fast::kf_pencil<64, 16>;
    case 128: return (const void*)fast::kf_pencil<128, 16>;
    default: return (const void*)fast::kf_pencil<256, 16>;
  }
}

static cudaError_t iteration(Run& r, int w, const Wig* wig, bool with_source, float2 A, const StopRule& rule,
                             const Hist& h) {
  r.ia.w = wig[w];
  r.oa.w = wig[w];
  const float2* src = with_source ? r.src : nullptr;
  const float2* dEc = r.dE;
  const DevState* stc = r.st;
  {
    void* args[] = {&r.ia, &dEc, &src, &A, &r.T, &stc};
    const void* gen = r.sh.rset == kPow2 ? (const void*)k_fwd_inner<16, kPow2> : (const void*)k_fwd_inner<16, kMixed>;
    cudaError_t e = launch_inner(r, false, args, r.sh.fast ? fast_fwd(r.sh) : nullptr, gen,
                                 r.sh.fast ? fast::kThreads : r.sh.th);
    if (e != cudaSuccess) return e;
  }
  {
    void* args[] = {&r.oa, &r.T, &stc};
    if (r.sh.fast_pencil) {
      const int no = r.sh.mode3d ? r.g.nz : r.g.nx;
      cudaError_t e = cudaLaunchKernel(fast_pencil(no), dim3((unsigned)r.sh.grid_outer), dim3(16 * (no / 16)), args,
                                       r.sh.smem_outer, r.stream);
      if (e != cudaSuccess) return e;
    } else {
      const void* gen = r.sh.rset == kPow2 ? (const void*)k_outer<16, kPow2> : (const void*)k_outer<16, kMixed>;
      const int no = r.sh.mode3d ? r.g.nz : r.g.nx;
      long long e_ = (long long)r.g.nc * r.sh.ty * no;
      int th = (int)std::max(32LL, std::min(512LL, ((e_ + 15) / 16 + 31) / 32 * 32));
      cudaError_t e = cudaLaunchKernel(gen, dim3((unsigned)r.sh.grid_outer), dim3(th), args, r.sh.smem_outer, r.stream);
      if (e != cudaSuccess) return e;
    }
  }
  {
    const float2* Tc = r.T;
    void* args[] = {&r.ia, &Tc, &r.dE, &r.E, &r.gamma, &stc, &r.partials};
    const void* gen = r.sh.rset == kPow2 ? (const void*)k_inv_inner<16, kPow2> : (const void*)k_inv_inner<16, kMixed>;
    cudaError_t e =
        launch_inner(r, true, args, r.sh.fast ? fast_inv(r.sh) : nullptr, gen, r.sh.fast ? fast::kThreads : r.sh.th);
    if (e != cudaSuccess) return e;
  }
  k_finish_iteration<<<1, 256, 0, r.stream>>>(r.st, rule, h, r.partials, (int)r.sh.grid_inner);
  return cudaGetLastError();
}

}  // namespace noalloc
}  // namespace ws

using namespace ws;
using namespace ws::noalloc;

extern "C" const char* ws_noalloc_last_error(void) { return t_error.c_str(); }

extern "C" int64_t ws_noalloc_scratch_bytes(void) { return (int64_t)kScratchBytes; }

extern "C" int ws_run_algorithm_noalloc(const int64_t N[4], const ws_complex* gamma, int64_t n_wiggles,
                                        const ws_wiggle* wiggles, const ws_complex* source_field, float epsilon,
                                        ws_complex k02e, const int64_t roi[8], int64_t max_iterations,
                                        double energy_threshold, int64_t energy_interval, ws_complex* E_out,
                                        double* diff_energy_out, int64_t* n_iterations, int* converged,
                                        void* stream) {
  if (!N || !gamma || !wiggles || !source_field || !roi || !E_out || !diff_energy_out)
    return fail(WS_ERR_INVALID_ARGUMENT, "null argument");
  if (n_wiggles < 1 || n_wiggles > 64) return fail(WS_ERR_INVALID_ARGUMENT, "Nwiggles must be in [1, 64]");
  if (max_iterations < 1 || max_iterations > 100000000LL || energy_interval < 1)
    return fail(WS_ERR_INVALID_ARGUMENT, "bad max_iterations or energy_interval");
  Geom g{};
  for (int d = 0; d < 4; ++d)
    if (N[d] < 1) return fail(WS_ERR_INVALID_ARGUMENT, "N must be positive");
  if (N[3] != 1 && N[3] != 3) return fail(WS_ERR_INVALID_ARGUMENT, "N(4) must be 1 or 3");
  if (N[0] > 65536 || N[1] > 65536 || N[2] > 65536) return fail(WS_ERR_UNSUPPORTED, "dimension above 65536");
  g.ny = (int)N[0];
  g.nx = (int)N[1];
  g.nz = (int)N[2];
  g.nc = (int)N[3];
  g.npts = (long long)g.ny * g.nx * g.nz;
  for (int d = 0; d < 4; ++d) {
    if (roi[2 * d] < 1 || roi[2 * d + 1] < roi[2 * d] || roi[2 * d + 1] > N[d])
      return fail(WS_ERR_INVALID_ARGUMENT, "roi outside the grid");
    g.r0[d] = (int)(roi[2 * d] - 1);
    g.r1[d] = (int)roi[2 * d + 1];
  }
  FftPlan py{}, pxl{}, po{}, px{};
  Shape sh;
  if (shape_for(g, sh) != WS_OK) return fail(WS_ERR_UNSUPPORTED, "grid shape not supported");
  const int no = sh.mode3d ? g.nz : g.nx;
  const int nxl = sh.mode3d ? g.nx / sh.csize : 1;
  if (!plan(g.ny, py) || !plan(g.nx, px) || !plan(nxl, pxl) || !plan(no, po))
    return fail(WS_ERR_UNSUPPORTED, "grid dimension has a prime factor above 13");
  // scratch layout: dE | T | twiddles (y, x, x-local, outer) | state | per-block energies
  const size_t field = (size_t)g.npts * g.nc;
  const size_t ntw = (size_t)g.ny + g.nx + nxl + no;
  const size_t need = 2 * field * sizeof(float2) + ntw * sizeof(float2) + 256 + sizeof(DevState) + 256 +
                      (size_t)sh.grid_inner * sizeof(double) + 256 + sizeof(int);
  if (need > kScratchBytes)
    return fail(WS_ERR_INVALID_ARGUMENT, "grid too large for the static scratch array (" +
                                             std::to_string(need) + " > " + std::to_string(kScratchBytes) +
                                             " bytes: at most about " + std::to_string(kScratchBytes / 16) +
                                             " field elements)");
  int dev = 0;
  NA_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return fail(WS_ERR_INVALID_ARGUMENT, "device ordinal above 63");
  int rc = WS_OK;
  {
    // the per-device lookup runs once; the lock keeps two host threads that
    // make their first call on a device at the same time from racing on it
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[dev]) {
      void* p = nullptr;
      NA_CUDA(cudaGetSymbolAddress(&p, g_ws_scratch));  // device address of the array on this device
      g_scratch_addr[dev] = p;
    }
    rc = set_attributes(dev);
  }
  if (rc) return rc;
  cudaStream_t s = (cudaStream_t)stream;
  char* base = (char*)g_scratch_addr[dev];
  Run r{};
  r.g = g;
  r.sh = sh;
  r.dE = (float2*)base;
  r.T = r.dE + field;
  float2* tw = r.T + field;
  r.st = (DevState*)(((uintptr_t)(tw + ntw) + 255) & ~(uintptr_t)255);
  r.partials = (double*)(((uintptr_t)(r.st + 1) + 255) & ~(uintptr_t)255);
  // set by a fast kernel whose bounded cluster or barrier wait gave up
  int* d_err = (int*)(((uintptr_t)(r.partials + sh.grid_inner) + 255) & ~(uintptr_t)255);
  r.E = (float2*)E_out;
  r.src = (float2*)source_field;
  r.gamma = (const float2*)gamma;
  r.stream = s;
  // twiddle tables on the device
  float2* twy = tw;
  float2* twx = twy + g.ny;
  float2* twxl = twx + g.nx;
  float2* two = twxl + nxl;
  const int lens[4] = {g.ny, g.nx, nxl, no};
  float2* outs[4] = {twy, twx, twxl, two};
  for (int i = 0; i < 4; ++i) {
    k_twiddles<<<std::max(1, std::min(1024, (lens[i] + 255) / 256)), 256, 0, s>>>(outs[i], lens[i]);
    NA_CUDA(cudaGetLastError());
  }
  py.tw = twy;
  pxl.tw = twxl;
  po.tw = two;
  // clear what must start at zero: dE, E (the caller's output), the loop state
  NA_CUDA(cudaMemsetAsync(r.dE, 0, field * sizeof(float2), s));
  NA_CUDA(cudaMemsetAsync(r.E, 0, field * sizeof(float2), s));
  NA_CUDA(cudaMemsetAsync(d_err, 0, sizeof(int), s));
  k_reset_state<<<1, 32, 0, s>>>(r.st, 1);
  NA_CUDA(cudaGetLastError());
  Wig wig[64];
  for (int w = 0; w < n_wiggles; ++w) {
    const ws_wiggle& W = wiggles[w];
    if (!W.pxe || !W.pye || !W.pze || !W.gx || !W.gy || !W.gz) return fail(WS_ERR_INVALID_ARGUMENT, "null wiggle");
    wig[w] = Wig{W.pxe, W.pye, W.pze, (const float2*)W.gx, (const float2*)W.gy, (const float2*)W.gz};
  }
  r.ia.g = g;
  r.ia.py = py;
  r.ia.pxl = pxl;
  r.ia.twx = twx;
  r.ia.csize = sh.csize;
  r.ia.mode3d = sh.mode3d;
  r.ia.ncols = sh.ncols;
  r.ia.bpr = (int)sh.grid_inner;  // a single right-hand side
  r.ia.fstride = 0;
  r.ia.err = d_err;
  r.oa.g = g;
  r.oa.po = po;
  r.oa.k02e = make_float2(k02e.re, k02e.im);
  r.oa.norm = (float)(1.0 / (double)g.npts);
  r.oa.ty = sh.ty;
  r.oa.mode3d = sh.mode3d;
  r.oa.bpr = (int)sh.grid_outer;
  r.oa.fstride = 0;
  StopRule rule{};
  rule.nw = (int)n_wiggles;
  rule.fresh = 0;
  rule.nan_stop = 1;
  rule.interval = (int)std::min<int64_t>(energy_interval, 1 << 30);
  rule.max_iter = max_iterations;
  rule.threshold = energy_threshold;
  Hist h{diff_energy_out, nullptr, max_iterations + n_wiggles, 0};
  const float2 A = make_float2(0.f, (float)(1.0f / epsilon / (float)n_wiggles));
  const long long max_cycles = (max_iterations + n_wiggles - 1) / n_wiggles + 1;
  DevState hs{};
  int kerr = 0;
  long long it = 0;
  for (long long cycle = 0;; ++cycle) {
    if (cycle >= max_cycles) return fail(WS_ERR_CUDA, "loop did not stop within max_iterations (internal error)");
    for (int i = 0; i < n_wiggles; ++i, ++it) NA_CUDA(iteration(r, i, wig, it < n_wiggles, A, rule, h));
    NA_CUDA(cudaMemcpyAsync(&hs, r.st, sizeof(DevState), cudaMemcpyDeviceToHost, s));
    NA_CUDA(cudaMemcpyAsync(&kerr, d_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    NA_CUDA(cudaStreamSynchronize(s));
    if (kerr) return fail(WS_ERR_CUDA, "a cluster exchange of the FFT kernels timed out");
    if (hs.done) break;
  }
  if (n_iterations) *n_iterations = hs.it - 1;
  if (converged) *converged = hs.converged;
  if (hs.status == WS_ERR_DIVERGED) return fail(WS_ERR_DIVERGED, "residual energy is not finite");
  return WS_OK;
}
