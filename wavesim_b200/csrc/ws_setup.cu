// Medium set-up on the device (no counterpart in the reference, which does
// it in MATLAB on the host): from the refractive index of the ROI to the
// full-grid gamma = (i/epsilon) V .* F of WaveSimBase.m:58-81 and 217-258,
//   e_r = n^2 (Medium.m:44), replicated into the boundary layers
//   (padarray 'replicate', Medium.m:62), V = e_r k0^2 - k0c^2 - i epsilon
//   (WaveSimBase.m:72-73), F = fy(y) fx(x) fz(z) the separable ARL edge
//   window (WaveSimBase.m:217-258, the 1-D windows come from the host),
// in double precision, rounded to complex64 once at the end as the host
// path does.  Plus the two reductions the host needs for k0c and epsilon
// (Medium.m:45-47, WaveSimBase.m:201-215).
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "wavesim_b200.h"

namespace {

thread_local std::string t_err;

int setup_fail(int code, const std::string& msg) {
  t_err = msg;
  return code;
}

// order-preserving map of doubles to unsigned 64-bit keys (for atomicMax/Min)
__device__ __forceinline__ unsigned long long dkey(double v) {
  const unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__host__ __device__ inline double dval(unsigned long long k) {
  const unsigned long long b = (k >> 63) ? (k & 0x7fffffffffffffffull) : ~k;
  double d;
  memcpy(&d, &b, sizeof d);
  return d;
}

__device__ __forceinline__ double2 load_n(const void* n, int is_complex, long long i) {
  if (is_complex) return reinterpret_cast<const double2*>(n)[i];
  return make_double2(reinterpret_cast<const double*>(n)[i], 0.0);
}

// out[0] = min real(n^2), out[1] = max real(n^2), out[2] = max |n^2 k0^2 - k0c^2|
// (the last only when k0sq > 0); out[] as order-preserving keys
__global__ void k_medium_reduce(const void* __restrict__ n, int is_complex, long long count, double k0sq,
                                double k0c2, unsigned long long* __restrict__ out) {
  double mn = 1e300, mx = -1e300, ma = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < count;
       i += (long long)gridDim.x * blockDim.x) {
    const double2 v = load_n(n, is_complex, i);
    const double er = v.x * v.x - v.y * v.y, ei = 2.0 * v.x * v.y;
    mn = fmin(mn, er);
    mx = fmax(mx, er);
    if (k0sq > 0) ma = fmax(ma, hypot(er * k0sq - k0c2, ei * k0sq));
  }
  for (int o = 16; o > 0; o >>= 1) {
    mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
    mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    ma = fmax(ma, __shfl_xor_sync(0xffffffffu, ma, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(out, dkey(mn));
    atomicMax(out + 1, dkey(mx));
    atomicMax(out + 2, dkey(ma));
  }
}

struct GammaArgs {
  int N[3];   // grid (y, x, z)
  int R[3];   // ROI size
  int lo[3];  // first ROI index (0-based)
  double k0sq, k0c2, eps;
};

__global__ void k_build_gamma(const void* __restrict__ n, int is_complex, const float* __restrict__ fy,
                              const float* __restrict__ fx, const float* __restrict__ fz, GammaArgs a,
                              float2* __restrict__ gamma) {
  const long long total = (long long)a.N[0] * a.N[1] * a.N[2];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
       i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i % a.N[0]);
    const long long r = i / a.N[0];
    const int x = (int)(r % a.N[1]);
    const int z = (int)(r / a.N[1]);
    const int yc = min(max(y - a.lo[0], 0), a.R[0] - 1);
    const int xc = min(max(x - a.lo[1], 0), a.R[1] - 1);
    const int zc = min(max(z - a.lo[2], 0), a.R[2] - 1);
    const double2 v = load_n(n, is_complex, yc + (long long)a.R[0] * (xc + (long long)a.R[1] * zc));
    const double er = v.x * v.x - v.y * v.y, ei = 2.0 * v.x * v.y;
    // V = e_r k0^2 - k0c^2 - i eps, gamma = (i / eps) V F
    const double vr = er * a.k0sq - a.k0c2, vi = ei * a.k0sq - a.eps;
    const double f = (double)fy[y] * (double)fx[x] * (double)fz[z];
    gamma[i] = make_float2((float)(-vi / a.eps * f), (float)(vr / a.eps * f));
  }
}

unsigned blocks_for(long long n) {
  long long b = (n + 255) / 256;
  return (unsigned)(b < 1 ? 1 : (b > 148 * 16 ? 148 * 16 : b));
}

}  // namespace

extern "C" {

const char* ws_setup_last_error(void) { return t_err.c_str(); }

int ws_medium_reduce(const void* n, int is_complex, int64_t count, double k0sq, double k0c2, double out[3],
                     void* stream) {
  if (!n || !out || count < 1) return setup_fail(WS_ERR_INVALID_ARGUMENT, "ws_medium_reduce: bad arguments");
  unsigned long long* d = nullptr;
  cudaError_t e = cudaMallocAsync(&d, 3 * sizeof(unsigned long long), (cudaStream_t)stream);
  if (e != cudaSuccess) return setup_fail(WS_ERR_OUT_OF_MEMORY, cudaGetErrorString(e));
  const unsigned long long init[3] = {~0ull, 0ull, 0ull};
  cudaMemcpyAsync(d, init, sizeof(init), cudaMemcpyHostToDevice, (cudaStream_t)stream);
  k_medium_reduce<<<blocks_for(count), 256, 0, (cudaStream_t)stream>>>(n, is_complex, count, k0sq, k0c2, d);
  unsigned long long h[3] = {0, 0, 0};
  cudaMemcpyAsync(h, d, sizeof(h), cudaMemcpyDeviceToHost, (cudaStream_t)stream);
  e = cudaStreamSynchronize((cudaStream_t)stream);
  cudaFreeAsync(d, (cudaStream_t)stream);
  if (e != cudaSuccess) return setup_fail(WS_ERR_CUDA, cudaGetErrorString(e));
  for (int i = 0; i < 3; ++i) out[i] = dval(h[i]);
  if (!(k0sq > 0)) out[2] = 0.0;
  return WS_OK;
}

int ws_build_gamma(const void* n, int is_complex, const int64_t roi_size[3], const int64_t N[3],
                   const int64_t roi_lo[3], const float* fy, const float* fx, const float* fz, double k0sq,
                   double k0c2, double epsilon, void* gamma, void* stream) {
  if (!n || !roi_size || !N || !roi_lo || !fy || !fx || !fz || !gamma || !(epsilon > 0))
    return setup_fail(WS_ERR_INVALID_ARGUMENT, "ws_build_gamma: bad arguments");
  GammaArgs a{};
  for (int d = 0; d < 3; ++d) {
    if (N[d] < 1 || N[d] > (1 << 30) || roi_size[d] < 1 || roi_lo[d] < 0 || roi_lo[d] + roi_size[d] > N[d])
      return setup_fail(WS_ERR_INVALID_ARGUMENT, "ws_build_gamma: the ROI must lie inside the grid");
    a.N[d] = (int)N[d];
    a.R[d] = (int)roi_size[d];
    a.lo[d] = (int)roi_lo[d];
  }
  a.k0sq = k0sq;
  a.k0c2 = k0c2;
  a.eps = epsilon;
  k_build_gamma<<<blocks_for((long long)N[0] * N[1] * N[2]), 256, 0, (cudaStream_t)stream>>>(
      n, is_complex, fy, fx, fz, a, (float2*)gamma);
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return setup_fail(WS_ERR_CUDA, cudaGetErrorString(e));
  return WS_OK;
}

}  // extern "C"
