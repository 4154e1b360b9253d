// Tensor-core kernels of the learned warm start (sm_100a, tcgen05 + TMEM).
//
// ws_gemm_bf16: C[M][N] (fp32) = A[M][K] . B[N][K]^T with A and B bf16,
// K contiguous (K-major), K a multiple of 64.  One block computes a
// 128 x 128 tile with 4 warps:
//   * the threads stage A and B tiles of 128 x 64 bf16 into shared memory in
//     the 128-byte swizzled K-major layout the tensor core reads (16-byte
//     chunk c of row r at r*128 + ((c ^ (r & 7)) * 16), 1024-byte atoms),
//     double buffered;
//   * one thread issues tcgen05.mma (kind::f16, M = 128, N = 128, K = 16,
//     four per 64-wide K step) accumulating in tensor memory (128 lanes x 128
//     fp32 columns) and tcgen05.commit's to the stage's mbarrier;
//   * the epilogue reads the accumulator with tcgen05.ld (warp w owns lanes
//     32w..32w+31, i.e. rows) and applies bias / activation on the way out.
// Every mbarrier wait is bounded (about 2 s of clock); on expiry the kernel
// records an error flag, still frees its tensor memory and returns.
//
// The convolution layers of the network are implicit in these GEMMs:
// forward  out[vox][co]   = im2col(in)[vox][27 ci] . W[co][27 ci]^T
// dgrad    dcol[vox][27ci] = dout[vox][co] . Wt[27 ci][co]^T, then col2im
// wgrad    dW[co][27 ci]   = doutT[co][vox] . colT[27 ci][vox]^T
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "wavesim_b200.h"

namespace ws {
namespace net {

constexpr int BM = 128, BN = 128, BK = 64;
constexpr int kGemmThreads = 128;
constexpr unsigned kTileBytes = BM * BK * 2;  // 16 KB per operand tile
constexpr unsigned kSmemBytes = 4 * kTileBytes + 1024;

thread_local std::string t_err;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// UMMA shared-memory descriptor: K-major, 128-byte swizzle, 8-row groups
// 1024 bytes apart (stride byte offset), descriptor version 1.
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr) {
  uint64_t d = 0;
  d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
  d |= (uint64_t)1 << 16;                         // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)((1024u >> 4) & 0x3FFFu) << 32;  // stride byte offset
  d |= (uint64_t)1 << 46;                         // version
  d |= (uint64_t)2 << 61;                         // SWIZZLE_128B
  return d;
}

// instruction descriptor: D f32, A bf16, B bf16, both K-major, N = 128, M = 128
constexpr uint32_t kIdesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

// Waits for phase `parity` of the barrier; gives up after ~2e9 cycles.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t addr = smem_u32(bar);
  const long long t0 = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > 2000000000LL) return false;
  }
}

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
      ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc));
}

__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Stage rows [r0, r0 + 128) x columns [k0, k0 + 64) of a K-major bf16
// matrix (rows >= nrows are zero) into a swizzled tile.
__device__ __forceinline__ void stage_tile(uint8_t* tile, const __nv_bfloat16* __restrict__ X, long long ld, int r0,
                                           int nrows, int k0, int tid) {
#pragma unroll
  for (int i = 0; i < (BM * 8) / kGemmThreads; ++i) {
    const int q = tid + kGemmThreads * i;
    const int row = q >> 3, c = q & 7;
    uint4 val = make_uint4(0u, 0u, 0u, 0u);
    if (r0 + row < nrows) val = __ldg(reinterpret_cast<const uint4*>(X + (long long)(r0 + row) * ld + k0 + c * 8));
    *reinterpret_cast<uint4*>(tile + row * 128 + ((c ^ (row & 7)) << 4)) = val;
  }
}

// Epilogue modes
enum { EPI_STORE = 0, EPI_BIAS_RELU_BF16 = 1, EPI_BIAS_BF16 = 2, EPI_BIAS_F32 = 3 };

__global__ void __launch_bounds__(kGemmThreads, 1)
    k_gemm_bf16(const __nv_bfloat16* __restrict__ A, const __nv_bfloat16* __restrict__ B, float* __restrict__ C,
                __nv_bfloat16* __restrict__ Cb, const float* __restrict__ bias, int M, int N, int K, long long lda,
                long long ldb, long long ldc, int mode, int* __restrict__ err) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  uint8_t* sA[2] = {base, base + kTileBytes};
  uint8_t* sB[2] = {base + 2 * kTileBytes, base + 3 * kTileBytes};
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmem_base_s;
  __shared__ int failed;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                 "r"(BN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    mbar_init(&mbar[0], 1);
    mbar_init(&mbar[1], 1);
    failed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_s;
  const int nk = K / BK;
  for (int kt = 0; kt < nk; ++kt) {
    const int s = kt & 1;
    if (kt >= 2) {
      // the MMAs that read this stage two steps ago must be done
      if (tid == 0 && !mbar_wait(&mbar[s], (uint32_t)(((kt >> 1) - 1) & 1))) failed = 1;
      __syncthreads();
      if (failed) break;
    }
    stage_tile(sA[s], A, lda, m0, M, kt * BK, tid);
    stage_tile(sB[s], B, ldb, n0, N, kt * BK, tid);
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = smem_u32(sA[s]), b0 = smem_u32(sB[s]);
#pragma unroll
      for (int k = 0; k < BK / 16; ++k)
        mma_bf16(tmem, make_desc(a0 + 32 * k), make_desc(b0 + 32 * k), kIdesc, (kt > 0 || k > 0) ? 1u : 0u);
      mma_commit(&mbar[s]);
    }
  }
  if (!failed && nk > 0) {
    const int s = (nk - 1) & 1;
    if (tid == 0 && !mbar_wait(&mbar[s], (uint32_t)(((nk - 1) >> 1) & 1))) failed = 1;
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!failed) {
    const int row = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c0 = 0; c0 < BN; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      if (row < M) {
#pragma unroll
        for (int j = 0; j < 16; ++j) {
          const int col = n0 + c0 + j;
          if (col >= N) continue;
          float x = v[j];
          if (mode != EPI_STORE && bias) x += bias[col];
          if (mode == EPI_BIAS_RELU_BF16) x = fmaxf(x, 0.f);
          if (mode == EPI_BIAS_RELU_BF16 || mode == EPI_BIAS_BF16)
            Cb[(long long)row * ldc + col] = __float2bfloat16_rn(x);
          else
            C[(long long)row * ldc + col] = x;
        }
      }
    }
  } else if (tid == 0) {
    atomicExch(err, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(BN));
}


// ----------------------------------------------------------------------------
// Layer kernels (channels-last activations: x[((b*D + z)*H + y)*W + x][c])
// ----------------------------------------------------------------------------
struct Vol {
  int b, d, h, w;  // batch, depth (z), height (y), width (x)
};

__device__ __forceinline__ long long vox_index(const Vol& v, int b, int z, int y, int x) {
  return (((long long)b * v.d + z) * v.h + y) * v.w + x;
}

// im2col for a 3x3x3 convolution with zero padding 1:
// col[vox][((dz*3 + dy)*3 + dx)*C + c] = in[vox + (dz-1, dy-1, dx-1)][c], K padded to kp with zeros.
__global__ void k_im2col3(const __nv_bfloat16* __restrict__ in, __nv_bfloat16* __restrict__ col, Vol v, int C, int kp) {
  const long long nvox = (long long)v.b * v.d * v.h * v.w;
  const long long total = nvox * kp;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const long long vox = i / kp;
    const int k = (int)(i - vox * kp);
    __nv_bfloat16 val = __float2bfloat16_rn(0.f);
    if (k < 27 * C) {
      const int tap = k / C, c = k - tap * C;
      const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
      long long r = vox;
      const int x = (int)(r % v.w); r /= v.w;
      const int y = (int)(r % v.h); r /= v.h;
      const int z = (int)(r % v.d);
      const int b = (int)(r / v.d);
      const int zz = z + dz, yy = y + dy, xx = x + dx;
      if (zz >= 0 && zz < v.d && yy >= 0 && yy < v.h && xx >= 0 && xx < v.w)
        val = in[vox_index(v, b, zz, yy, xx) * C + c];
    }
    col[i] = val;
  }
}

// Gradient of im2col3 (a gather, no atomics):
// din[u][c] = sum over taps t of dcol[u - (t - 1)][t*C + c].
__global__ void k_col2im3(const float* __restrict__ dcol, float* __restrict__ din, Vol v, int C, int kp) {
  const long long nvox = (long long)v.b * v.d * v.h * v.w;
  const long long total = nvox * C;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const long long u = i / C;
    const int c = (int)(i - u * C);
    long long r = u;
    const int x = (int)(r % v.w); r /= v.w;
    const int y = (int)(r % v.h); r /= v.h;
    const int z = (int)(r % v.d);
    const int b = (int)(r / v.d);
    float acc = 0.f;
    for (int t = 0; t < 27; ++t) {
      const int dz = t / 9 - 1, dy = (t / 3) % 3 - 1, dx = t % 3 - 1;
      const int zz = z - dz, yy = y - dy, xx = x - dx;
      if (zz >= 0 && zz < v.d && yy >= 0 && yy < v.h && xx >= 0 && xx < v.w)
        acc += dcol[vox_index(v, b, zz, yy, xx) * kp + t * C + c];
    }
    din[i] = acc;
  }
}

// out[r][c] = in[c][r] (bf16 or fp32 source, bf16 out), rows padded: in is rows x cols with leading dim ldi
__global__ void k_transpose_f32_bf16(const float* __restrict__ in, __nv_bfloat16* __restrict__ out, long long rows,
                                     long long cols, long long ldo) {
  // out[c][r] = in[r][c] for r < rows, c < cols; out has leading dimension ldo (>= rows, padded entries set to 0)
  const long long total = cols * ldo;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const long long c = i / ldo, r = i - c * ldo;
    out[i] = r < rows ? __float2bfloat16_rn(in[r * cols + c]) : __float2bfloat16_rn(0.f);
  }
}
__global__ void k_transpose_bf16(const __nv_bfloat16* __restrict__ in, __nv_bfloat16* __restrict__ out, long long rows,
                                 long long cols, long long ldi, long long ldo) {
  const long long total = cols * ldo;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const long long c = i / ldo, r = i - c * ldo;
    out[i] = r < rows ? in[r * ldi + c] : __float2bfloat16_rn(0.f);
  }
}

// 2x2x2 average pooling (channels-last) and its gradient
__global__ void k_avgpool2(const __nv_bfloat16* __restrict__ in, __nv_bfloat16* __restrict__ out, Vol vo, int C) {
  const long long total = (long long)vo.b * vo.d * vo.h * vo.w * C;
  const Vol vi{vo.b, vo.d * 2, vo.h * 2, vo.w * 2};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    long long r = i / C;
    const int x = (int)(r % vo.w); r /= vo.w;
    const int y = (int)(r % vo.h); r /= vo.h;
    const int z = (int)(r % vo.d);
    const int b = (int)(r / vo.d);
    float acc = 0.f;
    for (int q = 0; q < 8; ++q)
      acc += __bfloat162float(in[vox_index(vi, b, 2 * z + (q >> 2), 2 * y + ((q >> 1) & 1), 2 * x + (q & 1)) * C + c]);
    out[i] = __float2bfloat16_rn(0.125f * acc);
  }
}
__global__ void k_avgpool2_grad(const float* __restrict__ dout, float* __restrict__ din, Vol vi, int C) {
  const long long total = (long long)vi.b * vi.d * vi.h * vi.w * C;
  const Vol vo{vi.b, vi.d / 2, vi.h / 2, vi.w / 2};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    long long r = i / C;
    const int x = (int)(r % vi.w); r /= vi.w;
    const int y = (int)(r % vi.h); r /= vi.h;
    const int z = (int)(r % vi.d);
    const int b = (int)(r / vi.d);
    din[i] = 0.125f * dout[vox_index(vo, b, z / 2, y / 2, x / 2) * C + c];
  }
}
// nearest x2 upsampling of `a` (Ca channels at half resolution) concatenated with `skip` (Cs channels)
__global__ void k_upcat(const __nv_bfloat16* __restrict__ a, const __nv_bfloat16* __restrict__ skip,
                        __nv_bfloat16* __restrict__ out, Vol vo, int Ca, int Cs) {
  const int C = Ca + Cs;
  const long long total = (long long)vo.b * vo.d * vo.h * vo.w * C;
  const Vol vh{vo.b, vo.d / 2, vo.h / 2, vo.w / 2};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % C);
    const long long u = i / C;
    if (c < Ca) {
      long long r = u;
      const int x = (int)(r % vo.w); r /= vo.w;
      const int y = (int)(r % vo.h); r /= vo.h;
      const int z = (int)(r % vo.d);
      const int b = (int)(r / vo.d);
      out[i] = a[vox_index(vh, b, z / 2, y / 2, x / 2) * Ca + c];
    } else {
      out[i] = skip[u * Cs + (c - Ca)];
    }
  }
}
// gradient of k_upcat: da (half resolution, summed over the 8 children) and dskip
__global__ void k_upcat_grad(const float* __restrict__ dout, float* __restrict__ da, float* __restrict__ dskip,
                             Vol vo, int Ca, int Cs) {
  const int C = Ca + Cs;
  const Vol vh{vo.b, vo.d / 2, vo.h / 2, vo.w / 2};
  const long long nh = (long long)vh.b * vh.d * vh.h * vh.w * Ca;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nh; i += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(i % Ca);
    long long r = i / Ca;
    const int x = (int)(r % vh.w); r /= vh.w;
    const int y = (int)(r % vh.h); r /= vh.h;
    const int z = (int)(r % vh.d);
    const int b = (int)(r / vh.d);
    float acc = 0.f;
    for (int q = 0; q < 8; ++q)
      acc += dout[vox_index(vo, b, 2 * z + (q >> 2), 2 * y + ((q >> 1) & 1), 2 * x + (q & 1)) * C + c];
    da[i] = acc;
  }
  const long long ns = (long long)vo.b * vo.d * vo.h * vo.w * Cs;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < ns; i += (long long)gridDim.x * blockDim.x) {
    const long long u = i / Cs;
    const int c = (int)(i - u * Cs);
    dskip[i] = dout[u * C + Ca + c];
  }
}
// dx = dy * (y > 0) for a ReLU output y (bf16); in place on dy allowed
__global__ void k_relu_grad(float* __restrict__ dy, const __nv_bfloat16* __restrict__ y, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    if (!(__bfloat162float(y[i]) > 0.f)) dy[i] = 0.f;
}
// db[c] = sum over rows of dy[row][c]
__global__ void k_bias_grad(const float* __restrict__ dy, float* __restrict__ db, long long rows, int C) {
  const int c = blockIdx.x;
  float acc = 0.f;
  for (long long r = threadIdx.x; r < rows; r += blockDim.x) acc += dy[r * C + c];
  __shared__ float red[256];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) db[c] = red[0];
}
// Adam on fp32 master weights; writes the bf16 copy used by the GEMMs
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ g, float* __restrict__ m, float* __restrict__ v,
                       __nv_bfloat16* __restrict__ wb, long long n, float lr, float b1, float b2, float eps, float bc1,
                       float bc2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float wi = w[i] - lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    w[i] = wi;
    if (wb) wb[i] = __float2bfloat16_rn(wi);
  }
}
// mean squared error of pred (fp32, rows x cols with leading dim ldp) against target; grad = 2 (pred - t) / n
__global__ void k_mse(const float* __restrict__ pred, const float* __restrict__ t, float* __restrict__ grad,
                      double* __restrict__ loss, long long rows, int cols, long long ldp) {
  const long long n = rows * cols;
  double acc = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const long long r = i / cols;
    const int c = (int)(i - r * cols);
    const float d = pred[r * ldp + c] - t[i];
    grad[r * ldp + c] = 2.f * d / (float)n;
    acc += (double)d * d;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, acc / (double)n);
}
__global__ void k_f32_to_bf16(const float* __restrict__ in, __nv_bfloat16* __restrict__ out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = __float2bfloat16_rn(in[i]);
}

static unsigned grid_for(long long n) {
  long long g = (n + 255) / 256;
  return (unsigned)(g < 1 ? 1 : (g > 148 * 32 ? 148 * 32 : g));
}

}  // namespace net
}  // namespace ws

using namespace ws::net;

extern "C" const char* ws_net_last_error(void) { return t_err.c_str(); }

// C = A . B^T (see the file comment); mode selects the epilogue: 0 store fp32
// C; 1 bias + ReLU -> bf16 Cb; 2 bias -> bf16 Cb; 3 bias -> fp32 C.
// err_flag (device int, may be NULL) is set to 1 if a wait timed out.
extern "C" int ws_gemm_bf16(const void* A, const void* B, float* C, void* Cb, const float* bias, int64_t M,
                            int64_t N, int64_t K, int64_t lda, int64_t ldb, int64_t ldc, int mode, int* err_flag,
                            void* stream) {
  if (M < 1 || N < 1 || K < 64 || K % 64 != 0 || M > (1LL << 30) || N > (1LL << 30)) {
    t_err = "ws_gemm_bf16: need M, N >= 1 and K a positive multiple of 64";
    return WS_ERR_INVALID_ARGUMENT;
  }
  if (lda % 8 || ldb % 8 || ((uintptr_t)A & 15) || ((uintptr_t)B & 15)) {
    t_err = "ws_gemm_bf16: A and B rows must be 16-byte aligned";
    return WS_ERR_INVALID_ARGUMENT;
  }
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_gemm_bf16, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes);
    if (e != cudaSuccess) {
      t_err = std::string("ws_gemm_bf16: ") + cudaGetErrorString(e);
      return WS_ERR_CUDA;
    }
    attr = true;
  }
  static int* dummy = nullptr;
  if (!err_flag) {
    if (!dummy && cudaMalloc(&dummy, sizeof(int)) != cudaSuccess) return WS_ERR_OUT_OF_MEMORY;
    err_flag = dummy;
  }
  dim3 grid((unsigned)((N + BN - 1) / BN), (unsigned)((M + BM - 1) / BM));
  k_gemm_bf16<<<grid, kGemmThreads, kSmemBytes, (cudaStream_t)stream>>>(
      (const __nv_bfloat16*)A, (const __nv_bfloat16*)B, C, (__nv_bfloat16*)Cb, bias, (int)M, (int)N, (int)K, lda, ldb,
      ldc, mode, err_flag);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    t_err = std::string("ws_gemm_bf16: ") + cudaGetErrorString(e);
    return WS_ERR_CUDA;
  }
  return WS_OK;
}

// Layer entry points: device pointers, channels-last volumes of
// (b, d, h, w) voxels, launched on `stream`.  Return WS_OK or WS_ERR_CUDA.
#define NET_LAUNCH_CHECK()                                   \
  do {                                                       \
    cudaError_t e__ = cudaGetLastError();                    \
    if (e__ != cudaSuccess) {                                \
      t_err = cudaGetErrorString(e__);                       \
      return WS_ERR_CUDA;                                    \
    }                                                        \
    return WS_OK;                                            \
  } while (0)

extern "C" int ws_net_im2col3(const void* in, void* col, int b, int d, int h, int w, int C, int kp, void* stream) {
  Vol v{b, d, h, w};
  k_im2col3<<<grid_for((long long)b * d * h * w * kp), 256, 0, (cudaStream_t)stream>>>(
      (const __nv_bfloat16*)in, (__nv_bfloat16*)col, v, C, kp);
  NET_LAUNCH_CHECK();
}
extern "C" int ws_net_col2im3(const float* dcol, float* din, int b, int d, int h, int w, int C, int kp, void* stream) {
  Vol v{b, d, h, w};
  k_col2im3<<<grid_for((long long)b * d * h * w * C), 256, 0, (cudaStream_t)stream>>>(dcol, din, v, C, kp);
  NET_LAUNCH_CHECK();
}
extern "C" int ws_net_transpose_f32_bf16(const float* in, void* out, int64_t rows, int64_t cols, int64_t ldo,
                                         void* stream) {
  k_transpose_f32_bf16<<<grid_for(cols * ldo), 256, 0, (cudaStream_t)stream>>>(in, (__nv_bfloat16*)out, rows, cols, ldo);
  NET_LAUNCH_CHECK();
}
extern "C" int ws_net_transpose_bf16(const void* in, void* out, int64_t rows, int64_t cols, int64_t ldi, int64_t ldo,
                                     void* stream) {
  k_transpose_bf16<<<grid_for(cols * ldo), 256, 0, (cudaStream_t)stream>>>((const __nv_bfloat16*)in,
                                                                           (__nv_bfloat16*)out, rows, cols, ldi, ldo);
  NET_LAUNCH_CHECK();
}
extern "C" int ws_net_avgpool2(const void* in, void* out, int b, int d, int h, int w, int C, void* stream) {
  Vol vo{b, d / 2, h / 2, w / 2};
  k_avgpool2<<<grid_for((long long)b * (d / 2) * (h / 2) * (w / 2) * C), 256, 0, (cudaStream_t)stream>>>(
      (const __nv_bfloat16*)in, (__nv_bfloat16*)out, vo, C);
  NET_LAUNCH_CHECK();
}
extern "C" int ws_net_avgpool2_grad(const float* dout, float* din, int b, int d, int h, int w, int C, void* stream) {
  Vol vi{b, d, h, w};
  k_avgpool2_grad<<<grid_for((long long)b * d * h * w * C), 256, 0, (cudaStream_t)stream>>>(dout, din, vi, C);
  NET_LAUNCH_CHECK();
}
extern "C" int ws_net_upcat(const void* a, const void* skip, void* out, int b, int d, int h, int w, int Ca, int Cs,
                            void* stream) {
  Vol vo{b, d, h, w};
  k_upcat<<<grid_for((long long)b * d * h * w * (Ca + Cs)), 256, 0, (cudaStream_t)stream>>>(
      (const __nv_bfloat16*)a, (const __nv_bfloat16*)skip, (__nv_bfloat16*)out, vo, Ca, Cs);
  NET_LAUNCH_CHECK();
}
extern "C" int ws_net_upcat_grad(const float* dout, float* da, float* dskip, int b, int d, int h, int w, int Ca,
                                 int Cs, void* stream) {
  Vol vo{b, d, h, w};
  k_upcat_grad<<<grid_for((long long)b * d * h * w * (Ca + Cs)), 256, 0, (cudaStream_t)stream>>>(dout, da, dskip, vo,
                                                                                                  Ca, Cs);
  NET_LAUNCH_CHECK();
}
extern "C" int ws_net_relu_grad(float* dy, const void* y, int64_t n, void* stream) {
  k_relu_grad<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(dy, (const __nv_bfloat16*)y, n);
  NET_LAUNCH_CHECK();
}
extern "C" int ws_net_bias_grad(const float* dy, float* db, int64_t rows, int C, void* stream) {
  k_bias_grad<<<C, 256, 0, (cudaStream_t)stream>>>(dy, db, rows, C);
  NET_LAUNCH_CHECK();
}
extern "C" int ws_net_adam(float* w, const float* g, float* m, float* v, void* wb, int64_t n, float lr, float b1,
                           float b2, float eps, int step, void* stream) {
  const float bc1 = 1.f - powf(b1, (float)step), bc2 = 1.f - powf(b2, (float)step);
  k_adam<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(w, g, m, v, (__nv_bfloat16*)wb, n, lr, b1, b2, eps, bc1, bc2);
  NET_LAUNCH_CHECK();
}
extern "C" int ws_net_mse(const float* pred, const float* target, float* grad, double* loss, int64_t rows, int cols,
                          int64_t ldp, void* stream) {
  k_mse<<<grid_for(rows * cols), 256, 0, (cudaStream_t)stream>>>(pred, target, grad, loss, rows, cols, ldp);
  NET_LAUNCH_CHECK();
}
extern "C" int ws_net_f32_to_bf16(const float* in, void* out, int64_t n, void* stream) {
  k_f32_to_bf16<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(in, (__nv_bfloat16*)out, n);
  NET_LAUNCH_CHECK();
}
