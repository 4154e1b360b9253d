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
// col[vox][((dz*3 + dy)*3 + dx)*C + c] = in[vox + (dz-1, dy-1, dx-1)][c], K
// padded to kp with zeros.  C % 8 == 0: one thread per 16-byte chunk (8
// channels of one tap) of a row, 32-bit voxel arithmetic.
__global__ void k_im2col3(const __nv_bfloat16* __restrict__ in, __nv_bfloat16* __restrict__ col, Vol v, int C, int kp) {
  const int cpr = kp >> 3;
  const long long nvox = (long long)v.b * v.d * v.h * v.w;
  const long long total = nvox * cpr;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const long long row = i / cpr;
    const int k = (int)(i - row * cpr) << 3;
    uint4 val = make_uint4(0u, 0u, 0u, 0u);
    const int tap = k / C;
    if (tap < 27) {
      const int c = k - tap * C;
      const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
      long long r = row;
      const int x = (int)(r % v.w); r /= v.w;
      const int y = (int)(r % v.h); r /= v.h;
      const int z = (int)(r % v.d);
      const int b = (int)(r / v.d);
      const int zz = z + dz, yy = y + dy, xx = x + dx;
      if (zz >= 0 && zz < v.d && yy >= 0 && yy < v.h && xx >= 0 && xx < v.w)
        val = *reinterpret_cast<const uint4*>(in + vox_index(v, b, zz, yy, xx) * C + c);
    }
    *reinterpret_cast<uint4*>(col + row * kp + k) = val;
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

// out[c][r] = in[r][c] through 32 x 32 shared-memory tiles (fp32 or bf16
// in, bf16 out); in has leading dimension ldi, out ldo >= rows, and out rows
// r >= rows (the padding up to ldo) are written as zeros.
template <typename TI>
__global__ void k_transpose_tiled(const TI* __restrict__ in, __nv_bfloat16* __restrict__ out, long long rows,
                                  long long cols, long long ldi, long long ldo) {
  __shared__ float tile[32][33];
  const long long r0 = (long long)blockIdx.x * 32, c0 = (long long)blockIdx.y * 32;
  const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8 threads
  for (int j = ty; j < 32; j += 8) {
    const long long r = r0 + j, c = c0 + tx;
    float val = 0.f;
    if (r < rows && c < cols) {
      if constexpr (sizeof(TI) == 4)
        val = (float)in[r * ldi + c];
      else
        val = __bfloat162float(in[r * ldi + c]);
    }
    tile[j][tx] = val;
  }
  __syncthreads();
  for (int j = ty; j < 32; j += 8) {
    const long long c = c0 + j, r = r0 + tx;
    if (c < cols && r < ldo) out[c * ldo + r] = __float2bfloat16_rn(tile[tx][j]);
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

// ----------------------------------------------------------------------------
// Implicit-GEMM 3x3x3 convolution (zero padding 1), forward:
//   out[vox][co] = sum_k A[vox][k] W[co][k],  k = tap * C + c,
//   tap = (dz * 3 + dy) * 3 + dx,  A[vox][k] = in[vox + (dz-1, dy-1, dx-1)][c]
// with A never written to memory: each 16-byte chunk (8 channels of one tap)
// of a 128-voxel x 64-k tile is gathered by cp.async straight into the
// 128-byte swizzled shared-memory layout the tensor core reads (zero-filled
// outside the volume).  The input may be the channel concat [nearest x2
// upsampling of U (Cu channels), X (Cx channels)] of a decoder level, read
// in place.  NT = output-channel tile (16..128), S-stage cp.async ring; one
// thread issues tcgen05.mma M=128 x N=NT x K=16 into tensor memory and
// commits each stage to its mbarrier, which the producers wait on (bounded)
// before they refill the stage.
// ----------------------------------------------------------------------------
struct ConvIn {
  const __nv_bfloat16* U;  // half-resolution part (Cu channels), may be null with Cu = 0
  const __nv_bfloat16* X;  // full-resolution part (Cx channels)
  int Cu, Cx;              // multiples of 8
  int b, d, h, w;          // output (and X) volume
};

__device__ __forceinline__ void cp_async16(uint32_t dst, const void* src, uint32_t nbytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(nbytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int NT>
struct ConvTile {
  static constexpr unsigned kA = BM * BK * 2;  // 16 KB
  static constexpr unsigned kB = NT * BK * 2;  // NT rows x 128 B
  static constexpr unsigned kStage = kA + kB;
  static constexpr uint32_t kCols = NT <= 32 ? 32 : (NT <= 64 ? 64 : 128);  // tensor-memory columns (power of 2)
  static constexpr uint32_t kIdesc =
      (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NT >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);
  static_assert(NT % 16 == 0 && NT >= 16 && NT <= 128, "N tile");
  static_assert(kB % 1024 == 0, "B tile must hold whole 8-row swizzle atoms");
};

template <int NT, int S>
constexpr unsigned conv_smem_bytes() {
  return S * ConvTile<NT>::kStage + 1024;
}

template <int NT, int S, bool UP>
__global__ void __launch_bounds__(kGemmThreads)
    k_conv3(ConvIn in, const __nv_bfloat16* __restrict__ W, const float* __restrict__ bias, float* __restrict__ out32,
            __nv_bfloat16* __restrict__ outb, int M, int Cout, int kp, int mode, int* __restrict__ err) {
  using T = ConvTile<NT>;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~(uintptr_t)1023);
  __shared__ __align__(8) uint64_t mbar[S];
  __shared__ uint32_t tmem_base_s;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.x * BM, n0 = blockIdx.y * NT;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base_s)),
                 "r"(T::kCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
#pragma unroll
    for (int i = 0; i < S; ++i) mbar_init(&mbar[i], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_base_s;
  const uint32_t sbase = smem_u32(base);

  // this thread's A chunk column and its 8 rows (voxels m0 + (tid >> 3) + 16 i)
  const int chunk = tid & 7;
  const int C = in.Cu + in.Cx;
  const int hd = in.d >> 1, hh = in.h >> 1, hw = in.w >> 1;
  // UP: the coordinates of each row (the upsampled part needs them per tap);
  // else the linear voxel index and a 27-bit mask of the taps that fall
  // inside the volume, so that a tap costs one add and one bit test per row
  constexpr int NR = UP ? 8 : 1;
  int vz[NR], vy[NR], vx[NR], vb[NR];
  int vlin[8];
  uint32_t vmask[8];
#pragma unroll
  for (int i = 0; i < 8; ++i) {
    const int vox = m0 + (tid >> 3) + 16 * i;
    int x = 0, y = 0, z = 0, b = -1;
    if (vox < M) {
      int r = vox;
      x = r % in.w; r /= in.w;
      y = r % in.h; r /= in.h;
      z = r % in.d;
      b = r / in.d;
    }
    if constexpr (UP) {
      vz[i] = z;
      vy[i] = y;
      vx[i] = x;
      vb[i] = b;
    } else {
      const uint32_t mz = (z > 0 ? 1u : 0u) | 2u | (z < in.d - 1 ? 4u : 0u);
      const uint32_t my = (y > 0 ? 1u : 0u) | 2u | (y < in.h - 1 ? 4u : 0u);
      const uint32_t mx = (x > 0 ? 1u : 0u) | 2u | (x < in.w - 1 ? 4u : 0u);
      uint32_t m = 0;
#pragma unroll
      for (int t = 0; t < 27; ++t) m |= ((mz >> (t / 9)) & (my >> ((t / 3) % 3)) & (mx >> (t % 3)) & 1u) << t;
      vmask[i] = b >= 0 ? m : 0u;
      vlin[i] = vox;
    }
  }
  const uint32_t swz = (uint32_t)((chunk ^ ((tid >> 3) & 7)) << 4);  // row & 7 is the same for all 8 rows

  auto load_stage = [&](int kt, int s) {
    const uint32_t sa = sbase + s * T::kStage, sb = sa + T::kA;
    const int k = kt * BK + chunk * 8;
    const int tap = k / C;
    const int ch = k - tap * C;
    const int dz = tap / 9 - 1, dy = (tap / 3) % 3 - 1, dx = tap % 3 - 1;
    if constexpr (UP) {
      const bool up = ch < in.Cu;
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int row = (tid >> 3) + 16 * i;
        const int z = vz[i] + dz, y = vy[i] + dy, x = vx[i] + dx;
        const bool ok = tap < 27 && vb[i] >= 0 && (unsigned)z < (unsigned)in.d && (unsigned)y < (unsigned)in.h &&
                        (unsigned)x < (unsigned)in.w;
        const __nv_bfloat16* src = in.X;
        if (ok) {
          if (up)
            src = in.U + ((((long long)vb[i] * hd + (z >> 1)) * hh + (y >> 1)) * hw + (x >> 1)) * in.Cu + ch;
          else
            src = in.X + ((((long long)vb[i] * in.d + z) * in.h + y) * in.w + x) * in.Cx + (ch - in.Cu);
        }
        cp_async16(sa + row * 128 + swz, src, ok ? 16u : 0u);
      }
    } else {
      const int toff = (dz * in.h + dy) * in.w + dx;
      const int tsh = tap < 27 ? tap : 31;  // bit 31 of a mask is never set
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int row = (tid >> 3) + 16 * i;
        const bool ok = (vmask[i] >> tsh) & 1u;
        const __nv_bfloat16* src = ok ? in.X + (long long)(vlin[i] + toff) * in.Cx + ch : in.X;
        cp_async16(sa + row * 128 + swz, src, ok ? 16u : 0u);
      }
    }
#pragma unroll
    for (int i = 0; i < (NT * 8) / kGemmThreads; ++i) {
      const int q = tid + kGemmThreads * i;
      const int row = q >> 3, c = q & 7;
      const bool ok = n0 + row < Cout;
      const __nv_bfloat16* src = ok ? W + (long long)(n0 + row) * kp + kt * BK + c * 8 : W;
      cp_async16(sb + row * 128 + ((c ^ (row & 7)) << 4), src, ok ? 16u : 0u);
    }
  };

  const int nk = kp / BK;
  bool failed = false;
#pragma unroll
  for (int p = 0; p < S - 1; ++p) {
    if (p < nk) load_stage(p, p);
    cp_async_commit();
  }
  for (int kt = 0; kt < nk; ++kt) {
    const int s = kt % S;
    const int kn = kt + S - 1;
    if (kn < nk) {
      // stage kn % S was last read by the MMAs of step kt - 1
      if (kt >= 1 && !mbar_wait(&mbar[(kt - 1) % S], (uint32_t)(((kt - 1) / S) & 1))) failed = true;
      if (!failed) load_stage(kn, kn % S);
    }
    cp_async_commit();
    cp_async_wait<S - 1>();  // this thread's chunks of step kt have landed
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (__syncthreads_or(failed)) {
      failed = true;
      break;
    }
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t a0 = sbase + s * T::kStage, b0 = a0 + T::kA;
#pragma unroll
      for (int k = 0; k < BK / 16; ++k)
        mma_bf16(tmem, make_desc(a0 + 32 * k), make_desc(b0 + 32 * k), T::kIdesc, (kt > 0 || k > 0) ? 1u : 0u);
      mma_commit(&mbar[s]);
    }
  }
  cp_async_wait<0>();
  if (!failed && nk > 0 && !mbar_wait(&mbar[(nk - 1) % S], (uint32_t)(((nk - 1) / S) & 1))) failed = true;
  failed = __syncthreads_or(failed);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (!failed) {
    const int row = m0 + warp * 32 + lane;
#pragma unroll 1
    for (int c0 = 0; c0 < NT; c0 += 16) {
      float v[16];
      tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)c0, v);
      const int col0 = n0 + c0;
      if (row >= M || col0 >= Cout) continue;
      if (mode != EPI_STORE && bias) {
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] += col0 + j < Cout ? bias[col0 + j] : 0.f;
      }
      if (mode == EPI_BIAS_RELU_BF16) {
#pragma unroll
        for (int j = 0; j < 16; ++j) v[j] = fmaxf(v[j], 0.f);
      }
      if (mode == EPI_BIAS_RELU_BF16 || mode == EPI_BIAS_BF16) {
        __nv_bfloat16* dst = outb + (long long)row * Cout + col0;
        if (col0 + 16 <= Cout && (Cout & 7) == 0) {
          uint32_t pk[8];
#pragma unroll
          for (int j = 0; j < 8; ++j) {
            __nv_bfloat162 t = __floats2bfloat162_rn(v[2 * j], v[2 * j + 1]);
            pk[j] = *reinterpret_cast<uint32_t*>(&t);
          }
          reinterpret_cast<uint4*>(dst)[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
          reinterpret_cast<uint4*>(dst)[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
        } else {
#pragma unroll
          for (int j = 0; j < 16; ++j)
            if (col0 + j < Cout) dst[j] = __float2bfloat16_rn(v[j]);
        }
      } else {
        float* dst = out32 + (long long)row * Cout + col0;
#pragma unroll
        for (int j = 0; j < 16; ++j)
          if (col0 + j < Cout) dst[j] = v[j];
      }
    }
  } else if (tid == 0) {
    atomicExch(err, 1);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(T::kCols));
}

// Network input features of a ROI (y fastest, then x, then z: the column-major
// order of the ROI, which is also the network's (z, x, y) voxel order):
// 8 bf16 channels per voxel [(n - n_bg) / 0.2, source amplitude, cos phi,
// sin phi, 0, 0, 0, 0] with phi(z) = k0 sum_{z' <= z} (n - n_bg) the phase of
// a straight ray from the z = 0 face.  src (ROI-sized, may be null: a plane
// of ones at z = 0).  One thread per (y, x) ray, marching in z.
__global__ void k_features(const float* __restrict__ n, const float* __restrict__ src, long long nray, int nz, float n_bg,
                           float k0, __nv_bfloat16* __restrict__ out) {
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < nray; t += (long long)gridDim.x * blockDim.x) {
    float phi = 0.f;
    for (int z = 0; z < nz; ++z) {
      const long long v = t + nray * z;
      const float dn = n[v] - n_bg;
      phi = fmaf(k0, dn, phi);
      float sp, cp;
      sincosf(phi, &sp, &cp);
      const float amp = src ? src[v] : (z == 0 ? 1.f : 0.f);
      __nv_bfloat162 p0 = __floats2bfloat162_rn(dn * 5.f, amp), p1 = __floats2bfloat162_rn(cp, sp);
      uint4 q = make_uint4(*reinterpret_cast<uint32_t*>(&p0), *reinterpret_cast<uint32_t*>(&p1), 0u, 0u);
      reinterpret_cast<uint4*>(out)[v] = q;
    }
  }
}

// Starting field psi0 on the full simulation grid (column-major, Ny x Nx x
// Nz) from the network output pred[vox][2] = envelope of the ROI field:
// psi0 = scale (pred_re + i pred_im) exp(i kz z_roi) inside the ROI; in the
// boundary layers the nearest ROI value times a cos^2 taper per dimension
// that falls to zero at the grid edge.
struct RoiMap {
  int N[3];   // grid (y, x, z)
  int r0[3];  // first ROI index (0-based)
  int rn[3];  // ROI size
};
__device__ __forceinline__ float taper(int j, int lo, int n, int N) {
  if (j < lo) {
    const float c = cospif(0.5f * (float)(lo - j) / (float)(lo + 1));
    return c * c;
  }
  const int hi = N - lo - n;
  if (j >= lo + n) {
    const float c = cospif(0.5f * (float)(j - (lo + n) + 1) / (float)(hi + 1));
    return c * c;
  }
  return 1.f;
}
__global__ void k_envelope_to_field(const float* __restrict__ pred, RoiMap m, float scale, float kz,
                                    float2* __restrict__ psi, int s2d) {
  const long long total = (long long)m.N[0] * m.N[1] * m.N[2];
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int y = (int)(i % m.N[0]);
    const long long r = i / m.N[0];
    const int x = (int)(r % m.N[1]);
    const int z = (int)(r / m.N[1]);
    const int yc = min(max(y - m.r0[0], 0), m.rn[0] - 1);
    const int xc = min(max(x - m.r0[1], 0), m.rn[1] - 1);
    const int zc = min(max(z - m.r0[2], 0), m.rn[2] - 1);
    const float w = scale * taper(y, m.r0[0], m.rn[0], m.N[0]) * taper(x, m.r0[1], m.rn[1], m.N[1]) *
                    taper(z, m.r0[2], m.rn[2], m.N[2]);
    long long v;
    if (s2d) {
      // half-resolution network output, sub-voxel s of the (z, x, y) volume at channels [2s, 2s + 2)
      const int hy = m.rn[0] >> 1, hx = m.rn[1] >> 1;
      const int s = ((zc & 1) * 2 + (xc & 1)) * 2 + (yc & 1);
      v = ((yc >> 1) + (long long)hy * ((xc >> 1) + (long long)hx * (zc >> 1))) * 8 + s;
    } else {
      v = yc + (long long)m.rn[0] * (xc + (long long)m.rn[1] * zc);
    }
    const float2 p = reinterpret_cast<const float2*>(pred)[v];
    float s, c;
    sincosf(kz * (float)zc, &s, &c);
    psi[i] = make_float2(w * (p.x * c - p.y * s), w * (p.x * s + p.y * c));
  }
}

// 2x2x2 average pooling, 8 channels (one 16-byte chunk) per thread
__global__ void k_avgpool2_v8(const __nv_bfloat16* __restrict__ in, __nv_bfloat16* __restrict__ out, Vol vo, int C) {
  const int cc = C >> 3;
  const long long total = (long long)vo.b * vo.d * vo.h * vo.w * cc;
  const int wi = vo.w * 2, hi = vo.h * 2;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int c8 = (int)(i % cc);
    long long r = i / cc;
    const int x = (int)(r % vo.w); r /= vo.w;
    const int y = (int)(r % vo.h); r /= vo.h;
    const long long bz = r;  // b * d + z of the output
    float acc[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const long long src = ((2 * bz + (q >> 2)) * hi + 2 * y + ((q >> 1) & 1)) * wi + 2 * x + (q & 1);
      const uint4 u = reinterpret_cast<const uint4*>(in + src * C)[c8];
      const __nv_bfloat162* h2 = reinterpret_cast<const __nv_bfloat162*>(&u);
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const float2 f = __bfloat1622float2(h2[j]);
        acc[2 * j] += f.x;
        acc[2 * j + 1] += f.y;
      }
    }
    uint32_t pk[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      __nv_bfloat162 t = __floats2bfloat162_rn(0.125f * acc[2 * j], 0.125f * acc[2 * j + 1]);
      pk[j] = *reinterpret_cast<uint32_t*>(&t);
    }
    reinterpret_cast<uint4*>(out)[i] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
  }
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
  if (C % 8 || kp % 8 || ((uintptr_t)in & 15) || ((uintptr_t)col & 15)) {
    t_err = "ws_net_im2col3: need C and kp multiples of 8 and 16-byte aligned buffers";
    return WS_ERR_INVALID_ARGUMENT;
  }
  Vol v{b, d, h, w};
  k_im2col3<<<grid_for((long long)b * d * h * w * (kp / 8)), 256, 0, (cudaStream_t)stream>>>(
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
  if (ldo < rows || (ldo + 31) / 32 > 0x7fffffff || (cols + 31) / 32 > 65535) {
    t_err = "ws_net_transpose_f32_bf16: bad sizes";
    return WS_ERR_INVALID_ARGUMENT;
  }
  dim3 grid((unsigned)((ldo + 31) / 32), (unsigned)((cols + 31) / 32));
  k_transpose_tiled<float><<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>(in, (__nv_bfloat16*)out, rows, cols, cols,
                                                                           ldo);
  NET_LAUNCH_CHECK();
}
extern "C" int ws_net_transpose_bf16(const void* in, void* out, int64_t rows, int64_t cols, int64_t ldi, int64_t ldo,
                                     void* stream) {
  if (ldo < rows || (ldo + 31) / 32 > 0x7fffffff || (cols + 31) / 32 > 65535) {
    t_err = "ws_net_transpose_bf16: bad sizes";
    return WS_ERR_INVALID_ARGUMENT;
  }
  dim3 grid((unsigned)((ldo + 31) / 32), (unsigned)((cols + 31) / 32));
  k_transpose_tiled<__nv_bfloat16><<<grid, dim3(32, 8), 0, (cudaStream_t)stream>>>(
      (const __nv_bfloat16*)in, (__nv_bfloat16*)out, rows, cols, ldi, ldo);
  NET_LAUNCH_CHECK();
}
extern "C" int ws_net_avgpool2(const void* in, void* out, int b, int d, int h, int w, int C, void* stream) {
  Vol vo{b, d / 2, h / 2, w / 2};
  if (C % 8 == 0 && ((uintptr_t)in & 15) == 0 && ((uintptr_t)out & 15) == 0) {
    k_avgpool2_v8<<<grid_for((long long)b * (d / 2) * (h / 2) * (w / 2) * (C / 8)), 256, 0, (cudaStream_t)stream>>>(
        (const __nv_bfloat16*)in, (__nv_bfloat16*)out, vo, C);
    NET_LAUNCH_CHECK();
  }
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

// Launches k_conv3 with the smallest output-channel tile that holds Cout
// (Cout > 128: tiles of 128 across blockIdx.y); voxel tiles across blockIdx.x.
template <int NT, int S, bool UP>
static int launch_conv3(const ConvIn& in, const void* W, const float* bias, float* out_f32, void* out_bf16, int M,
                        int Cout, int kp, int mode, int* err, cudaStream_t stream) {
  constexpr unsigned smem = conv_smem_bytes<NT, S>();
  static bool attr[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  if (!attr[dev]) {
    cudaError_t e = cudaFuncSetAttribute(k_conv3<NT, S, UP>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) {
      t_err = std::string("conv3: ") + cudaGetErrorString(e);
      return WS_ERR_CUDA;
    }
    attr[dev] = true;
  }
  const long long mt = ((long long)M + BM - 1) / BM, nt = ((long long)Cout + NT - 1) / NT;
  if (nt > 65535) {
    t_err = "conv3: too many output channels";
    return WS_ERR_INVALID_ARGUMENT;
  }
  k_conv3<NT, S, UP><<<dim3((unsigned)mt, (unsigned)nt), kGemmThreads, smem, stream>>>(
      in, (const __nv_bfloat16*)W, bias, out_f32, (__nv_bfloat16*)out_bf16, M, Cout, kp, mode, err);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    t_err = std::string("conv3: ") + cudaGetErrorString(e);
    return WS_ERR_CUDA;
  }
  return WS_OK;
}

template <bool UP>
static int conv3_dispatch(const ConvIn& in, const void* W, const float* bias, float* out_f32, void* out_bf16, int M,
                          int Cout, int kp, int mode, int* err, cudaStream_t st) {
  if (Cout <= 16) return launch_conv3<16, 4, UP>(in, W, bias, out_f32, out_bf16, M, Cout, kp, mode, err, st);
  if (Cout <= 32) return launch_conv3<32, 4, UP>(in, W, bias, out_f32, out_bf16, M, Cout, kp, mode, err, st);
  if (Cout <= 64) return launch_conv3<64, 4, UP>(in, W, bias, out_f32, out_bf16, M, Cout, kp, mode, err, st);
  if (Cout <= 96) return launch_conv3<96, 3, UP>(in, W, bias, out_f32, out_bf16, M, Cout, kp, mode, err, st);
  return launch_conv3<128, 3, UP>(in, W, bias, out_f32, out_bf16, M, Cout, kp, mode, err, st);
}

static int conv3_fwd(const ConvIn& in, const void* W, const float* bias, float* out_f32, void* out_bf16, int Cout,
                     int kp, int mode, int* err_flag, void* stream) {
  const long long M = (long long)in.b * in.d * in.h * in.w;
  const int C = in.Cu + in.Cx;
  if (in.b < 1 || in.d < 1 || in.h < 1 || in.w < 1 || in.Cu < 0 || in.Cx < 0 || in.Cu % 8 || in.Cx % 8 || C < 8 ||
      kp % 64 || kp < 27 * C || M > (1LL << 31) - 256 || Cout < 1 || mode < 0 || mode > 3 || !W || !in.X) {
    t_err = "conv3: need channel counts multiples of 8, kp >= 27 C a multiple of 64";
    return WS_ERR_INVALID_ARGUMENT;
  }
  if (in.Cu && (!in.U || ((in.d | in.h | in.w) & 1))) {
    t_err = "conv3: the upsampled input needs even output dimensions";
    return WS_ERR_INVALID_ARGUMENT;
  }
  if (((uintptr_t)in.X & 15) || ((uintptr_t)in.U & 15) || ((uintptr_t)W & 15)) {
    t_err = "conv3: inputs and weights must be 16-byte aligned";
    return WS_ERR_INVALID_ARGUMENT;
  }
  const bool f32 = mode == EPI_STORE || mode == EPI_BIAS_F32;
  if (f32 ? !out_f32 : !out_bf16) {
    t_err = "conv3: missing output for this mode";
    return WS_ERR_INVALID_ARGUMENT;
  }
  static int* dummy[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64) dev = 0;
  if (!err_flag) {
    if (!dummy[dev] && cudaMalloc(&dummy[dev], sizeof(int)) != cudaSuccess) return WS_ERR_OUT_OF_MEMORY;
    err_flag = dummy[dev];
  }
  cudaStream_t st = (cudaStream_t)stream;
  if (in.Cu) return conv3_dispatch<true>(in, W, bias, out_f32, out_bf16, (int)M, Cout, kp, mode, err_flag, st);
  return conv3_dispatch<false>(in, W, bias, out_f32, out_bf16, (int)M, Cout, kp, mode, err_flag, st);
}

// Forward 3x3x3 convolution (zero padding 1) as an implicit GEMM on the
// tensor cores (k_conv3).
extern "C" int ws_conv3_fwd_bf16(const void* X, const void* W, const float* bias, float* out_f32, void* out_bf16,
                                 int b, int d, int h, int w, int C, int Cout, int kp, int mode, int* err_flag,
                                 void* stream) {
  ConvIn in{nullptr, (const __nv_bfloat16*)X, 0, C, b, d, h, w};
  return conv3_fwd(in, W, bias, out_f32, out_bf16, Cout, kp, mode, err_flag, stream);
}

// The same on the channel concat [nearest x2 upsampling of U, X] (a decoder
// level), read in place.
extern "C" int ws_conv3_upcat_fwd_bf16(const void* U, const void* X, const void* W, const float* bias,
                                       float* out_f32, void* out_bf16, int b, int d, int h, int w, int Cu, int Cx,
                                       int Cout, int kp, int mode, int* err_flag, void* stream) {
  ConvIn in{(const __nv_bfloat16*)U, (const __nv_bfloat16*)X, Cu, Cx, b, d, h, w};
  return conv3_fwd(in, W, bias, out_f32, out_bf16, Cout, kp, mode, err_flag, stream);
}

// Network input features of a ROI (k_features): n and src (may be NULL)
// real fp32 Ny x Nx x Nz column-major; out bf16 [Ny*Nx*Nz][8].
extern "C" int ws_net_features(const float* n, const float* src, int ny, int nx, int nz, float n_bg, float k0,
                               void* out, void* stream) {
  if (!n || !out || ny < 1 || nx < 1 || nz < 1 || ((uintptr_t)out & 15)) {
    t_err = "ws_net_features: bad arguments";
    return WS_ERR_INVALID_ARGUMENT;
  }
  const long long nray = (long long)ny * nx;
  k_features<<<grid_for(nray), 256, 0, (cudaStream_t)stream>>>(n, src, nray, nz, n_bg, k0, (__nv_bfloat16*)out);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    t_err = cudaGetErrorString(e);
    return WS_ERR_CUDA;
  }
  return WS_OK;
}

// Full-grid starting field from the network's ROI envelope
// (k_envelope_to_field).  N = grid (Ny, Nx, Nz); roi0 = first ROI index
// (0-based), roin = ROI size, both (y, x, z); psi complex64 column-major.
extern "C" int ws_net_envelope_to_field(const float* pred, const int64_t N[3], const int64_t roi0[3],
                                        const int64_t roin[3], float scale, float kz, int s2d, void* psi,
                                        void* stream) {
  if (!pred || !N || !roi0 || !roin || !psi) {
    t_err = "ws_net_envelope_to_field: null argument";
    return WS_ERR_INVALID_ARGUMENT;
  }
  RoiMap m{};
  for (int d = 0; d < 3; ++d) {
    if (N[d] < 1 || N[d] > (1 << 30) || roin[d] < 1 || roi0[d] < 0 || roi0[d] + roin[d] > N[d]) {
      t_err = "ws_net_envelope_to_field: the ROI must lie inside the grid";
      return WS_ERR_INVALID_ARGUMENT;
    }
    m.N[d] = (int)N[d];
    m.r0[d] = (int)roi0[d];
    m.rn[d] = (int)roin[d];
  }
  if (s2d && ((roin[0] | roin[1] | roin[2]) & 1)) {
    t_err = "ws_net_envelope_to_field: a half-resolution output needs even ROI sides";
    return WS_ERR_INVALID_ARGUMENT;
  }
  k_envelope_to_field<<<grid_for(N[0] * N[1] * N[2]), 256, 0, (cudaStream_t)stream>>>(pred, m, scale, kz,
                                                                                      (float2*)psi, s2d);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) {
    t_err = cudaGetErrorString(e);
    return WS_ERR_CUDA;
  }
  return WS_OK;
}

namespace ws {
namespace net {
// Weights of the input-gradient convolution: the gradient of a 3x3x3
// convolution (zero padding 1) with respect to its input is the convolution
// of the output gradient with the tap-reversed, transposed weights,
// Wf[ci][t * Cpad + co] = W[co][(26 - t) * Cin + ci] (zero for co >= Cout).
__global__ void k_flip_weights(const __nv_bfloat16* __restrict__ W, int Cin, int Cout, int kp,
                               __nv_bfloat16* __restrict__ Wf, int Cpad, int kpf) {
  const long long total = (long long)Cin * kpf;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int ci = (int)(i / kpf);
    const int k = (int)(i - (long long)ci * kpf);
    const int t = k / Cpad, co = k - t * Cpad;
    __nv_bfloat16 v = __float2bfloat16_rn(0.f);
    if (t < 27 && co < Cout) v = W[(long long)co * kp + (26 - t) * Cin + ci];
    Wf[i] = v;
  }
}
// dy *= (y > 0) when y (a ReLU output) is given, in place (fp32), and a bf16
// copy with the channels padded to Cpad (zeros)
__global__ void k_relu_grad_bf16(float* __restrict__ dy, const __nv_bfloat16* __restrict__ y, long long rows, int C,
                                 __nv_bfloat16* __restrict__ out, int Cpad) {
  const long long total = rows * Cpad;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const long long r = i / Cpad;
    const int c = (int)(i - r * Cpad);
    float g = 0.f;
    if (c < C) {
      const long long j = r * C + c;
      g = dy[j];
      if (y && !(__bfloat162float(y[j]) > 0.f)) {
        g = 0.f;
        dy[j] = 0.f;
      }
    }
    out[i] = __float2bfloat16_rn(g);
  }
}
}  // namespace net
}  // namespace ws

// Tap-reversed, transposed weights for the input-gradient convolution
// (k_flip_weights): W bf16 [Cout][kp] -> Wf bf16 [Cin][kpf], kpf >= 27 Cpad.
extern "C" int ws_net_flip_weights(const void* W, int Cin, int Cout, int kp, void* Wf, int Cpad, int kpf,
                                   void* stream) {
  if (!W || !Wf || Cin < 1 || Cout < 1 || Cpad < Cout || kp < 27 * Cin || kpf < 27 * Cpad) {
    t_err = "ws_net_flip_weights: bad sizes";
    return WS_ERR_INVALID_ARGUMENT;
  }
  k_flip_weights<<<grid_for((long long)Cin * kpf), 256, 0, (cudaStream_t)stream>>>(
      (const __nv_bfloat16*)W, Cin, Cout, kp, (__nv_bfloat16*)Wf, Cpad, kpf);
  NET_LAUNCH_CHECK();
}
// dy *= (y > 0) (y may be NULL: no ReLU) and out = bf16(dy) with Cpad >= C channels
extern "C" int ws_net_relu_grad_bf16(float* dy, const void* y, int64_t rows, int C, void* out, int Cpad, void* stream) {
  if (!dy || !out || rows < 1 || C < 1 || Cpad < C) {
    t_err = "ws_net_relu_grad_bf16: bad arguments";
    return WS_ERR_INVALID_ARGUMENT;
  }
  k_relu_grad_bf16<<<grid_for(rows * Cpad), 256, 0, (cudaStream_t)stream>>>(dy, (const __nv_bfloat16*)y, rows, C,
                                                                            (__nv_bfloat16*)out, Cpad);
  NET_LAUNCH_CHECK();
}

namespace ws {
namespace net {
__global__ void k_add(float* __restrict__ y, const float* __restrict__ x, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] += x[i];
}
}  // namespace net
}  // namespace ws

// y += x (fp32)
extern "C" int ws_net_add(float* y, const float* x, int64_t n, void* stream) {
  if (!y || !x || n < 0) {
    t_err = "ws_net_add: bad arguments";
    return WS_ERR_INVALID_ARGUMENT;
  }
  if (n == 0) return WS_OK;
  k_add<<<grid_for(n), 256, 0, (cudaStream_t)stream>>>(y, x, n);
  NET_LAUNCH_CHECK();
}

namespace ws {
namespace net {
// Space to depth: a (b, d, h, w) x C volume -> (b, d/2, h/2, w/2) x 8C, the
// 2x2x2 sub-voxel s = ((z & 1) * 2 + (y & 1)) * 2 + (x & 1) at channels
// [s C, (s + 1) C).  One thread per 16-byte chunk (C % 8 == 0).
__global__ void k_space_to_depth(const __nv_bfloat16* __restrict__ in, __nv_bfloat16* __restrict__ out, Vol vo,
                                 int C) {
  const int cc = C >> 3;  // chunks per sub-voxel
  const long long total = (long long)vo.b * vo.d * vo.h * vo.w * 8 * cc;
  const Vol vi{vo.b, vo.d * 2, vo.h * 2, vo.w * 2};
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total; i += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(i % (8 * cc));
    long long r = i / (8 * cc);
    const int x = (int)(r % vo.w); r /= vo.w;
    const int y = (int)(r % vo.h); r /= vo.h;
    const int z = (int)(r % vo.d);
    const int b = (int)(r / vo.d);
    const int s = q / cc, c8 = q - s * cc;
    const long long src = vox_index(vi, b, 2 * z + (s >> 2), 2 * y + ((s >> 1) & 1), 2 * x + (s & 1));
    reinterpret_cast<uint4*>(out)[i] = reinterpret_cast<const uint4*>(in + src * C)[c8];
  }
}
}  // namespace net
}  // namespace ws

// (b, d, h, w) x C bf16 -> (b, d/2, h/2, w/2) x 8C (k_space_to_depth)
extern "C" int ws_net_space_to_depth(const void* in, void* out, int b, int d, int h, int w, int C, void* stream) {
  if (!in || !out || C % 8 || (d | h | w) & 1 || b < 1 || d < 2 || h < 2 || w < 2 || ((uintptr_t)in & 15) ||
      ((uintptr_t)out & 15)) {
    t_err = "ws_net_space_to_depth: need C % 8 == 0, even sides and 16-byte aligned buffers";
    return WS_ERR_INVALID_ARGUMENT;
  }
  Vol vo{b, d / 2, h / 2, w / 2};
  k_space_to_depth<<<grid_for((long long)b * d * h * w / 8 * C), 256, 0, (cudaStream_t)stream>>>(
      (const __nv_bfloat16*)in, (__nv_bfloat16*)out, vo, C);
  NET_LAUNCH_CHECK();
}
