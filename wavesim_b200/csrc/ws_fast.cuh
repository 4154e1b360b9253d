// Power-of-two fast path of the fused MBS kernels.
//
// Every thread owns 16 elements of one line of length N at a time, so a line
// has P = N/16 threads, and the radix schedule is fixed at compile time:
//   N = 16:          [16]
//   N = 32 ... 256:  [16, N/16]
//   N = 512 ... 4096:[16, 16, N/256]
// Thread p enters with v[r] = x[p + P r] (its first-stage inputs, loaded
// straight from global memory when the line is contiguous there) and leaves
// with v[m] = X[p + P m]: the same index set, so a forward transform, a
// pointwise multiply and an inverse transform chain in registers.  Only the
// exchanges between stages touch shared memory (one write and one read per
// element for N <= 256).  All index arithmetic is shifts and masks.
//
// Kernels (scalar or per-component planes, layout of the generic path):
//   kf_plane_fwd<N, C, DO_X>  K1: (y, x) planes of N x N (3-D, DO_X) or
//                              columns of length N (2-D); for C > 1 a plane is
//                              split over a cluster of C blocks and the x
//                              transform follows a DSMEM transpose (each
//                              element crosses once).
//   kf_pencil<NO, TY>         K2: outer-dimension pencils, Green's function.
//   kf_plane_inv<N, C, DO_X>  K3: inverse of K1 + unwiggle, mix, accumulate,
//                              ROI energy, stop rule.
#pragma once
#include <cuda.h>

#include "ws_kernels.cuh"

namespace ws {
namespace fast {

constexpr int kThreads = 256;

__host__ __device__ constexpr int ipow16(int e) { return e == 0 ? 1 : 16 * ipow16(e - 1); }

template <int N>
struct LinePlan {
  static_assert(N >= 16 && N <= 4096 && (N & (N - 1)) == 0, "power-of-two line of 16..4096");
  static constexpr int P = N / 16;
  static constexpr int NST = N <= 16 ? 1 : (N <= 256 ? 2 : 3);
  __host__ __device__ static constexpr int radix(int s) { return s < NST - 1 ? 16 : N / ipow16(NST - 1); }
  __host__ __device__ static constexpr int span(int s) { return ipow16(s); }
};

// line element i at base[i + i/16] (contiguous, padded)
struct ColLine {
  float2* base;
  __device__ __forceinline__ float2& at(int i) const { return base[i + (i >> 4)]; }
};
// line element i at base[i * stride] (interleaved lines)
struct RowLine {
  float2* base;
  int stride;
  __device__ __forceinline__ float2& at(int i) const { return base[i * stride]; }
};

// Ask the bulk-copy engine to pull [p, p + bytes) into L2 (no registers, no
// shared memory; p and bytes multiples of 16).
__device__ __forceinline__ void prefetch_l2(const void* p, unsigned bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(p), "r"(bytes) : "memory");
}

// Cluster exchange by push: st.async of a float2 into another block's shared
// memory, completing on that block's mbarrier (bytes counted), so that the
// sender never waits on a remote load and the receiver waits once.
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ uint32_t map_rank(uint32_t addr, int rank) {
  uint32_t r;
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(rank));
  return r;
}
__device__ __forceinline__ void st_async_f2(uint32_t raddr, float2 v, uint32_t rbar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v2.f32 [%0], {%1, %2}, [%3];" ::"r"(raddr),
               "f"(v.x), "f"(v.y), "r"(rbar)
               : "memory");
}
__device__ __forceinline__ void st_async_f4(uint32_t raddr, float2 u, float2 v, uint32_t rbar) {
  asm volatile("st.async.shared::cluster.mbarrier::complete_tx::bytes.v4.f32 [%0], {%1, %2, %3, %4}, [%5];" ::"r"(raddr),
               "f"(u.x), "f"(u.y), "f"(v.x), "f"(v.y), "r"(rbar)
               : "memory");
}
__device__ __forceinline__ void mbar_init_expect(uint64_t* bar, uint32_t bytes) {
  const uint32_t a = smem_addr(bar);
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(a));
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
// Waits for phase 0 of the barrier (the pushed bytes all arrived); gives up
// after about 5e7 clocks and then returns false.
__device__ __forceinline__ bool mbar_wait_cluster(uint64_t* bar) {
  const uint32_t a = smem_addr(bar);
  const long long t0 = clock64();
  while (true) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.acquire.cluster.shared::cta.b64 p, [%1], 0;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a)
        : "memory");
    if (done) return true;
    if (clock64() - t0 > 50000000LL) return false;
  }
}

struct SyncWarp {
  __device__ __forceinline__ void operator()() const { __syncwarp(); }
};
struct SyncBlock {
  __device__ __forceinline__ void operator()() const { __syncthreads(); }
};

template <int R, bool INV>
__device__ __forceinline__ void dft_slice(float2 (&v)[16], int off) {
  float2 u[R];
#pragma unroll
  for (int r = 0; r < R; ++r) u[r] = v[off + r];
  Dft<R, INV>::run(u);
#pragma unroll
  for (int r = 0; r < R; ++r) v[off + r] = u[r];
}

template <int N, bool INV, int S, class Line, class Sync>
__device__ __forceinline__ void line_stage(float2 (&v)[16], const Line& L, int p, const float2* __restrict__ tw,
                                           Sync sync) {
  using PL = LinePlan<N>;
  constexpr int R = PL::radix(S), Ns = PL::span(S), B = 16 / R, P = PL::P, NR = N / R;
  constexpr int TS = N / (Ns * R);
  if constexpr (S > 0) {
#pragma unroll
    for (int q = 0; q < B; ++q) {
      const int j = p + P * q;
#pragma unroll
      for (int r = 0; r < R; ++r) v[q * R + r] = L.at(j + r * NR);
      const int jm = j & (Ns - 1);
#pragma unroll
      for (int r = 1; r < R; ++r) {
        float2 w = __ldg(&tw[jm * r * TS]);
        if (INV) w.y = -w.y;
        v[q * R + r] = cmul(v[q * R + r], w);
      }
    }
  }
#pragma unroll
  for (int q = 0; q < B; ++q) dft_slice<R, INV>(v, q * R);
  if constexpr (S < PL::NST - 1) {
    sync();
#pragma unroll
    for (int q = 0; q < B; ++q) {
      const int j = p + P * q;
      const int jm = j & (Ns - 1);
      const int base = (j - jm) * R + jm;
#pragma unroll
      for (int r = 0; r < R; ++r) L.at(base + r * Ns) = v[q * R + r];
    }
    sync();
  } else if constexpr (B > 1) {
    float2 t[16];
#pragma unroll
    for (int q = 0; q < B; ++q)
#pragma unroll
      for (int r = 0; r < R; ++r) t[q + B * r] = v[q * R + r];
#pragma unroll
    for (int m = 0; m < 16; ++m) v[m] = t[m];
  }
}

// Lines of up to 256 points have two stages, and the second stage's twiddles
// of a thread depend on its p only: a persistent kernel that transforms many
// lines with the same p loads them once (load_tw2) and passes them to
// line_fft_tw2, which is line_fft with those registers in place of the
// table loads (the same values, so the same results).
template <int N>
__device__ __forceinline__ void load_tw2(float2 (&wt)[16], int p, const float2* __restrict__ tw) {
  using PL = LinePlan<N>;
  static_assert(PL::NST == 2, "two-stage lines");
  constexpr int R = PL::radix(1), Ns = PL::span(1), B = 16 / R, P = PL::P, TS = N / (Ns * R);
#pragma unroll
  for (int q = 0; q < B; ++q) {
    const int jm = (p + P * q) & (Ns - 1);
    wt[q * R] = make_float2(1.f, 0.f);
#pragma unroll
    for (int r = 1; r < R; ++r) wt[q * R + r] = __ldg(&tw[jm * r * TS]);
  }
}

// In: v[r] = x[p + P r].  Out: v[m] = X[p + P m] (unnormalised; INV: sign +1).
template <int N, bool INV, class Line, class Sync>
__device__ __forceinline__ void line_fft(float2 (&v)[16], const Line& L, int p, const float2* __restrict__ tw,
                                         Sync sync) {
  line_stage<N, INV, 0>(v, L, p, tw, sync);
  if constexpr (LinePlan<N>::NST > 1) line_stage<N, INV, 1>(v, L, p, tw, sync);
  if constexpr (LinePlan<N>::NST > 2) line_stage<N, INV, 2>(v, L, p, tw, sync);
}

template <int N, bool INV, class Line, class Sync>
__device__ __forceinline__ void line_fft_tw2(float2 (&v)[16], const Line& L, int p, const float2 (&wt)[16],
                                             Sync sync) {
  using PL = LinePlan<N>;
  static_assert(PL::NST == 2, "two-stage lines");
  constexpr int R0 = PL::radix(0), B0 = 16 / R0, Ns0 = PL::span(0);
  constexpr int R = PL::radix(1), Ns = PL::span(1), B = 16 / R, P = PL::P, NR = N / R;
  // stage 0 (as line_stage<N, INV, 0>)
#pragma unroll
  for (int q = 0; q < B0; ++q) dft_slice<R0, INV>(v, q * R0);
  sync();
#pragma unroll
  for (int q = 0; q < B0; ++q) {
    const int j = p + P * q;
    const int jm = j & (Ns0 - 1);
    const int base = (j - jm) * R0 + jm;
#pragma unroll
    for (int r = 0; r < R0; ++r) L.at(base + r * Ns0) = v[q * R0 + r];
  }
  sync();
  // stage 1 (as line_stage<N, INV, 1>, twiddles from wt)
#pragma unroll
  for (int q = 0; q < B; ++q) {
    const int j = p + P * q;
#pragma unroll
    for (int r = 0; r < R; ++r) v[q * R + r] = L.at(j + r * NR);
#pragma unroll
    for (int r = 1; r < R; ++r) {
      float2 w = wt[q * R + r];
      if (INV) w.y = -w.y;
      v[q * R + r] = cmul(v[q * R + r], w);
    }
  }
#pragma unroll
  for (int q = 0; q < B; ++q) dft_slice<R, INV>(v, q * R);
  if constexpr (B > 1) {
    float2 t[16];
#pragma unroll
    for (int q = 0; q < B; ++q)
#pragma unroll
      for (int r = 0; r < R; ++r) t[q + B * r] = v[q * R + r];
#pragma unroll
    for (int m = 0; m < 16; ++m) v[m] = t[m];
  }
}

// shared-memory tile geometry of the plane kernels
template <int N, int C, bool DO_X>
struct PlaneGeom {
  static constexpr int M = DO_X ? N / C : 0;   // columns held in phase A (2-D: a.ncols at run time)
  static constexpr int CS = N + N / 16 + 1;    // padded column stride (odd: row access conflict free)
  static constexpr int LR = N / C;             // rows held in the x phase (C > 1)
  // transposed tile: row kyl of column x at x * CS2 + kyl + 2 (kyl / 16); CS2
  // even, so that element pairs (kyl even) are 16-byte aligned
  static constexpr int CS2 = LR + 2 * (LR / 16) + (LR >= 32 ? 2 : 0);
  static constexpr int P = N / 16;
  static constexpr int LPR = kThreads / P;     // lines per round
  // K1's column scratch: one round of lines, plus a slot for idle lanes when
  // the block's columns are not a whole number of rounds
  static constexpr int SCR = (DO_X && M % LPR == 0) ? LPR : LPR + 1;
  static constexpr size_t smem_a = (size_t)(M + 1) * CS * sizeof(float2);  // + scratch column
  static constexpr size_t smem_b = (size_t)N * CS2 * sizeof(float2);
  // K1 with a cluster: one round of column scratch + the received rows
  static constexpr bool PUSH = C > 1 && DO_X;
  // (+ 16 bytes: the received tile starts on a 16-byte boundary for the pair pushes)
  static constexpr size_t smem_push = (size_t)SCR * CS * sizeof(float2) + 16 + smem_b;
  static constexpr size_t smem_max_ab = smem_a > smem_b ? smem_a : smem_b;
  static constexpr size_t smem = PUSH ? (smem_push > smem_max_ab ? smem_push : smem_max_ab) : smem_a;
  static_assert(kThreads % P == 0 || P > kThreads, "threads per line");
};

// ----------------------------------------------------------------------------
// K1
// ----------------------------------------------------------------------------
template <int N, int C, bool DO_X>
__global__ void __launch_bounds__(kThreads, 3)
    kf_plane_fwd(InnerArgs a, const float2* __restrict__ dE, const float2* __restrict__ src, float2 A,
                 float2* __restrict__ T, const DevState* __restrict__ st) {
  using G = PlaneGeom<N, C, DO_X>;
  constexpr int P = G::P, LPR = G::LPR;
  const int rhs = blockIdx.x / a.bpr, bid = blockIdx.x - rhs * a.bpr;
  st += rhs;
  if (load_done(st)) return;
  dE += rhs * a.fstride;
  if (src) src += rhs * a.fstride;
  T += rhs * a.fstride;
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x;
  const Geom& g = a.g;
  const int nx = g.nx;
  const int M = DO_X ? G::M : a.ncols;  // scratch column for idle lanes: index M
  int rank = 0, plane = 0, x0 = 0, z = 0, ncol;
  long long colbase;
  if constexpr (DO_X) {
    rank = C > 1 ? (int)(bid % C) : 0;
    plane = bid / C;
    x0 = rank * M;
    z = plane % g.nz;
    colbase = (long long)plane * nx + x0;
    ncol = M;
  } else {
    colbase = (long long)bid * M;
    ncol = (int)min((long long)M, (long long)nx * g.nc - colbase);
  }
  // Blocks run roughly in index order, a.pf of them at a time: pull the
  // columns block bid + a.pf will load into L2 now, so that HBM keeps
  // streaming while this block transforms (same right-hand side only).
  if (a.pf && bid + a.pf < a.bpr) {
    const int fb = bid + a.pf;
    long long fcol;
    int fn;
    if constexpr (DO_X) {
      fcol = (long long)(fb / C) * nx + (long long)(C > 1 ? fb % C : 0) * M;
      fn = M;
    } else {
      fcol = (long long)fb * M;
      fn = (int)min((long long)M, (long long)nx * g.nc - fcol);
    }
    for (int c = tid; c < fn; c += kThreads) {
      prefetch_l2(dE + (fcol + c) * N, N * sizeof(float2));
      if (src) prefetch_l2(src + (fcol + c) * N, N * sizeof(float2));
    }
  }
  constexpr bool PUSH = G::PUSH;
  // PUSH: [one round of column scratch, LPR + 1 columns][rows received from the cluster]
  float2* const smB =
      PUSH ? reinterpret_cast<float2*>((reinterpret_cast<uintptr_t>(sm + G::SCR * G::CS) + 15) & ~(uintptr_t)15) : sm;
  __shared__ __align__(8) uint64_t recv_bar;
  if constexpr (PUSH) {
    if (tid == 0) mbar_init_expect(&recv_bar, (uint32_t)(G::LR * N * sizeof(float2)));
    cg::this_cluster().sync();  // every block's barrier is armed before anyone pushes
  }
  const float2 gzz = a.w.gz[z];
  // phase A: y transform of each held column, straight from global memory
  for (int c0 = 0; c0 < ncol; c0 += LPR) {
    const int cl = c0 + tid / P, p = tid % P;
    const bool live = cl < ncol;
    float2 v[16];
    if (live) {
      const long long col = colbase + cl;
      const int x = DO_X ? x0 + cl : (int)(col % nx);
      const float2 gxz = cmul(a.w.gx[x], gzz);
      const float2* __restrict__ s = dE + col * N;
      const float2* __restrict__ sr = src ? src + col * N : nullptr;
#pragma unroll
      for (int r = 0; r < 16; ++r) {
        const int y = p + P * r;
        float2 e = s[y];
        if (sr) e = cadd(e, cmul(A, sr[y]));
        v[r] = cmul(cmul(e, gxz), a.w.gy[y]);
      }
    } else {
#pragma unroll
      for (int r = 0; r < 16; ++r) v[r] = make_float2(0.f, 0.f);
    }
    ColLine L{sm + (PUSH ? (live ? cl - c0 : LPR) : (live ? cl : M)) * G::CS};
    if constexpr (P <= 32) {
      line_fft<N, false>(v, L, p, a.py.tw, SyncWarp{});
    } else {
      line_fft<N, false>(v, L, p, a.py.tw, SyncBlock{});
    }
    if constexpr (PUSH) {
      // X[ky] of column x goes to the block holding row ky: rank ky / LR,
      // at x * CS2 + kyl (padded) of its received tile
      // in 16-byte pairs (ky, ky + 1): the even thread of a lane pair sends
      // the pairs of m < 8, the odd one those of m >= 8 (P is even, so the
      // partner lane p ^ 1 works on the same column)
      float2 w[16];
#pragma unroll
      for (int m = 0; m < 16; ++m) {
        w[m].x = __shfl_xor_sync(0xffffffffu, v[m].x, 1);
        w[m].y = __shfl_xor_sync(0xffffffffu, v[m].y, 1);
      }
      if (live) {
        const int x = x0 + cl;
        const uint32_t lbar = smem_addr(&recv_bar);
        const bool odd = p & 1;
#pragma unroll
        for (int h = 0; h < 8; ++h) {
          const int m = odd ? 8 + h : h;
          const int ky = (p & ~1) + P * m;  // even
          const int dst = ky / G::LR, kyl = ky - dst * G::LR;
          const uint32_t la = smem_addr(smB + x * G::CS2 + kyl + 2 * (kyl >> 4));
          const float2 lo = odd ? w[8 + h] : v[h], hi = odd ? v[8 + h] : w[h];  // constant indices
          st_async_f4(map_rank(la, dst), lo, hi, map_rank(lbar, dst));
        }
      }
    } else if constexpr (DO_X) {
#pragma unroll
      for (int m = 0; m < 16; ++m) L.at(p + P * m) = v[m];
    } else if (live) {
      float2* __restrict__ d = T + (colbase + cl) * N;
#pragma unroll
      for (int m = 0; m < 16; ++m) d[p + P * m] = v[m];
    }
  }
  if constexpr (DO_X) {
    // rows of the x transform: C == 1 -> column-major tile as is;
    // C > 1 -> the rows [rank*LR, (rank+1)*LR) of all N columns the cluster
    // pushed into smB, column-major with stride CS2.
    int xs = G::CS;
    if constexpr (PUSH) {
      if (!mbar_wait_cluster(&recv_bar)) {
        if (a.err) atomicExch(a.err, 1);
      }
      xs = G::CS2;
    } else {
      __syncthreads();
    }
    constexpr int ROWS = C > 1 ? G::LR : N;
    constexpr int RPR = kThreads / P;  // rows per round
    for (int r0 = 0; r0 < ROWS; r0 += RPR) {
      const int rl = r0 + tid % RPR, p = tid / RPR;
      RowLine L{smB + rl + (PUSH ? 2 : 1) * (rl >> 4), xs};
      float2 v[16];
#pragma unroll
      for (int r = 0; r < 16; ++r) v[r] = L.at(p + P * r);
      line_fft<N, false>(v, L, p, a.twx, SyncBlock{});
      const int ky = (C > 1 ? rank * G::LR : 0) + rl;
      float2* __restrict__ d = T + (long long)plane * nx * N + ky;
#pragma unroll
      for (int m = 0; m < 16; ++m) d[(long long)(p + P * m) * N] = v[m];
    }
  }
}

// ----------------------------------------------------------------------------
// K2: outer-dimension pencils of length NO, TY consecutive y per block
// ----------------------------------------------------------------------------
template <int NO, int TY>
__global__ void __launch_bounds__(TY*(NO / 16) < 1024 ? TY*(NO / 16) : 1024, 3)
    kf_pencil(OuterArgs a, float2* __restrict__ T, const DevState* __restrict__ st) {
  pdl_begin();
  constexpr int P = NO / 16;
  constexpr int TYS = TY + 1;
  const int rhs = blockIdx.x / a.bpr, bid = blockIdx.x - rhs * a.bpr;
  st += rhs;
  if (load_done(st)) return;
  T += rhs * a.fstride;
  extern __shared__ float2 sm[];
  const Geom& g = a.g;
  const int tid = threadIdx.x;
  const int yl = tid % TY, p = tid / TY;
  const int nyt = g.ny / TY;
  const int yt = bid % nyt;
  const int mid = a.mode3d ? bid / nyt : 0;
  const int ky = yt * TY + yl;
  const long long ps = a.mode3d ? (long long)g.ny * g.nx : (long long)g.ny;
  float2* __restrict__ base = T + ky + (long long)g.ny * mid;
  if (a.pf && bid + a.pf < a.bpr) {
    // the TY-element rows of pencil block bid + a.pf into L2 (see kf_plane_fwd)
    const int fb = bid + a.pf;
    const float2* fbase = T + (long long)(fb % nyt) * TY + (long long)g.ny * (a.mode3d ? fb / nyt : 0);
    for (int r = tid; r < NO; r += TY * P) prefetch_l2(fbase + ps * r, TY * sizeof(float2));
  }
  float2 v[16];
#pragma unroll
  for (int r = 0; r < 16; ++r) v[r] = base[ps * (p + P * r)];
  RowLine L{sm + yl, TYS};
  line_fft<NO, false>(v, L, p, a.po.tw, SyncBlock{});
  // f_g0_scalar with the 1/N of ifftn: E ./ (px^2 + py^2 + (pz^2 - k02e))
  const float py = a.w.pye[ky];
  const float pxm = a.mode3d ? a.w.pxe[mid] : 0.f;
  const float base2 = a.mode3d ? fmaf(pxm, pxm, py * py) : fmaf(py, py, a.w.pze[0] * a.w.pze[0]);
  const float di = -a.k02e.y;
  if (a.pstd) {
#pragma unroll
    for (int m = 0; m < 16; ++m) {  // PSTD Laplacian -|p|^2 / N (k02e = 0)
      const int ko = p + P * m;
      const float po = a.mode3d ? a.w.pze[ko] : a.w.pxe[ko];
      const float f = -fmaf(po, po, base2) * a.norm;
      v[m] = make_float2(f * v[m].x, f * v[m].y);
    }
  } else {
#pragma unroll
    for (int m = 0; m < 16; ++m) {
      const int ko = p + P * m;
      const float po = a.mode3d ? a.w.pze[ko] : a.w.pxe[ko];
      const float dr = fmaf(po, po, base2) - a.k02e.x;
      const float inv = __fdividef(a.norm, fmaf(dr, dr, di * di));
      v[m] = cmul(v[m], make_float2(dr * inv, -di * inv));
    }
  }
  line_fft<NO, true>(v, L, p, a.po.tw, SyncBlock{});
  if (a.pstd)
#pragma unroll
    for (int m = 0; m < 16; ++m) v[m].y = -v[m].y;
#pragma unroll
  for (int m = 0; m < 16; ++m) base[ps * (p + P * m)] = v[m];
}

// ----------------------------------------------------------------------------
// K3
// ----------------------------------------------------------------------------
template <int N, int C, bool DO_X>
__global__ void __launch_bounds__(kThreads, C >= 16 ? 3 : 2)
    kf_plane_inv(InnerArgs a, const float2* __restrict__ T, float2* __restrict__ dE, float2* __restrict__ E,
                 const float2* __restrict__ gamma, const DevState* __restrict__ st, double* __restrict__ partials) {
  using G = PlaneGeom<N, C, DO_X>;
  constexpr int P = G::P, LPR = G::LPR;
  const int rhs = blockIdx.x / a.bpr, bid = blockIdx.x - rhs * a.bpr;
  st += rhs;
  if (load_done(st)) return;
  // with a.acc2, E' takes dE'_{k-1} + dE'_k after even iterations k only
  const bool acc_now = !a.acc2 || (__ldcg(&st->it) & 1) == 0;
  T += rhs * a.fstride;
  dE += rhs * a.fstride;
  E += rhs * a.fstride;
  partials += (long long)rhs * a.bpr;
  gamma += rhs * a.gstride;  // a batch of media: each right-hand side has its own gamma
  extern __shared__ float2 sm[];
  __shared__ float red[kThreads / 32];
  const int tid = threadIdx.x;
  const Geom& g = a.g;
  const int nx = g.nx;
  const int M = DO_X ? G::M : a.ncols;
  int rank = 0, plane = 0, x0 = 0, z = 0, comp = 0, ncol;
  long long colbase;
  if constexpr (DO_X) {
    rank = C > 1 ? (int)(bid % C) : 0;
    plane = bid / C;
    x0 = rank * M;
    z = plane % g.nz;
    comp = plane / g.nz;
    colbase = (long long)plane * nx + x0;
    ncol = M;
  } else {
    colbase = (long long)bid * M;
    ncol = (int)min((long long)M, (long long)nx * g.nc - colbase);
  }
  // the epilogue's dE, E and gamma columns are contiguous: start pulling them
  // into L2 now so that they arrive while the transforms run
  if (tid == 0 && ncol > 0) {
    const long long c0 = colbase;
    const unsigned bytes = (unsigned)ncol * N * sizeof(float2);
    const int comp0 = DO_X ? comp : (int)(colbase / nx);
    const int comp1 = DO_X ? comp : (int)((colbase + ncol - 1) / nx);
    prefetch_l2(dE + c0 * N, bytes);
    if (acc_now) prefetch_l2(E + c0 * N, bytes);
    if (comp0 == comp1) prefetch_l2(gamma + c0 * N - (long long)comp0 * g.npts, bytes);
  }
  if (a.pf && bid + a.pf < a.bpr) {
    // the transform input of block bid + a.pf into L2 (see kf_plane_fwd)
    const int fb = bid + a.pf;
    if constexpr (DO_X) {
      const long long fplane = fb / C;
      if constexpr (C > 1) {
        const int frank = fb % C;
        for (int kx = tid; kx < nx; kx += kThreads)
          prefetch_l2(T + (fplane * nx + kx) * N + (long long)frank * G::LR, G::LR * sizeof(float2));
      } else {
        if (tid == 0) prefetch_l2(T + fplane * nx * N, (unsigned)((long long)nx * N * sizeof(float2)));
      }
    } else {
      const long long fcol = (long long)fb * M;
      const int fn = (int)min((long long)M, (long long)nx * g.nc - fcol);
      if (tid == 0 && fn > 0) prefetch_l2(T + fcol * N, (unsigned)fn * N * sizeof(float2));
    }
  }
  if constexpr (DO_X) {
    constexpr int ROWS = C > 1 ? G::LR : N;
    constexpr int RPR = kThreads / P;
    const int xs = C > 1 ? G::CS2 : G::CS;
    for (int r0 = 0; r0 < ROWS; r0 += RPR) {
      const int rl = r0 + tid % RPR, p = tid / RPR;
      const int ky = (C > 1 ? rank * G::LR : 0) + rl;
      const float2* __restrict__ s = T + (long long)plane * nx * N + ky;
      float2 v[16];
#pragma unroll
      for (int r = 0; r < 16; ++r) v[r] = s[(long long)(p + P * r) * N];
      RowLine L{sm + rl + (rl >> 4), xs};
      line_fft<N, true>(v, L, p, a.twx, SyncBlock{});
#pragma unroll
      for (int m = 0; m < 16; ++m) L.at(p + P * m) = v[m];
    }
    __syncthreads();
    if constexpr (C > 1) {
      cg::cluster_group cl = cg::this_cluster();
      constexpr int PER = G::M * N / kThreads;
      float2 hold[PER];
      cl.sync();
#pragma unroll
      for (int i = 0; i < PER; ++i) {
        const int e = tid + kThreads * i;
        const int ky = e % N, c = e / N;
        const float2* rs = cl.map_shared_rank(sm, ky / G::LR);
        const int kyl = ky % G::LR;
        hold[i] = rs[(x0 + c) * G::CS2 + kyl + (kyl >> 4)];
      }
      cl.sync();
#pragma unroll
      for (int i = 0; i < PER; ++i) {
        const int e = tid + kThreads * i;
        const int ky = e % N, c = e / N;
        sm[c * G::CS + ky + (ky >> 4)] = hold[i];
      }
      __syncthreads();
    }
  }
  const float2 gzz = a.w.gz[z];
  float esum = 0.f;
  for (int c0 = 0; c0 < ncol; c0 += LPR) {
    const int cl = c0 + tid / P, p = tid % P;
    const bool live = cl < ncol;
    float2 v[16];
    ColLine L{sm + (live ? cl : M) * G::CS};
    if constexpr (DO_X) {
#pragma unroll
      for (int r = 0; r < 16; ++r) v[r] = L.at(p + P * r);
    } else {
      if (live) {
        const float2* __restrict__ s = T + (colbase + cl) * N;
#pragma unroll
        for (int r = 0; r < 16; ++r) v[r] = s[p + P * r];
      } else {
#pragma unroll
        for (int r = 0; r < 16; ++r) v[r] = make_float2(0.f, 0.f);
      }
    }
    if constexpr (P <= 32) {
      line_fft<N, true>(v, L, p, a.py.tw, SyncWarp{});
    } else {
      line_fft<N, true>(v, L, p, a.py.tw, SyncBlock{});
    }
    if (live) {
      const long long col = colbase + cl;
      int x, c;
      if constexpr (DO_X) {
        x = x0 + cl;
        c = comp;
      } else {
        x = (int)(col % nx);
        c = (int)(col / nx);
      }
      const float2 gxz = cmul(a.w.gx[x], gzz);
      const bool in_xzc = x >= g.r0[1] && x < g.r1[1] && z >= g.r0[2] && z < g.r1[2] && c >= g.r0[3] && c < g.r1[3];
      const long long gcol = col * N;
      const float2* __restrict__ gmc = gamma + (gcol - (long long)c * g.npts);
      float2* __restrict__ dEc = dE + gcol;
      float2* __restrict__ Ec = E + gcol;
      // Eprop after the conjugate ramps (WaveSim.m:55), then f_mix (f_mix.m:3-4)
      // and E += dE; the loads of a half are issued together.
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        float2 gm[8], d0[8], e0[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int y = p + P * (8 * h + i);
          gm[i] = gmc[y];
          d0[i] = dEc[y];
          e0[i] = acc_now ? Ec[y] : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int m = 8 * h + i;
          const int y = p + P * m;
          const float2 ep = cmul_conj(cmul_conj(v[m], gxz), a.w.gy[y]);
          const float2 one_m = make_float2(1.f - kAlpha * gm[i].x, -kAlpha * gm[i].y);
          const float2 t = cmul(cmul(gm[i], gm[i]), ep);
          const float2 dn = cadd(cmul(one_m, d0[i]), make_float2(kAlpha * t.y, -kAlpha * t.x));
          dEc[y] = dn;
          if (acc_now) Ec[y] = cadd(e0[i], a.acc2 ? cadd(d0[i], dn) : dn);
          if (in_xzc && y >= g.r0[0] && y < g.r1[0]) esum = fmaf(dn.x, dn.x, fmaf(dn.y, dn.y, esum));
        }
      }
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) esum += __shfl_xor_sync(0xffffffffu, esum, o);
  if ((tid & 31) == 0) red[tid >> 5] = esum;
  __syncthreads();
  if (tid < 32) {
    float v = tid < kThreads / 32 ? red[tid] : 0.f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (tid == 0) partials[bid] = (double)v;
  }
}


// ----------------------------------------------------------------------------
// K3 of iteration k fused with K1 of iteration k + 1 (3-D planes on a cluster)
// ----------------------------------------------------------------------------
// The new increment dE'_k of a column, which K3's epilogue holds in registers
// as v[m] = dE'(y = p + P m), is exactly the input K1 of the next iteration
// loads for that column.  So after the epilogue the block adds the source of
// iteration k + 1 (if any), applies the next wiggle's ramps and runs the y
// transform in place in the column tile; the cluster then exchanges rows by
// pulling (two cluster barriers), and each block transforms its rows along x
// and writes them to T: the very slab it read at the start.  dE' is not read
// again, so an iteration moves 64 instead of 72 bytes per point, and the
// K1 launch disappears from the loop.
template <int N, int C>
__global__ void __launch_bounds__(kThreads, 2)
    kf_plane_fused(InnerArgs a, Wig w1, const float2* __restrict__ src1, float2 A, float2* __restrict__ T,
                   float2* __restrict__ dE, float2* __restrict__ E, const float2* __restrict__ gamma,
                   const DevState* __restrict__ st, double* __restrict__ partials) {
  static_assert(C > 1, "cluster planes only");
  using G = PlaneGeom<N, C, true>;
  constexpr int P = G::P, LPR = G::LPR, M = G::M, LR = G::LR;
  constexpr int RPR = kThreads / P;
  const int rhs = blockIdx.x / a.bpr, bid = blockIdx.x - rhs * a.bpr;
  st += rhs;
  if (load_done(st)) return;  // the same for every block of a cluster
  const bool acc_now = !a.acc2 || (__ldcg(&st->it) & 1) == 0;
  T += rhs * a.fstride;
  dE += rhs * a.fstride;
  E += rhs * a.fstride;
  if (src1) src1 += rhs * a.fstride;
  partials += (long long)rhs * a.bpr;
  gamma += rhs * a.gstride;  // a batch of media: each right-hand side has its own gamma
  extern __shared__ float2 sm[];
  __shared__ float red[kThreads / 32];
  const int tid = threadIdx.x;
  const Geom& g = a.g;
  const int nx = g.nx;
  const int rank = (int)(bid % C), plane = bid / C;
  const int x0 = rank * M, z = plane % g.nz, comp = plane / g.nz;
  const long long colbase = (long long)plane * nx + x0;
  float2* __restrict__ slab = T + (long long)plane * nx * N + rank * LR;  // rows [rank LR, +LR) of the plane
  if (tid == 0) {
    const unsigned bytes = (unsigned)M * N * sizeof(float2);
    prefetch_l2(dE + colbase * N, bytes);
    if (acc_now) prefetch_l2(E + colbase * N, bytes);
    prefetch_l2(gamma + colbase * N - (long long)comp * g.npts, bytes);
    if (src1) prefetch_l2(src1 + colbase * N, bytes);
  }
  cg::cluster_group cl = cg::this_cluster();
  // K3: inverse x transform of the block's rows
  for (int r0 = 0; r0 < LR; r0 += RPR) {
    const int rl = r0 + tid % RPR, p = tid / RPR;
    float2 v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = slab[(long long)(p + P * r) * N + rl];
    RowLine L{sm + rl + (rl >> 4), G::CS2};
    line_fft<N, true>(v, L, p, a.twx, SyncBlock{});
#pragma unroll
    for (int m = 0; m < 16; ++m) L.at(p + P * m) = v[m];
  }
  {
    constexpr int PER = M * N / kThreads;
    float2 hold[PER];
    cl.sync();
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int e = tid + kThreads * i;
      const int ky = e % N, c = e / N;
      const float2* rs = cl.map_shared_rank(sm, ky / LR);
      const int kyl = ky % LR;
      hold[i] = rs[(x0 + c) * G::CS2 + kyl + (kyl >> 4)];
    }
    cl.sync();
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int e = tid + kThreads * i;
      const int ky = e % N, c = e / N;
      sm[c * G::CS + ky + (ky >> 4)] = hold[i];
    }
  }
  __syncthreads();
  const float2 gzz = a.w.gz[z];
  const float2 gzz1 = w1.gz[z];
  float esum = 0.f;
  for (int c0 = 0; c0 < M; c0 += LPR) {
    const int cc = c0 + tid / P, p = tid % P;
    float2 v[16];
    ColLine L{sm + cc * G::CS};
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = L.at(p + P * r);
    if constexpr (P <= 32) {
      line_fft<N, true>(v, L, p, a.py.tw, SyncWarp{});
    } else {
      line_fft<N, true>(v, L, p, a.py.tw, SyncBlock{});
    }
    const int x = x0 + cc;
    const long long col = colbase + cc;
    const float2 gxz = cmul(a.w.gx[x], gzz);
    const bool in_xzc = x >= g.r0[1] && x < g.r1[1] && z >= g.r0[2] && z < g.r1[2] && comp >= g.r0[3] && comp < g.r1[3];
    const long long gcol = col * N;
    const float2* __restrict__ gmc = gamma + (gcol - (long long)comp * g.npts);
    float2* __restrict__ dEc = dE + gcol;
    float2* __restrict__ Ec = E + gcol;
    // K3's epilogue (unwiggle, f_mix, E' += dE', ROI energy); v[m] becomes dE'_k(y)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float2 gm[8], d0[8], e0[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int y = p + P * (8 * h + i);
        gm[i] = gmc[y];
        d0[i] = dEc[y];
        e0[i] = acc_now ? Ec[y] : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int m = 8 * h + i;
        const int y = p + P * m;
        const float2 ep = cmul_conj(cmul_conj(v[m], gxz), a.w.gy[y]);
        const float2 one_m = make_float2(1.f - kAlpha * gm[i].x, -kAlpha * gm[i].y);
        const float2 t = cmul(cmul(gm[i], gm[i]), ep);
        const float2 dn = cadd(cmul(one_m, d0[i]), make_float2(kAlpha * t.y, -kAlpha * t.x));
        dEc[y] = dn;
        if (acc_now) Ec[y] = cadd(e0[i], a.acc2 ? cadd(d0[i], dn) : dn);
        if (in_xzc && y >= g.r0[0] && y < g.r1[0]) esum = fmaf(dn.x, dn.x, fmaf(dn.y, dn.y, esum));
        v[m] = dn;
      }
    }
    // K1 of iteration k + 1 on the same column: source, next ramps, y transform
    const float2 gxz1 = cmul(w1.gx[x], gzz1);
    const float2* __restrict__ sr = src1 ? src1 + gcol : nullptr;
#pragma unroll
    for (int m = 0; m < 16; ++m) {
      const int y = p + P * m;
      float2 e = v[m];
      if (sr) e = cadd(e, cmul(A, sr[y]));
      v[m] = cmul(cmul(e, gxz1), w1.gy[y]);
    }
    if constexpr (P <= 32) {
      line_fft<N, false>(v, L, p, a.py.tw, SyncWarp{});
    } else {
      line_fft<N, false>(v, L, p, a.py.tw, SyncBlock{});
    }
#pragma unroll
    for (int m = 0; m < 16; ++m) L.at(p + P * m) = v[m];
  }
  // the ROI energy of dE'_k
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) esum += __shfl_xor_sync(0xffffffffu, esum, o);
  if ((tid & 31) == 0) red[tid >> 5] = esum;
  // rows [rank LR, +LR) of all N transformed columns, from the blocks holding them
  {
    constexpr int PER = LR * N / kThreads;
    float2 hold[PER];
    cl.sync();
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int e = tid + kThreads * i;
      const int kyl = e % LR, x = e / LR;
      const int ky = rank * LR + kyl;
      const float2* rs = cl.map_shared_rank(sm, x / M);
      hold[i] = rs[(x % M) * G::CS + ky + (ky >> 4)];
    }
    cl.sync();
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int e = tid + kThreads * i;
      const int kyl = e % LR, x = e / LR;
      sm[x * G::CS2 + kyl + (kyl >> 4)] = hold[i];
    }
  }
  __syncthreads();
  if (tid < 32) {
    float v = tid < kThreads / 32 ? red[tid] : 0.f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (tid == 0) partials[bid] = (double)v;
  }
  // K1's x transform of the block's rows, written over the slab K3 read
  for (int r0 = 0; r0 < LR; r0 += RPR) {
    const int rl = r0 + tid % RPR, p = tid / RPR;
    RowLine L{sm + rl + (rl >> 4), G::CS2};
    float2 v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = L.at(p + P * r);
    line_fft<N, false>(v, L, p, a.twx, SyncBlock{});
#pragma unroll
    for (int m = 0; m < 16; ++m) slab[(long long)(p + P * m) * N + rl] = v[m];
  }
}


// The fused step with K3's rows loaded by one tensor copy (TMA) into a dense
// tile instead of two rounds of per-thread loads.
template <int N, int C>
__global__ void __launch_bounds__(kThreads, 2)
    kf_plane_fused_tma(const __grid_constant__ CUtensorMap tslab, InnerArgs a, Wig w1, const float2* __restrict__ src1, float2 A, float2* __restrict__ T,
                   float2* __restrict__ dE, float2* __restrict__ E, const float2* __restrict__ gamma,
                   const DevState* __restrict__ st, double* __restrict__ partials) {
  static_assert(C > 1, "cluster planes only");
  using G = PlaneGeom<N, C, true>;
  constexpr int P = G::P, LPR = G::LPR, M = G::M, LR = G::LR;
  constexpr int RPR = kThreads / P;
  const int rhs = blockIdx.x / a.bpr, bid = blockIdx.x - rhs * a.bpr;
  st += rhs;
  if (load_done(st)) return;  // the same for every block of a cluster
  const bool acc_now = !a.acc2 || (__ldcg(&st->it) & 1) == 0;
  T += rhs * a.fstride;
  dE += rhs * a.fstride;
  E += rhs * a.fstride;
  if (src1) src1 += rhs * a.fstride;
  partials += (long long)rhs * a.bpr;
  gamma += rhs * a.gstride;  // a batch of media: each right-hand side has its own gamma
  extern __shared__ float2 sm[];
  __shared__ float red[kThreads / 32];
  const int tid = threadIdx.x;
  const Geom& g = a.g;
  const int nx = g.nx;
  const int rank = (int)(bid % C), plane = bid / C;
  const int x0 = rank * M, z = plane % g.nz, comp = plane / g.nz;
  const long long colbase = (long long)plane * nx + x0;
  float2* __restrict__ slab = T + (long long)plane * nx * N + rank * LR;  // rows [rank LR, +LR) of the plane
  // K3's rows arrive by one tensor copy: the box {2 LR floats, N columns} of
  // the 2-D view {2 Ny floats, Nx Nz Nc nrhs columns} of T, landing dense:
  // element (row kyl, x) at rt[x * LR + kyl]
  float2* const rt = reinterpret_cast<float2*>((reinterpret_cast<uintptr_t>(sm) + 127) & ~(uintptr_t)127);
  __shared__ __align__(8) uint64_t slab_bar;
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_addr(&slab_bar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(&slab_bar)),
                 "r"((uint32_t)(N * LR * sizeof(float2)))
                 : "memory");
    const int c0 = 2 * rank * LR;
    const int c1 = (int)((long long)rhs * (a.fstride / N) + (long long)plane * nx);
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            smem_addr(rt)),
        "l"(&tslab), "r"(c0), "r"(c1), "r"(smem_addr(&slab_bar))
        : "memory");
    const unsigned bytes = (unsigned)M * N * sizeof(float2);
    prefetch_l2(dE + colbase * N, bytes);
    if (acc_now) prefetch_l2(E + colbase * N, bytes);
    prefetch_l2(gamma + colbase * N - (long long)comp * g.npts, bytes);
    if (src1) prefetch_l2(src1 + colbase * N, bytes);
  }
  cg::cluster_group cl = cg::this_cluster();
  {
    // bounded wait for the rows (phase 0 of slab_bar)
    const uint32_t ba = smem_addr(&slab_bar);
    const long long t0 = clock64();
    bool ok = false;
    while (true) {
      uint32_t done;
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n\t"
          "selp.u32 %0, 1, 0, p;\n\t}"
          : "=r"(done)
          : "r"(ba)
          : "memory");
      if (done) {
        ok = true;
        break;
      }
      if (clock64() - t0 > 50000000LL) break;
    }
    if (!ok && a.err) atomicExch(a.err, 1);
  }
  // K3: inverse x transform of the block's rows, in place
  for (int r0 = 0; r0 < LR; r0 += RPR) {
    const int rl = r0 + tid % RPR, p = tid / RPR;
    float2 v[16];
    RowLine L{rt + rl, LR};
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = L.at(p + P * r);
    line_fft<N, true>(v, L, p, a.twx, SyncBlock{});
#pragma unroll
    for (int m = 0; m < 16; ++m) L.at(p + P * m) = v[m];
  }
  {
    constexpr int PER = M * N / kThreads;
    float2 hold[PER];
    cl.sync();
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int e = tid + kThreads * i;
      const int ky = e % N, c = e / N;
      const float2* rs = cl.map_shared_rank(rt, ky / LR);
      hold[i] = rs[(x0 + c) * LR + ky % LR];
    }
    cl.sync();
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int e = tid + kThreads * i;
      const int ky = e % N, c = e / N;
      sm[c * G::CS + ky + (ky >> 4)] = hold[i];
    }
  }
  __syncthreads();
  const float2 gzz = a.w.gz[z];
  const float2 gzz1 = w1.gz[z];
  float esum = 0.f;
  for (int c0 = 0; c0 < M; c0 += LPR) {
    const int cc = c0 + tid / P, p = tid % P;
    float2 v[16];
    ColLine L{sm + cc * G::CS};
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = L.at(p + P * r);
    if constexpr (P <= 32) {
      line_fft<N, true>(v, L, p, a.py.tw, SyncWarp{});
    } else {
      line_fft<N, true>(v, L, p, a.py.tw, SyncBlock{});
    }
    const int x = x0 + cc;
    const long long col = colbase + cc;
    const float2 gxz = cmul(a.w.gx[x], gzz);
    const bool in_xzc = x >= g.r0[1] && x < g.r1[1] && z >= g.r0[2] && z < g.r1[2] && comp >= g.r0[3] && comp < g.r1[3];
    const long long gcol = col * N;
    const float2* __restrict__ gmc = gamma + (gcol - (long long)comp * g.npts);
    float2* __restrict__ dEc = dE + gcol;
    float2* __restrict__ Ec = E + gcol;
    // K3's epilogue (unwiggle, f_mix, E' += dE', ROI energy); v[m] becomes dE'_k(y)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float2 gm[8], d0[8], e0[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int y = p + P * (8 * h + i);
        gm[i] = gmc[y];
        d0[i] = dEc[y];
        e0[i] = acc_now ? Ec[y] : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int m = 8 * h + i;
        const int y = p + P * m;
        const float2 ep = cmul_conj(cmul_conj(v[m], gxz), a.w.gy[y]);
        const float2 one_m = make_float2(1.f - kAlpha * gm[i].x, -kAlpha * gm[i].y);
        const float2 t = cmul(cmul(gm[i], gm[i]), ep);
        const float2 dn = cadd(cmul(one_m, d0[i]), make_float2(kAlpha * t.y, -kAlpha * t.x));
        dEc[y] = dn;
        if (acc_now) Ec[y] = cadd(e0[i], a.acc2 ? cadd(d0[i], dn) : dn);
        if (in_xzc && y >= g.r0[0] && y < g.r1[0]) esum = fmaf(dn.x, dn.x, fmaf(dn.y, dn.y, esum));
        v[m] = dn;
      }
    }
    // K1 of iteration k + 1 on the same column: source, next ramps, y transform
    const float2 gxz1 = cmul(w1.gx[x], gzz1);
    const float2* __restrict__ sr = src1 ? src1 + gcol : nullptr;
#pragma unroll
    for (int m = 0; m < 16; ++m) {
      const int y = p + P * m;
      float2 e = v[m];
      if (sr) e = cadd(e, cmul(A, sr[y]));
      v[m] = cmul(cmul(e, gxz1), w1.gy[y]);
    }
    if constexpr (P <= 32) {
      line_fft<N, false>(v, L, p, a.py.tw, SyncWarp{});
    } else {
      line_fft<N, false>(v, L, p, a.py.tw, SyncBlock{});
    }
#pragma unroll
    for (int m = 0; m < 16; ++m) L.at(p + P * m) = v[m];
  }
  // the ROI energy of dE'_k
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) esum += __shfl_xor_sync(0xffffffffu, esum, o);
  if ((tid & 31) == 0) red[tid >> 5] = esum;
  // rows [rank LR, +LR) of all N transformed columns, from the blocks holding them
  {
    constexpr int PER = LR * N / kThreads;
    float2 hold[PER];
    cl.sync();
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int e = tid + kThreads * i;
      const int kyl = e % LR, x = e / LR;
      const int ky = rank * LR + kyl;
      const float2* rs = cl.map_shared_rank(sm, x / M);
      hold[i] = rs[(x % M) * G::CS + ky + (ky >> 4)];
    }
    cl.sync();
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int e = tid + kThreads * i;
      const int kyl = e % LR, x = e / LR;
      sm[x * G::CS2 + kyl + (kyl >> 4)] = hold[i];
    }
  }
  __syncthreads();
  if (tid < 32) {
    float v = tid < kThreads / 32 ? red[tid] : 0.f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (tid == 0) partials[bid] = (double)v;
  }
  // K1's x transform of the block's rows, written over the slab K3 read
  for (int r0 = 0; r0 < LR; r0 += RPR) {
    const int rl = r0 + tid % RPR, p = tid / RPR;
    RowLine L{sm + rl + (rl >> 4), G::CS2};
    float2 v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = L.at(p + P * r);
    line_fft<N, false>(v, L, p, a.twx, SyncBlock{});
#pragma unroll
    for (int m = 0; m < 16; ++m) slab[(long long)(p + P * m) * N + rl] = v[m];
  }
}


// The fused step split into passes that need no cluster (the default loop of
// 3-D power-of-two planes).  K3 of iteration k followed by K1 of iteration
// k + 1 is an inverse 2-D (y, x) transform, the pointwise epilogue and a
// forward 2-D transform of every z plane; run as
//   kt_xpencil<.., INV>  inverse x transforms (TMA-pipelined pencils along x)
//   kc_col_step<N, C>    per (x, z) column: inverse y transform, unwiggle,
//                        f_mix, E' += dE', ROI energy, the next iteration's
//                        source and ramps, forward y transform
//   kt_xpencil<.., FWD>  forward x transforms
// each pass reads and writes whole contiguous lines, so no block waits for
// another.  It moves 80 instead of 48 bytes per point, but each pass streams
// at close to the HBM bandwidth where the cluster exchange of the one-kernel
// step left it latency bound.
//
// kc_col_step covers the columns of the plane kernels' block (plane, rank):
// x0 = rank M .. x0 + M - 1 at z, with the same thread of each line, the same
// arithmetic in the same order (line_fft, the epilogue of kf_plane_fused) and
// the same per-block energy partial, so its fields equal the one-kernel
// step's bit for bit.
template <int N, int C>
__global__ void __launch_bounds__(kThreads, 2)
    kc_col_step(InnerArgs a, Wig w1, const float2* __restrict__ src1, float2 A, float2* __restrict__ T,
                float2* __restrict__ dE, float2* __restrict__ E, const float2* __restrict__ gamma,
                const DevState* __restrict__ st, double* __restrict__ partials) {
  pdl_begin();
  using G = PlaneGeom<N, C, true>;
  constexpr int P = G::P, LPR = G::LPR, M = G::M;
  static_assert(M % LPR == 0, "whole rounds of lines");
  // blocks in reverse order: the pass starts on the planes the inverse x
  // pencils wrote last (still in L2), and ends on the planes the forward x
  // pencils read first; a block's columns and energy partial do not change
  const int rb = (int)gridDim.x - 1 - (int)blockIdx.x;
  const int rhs = rb / a.bpr, bid = rb - rhs * a.bpr;
  st += rhs;
  if (load_done(st)) return;
  const bool acc_now = !a.acc2 || (__ldcg(&st->it) & 1) == 0;
  T += rhs * a.fstride;
  dE += rhs * a.fstride;
  E += rhs * a.fstride;
  if (src1) src1 += rhs * a.fstride;
  partials += (long long)rhs * a.bpr;
  gamma += rhs * a.gstride;  // a batch of media: each right-hand side has its own gamma
  __shared__ float2 sm[LPR * G::CS];  // one round of lines: the transforms' exchanges
  __shared__ float red[kThreads / 32];
  const int tid = threadIdx.x;
  const Geom& g = a.g;
  const int nx = g.nx;
  const int rank = (int)(bid % C), plane = bid / C;
  const int x0 = rank * M, z = plane % g.nz, comp = plane / g.nz;
  const long long colbase = (long long)plane * nx + x0;
  if (tid == 0) {
    // the block's M columns of gamma, dE' (and E', the next source) are
    // contiguous: pull them into L2 now, so that the epilogue's loads, which
    // wait for the inverse transform, find them there
    const long long off = colbase * N;
    constexpr unsigned bytes = (unsigned)(M * N * sizeof(float2));
    prefetch_l2(gamma + (off - (long long)comp * g.npts), bytes);
    prefetch_l2(dE + off, bytes);
    if (acc_now) prefetch_l2(E + off, bytes);
    if (src1) prefetch_l2(src1 + off, bytes);
  }
  // the y ramps of this and the next wiggle, read from shared memory: as
  // per-element global loads inside the epilogue they left the pass latency
  // bound (0.19 against 0.12 ms at 256^3)
  __shared__ float2 sgy[2 * N];
  for (int i = tid; i < N; i += kThreads) {
    sgy[i] = a.w.gy[i];
    sgy[N + i] = w1.gy[i];
  }
  __syncthreads();
  const float2 gzz = a.w.gz[z];
  const float2 gzz1 = w1.gz[z];
  float esum = 0.f;
  for (int c0 = 0; c0 < M; c0 += LPR) {
    const int cl = tid / P, cc = c0 + cl, p = tid % P;
    const int x = x0 + cc;
    const long long col = colbase + cc;
    const long long gcol = col * N;
    float2* __restrict__ Tc = T + gcol;
    float2 v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = Tc[p + P * r];
    ColLine L{sm + cl * G::CS};
    if constexpr (P <= 32) {
      line_fft<N, true>(v, L, p, a.py.tw, SyncWarp{});
    } else {
      line_fft<N, true>(v, L, p, a.py.tw, SyncBlock{});
    }
    const float2 gxz = cmul(a.w.gx[x], gzz);
    const bool in_xzc = x >= g.r0[1] && x < g.r1[1] && z >= g.r0[2] && z < g.r1[2] && comp >= g.r0[3] && comp < g.r1[3];
    const float2* __restrict__ gmc = gamma + (gcol - (long long)comp * g.npts);
    float2* __restrict__ dEc = dE + gcol;
    float2* __restrict__ Ec = E + gcol;
    // K3's epilogue (unwiggle, f_mix, E' += dE', ROI energy); v[m] becomes dE'_k(y)
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float2 gm[8], d0[8], e0[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int y = p + P * (8 * h + i);
        gm[i] = gmc[y];
        d0[i] = dEc[y];
        e0[i] = acc_now ? Ec[y] : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int m = 8 * h + i;
        const int y = p + P * m;
        const float2 ep = cmul_conj(cmul_conj(v[m], gxz), sgy[y]);
        const float2 one_m = make_float2(1.f - kAlpha * gm[i].x, -kAlpha * gm[i].y);
        const float2 t = cmul(cmul(gm[i], gm[i]), ep);
        const float2 dn = cadd(cmul(one_m, d0[i]), make_float2(kAlpha * t.y, -kAlpha * t.x));
        dEc[y] = dn;
        if (acc_now) Ec[y] = cadd(e0[i], a.acc2 ? cadd(d0[i], dn) : dn);
        if (in_xzc && y >= g.r0[0] && y < g.r1[0]) esum = fmaf(dn.x, dn.x, fmaf(dn.y, dn.y, esum));
        v[m] = dn;
      }
    }
    // K1 of iteration k + 1 on the same column: source, next ramps, y transform
    const float2 gxz1 = cmul(w1.gx[x], gzz1);
    const float2* __restrict__ sr = src1 ? src1 + gcol : nullptr;
#pragma unroll
    for (int m = 0; m < 16; ++m) {
      const int y = p + P * m;
      float2 e = v[m];
      if (sr) e = cadd(e, cmul(A, sr[y]));
      v[m] = cmul(cmul(e, gxz1), sgy[N + y]);
    }
    if constexpr (P <= 32) {
      line_fft<N, false>(v, L, p, a.py.tw, SyncWarp{});
    } else {
      line_fft<N, false>(v, L, p, a.py.tw, SyncBlock{});
    }
#pragma unroll
    for (int m = 0; m < 16; ++m) Tc[p + P * m] = v[m];
  }
  // the ROI energy of dE'_k, reduced as in the one-kernel step
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) esum += __shfl_xor_sync(0xffffffffu, esum, o);
  if ((tid & 31) == 0) red[tid >> 5] = esum;
  __syncthreads();
  if (tid < 32) {
    float v = tid < kThreads / 32 ? red[tid] : 0.f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (tid == 0) partials[bid] = (double)v;
  }
  if (a.fin) finish_in_last_block(const_cast<DevState*>(st), a.rule, a.hist, partials, a.bpr, rhs);
}

// The 2-D form: K2 already transforms along x, so K3 of iteration k and K1
// of iteration k + 1 meet in one column pass, and an iteration is K2 plus
// this kernel.  Block bid covers the 2-D column kernels' columns bid ncols
// ... bid ncols + ncols - 1 (column col = x + Nx c), the same lines and
// arithmetic as kf_plane_inv / kf_plane_fwd on a column (so the same
// fields bit for bit) and their energy partial.  Idle lanes of a partial
// last block work on a scratch column.  Dynamic shared memory:
// (LPR + 1) columns and the two y ramps (smem_col_step2d).
template <int N>
__host__ __device__ constexpr size_t smem_col_step2d() {
  return ((size_t)(kThreads / (N / 16) + 1) * PlaneGeom<N, 1, false>::CS + 2 * N) * sizeof(float2);
}
template <int N>
__global__ void __launch_bounds__(kThreads, 2)
    kc_col_step2d(InnerArgs a, Wig w1, const float2* __restrict__ src1, float2 A, float2* __restrict__ T,
                  float2* __restrict__ dE, float2* __restrict__ E, const float2* __restrict__ gamma,
                  const DevState* __restrict__ st, double* __restrict__ partials) {
  pdl_begin();
  using G = PlaneGeom<N, 1, false>;
  constexpr int P = G::P, LPR = G::LPR;
  const int rhs = blockIdx.x / a.bpr, bid = blockIdx.x - rhs * a.bpr;
  st += rhs;
  if (load_done(st)) return;
  const bool acc_now = !a.acc2 || (__ldcg(&st->it) & 1) == 0;
  T += rhs * a.fstride;
  dE += rhs * a.fstride;
  E += rhs * a.fstride;
  if (src1) src1 += rhs * a.fstride;
  partials += (long long)rhs * a.bpr;
  gamma += rhs * a.gstride;  // a batch of media: each right-hand side has its own gamma
  extern __shared__ float2 sm[];
  float2* const sgy = sm + (LPR + 1) * G::CS;
  __shared__ float red[kThreads / 32];
  const int tid = threadIdx.x;
  for (int i = tid; i < N; i += kThreads) {
    sgy[i] = a.w.gy[i];
    sgy[N + i] = w1.gy[i];
  }
  __syncthreads();
  const Geom& g = a.g;
  const int nx = g.nx;
  const int M = a.ncols;
  const long long colbase = (long long)bid * M;
  const int ncol = (int)min((long long)M, (long long)nx * g.nc - colbase);
  const int z = 0;
  const float2 gzz = a.w.gz[z];
  const float2 gzz1 = w1.gz[z];
  float esum = 0.f;
  for (int c0 = 0; c0 < ncol; c0 += LPR) {
    const int cl = tid / P, cc = c0 + cl, p = tid % P;
    const bool live = cc < ncol;
    const long long col = colbase + cc;
    const long long gcol = col * N;
    ColLine L{sm + (live ? cl : LPR) * G::CS};
    float2 v[16];
    if (live) {
#pragma unroll
      for (int r = 0; r < 16; ++r) v[r] = T[gcol + p + P * r];
    } else {
#pragma unroll
      for (int r = 0; r < 16; ++r) v[r] = make_float2(0.f, 0.f);
    }
    if constexpr (P <= 32) {
      line_fft<N, true>(v, L, p, a.py.tw, SyncWarp{});
    } else {
      line_fft<N, true>(v, L, p, a.py.tw, SyncBlock{});
    }
    if (live) {
      const int x = (int)(col % nx), c = (int)(col / nx);
      const float2 gxz = cmul(a.w.gx[x], gzz);
      const bool in_xzc = x >= g.r0[1] && x < g.r1[1] && z >= g.r0[2] && z < g.r1[2] && c >= g.r0[3] && c < g.r1[3];
      const float2* __restrict__ gmc = gamma + (gcol - (long long)c * g.npts);
      float2* __restrict__ dEc = dE + gcol;
      float2* __restrict__ Ec = E + gcol;
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        float2 gm[8], d0[8], e0[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int y = p + P * (8 * h + i);
          gm[i] = gmc[y];
          d0[i] = dEc[y];
          e0[i] = acc_now ? Ec[y] : make_float2(0.f, 0.f);
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const int m = 8 * h + i;
          const int y = p + P * m;
          const float2 ep = cmul_conj(cmul_conj(v[m], gxz), sgy[y]);
          const float2 one_m = make_float2(1.f - kAlpha * gm[i].x, -kAlpha * gm[i].y);
          const float2 t = cmul(cmul(gm[i], gm[i]), ep);
          const float2 dn = cadd(cmul(one_m, d0[i]), make_float2(kAlpha * t.y, -kAlpha * t.x));
          dEc[y] = dn;
          if (acc_now) Ec[y] = cadd(e0[i], a.acc2 ? cadd(d0[i], dn) : dn);
          if (in_xzc && y >= g.r0[0] && y < g.r1[0]) esum = fmaf(dn.x, dn.x, fmaf(dn.y, dn.y, esum));
          v[m] = dn;
        }
      }
      const float2 gxz1 = cmul(w1.gx[x], gzz1);
      const float2* __restrict__ sr = src1 ? src1 + gcol : nullptr;
#pragma unroll
      for (int m = 0; m < 16; ++m) {
        const int y = p + P * m;
        float2 e = v[m];
        if (sr) e = cadd(e, cmul(A, sr[y]));
        v[m] = cmul(cmul(e, gxz1), sgy[N + y]);
      }
    }
    if constexpr (P <= 32) {
      line_fft<N, false>(v, L, p, a.py.tw, SyncWarp{});
    } else {
      line_fft<N, false>(v, L, p, a.py.tw, SyncBlock{});
    }
    if (live) {
#pragma unroll
      for (int m = 0; m < 16; ++m) T[gcol + p + P * m] = v[m];
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) esum += __shfl_xor_sync(0xffffffffu, esum, o);
  if ((tid & 31) == 0) red[tid >> 5] = esum;
  __syncthreads();
  if (tid < 32) {
    float v = tid < kThreads / 32 ? red[tid] : 0.f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (tid == 0) partials[bid] = (double)v;
  }
  if (a.fin) finish_in_last_block(const_cast<DevState*>(st), a.rule, a.hist, partials, a.bpr, rhs);
}

// The same fused step with K1's half of the plane exchange pushed: each block
// sends its transformed columns to the row owners with st.async, completion
// counted in bytes on the receiver's mbarrier (as in kf_plane_fwd), instead of
// two more cluster barriers, whose release would wait for the epilogue's
// global stores.  The received rows land in the region that held K3's rows,
// dead after K3's exchange; the column tile is separate, so the tiles must be
// small: 256^2 planes on 16 blocks (16 columns and 16 rows each).
template <int N, int C>
struct FusedPushGeom {
  using G = PlaneGeom<N, C, true>;
  static constexpr size_t col_bytes = (size_t)G::M * G::CS * sizeof(float2);  // one round of columns
  static constexpr size_t row_bytes = (size_t)N * G::CS2 * sizeof(float2);
  static constexpr size_t smem = col_bytes + row_bytes;
  static_assert(G::M == G::LPR, "one round of columns");
  static_assert(col_bytes % 16 == 0, "the row tile starts on a 16-byte boundary");
};

template <int N, int C>
__global__ void __launch_bounds__(kThreads, 2)
    kf_plane_fused_push(InnerArgs a, Wig w1, const float2* __restrict__ src1, float2 A, float2* __restrict__ T,
                        float2* __restrict__ dE, float2* __restrict__ E, const float2* __restrict__ gamma,
                        const DevState* __restrict__ st, double* __restrict__ partials) {
  using G = PlaneGeom<N, C, true>;
  using F = FusedPushGeom<N, C>;
  constexpr int P = G::P, M = G::M, LR = G::LR;
  constexpr int RPR = kThreads / P;
  const int rhs = blockIdx.x / a.bpr, bid = blockIdx.x - rhs * a.bpr;
  st += rhs;
  if (load_done(st)) return;  // the same for every block of a cluster
  const bool acc_now = !a.acc2 || (__ldcg(&st->it) & 1) == 0;
  T += rhs * a.fstride;
  dE += rhs * a.fstride;
  E += rhs * a.fstride;
  if (src1) src1 += rhs * a.fstride;
  partials += (long long)rhs * a.bpr;
  gamma += rhs * a.gstride;  // a batch of media: each right-hand side has its own gamma
  extern __shared__ float2 sm[];
  float2* const ct = sm;                                       // columns [x0, x0 + M), stride CS
  float2* const rt = sm + F::col_bytes / sizeof(float2);       // rows: K3's, then the pushed ones; stride CS2
  __shared__ float red[kThreads / 32];
  __shared__ __align__(8) uint64_t recv_bar;
  const int tid = threadIdx.x;
  const Geom& g = a.g;
  const int nx = g.nx;
  const int rank = (int)(bid % C), plane = bid / C;
  const int x0 = rank * M, z = plane % g.nz, comp = plane / g.nz;
  const long long colbase = (long long)plane * nx + x0;
  float2* __restrict__ slab = T + (long long)plane * nx * N + rank * LR;
  if (tid == 0) {
    mbar_init_expect(&recv_bar, (uint32_t)(LR * N * sizeof(float2)));
    const unsigned bytes = (unsigned)M * N * sizeof(float2);
    prefetch_l2(dE + colbase * N, bytes);
    if (acc_now) prefetch_l2(E + colbase * N, bytes);
    prefetch_l2(gamma + colbase * N - (long long)comp * g.npts, bytes);
    if (src1) prefetch_l2(src1 + colbase * N, bytes);
  }
  cg::cluster_group cl = cg::this_cluster();
  // K3: inverse x transform of the block's rows
  for (int r0 = 0; r0 < LR; r0 += RPR) {
    const int rl = r0 + tid % RPR, p = tid / RPR;
    float2 v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = slab[(long long)(p + P * r) * N + rl];
    RowLine L{rt + rl + (rl >> 4), G::CS2};
    line_fft<N, true>(v, L, p, a.twx, SyncBlock{});
#pragma unroll
    for (int m = 0; m < 16; ++m) L.at(p + P * m) = v[m];
  }
  {
    constexpr int PER = M * N / kThreads;
    float2 hold[PER];
    cl.sync();  // also publishes every block's armed recv_bar
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int e = tid + kThreads * i;
      const int ky = e % N, c = e / N;
      const float2* rs = cl.map_shared_rank(rt, ky / LR);
      const int kyl = ky % LR;
      hold[i] = rs[(x0 + c) * G::CS2 + kyl + (kyl >> 4)];
    }
    cl.sync();  // every row tile is dead from here on: pushes may land in it
#pragma unroll
    for (int i = 0; i < PER; ++i) {
      const int e = tid + kThreads * i;
      const int ky = e % N, c = e / N;
      ct[c * G::CS + ky + (ky >> 4)] = hold[i];
    }
  }
  __syncthreads();
  float esum = 0.f;
  {
    const int cc = tid / P, p = tid % P;
    float2 v[16];
    ColLine L{ct + cc * G::CS};
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = L.at(p + P * r);
    if constexpr (P <= 32) {
      line_fft<N, true>(v, L, p, a.py.tw, SyncWarp{});
    } else {
      line_fft<N, true>(v, L, p, a.py.tw, SyncBlock{});
    }
    const int x = x0 + cc;
    const long long col = colbase + cc;
    const float2 gxz = cmul(a.w.gx[x], a.w.gz[z]);
    const bool in_xzc = x >= g.r0[1] && x < g.r1[1] && z >= g.r0[2] && z < g.r1[2] && comp >= g.r0[3] && comp < g.r1[3];
    const long long gcol = col * N;
    const float2* __restrict__ gmc = gamma + (gcol - (long long)comp * g.npts);
    float2* __restrict__ dEc = dE + gcol;
    float2* __restrict__ Ec = E + gcol;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      float2 gm[8], d0[8], e0[8];
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int y = p + P * (8 * h + i);
        gm[i] = gmc[y];
        d0[i] = dEc[y];
        e0[i] = acc_now ? Ec[y] : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int i = 0; i < 8; ++i) {
        const int m = 8 * h + i;
        const int y = p + P * m;
        const float2 ep = cmul_conj(cmul_conj(v[m], gxz), a.w.gy[y]);
        const float2 one_m = make_float2(1.f - kAlpha * gm[i].x, -kAlpha * gm[i].y);
        const float2 t = cmul(cmul(gm[i], gm[i]), ep);
        const float2 dn = cadd(cmul(one_m, d0[i]), make_float2(kAlpha * t.y, -kAlpha * t.x));
        dEc[y] = dn;
        if (acc_now) Ec[y] = cadd(e0[i], a.acc2 ? cadd(d0[i], dn) : dn);
        if (in_xzc && y >= g.r0[0] && y < g.r1[0]) esum = fmaf(dn.x, dn.x, fmaf(dn.y, dn.y, esum));
        v[m] = dn;
      }
    }
    // K1 of iteration k + 1 on the same column
    const float2 gxz1 = cmul(w1.gx[x], w1.gz[z]);
    const float2* __restrict__ sr = src1 ? src1 + gcol : nullptr;
#pragma unroll
    for (int m = 0; m < 16; ++m) {
      const int y = p + P * m;
      float2 e = v[m];
      if (sr) e = cadd(e, cmul(A, sr[y]));
      v[m] = cmul(cmul(e, gxz1), w1.gy[y]);
    }
    if constexpr (P <= 32) {
      line_fft<N, false>(v, L, p, a.py.tw, SyncWarp{});
    } else {
      line_fft<N, false>(v, L, p, a.py.tw, SyncBlock{});
    }
    // X[ky] of column x to the block holding row ky, in 16-byte pairs (ky, ky + 1)
    // as in kf_plane_fwd
    float2 w[16];
#pragma unroll
    for (int m = 0; m < 16; ++m) {
      w[m].x = __shfl_xor_sync(0xffffffffu, v[m].x, 1);
      w[m].y = __shfl_xor_sync(0xffffffffu, v[m].y, 1);
    }
    const uint32_t lbar = smem_addr(&recv_bar);
    const bool odd = p & 1;
#pragma unroll
    for (int h = 0; h < 8; ++h) {
      const int m = odd ? 8 + h : h;
      const int ky = (p & ~1) + P * m;
      const int dst = ky / LR, kyl = ky - dst * LR;
      const uint32_t la = smem_addr(rt + x * G::CS2 + kyl + 2 * (kyl >> 4));
      const float2 lo = odd ? w[8 + h] : v[h], hi = odd ? v[8 + h] : w[h];
      st_async_f4(map_rank(la, dst), lo, hi, map_rank(lbar, dst));
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) esum += __shfl_xor_sync(0xffffffffu, esum, o);
  if ((tid & 31) == 0) red[tid >> 5] = esum;
  if (!mbar_wait_cluster(&recv_bar)) {
    if (a.err) atomicExch(a.err, 1);
  }
  __syncthreads();
  if (tid < 32) {
    float v = tid < kThreads / 32 ? red[tid] : 0.f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (tid == 0) partials[bid] = (double)v;
  }
  // K1's x transform of the received rows, written over the slab K3 read
  for (int r0 = 0; r0 < LR; r0 += RPR) {
    const int rl = r0 + tid % RPR, p = tid / RPR;
    RowLine L{rt + rl + 2 * (rl >> 4), G::CS2};
    float2 v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = L.at(p + P * r);
    line_fft<N, false>(v, L, p, a.twx, SyncBlock{});
#pragma unroll
    for (int m = 0; m < 16; ++m) slab[(long long)(p + P * m) * N + rl] = v[m];
  }
  // (no block leaves before every push into it has arrived: recv_bar)
}

}  // namespace fast
}  // namespace ws
