// Shared-memory mixed-radix FFT engine for the MBS kernels.
//
// Many 1-D transforms ("lines") of one length n live in a shared-memory tile
// and are transformed in place by Stockham autosort stages.  A stage of radix
// R with span Ns (the product of the radices before it) takes butterfly j of a
// line from the inputs j + r*n/R, multiplies input r by W_{Ns R}^{(j mod Ns) r},
// runs an R-point DFT in registers and writes output r to
//   (j - j mod Ns) * R + (j mod Ns) + r * Ns.
// Threads read all of their inputs, synchronise, then write; so one buffer
// suffices and a 128 KB tile needs no ping-pong copy.
//
// Two tile layouts (both padded by one slot every 16 elements along the
// contiguous index, which keeps the strided accesses of a stage free of bank
// conflicts):
//   contiguous lines: addr(l, i) = l * stride + i + (i >> 4)    (y columns)
//   interleaved lines: addr(l, i) = i * stride + l + (l >> 4)   (x rows, z pencils)
// For interleaved lines consecutive threads take consecutive lines, so a warp
// touches consecutive addresses whatever the element stride.
#pragma once
#include <cuda_runtime.h>
#include "ws_codelets.cuh"

namespace ws {

constexpr int kMaxStages = 12;

__host__ __device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(fmaf(a.x, b.x, -a.y * b.y), fmaf(a.x, b.y, a.y * b.x));
}
__host__ __device__ __forceinline__ float2 cmul_conj(float2 a, float2 b) {  // a * conj(b)
  return make_float2(fmaf(a.x, b.x, a.y * b.y), fmaf(a.y, b.x, -a.x * b.y));
}
__host__ __device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__host__ __device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__host__ __device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

// One transform length and its radix schedule.  tw[k] = exp(-2 pi i k / n),
// computed on the host in double precision and stored as float.
struct FftPlan {
  int n;
  int nst;
  int radix[kMaxStages];
  const float2* tw;
};

struct Lines {
  int nlines;
  int stride;
  int contiguous;
  __device__ __forceinline__ int addr(int l, int i) const {
    return contiguous ? l * stride + i + (i >> 4) : i * stride + l + (l >> 4);
  }
};

// padded length of a contiguous run of n elements
__host__ __device__ __forceinline__ int padded(int n) { return n + ((n + 15) >> 4); }

template <int R, int Q, bool INV>
__device__ __forceinline__ void fft_stage(float2* __restrict__ s, const Lines L, int n, int Ns,
                                          const float2* __restrict__ tw, int tid, int nthr) {
  const int nb = n / R;
  const int total = L.nlines * nb;
  const int tstride = n / (Ns * R);
  float2 v[Q][R];
  int ob[Q], lb[Q];
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    const int b = tid + q * nthr;
    lb[q] = -1;
    if (b < total) {
      int l, j;
      if (L.contiguous) {
        l = b / nb;
        j = b - l * nb;
      } else {
        j = b / L.nlines;
        l = b - j * L.nlines;
      }
#pragma unroll
      for (int r = 0; r < R; ++r) v[q][r] = s[L.addr(l, j + r * nb)];
      const int jm = j % Ns;
      if (jm != 0) {
#pragma unroll
        for (int r = 1; r < R; ++r) {
          float2 w = __ldg(&tw[jm * r * tstride]);
          if (INV) w.y = -w.y;
          v[q][r] = cmul(v[q][r], w);
        }
      }
      Dft<R, INV>::run(v[q]);
      ob[q] = (j - jm) * R + jm;
      lb[q] = l;
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < Q; ++q) {
    if (lb[q] >= 0) {
#pragma unroll
      for (int r = 0; r < R; ++r) s[L.addr(lb[q], ob[q] + r * Ns)] = v[q][r];
    }
  }
  __syncthreads();
}

// Radix sets a kernel is compiled for.  kPow2 kernels (radices 16, 8, 4, 2)
// keep at most 16 elements per thread in registers and may run 1024 threads;
// kMixed kernels add 3, 5, 6, 7, 9, 10, 11, 12, 13 and run at most 512 threads
// (128 registers per thread).
constexpr int kPow2 = 0;
constexpr int kMixed = 1;

// Runs every stage of plan p on the lines L of tile s.  All threads of the
// block must call it.  EMAX bounds ceil(elements / threads) of the tile.
template <bool INV, int EMAX, int RSET>
__device__ __forceinline__ void fft_lines(float2* __restrict__ s, const Lines L, const FftPlan& p, int tid, int nthr) {
  int Ns = 1;
  for (int st = 0; st < p.nst; ++st) {
    const int R = p.radix[st];
    switch (R) {
#define WS_STAGE(RR) \
  case RR:           \
    fft_stage<RR, (EMAX + RR - 1) / RR, INV>(s, L, p.n, Ns, p.tw, tid, nthr); \
    break;
      WS_STAGE(16)
      WS_STAGE(8)
      WS_STAGE(4)
      WS_STAGE(2)
#undef WS_STAGE
      default:
        if constexpr (RSET == kMixed) {
          switch (R) {
#define WS_STAGE(RR) \
  case RR:           \
    fft_stage<RR, (EMAX + RR - 1) / RR, INV>(s, L, p.n, Ns, p.tw, tid, nthr); \
    break;
            WS_STAGE(3)
            WS_STAGE(5)
            WS_STAGE(6)
            WS_STAGE(7)
            WS_STAGE(9)
            WS_STAGE(10)
            WS_STAGE(11)
            WS_STAGE(12)
            WS_STAGE(13)
#undef WS_STAGE
            default:
              break;
          }
        }
        break;
    }
    Ns *= R;
  }
}

}  // namespace ws
