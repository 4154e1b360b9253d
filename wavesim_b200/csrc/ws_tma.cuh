// K2 as a persistent, TMA-pipelined kernel (sm_100a): the outer-dimension
// (z) pencils of a 3-D grid, TY consecutive y per tile.  Each block walks
// its tiles t = blockIdx.x, blockIdx.x + gridDim.x, ...; while it
// transforms one tile (FFT along z, Green's function, inverse FFT; registers
// plus an in-place exchange in the tile's own buffer), the tensor-memory
// access unit holds the loads of the next S - 2 tiles (S - 1 in the second
// half) and the store of the previous one, so that HBM never waits for the
// arithmetic.
//   load:  cp.async.bulk.tensor.3d, box {2 TY floats, 1, NO} of the map
//          {2 Ny floats, Nx, Nz * nrhs} over T, completing on the buffer's
//          mbarrier with the byte count
//   store: cp.async.bulk.tensor.3d from the same buffer, bulk group; a buffer
//          is reloaded only after the store that reads it has read it
//          (cp.async.bulk.wait_group.read)
// The tensor map spans this GPU's own T only (no multicast).  Every wait is
// bounded: a block whose load does not arrive in a.wait_clocks clocks (5e7 by
// default) sets *err, drains its copies (with the default bound, so that no
// copy outlives its block) and returns.
#pragma once
#include <cuda.h>

#include "ws_mixed.cuh"

namespace ws {
namespace tma {

__device__ __forceinline__ void load_3d(uint32_t dst, const CUtensorMap* map, int c0, int c1, int c2, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(
          dst),
      "l"(map), "r"(c0), "r"(c1), "r"(c2), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void store_3d(const CUtensorMap* map, int c0, int c1, int c2, uint32_t src) {
  asm volatile("cp.async.bulk.tensor.3d.global.shared::cta.bulk_group [%0, {%1, %2, %3}], [%4];" ::"l"(map), "r"(c0),
               "r"(c1), "r"(c2), "r"(src)
               : "memory");
}
__device__ __forceinline__ void bulk_commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }
// every committed store group has read its shared memory
__device__ __forceinline__ void bulk_wait_read_0() { asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory"); }
__device__ __forceinline__ void bulk_wait_all() { asm volatile("cp.async.bulk.wait_group 0;" ::: "memory"); }
__device__ __forceinline__ void expect_bytes(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fast::smem_addr(bar)), "r"(bytes)
               : "memory");
}
constexpr long long kWaitClocks = 50000000LL;  // ~25 ms at 2 GHz: the default bound of every wait

// phase with parity `parity` of the barrier complete; false after `limit`
// clocks.  With the default bound the thread may be suspended inside
// mbarrier.try_wait until the phase completes; a shorter bound polls with
// the non-blocking mbarrier.test_wait, so that the bound itself decides.
__device__ __forceinline__ bool wait_parity(uint64_t* bar, uint32_t parity, long long limit = kWaitClocks) {
  const uint32_t a = fast::smem_addr(bar);
  const long long t0 = clock64();
  const bool poll = limit < kWaitClocks;
  while (true) {
    uint32_t done;
    if (poll)
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "mbarrier.test_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
          "selp.u32 %0, 1, 0, p;\n\t}"
          : "=r"(done)
          : "r"(a), "r"(parity)
          : "memory");
    else
      asm volatile(
          "{\n\t.reg .pred p;\n\t"
          "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
          "selp.u32 %0, 1, 0, p;\n\t}"
          : "=r"(done)
          : "r"(a), "r"(parity)
          : "memory");
    if (done) return true;
    if (clock64() - t0 > limit) return false;
  }
}

template <int NO, int TY, int S>
struct PencilTile {
  static_assert(NO >= 32 && NO <= 256, "a TMA box dimension holds at most 256 elements");
  static_assert(2 * TY * 4 % 16 == 0 && 2 * TY <= 256, "inner box extent");
  static constexpr int P = NO / 16;
  static constexpr int kThreads = TY * P;
  static constexpr unsigned kTileBytes = NO * TY * sizeof(float2);
  // S tile buffers, [z][y] as the TMA box lands (128-byte aligned)
  static constexpr size_t smem = S * (size_t)kTileBytes + 128;
  // blocks per SM the tiles leave room for (228 KB of shared memory, 1 KB
  // reserved per block, at most 4): the register bound of the kernels
  static constexpr int kMinBlocks = (int)(228 * 1024 / (smem + 3 * 1024)) >= 4 ? 4
                                    : ((int)(228 * 1024 / (smem + 3 * 1024)) >= 3 ? 3 : 2);
};

template <int NO, int TY, int S>
__global__ void __launch_bounds__(PencilTile<NO, TY, S>::kThreads, PencilTile<NO, TY, S>::kMinBlocks)
    kt_pencil(const __grid_constant__ CUtensorMap tmap, OuterArgs a, const DevState* __restrict__ st, int ntiles,
              int* __restrict__ err) {
  pdl_begin();
  using PT = PencilTile<NO, TY, S>;
  constexpr int P = PT::P;
  extern __shared__ uint8_t smem_raw[];
  float2* const buf0 = reinterpret_cast<float2*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
  __shared__ __align__(8) uint64_t full[S];
  const Geom& g = a.g;
  const int tid = threadIdx.x;
  const int yl = tid % TY, p = tid / TY;
  const int nyt = g.ny / TY;
  const int per_rhs = nyt * g.nx;
  if (tid == 0) {
#pragma unroll
    for (int b = 0; b < S; ++b) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(fast::smem_addr(&full[b])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  // tile t -> (rhs, x = mid, y tile)
  auto coords = [&](int t, int& rhs, int& mid, int& yt) {
    rhs = t / per_rhs;
    const int r = t - rhs * per_rhs;
    mid = r / nyt;
    yt = r - mid * nyt;
  };
  auto issue = [&](int t, int b) {
    int rhs, mid, yt;
    coords(t, rhs, mid, yt);
    expect_bytes(&full[b], PT::kTileBytes);
    load_3d(fast::smem_addr(buf0 + b * NO * TY), &tmap, 2 * TY * yt, mid, rhs * g.nz, fast::smem_addr(&full[b]));
  };
  const int G = gridDim.x;
  const int mine = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / G + 1 : 0;  // tiles of this block
  if (tid == 0)
    for (int i = 0; i < S - 1 && i < mine; ++i) issue(blockIdx.x + i * G, i);
  float2 wt[16];  // the second stage's twiddles of this thread, the same for every tile
  fast::load_tw2<NO>(wt, p, a.po.tw);
  // this thread's part of the Green's function: pz^2 - Re(k0^2 + i eps) for its 16 z
  float pz2[16];
#pragma unroll
  for (int m = 0; m < 16; ++m) {
    const float po = a.w.pze[p + P * m];
    pz2[m] = fmaf(po, po, -a.k02e.x);
  }
  const float di = -a.k02e.y;
  int i = 0;
  bool ok = true;
  for (; i < mine; ++i) {
    const int b = i % S;
    const int t = blockIdx.x + i * G;
    float2* const buf = buf0 + b * NO * TY;
    ok = wait_parity(&full[b], (uint32_t)((i / S) & 1), a.wait_clocks > 0 ? a.wait_clocks : kWaitClocks);
    if (__syncthreads_or(!ok)) {
      ok = false;
      break;
    }
    // tile i + S - 1 goes into the buffer of tile i - 1 (no thread reads it
    // any more), once the store of tile i - 1 has read it: issued half way
    // through tile i, so that the load overlaps the inverse transform too
    auto refill = [&]() {
      const int nxt = i + S - 1;
      if (tid == 0 && nxt < mine) {
        bulk_wait_read_0();
        issue(blockIdx.x + nxt * G, nxt % S);
      }
    };
    int rhs, mid, yt;
    coords(t, rhs, mid, yt);
    const bool live = !load_done(st + rhs);
    if (!live) refill();
    if (live) {
      float2 v[16];
#pragma unroll
      for (int q = 0; q < 16; ++q) v[q] = buf[(p + P * q) * TY + yl];
      // the exchanges go through the tile's own buffer (each starts with a
      // block barrier, so every input has been read before it is overwritten)
      fast::RowLine L{buf + yl, TY};
      fast::line_fft_tw2<NO, false>(v, L, p, wt, fast::SyncBlock{});
      // f_g0_scalar with the 1/N of ifftn: E ./ (px^2 + py^2 + (pz^2 - k02e))
      const float py = a.w.pye[yt * TY + yl];
      const float pxm = a.w.pxe[mid];
      const float base2 = fmaf(pxm, pxm, py * py);
#pragma unroll
      for (int m = 0; m < 16; ++m) {
        const float dr = base2 + pz2[m];
        if (a.pstd) {
          v[m] = make_float2(-dr * a.norm * v[m].x, -dr * a.norm * v[m].y);  // PSTD Laplacian (k02e = 0)
        } else {
          const float inv = __fdividef(a.norm, fmaf(dr, dr, di * di));
          v[m] = cmul(v[m], make_float2(dr * inv, -di * inv));
        }
      }
      refill();
      fast::line_fft_tw2<NO, true>(v, L, p, wt, fast::SyncBlock{});
      if (a.pstd)
#pragma unroll
        for (int m = 0; m < 16; ++m) v[m].y = -v[m].y;
      // thread (p, yl) wrote back exactly the elements it read last
#pragma unroll
      for (int m = 0; m < 16; ++m) buf[(p + P * m) * TY + yl] = v[m];
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");  // visible to the TMA store
    }
    __syncthreads();
    if (tid == 0 && live) {
      store_3d(&tmap, 2 * TY * yt, mid, rhs * g.nz, fast::smem_addr(buf));
      bulk_commit();
    }
  }
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
    // drain the loads still in flight: tiles i .. min(i + S - 2, mine - 1); a
    // load that never arrives is abandoned after the same bound
    for (int j = i; j < mine && j < i + S - 1; ++j) (void)wait_parity(&full[j % S], (uint32_t)((j / S) & 1));
  }
  if (tid == 0) bulk_wait_all();
}


// The x transforms of the split fused step (ws_fast.cuh, kc_col_step): the
// same persistent pipeline as kt_pencil, along x instead of z and with one
// transform (forward, or inverse unnormalised) and no Green's function.  A
// tile is TY consecutive y of one x line: the box {2 TY floats, NO, 1} of the
// map {2 Ny floats, Nx, Nz Nc nrhs} over T, at (2 TY yt, 0, rhs Nz Nc + zc).
// Thread (p, yl) holds x = p + P r of row yl and transforms it with the
// plane kernels' line_fft and x twiddles, so the result is theirs bit for
// bit.  The map covers this GPU's T only; no multicast.
template <int NO, int TY, int S, bool INV>
__global__ void __launch_bounds__(PencilTile<NO, TY, S>::kThreads, PencilTile<NO, TY, S>::kMinBlocks)
    kt_xpencil(const __grid_constant__ CUtensorMap tmap, Geom g, const float2* __restrict__ twx,
               const DevState* __restrict__ st, int ntiles, long long wait_clocks, int* __restrict__ err) {
  pdl_begin();
  using PT = PencilTile<NO, TY, S>;
  constexpr int P = PT::P;
  extern __shared__ uint8_t smem_raw[];
  float2* const buf0 = reinterpret_cast<float2*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
  __shared__ __align__(8) uint64_t full[S];
  const int tid = threadIdx.x;
  const int yl = tid % TY, p = tid / TY;
  const int nyt = g.ny / TY;
  const int nzc = g.nz * g.nc;
  const int per_rhs = nyt * nzc;
  if (tid == 0) {
#pragma unroll
    for (int b = 0; b < S; ++b) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(fast::smem_addr(&full[b])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto coords = [&](int t, int& rhs, int& zc, int& yt) {
    rhs = t / per_rhs;
    const int r = t - rhs * per_rhs;
    zc = r / nyt;
    yt = r - zc * nyt;
  };
  auto issue = [&](int t, int b) {
    int rhs, zc, yt;
    coords(t, rhs, zc, yt);
    expect_bytes(&full[b], PT::kTileBytes);
    load_3d(fast::smem_addr(buf0 + b * NO * TY), &tmap, 2 * TY * yt, 0, rhs * nzc + zc, fast::smem_addr(&full[b]));
  };
  const int G = gridDim.x;
  const int mine = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / G + 1 : 0;
  if (tid == 0)
    for (int i = 0; i < S - 1 && i < mine; ++i) issue(blockIdx.x + i * G, i);
  // the second stage's twiddles of this thread, the same for every tile
  float2 wt[16];
  fast::load_tw2<NO>(wt, p, twx);
  const long long limit = wait_clocks > 0 ? wait_clocks : kWaitClocks;
  int i = 0;
  bool ok = true;
  for (; i < mine; ++i) {
    const int b = i % S;
    const int t = blockIdx.x + i * G;
    float2* const buf = buf0 + b * NO * TY;
    ok = wait_parity(&full[b], (uint32_t)((i / S) & 1), limit);
    if (__syncthreads_or(!ok)) {
      ok = false;
      break;
    }
    auto refill = [&]() {
      const int nxt = i + S - 1;
      if (tid == 0 && nxt < mine) {
        bulk_wait_read_0();
        issue(blockIdx.x + nxt * G, nxt % S);
      }
    };
    int rhs, zc, yt;
    coords(t, rhs, zc, yt);
    const bool live = !load_done(st + rhs);
    float2 v[16];
    if (live) {
#pragma unroll
      for (int q = 0; q < 16; ++q) v[q] = buf[(p + P * q) * TY + yl];
    }
    // tile i + S - 1 goes into the buffer of tile i - 1 once its store has read it
    refill();
    if (live) {
      fast::line_fft_tw2<NO, INV>(v, fast::RowLine{buf + yl, TY}, p, wt, fast::SyncBlock{});
#pragma unroll
      for (int m = 0; m < 16; ++m) buf[(p + P * m) * TY + yl] = v[m];
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0 && live) {
      store_3d(&tmap, 2 * TY * yt, 0, rhs * nzc + zc, fast::smem_addr(buf));
      bulk_commit();
    }
  }
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
    for (int j = i; j < mine && j < i + S - 1; ++j) (void)wait_parity(&full[j % S], (uint32_t)((j / S) & 1));
  }
  if (tid == 0) bulk_wait_all();
}

// kt_xpencil for the mixed-radix lines (ws_mixed.cuh): TY y of one x line
// of N = PL::N points per tile, PL::E elements per thread.
template <class PL, int TY, int S>
struct MixedXTile {
  static constexpr int NO = PL::N, P = PL::P, E = PL::E;
  static_assert(NO <= 256, "a TMA box dimension holds at most 256 elements");
  static_assert(2 * TY * 4 % 16 == 0 && 2 * TY <= 256, "inner box extent");
  static constexpr int kThreads = TY * P;
  static constexpr unsigned kTileBytes = NO * TY * sizeof(float2);
  static constexpr size_t smem = S * (size_t)kTileBytes + 128;
};

template <class PL, int TY, int S, bool INV>
__global__ void __launch_bounds__(MixedXTile<PL, TY, S>::kThreads, 2)
    kt_xpencil_m(const __grid_constant__ CUtensorMap tmap, Geom g, const float2* __restrict__ twx,
                 const DevState* __restrict__ st, int ntiles, long long wait_clocks, int* __restrict__ err) {
  pdl_begin();
  using PT = MixedXTile<PL, TY, S>;
  constexpr int NO = PT::NO, P = PT::P, E = PT::E;
  extern __shared__ uint8_t smem_raw[];
  float2* const buf0 = reinterpret_cast<float2*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
  __shared__ __align__(8) uint64_t full[S];
  const int tid = threadIdx.x;
  const int yl = tid % TY, p = tid / TY;
  const int nyt = g.ny / TY;
  const int nzc = g.nz * g.nc;
  const int per_rhs = nyt * nzc;
  if (tid == 0) {
#pragma unroll
    for (int b = 0; b < S; ++b) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(fast::smem_addr(&full[b])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto coords = [&](int t, int& rhs, int& zc, int& yt) {
    rhs = t / per_rhs;
    const int r = t - rhs * per_rhs;
    zc = r / nyt;
    yt = r - zc * nyt;
  };
  auto issue = [&](int t, int b) {
    int rhs, zc, yt;
    coords(t, rhs, zc, yt);
    expect_bytes(&full[b], PT::kTileBytes);
    load_3d(fast::smem_addr(buf0 + b * NO * TY), &tmap, 2 * TY * yt, 0, rhs * nzc + zc, fast::smem_addr(&full[b]));
  };
  const int G = gridDim.x;
  const int mine = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / G + 1 : 0;
  if (tid == 0)
    for (int i = 0; i < S - 1 && i < mine; ++i) issue(blockIdx.x + i * G, i);
  const long long limit = wait_clocks > 0 ? wait_clocks : kWaitClocks;
  int i = 0;
  bool ok = true;
  for (; i < mine; ++i) {
    const int b = i % S;
    const int t = blockIdx.x + i * G;
    float2* const buf = buf0 + b * NO * TY;
    ok = wait_parity(&full[b], (uint32_t)((i / S) & 1), limit);
    if (__syncthreads_or(!ok)) {
      ok = false;
      break;
    }
    auto refill = [&]() {
      const int nxt = i + S - 1;
      if (tid == 0 && nxt < mine) {
        bulk_wait_read_0();
        issue(blockIdx.x + nxt * G, nxt % S);
      }
    };
    int rhs, zc, yt;
    coords(t, rhs, zc, yt);
    const bool live = !load_done(st + rhs);
    float2 v[E];
    if (live) {
#pragma unroll
      for (int q = 0; q < E; ++q) v[q] = buf[(p + P * q) * TY + yl];
    }
    refill();
    if (live) {
      mixed::line_fft<PL, INV>(v, fast::RowLine{buf + yl, TY}, p, twx, fast::SyncBlock{});
#pragma unroll
      for (int m = 0; m < E; ++m) buf[(p + P * m) * TY + yl] = v[m];
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0 && live) {
      store_3d(&tmap, 2 * TY * yt, 0, rhs * nzc + zc, fast::smem_addr(buf));
      bulk_commit();
    }
  }
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
    for (int j = i; j < mine && j < i + S - 1; ++j) (void)wait_parity(&full[j % S], (uint32_t)((j / S) & 1));
  }
  if (tid == 0) bulk_wait_all();
}

// The vector form (WaveSimVector, 3 components): a tile is the three
// component boxes of the same (x, y tile), at z offsets c Nz of the map
// {2 Ny floats, Nx, Nz Nc nrhs}; each line is transformed with the
// register-resident mixed-radix schedule (ws_mixed.cuh) one component at a
// time, the dyadic Green's function (f_g0_vector.m) applied at every k point
// of the three transformed boxes, the inverse transforms, and the three
// boxes stored back.  The rest is kt_pencil.
template <class PL, int TY, int S>
struct VecPencilTile {
  static constexpr int NO = PL::N, P = PL::P, E = PL::E;
  static_assert(NO <= 256, "a TMA box dimension holds at most 256 elements");
  static_assert(2 * TY * 4 % 16 == 0 && 2 * TY <= 256, "inner box extent");
  static constexpr int kThreads = TY * P;
  static constexpr unsigned kBoxBytes = NO * TY * sizeof(float2);
  static constexpr unsigned kTileBytes = 3 * kBoxBytes;
  static constexpr size_t smem = S * (size_t)kTileBytes + 128;
  // blocks per SM the tiles leave room for (228 KB, 1 KB reserved per block,
  // at most 4): the register bound of the kernel
  static constexpr int kFit = (int)(228 * 1024 / (smem + 3 * 1024));
  static constexpr int kMinBlocks = kFit >= 4 ? 4 : (kFit >= 1 ? kFit : 1);
};

template <class PL, int TY, int S>
__global__ void __launch_bounds__(VecPencilTile<PL, TY, S>::kThreads, VecPencilTile<PL, TY, S>::kMinBlocks)
    kt_pencil_vec(const __grid_constant__ CUtensorMap tmap, OuterArgs a, const DevState* __restrict__ st, int ntiles,
                  int* __restrict__ err) {
  pdl_begin();
  using PT = VecPencilTile<PL, TY, S>;
  constexpr int NO = PT::NO, P = PT::P, E = PT::E;
  extern __shared__ uint8_t smem_raw[];
  float2* const buf0 = reinterpret_cast<float2*>((reinterpret_cast<uintptr_t>(smem_raw) + 127) & ~(uintptr_t)127);
  __shared__ __align__(8) uint64_t full[S];
  const Geom& g = a.g;
  const int tid = threadIdx.x;
  const int yl = tid % TY, p = tid / TY;
  const int nyt = g.ny / TY;
  const int per_rhs = nyt * g.nx;
  if (tid == 0) {
#pragma unroll
    for (int b = 0; b < S; ++b) asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(fast::smem_addr(&full[b])));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  auto coords = [&](int t, int& rhs, int& mid, int& yt) {
    rhs = t / per_rhs;
    const int r = t - rhs * per_rhs;
    mid = r / nyt;
    yt = r - mid * nyt;
  };
  auto box = [&](int b, int c) { return buf0 + (b * 3 + c) * NO * TY; };
  auto issue = [&](int t, int b) {
    int rhs, mid, yt;
    coords(t, rhs, mid, yt);
    expect_bytes(&full[b], PT::kTileBytes);
#pragma unroll
    for (int c = 0; c < 3; ++c)
      load_3d(fast::smem_addr(box(b, c)), &tmap, 2 * TY * yt, mid, (rhs * 3 + c) * g.nz, fast::smem_addr(&full[b]));
  };
  const int G = gridDim.x;
  const int mine = blockIdx.x < ntiles ? (ntiles - 1 - blockIdx.x) / G + 1 : 0;
  if (tid == 0)
    for (int i = 0; i < S - 1 && i < mine; ++i) issue(blockIdx.x + i * G, i);
  const float kk = fmaf(a.k02e.x, a.k02e.x, a.k02e.y * a.k02e.y);
  const float di = -a.k02e.y;
  int i = 0;
  bool ok = true;
  for (; i < mine; ++i) {
    const int b = i % S;
    const int t = blockIdx.x + i * G;
    ok = wait_parity(&full[b], (uint32_t)((i / S) & 1), a.wait_clocks > 0 ? a.wait_clocks : kWaitClocks);
    if (__syncthreads_or(!ok)) {
      ok = false;
      break;
    }
    auto refill = [&]() {
      const int nxt = i + S - 1;
      if (tid == 0 && nxt < mine) {
        bulk_wait_read_0();
        issue(blockIdx.x + nxt * G, nxt % S);
      }
    };
    int rhs, mid, yt;
    coords(t, rhs, mid, yt);
    const bool live = !load_done(st + rhs);
    if (!live) refill();
    if (live) {
      // one component at a time: each line's spectrum goes back to its own
      // box (thread (p, yl) writes exactly the elements it read in the last
      // stage, so no other thread still needs them), which keeps a single
      // line in registers instead of three
#pragma unroll 1
      for (int c = 0; c < 3; ++c) {
        float2 v[E];
#pragma unroll
        for (int r = 0; r < E; ++r) v[r] = box(b, c)[(p + P * r) * TY + yl];
        mixed::line_fft<PL, false>(v, fast::RowLine{box(b, c) + yl, TY}, p, a.po.tw, fast::SyncBlock{});
#pragma unroll
        for (int m = 0; m < E; ++m) box(b, c)[(p + P * m) * TY + yl] = v[m];
      }
      // f_g0_vector with the 1/N of ifftn: div = (p . E) / k02e; E_i <- (E_i - p_i div) / (|p|^2 - k02e),
      // on this thread's own k points of the three boxes
      const float px = a.w.pxe[mid], py = a.w.pye[yt * TY + yl];
#pragma unroll 4
      for (int m = 0; m < E; ++m) {
        const int k = (p + P * m) * TY + yl;
        const float pz = a.w.pze[p + P * m];
        const float dr = fmaf(px, px, fmaf(py, py, pz * pz)) - a.k02e.x;
        const float inv = __fdividef(a.norm, fmaf(dr, dr, di * di));
        const float2 g0 = make_float2(dr * inv, -di * inv);
        const float2 ex = box(b, 0)[k], ey = box(b, 1)[k], ez = box(b, 2)[k];
        const float2 pe =
            make_float2(fmaf(px, ex.x, fmaf(py, ey.x, pz * ez.x)), fmaf(px, ex.y, fmaf(py, ey.y, pz * ez.y)));
        const float2 dv =
            make_float2((pe.x * a.k02e.x + pe.y * a.k02e.y) / kk, (pe.y * a.k02e.x - pe.x * a.k02e.y) / kk);
        box(b, 0)[k] = cmul(g0, make_float2(ex.x - px * dv.x, ex.y - px * dv.y));
        box(b, 1)[k] = cmul(g0, make_float2(ey.x - py * dv.x, ey.y - py * dv.y));
        box(b, 2)[k] = cmul(g0, make_float2(ez.x - pz * dv.x, ez.y - pz * dv.y));
      }
      refill();
#pragma unroll 1
      for (int c = 0; c < 3; ++c) {
        float2 v[E];
#pragma unroll
        for (int r = 0; r < E; ++r) v[r] = box(b, c)[(p + P * r) * TY + yl];
        mixed::line_fft<PL, true>(v, fast::RowLine{box(b, c) + yl, TY}, p, a.po.tw, fast::SyncBlock{});
#pragma unroll
        for (int m = 0; m < E; ++m) box(b, c)[(p + P * m) * TY + yl] = v[m];
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncthreads();
    if (tid == 0 && live) {
#pragma unroll
      for (int c = 0; c < 3; ++c) store_3d(&tmap, 2 * TY * yt, mid, (rhs * 3 + c) * g.nz, fast::smem_addr(box(b, c)));
      bulk_commit();
    }
  }
  if (!ok) {
    if (tid == 0) atomicExch(err, 1);
    for (int j = i; j < mine && j < i + S - 1; ++j) (void)wait_parity(&full[j % S], (uint32_t)((j / S) & 1));
  }
  if (tid == 0) bulk_wait_all();
}

}  // namespace tma
}  // namespace ws
