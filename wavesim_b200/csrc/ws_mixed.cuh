// Register-resident fused MBS kernels for line lengths that are not powers
// of two (and for the vector Green's function), e.g. the 192^3 x 3 grid of
// a WaveSimVector problem with a 16-pixel boundary.
//
// A line of N points is held by P = N / E threads with E elements each, and
// transformed by a Stockham schedule fixed at compile time: up to four
// radices R0 R1 R2 R3 = N, each dividing E (192 = 12 x 4 x 4 with E = 12;
// 160 = 10 x 4 x 4 with E = 20; 224 = 14 x 4 x 4 with E = 28).  Thread p
// enters with v[r] = x[p + P r] and leaves with v[m] = X[p + P m], as in the
// power-of-two kernels.  Each stage runs E / R butterflies j = p + P q per
// thread; stage 0 takes their inputs x[j + r N/R0] = v[q + (E/R0) r] from
// registers, a later stage reads the R inputs x[j + r N/R] from shared
// memory and multiplies them by W_{Ns R}^{(j mod Ns) r} (Ns = product of the
// earlier radices); every stage but the last writes output r of butterfly j
// to (j - j mod Ns) R + j mod Ns + r Ns.
//
//   km_plane_fwd<PL, C>  K1: (y, x) planes on a cluster of C blocks; y
//                        transforms of N / C columns per block, then each
//                        block pulls its N / C rows from the cluster
//                        (distributed shared memory) for the x transforms.
//   km_pencil<PL, TY, NC> K2: z pencils of NC components, scalar or dyadic
//                        Green's function (f_g0_scalar.m / f_g0_vector.m).
//   km_plane_inv<PL, C>  K3: the inverse of K1, then the epilogue of the
//                        power-of-two K3 (unwiggle, f_mix, E' += dE', ROI energy).
#pragma once
#include "ws_fast.cuh"

namespace ws {
namespace mixed {

constexpr int kThreads = 256;

// Column lines of the column passes (kmc_col_step, the 2-D kernels): element
// i of a line at i + (i >> SH), lines CS elements apart.  The shift and
// stride minimise the shared-memory wavefronts of the lines' exchanges
// (colpad_model.py: every stage's accesses, half-warp by half-warp, 8-byte
// banks): 224 points 2496 against 3968 with the planes' (i >> 4, N + N/16 + 1),
// 160: 1824 against 3520, 96: 1024 against 1792, 192: 1152 against 1344,
// 576: 3456 against 4032; the others keep the planes' layout.
template <int N>
struct ColPad {
  static constexpr int SH = 4, CS = N + N / 16 + 1;
};
template <> struct ColPad<96> { static constexpr int SH = 5, CS = 104; };
template <> struct ColPad<160> { static constexpr int SH = 5, CS = 168; };
template <> struct ColPad<192> { static constexpr int SH = 5, CS = 197; };
template <> struct ColPad<224> { static constexpr int SH = 5, CS = 232; };
template <> struct ColPad<576> { static constexpr int SH = 5, CS = 593; };

template <int N>
struct ColLineP {
  float2* base;
  static_assert(ColPad<N>::CS >= (N - 1) + ((N - 1) >> ColPad<N>::SH) + 1, "a line fits its stride");
  __device__ __forceinline__ float2& at(int i) const { return base[i + (i >> ColPad<N>::SH)]; }
};

// The epilogues issue their loads (gamma, dE', E') in NH groups of H = E / NH
// elements: halves up to 12 elements per thread, quarters beyond, so that
// fewer loads are in flight in registers at once.
template <int E>
constexpr int kEpilogueParts = E > 12 && E % 4 == 0 ? 4 : 2;

template <int N_, int E_, int R0, int R1, int R2 = 1, int R3 = 1>
struct Plan {
  static constexpr int N = N_, E = E_, P = N_ / E_;
  static constexpr int NST = R3 > 1 ? 4 : (R2 > 1 ? 3 : (R1 > 1 ? 2 : 1));
  __host__ __device__ static constexpr int radix(int s) {
    return s == 0 ? R0 : (s == 1 ? R1 : (s == 2 ? R2 : R3));
  }
  __host__ __device__ static constexpr int span(int s) {
    return s == 0 ? 1 : (s == 1 ? R0 : (s == 2 ? R0 * R1 : R0 * R1 * R2));
  }
  static_assert(R0 * R1 * R2 * R3 == N_ && N_ % E_ == 0, "the radices multiply to N, E divides N");
  static_assert(E_ % R0 == 0 && E_ % R1 == 0 && E_ % R2 == 0 && E_ % R3 == 0, "every radix divides E");
  static_assert(NST > 1 || R0 == E_, "a one-stage line is one butterfly per thread");
};

template <int R, bool INV, int E>
__device__ __forceinline__ void dft_at(float2 (&v)[E], int off) {
  float2 u[R];
#pragma unroll
  for (int r = 0; r < R; ++r) u[r] = v[off + r];
  Dft<R, INV>::run(u);
#pragma unroll
  for (int r = 0; r < R; ++r) v[off + r] = u[r];
}

template <class PL, bool INV, int S, class Line, class Sync>
__device__ __forceinline__ void stage(float2 (&v)[PL::E], const Line& L, int p, const float2* __restrict__ tw,
                                      Sync sync) {
  constexpr int E = PL::E, N = PL::N, P = PL::P;
  constexpr int R = PL::radix(S), Ns = PL::span(S), B = E / R, NR = N / R, TS = N / (Ns * R);
  if constexpr (S == 0 && B > 1) {
    // butterfly q takes v[q + B r]; gather it to v[q R + r]
    float2 t[E];
#pragma unroll
    for (int m = 0; m < E; ++m) t[m] = v[m];
#pragma unroll
    for (int q = 0; q < B; ++q)
#pragma unroll
      for (int r = 0; r < R; ++r) v[q * R + r] = t[q + B * r];
  }
  if constexpr (S > 0) {
#pragma unroll
    for (int q = 0; q < B; ++q) {
      const int j = p + P * q;
#pragma unroll
      for (int r = 0; r < R; ++r) v[q * R + r] = L.at(j + r * NR);
      const int jm = j % Ns;
#pragma unroll
      for (int r = 1; r < R; ++r) {
        float2 w = __ldg(&tw[jm * r * TS]);
        if (INV) w.y = -w.y;
        v[q * R + r] = cmul(v[q * R + r], w);
      }
    }
  }
#pragma unroll
  for (int q = 0; q < B; ++q) dft_at<R, INV>(v, q * R);
  if constexpr (S < PL::NST - 1) {
    sync();
#pragma unroll
    for (int q = 0; q < B; ++q) {
      const int j = p + P * q;
      const int jm = j % Ns;
      const int base = (j - jm) * R + jm;
#pragma unroll
      for (int r = 0; r < R; ++r) L.at(base + r * Ns) = v[q * R + r];
    }
    sync();
  } else if constexpr (B > 1) {
    float2 t[E];
#pragma unroll
    for (int q = 0; q < B; ++q)
#pragma unroll
      for (int r = 0; r < R; ++r) t[q + B * r] = v[q * R + r];
#pragma unroll
    for (int m = 0; m < E; ++m) v[m] = t[m];
  }
}

// In: v[r] = x[p + P r].  Out: v[m] = X[p + P m] (unnormalised; INV: sign +1).
template <class PL, bool INV, class Line, class Sync>
__device__ __forceinline__ void line_fft(float2 (&v)[PL::E], const Line& L, int p, const float2* __restrict__ tw,
                                         Sync sync) {
  stage<PL, INV, 0>(v, L, p, tw, sync);
  if constexpr (PL::NST > 1) stage<PL, INV, 1>(v, L, p, tw, sync);
  if constexpr (PL::NST > 2) stage<PL, INV, 2>(v, L, p, tw, sync);
  if constexpr (PL::NST > 3) stage<PL, INV, 3>(v, L, p, tw, sync);
}

// Shared-memory tiles of the plane kernels (one buffer, used twice):
//   column tile: column cl of the block at cl * CS, element y at y + y / 16
//   row tile:    element (row kyl, x) at x * RS + kyl
template <class PL, int C>
struct MGeom {
  static constexpr int N = PL::N, P = PL::P;
  static constexpr int M = N / C;   // columns per block
  static constexpr int LR = N / C;  // rows per block
  static constexpr int CS = N + N / 16 + 1;
  static constexpr int RS = LR + 1;
  static constexpr int LPR = kThreads / P;  // lines per round
  static constexpr int PER = LR * N / kThreads;  // elements each thread carries across the cluster
  static constexpr size_t smem = sizeof(float2) * (size_t)(M * CS > N * RS ? M * CS : N * RS);
  static_assert(N % C == 0 && M % LPR == 0 && (LR * N) % kThreads == 0, "plane split");
  static_assert(kThreads % P == 0 && (P <= 32 ? 32 % P == 0 : true), "threads per line");
};

template <int P>
struct LineSync {
  using type = fast::SyncBlock;
};
template <>
struct LineSync<16> {
  using type = fast::SyncWarp;
};
template <>
struct LineSync<8> {
  using type = fast::SyncWarp;
};

// K1 --------------------------------------------------------------------------
template <class PL, int C>
__global__ void __launch_bounds__(kThreads, 3)
    km_plane_fwd(InnerArgs a, const float2* __restrict__ dE, const float2* __restrict__ src, float2 A,
                 float2* __restrict__ T, const DevState* __restrict__ st) {
  using G = MGeom<PL, C>;
  constexpr int N = PL::N, E = PL::E, P = PL::P, M = G::M, LR = G::LR, LPR = G::LPR;
  const int rhs = blockIdx.x / a.bpr, bid = blockIdx.x - rhs * a.bpr;
  st += rhs;
  if (load_done(st)) return;  // the same for every block of a cluster (one right-hand side)
  dE += rhs * a.fstride;
  if (src) src += rhs * a.fstride;
  T += rhs * a.fstride;
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x;
  const Geom& g = a.g;
  const int rank = bid % C, plane = bid / C, z = plane % g.nz;
  const int x0 = rank * M;
  const long long colbase = (long long)plane * N + x0;
  const float2 gzz = a.w.gz[z];
  // y transforms of the block's columns, straight from global memory
  for (int c0 = 0; c0 < M; c0 += LPR) {
    const int cl = c0 + tid / P, p = tid % P;
    const long long col = colbase + cl;
    const float2 gxz = cmul(a.w.gx[x0 + cl], gzz);
    const float2* __restrict__ s = dE + col * N;
    const float2* __restrict__ sr = src ? src + col * N : nullptr;
    float2 v[E];
#pragma unroll
    for (int r = 0; r < E; ++r) {
      const int y = p + P * r;
      float2 e = s[y];
      if (sr) e = cadd(e, cmul(A, sr[y]));
      v[r] = cmul(cmul(e, gxz), a.w.gy[y]);
    }
    fast::ColLine L{sm + cl * G::CS};
    line_fft<PL, false>(v, L, p, a.py.tw, typename LineSync<P>::type{});
#pragma unroll
    for (int m = 0; m < E; ++m) L.at(p + P * m) = v[m];
  }
  cg::cluster_group cluster = cg::this_cluster();
  cluster.sync();
  // rows [rank LR, rank LR + LR) of all N columns, from the blocks holding them
  float2 hold[G::PER];
#pragma unroll
  for (int i = 0; i < G::PER; ++i) {
    const int e = tid + kThreads * i;
    const int kyl = e % LR, x = e / LR;
    const int ky = rank * LR + kyl;
    const float2* rs = cluster.map_shared_rank(sm, x / M);
    hold[i] = rs[(x % M) * G::CS + ky + (ky >> 4)];
  }
  cluster.sync();
#pragma unroll
  for (int i = 0; i < G::PER; ++i) {
    const int e = tid + kThreads * i;
    sm[(e / LR) * G::RS + e % LR] = hold[i];
  }
  __syncthreads();
  constexpr int RPR = kThreads / P;
  for (int r0 = 0; r0 < LR; r0 += RPR) {
    const int rl = r0 + tid % RPR, p = tid / RPR;
    fast::RowLine L{sm + rl, G::RS};
    float2 v[E];
#pragma unroll
    for (int r = 0; r < E; ++r) v[r] = L.at(p + P * r);
    line_fft<PL, false>(v, L, p, a.twx, fast::SyncBlock{});
    float2* __restrict__ d = T + (long long)plane * N * N + rank * LR + rl;
#pragma unroll
    for (int m = 0; m < E; ++m) d[(long long)(p + P * m) * N] = v[m];
  }
}

// K2 --------------------------------------------------------------------------
// D3: z pencils of a 3-D grid; otherwise x pencils of a 2-D grid (a
// compile-time choice: the run-time branch cost the 3-D pencils registers
// and 25-35% of their speed)
template <class PL, int TY, int NC, bool D3 = true>
__global__ void __launch_bounds__(TY* PL::P, NC == 1 ? 2 : 1)
    km_pencil(OuterArgs a, float2* __restrict__ T, const DevState* __restrict__ st) {
  pdl_begin();
  constexpr int E = PL::E, P = PL::P, TYS = TY + 1;
  const int rhs = blockIdx.x / a.bpr, bid = blockIdx.x - rhs * a.bpr;
  st += rhs;
  if (load_done(st)) return;
  T += rhs * a.fstride;
  extern __shared__ float2 sm[];
  const Geom& g = a.g;
  const int tid = threadIdx.x;
  const int yl = tid % TY, p = tid / TY;
  const int nyt = g.ny / TY;
  // 3-D: z pencils of column x = mid; 2-D: x pencils (mid = 0)
  const int yt = bid % nyt, mid = D3 ? bid / nyt : 0;
  const int ky = yt * TY + yl;
  const long long ps = D3 ? (long long)g.ny * g.nx : (long long)g.ny;
  float2* __restrict__ base = T + ky + (long long)g.ny * mid;
  float2 v[NC][E];
#pragma unroll
  for (int c = 0; c < NC; ++c)
#pragma unroll
    for (int r = 0; r < E; ++r) v[c][r] = base[ps * (p + P * r) + g.npts * c];
  fast::RowLine L{sm + yl, TYS};
#pragma unroll
  for (int c = 0; c < NC; ++c) line_fft<PL, false>(v[c], L, p, a.po.tw, fast::SyncBlock{});
  const float pxm = a.w.pxe[mid], py = a.w.pye[ky], pz0 = a.w.pze[0];
  const float di = -a.k02e.y;
#pragma unroll
  for (int m = 0; m < E; ++m) {
    // the pencil's own coordinate: z in 3-D, x in 2-D
    const float px = D3 ? pxm : a.w.pxe[p + P * m];
    const float pz = D3 ? a.w.pze[p + P * m] : pz0;
    const float dr = fmaf(px, px, fmaf(py, py, pz * pz)) - a.k02e.x;
    const float inv = __fdividef(a.norm, fmaf(dr, dr, di * di));
    const float2 g0 = make_float2(dr * inv, -di * inv);
    if constexpr (NC == 1) {
      // f_g0_scalar with the 1/N of ifftn: E ./ (px^2 + py^2 + (pz^2 - k02e)),
      // or the PSTD Laplacian (k02e = 0)
      v[0][m] = a.pstd ? make_float2(-dr * a.norm * v[0][m].x, -dr * a.norm * v[0][m].y) : cmul(v[0][m], g0);
    } else {
      // f_g0_vector: div = (p . E) / k02e; E_i <- (E_i - p_i div) / (|p|^2 - k02e)
      const float2 ex = v[0][m], ey = v[1][m], ez = v[2][m];
      const float2 pe =
          make_float2(fmaf(px, ex.x, fmaf(py, ey.x, pz * ez.x)), fmaf(px, ex.y, fmaf(py, ey.y, pz * ez.y)));
      const float kk = fmaf(a.k02e.x, a.k02e.x, a.k02e.y * a.k02e.y);
      const float2 dv =
          make_float2((pe.x * a.k02e.x + pe.y * a.k02e.y) / kk, (pe.y * a.k02e.x - pe.x * a.k02e.y) / kk);
      v[0][m] = cmul(g0, make_float2(ex.x - px * dv.x, ex.y - px * dv.y));
      v[1][m] = cmul(g0, make_float2(ey.x - py * dv.x, ey.y - py * dv.y));
      v[2][m] = cmul(g0, make_float2(ez.x - pz * dv.x, ez.y - pz * dv.y));
    }
  }
#pragma unroll
  for (int c = 0; c < NC; ++c) line_fft<PL, true>(v[c], L, p, a.po.tw, fast::SyncBlock{});
  if (NC == 1 && a.pstd)
#pragma unroll
    for (int m = 0; m < E; ++m) v[0][m].y = -v[0][m].y;
#pragma unroll
  for (int c = 0; c < NC; ++c)
#pragma unroll
    for (int m = 0; m < E; ++m) base[ps * (p + P * m) + g.npts * c] = v[c][m];
}

// K3 --------------------------------------------------------------------------
template <class PL, int C>
__global__ void __launch_bounds__(kThreads, 2)
    km_plane_inv(InnerArgs a, const float2* __restrict__ T, float2* __restrict__ dE, float2* __restrict__ E,
                 const float2* __restrict__ gamma, const DevState* __restrict__ st, double* __restrict__ partials) {
  using G = MGeom<PL, C>;
  constexpr int N = PL::N, EL = PL::E, P = PL::P, M = G::M, LR = G::LR, LPR = G::LPR;
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
  const int rank = bid % C, plane = bid / C, z = plane % g.nz, comp = plane / g.nz;
  const int x0 = rank * M;
  const long long colbase = (long long)plane * N + x0;
  // inverse x transforms of the block's rows, straight from global memory
  constexpr int RPR = kThreads / P;
  for (int r0 = 0; r0 < LR; r0 += RPR) {
    const int rl = r0 + tid % RPR, p = tid / RPR;
    const float2* __restrict__ s = T + (long long)plane * N * N + rank * LR + rl;
    float2 v[EL];
#pragma unroll
    for (int r = 0; r < EL; ++r) v[r] = s[(long long)(p + P * r) * N];
    fast::RowLine L{sm + rl, G::RS};
    line_fft<PL, true>(v, L, p, a.twx, fast::SyncBlock{});
#pragma unroll
    for (int m = 0; m < EL; ++m) L.at(p + P * m) = v[m];
  }
  cg::cluster_group cluster = cg::this_cluster();
  cluster.sync();
  // columns [x0, x0 + M) of all N rows, from the blocks holding them
  float2 hold[G::PER];
#pragma unroll
  for (int i = 0; i < G::PER; ++i) {
    const int e = tid + kThreads * i;
    const int ky = e % N, c = e / N;
    const float2* rs = cluster.map_shared_rank(sm, ky / LR);
    hold[i] = rs[(x0 + c) * G::RS + ky % LR];
  }
  cluster.sync();
#pragma unroll
  for (int i = 0; i < G::PER; ++i) {
    const int e = tid + kThreads * i;
    const int ky = e % N, c = e / N;
    sm[c * G::CS + ky + (ky >> 4)] = hold[i];
  }
  __syncthreads();
  const float2 gzz = a.w.gz[z];
  float esum = 0.f;
  for (int c0 = 0; c0 < M; c0 += LPR) {
    const int cl = c0 + tid / P, p = tid % P;
    fast::ColLine L{sm + cl * G::CS};
    float2 v[EL];
#pragma unroll
    for (int r = 0; r < EL; ++r) v[r] = L.at(p + P * r);
    line_fft<PL, true>(v, L, p, a.py.tw, typename LineSync<P>::type{});
    const int x = x0 + cl;
    const long long col = colbase + cl;
    const float2 gxz = cmul(a.w.gx[x], gzz);
    const bool in_xzc =
        x >= g.r0[1] && x < g.r1[1] && z >= g.r0[2] && z < g.r1[2] && comp >= g.r0[3] && comp < g.r1[3];
    const long long gcol = col * N;
    const float2* __restrict__ gmc = gamma + (gcol - (long long)comp * g.npts);
    float2* __restrict__ dEc = dE + gcol;
    float2* __restrict__ Ec = E + gcol;
    // Eprop after the conjugate ramps (WaveSim.m:55), then f_mix (f_mix.m:3-4)
    // and E += dE; the loads of a half are issued together.
    constexpr int NH = kEpilogueParts<EL>, H = EL / NH;
#pragma unroll
    for (int h = 0; h < NH; ++h) {
      float2 gm[H], d0[H], e0[H];
#pragma unroll
      for (int i = 0; i < H; ++i) {
        const int y = p + P * (H * h + i);
        gm[i] = gmc[y];
        d0[i] = dEc[y];
        e0[i] = acc_now ? Ec[y] : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int i = 0; i < H; ++i) {
        const int m = H * h + i;
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


// K3 fused with K1 of the next iteration (as fast::kf_plane_fused): after
// K3's epilogue a column's new increment is in registers as K1 loads it, so
// the block adds the next source, applies the next wiggle's ramps, transforms
// the column along y in place, exchanges rows across the cluster (pull
// between two cluster barriers) and writes the x transform of its rows over
// the slab of T it read at the start.  Bit-identical to km_plane_inv followed
// by km_plane_fwd.
template <class PL, int C>
__global__ void __launch_bounds__(kThreads, 2)
    km_plane_fused(InnerArgs a, Wig w1, const float2* __restrict__ src1, float2 A, float2* __restrict__ T,
                   float2* __restrict__ dE, float2* __restrict__ E, const float2* __restrict__ gamma,
                   const DevState* __restrict__ st, double* __restrict__ partials) {
  using G = MGeom<PL, C>;
  constexpr int N = PL::N, EL = PL::E, P = PL::P, M = G::M, LR = G::LR, LPR = G::LPR;
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
  const int rank = bid % C, plane = bid / C, z = plane % g.nz, comp = plane / g.nz;
  const int x0 = rank * M;
  const long long colbase = (long long)plane * N + x0;
  float2* __restrict__ slab = T + (long long)plane * N * N + rank * LR;  // rows [rank LR, +LR) of the plane
  cg::cluster_group cluster = cg::this_cluster();
  // K3: inverse x transforms of the block's rows
  for (int r0 = 0; r0 < LR; r0 += RPR) {
    const int rl = r0 + tid % RPR, p = tid / RPR;
    float2 v[EL];
#pragma unroll
    for (int r = 0; r < EL; ++r) v[r] = slab[(long long)(p + P * r) * N + rl];
    fast::RowLine L{sm + rl, G::RS};
    line_fft<PL, true>(v, L, p, a.twx, fast::SyncBlock{});
#pragma unroll
    for (int m = 0; m < EL; ++m) L.at(p + P * m) = v[m];
  }
  {
    float2 hold[G::PER];
    cluster.sync();
#pragma unroll
    for (int i = 0; i < G::PER; ++i) {
      const int e = tid + kThreads * i;
      const int ky = e % N, c = e / N;
      const float2* rs = cluster.map_shared_rank(sm, ky / LR);
      hold[i] = rs[(x0 + c) * G::RS + ky % LR];
    }
    cluster.sync();
#pragma unroll
    for (int i = 0; i < G::PER; ++i) {
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
    const int cl = c0 + tid / P, p = tid % P;
    fast::ColLine L{sm + cl * G::CS};
    float2 v[EL];
#pragma unroll
    for (int r = 0; r < EL; ++r) v[r] = L.at(p + P * r);
    line_fft<PL, true>(v, L, p, a.py.tw, typename LineSync<P>::type{});
    const int x = x0 + cl;
    const long long gcol = (colbase + cl) * N;
    const float2 gxz = cmul(a.w.gx[x], gzz);
    const bool in_xzc =
        x >= g.r0[1] && x < g.r1[1] && z >= g.r0[2] && z < g.r1[2] && comp >= g.r0[3] && comp < g.r1[3];
    const float2* __restrict__ gmc = gamma + (gcol - (long long)comp * g.npts);
    float2* __restrict__ dEc = dE + gcol;
    float2* __restrict__ Ec = E + gcol;
    // K3's epilogue; v[m] becomes dE'_k(y = p + P m)
    constexpr int NH = kEpilogueParts<EL>, H = EL / NH;
#pragma unroll
    for (int h = 0; h < NH; ++h) {
      float2 gm[H], d0[H], e0[H];
#pragma unroll
      for (int i = 0; i < H; ++i) {
        const int y = p + P * (H * h + i);
        gm[i] = gmc[y];
        d0[i] = dEc[y];
        e0[i] = acc_now ? Ec[y] : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int i = 0; i < H; ++i) {
        const int m = H * h + i;
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
    for (int m = 0; m < EL; ++m) {
      const int y = p + P * m;
      float2 e = v[m];
      if (sr) e = cadd(e, cmul(A, sr[y]));
      v[m] = cmul(cmul(e, gxz1), w1.gy[y]);
    }
    line_fft<PL, false>(v, L, p, a.py.tw, typename LineSync<P>::type{});
#pragma unroll
    for (int m = 0; m < EL; ++m) L.at(p + P * m) = v[m];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) esum += __shfl_xor_sync(0xffffffffu, esum, o);
  if ((tid & 31) == 0) red[tid >> 5] = esum;
  // rows [rank LR, rank LR + LR) of all N transformed columns
  {
    float2 hold[G::PER];
    cluster.sync();
#pragma unroll
    for (int i = 0; i < G::PER; ++i) {
      const int e = tid + kThreads * i;
      const int kyl = e % LR, x = e / LR;
      const int ky = rank * LR + kyl;
      const float2* rs = cluster.map_shared_rank(sm, x / M);
      hold[i] = rs[(x % M) * G::CS + ky + (ky >> 4)];
    }
    cluster.sync();
#pragma unroll
    for (int i = 0; i < G::PER; ++i) {
      const int e = tid + kThreads * i;
      sm[(e / LR) * G::RS + e % LR] = hold[i];
    }
  }
  __syncthreads();
  if (tid < 32) {
    float v = tid < kThreads / 32 ? red[tid] : 0.f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (tid == 0) partials[bid] = (double)v;
  }
  // K1's x transforms, written over the slab K3 read
  for (int r0 = 0; r0 < LR; r0 += RPR) {
    const int rl = r0 + tid % RPR, p = tid / RPR;
    fast::RowLine L{sm + rl, G::RS};
    float2 v[EL];
#pragma unroll
    for (int r = 0; r < EL; ++r) v[r] = L.at(p + P * r);
    line_fft<PL, false>(v, L, p, a.twx, fast::SyncBlock{});
#pragma unroll
    for (int m = 0; m < EL; ++m) slab[(long long)(p + P * m) * N + rl] = v[m];
  }
}

// The fused step with K3's rows loaded by one tensor copy (TMA) into a dense
// tile instead of per-thread loads.
template <class PL, int C>
__global__ void __launch_bounds__(kThreads, 2)
    km_plane_fused_tma(const __grid_constant__ CUtensorMap tslab, InnerArgs a, Wig w1, const float2* __restrict__ src1, float2 A, float2* __restrict__ T,
                   float2* __restrict__ dE, float2* __restrict__ E, const float2* __restrict__ gamma,
                   const DevState* __restrict__ st, double* __restrict__ partials) {
  using G = MGeom<PL, C>;
  constexpr int N = PL::N, EL = PL::E, P = PL::P, M = G::M, LR = G::LR, LPR = G::LPR;
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
  const int rank = bid % C, plane = bid / C, z = plane % g.nz, comp = plane / g.nz;
  const int x0 = rank * M;
  const long long colbase = (long long)plane * N + x0;
  float2* __restrict__ slab = T + (long long)plane * N * N + rank * LR;  // rows [rank LR, +LR) of the plane
  cg::cluster_group cluster = cg::this_cluster();
  // K3's rows by one tensor copy: the box {2 LR floats, N columns} of the
  // 2-D view {2 Ny floats, Nx Nz Nc nrhs columns} of T, landing dense:
  // element (row kyl, x) at rt[x * LR + kyl]
  float2* const rt = reinterpret_cast<float2*>((reinterpret_cast<uintptr_t>(sm) + 127) & ~(uintptr_t)127);
  __shared__ __align__(8) uint64_t slab_bar;
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(fast::smem_addr(&slab_bar)));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (tid == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(fast::smem_addr(&slab_bar)),
                 "r"((uint32_t)(N * LR * sizeof(float2)))
                 : "memory");
    const int c0 = 2 * rank * LR;
    const int c1 = (int)((long long)rhs * (a.fstride / N) + (long long)plane * N);
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
            fast::smem_addr(rt)),
        "l"(&tslab), "r"(c0), "r"(c1), "r"(fast::smem_addr(&slab_bar))
        : "memory");
  }
  {
    const uint32_t ba = fast::smem_addr(&slab_bar);
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
  // K3: inverse x transforms of the block's rows, in place
  for (int r0 = 0; r0 < LR; r0 += RPR) {
    const int rl = r0 + tid % RPR, p = tid / RPR;
    float2 v[EL];
    fast::RowLine L{rt + rl, LR};
#pragma unroll
    for (int r = 0; r < EL; ++r) v[r] = L.at(p + P * r);
    line_fft<PL, true>(v, L, p, a.twx, fast::SyncBlock{});
#pragma unroll
    for (int m = 0; m < EL; ++m) L.at(p + P * m) = v[m];
  }
  {
    float2 hold[G::PER];
    cluster.sync();
#pragma unroll
    for (int i = 0; i < G::PER; ++i) {
      const int e = tid + kThreads * i;
      const int ky = e % N, c = e / N;
      const float2* rs = cluster.map_shared_rank(rt, ky / LR);
      hold[i] = rs[(x0 + c) * LR + ky % LR];
    }
    cluster.sync();
#pragma unroll
    for (int i = 0; i < G::PER; ++i) {
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
    const int cl = c0 + tid / P, p = tid % P;
    fast::ColLine L{sm + cl * G::CS};
    float2 v[EL];
#pragma unroll
    for (int r = 0; r < EL; ++r) v[r] = L.at(p + P * r);
    line_fft<PL, true>(v, L, p, a.py.tw, typename LineSync<P>::type{});
    const int x = x0 + cl;
    const long long gcol = (colbase + cl) * N;
    const float2 gxz = cmul(a.w.gx[x], gzz);
    const bool in_xzc =
        x >= g.r0[1] && x < g.r1[1] && z >= g.r0[2] && z < g.r1[2] && comp >= g.r0[3] && comp < g.r1[3];
    const float2* __restrict__ gmc = gamma + (gcol - (long long)comp * g.npts);
    float2* __restrict__ dEc = dE + gcol;
    float2* __restrict__ Ec = E + gcol;
    // K3's epilogue; v[m] becomes dE'_k(y = p + P m)
    constexpr int NH = kEpilogueParts<EL>, H = EL / NH;
#pragma unroll
    for (int h = 0; h < NH; ++h) {
      float2 gm[H], d0[H], e0[H];
#pragma unroll
      for (int i = 0; i < H; ++i) {
        const int y = p + P * (H * h + i);
        gm[i] = gmc[y];
        d0[i] = dEc[y];
        e0[i] = acc_now ? Ec[y] : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int i = 0; i < H; ++i) {
        const int m = H * h + i;
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
    for (int m = 0; m < EL; ++m) {
      const int y = p + P * m;
      float2 e = v[m];
      if (sr) e = cadd(e, cmul(A, sr[y]));
      v[m] = cmul(cmul(e, gxz1), w1.gy[y]);
    }
    line_fft<PL, false>(v, L, p, a.py.tw, typename LineSync<P>::type{});
#pragma unroll
    for (int m = 0; m < EL; ++m) L.at(p + P * m) = v[m];
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) esum += __shfl_xor_sync(0xffffffffu, esum, o);
  if ((tid & 31) == 0) red[tid >> 5] = esum;
  // rows [rank LR, rank LR + LR) of all N transformed columns
  {
    float2 hold[G::PER];
    cluster.sync();
#pragma unroll
    for (int i = 0; i < G::PER; ++i) {
      const int e = tid + kThreads * i;
      const int kyl = e % LR, x = e / LR;
      const int ky = rank * LR + kyl;
      const float2* rs = cluster.map_shared_rank(sm, x / M);
      hold[i] = rs[(x % M) * G::CS + ky + (ky >> 4)];
    }
    cluster.sync();
#pragma unroll
    for (int i = 0; i < G::PER; ++i) {
      const int e = tid + kThreads * i;
      sm[(e / LR) * G::RS + e % LR] = hold[i];
    }
  }
  __syncthreads();
  if (tid < 32) {
    float v = tid < kThreads / 32 ? red[tid] : 0.f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (tid == 0) partials[bid] = (double)v;
  }
  // K1's x transforms, written over the slab K3 read
  for (int r0 = 0; r0 < LR; r0 += RPR) {
    const int rl = r0 + tid % RPR, p = tid / RPR;
    fast::RowLine L{sm + rl, G::RS};
    float2 v[EL];
#pragma unroll
    for (int r = 0; r < EL; ++r) v[r] = L.at(p + P * r);
    line_fft<PL, false>(v, L, p, a.twx, fast::SyncBlock{});
#pragma unroll
    for (int m = 0; m < EL; ++m) slab[(long long)(p + P * m) * N + rl] = v[m];
  }
}

// The column pass of the split fused step (see fast::kc_col_step) for the
// mixed-radix planes: the columns of block (plane, rank) of km_plane_fused,
// the same arithmetic in the same order and the same energy partial, with
// the y ramps of both wiggles read from shared memory (dynamic: LPR column
// lines, then the 2 N ramps; smem_col_step bytes).
template <class PL, int C>
constexpr size_t smem_col_step() {
  return sizeof(float2) * ((size_t)MGeom<PL, C>::LPR * ColPad<PL::N>::CS + 2 * PL::N);
}

template <class PL, int C>
__global__ void __launch_bounds__(kThreads, 2)
    kmc_col_step(InnerArgs a, Wig w1, const float2* __restrict__ src1, float2 A, float2* __restrict__ T,
                 float2* __restrict__ dE, float2* __restrict__ E, const float2* __restrict__ gamma,
                 const DevState* __restrict__ st, double* __restrict__ partials) {
  pdl_begin();
  using G = MGeom<PL, C>;
  constexpr int N = PL::N, EL = PL::E, P = PL::P, M = G::M, LPR = G::LPR;
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
  extern __shared__ float2 smc[];
  float2* const sm = smc;
  float2* const sgy = smc + LPR * ColPad<N>::CS;
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
    fast::prefetch_l2(gamma + (off - (long long)comp * g.npts), bytes);
    fast::prefetch_l2(dE + off, bytes);
    if (acc_now) fast::prefetch_l2(E + off, bytes);
    if (src1) fast::prefetch_l2(src1 + off, bytes);
  }
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
    const long long gcol = (colbase + cc) * N;
    float2* __restrict__ Tc = T + gcol;
    ColLineP<N> L{sm + cl * ColPad<N>::CS};
    float2 v[EL];
#pragma unroll
    for (int r = 0; r < EL; ++r) v[r] = Tc[p + P * r];
    line_fft<PL, true>(v, L, p, a.py.tw, typename LineSync<P>::type{});
    const float2 gxz = cmul(a.w.gx[x], gzz);
    const bool in_xzc =
        x >= g.r0[1] && x < g.r1[1] && z >= g.r0[2] && z < g.r1[2] && comp >= g.r0[3] && comp < g.r1[3];
    const float2* __restrict__ gmc = gamma + (gcol - (long long)comp * g.npts);
    float2* __restrict__ dEc = dE + gcol;
    float2* __restrict__ Ec = E + gcol;
    constexpr int NH = kEpilogueParts<EL>, H = EL / NH;
#pragma unroll
    for (int h = 0; h < NH; ++h) {
      float2 gm[H], d0[H], e0[H];
#pragma unroll
      for (int i = 0; i < H; ++i) {
        const int y = p + P * (H * h + i);
        gm[i] = gmc[y];
        d0[i] = dEc[y];
        e0[i] = acc_now ? Ec[y] : make_float2(0.f, 0.f);
      }
#pragma unroll
      for (int i = 0; i < H; ++i) {
        const int m = H * h + i;
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
    for (int m = 0; m < EL; ++m) {
      const int y = p + P * m;
      float2 e = v[m];
      if (sr) e = cadd(e, cmul(A, sr[y]));
      v[m] = cmul(cmul(e, gxz1), sgy[N + y]);
    }
    line_fft<PL, false>(v, L, p, a.py.tw, typename LineSync<P>::type{});
#pragma unroll
    for (int m = 0; m < EL; ++m) Tc[p + P * m] = v[m];
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

// 2-D grids on the mixed-radix lines: the y transforms of whole columns, as
// the power-of-two kf_plane_fwd / kf_plane_inv / kc_col_step2d do them for
// 2-D (K2 transforms along x).  Block bid covers the columns bid M ... bid M
// + M - 1 (M = a.ncols = LPR, column col = x + Nx c) in one round of lines;
// idle lanes of a partial last block transform a scratch column.
//   kmc_col_fwd2d<PL>   K1: source share, ramps, forward y transform
//   kmc_col_inv2d<PL>   K3: inverse y transform, unwiggle, f_mix, E' += dE',
//                       ROI energy
//   kmc_col_step2d<PL>  K3 of an iteration and K1 of the next in one pass
//                       (the ramps of both wiggles in shared memory), the
//                       same arithmetic in the same order, so its fields
//                       equal the separate kernels' bit for bit
template <class PL>
struct MGeom2d {
  static constexpr int N = PL::N, P = PL::P;
  static constexpr int CS = ColPad<N>::CS;
  static constexpr int LPR = kThreads / P;
  static_assert(kThreads % P == 0 && (P <= 32 ? 32 % P == 0 : true), "threads per line");
};

// dynamic shared memory of kmc_col_step2d: LPR + 1 columns and the two y ramps
template <class PL>
constexpr size_t smem_col_step2d() {
  return sizeof(float2) * ((size_t)(MGeom2d<PL>::LPR + 1) * MGeom2d<PL>::CS + 2 * PL::N);
}

enum { kCol2dFwd = 0, kCol2dInv = 1, kCol2dStep = 2 };

template <class PL, int MODE>
__device__ __forceinline__ void col2d(const InnerArgs& a, const Wig& w1, const float2* __restrict__ din,
                                      const float2* __restrict__ src, float2 A, float2* __restrict__ T,
                                      float2* __restrict__ dE, float2* __restrict__ E,
                                      const float2* __restrict__ gamma, const DevState* __restrict__ st,
                                      double* __restrict__ partials) {
  using G = MGeom2d<PL>;
  constexpr int N = PL::N, EL = PL::E, P = PL::P, LPR = G::LPR;
  using Sync = typename LineSync<P>::type;
  const int rhs = blockIdx.x / a.bpr, bid = blockIdx.x - rhs * a.bpr;
  st += rhs;
  if (load_done(st)) return;
  T += rhs * a.fstride;
  if (src) src += rhs * a.fstride;
  bool acc_now = false;
  if constexpr (MODE == kCol2dFwd) {
    din += rhs * a.fstride;
  } else {
    acc_now = !a.acc2 || (__ldcg(&st->it) & 1) == 0;
    dE += rhs * a.fstride;
    E += rhs * a.fstride;
    partials += (long long)rhs * a.bpr;
    gamma += rhs * a.gstride;  // a batch of media: each right-hand side has its own gamma
  }
  extern __shared__ float2 smx[];
  float2* const sgy = smx + (LPR + 1) * G::CS;  // kCol2dStep only
  __shared__ float red[kThreads / 32];
  const int tid = threadIdx.x;
  if constexpr (MODE == kCol2dStep) {
    for (int i = tid; i < N; i += kThreads) {
      sgy[i] = a.w.gy[i];
      sgy[N + i] = w1.gy[i];
    }
    __syncthreads();
  }
  const Geom& g = a.g;
  const int nx = g.nx;
  const int M = a.ncols;
  const long long colbase = (long long)bid * M;
  const int ncol = (int)min((long long)M, (long long)nx * g.nc - colbase);
  const float2 gzz = a.w.gz[0];
  float esum = 0.f;
  for (int c0 = 0; c0 < ncol; c0 += LPR) {
    const int cl = tid / P, cc = c0 + cl, p = tid % P;
    const bool live = cc < ncol;
    const long long col = colbase + cc;
    const long long gcol = col * N;
    ColLineP<N> L{smx + (live ? cl : LPR) * G::CS};
    float2 v[EL];
    if constexpr (MODE == kCol2dFwd) {
      if (live) {
        const int x = (int)(col % nx);
        const float2 gxz = cmul(a.w.gx[x], gzz);
#pragma unroll
        for (int r = 0; r < EL; ++r) {
          const int y = p + P * r;
          float2 e = din[gcol + y];
          if (src) e = cadd(e, cmul(A, src[gcol + y]));
          v[r] = cmul(cmul(e, gxz), a.w.gy[y]);
        }
      } else {
#pragma unroll
        for (int r = 0; r < EL; ++r) v[r] = make_float2(0.f, 0.f);
      }
      line_fft<PL, false>(v, L, p, a.py.tw, Sync{});
      if (live) {
#pragma unroll
        for (int m = 0; m < EL; ++m) T[gcol + p + P * m] = v[m];
      }
    } else {
      if (live) {
#pragma unroll
        for (int r = 0; r < EL; ++r) v[r] = T[gcol + p + P * r];
      } else {
#pragma unroll
        for (int r = 0; r < EL; ++r) v[r] = make_float2(0.f, 0.f);
      }
      line_fft<PL, true>(v, L, p, a.py.tw, Sync{});
      if (live) {
        const int x = (int)(col % nx), c = (int)(col / nx);
        const float2 gxz = cmul(a.w.gx[x], gzz);
        const bool in_xzc = x >= g.r0[1] && x < g.r1[1] && 0 >= g.r0[2] && 0 < g.r1[2] && c >= g.r0[3] && c < g.r1[3];
        const float2* __restrict__ gmc = gamma + (gcol - (long long)c * g.npts);
        float2* __restrict__ dEc = dE + gcol;
        float2* __restrict__ Ec = E + gcol;
        constexpr int NH = kEpilogueParts<EL>, H = EL / NH;
#pragma unroll
        for (int h = 0; h < NH; ++h) {
          float2 gm[H], d0[H], e0[H];
#pragma unroll
          for (int i = 0; i < H; ++i) {
            const int y = p + P * (H * h + i);
            gm[i] = gmc[y];
            d0[i] = dEc[y];
            e0[i] = acc_now ? Ec[y] : make_float2(0.f, 0.f);
          }
#pragma unroll
          for (int i = 0; i < H; ++i) {
            const int m = H * h + i;
            const int y = p + P * m;
            const float2 gyy = MODE == kCol2dStep ? sgy[y] : a.w.gy[y];
            const float2 ep = cmul_conj(cmul_conj(v[m], gxz), gyy);
            const float2 one_m = make_float2(1.f - kAlpha * gm[i].x, -kAlpha * gm[i].y);
            const float2 t = cmul(cmul(gm[i], gm[i]), ep);
            const float2 dn = cadd(cmul(one_m, d0[i]), make_float2(kAlpha * t.y, -kAlpha * t.x));
            dEc[y] = dn;
            if (acc_now) Ec[y] = cadd(e0[i], a.acc2 ? cadd(d0[i], dn) : dn);
            if (in_xzc && y >= g.r0[0] && y < g.r1[0]) esum = fmaf(dn.x, dn.x, fmaf(dn.y, dn.y, esum));
            v[m] = dn;
          }
        }
        if constexpr (MODE == kCol2dStep) {
          // K1 of the next iteration on the same column: source, next ramps
          const float2 gxz1 = cmul(w1.gx[x], w1.gz[0]);
          const float2* __restrict__ sr = src ? src + gcol : nullptr;
#pragma unroll
          for (int m = 0; m < EL; ++m) {
            const int y = p + P * m;
            float2 e = v[m];
            if (sr) e = cadd(e, cmul(A, sr[y]));
            v[m] = cmul(cmul(e, gxz1), sgy[N + y]);
          }
        }
      }
      if constexpr (MODE == kCol2dStep) {
        line_fft<PL, false>(v, L, p, a.py.tw, Sync{});
        if (live) {
#pragma unroll
          for (int m = 0; m < EL; ++m) T[gcol + p + P * m] = v[m];
        }
      }
    }
  }
  if constexpr (MODE != kCol2dFwd) {
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
    if (MODE == kCol2dStep && a.fin)
      finish_in_last_block(const_cast<DevState*>(st), a.rule, a.hist, partials, a.bpr, rhs);
  }
}

template <class PL>
__global__ void __launch_bounds__(kThreads, 2)
    kmc_col_fwd2d(InnerArgs a, const float2* __restrict__ dE, const float2* __restrict__ src, float2 A,
                  float2* __restrict__ T, const DevState* __restrict__ st) {
  pdl_begin();
  col2d<PL, kCol2dFwd>(a, a.w, dE, src, A, T, nullptr, nullptr, nullptr, st, nullptr);
}

template <class PL>
__global__ void __launch_bounds__(kThreads, 2)
    kmc_col_inv2d(InnerArgs a, const float2* __restrict__ T, float2* __restrict__ dE, float2* __restrict__ E,
                  const float2* __restrict__ gamma, const DevState* __restrict__ st, double* __restrict__ partials) {
  pdl_begin();
  col2d<PL, kCol2dInv>(a, a.w, nullptr, nullptr, make_float2(0.f, 0.f), const_cast<float2*>(T), dE, E, gamma,
                       st, partials);
}

template <class PL>
__global__ void __launch_bounds__(kThreads, 2)
    kmc_col_step2d(InnerArgs a, Wig w1, const float2* __restrict__ src1, float2 A, float2* __restrict__ T,
                   float2* __restrict__ dE, float2* __restrict__ E, const float2* __restrict__ gamma,
                   const DevState* __restrict__ st, double* __restrict__ partials) {
  pdl_begin();
  col2d<PL, kCol2dStep>(a, w1, nullptr, src1, A, T, dE, E, gamma, st, partials);
}

}  // namespace mixed
}  // namespace ws
