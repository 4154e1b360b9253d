// C ABI of the B200 MBS loop (declared in include/wavesim_b200.h).
//
// Host runtime: FFT planning (radix schedules, twiddle tables, tile and
// cluster shapes), device buffers, the per-solver CUDA stream, and the loop
// driver.  The loop runs either as one CUDA graph (first wiggle cycle with the
// source, then a device-side while node over the steady cycle whose condition
// the last block of the cycle's final K3 sets) or, when a host callback needs
// the history, as launches from a host loop.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <mutex>
#include <vector>

#include "wavesim_b200.h"
#include "ws_fast.cuh"
#include "ws_kernels.cuh"
#include "ws_mixed.cuh"
#include "ws_tma.cuh"

namespace ws {

constexpr int kEmax = 16;           // max elements per thread per FFT stage
constexpr int kMaxThreadsPow2 = 512;
constexpr int kMaxThreadsMixed = 512;
constexpr size_t kSmemBudget = 150 * 1024;  // per-block tile budget (bytes)
constexpr int kNumSms = 148;

thread_local std::string g_last_error;

static int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define WS_CUDA(call)                                                                          \
  do {                                                                                         \
    cudaError_t err__ = (call);                                                                \
    if (err__ != cudaSuccess) {                                                                \
      return fail(err__ == cudaErrorMemoryAllocation ? WS_ERR_OUT_OF_MEMORY : WS_ERR_CUDA,     \
                  std::string(#call) + ": " + cudaGetErrorString(err__));                      \
    }                                                                                          \
  } while (0)

// ---------------------------------------------------------------------------
// planning
// ---------------------------------------------------------------------------
// Radix schedules of the generic kernels: 0 the largest radices first (the
// default), 1 radices of at most 8 first (more, lighter stages), 2 the
// default radices in reverse order.  Any order is a valid Stockham schedule;
// the autotuner picks one by time.
constexpr int kNumSchedules = 3;
static bool plan_radices(int n, std::vector<int>& out, int sched = 0) {
  out.clear();
  static const int pref0[] = {16, 12, 13, 11, 10, 9, 8, 7, 6, 5, 4, 3, 2};
  static const int pref1[] = {8, 7, 6, 5, 4, 3, 9, 10, 11, 12, 13, 16, 2};
  const int* pref = sched == 1 ? pref1 : pref0;
  while (n > 1) {
    bool found = false;
    for (int i = 0; i < 13; ++i) {
      const int r = pref[i];
      if (n % r == 0) {
        out.push_back(r);
        n /= r;
        found = true;
        break;
      }
    }
    if (!found) return false;
  }
  if (sched == 2) std::reverse(out.begin(), out.end());
  return (int)out.size() <= kMaxStages;
}

static bool length_supported(int n) {
  std::vector<int> r;
  return n >= 1 && n <= 65536 && plan_radices(n, r);
}

// Fast power-of-two kernels (ws_fast.cuh), instantiated for these shapes.
struct FastInner {
  int n, c, do_x;
  const void* fwd;
  const void* inv;
  size_t smem;      // bytes (3-D, enough for both kernels); 2-D: bytes per held column, one extra column of scratch
  size_t smem_fwd, smem_inv;  // 3-D: what each kernel needs
  const void* fused = nullptr;  // K3 of one iteration + K1 of the next (3-D planes on a cluster), or null
  size_t smem_fused = 0;
  const void* fused_tma = nullptr;  // the same with K3's rows loaded by a tensor copy (first argument: the map)
  const void* col_step = nullptr;   // the column pass of the split fused step (kc_col_step), or null
  size_t smem_col = 0;              // its dynamic shared memory (kc_col_step2d, kmc_col_step)
  int lines = 0;                    // 2-D: columns per block (0: 4096 / N, 16 elements per thread)
};
struct FastPencil {
  int no, ty;
  const void* fn;
  int nc;        // components it transforms together (1, or 3 with the dyadic Green's function)
  int threads;
  size_t smem;
  int dims;      // 3: z pencils of 3-D grids only; 2: x pencils of 2-D grids only; 0: both
};

template <int N, int C, bool DX>
static FastInner fast_inner() {
  using G = fast::PlaneGeom<N, C, DX>;
  FastInner f{N, C, DX ? 1 : 0, (const void*)fast::kf_plane_fwd<N, C, DX>,
              (const void*)fast::kf_plane_inv<N, C, DX>, DX ? G::smem : (size_t)G::CS * sizeof(float2),
              DX ? (G::PUSH ? G::smem_push : G::smem_a) : 0, DX ? G::smem_max_ab : 0};
  if constexpr (DX) {
    f.col_step = (const void*)fast::kc_col_step<N, C>;
  } else {
    f.col_step = (const void*)fast::kc_col_step2d<N>;
    f.smem_col = fast::smem_col_step2d<N>();
  }
  if constexpr (DX && C > 1) {
    if constexpr (C >= 16) {  // small tiles: the column tile and the row tile fit side by side
      f.fused = (const void*)fast::kf_plane_fused_push<N, C>;
      f.smem_fused = fast::FusedPushGeom<N, C>::smem;
    } else {
      f.fused = (const void*)fast::kf_plane_fused<N, C>;
      f.fused_tma = (const void*)fast::kf_plane_fused_tma<N, C>;
      f.smem_fused = G::smem_max_ab;
    }
  }
  return f;
}
template <int NO, int TY>
static FastPencil fast_pencil() {
  return FastPencil{NO, TY, (const void*)fast::kf_pencil<NO, TY>, 1, TY * (NO / 16),
                    (size_t)(TY + 1) * NO * sizeof(float2), 0};
}
// mixed-radix / vector kernels (ws_mixed.cuh)
using Plan192 = mixed::Plan<192, 12, 12, 4, 4>;
using Plan96 = mixed::Plan<96, 12, 12, 4, 2>;
using Plan160 = mixed::Plan<160, 20, 10, 4, 4>;
using Plan224 = mixed::Plan<224, 28, 14, 4, 4>;
// (radix orders by register use: 5 x 4 x 4 x 4 spilled 416 bytes a thread in
// the 2-D column pass, 4 x 4 x 4 x 5 16; 7 x 4 x 4 x 4 84, 14 x 4 x 4 x 2 40)
using Plan320 = mixed::Plan<320, 20, 4, 4, 4, 5>;
using Plan448 = mixed::Plan<448, 28, 14, 4, 4, 2>;
using Plan576 = mixed::Plan<576, 36, 12, 12, 4>;
template <class PL, int C>
static FastInner mixed_inner() {
  using G = mixed::MGeom<PL, C>;
  FastInner f{PL::N, C, 1, (const void*)mixed::km_plane_fwd<PL, C>, (const void*)mixed::km_plane_inv<PL, C>,
              G::smem, G::smem, G::smem};
  f.fused = (const void*)mixed::km_plane_fused<PL, C>;
  f.fused_tma = (const void*)mixed::km_plane_fused_tma<PL, C>;
  f.col_step = (const void*)mixed::kmc_col_step<PL, C>;
  f.smem_col = mixed::smem_col_step<PL, C>();
  f.smem_fused = G::smem;
  static_assert((size_t)PL::N * G::LR * sizeof(float2) + 128 <= G::smem, "the dense row tile fits");
  return f;
}
// 2-D columns on the mixed-radix lines (kmc_col_*2d), one round of lines per block
template <class PL>
static FastInner mixed_inner2d() {
  using G = mixed::MGeom2d<PL>;
  FastInner f{PL::N, 1, 0, (const void*)mixed::kmc_col_fwd2d<PL>, (const void*)mixed::kmc_col_inv2d<PL>,
              (size_t)G::CS * sizeof(float2), 0, 0};
  f.col_step = (const void*)mixed::kmc_col_step2d<PL>;
  f.smem_col = mixed::smem_col_step2d<PL>();
  f.lines = G::LPR;
  return f;
}
// z pencils of 3-D grids (one or three components), and x pencils of 2-D grids (one)
template <class PL, int TY, int NC>
static FastPencil mixed_pencil() {
  return FastPencil{PL::N, TY, (const void*)mixed::km_pencil<PL, TY, NC, true>, NC, TY * PL::P,
                    (size_t)(TY + 1) * PL::N * sizeof(float2), 3};
}
template <class PL, int TY>
static FastPencil mixed_pencil2d() {
  return FastPencil{PL::N, TY, (const void*)mixed::km_pencil<PL, TY, 1, false>, 1, TY * PL::P,
                    (size_t)(TY + 1) * PL::N * sizeof(float2), 2};
}

static const std::vector<FastInner>& fast_inner_table() {
  static const std::vector<FastInner> t = {
      fast_inner<64, 1, true>(),     fast_inner<128, 2, true>(),    fast_inner<256, 8, true>(),
      fast_inner<256, 16, true>(),
      fast_inner<64, 1, false>(),    fast_inner<128, 1, false>(),   fast_inner<256, 1, false>(),
      fast_inner<512, 1, false>(),   fast_inner<1024, 1, false>(),  fast_inner<2048, 1, false>(),
      mixed_inner<Plan192, 6>(),     mixed_inner<Plan96, 1>(),      mixed_inner<Plan160, 5>(),
      mixed_inner<Plan224, 7>(),
      mixed_inner2d<Plan192>(),      mixed_inner2d<Plan320>(),      mixed_inner2d<Plan448>(),
      mixed_inner2d<Plan576>()};
  return t;
}
// Persistent TMA-pipelined K2 (ws_tma.cuh) for z pencils of a 3-D grid.
struct TmaPencil {
  int no, ty, stages;
  const void* fn;
  size_t smem;
  int threads;
  int nc = 1;  // components (3: the vector form, kt_pencil_vec)
};
template <int NO, int TY, int S>
static TmaPencil tma_pencil() {
  using PT = tma::PencilTile<NO, TY, S>;
  return TmaPencil{NO, TY, S, (const void*)tma::kt_pencil<NO, TY, S>, PT::smem, PT::kThreads};
}
template <class PL, int TY, int S>
static TmaPencil tma_pencil_vec() {
  using PT = tma::VecPencilTile<PL, TY, S>;
  return TmaPencil{PL::N, TY, S, (const void*)tma::kt_pencil_vec<PL, TY, S>, PT::smem, PT::kThreads, 3};
}
// The x passes of the split fused step (kt_xpencil, ws_tma.cuh).
struct XPencil {
  int no, ty, stages;
  const void* fwd;
  const void* inv;
  size_t smem;
  int threads;
};
template <int NO, int TY, int S>
static XPencil x_pencil() {
  using PT = tma::PencilTile<NO, TY, S>;
  return XPencil{NO, TY, S, (const void*)tma::kt_xpencil<NO, TY, S, false>,
                 (const void*)tma::kt_xpencil<NO, TY, S, true>, PT::smem, PT::kThreads};
}
template <class PL, int TY, int S>
static XPencil x_pencil_m() {
  using PT = tma::MixedXTile<PL, TY, S>;
  return XPencil{PL::N, TY, S, (const void*)tma::kt_xpencil_m<PL, TY, S, false>,
                 (const void*)tma::kt_xpencil_m<PL, TY, S, true>, PT::smem, PT::kThreads};
}
static const std::vector<XPencil>& x_pencil_table() {
  // the first match of (no, ty) is the default
  static const std::vector<XPencil> t = {x_pencil<64, 16, 3>(), x_pencil<128, 16, 3>(), x_pencil<256, 8, 3>(),
                                         x_pencil<256, 8, 4>(), x_pencil<256, 16, 3>(), x_pencil<256, 8, 2>(),
                                         x_pencil_m<Plan192, 8, 4>(),
                                         x_pencil_m<Plan192, 16, 3>(), x_pencil_m<Plan96, 16, 3>(),
                                         x_pencil_m<Plan160, 16, 3>(), x_pencil_m<Plan224, 16, 3>()};
  return t;
}
using Plan192t = mixed::Plan<192, 12, 12, 4, 4>;
static const std::vector<TmaPencil>& tma_pencil_table() {
  // the first match of (no, ty) is the default; the autotuner tries the rest
  // (at 256: 8 y x 3 stages, 4 blocks of 128 threads per SM at 128 registers,
  // measured 0.0667 ms against 0.0732 for 8 x 4 stages at 3 blocks per SM,
  // 0.070 for 16 x 3, 0.081 for 4 x 4 and 0.096 for 8 x 6)
  static const std::vector<TmaPencil> t = {tma_pencil<64, 16, 3>(), tma_pencil<128, 16, 3>(),
                                           tma_pencil<256, 8, 3>(),  tma_pencil<256, 8, 4>(),
                                           tma_pencil<256, 8, 2>(),  tma_pencil<256, 16, 3>(),
                                           tma_pencil<256, 16, 2>(), tma_pencil<256, 8, 6>(),
                                           tma_pencil<256, 4, 4>(),
                                           // 192 x 3 components, one at a time in registers: 8 y x 2 stages
                                           // (3 blocks per SM) measured 0.120 ms at 192^3 against 0.143
                                           // (8 x 3), 0.154 (4 x 3) and 0.145 (16 x 2); all three lines in
                                           // registers took 0.131 at best
                                           tma_pencil_vec<Plan192t, 8, 2>(), tma_pencil_vec<Plan192t, 8, 3>(),
                                           tma_pencil_vec<Plan192t, 4, 3>(), tma_pencil_vec<Plan192t, 16, 2>()};
  return t;
}

static const std::vector<FastPencil>& fast_pencil_table() {
  static const std::vector<FastPencil> t = {
      fast_pencil<32, 16>(),  fast_pencil<64, 16>(),  fast_pencil<128, 16>(),
      fast_pencil<256, 16>(), fast_pencil<512, 8>(),  fast_pencil<1024, 4>(),
      mixed_pencil<Plan192, 8, 3>(),   // (a TY = 8 variant first: the later TY = 16 is the default)
      mixed_pencil<Plan192, 16, 1>(),
      mixed_pencil<Plan192, 16, 3>(),
      mixed_pencil<Plan96, 16, 1>(),
      mixed_pencil<Plan96, 16, 3>(),
      mixed_pencil<Plan160, 16, 1>(),
      mixed_pencil<Plan224, 16, 1>(),
      mixed_pencil2d<Plan192, 16>(),
      mixed_pencil2d<Plan320, 8>(),
      mixed_pencil2d<Plan448, 8>(),
      mixed_pencil2d<Plan576, 8>(),
      mixed_pencil<mixed::Plan<64, 16, 16, 4>, 16, 3>(),
      mixed_pencil<mixed::Plan<128, 16, 16, 8>, 16, 3>(),
      mixed_pencil<mixed::Plan<256, 16, 16, 16>, 16, 3>()};
  return t;
}

struct Layout {
  const FastInner* fi = nullptr;   // fast K1/K3, or null (generic)
  const FastPencil* fp = nullptr;  // fast K2, or null (generic)
  const TmaPencil* tp = nullptr;   // persistent TMA K2 (takes precedence over fp), or null
  const XPencil* xp = nullptr;     // x passes of the split fused step, or null (one-kernel fused step)
  int rset = kPow2;  // radix set of every plan of the solver
  int mode3d = 0;
  int csize = 1;     // 3-D: blocks (cluster) per plane
  int ncols = 1;     // 2-D: columns per block
  int ty = 16;       // outer pass: consecutive y per block
  int th_inner = 256, th_outer = 256;
  size_t smem_inner = 0, smem_outer = 0;
  long long grid_inner = 0, grid_outer = 0;
};

static bool is_pow2(long long n) { return n >= 1 && (n & (n - 1)) == 0; }

// Overrides of the layout heuristics, for the autotuner (0 = heuristic).
struct LayoutChoice {
  int inner = 0;  // 1: fast inner kernels when a shape matches, 2: generic
  int outer = 0;  // 1: fast pencil when a shape matches, 2: generic, 3 + k: TMA pencil of k stages
  int csize = 0;  // 3-D generic: smallest blocks per plane to try
  int ncols = 0;  // 2-D generic: columns per block
  int ty = 0;     // generic outer: consecutive y per block
  int sched = 0;  // radix schedule of the generic kernels' plans (plan_radices)
  int xp = 0;     // split step: 1 + index of the x pencil in x_pencil_table (0: the default)
  bool operator==(const LayoutChoice& o) const {
    return inner == o.inner && outer == o.outer && csize == o.csize && ncols == o.ncols && ty == o.ty &&
           sched == o.sched && xp == o.xp;
  }
};

static int make_layout(const Geom& g, Layout& L, std::string& why, const LayoutChoice& ch = LayoutChoice{}) {
  L = Layout{};
  L.mode3d = g.nz > 1;
  L.rset = kPow2;
  for (long long n : {(long long)g.ny, (long long)g.nx, (long long)g.nz})
    if (!is_pow2(n)) L.rset = kMixed;
  const int kMaxThreads = L.rset == kPow2 ? kMaxThreadsPow2 : kMaxThreadsMixed;
  auto threads_for = [&](long long elems) {
    long long t = (elems + kEmax - 1) / kEmax;
    t = ((t + 31) / 32) * 32;
    return (int)std::max(32LL, std::min((long long)kMaxThreads, t));
  };
  const int ny = g.ny;
  const size_t col_bytes = (size_t)padded(ny) * sizeof(float2);
  if (L.mode3d) {
    // smallest divisor C of Nx (<= 16) whose tile fits
    int best = 0;
    for (int c = ch.csize ? ch.csize : 1; c <= 16; ++c) {
      if (g.nx % c) continue;
      const long long cols = g.nx / c;
      const long long elems = cols * ny;
      if (elems > (long long)kMaxThreads * kEmax) continue;
      if (cols * col_bytes > kSmemBudget) continue;
      if (c > 1 && !length_supported((int)cols)) continue;
      best = c;
      break;
    }
    if (!best) {
      why = "an Ny x Nx plane of this size does not fit a cluster of 16 blocks";
      return WS_ERR_UNSUPPORTED;
    }
    L.csize = best;
    const long long cols = g.nx / best;
    L.th_inner = threads_for(cols * ny);
    L.smem_inner = cols * col_bytes;
    L.grid_inner = (long long)g.nz * g.nc * best;
  } else {
    const long long total_cols = (long long)g.nx * g.nc;
    const long long max_cols_fit = std::max(1LL, std::min((long long)(kSmemBudget / col_bytes),
                                                          (long long)kMaxThreads * kEmax / (long long)ny));
    if ((long long)ny > (long long)kMaxThreads * kEmax || col_bytes > kSmemBudget) {
      why = "Ny too large for one block";
      return WS_ERR_UNSUPPORTED;
    }
    // aim for >= 2 blocks per SM, at most ~8K elements per block
    long long want = std::max(1LL, std::min(max_cols_fit, (8192LL + ny - 1) / ny));
    while (want > 1 && (total_cols + want - 1) / want < 2 * kNumSms) want /= 2;
    if (ch.ncols) want = std::max(1LL, std::min<long long>(ch.ncols, max_cols_fit));
    L.ncols = (int)want;
    L.th_inner = threads_for((long long)want * ny);
    L.smem_inner = want * col_bytes;
    L.grid_inner = (total_cols + want - 1) / want;
  }
  // outer pass
  const int no = L.mode3d ? g.nz : g.nx;
  const long long mids = L.mode3d ? g.nx : 1;
  int ty = 16;
  while (ty > 1 && ((long long)padded(g.nc * ty) * no * sizeof(float2) > kSmemBudget ||
                    (long long)g.nc * ty * no > (long long)kMaxThreads * kEmax))
    ty /= 2;
  if (ty > g.ny) ty = std::max(1, g.ny);
  while (ty > 4 && ((g.ny + ty - 1) / ty) * mids < 2 * kNumSms) ty /= 2;
  if (ch.ty) ty = std::max(1, std::min(ch.ty, g.ny));
  if ((long long)padded(g.nc * ty) * no * sizeof(float2) > kSmemBudget ||
      (long long)g.nc * ty * no > (long long)kMaxThreads * kEmax) {
    why = "outer dimension too long for one block";
    return WS_ERR_UNSUPPORTED;
  }
  L.ty = ty;
  L.th_outer = threads_for((long long)g.nc * ty * no);
  L.smem_outer = (size_t)padded(g.nc * ty) * no * sizeof(float2);
  L.grid_outer = (long long)((g.ny + ty - 1) / ty) * mids;
  // fast power-of-two kernels where a shape matches
  const char* path = std::getenv("WAVESIM_B200_PATH");
  if (path && std::strcmp(path, "generic") == 0) return WS_OK;
  // 3-D: the first plane kernel of the grid's size, or the one with the
  // cluster size asked for (autotuner: ch.csize; WAVESIM_B200_CLUSTER)
  int want_c = ch.csize;
  if (!want_c)
    if (const char* e = std::getenv("WAVESIM_B200_CLUSTER")) want_c = std::atoi(e);
  const FastInner* first3 = nullptr;
  const FastInner* pick3 = nullptr;
  for (const FastInner& f : fast_inner_table()) {
    if (ch.inner == 2) break;
    if (L.mode3d && f.do_x && g.ny == f.n && g.nx == f.n) {
      if (!first3) first3 = &f;
      if (want_c && f.c == want_c) pick3 = &f;
    }
    if (!L.mode3d && !f.do_x && g.ny == f.n) L.fi = &f;
  }
  if (L.mode3d) L.fi = pick3 ? pick3 : first3;
  if (L.fi && !L.mode3d) {
    // one round of lines per block: 256 threads, 16 elements each (mixed-radix lines: E each)
    const long long total_cols = (long long)g.nx * g.nc;
    const long long want = L.fi->lines ? L.fi->lines : std::max(1, 4096 / g.ny);
    L.ncols = (int)want;
    L.grid_inner = (total_cols + want - 1) / want;
  }
  if (L.fi && L.mode3d) L.grid_inner = (long long)g.nz * g.nc * L.fi->c;
  if (ch.outer != 2) {
    // the last pencil of the shape, or the one with the y tile asked for
    // (autotuner: outer = 1 with ty; WAVESIM_B200_PENCIL_TY)
    int want_ty = ch.outer == 1 ? ch.ty : 0;
    if (!want_ty)
      if (const char* e = std::getenv("WAVESIM_B200_PENCIL_TY")) want_ty = std::atoi(e);
    for (const FastPencil& f : fast_pencil_table())
      if (f.no == no && g.ny % f.ty == 0 && f.nc == g.nc && (f.dims == 0 || f.dims == (L.mode3d ? 3 : 2)) && (!want_ty || f.ty == want_ty))
        L.fp = &f;
  }
  if (L.fp) L.grid_outer = (long long)(g.ny / L.fp->ty) * mids;  // blocks of the fast pencil kernel
  // the TMA pencil where a shape matches: by default (WAVESIM_B200_K2=plain keeps kf_pencil), or the
  // autotuner's choice of stages
  const char* k2 = std::getenv("WAVESIM_B200_K2");
  const bool tma_ok = L.mode3d && (ch.outer == 0 || ch.outer >= 3) &&
                      !(ch.outer == 0 && k2 && std::strcmp(k2, "plain") == 0);
  int want_tty = 0, want_ts = 0;  // WAVESIM_B200_TMA_TY / _TMA_STAGES: the y tile and stages of the TMA pencil
  if (const char* e = std::getenv("WAVESIM_B200_TMA_TY")) want_tty = std::atoi(e);
  if (const char* e = std::getenv("WAVESIM_B200_TMA_STAGES")) want_ts = std::atoi(e);
  if (tma_ok)
    for (const TmaPencil& f : tma_pencil_table())
      if (f.no == no && f.nc == g.nc && g.ny % f.ty == 0 && (ch.outer < 3 || f.stages == ch.outer - 3) &&
          (!want_tty || f.ty == want_tty) && (!want_ts || f.stages == want_ts)) {
        L.tp = &f;
        break;
      }
  // the split fused step (x pencils + column pass) on power-of-two planes;
  // WAVESIM_B200_STEP=cluster keeps the one-kernel step with the cluster
  // exchange, WAVESIM_B200_XTY picks the x pencils' y tile
  const char* step = std::getenv("WAVESIM_B200_STEP");
  int want_xty = 0, want_xs = 0;  // WAVESIM_B200_XTY / _XSTAGES: the y tile and stages of the x pencils
  if (const char* e = std::getenv("WAVESIM_B200_XTY")) want_xty = std::atoi(e);
  if (const char* e = std::getenv("WAVESIM_B200_XSTAGES")) want_xs = std::atoi(e);
  if (L.mode3d && L.fi && L.fi->col_step && !(step && std::strcmp(step, "cluster") == 0)) {
    const auto& xt = x_pencil_table();
    if (ch.xp > 0 && ch.xp <= (int)xt.size()) {
      const XPencil& f = xt[ch.xp - 1];
      if (f.no != g.nx || g.ny % f.ty) {
        why = "the x pencil asked for does not fit the grid";
        return WS_ERR_UNSUPPORTED;
      }
      L.xp = &f;
    } else {
      for (const XPencil& f : xt)
        if (f.no == g.nx && g.ny % f.ty == 0 && (!want_xty || f.ty == want_xty) && (!want_xs || f.stages == want_xs)) {
          L.xp = &f;
          break;
        }
    }
  }
  return WS_OK;
}

// ---------------------------------------------------------------------------
// solver object
// ---------------------------------------------------------------------------
struct GraphKey {
  double threshold = -1;
  long long max_iter = -1;
  int interval = -1, stop_rule = -1, nan_stop = -1, nrhs = -1, warm = -1;
  double warm_ratio = -1;
  bool operator==(const GraphKey& o) const {
    return threshold == o.threshold && max_iter == o.max_iter && interval == o.interval &&
           stop_rule == o.stop_rule && nan_stop == o.nan_stop && nrhs == o.nrhs && warm == o.warm &&
           warm_ratio == o.warm_ratio;
  }
};

struct Solver {
  int device = 0;
  cudaStream_t stream = nullptr;
  Geom g{};
  Layout lay;
  int nw = 0;
  float eps = 0.f;
  float2 k02e{};
  std::vector<Wig> wig;
  float* d_wigf = nullptr;   // all pxe/pye/pze
  float2* d_wigc = nullptr;  // all gx/gy/gz
  float2* d_gamma = nullptr;      // n_media gammas of npts elements each
  int n_media = 1;                // > 1: a batch of media, right-hand side r on gamma r
  // per right-hand side (batch of nrhs, capacity batch_cap): fields at r * field elements
  float2 *d_E = nullptr, *d_dE = nullptr, *d_T = nullptr, *d_src = nullptr;
  int batch_cap = 0;
  int nrhs = 1;
  float2* d_stage = nullptr;
  size_t stage_cap = 0;
  float2* d_out = nullptr;
  size_t out_cap = 0;
  DevState* d_state = nullptr;
  double* d_hist = nullptr;  // diff | fresh
  long long hist_cap = 0;
  double* d_energy = nullptr;
  double* d_partials = nullptr;  // per-block ROI energy of K3
  long long partials_cap = 0;    // elements of d_partials
  float2* d_init = nullptr;      // warm starts: v = gamma psi0 / Nw per right-hand side (batch_cap of them)
  int* d_err = nullptr;          // set by a fast kernel whose cluster exchange or TMA wait gave up
  CUtensorMap tmap_T{};          // T as {2 Ny floats, Nx, Nz * tmap_nrhs}, for the TMA pencil
  const void* tmap_base = nullptr;
  int tmap_nrhs = 0;
  const void* tmap_kernel = nullptr;  // the TMA pencil the map and tma_blocks were made for
  int tma_blocks = 0;            // resident blocks of the TMA pencil (its persistent grid)
  CUtensorMap tmap_X{};          // T as {2 Ny floats, Nx, Nz Nc nrhs}, box {2 TY, Nx, 1}, for the x pencils
  const void* xmap_base = nullptr;
  int xmap_nrhs = 0;
  const void* xmap_kernel = nullptr;
  int x_blocks = 0;              // resident blocks of the x pencil (its persistent grid)
  CUtensorMap tmap_slab{};       // T as 2-D {2 Ny floats, Nx Nz Nc nrhs}, box {2 LR, N}, for kf_plane_fused_tma
  const void* slab_base = nullptr;
  int slab_nrhs = 0;
  const void* slab_kernel = nullptr;
  int fused_tma = 1;             // the fused step loads K3's rows by a tensor copy (WAVESIM_B200_FUSED_TMA=0: not)
  int pf_inner = 0, pf_outer = 0;  // L2 prefetch distance of the fast kernels, in blocks (0: off)
  bool warm = false;             // the current solve starts from d_init
  int pstd = 0;                  // a PSTD stepper's solver: K2 applies the Laplacian (see ws_pstd_*)
  int fuse = 0;                  // the loop runs K3 of each iteration fused with K1 of the next
  LayoutChoice tuned{};          // the autotuner's choice (all zero: the heuristics)
  double warm_ratio = 0.0;       // discard threshold of the current solve
  long long wait_clocks = 0;     // bound of the TMA pencils' tile waits (0: the default)
  int fin_fuse = 0;              // WAVESIM_B200_FIN=1: the column pass's last block runs the stop rule instead
                                 // of k_finish_iteration (measured: 256^3 46.05 against 45.63 ms, 1024^2
                                 // 8.83 against 8.74 ms, 320^2 5.52 against 5.40 ms; off)
  int pdl = 0;                   // WAVESIM_B200_PDL=1: launch the loop's kernels with programmatic
                                 // dependent launch (measured: 256^3 solve 46.3 against 44.3 ms,
                                 // 96^3 3.38 against 2.80 ms, 1024^2 8.50 against 8.71 ms; off)
  float2* d_tw = nullptr;
  FftPlan py{}, pxl{}, po{};
  const float2* twx = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  GraphKey gkey;
  cudaEvent_t ev[8] = {};
};

static void free_graph(Solver* s) {
  if (s->gexec) cudaGraphExecDestroy(s->gexec);
  if (s->graph) cudaGraphDestroy(s->graph);
  s->gexec = nullptr;
  s->graph = nullptr;
}

// The fused K3 + K1 step is used where the layout has one (3-D fast planes on
// a cluster); WAVESIM_B200_FUSE=0 keeps the three kernels separate.
static void update_fuse(Solver* s) {
  const char* e = std::getenv("WAVESIM_B200_FUSE");
  const bool on3 = s->lay.fi && (s->lay.fi->fused || s->lay.xp) && s->lay.mode3d;
  const bool on2 = s->lay.fi && !s->lay.mode3d && s->lay.fi->col_step;  // 2-D: K2 + the column pass
  const int f = ((on3 || on2) && !s->pstd && !(e && std::strcmp(e, "0") == 0)) ? 1 : 0;
  if (f != s->fuse) free_graph(s);
  s->fuse = f;
}

static void destroy_solver(Solver* s) {
  if (!s) return;
  cudaSetDevice(s->device);
  free_graph(s);
  void* ptrs[] = {s->d_wigf, s->d_wigc,  s->d_gamma,  s->d_E,        s->d_dE, s->d_T,   s->d_src,
                  s->d_stage, s->d_out, s->d_state, s->d_hist, s->d_energy, s->d_tw, s->d_partials, s->d_init,
                  s->d_err};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  for (auto& e : s->ev)
    if (e) cudaEventDestroy(e);
  if (s->stream) cudaStreamDestroy(s->stream);
  delete s;
}

static int build_plan(int n, const std::vector<float2>& tw_all_offset_dummy, FftPlan& p, int sched = 0) {
  (void)tw_all_offset_dummy;
  std::vector<int> r;
  if (!plan_radices(n, r, sched)) return WS_ERR_UNSUPPORTED;
  p.n = n;
  p.nst = (int)r.size();
  for (int i = 0; i < kMaxStages; ++i) p.radix[i] = i < (int)r.size() ? r[i] : 1;
  return WS_OK;
}

static void push_twiddles(std::vector<float2>& all, int n, size_t& off) {
  off = all.size();
  for (int k = 0; k < n; ++k) {
    const double a = -2.0 * M_PI * (double)k / (double)n;
    all.push_back(make_float2((float)std::cos(a), (float)std::sin(a)));
  }
}

template <typename K>
static cudaError_t allow_dynamic_smem(K kernel, int optin) {
  cudaFuncAttributes fa{};
  cudaError_t e = cudaFuncGetAttributes(&fa, (const void*)kernel);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute((const void*)kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              optin - (int)fa.sharedSizeBytes);
}

template <int RS>
static cudaError_t set_attributes_for(int optin) {
  cudaError_t e;
  if ((e = allow_dynamic_smem(k_fwd_inner<kEmax, RS>, optin))) return e;
  if ((e = allow_dynamic_smem(k_inv_inner<kEmax, RS>, optin))) return e;
  if ((e = allow_dynamic_smem(k_outer<kEmax, RS>, optin))) return e;
  if ((e = cudaFuncSetAttribute(k_fwd_inner<kEmax, RS>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1))) return e;
  return cudaFuncSetAttribute(k_inv_inner<kEmax, RS>, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
}

static int set_kernel_attributes() {
  // per device: attributes are per-context
  static int done_mask = 0;
  int dev = 0;
  WS_CUDA(cudaGetDevice(&dev));
  if (dev < 31 && (done_mask >> dev) & 1) return WS_OK;
  int optin = 0;
  WS_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
  WS_CUDA(set_attributes_for<kPow2>(optin));
  WS_CUDA(set_attributes_for<kMixed>(optin));
  for (const FastInner& f : fast_inner_table()) {
    WS_CUDA(allow_dynamic_smem(f.fwd, optin));
    WS_CUDA(allow_dynamic_smem(f.inv, optin));
    WS_CUDA(cudaFuncSetAttribute(f.fwd, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    WS_CUDA(cudaFuncSetAttribute(f.inv, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    if (f.fused) {
      WS_CUDA(allow_dynamic_smem(f.fused, optin));
      WS_CUDA(cudaFuncSetAttribute(f.fused, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    }
    if (f.col_step) WS_CUDA(allow_dynamic_smem(f.col_step, optin));
    if (f.fused_tma) {
      WS_CUDA(allow_dynamic_smem(f.fused_tma, optin));
      WS_CUDA(cudaFuncSetAttribute(f.fused_tma, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    }
  }
  for (const FastPencil& f : fast_pencil_table()) WS_CUDA(allow_dynamic_smem(f.fn, optin));
  for (const TmaPencil& f : tma_pencil_table()) WS_CUDA(allow_dynamic_smem(f.fn, optin));
  for (const XPencil& f : x_pencil_table()) {
    WS_CUDA(allow_dynamic_smem(f.fwd, optin));
    WS_CUDA(allow_dynamic_smem(f.inv, optin));
  }
  if (dev < 31) done_mask |= 1 << dev;
  return WS_OK;
}

static int check_args(const int64_t N[4], int64_t n_wiggles, const ws_wiggle* wiggles, const ws_complex* gamma,
                      const int64_t roi[8], Geom& g) {
  if (!N || !gamma || !wiggles || !roi) return fail(WS_ERR_INVALID_ARGUMENT, "null argument");
  for (int i = 0; i < 4; ++i)
    if (N[i] < 1) return fail(WS_ERR_INVALID_ARGUMENT, "N must be positive");
  if (N[3] != 1 && N[3] != 3) return fail(WS_ERR_INVALID_ARGUMENT, "N(4) must be 1 (scalar) or 3 (vector)");
  if (N[0] > 65536 || N[1] > 65536 || N[2] > 65536)
    return fail(WS_ERR_UNSUPPORTED, "grid dimension larger than 65536");
  if (n_wiggles < 1 || n_wiggles > 64) return fail(WS_ERR_INVALID_ARGUMENT, "Nwiggles must be in [1, 64]");
  g.ny = (int)N[0];
  g.nx = (int)N[1];
  g.nz = (int)N[2];
  g.nc = (int)N[3];
  g.npts = (long long)g.ny * g.nx * g.nz;
  if (g.npts * g.nc > (1LL << 31)) return fail(WS_ERR_UNSUPPORTED, "grid larger than 2^31 elements");
  for (int d = 0; d < 4; ++d) {
    const int64_t a = roi[2 * d], b = roi[2 * d + 1];
    if (a < 1 || b < a || b > N[d]) return fail(WS_ERR_INVALID_ARGUMENT, "roi outside the grid");
    g.r0[d] = (int)(a - 1);
    g.r1[d] = (int)b;
  }
  for (int d = 0; d < 3; ++d)
    if (!length_supported((int)N[d]))
      return fail(WS_ERR_UNSUPPORTED, "grid dimension " + std::to_string(N[d]) +
                                          " has a prime factor above 13 (use an efficient size)");
  return WS_OK;
}

static cudaMemcpyKind kind_from(int memory) { return memory == WS_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice; }

static size_t field_elems(const Solver* s) { return (size_t)s->g.npts * s->g.nc; }

// Buffers for nrhs right-hand sides (kept when large enough).
// d_partials holds at least n per-block energies (graphs hold the old pointer)
static int ensure_partials(Solver* s, long long n) {
  if (n <= s->partials_cap) return WS_OK;
  double* p = nullptr;
  WS_CUDA(cudaMalloc(&p, (size_t)n * sizeof(double)));
  if (s->d_partials) cudaFree(s->d_partials);
  s->d_partials = p;
  s->partials_cap = n;
  free_graph(s);
  return WS_OK;
}

static int ensure_batch(Solver* s, int nrhs) {
  if (nrhs <= s->batch_cap) return WS_OK;
  void* old[] = {s->d_E, s->d_dE, s->d_T, s->d_src, s->d_state, s->d_energy, s->d_partials, s->d_init};
  for (void* p : old)
    if (p) cudaFree(p);
  s->d_E = s->d_dE = s->d_T = s->d_src = s->d_init = nullptr;
  s->d_state = nullptr;
  s->d_energy = s->d_partials = nullptr;
  s->batch_cap = 0;
  if (s->d_hist) cudaFree(s->d_hist);
  s->d_hist = nullptr;
  s->hist_cap = 0;
  free_graph(s);
  const size_t nb = field_elems(s) * nrhs * sizeof(float2);
  WS_CUDA(cudaMalloc(&s->d_E, nb));
  WS_CUDA(cudaMalloc(&s->d_dE, nb));
  WS_CUDA(cudaMalloc(&s->d_T, nb));
  WS_CUDA(cudaMalloc(&s->d_src, nb));
  WS_CUDA(cudaMalloc(&s->d_state, nrhs * sizeof(DevState)));
  WS_CUDA(cudaMalloc(&s->d_energy, nrhs * sizeof(double)));
  s->partials_cap = std::max<long long>(1, s->lay.grid_inner) * nrhs;
  WS_CUDA(cudaMalloc(&s->d_partials, (size_t)s->partials_cap * sizeof(double)));
  WS_CUDA(cudaMemset(s->d_E, 0, nb));
  WS_CUDA(cudaMemset(s->d_dE, 0, nb));
  WS_CUDA(cudaMemset(s->d_state, 0, nrhs * sizeof(DevState)));
  s->batch_cap = nrhs;
  return WS_OK;
}

static int create_solver(const int64_t N[4], const ws_complex* gamma, int64_t n_wiggles, const ws_wiggle* wiggles,
                         float epsilon, ws_complex k02e, const int64_t roi[8], int memory, int device, Solver** out) {
  Geom g{};
  int rc = check_args(N, n_wiggles, wiggles, gamma, roi, g);
  if (rc) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(WS_ERR_NO_DEVICE, "no CUDA device");
  if (device < 0 || device >= ndev) return fail(WS_ERR_INVALID_ARGUMENT, "bad device ordinal");
  WS_CUDA(cudaSetDevice(device));
  rc = set_kernel_attributes();
  if (rc) return rc;
  Solver* s = new Solver();
  s->device = device;
  s->g = g;
  s->nw = (int)n_wiggles;
  s->eps = epsilon;
  s->k02e = make_float2(k02e.re, k02e.im);
  std::string why;
  rc = make_layout(g, s->lay, why);
  if (rc) {
    destroy_solver(s);
    return fail(rc, why);
  }
  update_fuse(s);
  {
    // L2 prefetch distance of the fast kernels: about one wave of resident
    // blocks (2 per SM), a whole number of clusters.  WAVESIM_B200_PREFETCH
    // sets the waves' size in blocks per SM (0 switches the prefetch off).
    int per_sm = 2;
    if (const char* e = std::getenv("WAVESIM_B200_PREFETCH")) per_sm = std::max(0, std::atoi(e));
    const int c = s->lay.fi ? std::max(1, s->lay.fi->c) : 1;
    s->pf_inner = (per_sm * kNumSms / c) * c;
    s->pf_outer = per_sm * kNumSms;
    if (const char* e = std::getenv("WAVESIM_B200_FUSED_TMA")) s->fused_tma = std::atoi(e) ? 1 : 0;
    if (const char* e = std::getenv("WAVESIM_B200_PDL")) s->pdl = std::atoi(e) ? 1 : 0;
    if (const char* e = std::getenv("WAVESIM_B200_FIN")) s->fin_fuse = std::atoi(e) ? 1 : 0;
  }
#define WS_TRY(call)                 \
  do {                               \
    cudaError_t e__ = (call);        \
    if (e__ != cudaSuccess) {        \
      destroy_solver(s);             \
      return fail(e__ == cudaErrorMemoryAllocation ? WS_ERR_OUT_OF_MEMORY : WS_ERR_CUDA, \
                  std::string(#call) + ": " + cudaGetErrorString(e__)); \
    }                                \
  } while (0)
  WS_TRY(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
  WS_TRY(cudaMalloc(&s->d_err, sizeof(int)));
  WS_TRY(cudaMemset(s->d_err, 0, sizeof(int)));
  for (auto& e : s->ev) WS_TRY(cudaEventCreate(&e));
  // plans and twiddle tables
  std::vector<float2> tw;
  size_t off_y, off_x, off_xl, off_o;
  const int no = s->lay.mode3d ? g.nz : g.nx;
  const int nxl = s->lay.mode3d ? g.nx / s->lay.csize : 1;
  push_twiddles(tw, g.ny, off_y);
  push_twiddles(tw, g.nx, off_x);
  push_twiddles(tw, nxl, off_xl);
  push_twiddles(tw, no, off_o);
  WS_TRY(cudaMalloc(&s->d_tw, tw.size() * sizeof(float2)));
  WS_TRY(cudaMemcpy(s->d_tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice));
  build_plan(g.ny, tw, s->py);
  s->py.tw = s->d_tw + off_y;
  build_plan(nxl, tw, s->pxl);
  s->pxl.tw = s->d_tw + off_xl;
  build_plan(no, tw, s->po);
  s->po.tw = s->d_tw + off_o;
  s->twx = s->d_tw + off_x;
  // wiggles
  const size_t nf = (size_t)g.nx + g.ny + g.nz;
  WS_TRY(cudaMalloc(&s->d_wigf, nf * n_wiggles * sizeof(float)));
  WS_TRY(cudaMalloc(&s->d_wigc, nf * n_wiggles * sizeof(float2)));
  const cudaMemcpyKind kind = kind_from(memory);
  for (int w = 0; w < n_wiggles; ++w) {
    const ws_wiggle& W = wiggles[w];
    if (!W.pxe || !W.pye || !W.pze || !W.gx || !W.gy || !W.gz) {
      destroy_solver(s);
      return fail(WS_ERR_INVALID_ARGUMENT, "null wiggle array");
    }
    float* f = s->d_wigf + nf * w;
    float2* c = s->d_wigc + nf * w;
    WS_TRY(cudaMemcpy(f, W.pxe, g.nx * sizeof(float), kind));
    WS_TRY(cudaMemcpy(f + g.nx, W.pye, g.ny * sizeof(float), kind));
    WS_TRY(cudaMemcpy(f + g.nx + g.ny, W.pze, g.nz * sizeof(float), kind));
    WS_TRY(cudaMemcpy(c, W.gx, g.nx * sizeof(float2), kind));
    WS_TRY(cudaMemcpy(c + g.nx, W.gy, g.ny * sizeof(float2), kind));
    WS_TRY(cudaMemcpy(c + g.nx + g.ny, W.gz, g.nz * sizeof(float2), kind));
    s->wig.push_back(Wig{f, f + g.nx, f + g.nx + g.ny, c, c + g.nx, c + g.nx + g.ny});
  }
  WS_TRY(cudaMalloc(&s->d_gamma, (size_t)g.npts * sizeof(float2)));
  WS_TRY(cudaMemcpy(s->d_gamma, gamma, (size_t)g.npts * sizeof(float2), kind));
#undef WS_TRY
  const int rc2 = ensure_batch(s, 1);
  if (rc2) {
    destroy_solver(s);
    return rc2;
  }
  *out = s;
  return WS_OK;
}

// A new medium (gamma, wiggles, epsilon, k02e, roi) of the same grid and
// wiggle count into an existing solver: uploads only, no allocation.  The
// solver's stream must be idle (it is after a solve returns).
static int reload_medium(Solver* s, const int64_t N[4], const ws_complex* gamma, int64_t n_wiggles,
                         const ws_wiggle* wiggles, float epsilon, ws_complex k02e, const int64_t roi[8], int memory) {
  Geom g{};
  int rc = check_args(N, n_wiggles, wiggles, gamma, roi, g);
  if (rc) return rc;
  WS_CUDA(cudaSetDevice(s->device));
  const cudaMemcpyKind kind = kind_from(memory);
  const size_t nf = (size_t)g.nx + g.ny + g.nz;
  for (int w = 0; w < n_wiggles; ++w) {
    const ws_wiggle& W = wiggles[w];
    if (!W.pxe || !W.pye || !W.pze || !W.gx || !W.gy || !W.gz) return fail(WS_ERR_INVALID_ARGUMENT, "null wiggle array");
    float* f = s->d_wigf + nf * w;
    float2* c = s->d_wigc + nf * w;
    WS_CUDA(cudaMemcpy(f, W.pxe, g.nx * sizeof(float), kind));
    WS_CUDA(cudaMemcpy(f + g.nx, W.pye, g.ny * sizeof(float), kind));
    WS_CUDA(cudaMemcpy(f + g.nx + g.ny, W.pze, g.nz * sizeof(float), kind));
    WS_CUDA(cudaMemcpy(c, W.gx, g.nx * sizeof(float2), kind));
    WS_CUDA(cudaMemcpy(c + g.nx, W.gy, g.ny * sizeof(float2), kind));
    WS_CUDA(cudaMemcpy(c + g.nx + g.ny, W.gz, g.nz * sizeof(float2), kind));
  }
  WS_CUDA(cudaMemcpy(s->d_gamma, gamma, (size_t)g.npts * sizeof(float2), kind));
  const float2 k = make_float2(k02e.re, k02e.im);
  bool same = s->eps == epsilon && s->k02e.x == k.x && s->k02e.y == k.y;
  for (int d = 0; d < 4; ++d) same = same && s->g.r0[d] == g.r0[d] && s->g.r1[d] == g.r1[d];
  if (!same) {
    // scalars and the roi are kernel arguments inside the graph
    s->eps = epsilon;
    s->k02e = k;
    s->g = g;
    free_graph(s);
  }
  return WS_OK;
}

static InnerArgs inner_args(const Solver* s, int w) {
  InnerArgs a{};
  a.g = s->g;
  a.w = s->wig[w];
  a.py = s->py;
  a.pxl = s->pxl;
  a.twx = s->twx;
  a.csize = s->lay.csize;
  a.mode3d = s->lay.mode3d;
  a.ncols = s->lay.ncols;
  a.bpr = (int)s->lay.grid_inner;
  a.fstride = (long long)field_elems(s);
  a.err = s->d_err;
  a.gstride = s->n_media > 1 ? (long long)s->g.npts : 0;
  a.pf = 0;  // K3 (and the generic kernels) measured slower with it
  // E' += dE' in pairs when every stop (a multiple of Nw) falls after an even iteration
  a.acc2 = (s->nw % 2 == 0) ? 1 : 0;
  return a;
}

static OuterArgs outer_args(const Solver* s, int w) {
  OuterArgs a{};
  a.g = s->g;
  a.w = s->wig[w];
  a.po = s->po;
  a.k02e = s->k02e;
  a.norm = (float)(1.0 / ((double)s->g.npts));
  a.ty = s->lay.ty;
  a.mode3d = s->lay.mode3d;
  a.bpr = (int)s->lay.grid_outer;
  a.fstride = (long long)field_elems(s);
  a.pf = 0;  // K2 measured slower with it
  a.pstd = s->pstd;
  a.wait_clocks = s->wait_clocks;
  return a;
}

template <int RS>
static cudaError_t launch_k1_t(const Solver* s, int w, const float2* in, const float2* src, float2* out,
                              float a_mult) {
  const float2 A = make_float2(0.f, a_mult * (float)(1.0f / s->eps / (float)s->nw));  // 1i/epsilon/Nwiggles
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)(s->lay.grid_inner * s->nrhs));
  cfg.blockDim = dim3(s->lay.th_inner);
  cfg.dynamicSmemBytes = s->lay.smem_inner;
  cfg.stream = s->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = s->lay.mode3d ? s->lay.csize : 1;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_fwd_inner<kEmax, RS>, inner_args(s, w), in, src, A, out,
                            (const DevState*)s->d_state);
}

template <int RS>
static cudaError_t launch_k2_t(const Solver* s, int w) {
  k_outer<kEmax, RS><<<(unsigned)(s->lay.grid_outer * s->nrhs), s->lay.th_outer, s->lay.smem_outer, s->stream>>>(
      outer_args(s, w), s->d_T, s->d_state);
  return cudaGetLastError();
}

template <int RS>
static cudaError_t launch_k3_t(const Solver* s, int w) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)(s->lay.grid_inner * s->nrhs));
  cfg.blockDim = dim3(s->lay.th_inner);
  cfg.dynamicSmemBytes = s->lay.smem_inner;
  cfg.stream = s->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = s->lay.mode3d ? s->lay.csize : 1;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, k_inv_inner<kEmax, RS>, inner_args(s, w), (const float2*)s->d_T, s->d_dE,
                            s->d_E, (const float2*)s->d_gamma, (const DevState*)s->d_state, s->d_partials);
}

static size_t fast_inner_smem(const Solver* s, bool fwd) {
  const FastInner* f = s->lay.fi;
  return f->do_x ? (fwd ? f->smem_fwd : f->smem_inv) : f->smem * (size_t)(s->lay.ncols + 1);
}

static cudaError_t launch_fast_inner(const Solver* s, const void* fn, void** args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)(s->lay.grid_inner * s->nrhs));
  cfg.blockDim = dim3(fast::kThreads);
  cfg.dynamicSmemBytes = fast_inner_smem(s, fn == s->lay.fi->fwd);
  cfg.stream = s->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = s->lay.fi->do_x ? s->lay.fi->c : 1;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelExC(&cfg, fn, args);
}

// A loop kernel that begins with pdl_begin(): launched with programmatic
// stream serialisation, so that it may be scheduled while the kernel before
// it finishes (it waits for that kernel's completion before touching global
// memory); captured into the loop's graph as a programmatic edge.
static cudaError_t launch_pdl(const Solver* s, const void* fn, dim3 grid, dim3 block, void** args, size_t smem) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = s->pdl ? 1 : 0;
  return cudaLaunchKernelExC(&cfg, fn, args);
}

// K1 on explicit buffers: out = inner FFT of (in + a_mult A src) times the
// ramps of wiggle w (A = i/epsilon/Nw, the reference's per-iteration share of
// the source; a_mult = Nw gives the whole source, for the warm start's
// residual probe)
static cudaError_t launch_k1_io(const Solver* s, int w, const float2* in, const float2* src, float2* out,
                                float a_mult = 1.f) {
  if (s->lay.fi) {
    InnerArgs a = inner_args(s, w);
    a.ncols = s->lay.ncols;
    a.pf = s->pf_inner;  // K1 only: its loads come first, so the next wave's columns are worth pulling early
    float2 A = make_float2(0.f, a_mult * (float)(1.0f / s->eps / (float)s->nw));
    const DevState* st = s->d_state;
    void* args[] = {&a, &in, &src, &A, &out, &st};
    return launch_fast_inner(s, s->lay.fi->fwd, args);
  }
  return s->lay.rset == kPow2 ? launch_k1_t<kPow2>(s, w, in, src, out, a_mult)
                              : launch_k1_t<kMixed>(s, w, in, src, out, a_mult);
}
static cudaError_t launch_k1(const Solver* s, int w, bool with_source) {
  return launch_k1_io(s, w, s->d_dE, with_source ? s->d_src : nullptr, s->d_T);
}
// cuTensorMapEncodeTiled through the runtime's driver entry point (no link
// against libcuda)
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
static EncodeTiledFn encode_tiled() {
  static EncodeTiledFn fn = [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess)
      f = nullptr;
    return reinterpret_cast<EncodeTiledFn>(f);
  }();
  return fn;
}

// T of the current batch as a 3-D float tensor {2 Ny, Nx, Nz Nc nrhs}, box
// {2 TY, 1, Nz}: every x coordinate the kernel issues is 2 TY yt floats, a
// multiple of 16 floats (TY >= 8), so each copy starts on a 64-byte boundary.
static cudaError_t ensure_tmap(Solver* s) {
  const TmaPencil* f = s->lay.tp;
  if (s->tmap_base == s->d_T && s->tmap_nrhs == s->nrhs && s->tmap_kernel == f->fn) return cudaSuccess;
  s->tmap_kernel = nullptr;
  s->tma_blocks = 0;
  EncodeTiledFn enc = encode_tiled();
  if (!enc) return cudaErrorNotSupported;
  const Geom& g = s->g;
  const cuuint64_t dims[3] = {(cuuint64_t)2 * g.ny, (cuuint64_t)g.nx, (cuuint64_t)g.nz * g.nc * s->nrhs};
  const cuuint64_t strides[2] = {(cuuint64_t)g.ny * sizeof(float2), (cuuint64_t)g.ny * g.nx * sizeof(float2)};
  const cuuint32_t box[3] = {(cuuint32_t)(2 * f->ty), 1u, (cuuint32_t)f->no};
  const cuuint32_t estr[3] = {1u, 1u, 1u};
  if (enc(&s->tmap_T, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, s->d_T, dims, strides, box, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return cudaErrorInvalidValue;
  s->tmap_base = s->d_T;
  s->tmap_nrhs = s->nrhs;
  s->tmap_kernel = f->fn;
  return cudaSuccess;
}

static cudaError_t launch_k2_tma(const Solver* cs, int w) {
  Solver* s = const_cast<Solver*>(cs);  // the tensor-map cache only
  const TmaPencil* f = s->lay.tp;
  cudaError_t e = ensure_tmap(s);
  if (e != cudaSuccess) return e;
  if (s->tma_blocks <= 0) {
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f->fn, f->threads, f->smem);
    if (e != cudaSuccess) return e;
    s->tma_blocks = std::max(1, per_sm) * kNumSms;
  }
  OuterArgs a = outer_args(s, w);
  int ntiles = s->nrhs * s->g.nx * (s->g.ny / f->ty);
  const unsigned grid = (unsigned)std::min(ntiles, s->tma_blocks);
  const DevState* st = s->d_state;
  int* err = s->d_err;
  void* args[] = {&s->tmap_T, &a, &st, &ntiles, &err};
  return launch_pdl(s, f->fn, dim3(grid), dim3(f->threads), args, f->smem);
}

static cudaError_t launch_k2(const Solver* s, int w) {
  if (s->lay.tp) return launch_k2_tma(s, w);
  if (s->lay.fp) {
    OuterArgs a = outer_args(s, w);
    const FastPencil* f = s->lay.fp;
    const unsigned grid = (unsigned)(s->lay.grid_outer * s->nrhs);
    float2* T = s->d_T;
    const DevState* st = s->d_state;
    void* args[] = {&a, &T, &st};
    return launch_pdl(s, f->fn, dim3(grid), dim3(f->threads), args, f->smem);
  }
  return s->lay.rset == kPow2 ? launch_k2_t<kPow2>(s, w) : launch_k2_t<kMixed>(s, w);
}
static cudaError_t launch_k3_only(const Solver* s, int w) {
  cudaError_t e;
  if (s->lay.fi) {
    InnerArgs a = inner_args(s, w);
    a.ncols = s->lay.ncols;
    const float2* T = s->d_T;
    float2* dE = s->d_dE;
    float2* E = s->d_E;
    const float2* gamma = s->d_gamma;
    const DevState* st = s->d_state;
    double* partials = s->d_partials;
    void* args[] = {&a, &T, &dE, &E, &gamma, &st, &partials};
    e = launch_fast_inner(s, s->lay.fi->inv, args);
  } else {
    e = s->lay.rset == kPow2 ? launch_k3_t<kPow2>(s, w) : launch_k3_t<kMixed>(s, w);
  }
  return e;
}

static cudaError_t launch_finish(const Solver* s, const StopRule& rule, const Hist& h) {
  DevState* st = s->d_state;
  StopRule r = rule;
  Hist hh = h;
  const double* partials = s->d_partials;
  int nparts = (int)s->lay.grid_inner;
  void* args[] = {&st, &r, &hh, &partials, &nparts};
  cudaError_t e0 = launch_pdl(s, (const void*)k_finish_iteration, dim3(s->nrhs), dim3(256), args, 0);
  if (e0 != cudaSuccess) return e0;
  return cudaGetLastError();
}

static cudaError_t launch_k3(const Solver* s, int w, const StopRule& rule, const Hist& h) {
  cudaError_t e = launch_k3_only(s, w);
  if (e != cudaSuccess) return e;
  return launch_finish(s, rule, h);
}

static cudaError_t launch_iteration(const Solver* s, int it0, bool with_source, const StopRule& rule,
                                    const Hist& h);

// K3 of the iteration with wiggle w fused with K1 of the next (wiggle w1,
// with the source when that iteration is one of the first Nw)
// T as a 2-D float tensor {2 Ny, Nx Nz Nc nrhs} (one row per y column), box
// {2 LR, N}: the x coordinate of every copy is 2 LR rank floats (a multiple
// of 128 bytes), the row coordinate rhs Nx Nz Nc + plane Nx >= 0.
static cudaError_t ensure_slab_map(Solver* s) {
  const FastInner* f = s->lay.fi;
  if (s->slab_base == s->d_T && s->slab_nrhs == s->nrhs && s->slab_kernel == f->fused_tma) return cudaSuccess;
  EncodeTiledFn enc = encode_tiled();
  if (!enc) return cudaErrorNotSupported;
  const Geom& g = s->g;
  const int LR = g.ny / f->c;
  const cuuint64_t dims[2] = {(cuuint64_t)2 * g.ny, (cuuint64_t)g.nx * g.nz * g.nc * s->nrhs};
  const cuuint64_t strides[1] = {(cuuint64_t)g.ny * sizeof(float2)};
  const cuuint32_t box[2] = {(cuuint32_t)(2 * LR), (cuuint32_t)g.nx};
  const cuuint32_t estr[2] = {1u, 1u};
  if (enc(&s->tmap_slab, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, s->d_T, dims, strides, box, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return cudaErrorInvalidValue;
  s->slab_base = s->d_T;
  s->slab_nrhs = s->nrhs;
  s->slab_kernel = f->fused_tma;
  return cudaSuccess;
}

static cudaError_t launch_k3k1(const Solver* s, int w, int w1, bool src_next) {
  const bool tma = s->fused_tma && s->lay.fi->fused_tma;
  if (tma) {
    cudaError_t e = ensure_slab_map(const_cast<Solver*>(s));  // the map cache only
    if (e != cudaSuccess) return e;
  }
  InnerArgs a = inner_args(s, w);
  a.ncols = s->lay.ncols;
  Wig W1 = s->wig[w1];
  const float2* src1 = src_next ? s->d_src : nullptr;
  float2 A = make_float2(0.f, (float)(1.0f / s->eps / (float)s->nw));
  float2* T = s->d_T;
  float2* dE = s->d_dE;
  float2* E = s->d_E;
  const float2* gamma = s->d_gamma;
  const DevState* st = s->d_state;
  double* partials = s->d_partials;
  void* args[] = {&a, &W1, &src1, &A, &T, &dE, &E, &gamma, &st, &partials};
  void* args_tma[] = {const_cast<CUtensorMap*>(&s->tmap_slab), &a, &W1, &src1, &A, &T, &dE, &E, &gamma, &st,
                      &partials};
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = dim3((unsigned)(s->lay.grid_inner * s->nrhs));
  cfg.blockDim = dim3(fast::kThreads);
  cfg.dynamicSmemBytes = s->lay.fi->smem_fused;
  cfg.stream = s->stream;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = s->lay.fi->c;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return tma ? cudaLaunchKernelExC(&cfg, s->lay.fi->fused_tma, args_tma)
             : cudaLaunchKernelExC(&cfg, s->lay.fi->fused, args);
}

// T of the current batch as a 3-D float tensor {2 Ny, Nx, Nz Nc nrhs}, box
// {2 TY, Nx, 1}, for the x pencils: every x coordinate the kernel issues is
// 2 TY yt floats (a multiple of 16 floats, TY >= 8), the others 0 and the
// plane index, both >= 0.
static cudaError_t ensure_xmap(Solver* s) {
  const XPencil* f = s->lay.xp;
  if (s->xmap_base == s->d_T && s->xmap_nrhs == s->nrhs && s->xmap_kernel == f->fwd) return cudaSuccess;
  s->xmap_kernel = nullptr;
  s->x_blocks = 0;
  EncodeTiledFn enc = encode_tiled();
  if (!enc) return cudaErrorNotSupported;
  const Geom& g = s->g;
  const cuuint64_t dims[3] = {(cuuint64_t)2 * g.ny, (cuuint64_t)g.nx, (cuuint64_t)g.nz * g.nc * s->nrhs};
  const cuuint64_t strides[2] = {(cuuint64_t)g.ny * sizeof(float2), (cuuint64_t)g.ny * g.nx * sizeof(float2)};
  const cuuint32_t box[3] = {(cuuint32_t)(2 * f->ty), (cuuint32_t)f->no, 1u};
  const cuuint32_t estr[3] = {1u, 1u, 1u};
  if (enc(&s->tmap_X, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, s->d_T, dims, strides, box, estr,
          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
    return cudaErrorInvalidValue;
  s->xmap_base = s->d_T;
  s->xmap_nrhs = s->nrhs;
  s->xmap_kernel = f->fwd;
  return cudaSuccess;
}

// The x transforms of every (y, z) line of T in place: forward or inverse.
static cudaError_t launch_xpencil(const Solver* cs, bool inv) {
  Solver* s = const_cast<Solver*>(cs);  // the tensor-map cache only
  const XPencil* f = s->lay.xp;
  cudaError_t e = ensure_xmap(s);
  if (e != cudaSuccess) return e;
  if (s->x_blocks <= 0) {
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, f->fwd, f->threads, f->smem);
    if (e != cudaSuccess) return e;
    s->x_blocks = std::max(1, per_sm) * kNumSms;
  }
  int ntiles = s->nrhs * s->g.nz * s->g.nc * (s->g.ny / f->ty);
  const unsigned grid = (unsigned)std::min(ntiles, s->x_blocks);
  Geom g = s->g;
  const float2* tw = s->twx;
  const DevState* st = s->d_state;
  long long wc = s->wait_clocks;
  int* err = s->d_err;
  void* args[] = {&s->tmap_X, &g, &tw, &st, &ntiles, &wc, &err};
  return launch_pdl(s, inv ? f->inv : f->fwd, dim3(grid), dim3(f->threads), args, f->smem);
}

// The column pass of the split fused step (kc_col_step): the columns of every
// plane kernel block, no cluster.
// With rule and h, the pass's last block per right-hand side also runs the
// stop rule (finish_in_last_block), in place of k_finish_iteration.
static cudaError_t launch_colstep(const Solver* s, int w, int w1, bool src_next, const StopRule* rule = nullptr,
                                  const Hist* h = nullptr) {
  InnerArgs a = inner_args(s, w);
  a.ncols = s->lay.ncols;
  if (rule && h) {
    a.fin = 1;
    a.rule = *rule;
    a.hist = *h;
  }
  Wig W1 = s->wig[w1];
  const float2* src1 = src_next ? s->d_src : nullptr;
  float2 A = make_float2(0.f, (float)(1.0f / s->eps / (float)s->nw));
  float2* T = s->d_T;
  float2* dE = s->d_dE;
  float2* E = s->d_E;
  const float2* gamma = s->d_gamma;
  const DevState* st = s->d_state;
  double* partials = s->d_partials;
  void* args[] = {&a, &W1, &src1, &A, &T, &dE, &E, &gamma, &st, &partials};
  return launch_pdl(s, s->lay.fi->col_step, dim3((unsigned)(s->lay.grid_inner * s->nrhs)), dim3(fast::kThreads), args,
                    s->lay.fi->smem_col);
}

// K3 of an iteration and K1 of the next: one kernel on a cluster, or the
// split step (inverse x pencils, column pass, forward x pencils).
static cudaError_t launch_step(const Solver* s, int w, int w1, bool src_next, const StopRule* rule = nullptr,
                               const Hist* h = nullptr) {
  if (!s->lay.mode3d) return launch_colstep(s, w, w1, src_next, rule, h);  // 2-D: K2 already transformed along x
  if (!s->lay.xp) return launch_k3k1(s, w, w1, src_next);
  cudaError_t e = launch_xpencil(s, true);
  if (e != cudaSuccess) return e;
  if ((e = launch_colstep(s, w, w1, src_next, rule, h)) != cudaSuccess) return e;
  return launch_xpencil(s, false);
}

// Whether the loop's column pass runs the stop rule itself (2-D, or the
// split step of 3-D planes; WAVESIM_B200_FIN=1).
static bool finish_in_step(const Solver* s) { return s->fin_fuse && (!s->lay.mode3d || s->lay.xp); }

// One iteration of the fused loop: T already holds K1's output for it.
static cudaError_t launch_iteration_fused(const Solver* s, int i, bool src_next, const StopRule& rule,
                                          const Hist& h) {
  const int w = i % s->nw, w1 = (i + 1) % s->nw;
  cudaError_t e = launch_k2(s, w);
  if (e != cudaSuccess) return e;
  if (finish_in_step(s)) return launch_step(s, w, w1, src_next, &rule, &h);
  if ((e = launch_step(s, w, w1, src_next)) != cudaSuccess) return e;
  return launch_finish(s, rule, h);
}

// A steady iteration (no source) of the loop, fused or not.
static cudaError_t launch_steady(const Solver* s, int i, const StopRule& rule, const Hist& h) {
  return s->fuse ? launch_iteration_fused(s, i, false, rule, h) : launch_iteration(s, i, false, rule, h);
}

static cudaError_t launch_iteration(const Solver* s, int it0, bool with_source, const StopRule& rule,
                                    const Hist& h) {
  const int w = it0 % s->nw;
  cudaError_t e = launch_k1(s, w, with_source);
  if (e != cudaSuccess) return e;
  e = launch_k2(s, w);
  if (e != cudaSuccess) return e;
  return launch_k3(s, w, rule, h);
}

// Energy histories: per right-hand side r, diff at r * 2cap and fresh at r * 2cap + cap.
static int ensure_hist(Solver* s, long long cap) {
  if (s->hist_cap >= cap) return WS_OK;
  if (s->d_hist) cudaFree(s->d_hist);
  s->d_hist = nullptr;
  s->hist_cap = 0;
  free_graph(s);  // graphs hold the old pointer
  WS_CUDA(cudaMalloc(&s->d_hist, 2 * cap * std::max(1, s->batch_cap) * sizeof(double)));
  s->hist_cap = cap;
  return WS_OK;
}

// The prologue and first wiggle cycle of a solve (with the source).  Cold:
// the reference's iterations 1..Nw from E' = dE' = 0.  Warm (d_init holds
// v = u/Nw, see k_warm_scale): a cold probe iteration for diff_energy(1),
// the residual probe of the start and the discard check (k_warm_resid_*,
// k_warm_check), the restart from dE' = v, E' = 0, iterations 1..Nw with the
// source and the shift dE' -= v.
static cudaError_t launch_prologue(const Solver* s, const StopRule& rule, const Hist& h) {
  const size_t nbytes = field_elems(s) * s->nrhs * sizeof(float2);
  cudaError_t e;
  if ((e = cudaMemsetAsync(s->d_E, 0, nbytes, s->stream)) != cudaSuccess) return e;
  if ((e = cudaMemsetAsync(s->d_dE, 0, nbytes, s->stream)) != cudaSuccess) return e;
  k_reset_state<<<1, 256, 0, s->stream>>>(s->d_state, s->nrhs);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  if (s->warm) {
    if ((e = launch_iteration(s, 0, true, rule, h)) != cudaSuccess) return e;  // the probe
    const long long n = (long long)field_elems(s) * s->nrhs;
    const unsigned blocks = (unsigned)std::min<long long>((n + 255) / 256, 8 * kNumSms);
    const float nw = (float)s->nw;
    if (s->warm_ratio > 0.0) {
      // residual of the start: one iteration from dE' = u with the whole source
      k_warm_resid_begin<<<blocks, 256, 0, s->stream>>>(s->d_dE, s->d_init, n, nw);
      if ((e = cudaGetLastError()) != cudaSuccess) return e;
      if ((e = launch_k1_io(s, 0, s->d_dE, s->d_src, s->d_T, nw)) != cudaSuccess) return e;
      if ((e = launch_k2(s, 0)) != cudaSuccess) return e;
      if ((e = launch_k3_only(s, 0)) != cudaSuccess) return e;
      const long long fe = (long long)field_elems(s);
      const unsigned bpr = (unsigned)std::max<long long>(1, std::min<long long>((fe + 255) / 256, 4 * kNumSms));
      k_warm_resid_energy<<<dim3(bpr, s->nrhs), 256, 0, s->stream>>>(s->d_dE, s->d_init, s->g, fe, nw,
                                                                     s->d_state);
    }
    k_warm_begin<<<blocks, 256, 0, s->stream>>>(s->d_dE, s->d_E, s->d_init, n);
    k_warm_restart<<<1, 256, 0, s->stream>>>(s->d_state, s->nrhs);
    if (s->warm_ratio > 0.0)
      k_warm_check<<<1, 256, 0, s->stream>>>(s->d_state, s->nrhs, s->warm_ratio, (double)s->nw * s->nw);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (s->fuse) {
    // K1 of the first iteration, then each fused step also computes K1 of the
    // next iteration (with the source while that one is among the first Nw)
    if ((e = launch_k1(s, 0, true)) != cudaSuccess) return e;
    for (int i = 0; i < s->nw; ++i)
      if ((e = launch_iteration_fused(s, i, i + 1 < s->nw, rule, h)) != cudaSuccess) return e;
  } else {
    for (int i = 0; i < s->nw; ++i)
      if ((e = launch_iteration(s, i, true, rule, h)) != cudaSuccess) return e;
  }
  if (s->warm) {
    const long long fe = (long long)field_elems(s);
    const unsigned bpr = (unsigned)std::max<long long>(1, std::min<long long>((fe + 255) / 256, 4 * kNumSms));
    k_warm_shift<<<dim3(bpr, s->nrhs), 256, 0, s->stream>>>(s->d_dE, s->d_init, s->g, fe, s->d_state);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    // the shift changed dE': the fused loop's T is recomputed from it
    if (s->fuse && (e = launch_k1(s, 0, false)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

static int build_graph(Solver* s, const StopRule& rule, const Hist& h) {
  free_graph(s);
  // the stop rule can only end the loop at a multiple of Nw, at the latest at
  // the first multiple >= max_iter: this many cycles always suffice
  const long long max_cycles = (rule.max_iter + s->nw - 1) / s->nw + 1;
  cudaGraph_t graph;
  WS_CUDA(cudaGraphCreate(&graph, 0));
  cudaGraphConditionalHandle cond;
  cudaError_t e = cudaGraphConditionalHandleCreate(&cond, graph, 1, cudaGraphCondAssignDefault);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    return fail(WS_ERR_CUDA, std::string("cudaGraphConditionalHandleCreate: ") + cudaGetErrorString(e));
  }
  // prologue + first cycle (with the source)
  e = cudaStreamBeginCaptureToGraph(s->stream, graph, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    e = launch_prologue(s, rule, h);
    if (e == cudaSuccess) {
      k_cycle_guard<<<1, 32, 0, s->stream>>>(s->d_state, s->nrhs, cond, max_cycles);
      e = cudaGetLastError();
    }
    cudaGraph_t g2 = graph;
    cudaError_t e2 = cudaStreamEndCapture(s->stream, &g2);
    if (e == cudaSuccess) e = e2;
  }
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    return fail(WS_ERR_CUDA, std::string("graph capture (first cycle): ") + cudaGetErrorString(e));
  }
  // sink node of the captured chain
  size_t nn = 0;
  cudaGraphGetNodes(graph, nullptr, &nn);
  std::vector<cudaGraphNode_t> nodes(nn);
  cudaGraphGetNodes(graph, nodes.data(), &nn);
  std::vector<cudaGraphNode_t> sinks;
  for (auto n : nodes) {
    size_t nd = 0;
    cudaGraphNodeGetDependentNodes(n, nullptr, &nd);
    if (nd == 0) sinks.push_back(n);
  }
  cudaGraphNodeParams cp{};
  cp.type = cudaGraphNodeTypeConditional;
  cp.conditional.handle = cond;
  cp.conditional.type = cudaGraphCondTypeWhile;
  cp.conditional.size = 1;
  cudaGraphNode_t cnode;
  e = cudaGraphAddNode(&cnode, graph, sinks.data(), sinks.size(), &cp);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    return fail(WS_ERR_CUDA, std::string("cudaGraphAddNode(while): ") + cudaGetErrorString(e));
  }
  cudaGraph_t body = cp.conditional.phGraph_out[0];
  e = cudaStreamBeginCaptureToGraph(s->stream, body, nullptr, nullptr, 0, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    for (int i = 0; i < s->nw && e == cudaSuccess; ++i) e = launch_steady(s, i, rule, h);
    if (e == cudaSuccess) {
      k_cycle_guard<<<1, 32, 0, s->stream>>>(s->d_state, s->nrhs, cond, max_cycles);
      e = cudaGetLastError();
    }
    cudaGraph_t b2 = body;
    cudaError_t e2 = cudaStreamEndCapture(s->stream, &b2);
    if (e == cudaSuccess) e = e2;
  }
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    return fail(WS_ERR_CUDA, std::string("graph capture (while body): ") + cudaGetErrorString(e));
  }
  e = cudaGraphInstantiate(&s->gexec, graph, 0);
  if (e != cudaSuccess) {
    cudaGraphDestroy(graph);
    s->gexec = nullptr;
    return fail(WS_ERR_CUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(e));
  }
  s->graph = graph;
  return WS_OK;
}

// Source.add_to for every block of every right-hand side into the dense
// source fields (r at r * field elements); source energies into energy[r].
static int upload_sources(Solver* s, int nrhs, const int64_t* counts, const ws_source_block* src, int memory,
                          std::vector<double>& energy) {
  const Geom& g = s->g;
  const size_t F = field_elems(s);
  WS_CUDA(cudaMemsetAsync(s->d_src, 0, F * nrhs * sizeof(float2), s->stream));
  WS_CUDA(cudaMemsetAsync(s->d_energy, 0, nrhs * sizeof(double), s->stream));
  size_t need = 0;
  long long total = 0;
  for (int r = 0; r < nrhs; ++r) total += counts[r];
  for (long long b = 0; b < total; ++b) {
    const ws_source_block& B = src[b];
    size_t n = 1;
    for (int d = 0; d < 4; ++d) {
      const int64_t lim = d == 0 ? g.ny : d == 1 ? g.nx : d == 2 ? g.nz : g.nc;
      if (B.size[d] < 1 || B.position[d] < 1 || B.position[d] + B.size[d] - 1 > lim)
        return fail(WS_ERR_INVALID_ARGUMENT, "source block outside the grid (crop it first, Source.m:81-103)");
      n *= (size_t)B.size[d];
    }
    if (!B.values) return fail(WS_ERR_INVALID_ARGUMENT, "null source values");
    need = std::max(need, n);
  }
  if (need > s->stage_cap && memory != WS_DEVICE) {
    if (s->d_stage) cudaFree(s->d_stage);
    s->d_stage = nullptr;
    s->stage_cap = 0;
    WS_CUDA(cudaMalloc(&s->d_stage, need * sizeof(float2)));
    s->stage_cap = need;
  }
  long long b = 0;
  for (int r = 0; r < nrhs; ++r) {
    for (int64_t k = 0; k < counts[r]; ++k, ++b) {
      const ws_source_block& B = src[b];
      const size_t n = (size_t)(B.size[0] * B.size[1] * B.size[2] * B.size[3]);
      const float2* vals = (const float2*)B.values;
      if (memory != WS_DEVICE) {
        WS_CUDA(cudaMemcpyAsync(s->d_stage, B.values, n * sizeof(float2), cudaMemcpyHostToDevice, s->stream));
        vals = s->d_stage;
      }
      const int th = 256;
      const long long blocks = std::min<long long>((n + th - 1) / th, 4096);
      k_scatter_source<<<(unsigned)std::max(1LL, blocks), th, 0, s->stream>>>(
          s->d_src + F * r, vals, g, (int)B.position[0] - 1, (int)B.position[1] - 1, (int)B.position[2] - 1,
          (int)B.position[3] - 1, (int)B.size[0], (int)B.size[1], (int)B.size[2], (int)B.size[3], s->d_energy + r);
      WS_CUDA(cudaGetLastError());
      if (memory != WS_DEVICE) WS_CUDA(cudaStreamSynchronize(s->stream));  // staging buffer reuse
    }
  }
  energy.assign(nrhs, 0.0);
  WS_CUDA(cudaMemcpyAsync(energy.data(), s->d_energy, nrhs * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  WS_CUDA(cudaStreamSynchronize(s->stream));
  return WS_OK;
}

// One plane-wave block per right-hand side into the dense source fields.
static int generate_plane_waves(Solver* s, int nrhs, const ws_plane_wave* waves, std::vector<double>& energy) {
  const Geom& g = s->g;
  const size_t F = field_elems(s);
  WS_CUDA(cudaMemsetAsync(s->d_src, 0, F * nrhs * sizeof(float2), s->stream));
  WS_CUDA(cudaMemsetAsync(s->d_energy, 0, nrhs * sizeof(double), s->stream));
  for (int r = 0; r < nrhs; ++r) {
    const ws_plane_wave& W = waves[r];
    PlaneWaveArgs a{};
    long long n = 1;
    for (int d = 0; d < 4; ++d) {
      const int64_t lim = d == 0 ? g.ny : d == 1 ? g.nx : d == 2 ? g.nz : g.nc;
      if (W.size[d] < 1 || W.position[d] < 1 || W.position[d] + W.size[d] - 1 > lim)
        return fail(WS_ERR_INVALID_ARGUMENT, "plane-wave block outside the grid (crop it first, Source.m:81-103)");
      a.p[d] = (int)W.position[d] - 1;
      a.sz[d] = (int)W.size[d];
      n *= W.size[d];
    }
    a.amp_re = W.amplitude.re;
    a.amp_im = W.amplitude.im;
    a.phase0 = W.phase0;
    for (int d = 0; d < 3; ++d) a.phase[d] = W.phase[d];
    const long long blocks = std::min<long long>((n + 255) / 256, 4096);
    k_plane_wave_source<<<(unsigned)std::max(1LL, blocks), 256, 0, s->stream>>>(s->d_src + F * r, g, a,
                                                                                s->d_energy + r);
    WS_CUDA(cudaGetLastError());
  }
  energy.assign(nrhs, 0.0);
  WS_CUDA(cudaMemcpyAsync(energy.data(), s->d_energy, nrhs * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  WS_CUDA(cudaStreamSynchronize(s->stream));
  return WS_OK;
}

static size_t roi_elems(const Geom& g) {
  return (size_t)(g.r1[0] - g.r0[0]) * (g.r1[1] - g.r0[1]) * (g.r1[2] - g.r0[2]) * (g.r1[3] - g.r0[3]);
}

// One batch of nrhs right-hand sides on the solver's medium.  Each one follows
// the reference loop and stop rule on its own; a converged one stops working
// while the others continue.
static int solve_batch(Solver* s, int nrhs, const int64_t* counts, const ws_source_block* src, int source_memory,
                       const ws_solve_options* o, ws_complex* E_out, int out_memory, double* diff_out,
                       int64_t diff_cap, int64_t* n_it, int* converged, const ws_plane_wave* waves = nullptr) {
  WS_CUDA(cudaSetDevice(s->device));
  ws_solve_options opt;
  ws_default_options(&opt);
  if (o) opt = *o;
  if (nrhs < 1 || nrhs > 65536) return fail(WS_ERR_INVALID_ARGUMENT, "number of right-hand sides must be in [1, 65536]");
  if (s->n_media > 1 && nrhs != s->n_media)
    return fail(WS_ERR_INVALID_ARGUMENT, "a solver of several media takes one right-hand side per medium");
  if (opt.max_iterations < 1 || opt.max_iterations > 100000000LL)
    return fail(WS_ERR_INVALID_ARGUMENT, "max_iterations must be in [1, 1e8]");
  if (opt.energy_interval < 1) return fail(WS_ERR_INVALID_ARGUMENT, "energy_interval must be >= 1");
  if (!waves) {
    if (!counts || !src) return fail(WS_ERR_NO_SOURCE, "no source blocks");
    for (int r = 0; r < nrhs; ++r)
      if (counts[r] < 1) return fail(WS_ERR_NO_SOURCE, "a right-hand side has no source blocks");
  }
  const bool want_cb = opt.callback && opt.callback_type && std::strcmp(opt.callback_type, "NoCallback") != 0;
  if (want_cb && nrhs > 1) return fail(WS_ERR_INVALID_ARGUMENT, "callbacks need a single right-hand side");
  if (s->lay.grid_inner * (long long)nrhs > (1LL << 31) - 1 || s->lay.grid_outer * (long long)nrhs > (1LL << 31) - 1)
    return fail(WS_ERR_INVALID_ARGUMENT, "batch too large for one launch");
  int rc = ensure_batch(s, nrhs);
  if (rc) return rc;
  rc = ensure_partials(s, s->lay.grid_inner * (long long)nrhs);
  if (rc) return rc;
  if (s->nrhs != nrhs) free_graph(s);
  s->nrhs = nrhs;
  std::vector<double> src_energy;
  rc = waves ? generate_plane_waves(s, nrhs, waves, src_energy)
             : upload_sources(s, nrhs, counts, src, source_memory, src_energy);
  if (rc) return rc;
  for (int r = 0; r < nrhs; ++r)
    if (!(src_energy[r] > 0)) return fail(WS_ERR_NO_SOURCE, "There is no source inside the grid boundaries");
  // the loop can run at most max_iterations + Nw - 1 iterations
  const long long cap = opt.max_iterations + s->nw;
  rc = ensure_hist(s, cap);
  if (rc) return rc;
  StopRule rule{};
  rule.nw = s->nw;
  rule.fresh = opt.stop_rule == WS_STOP_FRESH;
  rule.nan_stop = opt.stop_on_nonfinite ? 1 : 0;
  rule.interval = (int)std::min<int64_t>(opt.energy_interval, 1 << 30);
  rule.max_iter = opt.max_iterations;
  rule.threshold = opt.energy_threshold;
  const long long hs_stride = 2 * s->hist_cap;
  Hist h{s->d_hist, s->d_hist + s->hist_cap, s->hist_cap, hs_stride};
  std::vector<DevState> hs(nrhs);
  s->warm = opt.initial_field != nullptr;
  s->warm_ratio = opt.warm_discard_ratio;
  if (s->warm) {
    const long long fe = (long long)field_elems(s);
    if (!s->d_init) WS_CUDA(cudaMalloc(&s->d_init, fe * s->batch_cap * sizeof(float2)));
    WS_CUDA(cudaMemcpyAsync(s->d_init, opt.initial_field, fe * nrhs * sizeof(float2),
                            opt.initial_memory == WS_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                            s->stream));
    const long long n = fe * nrhs;
    k_warm_scale<<<(unsigned)std::min<long long>((n + 255) / 256, 8 * kNumSms), 256, 0, s->stream>>>(
        s->d_init, s->d_gamma, n, s->g.npts, 1.0f / (float)s->nw, opt.initial_is_eprime ? 1 : 0,
        (long long)field_elems(s), s->n_media > 1 ? (long long)s->g.npts : 0LL);
    WS_CUDA(cudaGetLastError());
  }
  if (opt.use_graph && !want_cb) {
    GraphKey key{rule.threshold, rule.max_iter, rule.interval, opt.stop_rule, rule.nan_stop, nrhs,
                 s->warm ? 1 : 0, s->warm ? s->warm_ratio : 0.0};
    if (!s->gexec || !(key == s->gkey)) {
      rc = build_graph(s, rule, h);
      if (rc) return rc;
      s->gkey = key;
    }
    WS_CUDA(cudaGraphLaunch(s->gexec, s->stream));
  } else {
    std::vector<double> hist;
    long long it = 0;
    const long long cb_int = std::max<int64_t>(1, opt.callback_interval);
    const long long max_cycles = (rule.max_iter + s->nw - 1) / s->nw + 1;
    for (long long cycle = 0;; ++cycle) {
      if (cycle >= max_cycles) return fail(WS_ERR_CUDA, "loop did not stop within max_iterations (internal error)");
      if (cycle == 0) {
        WS_CUDA(launch_prologue(s, rule, h));
        it += s->nw;
      } else {
        for (int i = 0; i < s->nw; ++i) {
          WS_CUDA(launch_steady(s, (int)(it % s->nw), rule, h));
          ++it;
        }
      }
      WS_CUDA(cudaMemcpyAsync(hs.data(), s->d_state, nrhs * sizeof(DevState), cudaMemcpyDeviceToHost, s->stream));
      WS_CUDA(cudaStreamSynchronize(s->stream));
      if (want_cb) {
        const long long done_it = hs[0].it - 1;
        hist.resize(done_it);
        WS_CUDA(cudaMemcpy(hist.data(), s->d_hist, done_it * sizeof(double), cudaMemcpyDeviceToHost));
        for (long long k = done_it - s->nw + 1; k <= done_it; ++k)
          if (k >= 1 && (k % cb_int == 0 || (hs[0].done && k == done_it)))
            opt.callback(opt.callback_type, hist.data(), k, opt.energy_threshold, opt.user_data);
      }
      bool all = true;
      for (const DevState& d : hs) all = all && d.done;
      if (all) break;
    }
  }
  WS_CUDA(cudaMemcpyAsync(hs.data(), s->d_state, nrhs * sizeof(DevState), cudaMemcpyDeviceToHost, s->stream));
  int kerr = 0;
  WS_CUDA(cudaMemcpyAsync(&kerr, s->d_err, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
  WS_CUDA(cudaStreamSynchronize(s->stream));
  if (kerr) {
    cudaMemset(s->d_err, 0, sizeof(int));
    return fail(WS_ERR_CUDA, "a bounded wait of the FFT kernels (cluster exchange or TMA tile load) timed out");
  }
  bool diverged = false;
  for (int r = 0; r < nrhs; ++r) {
    const long long n_iter = hs[r].it - 1;
    if (n_it) n_it[r] = n_iter;
    if (converged) converged[r] = hs[r].converged;
    diverged = diverged || hs[r].status == WS_ERR_DIVERGED;
    if (diff_out && n_iter > 0)
      WS_CUDA(cudaMemcpy(diff_out + r * diff_cap, s->d_hist + r * hs_stride,
                         std::min<long long>(std::min(n_iter, cap), diff_cap) * sizeof(double),
                         cudaMemcpyDeviceToHost));
  }
  if (E_out) {
    const Geom& g = s->g;
    const cudaMemcpyKind k = out_memory == WS_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    const size_t F = field_elems(s);
    if (opt.output == WS_OUTPUT_FIELD) {
      const size_t n = roi_elems(g);
      for (int r = 0; r < nrhs; ++r) {
        float2* dst = (float2*)E_out + n * r;
        if (out_memory != WS_DEVICE) {
          if (n > s->out_cap) {
            if (s->d_out) cudaFree(s->d_out);
            s->d_out = nullptr;
            s->out_cap = 0;
            WS_CUDA(cudaMalloc(&s->d_out, n * sizeof(float2)));
            s->out_cap = n;
          }
          dst = s->d_out;
        }
        const long long blocks = std::min<long long>(((long long)n + 255) / 256, 8 * kNumSms);
        k_finalize<<<(unsigned)blocks, 256, 0, s->stream>>>(
            s->d_E + F * r, s->d_gamma + (s->n_media > 1 ? (long long)r * s->g.npts : 0LL), g, dst);
        WS_CUDA(cudaGetLastError());
        if (out_memory != WS_DEVICE)
          WS_CUDA(cudaMemcpyAsync((float2*)E_out + n * r, s->d_out, n * sizeof(float2), k, s->stream));
        WS_CUDA(cudaStreamSynchronize(s->stream));
      }
    } else {
      WS_CUDA(cudaMemcpyAsync(E_out, s->d_E, F * nrhs * sizeof(float2), k, s->stream));
    }
    WS_CUDA(cudaStreamSynchronize(s->stream));
  }
  if (diverged) return fail(WS_ERR_DIVERGED, "residual energy is not finite");
  return WS_OK;
}

static int solve(Solver* s, int64_t n_blocks, const ws_source_block* src, int source_memory,
                 const ws_solve_options* o, ws_complex* E_out, int out_memory, double* diff_out, int64_t* n_it,
                 int* converged) {
  if (n_blocks < 1 || !src) return fail(WS_ERR_NO_SOURCE, "no source blocks");
  const int64_t counts[1] = {n_blocks};
  const int64_t maxit = o ? o->max_iterations : 100000;
  return solve_batch(s, 1, counts, src, source_memory, o, E_out, out_memory, diff_out, maxit + s->nw, n_it,
                     converged);
}

}  // namespace ws

using namespace ws;

// ws_run_algorithm's solver of the previous call, per device
static constexpr int kRunCacheDevices = 64;
static Solver* g_run_cache[kRunCacheDevices] = {};
static std::mutex g_run_mu;

extern "C" {

void ws_default_options(ws_solve_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->max_iterations = 100000;
  o->energy_threshold = 1e-2;
  o->energy_interval = 8;
  o->stop_rule = WS_STOP_REFERENCE;
  o->output = WS_OUTPUT_EPRIME;
  o->stop_on_nonfinite = 1;
  o->use_graph = 1;
  o->callback_type = "NoCallback";
  o->callback_interval = 50;
}

const char* ws_version(void) { return "wavesim_b200 0.1.0 (sm_100a)"; }

const char* ws_last_error(void) { return g_last_error.c_str(); }

int ws_size_supported(const int64_t N[4]) {
  if (!N || (N[3] != 1 && N[3] != 3)) return 0;
  Geom g{};
  g.ny = (int)N[0];
  g.nx = (int)N[1];
  g.nz = (int)N[2];
  g.nc = (int)N[3];
  for (int d = 0; d < 3; ++d)
    if (N[d] < 1 || !length_supported((int)N[d])) return 0;
  Layout L;
  std::string why;
  return make_layout(g, L, why) == WS_OK;
}

int ws_solver_create(const int64_t N[4], const ws_complex* gamma, int64_t n_wiggles, const ws_wiggle* wiggles,
                     float epsilon, ws_complex k02e, const int64_t roi[8], int memory, int device, ws_solver* out) {
  if (!out) return fail(WS_ERR_INVALID_ARGUMENT, "null output handle");
  *out = nullptr;
  Solver* s = nullptr;
  const int rc = create_solver(N, gamma, n_wiggles, wiggles, epsilon, k02e, roi, memory, device, &s);
  if (rc) return rc;
  *out = reinterpret_cast<ws_solver>(s);
  return WS_OK;
}

int ws_solver_create_media(const int64_t N[4], int64_t n_media, const ws_complex* gammas, int64_t n_wiggles,
                           const ws_wiggle* wiggles, float epsilon, ws_complex k02e, const int64_t roi[8], int memory,
                           int device, ws_solver* out) {
  if (!out) return fail(WS_ERR_INVALID_ARGUMENT, "null output handle");
  *out = nullptr;
  if (n_media < 1 || n_media > 65536) return fail(WS_ERR_INVALID_ARGUMENT, "n_media must be in [1, 65536]");
  if (!gammas) return fail(WS_ERR_INVALID_ARGUMENT, "null gammas");
  Solver* s = nullptr;
  const int rc = create_solver(N, gammas, n_wiggles, wiggles, epsilon, k02e, roi, memory, device, &s);
  if (rc) return rc;
  if (n_media > 1) {
    const size_t bytes = (size_t)s->g.npts * sizeof(float2);
    cudaFree(s->d_gamma);
    s->d_gamma = nullptr;
    cudaError_t e = cudaMalloc(&s->d_gamma, bytes * (size_t)n_media);
    if (e == cudaSuccess)
      e = cudaMemcpy(s->d_gamma, gammas, bytes * (size_t)n_media,
                     memory == WS_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice);
    if (e != cudaSuccess) {
      destroy_solver(s);
      return fail(e == cudaErrorMemoryAllocation ? WS_ERR_OUT_OF_MEMORY : WS_ERR_CUDA,
                  std::string("media gammas: ") + cudaGetErrorString(e));
    }
    s->n_media = (int)n_media;
  }
  *out = reinterpret_cast<ws_solver>(s);
  return WS_OK;
}

int ws_solver_solve(ws_solver h, int64_t n_blocks, const ws_source_block* source, int source_memory,
                    const ws_solve_options* opts, ws_complex* E_out, int out_memory, double* diff_energy_out,
                    int64_t* n_iterations, int* converged) {
  if (!h) return fail(WS_ERR_INVALID_ARGUMENT, "null solver");
  return solve(reinterpret_cast<Solver*>(h), n_blocks, source, source_memory, opts, E_out, out_memory,
               diff_energy_out, n_iterations, converged);
}

int ws_solver_solve_batch(ws_solver h, int64_t n_rhs, const int64_t* block_counts, const ws_source_block* blocks,
                          int source_memory, const ws_solve_options* opts, ws_complex* E_out, int out_memory,
                          double* diff_energy_out, int64_t diff_capacity, int64_t* n_iterations, int* converged) {
  if (!h) return fail(WS_ERR_INVALID_ARGUMENT, "null solver");
  return solve_batch(reinterpret_cast<Solver*>(h), (int)n_rhs, block_counts, blocks, source_memory, opts, E_out,
                     out_memory, diff_energy_out, diff_capacity, n_iterations, converged);
}

int ws_solver_solve_plane_waves(ws_solver h, int64_t n_rhs, const ws_plane_wave* waves, const ws_solve_options* opts,
                                ws_complex* E_out, int out_memory, double* diff_energy_out, int64_t diff_capacity,
                                int64_t* n_iterations, int* converged) {
  if (!h) return fail(WS_ERR_INVALID_ARGUMENT, "null solver");
  if (!waves) return fail(WS_ERR_NO_SOURCE, "no plane waves");
  return solve_batch(reinterpret_cast<Solver*>(h), (int)n_rhs, nullptr, nullptr, WS_HOST, opts, E_out, out_memory,
                     diff_energy_out, diff_capacity, n_iterations, converged, waves);
}

int ws_solver_buffers(ws_solver h, void** E_prime, void** stream) {
  if (!h) return fail(WS_ERR_INVALID_ARGUMENT, "null solver");
  Solver* s = reinterpret_cast<Solver*>(h);
  if (E_prime) *E_prime = s->d_E;
  if (stream) *stream = s->stream;
  return WS_OK;
}

int ws_solver_set_wait_limit(ws_solver h, int64_t clocks) {
  if (!h) return fail(WS_ERR_INVALID_ARGUMENT, "null solver");
  if (clocks < 0) return fail(WS_ERR_INVALID_ARGUMENT, "clocks must be >= 0");
  Solver* s = reinterpret_cast<Solver*>(h);
  if (s->wait_clocks != (long long)clocks) free_graph(s);  // the graph holds the kernels' arguments
  s->wait_clocks = (long long)clocks;
  return WS_OK;
}

int ws_solver_launches_per_iteration(ws_solver h) {
  if (!h) return 0;
  const Solver* s = reinterpret_cast<Solver*>(h);
  // K2, K3 + next K1 (one kernel, or the split step's three), stop rule; or K1, K2, K3, stop rule
  if (!s->fuse) return 4;                                   // K1, K2, K3, the stop rule
  if (s->lay.mode3d && !s->lay.xp) return 3;                // K2, K3K1 on a cluster, the stop rule
  const int step = s->lay.mode3d ? 4 : 2;                   // K2 (+ x pencils), the column pass (+ x pencils)
  return finish_in_step(s) ? step : step + 1;
}

int ws_solver_fused(ws_solver h) {
  if (!h) return 0;
  return reinterpret_cast<Solver*>(h)->fuse ? 1 : 0;
}

int ws_solver_time_fused(ws_solver h, int n_iterations, float* ms_out, double* bytes_out) {
  if (!h || !ms_out || n_iterations < 1) return fail(WS_ERR_INVALID_ARGUMENT, "bad argument");
  Solver* s = reinterpret_cast<Solver*>(h);
  if (!s->fuse) return fail(WS_ERR_UNSUPPORTED, "this solver's loop does not fuse K3 with K1");
  WS_CUDA(cudaSetDevice(s->device));
  const long long cap = n_iterations + 1;
  if (s->hist_cap < cap) {
    const int rc = ensure_hist(s, cap);
    if (rc) return rc;
  }
  StopRule rule{s->nw, 1, 0, 1, (long long)1 << 62, -1.0};
  Hist hh{s->d_hist, s->d_hist + s->hist_cap, 0, 0};  // cap 0: history untouched
  s->nrhs = 1;
  k_resume_state<<<1, 32, 0, s->stream>>>(s->d_state);
  WS_CUDA(launch_k1(s, 0, false));
  float acc = 0.f;
  for (int i = 0; i < n_iterations; ++i) {
    const int w = i % s->nw;
    WS_CUDA(launch_k2(s, w));
    WS_CUDA(cudaEventRecord(s->ev[0], s->stream));
    WS_CUDA(launch_step(s, w, (i + 1) % s->nw, false));
    WS_CUDA(cudaEventRecord(s->ev[1], s->stream));
    WS_CUDA(launch_finish(s, rule, hh));
    WS_CUDA(cudaEventSynchronize(s->ev[1]));
    float t;
    WS_CUDA(cudaEventElapsedTime(&t, s->ev[0], s->ev[1]));
    acc += t;
  }
  *ms_out = acc / n_iterations;
  if (bytes_out) {
    const double n = (double)s->g.npts * s->g.nc;
    // K3's bytes (as ws_solver_time_kernels) plus the write of T for the next
    // iteration; the split step also reads and writes T in each x pass
    *bytes_out = (s->nw % 2 == 0 ? 40.0 : 48.0) * n + 8.0 * (double)s->g.npts + (s->lay.xp ? 32.0 * n : 0.0);
  }
  return WS_OK;
}

int ws_solver_time_split(ws_solver h, int n_iterations, float ms_out[3], double bytes_out[3]) {
  if (!h || !ms_out || n_iterations < 1) return fail(WS_ERR_INVALID_ARGUMENT, "bad argument");
  Solver* s = reinterpret_cast<Solver*>(h);
  if (!s->fuse || !s->lay.xp) return fail(WS_ERR_UNSUPPORTED, "this solver's loop does not run the split step");
  WS_CUDA(cudaSetDevice(s->device));
  const long long cap = n_iterations + 1;
  if (s->hist_cap < cap) {
    const int rc = ensure_hist(s, cap);
    if (rc) return rc;
  }
  StopRule rule{s->nw, 1, 0, 1, (long long)1 << 62, -1.0};
  Hist hh{s->d_hist, s->d_hist + s->hist_cap, 0, 0};  // cap 0: history untouched
  s->nrhs = 1;
  k_resume_state<<<1, 32, 0, s->stream>>>(s->d_state);
  WS_CUDA(launch_k1(s, 0, false));
  float acc[3] = {0, 0, 0};
  for (int i = 0; i < n_iterations; ++i) {
    const int w = i % s->nw;
    WS_CUDA(launch_k2(s, w));
    WS_CUDA(cudaEventRecord(s->ev[0], s->stream));
    WS_CUDA(launch_xpencil(s, true));
    WS_CUDA(cudaEventRecord(s->ev[1], s->stream));
    WS_CUDA(launch_colstep(s, w, (i + 1) % s->nw, false));
    WS_CUDA(cudaEventRecord(s->ev[2], s->stream));
    WS_CUDA(launch_xpencil(s, false));
    WS_CUDA(cudaEventRecord(s->ev[3], s->stream));
    WS_CUDA(launch_finish(s, rule, hh));
    WS_CUDA(cudaEventSynchronize(s->ev[3]));
    float t;
    for (int k = 0; k < 3; ++k) {
      WS_CUDA(cudaEventElapsedTime(&t, s->ev[k], s->ev[k + 1]));
      acc[k] += t;
    }
  }
  for (int k = 0; k < 3; ++k) ms_out[k] = acc[k] / n_iterations;
  if (bytes_out) {
    const double n = (double)s->g.npts * s->g.nc;
    bytes_out[0] = 16.0 * n;  // read T, write T
    // read T, dE, gamma, write dE, T; E' read and written after even iterations only (the mean)
    bytes_out[1] = (s->nw % 2 == 0 ? 40.0 : 48.0) * n + 8.0 * (double)s->g.npts;
    bytes_out[2] = 16.0 * n;
  }
  return WS_OK;
}

int ws_solver_time_kernels(ws_solver h, int n_iterations, float ms_out[3], double bytes_out[3]) {
  if (!h || !ms_out || n_iterations < 1) return fail(WS_ERR_INVALID_ARGUMENT, "bad argument");
  Solver* s = reinterpret_cast<Solver*>(h);
  WS_CUDA(cudaSetDevice(s->device));
  const long long cap = n_iterations + 1;
  if (s->hist_cap < cap) {
    const int rc = ensure_hist(s, cap);
    if (rc) return rc;
  }
  StopRule rule{s->nw, 1, 0, 1, (long long)1 << 62, -1.0};
  Hist hh{s->d_hist, s->d_hist + s->hist_cap, 0, 0};  // cap 0: history untouched
  s->nrhs = 1;  // time the first right-hand side alone
  k_resume_state<<<1, 32, 0, s->stream>>>(s->d_state);
  float acc[3] = {0, 0, 0};
  for (int i = 0; i < n_iterations; ++i) {
    const int w = i % s->nw;
    WS_CUDA(cudaEventRecord(s->ev[0], s->stream));
    WS_CUDA(launch_k1(s, w, false));
    WS_CUDA(cudaEventRecord(s->ev[1], s->stream));
    WS_CUDA(launch_k2(s, w));
    WS_CUDA(cudaEventRecord(s->ev[2], s->stream));
    WS_CUDA(launch_k3_only(s, w));
    WS_CUDA(cudaEventRecord(s->ev[3], s->stream));
    WS_CUDA(launch_finish(s, rule, hh));
    WS_CUDA(cudaEventSynchronize(s->ev[3]));
    float t;
    for (int k = 0; k < 3; ++k) {
      WS_CUDA(cudaEventElapsedTime(&t, s->ev[k], s->ev[k + 1]));
      acc[k] += t;
    }
  }
  for (int k = 0; k < 3; ++k) ms_out[k] = acc[k] / n_iterations;
  if (bytes_out) {
    const double n = (double)s->g.npts * s->g.nc;
    bytes_out[0] = 16.0 * n;                                // read dE, write T
    bytes_out[1] = 16.0 * n;                                // read T, write T
    // read T, dE, gamma, write dE; E read and written every iteration, or
    // every second one when E' takes the increments in pairs (the mean)
    bytes_out[2] = (s->nw % 2 == 0 ? 32.0 : 40.0) * n + 8.0 * (double)s->g.npts;
  }
  return WS_OK;
}

int ws_solver_warm_report(ws_solver h, int64_t rhs, double* cold_first_energy, double* warm_cycle_energy,
                          int* discarded) {
  if (!h) return fail(WS_ERR_INVALID_ARGUMENT, "null solver");
  Solver* s = reinterpret_cast<Solver*>(h);
  if (rhs < 0 || rhs >= s->nrhs) return fail(WS_ERR_INVALID_ARGUMENT, "right-hand side out of range");
  WS_CUDA(cudaSetDevice(s->device));
  DevState st{};
  WS_CUDA(cudaMemcpy(&st, s->d_state + rhs, sizeof(DevState), cudaMemcpyDeviceToHost));
  if (cold_first_energy) *cold_first_energy = st.diff1;
  if (warm_cycle_energy) *warm_cycle_energy = s->warm ? st.warm_e : -1.0;
  if (discarded) *discarded = s->warm ? st.discarded : 0;
  return WS_OK;
}

int ws_solver_warm_residual(ws_solver h, int64_t rhs, double* cold_residual_energy, double* warm_residual_energy) {
  if (!h) return fail(WS_ERR_INVALID_ARGUMENT, "null solver");
  Solver* s = reinterpret_cast<Solver*>(h);
  if (rhs < 0 || rhs >= s->nrhs) return fail(WS_ERR_INVALID_ARGUMENT, "right-hand side out of range");
  WS_CUDA(cudaSetDevice(s->device));
  DevState st{};
  WS_CUDA(cudaMemcpy(&st, s->d_state + rhs, sizeof(DevState), cudaMemcpyDeviceToHost));
  const bool have = s->warm && s->warm_ratio > 0.0;
  if (cold_residual_energy) *cold_residual_energy = have ? (double)s->nw * s->nw * st.diff1 : -1.0;
  if (warm_residual_energy) *warm_residual_energy = have ? st.warm_r : -1.0;
  return WS_OK;
}

// ---------------------------------------------------------------------------
// Autotuner: among the kernel layouts this grid supports (fast power-of-two
// kernels or the generic mixed-radix ones for the inner and the outer pass,
// the generic outer pass's y tile, the 2-D columns per block), keep the
// fastest inner and the fastest outer pass.  Each candidate first runs one
// iteration from a fixed field and must reproduce the current layout's
// increment to 1e-4; only then is it timed.
// ---------------------------------------------------------------------------
}  // extern "C"

namespace ws {
static __global__ void k_fill_pattern(float2* __restrict__ a, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    unsigned h = (unsigned)(i * 2654435761u) ^ (unsigned)(i >> 32) * 2246822519u;
    h ^= h >> 15;
    h *= 2246822519u;
    h ^= h >> 13;
    a[i] = make_float2((float)(h & 0xffff) / 65536.f - 0.5f, (float)(h >> 16) / 65536.f - 0.5f);
  }
}
// out[0] = max |a - b|, out[1] = max |b| (float bits of non-negative values compare as unsigned)
static __global__ void k_max_diff(const float2* __restrict__ a, const float2* __restrict__ b, long long n,
                                  unsigned* __restrict__ out) {
  float d = 0.f, m = 0.f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 u = a[i], v = b[i];
    d = fmaxf(d, fmaxf(fabsf(u.x - v.x), fabsf(u.y - v.y)));
    m = fmaxf(m, fmaxf(fabsf(v.x), fabsf(v.y)));
  }
  if (!(d == d)) d = __int_as_float(0x7f800000);  // NaN counts as a mismatch
  atomicMax(out, __float_as_uint(d));
  atomicMax(out + 1, __float_as_uint(m));
}

// One iteration (wiggle 0, no source) from the fixed pattern; dE' -> out.
// One iteration of the loop as it runs with the solver's current layout
// (the fused step where there is one), from a fixed pattern; the new
// increment dE' into `out`.
static int tune_probe(Solver* s, const StopRule& rule, const Hist& hh, float2* out) {
  const long long n = (long long)field_elems(s);
  const unsigned blocks = (unsigned)std::min<long long>((n + 255) / 256, 8 * kNumSms);
  k_fill_pattern<<<blocks, 256, 0, s->stream>>>(s->d_dE, n);
  k_resume_state<<<1, 32, 0, s->stream>>>(s->d_state);
  WS_CUDA(cudaGetLastError());
  WS_CUDA(launch_k1(s, 0, false));
  WS_CUDA(launch_k2(s, 0));
  if (s->fuse) {
    WS_CUDA(launch_step(s, 0, 1 % s->nw, false));
  } else {
    WS_CUDA(launch_k3_only(s, 0));
  }
  WS_CUDA(launch_finish(s, rule, hh));
  WS_CUDA(cudaMemcpyAsync(out, s->d_dE, n * sizeof(float2), cudaMemcpyDeviceToDevice, s->stream));
  WS_CUDA(cudaStreamSynchronize(s->stream));
  return WS_OK;
}

// Mean device time of the loop's kernels: K1, K2, K3, or (fused) 0, K2 and
// the step.
static int tune_time(Solver* s, const StopRule& rule, const Hist& hh, int iters, float ms[3]) {
  k_resume_state<<<1, 32, 0, s->stream>>>(s->d_state);
  float acc[3] = {0, 0, 0};
  if (s->fuse) {
    WS_CUDA(launch_k1(s, 0, false));
    for (int i = 0; i < iters; ++i) {
      const int w = i % s->nw;
      WS_CUDA(cudaEventRecord(s->ev[0], s->stream));
      WS_CUDA(launch_k2(s, w));
      WS_CUDA(cudaEventRecord(s->ev[1], s->stream));
      WS_CUDA(launch_step(s, w, (i + 1) % s->nw, false));
      WS_CUDA(cudaEventRecord(s->ev[2], s->stream));
      WS_CUDA(launch_finish(s, rule, hh));
      WS_CUDA(cudaEventSynchronize(s->ev[2]));
      float t;
      WS_CUDA(cudaEventElapsedTime(&t, s->ev[0], s->ev[1]));
      acc[1] += t;
      WS_CUDA(cudaEventElapsedTime(&t, s->ev[1], s->ev[2]));
      acc[2] += t;
    }
    for (int k = 0; k < 3; ++k) ms[k] = acc[k] / iters;
    return WS_OK;
  }
  for (int i = 0; i < iters; ++i) {
    const int w = i % s->nw;
    WS_CUDA(cudaEventRecord(s->ev[0], s->stream));
    WS_CUDA(launch_k1(s, w, false));
    WS_CUDA(cudaEventRecord(s->ev[1], s->stream));
    WS_CUDA(launch_k2(s, w));
    WS_CUDA(cudaEventRecord(s->ev[2], s->stream));
    WS_CUDA(launch_k3_only(s, w));
    WS_CUDA(cudaEventRecord(s->ev[3], s->stream));
    WS_CUDA(launch_finish(s, rule, hh));
    WS_CUDA(cudaEventSynchronize(s->ev[3]));
    float t;
    for (int k = 0; k < 3; ++k) {
      WS_CUDA(cudaEventElapsedTime(&t, s->ev[k], s->ev[k + 1]));
      acc[k] += t;
    }
  }
  for (int k = 0; k < 3; ++k) ms[k] = acc[k] / iters;
  return WS_OK;
}
// The generic kernels' plans with radix schedule `sched` (same lengths and
// twiddle tables).
static void apply_sched(Solver* s, int sched) {
  std::vector<float2> none;
  FftPlan* plans[3] = {&s->py, &s->pxl, &s->po};
  for (FftPlan* p : plans) {
    const float2* tw = p->tw;
    if (p->n >= 1) build_plan(p->n, none, *p, sched);
    p->tw = tw;
  }
}

// Makes `c` the solver's layout (kernels, plans, fused loop); false if the
// grid does not allow it.
static bool apply_choice(Solver* s, const LayoutChoice& c) {
  Layout L;
  std::string why;
  if (make_layout(s->g, L, why, c) != WS_OK) return false;
  // the generic 3-D kernels transform x-local lines of Nx / csize points with
  // the plan and twiddles made for the solver's first layout: a layout with
  // another cluster size would run them on lines of another length
  if (L.mode3d && !L.fi && s->g.nx / L.csize != s->pxl.n) return false;
  if (ensure_partials(s, L.grid_inner * std::max(1, s->batch_cap)) != WS_OK) return false;
  s->lay = L;
  apply_sched(s, c.sched);
  update_fuse(s);
  free_graph(s);
  return true;
}
}  // namespace ws

extern "C" {

int ws_solver_autotune(ws_solver h, int n_iterations, int* n_tried, float* ms_before, float* ms_after) {
  if (!h || n_iterations < 1) return fail(WS_ERR_INVALID_ARGUMENT, "bad argument");
  Solver* s = reinterpret_cast<Solver*>(h);
  WS_CUDA(cudaSetDevice(s->device));
  if (s->hist_cap < 2) {
    const int rc = ensure_hist(s, 2);
    if (rc) return rc;
  }
  StopRule rule{s->nw, 1, 0, 1, (long long)1 << 62, -1.0};
  Hist hh{s->d_hist, s->d_hist + s->hist_cap, 0, 0};  // cap 0: history untouched
  s->nrhs = 1;
  free_graph(s);
  const long long n = (long long)field_elems(s);
  float2* ref = nullptr;
  float2* got = nullptr;
  unsigned* dmax = nullptr;
  auto cleanup = [&]() {
    if (ref) cudaFree(ref);
    if (got) cudaFree(got);
    if (dmax) cudaFree(dmax);
  };
  if (cudaMalloc(&ref, n * sizeof(float2)) != cudaSuccess || cudaMalloc(&got, n * sizeof(float2)) != cudaSuccess ||
      cudaMalloc(&dmax, 2 * sizeof(unsigned)) != cudaSuccess) {
    cleanup();
    return fail(WS_ERR_OUT_OF_MEMORY, "autotune: no memory for the probe fields");
  }
  const Layout base = s->lay;
  int rc = tune_probe(s, rule, hh, ref);
  float base_ms[3];
  if (!rc) rc = tune_time(s, rule, hh, n_iterations, base_ms);
  if (rc) {
    cleanup();
    return rc;
  }
  // candidates
  std::vector<LayoutChoice> inner_c, outer_c;
  inner_c.push_back(LayoutChoice{1, 0, 0, 0, 0});
  inner_c.push_back(LayoutChoice{2, 0, 0, 0, 0});
  if (base.mode3d)
    for (int c : {8, 16}) inner_c.push_back(LayoutChoice{1, 0, c, 0, 0});  // fast planes on other cluster sizes
  if (!base.mode3d)
    for (int f : {4, 2, -2})
      inner_c.push_back(LayoutChoice{2, 0, 0, f > 0 ? std::max(1, base.ncols / f) : base.ncols * 2, 0});
  for (int k = 1; k < kNumSchedules; ++k) {  // the generic kernels' radix schedules
    LayoutChoice c{2, 0, 0, 0, 0};
    c.sched = k;
    inner_c.push_back(c);
  }
  if (base.mode3d) {  // the split step's x pencils
    const auto& xt = x_pencil_table();
    for (int i = 0; i < (int)xt.size(); ++i)
      if (xt[i].no == s->g.nx && s->g.ny % xt[i].ty == 0) {
        LayoutChoice c{1, 0, 0, 0, 0};
        c.xp = i + 1;
        inner_c.push_back(c);
      }
  }
  outer_c.push_back(LayoutChoice{0, 1, 0, 0, 0});
  outer_c.push_back(LayoutChoice{0, 1, 0, 0, 8});  // fast pencil with 8 y per block, where one exists
  for (int k : {2, 3}) outer_c.push_back(LayoutChoice{0, 3 + k, 0, 0, 0});
  for (int t : {1, 2, 4, 8, 16}) outer_c.push_back(LayoutChoice{0, 2, 0, 0, t});
  int tried = 0;
  LayoutChoice best_in{}, best_out{};
  float t_in = base_ms[0] + base_ms[2], t_out = base_ms[1];
  const LayoutChoice base_choice = s->tuned;
  auto evaluate = [&](const LayoutChoice& c, float ms[3]) -> bool {
    if (!apply_choice(s, c)) {
      apply_choice(s, base_choice);
      return false;
    }
    bool ok = tune_probe(s, rule, hh, got) == WS_OK;
    if (ok) {
      unsigned hmax[2] = {0, 0};
      cudaMemsetAsync(dmax, 0, 2 * sizeof(unsigned), s->stream);
      k_max_diff<<<(unsigned)std::min<long long>((n + 255) / 256, 8 * kNumSms), 256, 0, s->stream>>>(got, ref, n,
                                                                                                  dmax);
      ok = cudaMemcpyAsync(hmax, dmax, sizeof(hmax), cudaMemcpyDeviceToHost, s->stream) == cudaSuccess &&
           cudaStreamSynchronize(s->stream) == cudaSuccess;
      float d, m;
      std::memcpy(&d, &hmax[0], 4);
      std::memcpy(&m, &hmax[1], 4);
      ok = ok && d <= 1e-4f * m;
    }
    if (ok) ok = tune_time(s, rule, hh, n_iterations, ms) == WS_OK;
    apply_choice(s, base_choice);
    cudaGetLastError();  // a launch refused for a candidate must not leak into later calls
    ++tried;
    return ok;
  };
  for (const LayoutChoice& c : inner_c) {
    float ms[3];
    if (evaluate(c, ms) && ms[0] + ms[2] < 0.97f * t_in) {
      t_in = ms[0] + ms[2];
      best_in = c;
    }
  }
  for (const LayoutChoice& c : outer_c) {
    float ms[3];
    if (evaluate(c, ms) && ms[1] < 0.97f * t_out) {
      t_out = ms[1];
      best_out = c;
    }
  }
  LayoutChoice fin = best_in;
  fin.outer = best_out.outer;
  fin.ty = best_out.ty;
  float fin_ms[3] = {base_ms[0], base_ms[1], base_ms[2]};
  if (!(fin == base_choice)) {
    if (!evaluate(fin, fin_ms)) {
      fin = base_choice;
      std::memcpy(fin_ms, base_ms, sizeof(fin_ms));
    }
  }
  apply_choice(s, fin);
  s->tuned = fin;
  cleanup();
  if (n_tried) *n_tried = tried;
  if (ms_before) *ms_before = base_ms[0] + base_ms[1] + base_ms[2];
  if (ms_after) *ms_after = fin_ms[0] + fin_ms[1] + fin_ms[2];
  return WS_OK;
}

int ws_solver_get_layout(ws_solver h, int32_t choice[7]) {
  if (!h || !choice) return fail(WS_ERR_INVALID_ARGUMENT, "bad argument");
  const LayoutChoice& c = reinterpret_cast<Solver*>(h)->tuned;
  const int32_t v[7] = {c.inner, c.outer, c.csize, c.ncols, c.ty, c.sched, c.xp};
  std::memcpy(choice, v, sizeof(v));
  return WS_OK;
}

int ws_solver_set_layout(ws_solver h, const int32_t choice[7]) {
  if (!h || !choice) return fail(WS_ERR_INVALID_ARGUMENT, "bad argument");
  Solver* s = reinterpret_cast<Solver*>(h);
  LayoutChoice c{choice[0], choice[1], choice[2], choice[3], choice[4]};
  c.sched = choice[5];
  c.xp = choice[6];
  if (c.inner < 0 || c.inner > 2 || c.outer < 0 || c.outer > 9 || c.csize < 0 || c.csize > 16 || c.ncols < 0 ||
      c.ty < 0 || c.sched < 0 || c.sched >= kNumSchedules || c.xp < 0 || c.xp > (int)x_pencil_table().size())
    return fail(WS_ERR_INVALID_ARGUMENT, "layout choice out of range");
  WS_CUDA(cudaSetDevice(s->device));
  if (!apply_choice(s, c)) {
    apply_choice(s, s->tuned);
    return fail(WS_ERR_UNSUPPORTED, "this grid does not take that layout");
  }
  s->tuned = c;
  return WS_OK;
}

int ws_solver_destroy(ws_solver h) {
  destroy_solver(reinterpret_cast<Solver*>(h));
  return WS_OK;
}

int ws_run_algorithm(const int64_t N[4], const ws_complex* gamma, int64_t n_wiggles, const ws_wiggle* wiggles,
                     int64_t n_blocks, const ws_source_block* source, float epsilon, ws_complex k02e,
                     const int64_t roi[8], int64_t max_iterations, double energy_threshold,
                     const char* callback_string, int64_t callback_interval, ws_callback_fn callback,
                     void* user_data, int memory, ws_complex* E_out, double* diff_energy_out,
                     int64_t* n_iterations) {
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= kRunCacheDevices) return fail(WS_ERR_INVALID_ARGUMENT, "device ordinal beyond the call cache");
  std::lock_guard<std::mutex> lock(g_run_mu);
  // the solver of the previous call on this device is reused when the grid
  // and the wiggle count match: only the medium is uploaded again
  Solver*& s = g_run_cache[dev];
  int rc = WS_ERR_INVALID_ARGUMENT;
  if (s && N && s->g.ny == N[0] && s->g.nx == N[1] && s->g.nz == N[2] && s->g.nc == N[3] && s->nw == n_wiggles)
    rc = reload_medium(s, N, gamma, n_wiggles, wiggles, epsilon, k02e, roi, memory);
  if (rc) {
    destroy_solver(s);
    s = nullptr;
    rc = create_solver(N, gamma, n_wiggles, wiggles, epsilon, k02e, roi, memory, dev, &s);
    if (rc) {
      s = nullptr;
      return rc;
    }
  }
  ws_solve_options o;
  ws_default_options(&o);
  o.max_iterations = max_iterations;
  o.energy_threshold = energy_threshold;
  o.callback_type = callback_string ? callback_string : "NoCallback";
  o.callback_interval = callback_interval > 0 ? callback_interval : 50;
  o.energy_interval = std::min<int64_t>(8, o.callback_interval);  // Simulation.m:135
  o.callback = callback;
  o.user_data = user_data;
  rc = solve(s, n_blocks, source, memory, &o, E_out, memory, diff_energy_out, n_iterations, nullptr);
  if (rc && rc != WS_ERR_DIVERGED && rc != WS_ERR_NO_SOURCE && rc != WS_ERR_INVALID_ARGUMENT) {
    destroy_solver(s);  // after a CUDA error start afresh next time
    s = nullptr;
  }
  return rc;
}

void ws_run_algorithm_release(void) {
  std::lock_guard<std::mutex> lock(g_run_mu);
  for (Solver*& s : g_run_cache) {
    destroy_solver(s);
    s = nullptr;
  }
}

}  // extern "C"

// ---------------------------------------------------------------------------
// PSTD (PSTD.m): the reference's pseudo-spectral time-domain comparison
// solver, on the same FFT kernels.  One step (PSTD.m:103-117):
//   Etmp   = ifftn(-(px^2 + py^2 + pz^2) .* fftn(E)) + A(it) S
//   E_next = c2 E + c1 E_prev + c3 Etmp
// runs as K1 (inner FFT of E, unit ramps) -> K2 (outer FFT, Laplacian / N,
// inverse outer FFT, conjugate) -> K1 again (inner FFT of the conjugate, so
// that conj of its output is the inverse inner FFT) -> k_pstd_update (the
// leapfrog, the source, the step energy |E_next - E e^{i(arg A - arg A_prev)}|^2
// on the ROI) -> k_pstd_finish (Simulation.next with can_terminate =
// real(A) > 0.9, energy / |A|^2).  E and E_prev swap buffers every step; the
// source amplitudes A(it) of a chunk of steps come from the host.
// ---------------------------------------------------------------------------
namespace ws {

struct PstdStep {
  Geom g;
  const float2* T2;    // inner FFT of conj(W): conj(T2) = ifftn(k fftn(E))
  const float2* E;
  const float2* Eprev;
  float2* Enext;       // the buffer of Eprev
  const float2* c12;   // (c1, c2) per point
  const float* c3;
  const float2* src;   // dense source field
  const double2* amp;  // amp[k] = A at step it0 - 1 + k
  long long it0;
};

struct PstdRule {
  double threshold;
  long long max_iter;
  int interval;
};

static __global__ void __launch_bounds__(256) k_pstd_update(PstdStep a, const DevState* __restrict__ st,
                                                            double* __restrict__ partials) {
  if (load_done(st)) return;
  const long long k = (long long)__ldcg(&st->it) - a.it0 + 1;
  const double2 A = a.amp[k], Ap = a.amp[k - 1];
  const double dphi = atan2(A.y, A.x) - atan2(Ap.y, Ap.x);
  const float2 ps = make_float2((float)cos(dphi), (float)sin(dphi));
  const float2 Af = make_float2((float)A.x, (float)A.y);
  const Geom& g = a.g;
  float esum = 0.f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < g.npts;
       i += (long long)gridDim.x * blockDim.x) {
    float2 t = a.T2[i];
    t.y = -t.y;
    t = cadd(t, cmul(Af, a.src[i]));  // Source.add_to (Source.m:167-169)
    const float2 c12 = a.c12[i];
    const float c3 = a.c3[i];
    const float2 e = a.E[i], ep = a.Eprev[i];
    const float2 en = make_float2(c12.y * e.x + c12.x * ep.x + c3 * t.x, c12.y * e.y + c12.x * ep.y + c3 * t.y);
    a.Enext[i] = en;
    const int y = (int)(i % g.ny);
    const long long r = i / g.ny;
    const int x = (int)(r % g.nx), z = (int)(r / g.nx);
    if (y >= g.r0[0] && y < g.r1[0] && x >= g.r0[1] && x < g.r1[1] && z >= g.r0[2] && z < g.r1[2]) {
      const float2 d = make_float2(en.x - (e.x * ps.x - e.y * ps.y), en.y - (e.x * ps.y + e.y * ps.x));
      esum = fmaf(d.x, d.x, fmaf(d.y, d.y, esum));
    }
  }
  __shared__ float red[8];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) esum += __shfl_xor_sync(0xffffffffu, esum, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = esum;
  __syncthreads();
  if (threadIdx.x < 32) {
    float v = threadIdx.x < blockDim.x / 32 ? red[threadIdx.x] : 0.f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (threadIdx.x == 0) partials[blockIdx.x] = (double)v;
  }
}

// Simulation.next (Simulation.m:193-217) for PSTD.run_algorithm (PSTD.m:108-124)
static __global__ void k_pstd_finish(DevState* st, const double* __restrict__ partials, int nparts,
                                     const double2* __restrict__ amp, long long it0, PstdRule rule,
                                     double* __restrict__ hist, long long hist_cap) {
  __shared__ double red[32];
  if (load_done(st)) return;
  double e = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) e += partials[i];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = e;
  __syncthreads();
  if (threadIdx.x != 0) return;
  e = 0.0;
  for (int w = 0; w < (int)(blockDim.x + 31) / 32; ++w) e += red[w];
  const int it = st->it;
  const double2 A = amp[it - it0 + 1];
  if (st->calc_energy) st->last_step_energy = e / (A.x * A.x + A.y * A.y);
  const double d = st->last_step_energy;
  if (it - 1 < hist_cap) hist[it - 1] = d;
  if (it == 1) st->diff1 = d;
  const bool can_terminate = A.x > 0.9;  // MATLAB's A > 0.9 compares the real part
  if (can_terminate && d / st->diff1 < rule.threshold) {
    st->done = 1;
    st->converged = 1;
  } else if (can_terminate && it >= rule.max_iter) {
    st->done = 1;
    st->converged = 0;
  }
  st->calc_energy = ((it - 1) % rule.interval) == 0;
  st->it = it + 1;
}

// ROI crop times a phase factor (PSTD.m:126)
static __global__ void k_pstd_output(const float2* __restrict__ E, Geom g, float2 phase, float2* __restrict__ out) {
  const int ry = g.r1[0] - g.r0[0], rx = g.r1[1] - g.r0[1], rz = g.r1[2] - g.r0[2];
  const long long n = (long long)ry * rx * rz;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    long long r = i;
    const int y = (int)(r % ry) + g.r0[0];
    r /= ry;
    const int x = (int)(r % rx) + g.r0[1];
    const int z = (int)(r / rx) + g.r0[2];
    out[i] = cmul(E[y + (long long)g.ny * (x + (long long)g.nx * z)], phase);
  }
}

struct Pstd {
  Solver* s = nullptr;       // layout, twiddles, T, source, state, stream (K2 in Laplacian mode)
  float2* d_Ebuf = nullptr;  // two fields: step it reads E from (it - 1) % 2, writes E_next to it % 2
  float2* d_T2 = nullptr;
  float* d_c3 = nullptr;
  double2* d_amp = nullptr;
  double* d_hist = nullptr;
  long long hist_cap = 0;
  double* d_part = nullptr;
  int nparts = 0;
};

static void pstd_free(Pstd* p) {
  if (!p) return;
  if (p->s) {
    cudaSetDevice(p->s->device);
    void* ptrs[] = {p->d_Ebuf, p->d_T2, p->d_c3, p->d_amp, p->d_hist, p->d_part};
    for (void* q : ptrs)
      if (q) cudaFree(q);
    destroy_solver(p->s);
  }
  delete p;
}

static void pstd_default_amplitude(double ncycle, double* re, double* im, void*) {
  // PSTD.m:130-137
  const double env = 0.5 - 0.5 * std::cos(M_PI * std::min(ncycle / 100.0, 1.0));
  *re = std::cos(-2.0 * M_PI * ncycle) * env;
  *im = std::sin(-2.0 * M_PI * ncycle) * env;
}

constexpr int kPstdChunk = 256;  // steps launched between host checks of the stop flag

}  // namespace ws

extern "C" {

int ws_pstd_create(const int64_t N[3], const float* c1, const float* c2, const float* c3, const float* px,
                   const float* py, const float* pz, const int64_t roi[8], int device, ws_pstd* out) {
  if (!N || !c1 || !c2 || !c3 || !px || !py || !pz || !roi || !out)
    return fail(WS_ERR_INVALID_ARGUMENT, "null argument");
  *out = nullptr;
  const int64_t N4[4] = {N[0], N[1], N[2], 1};
  for (int d = 0; d < 3; ++d)
    if (N[d] < 1) return fail(WS_ERR_INVALID_ARGUMENT, "N must be positive");
  const size_t npts = (size_t)N[0] * N[1] * N[2];
  // the solver's gamma buffer holds (c1, c2); one wiggle with unit ramps and the plain Fourier ranges
  std::vector<float2> c12(npts);
  for (size_t i = 0; i < npts; ++i) c12[i] = make_float2(c1[i], c2[i]);
  std::vector<float2> one((size_t)std::max(N[0], std::max(N[1], N[2])), make_float2(1.f, 0.f));
  ws_wiggle w{px, py, pz, (const ws_complex*)one.data(), (const ws_complex*)one.data(),
              (const ws_complex*)one.data()};
  Pstd* p = new Pstd();
  int rc = create_solver(N4, (const ws_complex*)c12.data(), 1, &w, 1.0f, ws_complex{0.f, 0.f}, roi, WS_HOST, device,
                         &p->s);
  if (rc) {
    delete p;
    return rc;
  }
  Solver* s = p->s;
  s->pstd = 1;
  s->fuse = 0;
  p->nparts = (int)std::min<long long>(((long long)npts + 255) / 256, 8LL * kNumSms);
  cudaError_t e = cudaSuccess;
  if (e == cudaSuccess) e = cudaMalloc(&p->d_Ebuf, 2 * npts * sizeof(float2));
  if (e == cudaSuccess) e = cudaMalloc(&p->d_T2, npts * sizeof(float2));
  if (e == cudaSuccess) e = cudaMalloc(&p->d_c3, npts * sizeof(float));
  if (e == cudaSuccess) e = cudaMalloc(&p->d_amp, (kPstdChunk + 1) * sizeof(double2));
  if (e == cudaSuccess) e = cudaMalloc(&p->d_part, p->nparts * sizeof(double));
  if (e == cudaSuccess) e = cudaMemcpy(p->d_c3, c3, npts * sizeof(float), cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    pstd_free(p);
    return fail(e == cudaErrorMemoryAllocation ? WS_ERR_OUT_OF_MEMORY : WS_ERR_CUDA, cudaGetErrorString(e));
  }
  *out = reinterpret_cast<ws_pstd>(p);
  return WS_OK;
}

void ws_pstd_default_options(ws_pstd_options* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->max_iterations = 100000;
  o->energy_threshold = 1e-2;
  o->energy_interval = 8;
  o->iterations_per_cycle = 1.0;
}

int ws_pstd_run(ws_pstd h, int64_t n_blocks, const ws_source_block* source, int source_memory,
                const ws_pstd_options* opts, ws_complex* E_out, double* diff_energy_out, int64_t diff_capacity,
                int64_t* n_iterations, int* converged) {
  if (!h || !opts || !E_out) return fail(WS_ERR_INVALID_ARGUMENT, "null argument");
  if (opts->max_iterations < 1 || opts->energy_interval < 1 || !(opts->iterations_per_cycle > 0))
    return fail(WS_ERR_INVALID_ARGUMENT, "bad options");
  Pstd* p = reinterpret_cast<Pstd*>(h);
  Solver* s = p->s;
  WS_CUDA(cudaSetDevice(s->device));
  const Geom& g = s->g;
  if (n_blocks < 1 || !source) return fail(WS_ERR_NO_SOURCE, "There is no source inside the grid boundaries");
  std::vector<double> energy;
  int rc = upload_sources(s, 1, &n_blocks, source, source_memory, energy);
  if (rc) return rc;
  if (!(energy[0] > 0)) return fail(WS_ERR_NO_SOURCE, "There is no source inside the grid boundaries");
  const long long cap = std::max<long long>(0, diff_capacity);
  if (cap > p->hist_cap) {
    if (p->d_hist) cudaFree(p->d_hist);
    p->d_hist = nullptr;
    p->hist_cap = 0;
    WS_CUDA(cudaMalloc(&p->d_hist, cap * sizeof(double)));
    p->hist_cap = cap;
  }
  const size_t npts = (size_t)g.npts;
  WS_CUDA(cudaMemsetAsync(p->d_Ebuf, 0, 2 * npts * sizeof(float2), s->stream));
  DevState st0{};
  st0.it = 1;
  st0.calc_energy = 1;
  st0.last_step_energy = INFINITY;
  WS_CUDA(cudaMemcpyAsync(s->d_state, &st0, sizeof(st0), cudaMemcpyHostToDevice, s->stream));
  ws_amplitude_fn amp = opts->amplitude ? opts->amplitude : pstd_default_amplitude;
  const PstdRule rule{opts->energy_threshold, (long long)opts->max_iterations, (int)opts->energy_interval};
  std::vector<double2> hamp(kPstdChunk + 1);
  double2 a_last = make_double2(1.0, 0.0);  // PSTD.m:83: A = 1 before the first step
  long long it0 = 1;
  DevState hst{};
  const unsigned ublocks = (unsigned)p->nparts;
  // Simulation.next stops at max_iterations only on a step that may terminate
  // (real(A) > 0.9), as the reference does; past max_iterations plus a margin
  // of max(1000, 2 iterations_per_cycle) steps the run ends unconverged.
  const long long hard_stop =
      opts->max_iterations + std::max<long long>(1000, (long long)std::ceil(2 * opts->iterations_per_cycle));
  while (true) {
    const long long K = kPstdChunk;
    hamp[0] = a_last;
    for (long long k = 1; k <= K; ++k)
      amp((double)(it0 - 1 + k) / opts->iterations_per_cycle, &hamp[k].x, &hamp[k].y, opts->user_data);
    WS_CUDA(cudaMemcpyAsync(p->d_amp, hamp.data(), (K + 1) * sizeof(double2), cudaMemcpyHostToDevice, s->stream));
    for (long long k = 0; k < K; ++k) {
      const long long it = it0 + k;
      float2* E = p->d_Ebuf + (size_t)((it - 1) & 1) * npts;
      float2* Ep = p->d_Ebuf + (size_t)(it & 1) * npts;
      WS_CUDA(launch_k1_io(s, 0, E, nullptr, s->d_T));
      WS_CUDA(launch_k2(s, 0));
      WS_CUDA(launch_k1_io(s, 0, s->d_T, nullptr, p->d_T2));
      PstdStep a{g, p->d_T2, E, Ep, Ep, (const float2*)s->d_gamma, p->d_c3, s->d_src, p->d_amp, it0};
      k_pstd_update<<<ublocks, 256, 0, s->stream>>>(a, s->d_state, p->d_part);
      WS_CUDA(cudaGetLastError());
      k_pstd_finish<<<1, 256, 0, s->stream>>>(s->d_state, p->d_part, p->nparts, p->d_amp, it0, rule, p->d_hist,
                                              p->hist_cap < cap ? p->hist_cap : cap);
      WS_CUDA(cudaGetLastError());
    }
    WS_CUDA(cudaMemcpyAsync(&hst, s->d_state, sizeof(hst), cudaMemcpyDeviceToHost, s->stream));
    WS_CUDA(cudaStreamSynchronize(s->stream));
    if (hst.done || it0 + K > hard_stop) break;
    a_last = hamp[K];
    it0 += K;
  }
  int kerr = 0;
  WS_CUDA(cudaMemcpy(&kerr, s->d_err, sizeof(int), cudaMemcpyDeviceToHost));
  if (kerr) return fail(WS_ERR_CUDA, "a kernel's bounded wait gave up (cluster exchange or TMA load)");
  const long long last = hst.it - 1;  // the last step run
  double are = 1.0, aim = 0.0;
  amp((double)hst.it / opts->iterations_per_cycle, &are, &aim, opts->user_data);  // PSTD.m:125
  const double ph = -std::atan2(aim, are);
  const float2 phase = make_float2((float)std::cos(ph), (float)std::sin(ph));
  const long long nroi = (long long)(g.r1[0] - g.r0[0]) * (g.r1[1] - g.r0[1]) * (g.r1[2] - g.r0[2]);
  if (s->out_cap < (size_t)nroi) {
    if (s->d_out) cudaFree(s->d_out);
    s->d_out = nullptr;
    s->out_cap = 0;
    WS_CUDA(cudaMalloc(&s->d_out, nroi * sizeof(float2)));
    s->out_cap = nroi;
  }
  k_pstd_output<<<(unsigned)std::min<long long>((nroi + 255) / 256, 8LL * kNumSms), 256, 0, s->stream>>>(
      p->d_Ebuf + (size_t)(last & 1) * npts, g, phase, s->d_out);
  WS_CUDA(cudaGetLastError());
  WS_CUDA(cudaMemcpyAsync(E_out, s->d_out, nroi * sizeof(float2), cudaMemcpyDeviceToHost, s->stream));
  const long long nh = std::min<long long>(last, cap);
  if (diff_energy_out && nh > 0)
    WS_CUDA(cudaMemcpyAsync(diff_energy_out, p->d_hist, nh * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
  WS_CUDA(cudaStreamSynchronize(s->stream));
  if (n_iterations) *n_iterations = last;
  if (converged) *converged = hst.converged;
  return WS_OK;
}

int ws_pstd_destroy(ws_pstd h) {
  pstd_free(reinterpret_cast<Pstd*>(h));
  return WS_OK;
}

}  // extern "C"
