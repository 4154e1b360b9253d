// Fused MBS iteration kernels (sm_100a).
//
// One iteration of WaveSimBase.run_algorithm (WaveSimBase.m:165-189) is three
// passes over HBM.  "inner" dimensions are the ones a thread block (or a
// thread-block cluster) holds completely in shared memory; the "outer"
// dimension is transformed by pencils in the middle pass:
//   3-D grids (Nz > 1): inner = (y, x) planes, outer = z
//   2-D grids (Nz == 1): inner = y columns,   outer = x
//
// K1 k_fwd_inner : dE (+ i/(eps Nw) S in the first Nw iterations, Source.m:167-169)
//                  times the wiggle ramps gx gy gz (f_wiggle.m:5), forward FFT
//                  over the inner dimensions -> T
// K2 k_outer     : forward FFT over the outer dimension, Green's function
//                  (f_g0_scalar.m:6 or f_g0_vector.m:4-8, with the 1/N of
//                  ifftn folded in), inverse FFT over the outer dimension, in place on T
// K3 k_inv_inner : inverse FFT over the inner dimensions, conj ramps
//                  (WaveSim.m:55), f_mix (f_mix.m:3-4), E += dE, the ROI energy
//                  sum(|dE|^2) (Simulation.m:265-273) and, in the last block to
//                  finish, the stop rule of Simulation.next (Simulation.m:193-217).
//
// A 3-D plane that does not fit one block's shared memory is split over a
// cluster of C blocks along x: the x transform is then one radix-C step across
// the cluster through distributed shared memory plus a local transform of
// length Nx/C (forward: X[k1 + C k2] = sum_x' W_{Nx/C}^{x' k2} W_Nx^{k1 x'}
// sum_c x[x' + c Nx/C] W_C^{c k1}; the inverse mirrors it).
#pragma once
#include <cooperative_groups.h>
#include <cuda_runtime.h>
#include <math.h>
#include "ws_fft.cuh"

namespace ws {

namespace cg = cooperative_groups;

constexpr float kAlpha = 0.7f;  // private/f_mix.m:3

struct Geom {
  int ny, nx, nz, nc;
  long long npts;  // ny * nx * nz
  int r0[4], r1[4];  // roi, 0-based, [r0, r1) per (y, x, z, c)
};

struct Wig {
  const float* pxe;
  const float* pye;
  const float* pze;
  const float2* gx;
  const float2* gy;
  const float2* gz;
};

// Device-resident loop state (the fields of the reference's `state`).
struct DevState {
  int it;           // state.it, 1-based
  int done;         // !state.has_next
  int converged;    // state.converged
  int calc_energy;  // state.calculate_energy
  int status;       // 0 or WS_ERR_DIVERGED
  unsigned int blocks_done;
  long long cycles;  // wiggle cycles completed (loop guard)
  double e_acc;             // partial sums of this iteration's ROI energy
  double last_step_energy;  // state.last_step_energy
  double diff1;             // state.diff_energy(1)
  // warm starts (no counterpart in the reference)
  int diff1_locked;         // diff1 comes from the cold probe iteration; iteration 1 keeps it
  int discarded;            // given up at the end of the first wiggle cycle
  double warm_e;            // ROI energy of the true increment dE'_Nw of a warm start
  double warm_r;            // ROI energy of the warm start's initial residual (k_warm_resid_energy)
};

struct StopRule {
  int nw;          // numel(wiggles)
  int fresh;       // 1: WS_STOP_FRESH
  int nan_stop;    // 1: stop when the energy is not finite
  int interval;    // energy_calculation_interval
  long long max_iter;
  double threshold;
};

struct Hist {
  double* diff;   // state.diff_energy
  double* fresh;  // energy of every iteration
  long long cap;
  long long stride;  // distance between the histories of consecutive right-hand sides
};

struct InnerArgs {
  Geom g;
  Wig w;
  FftPlan py;   // length Ny
  FftPlan pxl;  // length Nx / csize (3-D only)
  const float2* twx;  // W_Nx^k table (cluster step)
  int csize;    // blocks per plane (cluster size), 3-D only
  int mode3d;
  int ncols;    // columns per block, 2-D only
  int bpr;      // blocks per right-hand side (a batch of sources runs as consecutive block ranges)
  long long fstride;  // elements between the fields of consecutive right-hand sides
  int pf;       // fast kernels: block b pulls the inputs of block b + pf into L2 (0: off)
  int acc2;     // K3: E' += dE' in pairs, every second iteration (Nw even; 0: every iteration)
  int* err;     // fast kernels: set to 1 when a cluster exchange wait gives up (may be null)
  long long gstride;  // elements between the gammas of consecutive right-hand sides (0: one shared gamma)
  int fin;            // column passes: the last block of a right-hand side runs the stop rule
  StopRule rule;      //   (finish_in_last_block) with this rule and history
  Hist hist;
};

struct OuterArgs {
  Geom g;
  Wig w;
  FftPlan po;   // length of the outer dimension
  float2 k02e;
  float norm;   // 1 / (Ny Nx Nz), the normalisation of ifftn
  int ty;       // consecutive y per block
  int mode3d;
  int bpr;
  long long fstride;
  int pf;       // fast kernels: block b pulls the inputs of block b + pf into L2 (0: off)
  int pstd;     // 1: PSTD Laplacian -(px^2 + py^2 + pz^2) / N instead of the Green's function
                // (k02e = 0), and the output conjugated (scalar fields only)
  long long wait_clocks;  // TMA pencils: clocks a tile load may take before the block gives up
                          // (<= 0: the default bound)
};

__device__ __forceinline__ int load_done(const DevState* st) { return __ldcg(&st->done); }

// Programmatic dependent launch: the loop's kernels are launched so that the
// next one may be scheduled while this one runs; each waits here, before it
// touches global memory, until the kernel before it has completed and its
// writes are visible (a no-op when launched without the attribute), then lets
// the kernel after it be scheduled.
__device__ __forceinline__ void pdl_begin() {
  asm volatile("griddepcontrol.wait;" ::: "memory");
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// One radix-C step across the cluster (C = a.csize > 1), in place on the
// shared tile.  Forward: out[x'] = sum_c u_c[x'] W_Nx^{rank (x' + c M)};
// inverse: out[x'] = sum_c u_c[x'] conj(W_Nx^{c (x' + rank M)}), M = Nx / C.
template <int EMAX, bool INV>
__device__ __forceinline__ void cluster_step(float2* sm, int ny, int LS, int ncol, int C, int rank, int nx,
                                             const float2* __restrict__ twx, int tid, int nthr) {
  cg::cluster_group cl = cg::this_cluster();
  cl.sync();
  float2 acc[EMAX];
  const int m = ncol * ny;
#pragma unroll
  for (int q = 0; q < EMAX; ++q) {
    const int e = tid + q * nthr;
    if (e < m) {
      const int xl = e / ny, y = e - xl * ny;
      const int ad = xl * LS + y + (y >> 4);
      float2 s = make_float2(0.f, 0.f);
      for (int c = 0; c < C; ++c) {
        const float2* rs = cl.map_shared_rank(sm, c);
        const float2 u = rs[ad];
        long long k = INV ? (long long)c * (xl + rank * ncol) : (long long)rank * (xl + c * ncol);
        float2 w = __ldg(&twx[k % nx]);
        if (INV) w.y = -w.y;
        s = cadd(s, cmul(u, w));
      }
      acc[q] = s;
    }
  }
  cl.sync();
#pragma unroll
  for (int q = 0; q < EMAX; ++q) {
    const int e = tid + q * nthr;
    if (e < m) {
      const int xl = e / ny, y = e - xl * ny;
      sm[xl * LS + y + (y >> 4)] = acc[q];
    }
  }
  __syncthreads();
}

// K1 -------------------------------------------------------------------------
template <int EMAX, int RSET>
__global__ void __launch_bounds__(512, 1) k_fwd_inner(InnerArgs a, const float2* __restrict__ dE,
                                                    const float2* __restrict__ src, float2 A,
                                                    float2* __restrict__ T, const DevState* __restrict__ st) {
  const int rhs = blockIdx.x / a.bpr, bid = blockIdx.x - rhs * a.bpr;
  st += rhs;
  if (load_done(st)) return;
  dE += rhs * a.fstride;
  if (src) src += rhs * a.fstride;
  T += rhs * a.fstride;
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x, nthr = blockDim.x;
  const Geom& g = a.g;
  const int ny = g.ny, LS = padded(ny);
  int ncol, plane = 0, rank = 0, x0 = 0, z = 0;
  long long colbase;
  if (a.mode3d) {
    rank = bid % a.csize;
    plane = bid / a.csize;
    ncol = g.nx / a.csize;
    x0 = rank * ncol;
    z = plane % g.nz;
    colbase = (long long)plane * g.nx + x0;
  } else {
    colbase = (long long)bid * a.ncols;
    ncol = (int)min((long long)a.ncols, (long long)g.nx * g.nc - colbase);
  }
  const int m = ncol * ny;
  const float2 gzz = a.w.gz[z];
  for (int e = tid; e < m; e += nthr) {
    const int xl = e / ny, y = e - xl * ny;
    const long long col = colbase + xl;
    const long long gi = col * ny + y;
    float2 v = dE[gi];
    if (src) v = cadd(v, cmul(A, src[gi]));
    const int x = a.mode3d ? x0 + xl : (int)(col % g.nx);
    v = cmul(cmul(cmul(v, a.w.gx[x]), a.w.gy[y]), gzz);
    sm[xl * LS + y + (y >> 4)] = v;
  }
  __syncthreads();
  fft_lines<false, EMAX, RSET>(sm, Lines{ncol, LS, 1}, a.py, tid, nthr);
  if (a.mode3d && g.nx > 1) {
    if (a.csize > 1) cluster_step<EMAX, false>(sm, ny, LS, ncol, a.csize, rank, g.nx, a.twx, tid, nthr);
    fft_lines<false, EMAX, RSET>(sm, Lines{ny, LS, 0}, a.pxl, tid, nthr);
  }
  for (int e = tid; e < m; e += nthr) {
    const int xl = e / ny, y = e - xl * ny;
    long long col;
    if (a.mode3d) {
      const int kx = a.csize > 1 ? rank + a.csize * xl : xl;
      col = (long long)plane * g.nx + kx;
    } else {
      col = colbase + xl;
    }
    T[col * ny + y] = sm[xl * LS + y + (y >> 4)];
  }
}

// K2 -------------------------------------------------------------------------
template <int EMAX, int RSET>
__global__ void __launch_bounds__(512, 1) k_outer(OuterArgs a, float2* __restrict__ T, const DevState* __restrict__ st) {
  const int rhs = blockIdx.x / a.bpr, bid = blockIdx.x - rhs * a.bpr;
  st += rhs;
  if (load_done(st)) return;
  T += rhs * a.fstride;
  extern __shared__ float2 sm[];
  const int tid = threadIdx.x, nthr = blockDim.x;
  const Geom& g = a.g;
  const int ty = a.ty, nc = g.nc;
  const int nyt = (g.ny + ty - 1) / ty;
  const int yt = bid % nyt;
  const int mid = a.mode3d ? bid / nyt : 0;
  const int y0 = yt * ty;
  const int no = a.mode3d ? g.nz : g.nx;
  const long long ps = a.mode3d ? (long long)g.ny * g.nx : (long long)g.ny;
  const long long base = y0 + (long long)g.ny * mid;
  const int L = nc * ty;
  const int RS = padded(L);
  const int m = no * L;
  for (int e = tid; e < m; e += nthr) {
    const int yl = e % ty, r = e / ty;
    const int c = r % nc, o = r / nc;
    const int l = c * ty + yl;
    float2 v = make_float2(0.f, 0.f);
    if (y0 + yl < g.ny) v = T[base + yl + ps * o + g.npts * c];
    sm[o * RS + l + (l >> 4)] = v;
  }
  __syncthreads();
  fft_lines<false, EMAX, RSET>(sm, Lines{L, RS, 0}, a.po, tid, nthr);
  // Green's function in the fully transformed (ky, kx, kz) space
  for (int e = tid; e < no * ty; e += nthr) {
    const int yl = e % ty, o = e / ty;
    const int ky = y0 + yl;
    if (ky >= g.ny) continue;
    const int kx = a.mode3d ? mid : o;
    const int kz = a.mode3d ? o : 0;
    const float px = a.w.pxe[kx], py = a.w.pye[ky], pz = a.w.pze[kz];
    if (nc == 1) {
      // f_g0_scalar: E ./ (px^2 + py^2 + (pz^2 - k02e))
      const float dr = fmaf(px, px, fmaf(py, py, pz * pz)) - a.k02e.x;
      const float di = -a.k02e.y;
      const int ad = o * RS + yl + (yl >> 4);
      if (a.pstd) {
        sm[ad] = make_float2(-dr * a.norm * sm[ad].x, -dr * a.norm * sm[ad].y);  // PSTD.m:68
      } else {
        const float inv = a.norm / fmaf(dr, dr, di * di);
        sm[ad] = cmul(sm[ad], make_float2(dr * inv, -di * inv));
      }
    } else {
      // f_g0_vector: div = (p . E) / k02e; E_i <- (E_i - p_i div) / (|p|^2 - k02e)
      const int l0 = yl, l1 = ty + yl, l2 = 2 * ty + yl;
      const int a0 = o * RS + l0 + (l0 >> 4), a1 = o * RS + l1 + (l1 >> 4), a2 = o * RS + l2 + (l2 >> 4);
      const float2 ex = sm[a0], ey = sm[a1], ez = sm[a2];
      const float2 pe = make_float2(fmaf(px, ex.x, fmaf(py, ey.x, pz * ez.x)), fmaf(px, ex.y, fmaf(py, ey.y, pz * ez.y)));
      const float kk = fmaf(a.k02e.x, a.k02e.x, a.k02e.y * a.k02e.y);
      const float2 div = make_float2((pe.x * a.k02e.x + pe.y * a.k02e.y) / kk, (pe.y * a.k02e.x - pe.x * a.k02e.y) / kk);
      const float dr = fmaf(px, px, fmaf(py, py, pz * pz)) - a.k02e.x;
      const float di = -a.k02e.y;
      const float inv = a.norm / fmaf(dr, dr, di * di);
      const float2 g0 = make_float2(dr * inv, -di * inv);
      sm[a0] = cmul(g0, make_float2(ex.x - px * div.x, ex.y - px * div.y));
      sm[a1] = cmul(g0, make_float2(ey.x - py * div.x, ey.y - py * div.y));
      sm[a2] = cmul(g0, make_float2(ez.x - pz * div.x, ez.y - pz * div.y));
    }
  }
  __syncthreads();
  fft_lines<true, EMAX, RSET>(sm, Lines{L, RS, 0}, a.po, tid, nthr);
  for (int e = tid; e < m; e += nthr) {
    const int yl = e % ty, r = e / ty;
    const int c = r % nc, o = r / nc;
    const int l = c * ty + yl;
    if (y0 + yl < g.ny) {
      float2 v = sm[o * RS + l + (l >> 4)];
      if (a.pstd) v.y = -v.y;
      T[base + yl + ps * o + g.npts * c] = v;
    }
  }
}

// Simulation.next (Simulation.m:193-217), run by one thread after the energy
// of iteration st->it is complete.
__device__ __forceinline__ void finish_iteration(DevState* st, const StopRule& rule, const Hist& h) {
  const double e = st->e_acc;
  st->e_acc = 0.0;
  const int it = st->it;
  if (h.fresh && it - 1 < h.cap) h.fresh[it - 1] = e;
  if (st->calc_energy || rule.fresh) st->last_step_energy = e;
  if (it == 1 && st->diff1_locked) st->last_step_energy = st->diff1;  // warm start: the cold diff_energy(1)
  const double d = st->last_step_energy;
  if (it - 1 < h.cap) h.diff[it - 1] = d;
  if (it == 1) st->diff1 = d;
  const bool can_terminate = (it % rule.nw) == 0;
  if (can_terminate && d / st->diff1 < rule.threshold) {
    st->done = 1;
    st->converged = 1;
  } else if (can_terminate && it >= rule.max_iter) {
    st->done = 1;
    st->converged = 0;
  }
  if (rule.nan_stop && !isfinite(e)) {
    st->done = 1;
    st->converged = 0;
    st->status = 6;  // WS_ERR_DIVERGED
  }
  st->calc_energy = ((it - 1) % rule.interval) == 0;
  st->it = it + 1;
  st->blocks_done = 0;
}

// The stop rule of an iteration run by the last block (of 256 threads) of
// the pass that wrote the iteration's energy partials, instead of a separate
// k_finish_iteration launch: each block counts itself in st->blocks_done
// after its partial is visible; the block that completes the count (all
// others have then finished, and read st->it before it changes) sums the
// partials in k_finish_iteration's order (thread i takes i, i + 256, ...,
// then the same tree) and runs finish_iteration, which clears the count.
// st and partials are those of the block's right-hand side.
__device__ __forceinline__ void finish_in_last_block(DevState* st, const StopRule& rule, Hist h,
                                                    const double* partials, int nparts, int rhs) {
  __shared__ unsigned s_last;
  __shared__ double red[256];
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s_last = atomicAdd(&st->blocks_done, 1u) == (unsigned)(nparts - 1) ? 1u : 0u;
  __syncthreads();
  if (!s_last) return;
  __threadfence();
  h.diff += rhs * h.stride;
  if (h.fresh) h.fresh += rhs * h.stride;
  double acc = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) acc += __ldcg(&partials[i]);
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    st->e_acc = red[0];
    finish_iteration(st, rule, h);
  }
}

// K3 -------------------------------------------------------------------------
template <int EMAX, int RSET>
__global__ void __launch_bounds__(512, 1) k_inv_inner(InnerArgs a, const float2* __restrict__ T, float2* __restrict__ dE,
                                                    float2* __restrict__ E, const float2* __restrict__ gamma,
                                                    const DevState* __restrict__ st, double* __restrict__ partials) {
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
  __shared__ float red[32];
  const int tid = threadIdx.x, nthr = blockDim.x;
  const Geom& g = a.g;
  const int ny = g.ny, LS = padded(ny);
  int ncol, plane = 0, rank = 0, x0 = 0, z = 0, comp = 0;
  long long colbase;
  if (a.mode3d) {
    rank = bid % a.csize;
    plane = bid / a.csize;
    ncol = g.nx / a.csize;
    x0 = rank * ncol;
    z = plane % g.nz;
    comp = plane / g.nz;
    colbase = (long long)plane * g.nx + x0;
  } else {
    colbase = (long long)bid * a.ncols;
    ncol = (int)min((long long)a.ncols, (long long)g.nx * g.nc - colbase);
  }
  const int m = ncol * ny;
  for (int e = tid; e < m; e += nthr) {
    const int xl = e / ny, y = e - xl * ny;
    long long col;
    if (a.mode3d) {
      const int kx = a.csize > 1 ? rank + a.csize * xl : xl;
      col = (long long)plane * g.nx + kx;
    } else {
      col = colbase + xl;
    }
    sm[xl * LS + y + (y >> 4)] = T[col * ny + y];
  }
  __syncthreads();
  if (a.mode3d && g.nx > 1) {
    fft_lines<true, EMAX, RSET>(sm, Lines{ny, LS, 0}, a.pxl, tid, nthr);
    if (a.csize > 1) cluster_step<EMAX, true>(sm, ny, LS, ncol, a.csize, rank, g.nx, a.twx, tid, nthr);
  }
  fft_lines<true, EMAX, RSET>(sm, Lines{ncol, LS, 1}, a.py, tid, nthr);
  const float2 gzz = a.w.gz[z];
  float esum = 0.f;
  for (int e = tid; e < m; e += nthr) {
    const int xl = e / ny, y = e - xl * ny;
    const long long col = colbase + xl;
    const long long gi = col * ny + y;
    int x, c;
    if (a.mode3d) {
      x = x0 + xl;
      c = comp;
    } else {
      x = (int)(col % g.nx);
      c = (int)(col / g.nx);
    }
    // Eprop after the inverse transform and the conjugate ramps (WaveSim.m:53-55)
    const float2 ep = cmul_conj(cmul_conj(cmul_conj(sm[xl * LS + y + (y >> 4)], a.w.gx[x]), a.w.gy[y]), gzz);
    const float2 gm = gamma[gi - (long long)c * g.npts];
    const float2 d0 = dE[gi];
    // f_mix: (1 - a gamma) dE - i a gamma^2 Eprop
    const float2 one_m = make_float2(1.f - kAlpha * gm.x, -kAlpha * gm.y);
    const float2 g2 = cmul(gm, gm);
    const float2 t = cmul(g2, ep);
    const float2 dn = cadd(cmul(one_m, d0), make_float2(kAlpha * t.y, -kAlpha * t.x));
    dE[gi] = dn;
    if (acc_now) {
      const float2 e0 = E[gi];
      E[gi] = cadd(e0, a.acc2 ? cadd(d0, dn) : dn);
    }
    if (y >= g.r0[0] && y < g.r1[0] && x >= g.r0[1] && x < g.r1[1] && z >= g.r0[2] && z < g.r1[2] &&
        c >= g.r0[3] && c < g.r1[3])
      esum = fmaf(dn.x, dn.x, fmaf(dn.y, dn.y, esum));
  }
  // block reduction of the ROI energy into this block's partial sum
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) esum += __shfl_xor_sync(0xffffffffu, esum, o);
  if ((tid & 31) == 0) red[tid >> 5] = esum;
  __syncthreads();
  if (tid < 32) {
    float v = tid < (nthr + 31) / 32 ? red[tid] : 0.f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (tid == 0) partials[bid] = (double)v;
  }
}

// The stop rule after each iteration: sums the per-block ROI energies of K3 in
// a fixed order (so the energy history is reproducible bit for bit) and runs
// Simulation.next (Simulation.m:193-217).  One block.
static __global__ void __launch_bounds__(256) k_finish_iteration(DevState* st, StopRule rule, Hist h,
                                                          const double* __restrict__ partials, int nparts) {
  pdl_begin();
  const int rhs = blockIdx.x;  // one block per right-hand side
  st += rhs;
  partials += (long long)rhs * nparts;
  h.diff += rhs * h.stride;
  if (h.fresh) h.fresh += rhs * h.stride;
  if (load_done(st)) return;
  __shared__ double red[256];
  double acc = 0.0;
  for (int i = threadIdx.x; i < nparts; i += blockDim.x) acc += partials[i];
  red[threadIdx.x] = acc;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if ((int)threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    st->e_acc = red[0];
    finish_iteration(st, rule, h);
  }
}

// Helpers --------------------------------------------------------------------
static __global__ void k_reset_state(DevState* st, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    DevState* s = st + i;
    s->it = 1;
    s->done = 0;
    s->converged = 0;
    s->calc_energy = 1;
    s->status = 0;
    s->blocks_done = 0;
    s->cycles = 0;
    s->e_acc = 0.0;
    s->last_step_energy = __longlong_as_double(0x7ff0000000000000LL);  // inf (Simulation.m:169)
    s->diff1 = 0.0;
    s->diff1_locked = 0;
    s->discarded = 0;
    s->warm_e = 0.0;
    s->warm_r = 0.0;
  }
}

// Warm start from a starting field u = gamma psi0 (no counterpart in the
// reference).  The loop's limit depends on how an increment enters the
// wiggle cycle, so a start is injected the way the reference injects its
// source: spread evenly over the first cycle, u/Nw per iteration.  With
// v = u/Nw that is exactly the cold first cycle run from dE' = v, E' = 0,
// followed by dE' -= v (the Nw extra v's that E' accumulated sum to u).  A
// zero start therefore reproduces the cold loop bit for bit.
//
// v <- gamma .* psi0 / Nw (or E'/Nw when the start is already primed); gamma
// is shared by the components and right-hand sides (npts points each).
static __global__ void k_warm_scale(float2* __restrict__ v, const float2* __restrict__ gamma, long long n,
                                    long long npts, float inv_nw, int primed, long long fe, long long gstride) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float2 u = primed ? v[i] : cmul(v[i], gamma[(i / fe) * gstride + (i % fe) % npts]);
    v[i] = make_float2(u.x * inv_nw, u.y * inv_nw);
  }
}

// After the cold probe iteration (which set diff_energy(1)): dE' <- v, E' <- 0
// and the loop restarts at iteration 1 with diff1 kept.
static __global__ void k_warm_begin(float2* __restrict__ dE, float2* __restrict__ E, const float2* __restrict__ v,
                                    long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    dE[i] = v[i];
    E[i] = make_float2(0.f, 0.f);
  }
}
static __global__ void k_warm_restart(DevState* st, int n) {
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    DevState* s = st + i;
    if (s->status) continue;  // the probe diverged: leave it stopped
    s->it = 1;
    s->done = 0;
    s->converged = 0;
    s->calc_energy = 1;
    s->blocks_done = 0;
    s->e_acc = 0.0;
    s->last_step_energy = __longlong_as_double(0x7ff0000000000000LL);
    s->diff1_locked = 1;
    s->discarded = 0;
    s->warm_e = 0.0;
  }
}

// End of the warm first cycle: dE' -= v (the true increment of iteration
// Nw), and its ROI energy into warm_e of right-hand side blockIdx.y.
static __global__ void __launch_bounds__(256) k_warm_shift(float2* __restrict__ dE, const float2* __restrict__ v,
                                                           Geom g, long long fstride, DevState* st) {
  const int r = blockIdx.y;
  dE += (long long)r * fstride;
  v += (long long)r * fstride;
  float acc = 0.f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < fstride; i += (long long)gridDim.x * blockDim.x) {
    const float2 d = csub(dE[i], v[i]);
    dE[i] = d;
    long long k = i;
    const int y = (int)(k % g.ny); k /= g.ny;
    const int x = (int)(k % g.nx); k /= g.nx;
    const int z = (int)(k % g.nz);
    const int c = (int)(k / g.nz);
    if (y >= g.r0[0] && y < g.r1[0] && x >= g.r0[1] && x < g.r1[1] && z >= g.r0[2] && z < g.r1[2] && c >= g.r0[3] &&
        c < g.r1[3])
      acc = fmaf(d.x, d.x, fmaf(d.y, d.y, acc));
  }
  __shared__ float red[8];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    atomicAdd(&st[r].warm_e, (double)t);
  }
}

// The initial residual of a warm start (no counterpart in the reference).
// With the whole source S (its Nw per-iteration parts A S summed) the loop is
// the Richardson iteration E'_k = T_w(E'_(k-1), Nw A S), T_w(x, s) =
// f_mix(x, G'_w(x + s)); a start u = Nw v has the residual
// r(u) = T_1(u, Nw A S) - u, and the cold start r(0) = Nw T_1(0, A S), Nw
// times the probe iteration's increment, of ROI energy Nw^2 diff_energy(1).
// k_warm_resid_begin sets dE' = u, one iteration with the source scaled by Nw
// follows (K1, K2, K3, no stop rule), and k_warm_resid_energy sums
// |dE' - u|^2 over the ROI into warm_r of right-hand side blockIdx.y.
static __global__ void k_warm_resid_begin(float2* __restrict__ dE, const float2* __restrict__ v, long long n,
                                          float nw) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dE[i] = make_float2(v[i].x * nw, v[i].y * nw);
}

static __global__ void __launch_bounds__(256) k_warm_resid_energy(const float2* __restrict__ dE,
                                                                  const float2* __restrict__ v, Geom g,
                                                                  long long fstride, float nw, DevState* st) {
  const int r = blockIdx.y;
  dE += (long long)r * fstride;
  v += (long long)r * fstride;
  float acc = 0.f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < fstride; i += (long long)gridDim.x * blockDim.x) {
    long long k = i;
    const int y = (int)(k % g.ny); k /= g.ny;
    const int x = (int)(k % g.nx); k /= g.nx;
    const int z = (int)(k % g.nz);
    const int c = (int)(k / g.nz);
    if (y >= g.r0[0] && y < g.r1[0] && x >= g.r0[1] && x < g.r1[1] && z >= g.r0[2] && z < g.r1[2] && c >= g.r0[3] &&
        c < g.r1[3]) {
      const float2 d = make_float2(dE[i].x - nw * v[i].x, dE[i].y - nw * v[i].y);
      acc = fmaf(d.x, d.x, fmaf(d.y, d.y, acc));
    }
  }
  __shared__ float red[8];
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    float t = 0.f;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w];
    atomicAdd(&st[r].warm_r, (double)t);
  }
}

// A warm start whose initial residual is worse than the cold start's (ROI
// energy above ratio x Nw^2 diff_energy(1), with 1e-3 of slack for rounding:
// a zero start has exactly the cold residual) is given up before its first
// cycle: the right-hand side stops unconverged, marked discarded, and the
// caller reruns it cold.  ratio <= 0 keeps every start.
static __global__ void k_warm_check(DevState* st, int n, double ratio, double nw2) {
  for (int r = threadIdx.x; r < n; r += blockDim.x) {
    DevState* d = st + r;
    if (ratio <= 0.0 || d->done) continue;
    if (!(d->warm_r <= ratio * nw2 * d->diff1 * (1.0 + 1e-3))) {
      d->done = 1;
      d->converged = 0;
      d->discarded = 1;
    }
  }
}

// Runs after each wiggle cycle of the graph: continues the device-side while
// loop only if the stop rule has not fired and fewer than max_cycles cycles
// have run, so the loop ends even if the stop logic were never reached.
static __global__ void k_cycle_guard(DevState* st, int n, cudaGraphConditionalHandle cond, long long max_cycles) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    const long long c = ++st->cycles;
    bool any = false;
    for (int i = 0; i < n; ++i) any |= !st[i].done;
    const bool go = any && c < max_cycles;
    if (!go)
      for (int i = 0; i < n; ++i) st[i].done = 1;
    cudaGraphSetConditional(cond, go ? 1u : 0u);
  }
}

static __global__ void k_resume_state(DevState* st) {
  if (threadIdx.x == 0 && blockIdx.x == 0) {
    st->done = 0;
    st->blocks_done = 0;
    st->e_acc = 0.0;
  }
}

// Source.add_to for one block (values at 0-based corner p, size s), into the
// dense source buffer; also accumulates the block energy (Source.m:57-67).
static __global__ void k_scatter_source(float2* __restrict__ dst, const float2* __restrict__ vals, Geom g, int p0, int p1,
                                 int p2, int p3, int s0, int s1, int s2, int s3, double* energy) {
  const long long n = (long long)s0 * s1 * s2 * s3;
  float esum = 0.f;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    long long r = i;
    const int a0 = (int)(r % s0); r /= s0;
    const int a1 = (int)(r % s1); r /= s1;
    const int a2 = (int)(r % s2); r /= s2;
    const int a3 = (int)r;
    const long long gi = (p0 + a0) + (long long)g.ny * ((p1 + a1) + (long long)g.nx * ((p2 + a2) + (long long)g.nz * (p3 + a3)));
    const float2 v = vals[i];
    dst[gi] = cadd(dst[gi], v);
    esum = fmaf(v.x, v.x, fmaf(v.y, v.y, esum));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) esum += __shfl_xor_sync(0xffffffffu, esum, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(energy, (double)esum);
}

// A plane-wave source block generated on the device: value(a) = amp exp(i
// (phase0 + sum_d phase[d] a_d)) over the block at 0-based corner p, size sz
// (no counterpart in the reference, whose sources are dense arrays).
struct PlaneWaveArgs {
  int p[4], sz[4];
  double amp_re, amp_im, phase0, phase[3];
};
static __global__ void k_plane_wave_source(float2* __restrict__ dst, Geom g, PlaneWaveArgs w, double* energy) {
  const long long n = (long long)w.sz[0] * w.sz[1] * w.sz[2] * w.sz[3];
  double esum = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    long long r = i;
    const int a0 = (int)(r % w.sz[0]); r /= w.sz[0];
    const int a1 = (int)(r % w.sz[1]); r /= w.sz[1];
    const int a2 = (int)(r % w.sz[2]); r /= w.sz[2];
    const int a3 = (int)r;
    const long long gi = (w.p[0] + a0) +
                         (long long)g.ny * ((w.p[1] + a1) + (long long)g.nx * ((w.p[2] + a2) + (long long)g.nz * (w.p[3] + a3)));
    double sp, cp;
    sincos(w.phase0 + w.phase[0] * a0 + w.phase[1] * a1 + w.phase[2] * a2, &sp, &cp);
    const float2 v = make_float2((float)(w.amp_re * cp - w.amp_im * sp), (float)(w.amp_re * sp + w.amp_im * cp));
    dst[gi] = cadd(dst[gi], v);
    esum += (double)v.x * v.x + (double)v.y * v.y;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) esum += __shfl_xor_sync(0xffffffffu, esum, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(energy, esum);
}

// E = E' ./ gamma on the roi (WaveSimBase.m:193,196), column-major output.
static __global__ void k_finalize(const float2* __restrict__ Ep, const float2* __restrict__ gamma, Geom g,
                           float2* __restrict__ out) {
  const int ry = g.r1[0] - g.r0[0], rx = g.r1[1] - g.r0[1], rz = g.r1[2] - g.r0[2], rc = g.r1[3] - g.r0[3];
  const long long n = (long long)ry * rx * rz * rc;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    long long r = i;
    const int y = (int)(r % ry) + g.r0[0]; r /= ry;
    const int x = (int)(r % rx) + g.r0[1]; r /= rx;
    const int z = (int)(r % rz) + g.r0[2]; r /= rz;
    const int c = (int)r + g.r0[3];
    const long long gi0 = y + (long long)g.ny * (x + (long long)g.nx * z);
    const float2 e = Ep[gi0 + (long long)c * g.npts];
    const float2 d = gamma[gi0];
    const float dd = fmaf(d.x, d.x, d.y * d.y);
    out[i] = make_float2((e.x * d.x + e.y * d.y) / dd, (e.y * d.x - e.x * d.y) / dd);
  }
}

}  // namespace ws
