/*
 * wavesim_b200 - C ABI of the B200 modified Born series (MBS) iteration loop.
 *
 * This library replaces the iteration loop of IvoVellekoop/wavesim
 * (WaveSimBase.run_algorithm, WaveSimBase.m:157-197, and its native
 * counterpart RunWaveSimAlgorithmMex, called at WaveSimBase.m:145-146) with
 * hand-written sm_100a CUDA kernels.  Everything the MATLAB side computes
 * before the loop (gamma, wiggle descriptors, epsilon, k02e, roi, the cropped
 * source) is passed in unchanged; everything it does after the loop
 * (E ./ gamma and the ROI crop, WaveSimBase.m:150-153) is done by the caller,
 * or by the library on request (WS_OUTPUT_FIELD).
 *
 * Memory layout: every array is MATLAB's column-major layout.  A field of
 * size N = [Ny, Nx, Nz, Nc] has element (y, x, z, c) (0-based) at
 * y + Ny*(x + Nx*(z + Nz*c)); complex values are interleaved (re, im) single
 * precision, as in a complex single gpuArray.
 *
 * Errors: functions return a ws_status; ws_last_error() gives a message for
 * the calling thread.  No C++ exception crosses this interface.
 * Threading: a ws_solver owns one CUDA stream and is not thread safe; distinct
 * solvers may be used from distinct threads.
 */
#ifndef WAVESIM_B200_H
#define WAVESIM_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum ws_status {
  WS_OK = 0,
  WS_ERR_INVALID_ARGUMENT = 1, /* bad size, pointer, roi, option */
  WS_ERR_UNSUPPORTED = 2,      /* grid size the FFT kernels do not handle */
  WS_ERR_CUDA = 3,             /* a CUDA runtime call failed */
  WS_ERR_OUT_OF_MEMORY = 4,
  WS_ERR_NO_SOURCE = 5,        /* no source energy inside the grid (Simulation.m:157-161) */
  WS_ERR_DIVERGED = 6,         /* residual energy became NaN or Inf */
  WS_ERR_NO_DEVICE = 7
} ws_status;

/* Where a pointer argument lives. */
enum { WS_HOST = 0, WS_DEVICE = 1 };

/* Stop rules.
 * WS_STOP_REFERENCE: Simulation.next (Simulation.m:193-217) exactly: the
 *   energy is refreshed at iterations 1, 2, 2+k*interval, the ratio to the
 *   first energy is tested only when it % Nwiggles == 0.
 * WS_STOP_FRESH: the same test at the same iterations, but with the energy of
 *   the current iteration (computed by every fused iteration at no cost). */
enum { WS_STOP_REFERENCE = 0, WS_STOP_FRESH = 1 };

/* What ws_solver_solve writes to E_out.
 * WS_OUTPUT_EPRIME: the full-grid accumulated field E' (what
 *   RunWaveSimAlgorithmMex returns; the caller divides by gamma and crops).
 * WS_OUTPUT_FIELD: E = E' ./ gamma cropped to the roi (Simulation.m:254-261),
 *   size (y1-y0+1)*(x1-x0+1)*(z1-z0+1)*(c1-c0+1). */
enum { WS_OUTPUT_EPRIME = 0, WS_OUTPUT_FIELD = 1 };

typedef struct ws_complex {
  float re;
  float im;
} ws_complex;

/* One wiggle descriptor (WaveSimBase.m:300-316): shifted Fourier coordinates
 * pre-divided by sqrt(epsilon) and the real-space phase ramps.
 * Lengths: pxe, gx: Nx; pye, gy: Ny; pze, gz: Nz. */
typedef struct ws_wiggle {
  const float* pxe;
  const float* pye;
  const float* pze;
  const ws_complex* gx;
  const ws_complex* gy;
  const ws_complex* gz;
} ws_wiggle;

/* One block of a Source object (Source.m:18-21) after Simulation.exec has
 * shifted and cropped it to the grid (Simulation.m:154-156): 1-based corner
 * position (y, x, z, polarization) in grid coordinates and the block size;
 * values are column-major. */
typedef struct ws_source_block {
  int64_t position[4];
  int64_t size[4];
  const ws_complex* values;
} ws_source_block;

/* Progress callback, the counterpart of SimulationCallback.m:1
 * (callbackType, diff_energy, ..., energy_threshold).  Called on the host
 * every callback_interval iterations and once at the end. */
typedef void (*ws_callback_fn)(const char* callback_type, const double* diff_energy, int64_t n_iterations,
                               double energy_threshold, void* user_data);

/* A plane-wave source block (no counterpart in the reference, whose sources
 * are dense arrays): value(a) = amplitude * exp(i (phase0 + phase[0] a_y +
 * phase[1] a_x + phase[2] a_z)) over the block at the 1-based grid corner
 * `position` (after the shift and crop of Simulation.exec), a the 0-based
 * offset within the block.  Generated on the device. */
typedef struct ws_plane_wave {
  int64_t position[4];
  int64_t size[4];
  ws_complex amplitude;
  double phase[3];
  double phase0;
} ws_plane_wave;

typedef struct ws_solve_options {
  int64_t max_iterations;        /* >= 1; the MEX call uses max_iterations or 100000 (WaveSimBase.m:127-131) */
  double energy_threshold;       /* Simulation.energy_threshold (Simulation.m:53) */
  int64_t energy_interval;       /* Simulation.energy_calculation_interval (default 8, Simulation.m:61,135) */
  int stop_rule;                 /* WS_STOP_REFERENCE or WS_STOP_FRESH */
  int output;                    /* WS_OUTPUT_EPRIME or WS_OUTPUT_FIELD */
  int stop_on_nonfinite;         /* 1: stop with WS_ERR_DIVERGED when the energy is NaN/Inf */
  int use_graph;                 /* 1: run the loop as one CUDA graph with a device-side while node */
  const char* callback_type;     /* "NoCallback" (default when NULL), "EnergyAdded", "EnergyAddedDisp", ... */
  int64_t callback_interval;     /* Simulation.callback_interval (default 50) */
  ws_callback_fn callback;       /* may be NULL */
  void* user_data;
  /* Warm start (no counterpart in the reference).  NULL: the reference's
   * cold start from zero.  Else one full-grid starting field per right-hand
   * side (Ny*Nx*Nz*Nc complex, column-major) in initial_memory: the field
   * psi0 itself, or E' = gamma .* psi0 when initial_is_eprime is 1 (e.g. the
   * E' output of an earlier solve).  The start enters the loop the way the
   * reference's source does, spread evenly over the first wiggle cycle
   * (u/Nw per iteration, u = gamma psi0); a zero start reproduces the cold
   * loop exactly.  One extra probe iteration, the cold first iteration, runs
   * first: its energy stays diff_energy(1), the stop rule's denominator.
   * diff_energy(2..Nw) are energies of the shifted increments dE' + u/Nw. */
  const ws_complex* initial_field;
  int initial_memory;            /* WS_HOST or WS_DEVICE */
  int initial_is_eprime;
  /* A warm start whose initial residual is worse than the cold start's is
   * given up before its first wiggle cycle: unconverged and marked discarded
   * (ws_solver_warm_report), to be rerun cold.  The residual of a start u
   * (E' variables) is r(u) = T(u, S) - u, T one reference iteration with the
   * first wiggle and the whole source, so r(0) is the cold start's; the test
   * is ROI energy |r(u)|^2 > warm_discard_ratio x |r(0)|^2 (1e-3 relative
   * slack for rounding).  It costs one iteration.  1.0 is the plain rule,
   * 0 keeps every start. */
  double warm_discard_ratio;
} ws_solve_options;

typedef struct ws_solver_s* ws_solver;

/* Fill opts with the reference defaults. */
void ws_default_options(ws_solve_options* opts);

/* Library version string. */
const char* ws_version(void);

/* Message of the last failed call on this thread ("" if none). */
const char* ws_last_error(void);

/* 1 if a grid of this size is supported by the FFT kernels. */
int ws_size_supported(const int64_t N[4]);

/*
 * ws_run_algorithm - one solve, the argument list of RunWaveSimAlgorithmMex
 * (WaveSimBase.m:145-146):
 *   [E, diff_energy] = RunWaveSimAlgorithmMex(N, gamma, Nwiggles, wiggles, source,
 *       epsilon, k02e, roi, maxIter, energy_threshold, callbackString, callback_interval)
 * N      : [Ny, Nx, Nz, Nc] (Nc = 1 scalar, 3 vector)
 * gamma  : Ny*Nx*Nz complex (shared by the Nc components)
 * roi    : MATLAB's 2x4 roi matrix in column-major order
 *          {y0, y1, x0, x1, z0, z1, c0, c1}, 1-based inclusive
 * memory : WS_HOST or WS_DEVICE for every array argument (gamma, wiggles,
 *          source values, E_out)
 * E_out  : Ny*Nx*Nz*Nc complex, receives E' (the caller divides by gamma)
 * diff_energy_out : capacity >= max_iterations + Nwiggles doubles (the loop
 *          stops at the first multiple of Nwiggles >= max_iterations);
 *          receives the per-iteration energy history; *n_iterations its length.
 * callback / user_data: may be NULL.
 * The device buffers of a call are kept (one set per device) and reused by
 * the next call on the same grid with the same wiggle count, which then
 * uploads only the medium; ws_run_algorithm_release frees them.
 */
int ws_run_algorithm(const int64_t N[4], const ws_complex* gamma, int64_t n_wiggles, const ws_wiggle* wiggles,
                     int64_t n_blocks, const ws_source_block* source, float epsilon, ws_complex k02e,
                     const int64_t roi[8], int64_t max_iterations, double energy_threshold,
                     const char* callback_string, int64_t callback_interval, ws_callback_fn callback,
                     void* user_data, int memory, ws_complex* E_out, double* diff_energy_out,
                     int64_t* n_iterations);

/* Frees the device buffers ws_run_algorithm keeps between calls. */
void ws_run_algorithm_release(void);

/* ws_solver_create - uploads (or references, for WS_DEVICE) the medium and
 * wiggle data once, plans the FFTs and allocates the iteration buffers, so
 * that repeated solves on one medium (sources, angles) pay set-up once.
 * Same meaning of arguments as ws_run_algorithm.  device: CUDA ordinal. */
int ws_solver_create(const int64_t N[4], const ws_complex* gamma, int64_t n_wiggles, const ws_wiggle* wiggles,
                     float epsilon, ws_complex k02e, const int64_t roi[8], int memory, int device,
                     ws_solver* out);

/* ws_solver_create_media - a solver for n_media media of one grid: gammas
 * holds n_media gamma arrays of Ny*Nx*Nz elements back to back (in
 * `memory`); everything else - wiggles, epsilon, k02e, roi - is shared, as it
 * is for media of one size whose refractive indices span the same range
 * (epsilon and k0c depend only on the extremes of n^2).  It is solved with
 * ws_solver_solve_batch, one right-hand side per medium (right-hand side r
 * on medium r), so every kernel launch covers all the media.  No counterpart
 * in the reference, whose callers run exec once per medium. */
int ws_solver_create_media(const int64_t N[4], int64_t n_media, const ws_complex* gammas, int64_t n_wiggles,
                           const ws_wiggle* wiggles, float epsilon, ws_complex k02e, const int64_t roi[8],
                           int memory, int device, ws_solver* out);

/* ws_solver_solve - runs the loop for one source.  source values live in
 * source_memory; E_out in out_memory.  diff_energy_out (host) may be NULL.
 * converged (may be NULL) receives 1 if the energy test stopped the loop. */
int ws_solver_solve(ws_solver s, int64_t n_blocks, const ws_source_block* source, int source_memory,
                    const ws_solve_options* opts, ws_complex* E_out, int out_memory, double* diff_energy_out,
                    int64_t* n_iterations, int* converged);

/* ws_solver_solve_batch - n_rhs right-hand sides (sources) on the solver's
 * medium in one set of launches: the blocks of right-hand side r are the
 * block_counts[r] entries that follow those of r-1 in `blocks`.  Each one runs
 * the reference loop with its own stop rule; one that has converged stops
 * working while the others go on.  Outputs are consecutive per right-hand
 * side: E_out (n_rhs fields, E' or the roi field per opts->output),
 * diff_energy_out (host, may be NULL: n_rhs x diff_capacity doubles),
 * n_iterations and converged (n_rhs entries each, may be NULL).  The batch
 * form of ws_solver_solve; no counterpart in the reference, whose callers run
 * exec once per source (e.g. examples/pulse2d.m:31-40).  Callbacks are not
 * supported for n_rhs > 1. */
int ws_solver_solve_batch(ws_solver s, int64_t n_rhs, const int64_t* block_counts, const ws_source_block* blocks,
                          int source_memory, const ws_solve_options* opts, ws_complex* E_out, int out_memory,
                          double* diff_energy_out, int64_t diff_capacity, int64_t* n_iterations, int* converged);

/* ws_solver_solve_batch with one plane-wave block per right-hand side
 * (waves[n_rhs]), generated on the device instead of uploaded: angle sweeps
 * on one medium (e.g. examples/pulse2d.m:31-40). */
int ws_solver_solve_plane_waves(ws_solver s, int64_t n_rhs, const ws_plane_wave* waves,
                                const ws_solve_options* opts, ws_complex* E_out, int out_memory,
                                double* diff_energy_out, int64_t diff_capacity, int64_t* n_iterations,
                                int* converged);

/* Device pointer of the solver's current E' buffer and the CUDA stream it
 * works on (both valid until ws_solver_destroy). */
int ws_solver_buffers(ws_solver s, void** E_prime, void** stream);

/* ws_solver_time_kernels - runs n_iterations further iterations on the
 * current state, one kernel launch at a time, and returns the mean device
 * time of each fused kernel in ms (CUDA events on the solver's stream):
 * ms_out[0] forward inner (wiggle + source + inner FFT),
 * ms_out[1] outer (FFT, Green's function, inverse FFT),
 * ms_out[2] inverse inner (inverse FFT, unwiggle, mix, accumulate, energy).
 * bytes_out[3] (may be NULL): algorithmic bytes each launch moves (for the
 * inverse inner kernel the mean of an odd and an even iteration: with an
 * even number of wiggles E' takes the increments in pairs, after even
 * iterations only, and every stop of the loop falls after an even one). */
int ws_solver_time_kernels(ws_solver s, int n_iterations, float ms_out[3], double bytes_out[3]);

/* Bound of the waits of the TMA-pipelined outer pass (K2 of 3-D grids): a
 * block whose tile load has not arrived after `clocks` SM clocks gives up,
 * waits for its copies still in flight (with the default bound), and the
 * solve returns WS_ERR_CUDA ("timed out") instead of hanging.  0 restores the
 * default (5e7 clocks, ~25 ms).  A very small bound makes the waits run out
 * on purpose: the failure path can be tested without a GPU fault.  No
 * counterpart in the reference. */
int ws_solver_set_wait_limit(ws_solver s, int64_t clocks);

/* Number of kernel launches one iteration makes. */
int ws_solver_launches_per_iteration(ws_solver s);

/* 1 if the solver's loop fuses K3 of an iteration with K1 of the next (the
 * one-kernel step on a cluster, the split step of 3-D planes, the column
 * pass of 2-D grids), 0 if it runs K1, K2 and K3 as separate kernels.  No
 * counterpart in the reference. */
int ws_solver_fused(ws_solver s);

/* Where the loop fuses K3 of an iteration with K1 of the next (3-D fast
 * planes on a cluster), the mean CUDA-event time of that kernel and its
 * algorithmic bytes per launch (K3's plus the write of T); otherwise
 * WS_ERR_UNSUPPORTED. */
int ws_solver_time_fused(ws_solver s, int n_iterations, float* ms_out, double* bytes_out);

/* Where the loop runs K3 of an iteration and K1 of the next as the split
 * step (3-D power-of-two planes: inverse x transforms, the column pass with
 * the y transforms and the pointwise epilogue, forward x transforms, each a
 * separate kernel that needs no cluster), the mean CUDA-event time of each of
 * the three kernels (ms_out[0..2], in that order) and their algorithmic bytes
 * per launch (the column pass: the mean of an odd and an even iteration);
 * otherwise WS_ERR_UNSUPPORTED.  No counterpart in the reference. */
int ws_solver_time_split(ws_solver s, int n_iterations, float ms_out[3], double bytes_out[3]);

/* After a warm-started solve of right-hand side `rhs`: the ROI energy of the
 * cold first increment (diff_energy(1), from the probe iteration), the ROI
 * energy of the true increment at the end of the warm first wiggle cycle,
 * and whether the start was discarded (by its initial residual, see
 * warm_discard_ratio).  Any pointer may be NULL; the
 * values are -1 / 0 after a cold solve.  No counterpart in the reference. */
int ws_solver_warm_report(ws_solver s, int64_t rhs, double* cold_first_energy, double* warm_cycle_energy,
                          int* discarded);

/* After a warm-started solve of right-hand side `rhs` with a discard test
 * (warm_discard_ratio > 0): the ROI energies of the cold start's initial
 * residual (Nw^2 diff_energy(1)) and of the warm start's (see
 * warm_discard_ratio).  -1 when no test ran.  No counterpart in the
 * reference. */
int ws_solver_warm_residual(ws_solver s, int64_t rhs, double* cold_residual_energy, double* warm_residual_energy);

/* Autotuner (no counterpart in the reference): times the kernel layouts the
 * solver's grid supports - the power-of-two fast kernels or the generic
 * mixed-radix ones for the inner and the outer pass, the generic kernels'
 * radix schedules, the split step's x pencils (y tile, stages), the TMA
 * pencil's stages, the generic outer pass's y tile, the 2-D columns per
 * block - over n_iterations iterations of the loop as it runs (the fused
 * step where there is one) each, keeps the fastest inner and outer pass,
 * and uses them from the next solve on.  A candidate must first reproduce one iteration of the current
 * layout to 1e-4.  Outputs (may be NULL): candidates tried, and the time of
 * one iteration (K1 + K2 + K3, ms) before and after.  Overwrites the solver's
 * fields; call it between solves. */
int ws_solver_autotune(ws_solver s, int n_iterations, int* n_tried, float* ms_before, float* ms_after);

/* The solver's layout choice as 7 integers (the autotuner's pick, or zeros
 * for the heuristics): inner kernels, outer kernel, cluster size, columns per
 * block, y per outer block, radix schedule of the generic kernels, x pencil
 * of the split step.  ws_solver_set_layout applies such a choice (e.g. one
 * cached from an earlier autotune of the same grid) without timing anything;
 * WS_ERR_UNSUPPORTED if this grid does not take it.  No counterpart in the
 * reference. */
int ws_solver_get_layout(ws_solver s, int32_t choice[7]);
int ws_solver_set_layout(ws_solver s, const int32_t choice[7]);

int ws_solver_destroy(ws_solver s);

/* ------------------------------------------------------------------------
 * PSTD: the reference's pseudo-spectral time-domain comparison solver
 * (PSTD.m:22-137) on the same FFT kernels.  Replaces PSTD.run_algorithm
 * (PSTD.m:79-127); the constructor's set-up (time step, coefficient maps,
 * Fourier ranges, PSTD.m:22-77) stays with the caller.
 * ------------------------------------------------------------------------ */
typedef struct ws_pstd_s* ws_pstd;

/* A(Ncycle), the source amplitude of PSTD.source_amplitude (PSTD.m:10). */
typedef void (*ws_amplitude_fn)(double ncycle, double* re, double* im, void* user_data);

typedef struct ws_pstd_options {
  int64_t max_iterations;        /* ceil(max_cycles * iterations_per_cycle) (Simulation.m:165); as in
                                    Simulation.next the run stops there only on a step with real(A) > 0.9 */
  double energy_threshold;       /* Simulation.energy_threshold */
  int64_t energy_interval;       /* Simulation.energy_calculation_interval */
  double iterations_per_cycle;   /* lambda / dt (PSTD.m:55); step it runs at Ncycle = it / this */
  ws_amplitude_fn amplitude;     /* NULL: PSTD.default_source (PSTD.m:130-137) */
  void* user_data;
} ws_pstd_options;

void ws_pstd_default_options(ws_pstd_options* opts);

/* N = grid (Ny, Nx, Nz); c1, c2, c3 = the real coefficient maps of the damped
 * leapfrog (PSTD.m:57-63, N(1) N(2) N(3) floats, column-major, host);
 * px, py, pz = SimulationGrid px_range (Nx), py_range (Ny), pz_range (Nz);
 * roi = 1-based [first; last] per dimension as in ws_solver_create. */
int ws_pstd_create(const int64_t N[3], const float* c1, const float* c2, const float* c3, const float* px,
                   const float* py, const float* pz, const int64_t roi[8], int device, ws_pstd* out);

/* Runs PSTD.run_algorithm for the source blocks (positions on the grid,
 * 1-based, cropped).  E_out (host) receives the ROI field times
 * exp(-i arg A(it_final / iterations_per_cycle)) (PSTD.m:125-126),
 * diff_energy_out (host, may be NULL) the first diff_capacity entries of
 * state.diff_energy. */
int ws_pstd_run(ws_pstd h, int64_t n_blocks, const ws_source_block* source, int source_memory,
                const ws_pstd_options* opts, ws_complex* E_out, double* diff_energy_out, int64_t diff_capacity,
                int64_t* n_iterations, int* converged);

int ws_pstd_destroy(ws_pstd h);

/*
 * Medium set-up on the device (no counterpart in the reference, which builds
 * gamma in MATLAB on the host; WaveSimBase.m:58-81, 201-258, Medium.m:44-62).
 * n is the refractive index of the ROI, Ny*Nx*Nz column-major, complex
 * double (is_complex = 1) or double, in device memory.
 *
 * ws_medium_reduce: out[0] = min real(n^2), out[1] = max real(n^2) (e_r_min,
 * e_r_max of Medium.m:45-47); with k0sq > 0 also out[2] = max |n^2 k0^2 -
 * k0c^2| (epsilon = max(out[2] / 0.95, 3), WaveSimBase.m:201-215).
 * ws_build_gamma: gamma = (i/epsilon)(e_r k0^2 - k0c^2 - i epsilon) fy fx fz
 * on the full Ny x Nx x Nz grid (complex64, device), e_r = n^2 replicated
 * into the boundary layers (the ROI starts at roi_lo, 0-based), fy/fx/fz the
 * 1-D ARL windows (device floats of lengths Ny, Nx, Nz).  Computed in double,
 * rounded once.  ws_setup_last_error gives the message of a failure.
 */
int ws_medium_reduce(const void* n, int is_complex, int64_t count, double k0sq, double k0c2, double out[3],
                     void* stream);
int ws_build_gamma(const void* n, int is_complex, const int64_t roi_size[3], const int64_t N[3],
                   const int64_t roi_lo[3], const float* fy, const float* fx, const float* fz, double k0sq,
                   double k0c2, double epsilon, void* gamma, void* stream);
const char* ws_setup_last_error(void);

/*
 * ws_run_algorithm_noalloc - the same loop as ws_run_algorithm for callers
 * that cannot allocate GPU memory (an application that owns the device
 * through its own memory pool, a real-time loop that forbids allocation after
 * start-up, a plug-in confined to the buffers it is handed).  No counterpart
 * in the reference.
 *
 * Every pointer is a device pointer except wiggles (a host array of
 * ws_wiggle whose members are device pointers), N, roi and the scalar outputs.
 * source_field is the dense source, Ny*Nx*Nz*Nc complex (the blocks summed
 * into one field, Source.add_to with factor 1).  E_out receives E' (full
 * grid), diff_energy_out (device, >= max_iterations + n_wiggles doubles) the
 * energy history.  stream: a cudaStream_t, or NULL for the default stream.
 *
 * The working arrays live in one statically allocated device array of
 * ws_noalloc_scratch_bytes() bytes (40 MiB), shared by all calls and kept by
 * every GPU that loads it until the process exits.  A grid needs 16 bytes per
 * field element plus twiddle tables: about 2.6 million elements at most;
 * larger grids return WS_ERR_INVALID_ARGUMENT.  Calls that overlap on the GPU
 * race on the shared array.  The first call on each device looks up the
 * array's address and should come before any stream capture.  Errors:
 * ws_noalloc_last_error().
 */
int ws_run_algorithm_noalloc(const int64_t N[4], const ws_complex* gamma, int64_t n_wiggles,
                             const ws_wiggle* wiggles, const ws_complex* source_field, float epsilon,
                             ws_complex k02e, const int64_t roi[8], int64_t max_iterations,
                             double energy_threshold, int64_t energy_interval, ws_complex* E_out,
                             double* diff_energy_out, int64_t* n_iterations, int* converged, void* stream);

/* Size in bytes of the static scratch array of ws_run_algorithm_noalloc. */
int64_t ws_noalloc_scratch_bytes(void);

/* Message of the last failed ws_run_algorithm_noalloc call on this thread. */
const char* ws_noalloc_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* WAVESIM_B200_H */
