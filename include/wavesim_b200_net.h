/*
 * wavesim_b200_net - kernels of the learned warm start (sm_100a).
 * No counterpart in the reference.
 *
 * A small 3-D convolutional encoder-decoder predicts the starting field of
 * the MBS loop (wavesim_b200/warmstart.py).  Its convolutions run on the
 * tcgen05 tensor cores (bf16 operands, fp32 accumulation in tensor memory):
 * the forward pass and the input gradient as implicit GEMMs that gather
 * their operand in the kernel (ws_conv3_fwd_bf16), the weight gradient as an
 * explicit GEMM (ws_gemm_bf16) of transposed im2col matrices.  The other
 * entry points are the layer kernels around them.
 *
 * Every pointer is a device pointer; activations are channels-last
 * [voxel][channel] with voxels in (b, z, y, x) order; `stream` is a
 * cudaStream_t (NULL: default stream).  Functions return a ws_status;
 * ws_net_last_error() gives the message of the last failure on the thread.
 * err_flag (a device int, may be NULL) is set to 1 when a tensor-core
 * completion wait of the kernel timed out (it then frees its tensor memory
 * and returns without writing its output).
 */
#ifndef WAVESIM_B200_NET_H
#define WAVESIM_B200_NET_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* C[M][N] = A[M][K] . B[N][K]^T, A and B bf16 with K contiguous (K a multiple
 * of 64, rows 16-byte aligned).  mode 0: fp32 C; 1: bias + ReLU -> bf16 Cb;
 * 2: bias -> bf16 Cb; 3: bias -> fp32 C. */
int ws_gemm_bf16(const void* A, const void* B, float* C, void* Cb, const float* bias, int64_t M, int64_t N,
                 int64_t K, int64_t lda, int64_t ldb, int64_t ldc, int mode, int* err_flag, void* stream);

/* 3x3x3 convolution, zero padding 1, as an implicit GEMM on the tensor cores:
 * out[vox][co] = sum_k A[vox][k] W[co][k] with A[vox][t*C + c] = X[vox +
 * offset(t)][c] gathered by the kernel (X bf16 [vox][C], C % 8 == 0), W bf16
 * [Cout][kp], kp = 27 C rounded up to 64.  mode as for ws_gemm_bf16: 0 and 3
 * write out_f32, 1 and 2 out_bf16, each [vox][Cout]. */
int ws_conv3_fwd_bf16(const void* X, const void* W, const float* bias, float* out_f32, void* out_bf16, int b, int d,
                      int h, int w, int C, int Cout, int kp, int mode, int* err_flag, void* stream);

/* The same convolution of the channel concat [nearest x2 upsampling of U, X]
 * (a decoder level) without writing the concat: U (b, d/2, h/2, w/2) x Cu,
 * X (b, d, h, w) x Cx, Cu and Cx multiples of 8, d, h, w even, kp >= 27
 * (Cu + Cx). */
int ws_conv3_upcat_fwd_bf16(const void* U, const void* X, const void* W, const float* bias, float* out_f32,
                            void* out_bf16, int b, int d, int h, int w, int Cu, int Cx, int Cout, int kp, int mode,
                            int* err_flag, void* stream);

/* Network input of a ROI: n (and src, may be NULL for a plane of ones at
 * z = 0) real fp32 Ny x Nx x Nz column-major; out bf16 [Ny*Nx*Nz][8] =
 * [(n - n_bg)/0.2, src, cos phi, sin phi, 0, 0, 0, 0], phi = k0 sum_{z' <= z}
 * (n - n_bg) the straight-ray phase from the z = 0 face. */
int ws_net_features(const float* n, const float* src, int ny, int nx, int nz, float n_bg, float k0, void* out,
                    void* stream);

/* Full-grid starting field psi0 (complex64, Ny x Nx x Nz column-major) from
 * the network output (the ROI envelope): scale * pred * exp(i kz z) in the
 * ROI, continued into the boundary layers by the nearest ROI value under a
 * cos^2 taper.  pred is [vox][2] with voxels in the ROI's column-major order,
 * or with s2d = 1 the half-resolution [hvox][16] of ws_net_space_to_depth
 * (sub-voxel s at columns 2s, 2s + 1).  N, roi0 (0-based first ROI index)
 * and roin (ROI size) as (y, x, z). */
int ws_net_envelope_to_field(const float* pred, const int64_t N[3], const int64_t roi0[3], const int64_t roin[3],
                             float scale, float kz, int s2d, void* psi, void* stream);

/* Space to depth: (b, d, h, w) x C bf16 -> (b, d/2, h/2, w/2) x 8C, the
 * 2x2x2 sub-voxel s = ((z & 1) 2 + (y & 1)) 2 + (x & 1) at channels
 * [s C, (s + 1) C); C % 8 == 0, even sides. */
int ws_net_space_to_depth(const void* in, void* out, int b, int d, int h, int w, int C, void* stream);

/* Weights of the input-gradient convolution: Wf[ci][t Cpad + co] =
 * W[co][(26 - t) Cin + ci], zero for co >= Cout; W bf16 [Cout][kp], Wf bf16
 * [Cin][kpf], kpf >= 27 Cpad. */
int ws_net_flip_weights(const void* W, int Cin, int Cout, int kp, void* Wf, int Cpad, int kpf, void* stream);

/* dy *= (y > 0) in place for the bf16 output y of a ReLU (y may be NULL) and
 * out = bf16(dy) [rows][Cpad], channels C..Cpad-1 zero. */
int ws_net_relu_grad_bf16(float* dy, const void* y, int64_t rows, int C, void* out, int Cpad, void* stream);

/* im2col of a 3x3x3 convolution with zero padding 1: col[vox][kp], entry
 * ((dz*3 + dy)*3 + dx)*C + c, zero for k >= 27 C (C, kp multiples of 8). */
int ws_net_im2col3(const void* in, void* col, int b, int d, int h, int w, int C, int kp, void* stream);
/* gradient of ws_net_im2col3 (fp32): din[u][c] = sum_t dcol[u - (t - 1)][t C + c] */
int ws_net_col2im3(const float* dcol, float* din, int b, int d, int h, int w, int C, int kp, void* stream);
/* out[c][r] = bf16(in[r][c]) (fp32 in, rows x cols), out rows zero-padded to ldo */
int ws_net_transpose_f32_bf16(const float* in, void* out, int64_t rows, int64_t cols, int64_t ldo, void* stream);
/* out[c][r] = in[r][c] (bf16, in with leading dimension ldi), out rows zero-padded to ldo */
int ws_net_transpose_bf16(const void* in, void* out, int64_t rows, int64_t cols, int64_t ldi, int64_t ldo,
                          void* stream);
/* 2x2x2 average pooling of a (b, d, h, w) volume, and its gradient */
int ws_net_avgpool2(const void* in, void* out, int b, int d, int h, int w, int C, void* stream);
int ws_net_avgpool2_grad(const float* dout, float* din, int b, int d, int h, int w, int C, void* stream);
/* out = [nearest x2 upsampling of a (Ca channels), skip (Cs channels)] on a
 * (b, d, h, w) volume, and its gradient */
int ws_net_upcat(const void* a, const void* skip, void* out, int b, int d, int h, int w, int Ca, int Cs, void* stream);
int ws_net_upcat_grad(const float* dout, float* da, float* dskip, int b, int d, int h, int w, int Ca, int Cs,
                      void* stream);
/* dy *= (y > 0) for the bf16 output y of a ReLU */
int ws_net_relu_grad(float* dy, const void* y, int64_t n, void* stream);
/* db[c] = sum_r dy[r][c] */
int ws_net_bias_grad(const float* dy, float* db, int64_t rows, int C, void* stream);
/* Adam step (bias-corrected, step >= 1) on fp32 weights, optional bf16 copy wb */
int ws_net_adam(float* w, const float* g, float* m, float* v, void* wb, int64_t n, float lr, float b1, float b2,
                float eps, int step, void* stream);
/* mean squared error: loss += mean((pred - target)^2), grad = 2 (pred - target) / n */
int ws_net_mse(const float* pred, const float* target, float* grad, double* loss, int64_t rows, int cols,
               int64_t ldp, void* stream);
/* out = bf16(in) */
int ws_net_f32_to_bf16(const float* in, void* out, int64_t n, void* stream);
/* y += x (fp32) */
int ws_net_add(float* y, const float* x, int64_t n, void* stream);
const char* ws_net_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* WAVESIM_B200_NET_H */
