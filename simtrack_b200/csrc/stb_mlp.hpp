// Surrogate MLP kernels: argument blocks and launch interfaces.
#pragma once
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "stb_status.hpp"

namespace stb {

enum GemmEpilogue : int {
  EPI_F32 = 0,        // C = acc (optionally stored transposed)
  EPI_BIAS_F32 = 1,   // C = acc + bias
  EPI_BIAS_GELU = 2,  // C = Z = acc + bias; H = HT^T = bf16(GELU(Z))
  EPI_DGELU = 3,      // dZ = acc * GELU'(Z); H = HT^T = bf16(dZ); C = dZ if C != NULL
};

struct GemmArgs {
  const __nv_bfloat16 *A;  // [M x K], row stride lda (K contiguous)
  const __nv_bfloat16 *B;  // [N x K], row stride ldb
  int lda, ldb;
  int M, N, K;             // N in {16, 32, ..., 256}; K a multiple of 16
  int mode;
  int transpose_out;       // EPI_F32: store C^T
  int n_valid;             // EPI_F32 / EPI_BIAS_F32: columns stored (bias applied); 0 = N
  float *C;
  int ldc;
  const float *bias;
  const float *Z;          // EPI_DGELU: saved pre-activation
  int ldz;
  __nv_bfloat16 *H;        // bf16 row-major output
  int ldh;
  __nv_bfloat16 *HT;       // bf16 transposed output
  int ldht;
  int *status;
};

size_t mlp_gemm_smem_bytes();
cudaError_t mlp_gemm_launch(const GemmArgs &g, cudaStream_t st);

// Elementwise kernels of the training step (stb_mlp_ops.cu).
cudaError_t mlp_pack_input(const float *x, int B, int nin, int ldin_pad, __nv_bfloat16 *X0, __nv_bfloat16 *X0T,
                           cudaStream_t st);
cudaError_t mlp_softmax_xent(const float *logits, int ld, const int32_t *labels, const float *weights, int B,
                             int nout, float inv_norm, float *loss_sum, float *probs, __nv_bfloat16 *dZ,
                             __nv_bfloat16 *dZT, int nout_pad, float *dz_f32, cudaStream_t st);
cudaError_t mlp_column_sums(const float *dz, int B, int N, int ld, float *out, cudaStream_t st);
cudaError_t mlp_adamw(float *w, const float *g, float *m, float *v, long n, float lr, float b1, float b2, float eps,
                      float wd, float bc1, float bc2, cudaStream_t st);
cudaError_t mlp_cast_weights(const float *w, int out, int in, int out_pad, int in_pad, __nv_bfloat16 *W,
                             __nv_bfloat16 *WT, cudaStream_t st);

}  // namespace stb
