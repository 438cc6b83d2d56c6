// Elementwise and reduction kernels of the surrogate's training step: input
// packing to padded bf16 (row-major and transposed), softmax cross-entropy
// with its logit gradient, bias-gradient column sums, AdamW on the FP32
// master weights and the bf16 weight copies the GEMMs consume.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "stb_mlp.hpp"

namespace stb {

namespace {

__global__ void pack_input_kernel(const float *x, int B, int nin, int ldp, __nv_bfloat16 *X0, __nv_bfloat16 *X0T) {
  const long total = (long)B * ldp;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int b = (int)(i / ldp), j = (int)(i % ldp);
    const __nv_bfloat16 v = __float2bfloat16_rn(j < nin ? x[(long)b * nin + j] : 0.0f);
    X0[i] = v;
    X0T[(long)j * B + b] = v;
  }
}

// Two-class (or nout-class) softmax cross-entropy, mean over the batch with
// optional per-sample weights.  dZ = w * (p - onehot) * inv_norm.
__global__ void softmax_xent_kernel(const float *logits, int ld, const int32_t *labels, const float *weights, int B,
                                    int nout, float inv_norm, float *loss_sum, float *probs, __nv_bfloat16 *dZ,
                                    __nv_bfloat16 *dZT, int nout_pad, float *dz_f32) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  float l = 0.0f;
  if (b < B) {
    const float *z = logits + (long)b * ld;
    float mx = z[0];
    for (int j = 1; j < nout; j++) mx = fmaxf(mx, z[j]);
    float s = 0.0f;
    for (int j = 0; j < nout; j++) s += expf(z[j] - mx);
    const float w = weights ? weights[b] : 1.0f;
    const int y = labels ? labels[b] : -1;
    for (int j = 0; j < nout_pad; j++) {
      float p = 0.0f, d = 0.0f;
      if (j < nout) {
        p = expf(z[j] - mx) / s;
        d = w * (p - (j == y ? 1.0f : 0.0f)) * inv_norm;
        if (probs) probs[(long)b * nout + j] = p;
      }
      if (dZ) {
        const __nv_bfloat16 h = __float2bfloat16_rn(d);
        dZ[(long)b * nout_pad + j] = h;
        dZT[(long)j * B + b] = h;
        if (dz_f32) dz_f32[(long)b * nout_pad + j] = d;
      }
    }
    if (y >= 0) l = w * (logf(s) + mx - z[y]) * inv_norm;
  }
  // warp reduction, one atomic per warp
  for (int o = 16; o > 0; o >>= 1) l += __shfl_down_sync(0xffffffffu, l, o);
  if ((threadIdx.x & 31) == 0 && loss_sum) atomicAdd(loss_sum, l);
}

// out[j] = sum_b dz[b][j]: one CTA per column.
__global__ void column_sums_kernel(const float *dz, int B, int N, int ld, float *out) {
  __shared__ float red[32];
  const int j = blockIdx.x;
  float s = 0.0f;
  for (int b = threadIdx.x; b < B; b += blockDim.x) s += dz[(long)b * ld + j];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x < 32) {
    s = threadIdx.x < (int)(blockDim.x >> 5) ? red[threadIdx.x] : 0.0f;
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (threadIdx.x == 0) out[j] = s;
  }
}

// Decoupled weight decay (Loshchilov & Hutter), bias-corrected moments.
__global__ void adamw_kernel(float *w, const float *g, float *m, float *v, long n, float lr, float b1, float b2,
                             float eps, float wd, float bc1, float bc2) {
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    const float mh = mi / bc1, vh = vi / bc2;
    w[i] = w[i] - lr * (mh / (sqrtf(vh) + eps) + wd * w[i]);
  }
}

__global__ void cast_weights_kernel(const float *w, int out, int in, int out_pad, int in_pad, __nv_bfloat16 *W,
                                    __nv_bfloat16 *WT) {
  const long total = (long)out_pad * in_pad;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total; i += (long)gridDim.x * blockDim.x) {
    const int o = (int)(i / in_pad), k = (int)(i % in_pad);
    const __nv_bfloat16 h = __float2bfloat16_rn((o < out && k < in) ? w[(long)o * in + k] : 0.0f);
    W[i] = h;
    WT[(long)k * out_pad + o] = h;
  }
}

int grid_for(long n, int block) {
  long g = (n + block - 1) / block;
  if (g > 4096) g = 4096;
  return g < 1 ? 1 : (int)g;
}

}  // namespace

cudaError_t mlp_pack_input(const float *x, int B, int nin, int ldp, __nv_bfloat16 *X0, __nv_bfloat16 *X0T,
                           cudaStream_t st) {
  pack_input_kernel<<<grid_for((long)B * ldp, 256), 256, 0, st>>>(x, B, nin, ldp, X0, X0T);
  return cudaGetLastError();
}

cudaError_t mlp_softmax_xent(const float *logits, int ld, const int32_t *labels, const float *weights, int B,
                             int nout, float inv_norm, float *loss_sum, float *probs, __nv_bfloat16 *dZ,
                             __nv_bfloat16 *dZT, int nout_pad, float *dz_f32, cudaStream_t st) {
  softmax_xent_kernel<<<(B + 255) / 256, 256, 0, st>>>(logits, ld, labels, weights, B, nout, inv_norm, loss_sum, probs,
                                                        dZ, dZT, nout_pad, dz_f32);
  return cudaGetLastError();
}

cudaError_t mlp_column_sums(const float *dz, int B, int N, int ld, float *out, cudaStream_t st) {
  column_sums_kernel<<<N, 256, 0, st>>>(dz, B, N, ld, out);
  return cudaGetLastError();
}

cudaError_t mlp_adamw(float *w, const float *g, float *m, float *v, long n, float lr, float b1, float b2, float eps,
                      float wd, float bc1, float bc2, cudaStream_t st) {
  adamw_kernel<<<grid_for(n, 256), 256, 0, st>>>(w, g, m, v, n, lr, b1, b2, eps, wd, bc1, bc2);
  return cudaGetLastError();
}

cudaError_t mlp_cast_weights(const float *w, int out, int in, int out_pad, int in_pad, __nv_bfloat16 *W,
                             __nv_bfloat16 *WT, cudaStream_t st) {
  cast_weights_kernel<<<grid_for((long)out_pad * in_pad, 256), 256, 0, st>>>(w, out, in, out_pad, in_pad, W, WT);
  return cudaGetLastError();
}

}  // namespace stb
