// Host side of the surrogate MLP (C ABI stb_mlp_*): parameter storage,
// forward / backward orchestration over the tcgen05 GEMM kernel and the
// elementwise kernels, and the AdamW step.
//
// Network: nin -> H -> H -> H -> nout, GELU after each hidden layer, softmax
// cross-entropy on the output.  FP32 master parameters; the GEMMs consume
// bf16 copies of weights, activations and gradients and accumulate in FP32.
// Input and output widths are padded to 16 (one MMA K step / the smallest N).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "simtrack_b200.h"
#include "stb_mlp.hpp"
#include "stb_runtime.hpp"

using bf16 = __nv_bfloat16;

struct stb_mlp {
  int device = 0;
  int nin = 0, H = 0, nout = 0, max_batch = 0;
  static constexpr int kPadIn = 16, kPadOut = 16;
  long nparams = 0;
  long off_W[4] = {0}, off_b[4] = {0};
  int dims_out[4] = {0}, dims_in[4] = {0}, pad_out[4] = {0}, pad_in[4] = {0};
  float *params = nullptr, *grads = nullptr, *m = nullptr, *v = nullptr;
  bf16 *W[4] = {nullptr}, *WT[4] = {nullptr};
  // activations (max_batch rows)
  bf16 *X0 = nullptr, *X0T = nullptr;
  float *Z[3] = {nullptr};
  bf16 *Hh[3] = {nullptr}, *HT[3] = {nullptr};
  float *logits = nullptr;
  bf16 *dZ[4] = {nullptr}, *dZT[4] = {nullptr};
  float *dzf[4] = {nullptr};
  float *loss = nullptr;
  int *status = nullptr;
  cudaStream_t stream = nullptr;
  std::vector<void *> allocs;
  float lr = 1e-3f, b1 = 0.9f, b2 = 0.999f, eps = 1e-8f, wd = 1e-2f;
  long step = 0;
};

namespace stb {
namespace {

void mlp_destroy(stb_mlp *p) {
  if (!p) return;
  int prev = -1;
  cudaGetDevice(&prev);
  cudaSetDevice(p->device);
  for (void *a : p->allocs) cudaFree(a);
  if (p->stream) cudaStreamDestroy(p->stream);
  if (prev >= 0) cudaSetDevice(prev);
  delete p;
}

template <class T>
T *dalloc(stb_mlp *p, long count) {
  void *d = nullptr;
  cuda_check(cudaMalloc(&d, sizeof(T) * (size_t)(count > 0 ? count : 1)), "cudaMalloc(mlp)");
  p->allocs.push_back(d);
  cuda_check(cudaMemset(d, 0, sizeof(T) * (size_t)(count > 0 ? count : 1)), "cudaMemset(mlp)");
  return (T *)d;
}

void refresh_bf16(stb_mlp *p) {
  for (int l = 0; l < 4; l++)
    cuda_check(mlp_cast_weights(p->params + p->off_W[l], p->dims_out[l], p->dims_in[l], p->pad_out[l], p->pad_in[l],
                                p->W[l], p->WT[l], p->stream),
               "cast weights");
}

stb_mlp *mlp_build(int nin, int hidden, int nout, int max_batch, unsigned long long seed, int device) {
  if (nin < 1 || nin > 16 || nout < 1 || nout > 16) throw Error(STB_EINVAL, "input and output widths must be 1..16");
  if (hidden < 16 || hidden > 256 || hidden % 16) throw Error(STB_EINVAL, "hidden width must be a multiple of 16 <= 256");
  if (max_batch < 16 || max_batch % 16) throw Error(STB_EINVAL, "max_batch must be a positive multiple of 16");
  std::unique_ptr<stb_mlp, void (*)(stb_mlp *)> p(new stb_mlp(), mlp_destroy);
  p->device = device;
  p->nin = nin;
  p->H = hidden;
  p->nout = nout;
  p->max_batch = max_batch;
  DeviceGuard g(device);
  cuda_check(cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking), "stream");
  const int H = hidden;
  int outs[4] = {H, H, H, nout}, ins[4] = {nin, H, H, H};
  int pouts[4] = {H, H, H, stb_mlp::kPadOut}, pins[4] = {stb_mlp::kPadIn, H, H, H};
  long off = 0;
  for (int l = 0; l < 4; l++) {
    p->dims_out[l] = outs[l];
    p->dims_in[l] = ins[l];
    p->pad_out[l] = pouts[l];
    p->pad_in[l] = pins[l];
    p->off_W[l] = off;
    off += (long)outs[l] * ins[l];
    p->off_b[l] = off;
    off += outs[l];
  }
  p->nparams = off;
  p->params = dalloc<float>(p.get(), off);
  p->grads = dalloc<float>(p.get(), off);
  p->m = dalloc<float>(p.get(), off);
  p->v = dalloc<float>(p.get(), off);
  // PyTorch nn.Linear default: U(-1/sqrt(in), 1/sqrt(in)) for weights and biases.
  std::mt19937_64 rng(seed);
  std::vector<float> host(off);
  for (int l = 0; l < 4; l++) {
    const float a = 1.0f / std::sqrt((float)ins[l]);
    std::uniform_real_distribution<float> U(-a, a);
    for (long i = 0; i < (long)outs[l] * ins[l]; i++) host[p->off_W[l] + i] = U(rng);
    for (int i = 0; i < outs[l]; i++) host[p->off_b[l] + i] = U(rng);
  }
  cuda_check(cudaMemcpy(p->params, host.data(), sizeof(float) * off, cudaMemcpyHostToDevice), "upload params");
  for (int l = 0; l < 4; l++) {
    p->W[l] = dalloc<bf16>(p.get(), (long)pouts[l] * pins[l]);
    p->WT[l] = dalloc<bf16>(p.get(), (long)pouts[l] * pins[l]);
  }
  const long B = max_batch;
  p->X0 = dalloc<bf16>(p.get(), B * stb_mlp::kPadIn);
  p->X0T = dalloc<bf16>(p.get(), B * stb_mlp::kPadIn);
  for (int l = 0; l < 3; l++) {
    p->Z[l] = dalloc<float>(p.get(), B * H);
    p->Hh[l] = dalloc<bf16>(p.get(), B * H);
    p->HT[l] = dalloc<bf16>(p.get(), B * H);
    p->dZ[l] = dalloc<bf16>(p.get(), B * H);
    p->dZT[l] = dalloc<bf16>(p.get(), B * H);
    p->dzf[l] = dalloc<float>(p.get(), B * H);
  }
  p->dZ[3] = dalloc<bf16>(p.get(), B * stb_mlp::kPadOut);
  p->dZT[3] = dalloc<bf16>(p.get(), B * stb_mlp::kPadOut);
  p->dzf[3] = dalloc<float>(p.get(), B * stb_mlp::kPadOut);
  p->logits = dalloc<float>(p.get(), B * stb_mlp::kPadOut);
  p->loss = dalloc<float>(p.get(), 1);
  p->status = dalloc<int>(p.get(), 1);
  refresh_bf16(p.get());
  cuda_check(cudaStreamSynchronize(p->stream), "mlp init");
  return p.release();
}

GemmArgs gemm(const bf16 *A, int lda, const bf16 *B, int ldb, int M, int N, int K, int mode, int *status) {
  GemmArgs g{};
  g.A = A;
  g.B = B;
  g.lda = lda;
  g.ldb = ldb;
  g.M = M;
  g.N = N;
  g.K = K;
  g.mode = mode;
  g.status = status;
  return g;
}

void run_gemm(stb_mlp *p, const GemmArgs &g) { cuda_check(mlp_gemm_launch(g, p->stream), "tcgen05 GEMM launch"); }

void check_batch(stb_mlp *p, int B) {
  if (B < 16 || B > p->max_batch || B % 16) throw Error(STB_EINVAL, "batch must be a multiple of 16 within max_batch");
}

// Forward pass; leaves Z, H, HT of every hidden layer and the logits.
void forward(stb_mlp *p, const float *x, int B) {
  const int H = p->H;
  cuda_check(mlp_pack_input(x, B, p->nin, stb_mlp::kPadIn, p->X0, p->X0T, p->stream), "pack input");
  const bf16 *in = p->X0;
  int ldin = stb_mlp::kPadIn;
  for (int l = 0; l < 3; l++) {
    GemmArgs g = gemm(in, ldin, p->W[l], p->pad_in[l], B, H, p->pad_in[l], EPI_BIAS_GELU, p->status);
    g.C = p->Z[l];
    g.ldc = H;
    g.bias = p->params + p->off_b[l];
    g.H = p->Hh[l];
    g.ldh = H;
    g.HT = p->HT[l];
    g.ldht = B;
    run_gemm(p, g);
    in = p->Hh[l];
    ldin = H;
  }
  GemmArgs g = gemm(p->Hh[2], H, p->W[3], H, B, stb_mlp::kPadOut, H, EPI_BIAS_F32, p->status);
  g.C = p->logits;
  g.ldc = stb_mlp::kPadOut;
  g.bias = p->params + p->off_b[3];
  g.n_valid = p->nout;
  run_gemm(p, g);
}

// Loss and parameter gradients (into p->grads) for one batch.
void backward(stb_mlp *p, const float *x, const int32_t *labels, const float *weights, int B, float *loss_host) {
  forward(p, x, B);
  cuda_check(cudaMemsetAsync(p->loss, 0, sizeof(float), p->stream), "reset loss");
  float norm = (float)B;
  if (weights) {
    std::vector<float> w(B);
    cuda_check(cudaMemcpyAsync(w.data(), weights, sizeof(float) * B, cudaMemcpyDeviceToHost, p->stream), "weights");
    cuda_check(cudaStreamSynchronize(p->stream), "weights");
    double s = 0;
    for (float v : w) s += v;
    norm = s > 0 ? (float)s : 1.0f;
  }
  cuda_check(mlp_softmax_xent(p->logits, stb_mlp::kPadOut, labels, weights, B, p->nout, 1.0f / norm, p->loss,
                              nullptr, p->dZ[3], p->dZT[3], stb_mlp::kPadOut, p->dzf[3], p->stream),
             "softmax cross-entropy");
  for (int l = 3; l >= 0; l--) {
    const bf16 *prevT = l > 0 ? p->HT[l - 1] : p->X0T;
    // dW_l = dZ_l^T * H_{l-1}: M = out_l, N = padded in_l, K = batch
    GemmArgs gw = gemm(p->dZT[l], B, prevT, B, p->dims_out[l], p->pad_in[l], B, EPI_F32, p->status);
    gw.C = p->grads + p->off_W[l];
    gw.ldc = p->dims_in[l];
    gw.n_valid = p->dims_in[l];
    run_gemm(p, gw);
    // db_l = sum over the batch of dZ_l
    cuda_check(mlp_column_sums(p->dzf[l], B, p->dims_out[l], p->pad_out[l], p->grads + p->off_b[l], p->stream),
               "bias gradient");
    if (l > 0) {
      // dH_{l-1} = dZ_l * W_l, then dZ_{l-1} = dH_{l-1} * GELU'(Z_{l-1})
      GemmArgs gd = gemm(p->dZ[l], p->pad_out[l], p->WT[l], p->pad_out[l], B, p->pad_in[l], p->pad_out[l], EPI_DGELU,
                         p->status);
      gd.Z = p->Z[l - 1];
      gd.ldz = p->H;
      gd.H = p->dZ[l - 1];
      gd.ldh = p->H;
      gd.HT = p->dZT[l - 1];
      gd.ldht = B;
      gd.C = p->dzf[l - 1];
      gd.ldc = p->H;
      run_gemm(p, gd);
    }
  }
  if (loss_host) {
    cuda_check(cudaMemcpyAsync(loss_host, p->loss, sizeof(float), cudaMemcpyDeviceToHost, p->stream), "loss");
  }
  cuda_check(cudaStreamSynchronize(p->stream), "mlp backward");
  int st = 0;
  cuda_check(cudaMemcpy(&st, p->status, sizeof(int), cudaMemcpyDeviceToHost), "status");
  if (st != 0) throw Error(st, "tcgen05 GEMM reported status " + std::to_string(st));
}

void adamw_step(stb_mlp *p) {
  p->step += 1;
  const float bc1 = 1.0f - std::pow(p->b1, (float)p->step), bc2 = 1.0f - std::pow(p->b2, (float)p->step);
  cuda_check(mlp_adamw(p->params, p->grads, p->m, p->v, p->nparams, p->lr, p->b1, p->b2, p->eps, p->wd, bc1, bc2,
                       p->stream),
             "adamw");
  refresh_bf16(p);
  cuda_check(cudaStreamSynchronize(p->stream), "adamw");
}

}  // namespace
}  // namespace stb

using namespace stb;

extern "C" {

int stb_mlp_create(int nin, int hidden, int nout, int max_batch, unsigned long long seed, int device, stb_mlp **out) {
  return guarded([&] {
    if (!out) throw Error(STB_EINVAL, "NULL output");
    *out = mlp_build(nin, hidden, nout, max_batch, seed, device);
    return STB_OK;
  });
}

int stb_mlp_free(stb_mlp *p) {
  return guarded([&] {
    mlp_destroy(p);
    return STB_OK;
  });
}

long stb_mlp_param_count(const stb_mlp *p) { return p ? p->nparams : -1; }

int stb_mlp_get_params(stb_mlp *p, float *host, int which) {
  return guarded([&] {
    if (!p || !host) throw Error(STB_EINVAL, "NULL argument");
    DeviceGuard g(p->device);
    const float *src = which == 1 ? p->grads : p->params;
    cuda_check(cudaMemcpy(host, src, sizeof(float) * p->nparams, cudaMemcpyDeviceToHost), "download");
    return STB_OK;
  });
}

int stb_mlp_set_params(stb_mlp *p, const float *host) {
  return guarded([&] {
    if (!p || !host) throw Error(STB_EINVAL, "NULL argument");
    DeviceGuard g(p->device);
    cuda_check(cudaMemcpy(p->params, host, sizeof(float) * p->nparams, cudaMemcpyHostToDevice), "upload");
    cuda_check(cudaMemset(p->m, 0, sizeof(float) * p->nparams), "reset moments");
    cuda_check(cudaMemset(p->v, 0, sizeof(float) * p->nparams), "reset moments");
    p->step = 0;
    refresh_bf16(p);
    cuda_check(cudaStreamSynchronize(p->stream), "set params");
    return STB_OK;
  });
}

int stb_mlp_set_adamw(stb_mlp *p, float lr, float beta1, float beta2, float eps, float weight_decay) {
  return guarded([&] {
    if (!p) throw Error(STB_EINVAL, "NULL mlp");
    p->lr = lr;
    p->b1 = beta1;
    p->b2 = beta2;
    p->eps = eps;
    p->wd = weight_decay;
    return STB_OK;
  });
}

int stb_mlp_forward(stb_mlp *p, const float *x, int B, float *probs) {
  return guarded([&] {
    if (!p || !x || !probs) throw Error(STB_EINVAL, "NULL argument");
    check_batch(p, B);
    DeviceGuard g(p->device);
    forward(p, x, B);
    cuda_check(mlp_softmax_xent(p->logits, stb_mlp::kPadOut, nullptr, nullptr, B, p->nout, 1.0f, nullptr, probs,
                                nullptr, nullptr, stb_mlp::kPadOut, nullptr, p->stream),
               "softmax");
    cuda_check(cudaStreamSynchronize(p->stream), "mlp forward");
    int st = 0;
    cuda_check(cudaMemcpy(&st, p->status, sizeof(int), cudaMemcpyDeviceToHost), "status");
    if (st != 0) throw Error(st, "tcgen05 GEMM reported status " + std::to_string(st));
    return STB_OK;
  });
}

int stb_mlp_gradients(stb_mlp *p, const float *x, const int32_t *labels, const float *weights, int B,
                      float *loss_host) {
  return guarded([&] {
    if (!p || !x || !labels) throw Error(STB_EINVAL, "NULL argument");
    check_batch(p, B);
    DeviceGuard g(p->device);
    backward(p, x, labels, weights, B, loss_host);
    return STB_OK;
  });
}

int stb_mlp_train_step(stb_mlp *p, const float *x, const int32_t *labels, const float *weights, int B,
                       float *loss_host) {
  return guarded([&] {
    if (!p || !x || !labels) throw Error(STB_EINVAL, "NULL argument");
    check_batch(p, B);
    DeviceGuard g(p->device);
    backward(p, x, labels, weights, B, loss_host);
    adamw_step(p);
    return STB_OK;
  });
}

int stb_mlp_gemm_test(const void *A, int lda, const void *Bm, int ldb, int M, int N, int K, float *C, int ldc,
                      int device) {
  return guarded([&] {
    DeviceGuard g(device);
    int *status = nullptr;
    cuda_check(cudaMalloc(&status, sizeof(int)), "cudaMalloc(status)");
    DevFree f{status};
    cuda_check(cudaMemset(status, 0, sizeof(int)), "reset status");
    GemmArgs ga = gemm((const bf16 *)A, lda, (const bf16 *)Bm, ldb, M, N, K, EPI_F32, status);
    ga.C = C;
    ga.ldc = ldc;
    cuda_check(mlp_gemm_launch(ga, 0), "tcgen05 GEMM launch");
    cuda_check(cudaDeviceSynchronize(), "tcgen05 GEMM");
    int st = 0;
    cuda_check(cudaMemcpy(&st, status, sizeof(int), cudaMemcpyDeviceToHost), "status");
    if (st != 0) throw Error(st, "tcgen05 GEMM reported status " + std::to_string(st));
    return STB_OK;
  });
}

}  // extern "C"
