// Learned solver settings: a small multilayer perceptron (in -> h1 -> h2 ->
// out, ReLU hidden layers, softmax output) that maps matrix features to a
// choice of solver settings (partition count, coupled / decoupled SPIKE).
// Training and inference run on the GPU with the kernels below; there is no
// library GEMM: the layers are a few thousand multiply-adds per sample.
//
// Every kernel is deterministic (no atomics): one thread per output value,
// sums in a fixed order.  Parameters are FP32, row-major W[o][i].
#include <cuda_runtime.h>

#include <cmath>
#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/sap_b200.h"
#include "common.cuh"

namespace sapb {

// y[b][o] = act(sum_i W[o][i] x[b][i] + bias[o]); act = ReLU when relu
static __global__ void k_dense_fwd(const float* __restrict__ W, const float* __restrict__ bias,
                                   const float* __restrict__ x, float* __restrict__ y, int batch, int in, int out,
                                   int relu) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= batch * out) return;
  const int b = t / out, o = t % out;
  float s = bias[o];
  for (int i = 0; i < in; i++) s += W[o * in + i] * x[b * in + i];
  y[t] = relu ? fmaxf(s, 0.f) : s;
}

// dx[b][i] = (sum_o W[o][i] dy[b][o]) * (relu'(x) when mask)
static __global__ void k_dense_bwd_x(const float* __restrict__ W, const float* __restrict__ dy,
                                     const float* __restrict__ xact, float* __restrict__ dx, int batch, int in,
                                     int out, int mask) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= batch * in) return;
  const int b = t / in, i = t % in;
  float s = 0.f;
  for (int o = 0; o < out; o++) s += W[o * in + i] * dy[b * out + o];
  dx[t] = (mask && xact[t] <= 0.f) ? 0.f : s;
}

// dW[o][i] = sum_b dy[b][o] x[b][i];  db[o] = sum_b dy[b][o]
static __global__ void k_dense_bwd_w(const float* __restrict__ dy, const float* __restrict__ x, float* __restrict__ dW,
                                     float* __restrict__ db, int batch, int in, int out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t < out * in) {
    const int o = t / in, i = t % in;
    float s = 0.f;
    for (int b = 0; b < batch; b++) s += dy[b * out + o] * x[b * in + i];
    dW[t] = s;
  } else if (t < out * in + out) {
    const int o = t - out * in;
    float s = 0.f;
    for (int b = 0; b < batch; b++) s += dy[b * out + o];
    db[o] = s;
  }
}

// softmax cross-entropy: dlogits = (softmax - onehot) / batch, loss[b]
static __global__ void k_softmax_ce(const float* __restrict__ logits, const int* __restrict__ label,
                                    float* __restrict__ dlogits, float* __restrict__ loss, int batch, int out) {
  const int b = blockIdx.x * blockDim.x + threadIdx.x;
  if (b >= batch) return;
  const float* z = logits + b * out;
  float m = z[0];
  for (int o = 1; o < out; o++) m = fmaxf(m, z[o]);
  float se = 0.f;
  for (int o = 0; o < out; o++) se += expf(z[o] - m);
  const float lse = m + logf(se);
  loss[b] = lse - z[label[b]];
  for (int o = 0; o < out; o++) {
    const float p = expf(z[o] - lse);
    dlogits[b * out + o] = (p - (o == label[b] ? 1.f : 0.f)) / (float)batch;
  }
}

// Adam (Kingma & Ba 2015) on a flat parameter vector
static __global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                              float* __restrict__ v, int n, float lr, float b1, float b2, float eps, float c1,
                              float c2) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= n) return;
  m[t] = b1 * m[t] + (1.f - b1) * g[t];
  v[t] = b2 * v[t] + (1.f - b2) * g[t] * g[t];
  p[t] -= lr * (m[t] / c1) / (sqrtf(v[t] / c2) + eps);
}

struct Mlp {
  int in = 0, h1 = 0, h2 = 0, out = 0;
  int nparam = 0;
  DBuf<float> prm, grd, am, av;  // flat: W1 b1 W2 b2 W3 b3
  DBuf<float> x, a1, a2, z, d1, d2, dz, loss;
  DBuf<int> lab;
  int cap = 0;
  int step = 0;
  cudaStream_t st = nullptr;
  float* W1() { return prm.get(); }
  float* B1() { return W1() + h1 * in; }
  float* W2() { return B1() + h1; }
  float* B2() { return W2() + h2 * h1; }
  float* W3() { return B2() + h2; }
  float* B3() { return W3() + out * h2; }
  float* G(int k) {  // gradient slice of parameter block k (same layout)
    const int off[6] = {0, h1 * in, h1 * in + h1, h1 * in + h1 + h2 * h1, h1 * in + h1 + h2 * h1 + h2,
                        h1 * in + h1 + h2 * h1 + h2 + out * h2};
    return grd.get() + off[k];
  }
  void ensure(int batch) {
    if (batch <= cap) return;
    cap = batch;
    x.alloc((size_t)batch * in);
    a1.alloc((size_t)batch * h1);
    a2.alloc((size_t)batch * h2);
    z.alloc((size_t)batch * out);
    d1.alloc((size_t)batch * h1);
    d2.alloc((size_t)batch * h2);
    dz.alloc((size_t)batch * out);
    loss.alloc(batch);
    lab.alloc(batch);
  }
  static int g(int n) { return (n + 127) / 128; }
  void forward(int batch) {
    k_dense_fwd<<<g(batch * h1), 128, 0, st>>>(W1(), B1(), x.get(), a1.get(), batch, in, h1, 1);
    SAPB_LAUNCHED();
    k_dense_fwd<<<g(batch * h2), 128, 0, st>>>(W2(), B2(), a1.get(), a2.get(), batch, h1, h2, 1);
    SAPB_LAUNCHED();
    k_dense_fwd<<<g(batch * out), 128, 0, st>>>(W3(), B3(), a2.get(), z.get(), batch, h2, out, 0);
    SAPB_LAUNCHED();
  }
  void backward(int batch) {
    k_softmax_ce<<<g(batch), 128, 0, st>>>(z.get(), lab.get(), dz.get(), loss.get(), batch, out);
    SAPB_LAUNCHED();
    k_dense_bwd_w<<<g(out * h2 + out), 128, 0, st>>>(dz.get(), a2.get(), G(4), G(5), batch, h2, out);
    SAPB_LAUNCHED();
    k_dense_bwd_x<<<g(batch * h2), 128, 0, st>>>(W3(), dz.get(), a2.get(), d2.get(), batch, h2, out, 1);
    SAPB_LAUNCHED();
    k_dense_bwd_w<<<g(h2 * h1 + h2), 128, 0, st>>>(d2.get(), a1.get(), G(2), G(3), batch, h1, h2);
    SAPB_LAUNCHED();
    k_dense_bwd_x<<<g(batch * h1), 128, 0, st>>>(W2(), d2.get(), a1.get(), d1.get(), batch, h1, h2, 1);
    SAPB_LAUNCHED();
    k_dense_bwd_w<<<g(h1 * in + h1), 128, 0, st>>>(d1.get(), x.get(), G(0), G(1), batch, in, h1);
    SAPB_LAUNCHED();
  }
};

}  // namespace sapb

using namespace sapb;

struct sap_mlp {
  Mlp m;
};

static thread_local std::string g_mlp_error;

#define MLP_TRY(...)                                    \
  try {                                                 \
    __VA_ARGS__;                                        \
    return SAP_OK;                                      \
  } catch (const sapb::Error& e) {                      \
    g_mlp_error = e.what();                             \
    return e.code;                                      \
  } catch (const std::exception& e) {                   \
    g_mlp_error = e.what();                             \
    return SAP_ERR_CUDA;                                \
  }

extern "C" {

const char* sap_mlp_last_error(void) { return g_mlp_error.c_str(); }

int sap_mlp_create(int in, int h1, int h2, int out, uint64_t seed, sap_mlp** res) {
  MLP_TRY({
    if (!res || in <= 0 || h1 <= 0 || h2 <= 0 || out <= 1 || in > 4096 || h1 > 4096 || h2 > 4096 || out > 4096)
      throw Error(SAP_ERR_INVALID_ARGUMENT, "invalid network shape");
    auto h = std::make_unique<sap_mlp>();
    Mlp& m = h->m;
    m.in = in;
    m.h1 = h1;
    m.h2 = h2;
    m.out = out;
    m.nparam = h1 * in + h1 + h2 * h1 + h2 + out * h2 + out;
    // He-uniform initial weights from a splitmix64 stream, zero biases
    std::vector<float> p(m.nparam, 0.f);
    uint64_t s = seed;
    auto next = [&]() {
      uint64_t z = (s += 0x9E3779B97F4A7C15ull);
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      z ^= z >> 31;
      return (double)(z >> 11) / 9007199254740992.0;
    };
    auto fill = [&](int off, int rows, int cols) {
      const double lim = std::sqrt(6.0 / cols);
      for (int k = 0; k < rows * cols; k++) p[off + k] = (float)((2.0 * next() - 1.0) * lim);
    };
    fill(0, h1, in);
    fill(h1 * in + h1, h2, h1);
    fill(h1 * in + h1 + h2 * h1 + h2, out, h2);
    m.prm.upload(p, nullptr);
    m.grd.alloc(m.nparam);
    m.am.alloc(m.nparam);
    m.av.alloc(m.nparam);
    m.am.zero(nullptr);
    m.av.zero(nullptr);
    SAPB_CUDA(cudaDeviceSynchronize());
    *res = h.release();
  });
}

int sap_mlp_destroy(sap_mlp* h) {
  delete h;
  return SAP_OK;
}

int sap_mlp_num_params(const sap_mlp* h) { return h ? h->m.nparam : 0; }

// Parameters as one host float array (W1 b1 W2 b2 W3 b3, W row-major [out][in]).
int sap_mlp_get_params(sap_mlp* h, float* out) {
  MLP_TRY({
    if (!h || !out) throw Error(SAP_ERR_INVALID_ARGUMENT, "null argument");
    SAPB_CUDA(cudaMemcpy(out, h->m.prm.get(), sizeof(float) * h->m.nparam, cudaMemcpyDeviceToHost));
  });
}

int sap_mlp_set_params(sap_mlp* h, const float* in) {
  MLP_TRY({
    if (!h || !in) throw Error(SAP_ERR_INVALID_ARGUMENT, "null argument");
    SAPB_CUDA(cudaMemcpy(h->m.prm.get(), in, sizeof(float) * h->m.nparam, cudaMemcpyHostToDevice));
  });
}

// logits[batch][out] for host features x[batch][in]
int sap_mlp_forward(sap_mlp* h, const float* x, int batch, float* logits) {
  MLP_TRY({
    if (!h || !x || !logits || batch <= 0) throw Error(SAP_ERR_INVALID_ARGUMENT, "invalid argument");
    Mlp& m = h->m;
    m.ensure(batch);
    SAPB_CUDA(cudaMemcpy(m.x.get(), x, sizeof(float) * batch * m.in, cudaMemcpyHostToDevice));
    m.forward(batch);
    SAPB_CUDA(cudaMemcpy(logits, m.z.get(), sizeof(float) * batch * m.out, cudaMemcpyDeviceToHost));
  });
}

// Mean cross-entropy loss and its gradient (flat, the parameter layout).
int sap_mlp_gradients(sap_mlp* h, const float* x, const int* labels, int batch, float* grads, float* loss) {
  MLP_TRY({
    if (!h || !x || !labels || batch <= 0) throw Error(SAP_ERR_INVALID_ARGUMENT, "invalid argument");
    Mlp& m = h->m;
    m.ensure(batch);
    for (int b = 0; b < batch; b++)
      if (labels[b] < 0 || labels[b] >= m.out) throw Error(SAP_ERR_INVALID_ARGUMENT, "label out of range");
    SAPB_CUDA(cudaMemcpy(m.x.get(), x, sizeof(float) * batch * m.in, cudaMemcpyHostToDevice));
    SAPB_CUDA(cudaMemcpy(m.lab.get(), labels, sizeof(int) * batch, cudaMemcpyHostToDevice));
    m.forward(batch);
    m.backward(batch);
    if (grads) SAPB_CUDA(cudaMemcpy(grads, m.grd.get(), sizeof(float) * m.nparam, cudaMemcpyDeviceToHost));
    if (loss) {
      std::vector<float> l(batch);
      SAPB_CUDA(cudaMemcpy(l.data(), m.loss.get(), sizeof(float) * batch, cudaMemcpyDeviceToHost));
      double s = 0;
      for (float v : l) s += v;
      *loss = (float)(s / batch);
    }
  });
}

// `epochs` full-batch Adam steps on (x, labels); returns the final mean loss.
int sap_mlp_train(sap_mlp* h, const float* x, const int* labels, int batch, int epochs, float lr, float* loss) {
  MLP_TRY({
    if (!h || !x || !labels || batch <= 0 || epochs < 0) throw Error(SAP_ERR_INVALID_ARGUMENT, "invalid argument");
    Mlp& m = h->m;
    m.ensure(batch);
    for (int b = 0; b < batch; b++)
      if (labels[b] < 0 || labels[b] >= m.out) throw Error(SAP_ERR_INVALID_ARGUMENT, "label out of range");
    SAPB_CUDA(cudaMemcpy(m.x.get(), x, sizeof(float) * batch * m.in, cudaMemcpyHostToDevice));
    SAPB_CUDA(cudaMemcpy(m.lab.get(), labels, sizeof(int) * batch, cudaMemcpyHostToDevice));
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int e = 0; e < epochs; e++) {
      m.forward(batch);
      m.backward(batch);
      m.step++;
      const float c1 = 1.f - std::pow(b1, (float)m.step), c2 = 1.f - std::pow(b2, (float)m.step);
      k_adam<<<Mlp::g(m.nparam), 128, 0, m.st>>>(m.prm.get(), m.grd.get(), m.am.get(), m.av.get(), m.nparam, lr, b1,
                                                 b2, eps, c1, c2);
      SAPB_LAUNCHED();
    }
    m.forward(batch);
    k_softmax_ce<<<Mlp::g(batch), 128, 0, m.st>>>(m.z.get(), m.lab.get(), m.dz.get(), m.loss.get(), batch, m.out);
    SAPB_LAUNCHED();
    std::vector<float> l(batch);
    SAPB_CUDA(cudaMemcpy(l.data(), m.loss.get(), sizeof(float) * batch, cudaMemcpyDeviceToHost));
    double s = 0;
    for (float v : l) s += v;
    if (loss) *loss = (float)(s / batch);
  });
}

}  // extern "C"
