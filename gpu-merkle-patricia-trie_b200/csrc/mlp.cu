// mlp.cu -- fp32 MLP kernels of the schedule selector (inference, masked-MSE
// gradient, Adam training) and their host wrapper.
//
// The network is tiny (<= 16 inputs, <= 64 hidden, <= 16 outputs, < 6.3k
// parameters), so one CTA holds the parameters, the Adam moments, the
// gradient and a 64-sample mini-batch's activations in shared memory and runs
// whole training epochs in a single launch.  Each gradient element is owned by
// one thread (no atomics): mini-batch reductions are loops over the samples in
// shared memory.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "mlp.h"

namespace gmpt {

void count_launch();

namespace {

constexpr int kMlpThreads = 256;
constexpr int kMlpMB = 64;

struct MlpDims {
  int I, H, O;
  __host__ __device__ int w1() const { return 0; }
  __host__ __device__ int b1() const { return H * I; }
  __host__ __device__ int w2() const { return H * I + H; }
  __host__ __device__ int b2() const { return H * I + H + H * H; }
  __host__ __device__ int w3() const { return H * I + 2 * H + H * H; }
  __host__ __device__ int b3() const { return H * I + 2 * H + H * H + O * H; }
  __host__ __device__ int np() const { return H * I + 2 * H + H * H + O * H + O; }
};

__host__ __device__ inline void epoch_ab(uint64_t seed, int epoch, uint64_t P, uint64_t &a, uint64_t &b) {
  const uint64_t h = mlp_splitmix(seed ^ (0x632BE59BD9B4E019ull * (uint64_t)(epoch + 1)));
  a = (h | 1ull) & (P - 1);
  if (a == 0) a = 1;
  b = mlp_splitmix(h) & (P - 1);
}

struct MlpSmem {
  float *P, *G, *Mo, *Vo;  // params, gradient, Adam moments
  float *X, *A1, *A2, *Y, *T, *M;
  int *sidx;
  float *red;
};

__device__ MlpSmem carve(float *base, MlpDims d, bool adam) {
  MlpSmem S;
  const int np = d.np();
  float *p = base;
  S.P = p;
  p += np;
  S.G = p;
  p += np;
  if (adam) {
    S.Mo = p;
    p += np;
    S.Vo = p;
    p += np;
  } else {
    S.Mo = S.Vo = nullptr;
  }
  S.X = p;
  p += kMlpMB * d.I;
  S.A1 = p;
  p += kMlpMB * d.H;
  S.A2 = p;
  p += kMlpMB * d.H;
  S.Y = p;
  p += kMlpMB * d.O;
  S.T = p;
  p += kMlpMB * d.O;
  S.M = p;
  p += kMlpMB * d.O;
  S.red = p;
  p += 64;
  S.sidx = reinterpret_cast<int *>(p);
  return S;
}

size_t smem_floats(MlpDims d, bool adam) {
  return (size_t)d.np() * (adam ? 4 : 2) + kMlpMB * (d.I + 2 * d.H + 3 * d.O) + 64 + kMlpMB;
}

__device__ float block_sum(float v, float *red) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  __syncthreads();
  if (lane == 0) red[w] = v;
  __syncthreads();
  if (w == 0) {
    v = lane < (int)(blockDim.x >> 5) ? red[lane] : 0.f;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) red[32] = v;
  }
  __syncthreads();
  return red[32];
}

// Forward + backward of the cnt samples S.sidx[0..cnt) of (X, T, M); adds
// the gradient of  norm * sum M (y - t)^2  to S.G (norm <= 0: 1 / sum M of
// this mini-batch).  Returns the unnormalised loss sum and the mask sum.
__device__ void mb_grad(const MlpSmem &S, MlpDims d, const float *X, const float *T, const float *M, int cnt,
                        float norm_in, float *loss_sum, float *mask_sum) {
  const int tid = threadIdx.x, nt = blockDim.x;
  const int I = d.I, H = d.H, O = d.O;
  const float *P = S.P;
  float *G = S.G;
  for (int e = tid; e < cnt * I; e += nt) S.X[e] = X[(size_t)S.sidx[e / I] * I + e % I];
  for (int e = tid; e < cnt * O; e += nt) {
    const size_t g = (size_t)S.sidx[e / O] * O + e % O;
    S.T[e] = T[g];
    S.M[e] = M[g];
  }
  __syncthreads();
  for (int e = tid; e < cnt * H; e += nt) {
    const int s = e / H, h = e % H;
    float z = P[d.b1() + h];
    for (int i = 0; i < I; ++i) z += P[d.w1() + h * I + i] * S.X[s * I + i];
    S.A1[e] = fmaxf(z, 0.f);
  }
  __syncthreads();
  for (int e = tid; e < cnt * H; e += nt) {
    const int s = e / H, h = e % H;
    float z = P[d.b2() + h];
    for (int k = 0; k < H; ++k) z += P[d.w2() + h * H + k] * S.A1[s * H + k];
    S.A2[e] = fmaxf(z, 0.f);
  }
  __syncthreads();
  for (int e = tid; e < cnt * O; e += nt) {
    const int s = e / O, o = e % O;
    float z = P[d.b3() + o];
    for (int h = 0; h < H; ++h) z += P[d.w3() + o * H + h] * S.A2[s * H + h];
    S.Y[e] = z;
  }
  __syncthreads();
  float ls = 0.f, ms = 0.f;
  for (int e = tid; e < cnt * O; e += nt) {
    const float r = S.Y[e] - S.T[e];
    ls += S.M[e] * r * r;
    ms += S.M[e];
  }
  ls = block_sum(ls, S.red);
  ms = block_sum(ms, S.red);
  const float norm = norm_in > 0.f ? norm_in : (ms > 0.f ? 1.f / ms : 0.f);
  for (int e = tid; e < cnt * O; e += nt) S.Y[e] = 2.f * norm * S.M[e] * (S.Y[e] - S.T[e]);  // dL/dy
  __syncthreads();
  for (int p = tid; p < O * H + O; p += nt) {
    float g = 0.f;
    if (p < O * H) {
      const int o = p / H, h = p % H;
      for (int s = 0; s < cnt; ++s) g += S.Y[s * O + o] * S.A2[s * H + h];
      G[d.w3() + p] += g;
    } else {
      const int o = p - O * H;
      for (int s = 0; s < cnt; ++s) g += S.Y[s * O + o];
      G[d.b3() + o] += g;
    }
  }
  __syncthreads();
  for (int e = tid; e < cnt * H; e += nt) {  // dZ2 over A2 (ReLU mask from A2 itself)
    const int s = e / H, h = e % H;
    float v = 0.f;
    if (S.A2[e] > 0.f)
      for (int o = 0; o < O; ++o) v += S.Y[s * O + o] * P[d.w3() + o * H + h];
    S.A2[e] = v;
  }
  __syncthreads();
  for (int p = tid; p < H * H + H; p += nt) {
    float g = 0.f;
    if (p < H * H) {
      const int h = p / H, k = p % H;
      for (int s = 0; s < cnt; ++s) g += S.A2[s * H + h] * S.A1[s * H + k];
      G[d.w2() + p] += g;
    } else {
      const int h = p - H * H;
      for (int s = 0; s < cnt; ++s) g += S.A2[s * H + h];
      G[d.b2() + h] += g;
    }
  }
  __syncthreads();
  for (int e = tid; e < cnt * H; e += nt) {  // dZ1 over A1
    const int s = e / H, k = e % H;
    float v = 0.f;
    if (S.A1[e] > 0.f)
      for (int h = 0; h < H; ++h) v += S.A2[s * H + h] * P[d.w2() + h * H + k];
    S.A1[e] = v;
  }
  __syncthreads();
  for (int p = tid; p < H * I + H; p += nt) {
    float g = 0.f;
    if (p < H * I) {
      const int h = p / I, i = p % I;
      for (int s = 0; s < cnt; ++s) g += S.A1[s * H + h] * S.X[s * I + i];
      G[d.w1() + p] += g;
    } else {
      const int h = p - H * I;
      for (int s = 0; s < cnt; ++s) g += S.A1[s * H + h];
      G[d.b1() + h] += g;
    }
  }
  __syncthreads();
  *loss_sum = ls;
  *mask_sum = ms;
}

__global__ void __launch_bounds__(kMlpThreads) k_mlp_forward(const float *P, const float *X, int n, MlpDims d,
                                                             float *Y) {
  extern __shared__ float sp[];
  for (int p = threadIdx.x; p < d.np(); p += blockDim.x) sp[p] = P[p];
  __syncthreads();
  const int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s >= n) return;
  float a1[kMlpMaxHidden], a2[kMlpMaxHidden];
  for (int h = 0; h < d.H; ++h) {
    float z = sp[d.b1() + h];
    for (int i = 0; i < d.I; ++i) z += sp[d.w1() + h * d.I + i] * X[(size_t)s * d.I + i];
    a1[h] = fmaxf(z, 0.f);
  }
  for (int h = 0; h < d.H; ++h) {
    float z = sp[d.b2() + h];
    for (int k = 0; k < d.H; ++k) z += sp[d.w2() + h * d.H + k] * a1[k];
    a2[h] = fmaxf(z, 0.f);
  }
  for (int o = 0; o < d.O; ++o) {
    float z = sp[d.b3() + o];
    for (int h = 0; h < d.H; ++h) z += sp[d.w3() + o * d.H + h] * a2[h];
    Y[(size_t)s * d.O + o] = z;
  }
}

__global__ void __launch_bounds__(kMlpThreads) k_mlp_grad(const float *P, const float *X, const float *T,
                                                          const float *M, int n, MlpDims d, float norm, float *G_out,
                                                          float *loss_out) {
  extern __shared__ float smem[];
  MlpSmem S = carve(smem, d, false);
  for (int p = threadIdx.x; p < d.np(); p += blockDim.x) {
    S.P[p] = P[p];
    S.G[p] = 0.f;
  }
  __syncthreads();
  float loss = 0.f;
  for (int base = 0; base < n; base += kMlpMB) {
    const int cnt = min(kMlpMB, n - base);
    for (int s = threadIdx.x; s < cnt; s += blockDim.x) S.sidx[s] = base + s;
    __syncthreads();
    float ls, ms;
    mb_grad(S, d, X, T, M, cnt, norm, &ls, &ms);
    loss += ls;
  }
  for (int p = threadIdx.x; p < d.np(); p += blockDim.x) G_out[p] = S.G[p];
  if (threadIdx.x == 0) *loss_out = loss * norm;
}

__global__ void __launch_bounds__(kMlpThreads) k_mlp_train(float *P, float *Mo, float *Vo, const float *X,
                                                           const float *T, const float *M, int n, MlpDims d,
                                                           int epochs, int batch, float lr, uint64_t seed,
                                                           double b1p, double b2p, float *loss_out) {
  extern __shared__ float smem[];
  MlpSmem S = carve(smem, d, true);
  __shared__ int sh_cnt;
  __shared__ unsigned long long sh_j;
  const int np = d.np();
  for (int p = threadIdx.x; p < np; p += blockDim.x) {
    S.P[p] = P[p];
    S.Mo[p] = Mo[p];
    S.Vo[p] = Vo[p];
  }
  __syncthreads();
  uint64_t P2 = 1;
  while (P2 < (uint64_t)n) P2 <<= 1;
  float last = 0.f;
  for (int ep = 0; ep < epochs; ++ep) {
    uint64_t a, b;
    epoch_ab(seed, ep, P2, a, b);
    float ep_loss = 0.f;
    int nmb = 0;
    uint64_t j = 0;
    while (true) {
      if (threadIdx.x == 0) {
        int c = 0;
        while (c < batch && j < P2) {
          const uint64_t idx = (a * j + b) & (P2 - 1);
          ++j;
          if (idx < (uint64_t)n) S.sidx[c++] = (int)idx;
        }
        sh_cnt = c;
        sh_j = j;
      }
      __syncthreads();
      const int cnt = sh_cnt;
      j = sh_j;
      if (cnt == 0) break;
      for (int p = threadIdx.x; p < np; p += blockDim.x) S.G[p] = 0.f;
      __syncthreads();
      float ls, ms;
      mb_grad(S, d, X, T, M, cnt, -1.f, &ls, &ms);
      ep_loss += ms > 0.f ? ls / ms : 0.f;
      ++nmb;
      b1p *= 0.9;
      b2p *= 0.999;
      const float c1 = (float)(1.0 - b1p), c2 = (float)(1.0 - b2p);
      for (int p = threadIdx.x; p < np; p += blockDim.x) {
        const float g = S.G[p];
        const float m = 0.9f * S.Mo[p] + 0.1f * g;
        const float v = 0.999f * S.Vo[p] + 0.001f * g * g;
        S.Mo[p] = m;
        S.Vo[p] = v;
        S.P[p] -= lr * (m / c1) / (sqrtf(v / c2) + 1e-8f);
      }
      __syncthreads();
    }
    last = nmb ? ep_loss / (float)nmb : 0.f;
  }
  for (int p = threadIdx.x; p < np; p += blockDim.x) {
    P[p] = S.P[p];
    Mo[p] = S.Mo[p];
    Vo[p] = S.Vo[p];
  }
  if (threadIdx.x == 0) *loss_out = last;
}

}  // namespace

Mlp::Mlp(int device, int n_in, int n_hidden, int n_out, uint64_t seed)
    : dev_(device), I_(n_in), H_(n_hidden), O_(n_out) {
  if (n_in < 1 || n_in > kMlpMaxIn || n_hidden < 1 || n_hidden > kMlpMaxHidden || n_out < 1 || n_out > kMlpMaxOut) {
    err_ = "mlp dimensions out of range (inputs <= 16, hidden <= 64, outputs <= 8)";
    return;
  }
  MlpDims d{I_, H_, O_};
  np_ = d.np();
  // He-uniform weights from a splitmix64 stream, zero biases
  std::vector<float> p(np_, 0.f);
  uint64_t st = seed;
  auto uni = [&]() {
    st = mlp_splitmix(st);
    return (double)(st >> 11) * (1.0 / 9007199254740992.0);
  };
  auto fill = [&](int off, int count, int fan_in) {
    const double lim = std::sqrt(6.0 / fan_in);
    for (int k = 0; k < count; ++k) p[off + k] = (float)((2.0 * uni() - 1.0) * lim);
  };
  fill(d.w1(), H_ * I_, I_);
  fill(d.w2(), H_ * H_, H_);
  fill(d.w3(), O_ * H_, H_);
  cudaError_t e = cudaSetDevice(dev_);
  if (e == cudaSuccess) e = cudaMalloc(&d_p_, sizeof(float) * np_);
  if (e == cudaSuccess) e = cudaMalloc(&d_m_, sizeof(float) * np_);
  if (e == cudaSuccess) e = cudaMalloc(&d_v_, sizeof(float) * np_);
  if (e == cudaSuccess) e = cudaMemcpy(d_p_, p.data(), sizeof(float) * np_, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemset(d_m_, 0, sizeof(float) * np_);
  if (e == cudaSuccess) e = cudaMemset(d_v_, 0, sizeof(float) * np_);
  if (e != cudaSuccess) err_ = std::string("mlp init: ") + cudaGetErrorString(e);
}

Mlp::~Mlp() {
  cudaSetDevice(dev_);
  for (float *q : {d_p_, d_m_, d_v_, d_buf_})
    if (q) cudaFree(q);
}

int Mlp::fail(const std::string &msg) {
  err_ = msg;
  return 1;
}

// copy k host float arrays into one device buffer; dst[i] = their device copies
int Mlp::stage(const float *const *src, const size_t *counts, int k, float **dst) {
  size_t total = 0;
  for (int i = 0; i < k; ++i) total += (counts[i] + 63) & ~size_t(63);
  if (total > buf_floats_) {
    if (d_buf_) cudaFree(d_buf_);
    d_buf_ = nullptr;
    buf_floats_ = 0;
    if (cudaMalloc(&d_buf_, sizeof(float) * total) != cudaSuccess) return fail("mlp buffer: out of device memory");
    buf_floats_ = total;
  }
  size_t at = 0;
  for (int i = 0; i < k; ++i) {
    dst[i] = d_buf_ + at;
    if (counts[i] &&
        cudaMemcpy(dst[i], src[i], sizeof(float) * counts[i], cudaMemcpyHostToDevice) != cudaSuccess)
      return fail("mlp copy");
    at += (counts[i] + 63) & ~size_t(63);
  }
  return 0;
}

int Mlp::get_params(float *out) {
  cudaSetDevice(dev_);
  return cudaMemcpy(out, d_p_, sizeof(float) * np_, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : fail("mlp copy");
}

int Mlp::set_params(const float *in) {
  cudaSetDevice(dev_);
  if (cudaMemcpy(d_p_, in, sizeof(float) * np_, cudaMemcpyHostToDevice) != cudaSuccess) return fail("mlp copy");
  cudaMemset(d_m_, 0, sizeof(float) * np_);
  cudaMemset(d_v_, 0, sizeof(float) * np_);
  steps_ = 0;
  return 0;
}

int Mlp::forward(const float *x, int n, float *y) {
  if (n <= 0) return 0;
  cudaSetDevice(dev_);
  std::vector<float> zeros((size_t)n * O_, 0.f);
  const float *src[2] = {x, zeros.data()};
  size_t cnt[2] = {(size_t)n * I_, (size_t)n * O_};
  float *d[2];
  if (stage(src, cnt, 2, d)) return 1;
  MlpDims dm{I_, H_, O_};
  count_launch(), k_mlp_forward<<<(n + kMlpThreads - 1) / kMlpThreads, kMlpThreads, sizeof(float) * np_>>>(
      d_p_, d[0], n, dm, d[1]);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(y, d[1], sizeof(float) * n * O_, cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? 0 : fail(std::string("mlp forward: ") + cudaGetErrorString(e));
}

int Mlp::loss_grad(const float *x, const float *t, const float *m, int n, float *loss, float *grad) {
  cudaSetDevice(dev_);
  double msum = 0;
  for (size_t i = 0; i < (size_t)n * O_; ++i) msum += m[i];
  const float norm = msum > 0 ? (float)(1.0 / msum) : 0.f;
  const float *src[4] = {x, t, m, nullptr};
  size_t cnt[4] = {(size_t)n * I_, (size_t)n * O_, (size_t)n * O_, (size_t)np_ + 64};
  float *d[4];
  std::vector<float> zeros(cnt[3], 0.f);
  src[3] = zeros.data();
  if (stage(src, cnt, 4, d)) return 1;
  MlpDims dm{I_, H_, O_};
  const size_t smem = sizeof(float) * smem_floats(dm, false);
  if (cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return fail("mlp grad smem");
  count_launch(), k_mlp_grad<<<1, kMlpThreads, smem>>>(d_p_, d[0], d[1], d[2], n, dm, norm, d[3], d[3] + np_);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(grad, d[3], sizeof(float) * np_, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(loss, d[3] + np_, sizeof(float), cudaMemcpyDeviceToHost);
  return e == cudaSuccess ? 0 : fail(std::string("mlp grad: ") + cudaGetErrorString(e));
}

int Mlp::train(const float *x, const float *t, const float *m, int n, int epochs, int batch, float lr, uint64_t seed,
               float *loss) {
  if (n <= 0 || epochs <= 0) return 0;
  if (batch < 1 || batch > kMlpMB) return fail("mlp train: batch must be in [1, 64]");
  cudaSetDevice(dev_);
  const float *src[4] = {x, t, m, nullptr};
  std::vector<float> zero(64, 0.f);
  src[3] = zero.data();
  size_t cnt[4] = {(size_t)n * I_, (size_t)n * O_, (size_t)n * O_, 64};
  float *d[4];
  if (stage(src, cnt, 4, d)) return 1;
  MlpDims dm{I_, H_, O_};
  const size_t smem = sizeof(float) * smem_floats(dm, true);
  if (cudaFuncSetAttribute(k_mlp_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
    return fail("mlp train smem");
  const double b1p = std::pow(0.9, (double)steps_), b2p = std::pow(0.999, (double)steps_);
  count_launch(), k_mlp_train<<<1, kMlpThreads, smem>>>(d_p_, d_m_, d_v_, d[0], d[1], d[2], n, dm, epochs, batch, lr,
                                                       seed, b1p, b2p, d[3]);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(loss, d[3], sizeof(float), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return fail(std::string("mlp train: ") + cudaGetErrorString(e));
  steps_ += (uint64_t)epochs * (uint64_t)((n + batch - 1) / batch);
  return 0;
}

}  // namespace gmpt
