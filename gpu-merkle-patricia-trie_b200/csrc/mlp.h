// mlp.h -- the schedule selector's network: a two-hidden-layer ReLU MLP in
// fp32 with hand-written CUDA inference, gradient and Adam training kernels.
//
// Parameters, flat: W1[H][I] b1[H] W2[H][H] b2[H] W3[O][H] b3[O].
// Loss over a set of samples: sum over (s, o) of M[s][o] * (y[s][o] - T[s][o])^2
// divided by sum of M (masked mean squared error: a sample carries a target
// only for the outputs that were measured).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>
#include <vector>

namespace gmpt {

constexpr int kMlpMaxIn = 16, kMlpMaxHidden = 64, kMlpMaxOut = 16;

class Mlp {
 public:
  Mlp(int device, int n_in, int n_hidden, int n_out, uint64_t seed);
  ~Mlp();
  Mlp(const Mlp &) = delete;
  Mlp &operator=(const Mlp &) = delete;

  int n_params() const { return np_; }
  int get_params(float *out);
  int set_params(const float *in);  // also clears the Adam state
  // y[n][O] for x[n][I] (host arrays)
  int forward(const float *x, int n, float *y);
  // masked-MSE loss and its gradient over all n samples (host arrays)
  int loss_grad(const float *x, const float *t, const float *m, int n, float *loss, float *grad);
  // Adam (beta1 0.9, beta2 0.999, eps 1e-8): `epochs` passes over the n
  // samples in mini-batches of `batch` (<= 64), in a per-epoch order fixed by
  // `seed` (mlp_epoch_order); one kernel launch.  *loss = mean mini-batch
  // loss of the last epoch.
  int train(const float *x, const float *t, const float *m, int n, int epochs, int batch, float lr, uint64_t seed,
            float *loss);
  uint64_t adam_steps() const { return steps_; }
  const std::string &error() const { return err_; }

 private:
  int dev_ = 0, I_ = 0, H_ = 0, O_ = 0, np_ = 0;
  uint64_t steps_ = 0;
  float *d_p_ = nullptr, *d_m_ = nullptr, *d_v_ = nullptr;
  float *d_buf_ = nullptr;
  size_t buf_floats_ = 0;
  std::string err_;
  int fail(const std::string &msg);
  int stage(const float *const *src, const size_t *counts, int k, float **dst);
};

// Position -> sample index of one training epoch: positions j of [0, P),
// P = 2^ceil(log2 n), map to (a * j + b) mod P with a odd (a bijection of
// [0, P)); images >= n are skipped.  a, b come from splitmix64 of
// (seed, epoch).  Shared by the kernel and the host so the order is testable.
__host__ __device__ inline uint64_t mlp_splitmix(uint64_t x) {
  x += 0x9E3779B97F4A7C15ull;
  x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
  x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
  return x ^ (x >> 31);
}

}  // namespace gmpt
