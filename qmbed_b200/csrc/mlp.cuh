// A small fully connected ReLU network (default 4 hidden layers of 128) that
// maps model parameters to spectral bounds, trained and evaluated on the GPU by
// this library's own kernels (FP32 parameters and activations, FP32
// accumulation in a fixed order, so results are bitwise reproducible).
#pragma once

#include <cstdint>
#include <vector>

#include "common.cuh"

namespace qmbed {

class Mlp {
 public:
  Mlp(int device, int inputs, int outputs, int width, int hidden_layers, uint64_t seed);
  ~Mlp();
  Mlp(const Mlp&) = delete;
  Mlp& operator=(const Mlp&) = delete;

  int inputs() const { return inputs_; }
  int outputs() const { return outputs_; }
  size_t parameter_count() const { return params_total_; }
  // Flattened parameters: per linear map, W (in x out, row-major) then b (out).
  void get_parameters(float* out) const;
  void set_parameters(const float* in);
  // Affine scaling of inputs and outputs: net input = (x - in_mean) / in_std,
  // prediction = net output * out_std + out_mean. Identity by default.
  void set_scaling(const std::vector<float>& in_mean, const std::vector<float>& in_std,
                   const std::vector<float>& out_mean, const std::vector<float>& out_std);
  void get_scaling(float* in_mean, float* in_std, float* out_mean, float* out_std) const;
  // Mean squared error of the network on (X, Y) in network units (no scaling)
  // and its gradient with respect to every parameter (flattened like above).
  float gradients(const float* X, const float* Y, int n, float* grads);
  // Adam training on scaled data; the scaling is fitted to (X, Y) first.
  // Returns the final full-batch loss in network units.
  float train(const float* X, const float* Y, int n, int epochs, int batch, float lr, uint64_t seed);
  // Predictions in physical units for host inputs.
  void predict(const float* X, int n, float* Y);

 private:
  void forward(int n, const float* x_dev);  // network units
  float loss_and_backward(int n, const float* y_dev);
  void ensure_batch(int n);

  int device_, inputs_, outputs_, width_, layers_;  // layers_ = linear maps
  std::vector<int> dims_;                           // layer widths, inputs .. outputs
  std::vector<size_t> w_off_, b_off_;
  size_t params_total_ = 0;
  DeviceBuffer params_, grads_, adam_m_, adam_v_;
  DeviceBuffer acts_, deltas_, io_, loss_;
  int batch_cap_ = 0;
  std::vector<size_t> act_off_;
  std::vector<float> in_mean_, in_std_, out_mean_, out_std_;
  cudaStream_t stream_ = nullptr;
};

}  // namespace qmbed
