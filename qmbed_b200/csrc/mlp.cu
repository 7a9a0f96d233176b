// Fully connected ReLU network: forward, backward and Adam on the GPU.
//
// Layer l maps A_l (batch x d_l) to Z_l = A_l W_l + b_l with W_l stored
// row-major (d_l x d_{l+1}); hidden layers apply ReLU, the output layer is
// linear. The loss is the mean squared error over batch x outputs. Every
// product is one strided tiled GEMM kernel whose output elements each sum
// their k terms in a fixed order (no atomics), so a training run is bitwise
// reproducible. Adam follows Kingma and Ba (ICLR 2015, Algorithm 1).
#include <algorithm>
#include <cmath>
#include <numeric>

#include "mlp.cuh"

namespace qmbed {

namespace {

constexpr int kTile = 16;

enum Epilogue : int { kPlain = 0, kBiasRelu = 1, kBias = 2, kMask = 3 };

// C[m * N + n] = epilogue(sum_k A[m * sam + k * sak] * B[k * sbk + n * sbn])
__global__ void gemm_kernel(int M, int N, int K, const float* __restrict__ A, int64_t sam, int64_t sak,
                            const float* __restrict__ B, int64_t sbk, int64_t sbn, float* __restrict__ C,
                            const float* __restrict__ bias, const float* __restrict__ mask, int epilogue) {
  __shared__ float As[kTile][kTile + 1];
  __shared__ float Bs[kTile][kTile + 1];
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int m = blockIdx.y * kTile + ty, n = blockIdx.x * kTile + tx;
  float acc = 0.0f;
  for (int k0 = 0; k0 < K; k0 += kTile) {
    const int ka = k0 + tx, kb = k0 + ty;
    const int am = blockIdx.y * kTile + ty, bn = blockIdx.x * kTile + tx;
    As[ty][tx] = (am < M && ka < K) ? A[am * sam + ka * sak] : 0.0f;
    Bs[ty][tx] = (kb < K && bn < N) ? B[kb * sbk + bn * sbn] : 0.0f;
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < kTile; ++kk) acc = fmaf(As[ty][kk], Bs[kk][tx], acc);
    __syncthreads();
  }
  if (m < M && n < N) {
    float v = acc;
    if (epilogue == kBiasRelu || epilogue == kBias) v += bias[n];
    if (epilogue == kBiasRelu) v = v > 0.0f ? v : 0.0f;
    if (epilogue == kMask) v = mask[static_cast<int64_t>(m) * N + n] > 0.0f ? v : 0.0f;
    C[static_cast<int64_t>(m) * N + n] = v;
  }
}

// out[n] = sum_m D[m * N + n]
__global__ void colsum_kernel(int M, int N, const float* __restrict__ D, float* __restrict__ out) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.0f;
  for (int m = 0; m < M; ++m) s += D[static_cast<int64_t>(m) * N + n];
  out[n] = s;
}

// delta = 2 (yhat - y) / count, loss[0] = sum (yhat - y)^2 / count (one block)
__global__ void mse_kernel(int count, const float* __restrict__ yhat, const float* __restrict__ y,
                           float* __restrict__ delta, float* __restrict__ loss) {
  __shared__ float part[256];
  float s = 0.0f;
  for (int i = threadIdx.x; i < count; i += blockDim.x) {
    const float d = yhat[i] - y[i];
    delta[i] = 2.0f * d / static_cast<float>(count);
    s += d * d;
  }
  part[threadIdx.x] = s;
  __syncthreads();
  for (int o = blockDim.x / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) part[threadIdx.x] += part[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) loss[0] = part[0] / static_cast<float>(count);
}

__global__ void adam_kernel(size_t n, float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (size_t i = static_cast<size_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n;
       i += static_cast<size_t>(gridDim.x) * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

uint64_t splitmix(uint64_t& s) {
  uint64_t z = (s += 0x9e3779b97f4a7c15ULL);
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

double unit(uint64_t& s) { return static_cast<double>(splitmix(s) >> 11) * (1.0 / 9007199254740992.0); }

void gemm(cudaStream_t s, int M, int N, int K, const float* A, int64_t sam, int64_t sak, const float* B, int64_t sbk,
          int64_t sbn, float* C, const float* bias, const float* mask, int epilogue) {
  const dim3 block(kTile, kTile), grid((N + kTile - 1) / kTile, (M + kTile - 1) / kTile);
  gemm_kernel<<<grid, block, 0, s>>>(M, N, K, A, sam, sak, B, sbk, sbn, C, bias, mask, epilogue);
  QMBED_LAUNCH_CHECK();
}

}  // namespace

Mlp::Mlp(int device, int inputs, int outputs, int width, int hidden_layers, uint64_t seed)
    : device_(device), inputs_(inputs), outputs_(outputs), width_(width), layers_(hidden_layers + 1) {
  if (inputs < 1 || outputs < 1 || width < 1 || hidden_layers < 0 || inputs > 4096 || width > 4096 || outputs > 4096)
    raise(QMBED_INVALID_OPTIONS, "network sizes must be positive (at most 4096 per layer)");
  QMBED_CUDA(cudaSetDevice(device_));
  QMBED_CUDA(cudaStreamCreateWithFlags(&stream_, cudaStreamNonBlocking));
  dims_.push_back(inputs);
  for (int l = 0; l < hidden_layers; ++l) dims_.push_back(width);
  dims_.push_back(outputs);
  for (int l = 0; l < layers_; ++l) {
    w_off_.push_back(params_total_);
    params_total_ += static_cast<size_t>(dims_[l]) * dims_[l + 1];
    b_off_.push_back(params_total_);
    params_total_ += static_cast<size_t>(dims_[l + 1]);
  }
  // He-uniform weights, zero biases, from a splitmix64 stream of the seed
  std::vector<float> p(params_total_, 0.0f);
  uint64_t state = seed;
  for (int l = 0; l < layers_; ++l) {
    const double limit = std::sqrt(6.0 / dims_[l]);
    for (size_t i = 0; i < static_cast<size_t>(dims_[l]) * dims_[l + 1]; ++i)
      p[w_off_[l] + i] = static_cast<float>((2.0 * unit(state) - 1.0) * limit);
  }
  params_.allocate(params_total_ * sizeof(float));
  grads_.allocate(params_total_ * sizeof(float));
  adam_m_.allocate(params_total_ * sizeof(float));
  adam_v_.allocate(params_total_ * sizeof(float));
  loss_.allocate(sizeof(float));
  set_parameters(p.data());
  in_mean_.assign(inputs, 0.0f);
  in_std_.assign(inputs, 1.0f);
  out_mean_.assign(outputs, 0.0f);
  out_std_.assign(outputs, 1.0f);
}

Mlp::~Mlp() {
  if (stream_) cudaStreamDestroy(stream_);
}

void Mlp::get_scaling(float* in_mean, float* in_std, float* out_mean, float* out_std) const {
  std::copy(in_mean_.begin(), in_mean_.end(), in_mean);
  std::copy(in_std_.begin(), in_std_.end(), in_std);
  std::copy(out_mean_.begin(), out_mean_.end(), out_mean);
  std::copy(out_std_.begin(), out_std_.end(), out_std);
}

void Mlp::get_parameters(float* out) const {
  QMBED_CUDA(cudaSetDevice(device_));
  QMBED_CUDA(cudaMemcpyAsync(out, params_.get(), params_total_ * sizeof(float), cudaMemcpyDeviceToHost, stream_));
  QMBED_CUDA(cudaStreamSynchronize(stream_));
}

void Mlp::set_parameters(const float* in) {
  QMBED_CUDA(cudaSetDevice(device_));
  QMBED_CUDA(cudaMemcpyAsync(params_.get(), in, params_total_ * sizeof(float), cudaMemcpyHostToDevice, stream_));
  QMBED_CUDA(cudaStreamSynchronize(stream_));
}

void Mlp::set_scaling(const std::vector<float>& in_mean, const std::vector<float>& in_std,
                      const std::vector<float>& out_mean, const std::vector<float>& out_std) {
  if (static_cast<int>(in_mean.size()) != inputs_ || static_cast<int>(in_std.size()) != inputs_ ||
      static_cast<int>(out_mean.size()) != outputs_ || static_cast<int>(out_std.size()) != outputs_)
    raise(QMBED_DIMENSION_MISMATCH, "scaling vectors do not match the network");
  in_mean_ = in_mean;
  in_std_ = in_std;
  out_mean_ = out_mean;
  out_std_ = out_std;
}

void Mlp::ensure_batch(int n) {
  if (n <= batch_cap_) return;
  act_off_.assign(dims_.size(), 0);
  size_t total = 0;
  for (size_t l = 0; l < dims_.size(); ++l) {
    act_off_[l] = total;
    total += static_cast<size_t>(n) * dims_[l];
  }
  acts_.allocate(total * sizeof(float));
  deltas_.allocate(total * sizeof(float));
  io_.allocate(static_cast<size_t>(n) * outputs_ * sizeof(float));
  batch_cap_ = n;
}

void Mlp::forward(int n, const float* x_dev) {
  float* acts = acts_.as<float>();
  const float* p = params_.as<float>();
  QMBED_CUDA(cudaMemcpyAsync(acts + act_off_[0], x_dev, static_cast<size_t>(n) * inputs_ * sizeof(float),
                             cudaMemcpyDeviceToDevice, stream_));
  for (int l = 0; l < layers_; ++l) {
    const int din = dims_[l], dout = dims_[l + 1];
    gemm(stream_, n, dout, din, acts + act_off_[l], din, 1, p + w_off_[l], dout, 1, acts + act_off_[l + 1],
         p + b_off_[l], nullptr, l + 1 < layers_ ? kBiasRelu : kBias);
  }
}

float Mlp::loss_and_backward(int n, const float* y_dev) {
  float* acts = acts_.as<float>();
  float* deltas = deltas_.as<float>();
  const float* p = params_.as<float>();
  float* g = grads_.as<float>();
  const int L = layers_;
  mse_kernel<<<1, 256, 0, stream_>>>(n * outputs_, acts + act_off_[L], y_dev, deltas + act_off_[L], loss_.as<float>());
  QMBED_LAUNCH_CHECK();
  for (int l = L - 1; l >= 0; --l) {
    const int din = dims_[l], dout = dims_[l + 1];
    // dW_l = A_l^T delta_{l+1}, db_l = column sums of delta_{l+1}
    gemm(stream_, din, dout, n, acts + act_off_[l], 1, din, deltas + act_off_[l + 1], dout, 1, g + w_off_[l], nullptr,
         nullptr, kPlain);
    colsum_kernel<<<(dout + 127) / 128, 128, 0, stream_>>>(n, dout, deltas + act_off_[l + 1], g + b_off_[l]);
    QMBED_LAUNCH_CHECK();
    // delta_l = (delta_{l+1} W_l^T) masked by the ReLU of A_l (hidden layers only)
    if (l > 0)
      gemm(stream_, n, din, dout, deltas + act_off_[l + 1], dout, 1, p + w_off_[l], 1, dout, deltas + act_off_[l],
           nullptr, acts + act_off_[l], kMask);
  }
  float loss = 0.0f;
  QMBED_CUDA(cudaMemcpyAsync(&loss, loss_.get(), sizeof(float), cudaMemcpyDeviceToHost, stream_));
  QMBED_CUDA(cudaStreamSynchronize(stream_));
  return loss;
}

float Mlp::gradients(const float* X, const float* Y, int n, float* grads) {
  if (n < 1) raise(QMBED_INVALID_OPTIONS, "a batch needs at least one sample");
  QMBED_CUDA(cudaSetDevice(device_));
  ensure_batch(n);
  DeviceBuffer x(static_cast<size_t>(n) * inputs_ * sizeof(float)), y(static_cast<size_t>(n) * outputs_ * sizeof(float));
  QMBED_CUDA(cudaMemcpyAsync(x.get(), X, x.bytes(), cudaMemcpyHostToDevice, stream_));
  QMBED_CUDA(cudaMemcpyAsync(y.get(), Y, y.bytes(), cudaMemcpyHostToDevice, stream_));
  forward(n, x.as<float>());
  const float loss = loss_and_backward(n, y.as<float>());
  QMBED_CUDA(cudaMemcpyAsync(grads, grads_.get(), params_total_ * sizeof(float), cudaMemcpyDeviceToHost, stream_));
  QMBED_CUDA(cudaStreamSynchronize(stream_));
  return loss;
}

float Mlp::train(const float* X, const float* Y, int n, int epochs, int batch, float lr, uint64_t seed) {
  if (n < 2 || epochs < 1 || batch < 1 || !(lr > 0.0f)) raise(QMBED_INVALID_OPTIONS, "training needs n >= 2, epochs, batch and lr > 0");
  QMBED_CUDA(cudaSetDevice(device_));
  batch = std::min(batch, n);
  // fit the scaling to the data
  auto fit = [&](const float* data, int cols, std::vector<float>& mean, std::vector<float>& sd) {
    mean.assign(cols, 0.0f);
    sd.assign(cols, 1.0f);
    for (int c = 0; c < cols; ++c) {
      double s = 0.0, s2 = 0.0;
      for (int i = 0; i < n; ++i) {
        const double v = data[static_cast<size_t>(i) * cols + c];
        s += v;
        s2 += v * v;
      }
      const double m = s / n, var = std::max(s2 / n - m * m, 0.0);
      mean[c] = static_cast<float>(m);
      sd[c] = static_cast<float>(std::max(std::sqrt(var), 1.0e-6));
    }
  };
  fit(X, inputs_, in_mean_, in_std_);
  fit(Y, outputs_, out_mean_, out_std_);
  std::vector<float> xs(static_cast<size_t>(n) * inputs_), ys(static_cast<size_t>(n) * outputs_);
  for (int i = 0; i < n; ++i) {
    for (int c = 0; c < inputs_; ++c)
      xs[static_cast<size_t>(i) * inputs_ + c] = (X[static_cast<size_t>(i) * inputs_ + c] - in_mean_[c]) / in_std_[c];
    for (int c = 0; c < outputs_; ++c)
      ys[static_cast<size_t>(i) * outputs_ + c] = (Y[static_cast<size_t>(i) * outputs_ + c] - out_mean_[c]) / out_std_[c];
  }
  ensure_batch(n);
  DeviceBuffer dx(xs.size() * sizeof(float)), dy(ys.size() * sizeof(float));
  QMBED_CUDA(cudaMemsetAsync(adam_m_.get(), 0, params_total_ * sizeof(float), stream_));
  QMBED_CUDA(cudaMemsetAsync(adam_v_.get(), 0, params_total_ * sizeof(float), stream_));
  std::vector<int> order(n);
  std::iota(order.begin(), order.end(), 0);
  std::vector<float> px(xs.size()), py(ys.size());
  uint64_t state = seed;
  const float b1 = 0.9f, b2 = 0.999f, eps = 1.0e-8f;
  double p1 = 1.0, p2 = 1.0;
  const int grid = static_cast<int>(std::min<size_t>((params_total_ + 255) / 256, 1024));
  for (int epoch = 0; epoch < epochs; ++epoch) {
    for (int i = n - 1; i > 0; --i) std::swap(order[i], order[splitmix(state) % static_cast<uint64_t>(i + 1)]);
    for (int i = 0; i < n; ++i) {
      std::copy_n(xs.begin() + static_cast<size_t>(order[i]) * inputs_, inputs_, px.begin() + static_cast<size_t>(i) * inputs_);
      std::copy_n(ys.begin() + static_cast<size_t>(order[i]) * outputs_, outputs_, py.begin() + static_cast<size_t>(i) * outputs_);
    }
    QMBED_CUDA(cudaMemcpyAsync(dx.get(), px.data(), dx.bytes(), cudaMemcpyHostToDevice, stream_));
    QMBED_CUDA(cudaMemcpyAsync(dy.get(), py.data(), dy.bytes(), cudaMemcpyHostToDevice, stream_));
    // cosine learning-rate decay over the run
    const float rate = lr * static_cast<float>(0.5 * (1.0 + std::cos(3.141592653589793 * epoch / epochs)));
    for (int start = 0; start + batch <= n; start += batch) {
      forward(batch, dx.as<float>() + static_cast<size_t>(start) * inputs_);
      float* acts = acts_.as<float>();
      float* deltas = deltas_.as<float>();
      const int count = batch * outputs_;
      mse_kernel<<<1, 256, 0, stream_>>>(count, acts + act_off_[layers_],
                                         dy.as<float>() + static_cast<size_t>(start) * outputs_,
                                         deltas + act_off_[layers_], loss_.as<float>());
      QMBED_LAUNCH_CHECK();
      const float* p = params_.as<float>();
      float* g = grads_.as<float>();
      for (int l = layers_ - 1; l >= 0; --l) {
        const int din = dims_[l], dout = dims_[l + 1];
        gemm(stream_, din, dout, batch, acts + act_off_[l], 1, din, deltas + act_off_[l + 1], dout, 1, g + w_off_[l],
             nullptr, nullptr, kPlain);
        colsum_kernel<<<(dout + 127) / 128, 128, 0, stream_>>>(batch, dout, deltas + act_off_[l + 1], g + b_off_[l]);
        QMBED_LAUNCH_CHECK();
        if (l > 0)
          gemm(stream_, batch, din, dout, deltas + act_off_[l + 1], dout, 1, p + w_off_[l], 1, dout,
               deltas + act_off_[l], nullptr, acts + act_off_[l], kMask);
      }
      p1 *= b1;
      p2 *= b2;
      adam_kernel<<<grid, 256, 0, stream_>>>(params_total_, params_.as<float>(), grads_.as<float>(),
                                             adam_m_.as<float>(), adam_v_.as<float>(), rate, b1, b2, eps,
                                             static_cast<float>(1.0 - p1), static_cast<float>(1.0 - p2));
      QMBED_LAUNCH_CHECK();
    }
  }
  // final full-batch loss in network units
  QMBED_CUDA(cudaMemcpyAsync(dx.get(), xs.data(), dx.bytes(), cudaMemcpyHostToDevice, stream_));
  QMBED_CUDA(cudaMemcpyAsync(dy.get(), ys.data(), dy.bytes(), cudaMemcpyHostToDevice, stream_));
  forward(n, dx.as<float>());
  return loss_and_backward(n, dy.as<float>());
}

void Mlp::predict(const float* X, int n, float* Y) {
  if (n < 1) return;
  QMBED_CUDA(cudaSetDevice(device_));
  ensure_batch(n);
  std::vector<float> xs(static_cast<size_t>(n) * inputs_), ys(static_cast<size_t>(n) * outputs_);
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < inputs_; ++c)
      xs[static_cast<size_t>(i) * inputs_ + c] = (X[static_cast<size_t>(i) * inputs_ + c] - in_mean_[c]) / in_std_[c];
  DeviceBuffer dx(xs.size() * sizeof(float));
  QMBED_CUDA(cudaMemcpyAsync(dx.get(), xs.data(), dx.bytes(), cudaMemcpyHostToDevice, stream_));
  forward(n, dx.as<float>());
  QMBED_CUDA(cudaMemcpyAsync(ys.data(), acts_.as<float>() + act_off_[layers_], ys.size() * sizeof(float),
                             cudaMemcpyDeviceToHost, stream_));
  QMBED_CUDA(cudaStreamSynchronize(stream_));
  for (int i = 0; i < n; ++i)
    for (int c = 0; c < outputs_; ++c)
      Y[static_cast<size_t>(i) * outputs_ + c] = ys[static_cast<size_t>(i) * outputs_ + c] * out_std_[c] + out_mean_[c];
}

}  // namespace qmbed
