// H.v on device buffers without any device allocation.
//
// The regular entry point (qmbed_gpu_operator_apply_device) allocates, on its
// first call for a symmetry sector with stored rows, a device vector holding
// x / sqrt(R) (R = orbit size). Some callers cannot let a library call
// cudaMalloc: applications that own all device memory through their own pool
// and budget, and latency-critical loops that must not pay the implicit device
// synchronisation of cudaMalloc/cudaFree. For them, the variant below takes
// that vector from a fixed array in this file instead.
#include <functional>
#include <mutex>
#include <string>

#include "../../include/qmbed_b200.h"
#include "operator.cuh"

namespace qmbed {
int noalloc_guarded(const std::function<void()>& body);
}

struct qmbed_operator_s;

namespace {

// 32 MiB of scratch, reserved in global memory of every GPU on which this
// library's device code is loaded, and held until the process exits. It
// bounds the input vector of symmetry sectors with stored rows: dimension x
// (2 if complex) x (8 for FP64, 4 for FP32) bytes.
constexpr size_t kNoAllocScratchBytes = size_t{1} << 25;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mutex;
void* g_scratch_address[kMaxDevices] = {};

// The device address of g_noalloc_scratch on `device`. In host code the
// symbol's name is only a host-side stand-in, so the address is looked up
// once per device, with that device current, and cached.
void* scratch_address(int device) {
  if (device < 0 || device >= kMaxDevices) qmbed::raise(qmbed::QMBED_INVALID_OPTIONS, "device index out of range");
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (!g_scratch_address[device]) {
    QMBED_CUDA(cudaSetDevice(device));
    void* address = nullptr;
    const cudaError_t status = cudaGetSymbolAddress(&address, g_noalloc_scratch);
    if (status != cudaSuccess || address == nullptr)
      qmbed::raise(qmbed::QMBED_CUDA_ERROR,
                   std::string("cudaGetSymbolAddress(g_noalloc_scratch): ") + cudaGetErrorString(status));
    g_scratch_address[device] = address;
  }
  return g_scratch_address[device];
}

}  // namespace

namespace qmbed {
const SpinOperator& operator_of(qmbed_operator_s* op);
}

extern "C" int qmbed_gpu_operator_apply_device_noalloc(qmbed_operator op, int precision, int complex_vectors,
                                                       const void* x, void* y, void* stream) {
  return qmbed::noalloc_guarded([&] {
    if (precision != 64 && precision != 32) qmbed::raise(qmbed::QMBED_INVALID_OPTIONS, "precision must be 64 or 32");
    const qmbed::SpinOperator& H = qmbed::operator_of(op);
    // The size limit applies where the scratch is used (symmetry sectors with
    // stored rows); apply_with_scratch checks it there.
    void* scratch = scratch_address(H.basis().device());
    H.apply_with_scratch(precision, complex_vectors != 0, x, y, static_cast<cudaStream_t>(stream), scratch,
                         kNoAllocScratchBytes);
  });
}
