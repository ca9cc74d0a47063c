// ops.cu -- small element-wise device helpers of the C ABI.
#include <cuda_runtime.h>

#include <algorithm>

#include "device.h"

namespace emg {
namespace {

__global__ void k_axpby(double* __restrict__ out, double a, const double* __restrict__ x, double b,
                        const double* __restrict__ y, int64_t n) {
  for (int64_t i = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x; i < n;
       i += static_cast<int64_t>(gridDim.x) * blockDim.x)
    out[i] = a * x[i] + b * y[i];
}

}  // namespace

int axpby_values(double* out, double a, const double* x, double b, const double* y, int64_t n,
                 cudaStream_t st) {
  if (n <= 0) return EMG_SUCCESS;
  const int grid = static_cast<int>(std::min<int64_t>((n + 255) / 256, 148 * 16));
  k_axpby<<<grid, 256, 0, st>>>(out, a, x, b, y, n);
  EMG_CK(cudaGetLastError());
  EMG_CK(cudaStreamSynchronize(st));
  return EMG_SUCCESS;
}

}  // namespace emg
