// Tensor-core trailing update of the FP32 LU (tcgen05, sm_100a).
// This header provides the buffers and the dispatch hook used by mixed.cuh;
// tc_update returns false when the tensor-core path is not taken, in which
// case the caller runs the FP32 SIMT update.
#pragma once
#include <cuda_runtime.h>

#include "linalg.cuh"

namespace nb200 {

struct TcWork {
  size_t total = 0;
  size_t bytes() const { return total; }
  void release() { total = 0; }
  cudaError_t ensure(int, int) { return cudaSuccess; }
};

inline size_t tc_bytes_per_system(size_t) { return 0; }

inline bool tc_update(TcWork&, BatchT<float2>, int, int, int, cudaStream_t, long long&) { return false; }

}  // namespace nb200
