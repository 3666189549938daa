// Internal interface of the peak-calling kernels (peaks.cu).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace tmb {

int max_filter_peaks(const float* scores, int n0, int n1, int n2, int size, float* tmp_a,
                     float* tmp_b, uint8_t* mask, cudaStream_t stream);
int64_t nms_workspace_bytes(int n);
int greedy_nms(const int64_t* coords, int n, int64_t min_distance, int32_t* out_idx,
               int32_t* out_count, void* workspace, cudaStream_t stream);

}  // namespace tmb
