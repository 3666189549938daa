// Internal interface of the rotation-scan plan (scan.cu).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "pytme_b200.h"
#include "fft_smem.cuh"

namespace tmb {

struct Scan;

fft::LinePlan make_line_plan(int n);
int scan_create(const tm_scan_desc* desc, Scan** out);
int scan_destroy(Scan* s);
int64_t scan_device_bytes(const Scan* s);
int scan_set_template(Scan* s, const float* tmpl, const float* mask, const float* filt,
                      cudaStream_t stream);
int scan_set_target(Scan* s, const float* target, cudaStream_t stream);
int scan_set_interpolation(Scan* s, int order, cudaStream_t stream);
int scan_set_xpass(Scan* s, int mode);
int scan_xpass_mode(const Scan* s);
int scan_set_zpass(Scan* s, int mode);
int scan_zpass_mode(const Scan* s);
int scan_set_ypass(Scan* s, int mode);
int scan_ypass_mode(const Scan* s);
int scan_set_wait_budget(Scan* s, uint32_t iters);
// default poll budget of a tensor-core wait (tc_common.cuh kWaitIters)
uint32_t tc_wait_iters_default();
int scan_check(Scan* s, cudaStream_t stream);
int scan_run(Scan* s, const float* matrices, int n, int32_t first_index, float* state_max,
             int32_t* state_rot, cudaStream_t stream);
int scan_set_timing(Scan* s, int enable);
int scan_set_graph(Scan* s, int enable);
int scan_get_timing(const Scan* s, double* ms, int64_t* launches);
int64_t scan_stage_bytes(const Scan* s, int stage, int nb);
int line_fft_test(const void* x, void* y, int n, int lines, int dir, cudaStream_t stream);

}  // namespace tmb
