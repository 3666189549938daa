// Internal (C++) interfaces of the device ops; the exported C ABI wraps these.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "pytme_b200.h"

namespace tmb {

const char* last_error();

constexpr int kStatChunks = 64;  // partial-sum blocks per batch item in template_stats

int rigid_transform(const float* data, const float* mask, int d0, int d1, int d2,
                    const float* matrices, int n_mat, float* out, float* out_mask, int o0,
                    int o1, int o2, cudaStream_t stream);

// Order 3: interpolation coefficients (SciPy spline_filter, mirror boundary) and the
// pull interpolation from coefficient arrays.
int spline_prefilter(const float* in, double* coef, int d0, int d1, int d2, int batch,
                     cudaStream_t stream);
int to_double(const float* in, double* out, int64_t n, cudaStream_t stream);
int rigid_transform_cubic(const double* coef, const double* mcoef, int d0, int d1, int d2,
                          const float* matrices, int n_mat, float* out, float* out_mask, int o0,
                          int o1, int o2, cudaStream_t stream);

// Bins of the whitening filter for a data spectrum of rfft shape data_ft_shape
// (n_bins <= 0: the reference's default).
int whitening_bins(const int* data_ft_shape, int n_bins);
// Whitening filter from the complex64 rfft of the data; work: 3 * bins doubles; factor
// (optional) multiplies the result before the rounding to float32.
int whitening_filter(const float2* data_rfft, const int* data_ft_shape, int n_bins,
                     const int* shape, int rfft, double* work, const float* factor, float* out,
                     cudaStream_t stream);
int build_filter(const tm_filter_component* comps, int n_comp, const int* shape, int rfft,
                 float* out, cudaStream_t stream);

int64_t stats_workspace_bytes(int batch);
// stats layout per item: {mean, std, n_obs, 0} (double) after the partial sums
int template_stats(const float* x, const float* m, int64_t m_item_stride, int e0, int e1, int e2,
                   int o1, int o2, int64_t item_stride, int batch, double n_obs, double* ws,
                   cudaStream_t stream);
int normalize_template(float* x, const float* m, int64_t m_item_stride, int e0, int e1, int e2,
                       int o1, int o2, int64_t item_stride, int batch, double n_obs, double* ws,
                       cudaStream_t stream);

int norm_scores(const float* arr, const float* exp_sq, const float* sq_exp, double n_obs,
                const float* n_obs_dev, double eps, float* out, int64_t n, cudaStream_t stream);

int max_score_over_rotations(const float* scores, float* max_scores, int32_t* rotations,
                             int32_t index, int64_t n, cudaStream_t stream);

int complex_multiply(const void* a, const void* b, void* out, int64_t n, cudaStream_t stream);
int apply_real_filter(void* spectra, const float* filt, int64_t n, int batch, cudaStream_t stream);
int scale_real(float* x, float s, int64_t n, cudaStream_t stream);
int plain_epilogue(const float* x, const float* inv_den, const float* cc_m, const float* cc_m2,
                   const double* stats, double eps, float scale, float* mx, int32_t* rot,
                   int32_t index, int64_t n, cudaStream_t stream);
int pad_box(const float* src, int t0, int t1, int t2, float* dst, int n1, int n2,
            cudaStream_t stream);

}  // namespace tmb
