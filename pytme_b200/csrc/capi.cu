// Exported C ABI (include/pytme_b200.h). Thin wrappers over the internal ops;
// argument checking lives here and in the ops.
#include "common.cuh"
#include "diagnostics.h"
#include "ops.cuh"
#include "peaks.cuh"
#include "refine.cuh"
#include "scan.cuh"
#include "xcorr_tc.cuh"

#include <cufft.h>

#include <string>

struct tm_fft_plan {
  cufftHandle fwd = 0, inv = 0;
  bool dbl = false;
  int64_t n_real = 0;   // elements per real array (all batches)
  int64_t n_item = 0;   // real elements per batch item
  int64_t n_ft = 0;     // complex elements per batch item
  int batch = 1;
};

struct tm_scan {
  tmb::Scan* impl = nullptr;
};

static cudaStream_t S(void* s) { return static_cast<cudaStream_t>(s); }

static tmb::RefineArgs refine_args(const tm_refine_desc* d) {
  tmb::RefineArgs a;
  a.tmpl = d->tmpl;
  a.mask = d->mask;
  a.rot = d->rot;
  a.shifts = d->shifts;
  a.corners = d->corners;
  a.P = d->n_peaks;
  a.target = d->target;
  a.eps = d->eps;
  a.outside = d->target_outside;
  for (int i = 0; i < 3; ++i) {
    a.t[i] = d->template_shape[i];
    a.n[i] = d->target_shape[i];
  }
  return a;
}

extern "C" {

int tm_version(void) { return 100; }

int tm_set_device_memory_limit(int64_t bytes) {
  tmb::set_device_memory_limit(bytes);
  return TM_OK;
}

int tm_last_error(char* buf, size_t len) {
  const char* msg = tmb::last_error();
  size_t n = strlen(msg);
  if (buf && len > 0) {
    size_t c = n < len - 1 ? n : len - 1;
    memcpy(buf, msg, c);
    buf[c] = '\0';
  }
  return (int)n;
}

int tm_rigid_transform(const float* data, const float* mask, int d0, int d1, int d2,
                       const float* matrices, int n_mat, float* out, float* out_mask, int o0,
                       int o1, int o2, void* stream) {
  return tmb::rigid_transform(data, mask, d0, d1, d2, matrices, n_mat, out, out_mask, o0, o1, o2,
                             S(stream));
}

int tm_spline_prefilter(const float* in, double* coef, int d0, int d1, int d2, int batch,
                        void* stream) {
  TM_REQUIRE(in, "tm_spline_prefilter: null input");
  return tmb::spline_prefilter(in, coef, d0, d1, d2, batch, S(stream));
}

int tm_rigid_transform_cubic(const double* coef, const double* mask_coef, int d0, int d1,
                             int d2, const float* matrices, int n_mat, float* out,
                             float* out_mask, int o0, int o1, int o2, void* stream) {
  return tmb::rigid_transform_cubic(coef, mask_coef, d0, d1, d2, matrices, n_mat, out, out_mask,
                                   o0, o1, o2, S(stream));
}

int64_t tm_normalize_template_workspace(int batch) {
  return batch > 0 ? tmb::stats_workspace_bytes(batch) : 0;
}

int tm_normalize_template(float* x, const float* mask, int64_t n, int batch,
                          int64_t mask_batch_stride, double n_obs, void* workspace,
                          void* stream) {
  TM_REQUIRE(x && mask && workspace, "tm_normalize_template: null pointer");
  TM_REQUIRE(n > 0 && n <= (int64_t)INT32_MAX && batch > 0,
             "tm_normalize_template: bad size n=%lld batch=%d", (long long)n, batch);
  TM_REQUIRE(mask_batch_stride == 0 || mask_batch_stride == n,
             "tm_normalize_template: mask_batch_stride must be 0 or n");
  return tmb::normalize_template(x, mask, mask_batch_stride, 1, 1, (int)n, 1, (int)n, n, batch,
                                n_obs, static_cast<double*>(workspace), S(stream));
}

int tm_norm_scores(const float* arr, const float* exp_sq, const float* sq_exp, double n_obs,
                   const float* n_obs_dev, double eps, float* out, int64_t n, void* stream) {
  TM_REQUIRE(n_obs_dev || n_obs > 0, "tm_norm_scores: n_obs must be positive");
  return tmb::norm_scores(arr, exp_sq, sq_exp, n_obs, n_obs_dev, eps, out, n, S(stream));
}

int tm_max_score_over_rotations(const float* scores, float* max_scores, int32_t* rotations,
                                int32_t rotation_index, int64_t n, void* stream) {
  return tmb::max_score_over_rotations(scores, max_scores, rotations, rotation_index, n,
                                      S(stream));
}

// ------------------------------------------------------------------ FFT plans
int tm_fft_plan_create(int ndim, const int* shape, int batch, int double_precision,
                       tm_fft_plan** plan) {
  TM_REQUIRE(plan && shape, "tm_fft_plan_create: null pointer");
  TM_REQUIRE(ndim >= 1 && ndim <= 3, "tm_fft_plan_create: ndim must be 1..3");
  TM_REQUIRE(batch >= 1, "tm_fft_plan_create: batch must be >= 1");
  *plan = nullptr;
  int n[3];
  int64_t nr = 1;
  for (int i = 0; i < ndim; ++i) {
    TM_REQUIRE(shape[i] > 0, "tm_fft_plan_create: shape must be positive");
    n[i] = shape[i];
    nr *= shape[i];
  }
  tm_fft_plan* p = new tm_fft_plan();
  p->dbl = double_precision != 0;
  p->n_real = nr * batch;
  p->n_item = nr;
  p->n_ft = nr / n[ndim - 1] * (n[ndim - 1] / 2 + 1);
  p->batch = batch;
  cufftResult r = cufftPlanMany(&p->fwd, ndim, n, nullptr, 1, 0, nullptr, 1, 0,
                                p->dbl ? CUFFT_D2Z : CUFFT_R2C, batch);
  if (r == CUFFT_SUCCESS)
    r = cufftPlanMany(&p->inv, ndim, n, nullptr, 1, 0, nullptr, 1, 0,
                      p->dbl ? CUFFT_Z2D : CUFFT_C2R, batch);
  if (r != CUFFT_SUCCESS) {
    tmb::set_error("tm_fft_plan_create: cuFFT error %d", (int)r);
    delete p;
    return r == CUFFT_ALLOC_FAILED ? TM_E_OOM : TM_E_CUFFT;
  }
  *plan = p;
  return TM_OK;
}

int tm_fft_plan_destroy(tm_fft_plan* p) {
  if (!p) return TM_OK;
  cufftDestroy(p->fwd);
  cufftDestroy(p->inv);
  delete p;
  return TM_OK;
}

int tm_fft_r2c(tm_fft_plan* p, const void* in, void* out, void* stream) {
  TM_REQUIRE(p && in && out, "tm_fft_r2c: null pointer");
  cufftSetStream(p->fwd, S(stream));
  cufftResult r = p->dbl ? cufftExecD2Z(p->fwd, (cufftDoubleReal*)in, (cufftDoubleComplex*)out)
                         : cufftExecR2C(p->fwd, (cufftReal*)in, (cufftComplex*)out);
  if (r != CUFFT_SUCCESS) { tmb::set_error("tm_fft_r2c: cuFFT error %d", (int)r); return TM_E_CUFFT; }
  return tmb::check_launch("tm_fft_r2c");
}

__global__ static void scale_d_kernel(double* x, double s, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] *= s;
}

int tm_fft_c2r(tm_fft_plan* p, void* in, void* out, double scale, void* stream) {
  TM_REQUIRE(p && in && out, "tm_fft_c2r: null pointer");
  cufftSetStream(p->inv, S(stream));
  cufftResult r = p->dbl ? cufftExecZ2D(p->inv, (cufftDoubleComplex*)in, (cufftDoubleReal*)out)
                         : cufftExecC2R(p->inv, (cufftComplex*)in, (cufftReal*)out);
  if (r != CUFFT_SUCCESS) { tmb::set_error("tm_fft_c2r: cuFFT error %d", (int)r); return TM_E_CUFFT; }
  if (scale != 1.0) {
    if (p->dbl) {
      int64_t blocks = tmb::ceil_div(p->n_real, 256);
      if (blocks > 148 * 16) blocks = 148 * 16;
      scale_d_kernel<<<(unsigned)blocks, 256, 0, S(stream)>>>((double*)out, scale, p->n_real);
    } else {
      TM_TRY(tmb::scale_real((float*)out, (float)scale, p->n_real, S(stream)));
    }
  }
  return tmb::check_launch("tm_fft_c2r");
}

// ------------------------------------------------------------------ scan
int tm_scan_create(const tm_scan_desc* desc, tm_scan** plan) {
  TM_REQUIRE(plan, "tm_scan_create: null plan pointer");
  *plan = nullptr;
  tmb::Scan* impl = nullptr;
  TM_TRY(tmb::scan_create(desc, &impl));
  *plan = new tm_scan{impl};
  return TM_OK;
}

int tm_scan_destroy(tm_scan* plan) {
  if (!plan) return TM_OK;
  tmb::scan_destroy(plan->impl);
  delete plan;
  return TM_OK;
}

int64_t tm_scan_device_bytes(const tm_scan* plan) {
  return plan ? tmb::scan_device_bytes(plan->impl) : 0;
}

int tm_scan_set_template(tm_scan* plan, const float* template_rev, const float* mask_rev,
                         const float* template_filter, void* stream) {
  TM_REQUIRE(plan, "tm_scan_set_template: null plan");
  return tmb::scan_set_template(plan->impl, template_rev, mask_rev, template_filter, S(stream));
}

int tm_scan_set_target(tm_scan* plan, const float* target, void* stream) {
  TM_REQUIRE(plan, "tm_scan_set_target: null plan");
  return tmb::scan_set_target(plan->impl, target, S(stream));
}

int tm_scan_set_interpolation(tm_scan* plan, int order, void* stream) {
  TM_REQUIRE(plan, "tm_scan_set_interpolation: null plan");
  return tmb::scan_set_interpolation(plan->impl, order, S(stream));
}

int tm_scan_set_xpass(tm_scan* plan, int mode) {
  TM_REQUIRE(plan, "tm_scan_set_xpass: null plan");
  return tmb::scan_set_xpass(plan->impl, mode);
}

int tm_scan_xpass_mode(const tm_scan* plan) {
  return plan ? tmb::scan_xpass_mode(plan->impl) : TM_E_INVALID;
}

int tm_scan_set_zpass(tm_scan* plan, int mode) {
  TM_REQUIRE(plan, "tm_scan_set_zpass: null plan");
  return tmb::scan_set_zpass(plan->impl, mode);
}

int tm_scan_zpass_mode(const tm_scan* plan) {
  return plan ? tmb::scan_zpass_mode(plan->impl) : TM_E_INVALID;
}

int tm_scan_set_ypass(tm_scan* plan, int mode) {
  TM_REQUIRE(plan, "tm_scan_set_ypass: null plan");
  return tmb::scan_set_ypass(plan->impl, mode);
}

int tm_scan_ypass_mode(const tm_scan* plan) {
  return plan ? tmb::scan_ypass_mode(plan->impl) : TM_E_INVALID;
}

int tm_scan_set_wait_budget(tm_scan* plan, uint32_t iters) {
  TM_REQUIRE(plan, "tm_scan_set_wait_budget: null plan");
  return tmb::scan_set_wait_budget(plan->impl, iters);
}

int tm_scan_check(tm_scan* plan, void* stream) {
  TM_REQUIRE(plan, "tm_scan_check: null plan");
  return tmb::scan_check(plan->impl, S(stream));
}

int tm_scan_run(tm_scan* plan, const float* matrices, int n, int32_t first_index,
                float* max_scores, int32_t* argmax, void* stream) {
  TM_REQUIRE(plan, "tm_scan_run: null plan");
  return tmb::scan_run(plan->impl, matrices, n, first_index, max_scores, argmax, S(stream));
}

int tm_scan_set_timing(tm_scan* plan, int enable) {
  TM_REQUIRE(plan, "tm_scan_set_timing: null plan");
  return tmb::scan_set_timing(plan->impl, enable);
}

int tm_scan_set_graph(tm_scan* plan, int enable) {
  TM_REQUIRE(plan, "tm_scan_set_graph: null plan");
  return tmb::scan_set_graph(plan->impl, enable);
}

int tm_scan_get_timing(const tm_scan* plan, double* ms, int64_t* launches) {
  TM_REQUIRE(plan, "tm_scan_get_timing: null plan");
  return tmb::scan_get_timing(plan->impl, ms, launches);
}

int64_t tm_scan_stage_bytes(const tm_scan* plan, int stage, int nb) {
  return plan ? tmb::scan_stage_bytes(plan->impl, stage, nb) : 0;
}

int tm_max_filter_peaks(const float* scores, int n0, int n1, int n2, int size, float* tmp_a,
                        float* tmp_b, uint8_t* mask, void* stream) {
  return tmb::max_filter_peaks(scores, n0, n1, n2, size, tmp_a, tmp_b, mask, S(stream));
}

int64_t tm_find_candidate_indices_workspace(int n) { return tmb::nms_workspace_bytes(n); }

int tm_find_candidate_indices(const int64_t* coords, int n, int64_t min_distance,
                              int32_t* out_idx, int32_t* out_count, void* workspace,
                              void* stream) {
  return tmb::greedy_nms(coords, n, min_distance, out_idx, out_count, workspace, S(stream));
}

int tm_xcorr_tc_test(const void* G, const void* C, int nb, int t0, int n0, int n1, int h2,
                     float scale, void* H, int half, void* stream) {
  TM_REQUIRE(G && C && H, "tm_xcorr_tc_test: null pointer");
  tmb::XcorrTcConfig cfg;
  TM_TRY(tmb::xcorr_tc_config(n0, t0, nb, &cfg));
  if (!cfg.ok) {
    tmb::set_error("tm_xcorr_tc_test: configuration n0=%d t0=%d nb=%d not supported", n0, t0, nb);
    return TM_E_UNSUPPORTED;
  }
  // the scan's layout: output rows padded to a multiple of 8 elements, then copied to the
  // caller's unpadded rows
  const int hp = (h2 + 7) / 8 * 8;
  const size_t esz = half ? 4 : 8;
  const size_t rows = (size_t)nb * n0 * n1;
  int* err = nullptr;
  void* Hp = nullptr;
  TM_TRY(tmb::cuda_status(cudaMalloc((void**)&err, sizeof(int)), "tm_xcorr_tc_test: alloc"));
  if (cudaMalloc(&Hp, rows * hp * esz) != cudaSuccess) {
    cudaGetLastError();
    cudaFree(err);
    tmb::set_error("tm_xcorr_tc_test: out of device memory");
    return TM_E_OOM;
  }
  cudaMemsetAsync(err, 0, sizeof(int), S(stream));
  int st = tmb::xcorr_tc_run(cfg, (const float2*)G, (const float2*)C, nb, t0, n0, n1, h2, hp,
                             scale, Hp, half != 0, err, S(stream));
  int herr = 0;
  if (st == TM_OK)
    st = tmb::cuda_status(cudaMemcpy2DAsync(H, h2 * esz, Hp, hp * esz, h2 * esz, rows,
                                            cudaMemcpyDeviceToDevice, S(stream)),
                          "tm_xcorr_tc_test: copy");
  if (st == TM_OK) {
    cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, S(stream));
    st = tmb::cuda_status(cudaStreamSynchronize(S(stream)), "tm_xcorr_tc_test");
  }
  cudaFree(Hp);
  cudaFree(err);
  if (st == TM_OK && herr) {
    tmb::set_error("tm_xcorr_tc_test: tensor-core wait timed out");
    st = TM_E_TIMEOUT;
  }
  return st;
}

int tm_line_fft_test(const void* x, void* y, int n, int lines, int dir, void* stream) {
  TM_REQUIRE(x && y, "tm_line_fft_test: null pointer");
  return tmb::line_fft_test(x, y, n, lines, dir, S(stream));
}


// ------------------------------------------------------------------ FFT filter
int tm_fft_filter(tm_fft_plan* p, float* x, void* spectrum, const float* filter, void* stream) {
  TM_REQUIRE(p && x && spectrum && filter, "tm_fft_filter: null pointer");
  TM_REQUIRE(!p->dbl, "tm_fft_filter: single-precision plans only");
  TM_TRY(tm_fft_r2c(p, x, spectrum, stream));
  TM_TRY(tmb::apply_real_filter(spectrum, filter, p->n_ft, p->batch, S(stream)));
  return tm_fft_c2r(p, spectrum, x, 1.0 / (double)p->n_item, stream);
}

// ------------------------------------------------------------------ refinement
int tm_build_filter(const tm_filter_component* components, int n_components, const int* shape,
                    int rfft, float* out, void* stream) {
  return tmb::build_filter(components, n_components, shape, rfft, out, S(stream));
}

int tm_whitening_bins(const int* data_ft_shape, int n_bins) {
  if (!data_ft_shape) return TM_E_INVALID;
  return tmb::whitening_bins(data_ft_shape, n_bins);
}

int tm_whitening_filter(const void* data_rfft, const int* data_ft_shape, int n_bins,
                        const int* shape, int rfft, double* work, const float* factor,
                        float* out, void* stream) {
  return tmb::whitening_filter(static_cast<const float2*>(data_rfft), data_ft_shape, n_bins,
                               shape, rfft, work, factor, out, S(stream));
}

int tm_euler_zyz(const float* angles, int n, float* rot, float* drot, void* stream) {
  return tmb::euler_zyz(angles, n, rot, drot, S(stream));
}

int tm_refine_rotate(const tm_refine_desc* d, float* tmpl_rot, void* stream) {
  TM_REQUIRE(d, "tm_refine_rotate: null descriptor");
  return tmb::refine_rotate(refine_args(d), tmpl_rot, S(stream));
}

int tm_refine_forward(const tm_refine_desc* d, const float* tmpl_filtered, double* sums,
                      float* scores, void* stream) {
  TM_REQUIRE(d, "tm_refine_forward: null descriptor");
  return tmb::refine_forward(refine_args(d), tmpl_filtered, sums, scores, S(stream));
}

int tm_refine_grad_filtered(const tm_refine_desc* d, const float* tmpl_filtered,
                            const double* sums, const float* grad_scores, float* grad_filtered,
                            void* stream) {
  TM_REQUIRE(d, "tm_refine_grad_filtered: null descriptor");
  return tmb::refine_grad_filtered(refine_args(d), tmpl_filtered, sums, grad_scores,
                                   grad_filtered, S(stream));
}

int tm_refine_backward(const tm_refine_desc* d, const float* tmpl_filtered,
                       const float* grad_rotated, const double* sums, const float* grad_scores,
                       const float* drot, double* grad_rot, double* grad_shift,
                       double* grad_angles, float* grad_tmpl, void* stream) {
  TM_REQUIRE(d, "tm_refine_backward: null descriptor");
  return tmb::refine_backward(refine_args(d), tmpl_filtered, grad_rotated, sums, grad_scores,
                              drot, grad_rot, grad_shift, grad_angles, grad_tmpl, S(stream));
}

}  // extern "C"
