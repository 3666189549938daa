/*
 * pytme_b200 C ABI: the exhaustive template-matching hot path of pyTME on
 * NVIDIA B200 (sm_100a).
 *
 * Conventions
 *   - Every function returns an int status: TM_OK (0) or a negative TM_E_* code;
 *     tm_last_error() returns the message of the calling thread's last failure.
 *   - Buffers are raw device pointers owned by the caller, C-contiguous,
 *     float32 unless stated otherwise. Shapes are (axis 0, axis 1, axis 2) with
 *     axis 2 fastest, the layout of a C-ordered NumPy array.
 *   - Work is enqueued on the caller's CUDA stream (`stream`, a cudaStream_t
 *     passed as void*; NULL is the legacy default stream) and is asynchronous
 *     unless a function says it synchronises.
 *   - A tm_scan plan owns its scratch memory and cuFFT plans; it may be used
 *     from one host thread at a time.
 *
 * Each entry point names the reference interface (KosinskiLab/pyTME 0.3.b0,
 * paths inside that project) whose behaviour it provides.
 */
#ifndef PYTME_B200_H
#define PYTME_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TM_OK 0
#define TM_E_INVALID (-1)     /* bad argument: null pointer, shape, size */
#define TM_E_OOM (-2)         /* device allocation failed */
#define TM_E_CUFFT (-3)       /* cuFFT plan or execution failed */
#define TM_E_CUDA (-4)        /* CUDA runtime / launch error */
#define TM_E_TIMEOUT (-5)     /* a bounded device wait gave up */
#define TM_E_UNSUPPORTED (-6) /* valid request outside what this build implements */

#define TM_SCORE_CC 0    /* tme/matching_scores.py cc_setup + corr_scoring */
#define TM_SCORE_FLC 1   /* flc_setup + flc_scoring (rotated mask) */
#define TM_SCORE_FLCSM 2 /* flcSphericalMask_setup + corr_scoring */

#define TM_PREC_FP32 0  /* complex64 intermediate spectra */
#define TM_PREC_MIXED 1 /* half2 intermediate spectra, FP32 arithmetic, FP64 denominator */

/* Library version (major*10000 + minor*100 + patch). */
int tm_version(void);

/* Copies the calling thread's last error message (NUL-terminated, truncated to
 * len). Returns the full message length. */
int tm_last_error(char* buf, size_t len);

/* Caps the device memory one scan plan may allocate (bytes; 0 removes the cap). A plan
 * that would need more fails in tm_scan_create with TM_E_OOM, as a failed allocation
 * does, before touching the device: for hosts that run within a fixed memory budget,
 * and to exercise the out-of-memory path. The reference has no such setting; its
 * allocation failures surface through device_memory_handler
 * (tme/matching_exhaustive.py:122-141), which this error path mirrors. */
int tm_set_device_memory_limit(int64_t bytes);

/* Order-1 rigid transform of `n_mat` copies of a (d0,d1,d2) volume.
 * Replaces NumpyFFTWBackend.rigid_transform / _rigid_transform with order=1
 * (tme/backends/npfftw_backend.py:357-449), i.e. scipy.ndimage.affine_transform
 * in mode "constant": out[b][o] = interp(data, M_b[:3,:3] o + M_b[:3,3]), zero when
 * a coordinate falls below 0 or above n-1 on any axis. `matrices` holds n_mat
 * row-major 4x4 float32 pull matrices on the device. Output b is the (o0,o1,o2)
 * array at out + b*o0*o1*o2; only its top-left (d0,d1,d2) box is written.
 * `mask`/`out_mask` (optional, both or neither) are transformed with the same
 * matrices, as the reference does for arr_mask. */
int tm_rigid_transform(const float* data, const float* mask, int d0, int d1, int d2,
                       const float* matrices, int n_mat, float* out, float* out_mask, int o0,
                       int o1, int o2, void* stream);

/* Order-3 path of the same method: SciPy's spline_filter (order 3, mirror boundary),
 * which affine_transform(prefilter=True) applies to the data
 * (tme/backends/npfftw_backend.py:381-388), writing `batch` coefficient volumes of
 * d0 x d1 x d2 doubles. */
int tm_spline_prefilter(const float* in, double* coef, int d0, int d1, int d2, int batch,
                        void* stream);
/* Order-3 rigid transform from coefficient volumes: `coef` from tm_spline_prefilter for
 * the data, `mask_coef` the mask itself as doubles (the reference does not prefilter
 * masks, :434-447). Otherwise as tm_rigid_transform (SciPy constant mode, mirrored
 * coefficients inside the support at the edges). */
int tm_rigid_transform_cubic(const double* coef, const double* mask_coef, int d0, int d1,
                             int d2, const float* matrices, int n_mat, float* out,
                             float* out_mask, int o0, int o1, int o2, void* stream);

/* In-place masked standardisation of `batch` volumes of n elements:
 * x = (x - mean) / std * mask with mean/std over mask weights, the reference's
 * normalize_template (tme/matching_utils.py:61-99). n_obs > 0 is used as the
 * observation count, otherwise sum(mask) is. mask_batch_stride is 0 to share one
 * mask across the batch or n for one mask per volume. Reductions run in double.
 * `workspace` must hold tm_normalize_template_workspace(batch) bytes of device
 * memory. */
int64_t tm_normalize_template_workspace(int batch);
int tm_normalize_template(float* x, const float* mask, int64_t n, int batch,
                          int64_t mask_batch_stride, double n_obs, void* workspace,
                          void* stream);

/* NumpyFFTWBackend.norm_scores (tme/backends/npfftw_backend.py:537-587) evaluated in
 * double: sd = sqrt(max(exp_sq/n - (sq_exp/n)^2, 0)); sd < eps -> 1;
 * out = arr / (sd * n). arr == NULL stands for the scalar 1. n_obs_dev, when not
 * NULL, points to a device float32 n_obs that overrides n_obs. */
int tm_norm_scores(const float* arr, const float* exp_sq, const float* sq_exp, double n_obs,
                   const float* n_obs_dev, double eps, float* out, int64_t n, void* stream);

/* NumpyFFTWBackend.max_score_over_rotations (tme/backends/npfftw_backend.py:503-535):
 * where scores > max_scores (strict), copy the score and set rotations to
 * rotation_index. Buffers must be 16-byte aligned. */
int tm_max_score_over_rotations(const float* scores, float* max_scores, int32_t* rotations,
                                int32_t rotation_index, int64_t n, void* stream);

/* ---- FFT plans (cuFFT) for the backend's rfftn / irfftn
 * (tme/backends/npfftw_backend.py:243-306). ndim in 1..3, shape is the real shape,
 * batch leading. Forward is unnormalised; tm_fft_c2r multiplies by `scale`
 * (pass 1/prod(shape) for NumPy's "backward" normalisation) and overwrites its
 * input. double_precision selects D2Z/Z2D. */
typedef struct tm_fft_plan tm_fft_plan;
int tm_fft_plan_create(int ndim, const int* shape, int batch, int double_precision,
                       tm_fft_plan** plan);
int tm_fft_plan_destroy(tm_fft_plan* plan);
int tm_fft_r2c(tm_fft_plan* plan, const void* in, void* out, void* stream);
int tm_fft_c2r(tm_fft_plan* plan, void* in, void* out, double scale, void* stream);
/* Template filter at template shape (_apply_filter_subset of _create_filter_func,
 * tme/matching_scores.py:90-135): x = irfftn(rfftn(x) * filter) in place for every
 * batch item of a single-precision plan. `filter` holds one real value per rfft
 * element of one item and is shared by all items; `spectrum` holds the plan's
 * complex output (batch x rfft elements). */
int tm_fft_filter(tm_fft_plan* plan, float* x, void* spectrum, const float* filter,
                  void* stream);

/* ---- rotation scan: the per-rotation loops of corr_scoring
 * (tme/matching_scores.py:491-626) and flc_scoring (:629-759) with the
 * MaxScoreOverRotations update (tme/analyzer/aggregation.py:142-189). */
typedef struct {
  int score;             /* TM_SCORE_* */
  int precision;         /* TM_PREC_* */
  int fast_shape[3];     /* transform shape (fast_shape of fourier_padding) */
  int template_shape[3]; /* template / mask shape */
  int batch;             /* rotations per launch group (fused path) */
  int plain;             /* 1: one rotation at a time with full cuFFT transforms */
  int has_template_filter; /* set by tm_scan_set_template */
} tm_scan_desc;

typedef struct tm_scan tm_scan;

/* Creates a plan and allocates its device scratch. Returns TM_E_UNSUPPORTED for
 * shapes the fused path does not handle (the plain path handles every shape). */
int tm_scan_create(const tm_scan_desc* desc, tm_scan** plan);
int tm_scan_destroy(tm_scan* plan);
/* Device bytes held by the plan (scratch plus persistent spectra). */
int64_t tm_scan_device_bytes(const tm_scan* plan);

/* Template and mask as the scoring loops see them (already reversed along every
 * axis, MatchingData.template, tme/matching_data.py:698-715), shape
 * template_shape; mask may be NULL for CC. template_filter (optional) is the
 * multiplicative filter at the template's rfft shape (t0, t1, t2//2+1), applied
 * to each rotated template before normalisation (_create_filter_func,
 * tme/matching_scores.py:44-150). Synchronises the stream. */
int tm_scan_set_template(tm_scan* plan, const float* template_rev, const float* mask_rev,
                         const float* template_filter, void* stream);

/* Target of shape fast_shape (top-left padded and already filtered). Computes
 * the target spectra and, for FLCSphericalMask, the inverse local-variance
 * denominator in double precision (flcSphericalMask_setup,
 * tme/matching_scores.py:390-450). Call after tm_scan_set_template.
 * Synchronises the stream. */
int tm_scan_set_target(tm_scan* plan, const float* target, void* stream);
/* interpolation_order of corr_scoring / flc_scoring (tme/matching_scores.py:600-608,
 * 731-740) as rigid_transform applies it (tme/backends/npfftw_backend.py:390-449):
 * 1 = trilinear (the default), 3 = cubic B-spline with the template prefiltered and
 * the rotated mask not. Other orders return TM_E_UNSUPPORTED. Synchronous with respect
 * to `stream` only when the template is already set (it then builds the coefficients). */
int tm_scan_set_interpolation(tm_scan* plan, int order, void* stream);
/* x pass of the fused CC / FLCSphericalMask scan (the axis-0 transforms and the product
 * with the target spectrum of corr_scoring, tme/matching_scores.py:610-618): mode 0 runs
 * it on the tensor cores as a per-column circular correlation, mode 1 as forward and
 * inverse FFTs on the CUDA cores, mode 2 restores the default (tensor cores for
 * mixed-precision plans whose x length is a multiple of 128, FFTs otherwise).
 * TM_E_UNSUPPORTED when mode 0 is not available for this plan. */
int tm_scan_set_xpass(tm_scan* plan, int mode);
/* The x pass the plan runs: 0 tensor cores, 1 FFT (TM_E_INVALID for a null plan). */
int tm_scan_xpass_mode(const tm_scan* plan);
/* z pass of the fused CC / FLCSphericalMask scan (the inverse transform along axis 2,
 * the score normalisation and the MaxScoreOverRotations update of corr_scoring,
 * tme/matching_scores.py:618-624, and tme/analyzer/aggregation.py:142-189): mode 0 runs
 * the c2r as a GEMM with a fixed operator on the tensor cores and reduces the maximum
 * over the group's rotations from tensor memory (the default for mixed-precision plans
 * with n2 <= 256 and at most 32 rotations per group), mode 1 as CUDA-core FFTs, mode 2
 * restores the default. TM_E_UNSUPPORTED when mode 0 is not available. */
int tm_scan_set_zpass(tm_scan* plan, int mode);
int tm_scan_zpass_mode(const tm_scan* plan);
/* y pass of the fused CC / FLCSphericalMask scan (the inverse transform along axis 1 of
 * corr_scoring's irfftn, tme/matching_scores.py:618-620): mode 0 runs it on the tensor
 * cores (radix 16 in FP32 registers, then radix n1/16 as an FP16 DFT GEMM, twiddles
 * between them; mixed-precision plans with n1 of 256 or 512; the default where
 * available), mode 1 as CUDA-core FFTs, mode 2 restores the default, mode 3 runs both
 * DFT stages on the tensor cores (needs the warp-specialised tensor-core x pass, which
 * then writes the y pass's input layout), mode 4 runs mode 0 in place on row-major
 * spectra (mode 0 reads the spectra that the warp-specialised x pass writes with x'
 * innermost and writes row-major rows into a second buffer for the z pass, where the
 * plan has one). tm_scan_ypass_mode reports 0, 1, 3 or 4.
 * TM_E_UNSUPPORTED when the requested form is not available. */
int tm_scan_set_ypass(tm_scan* plan, int mode);
int tm_scan_ypass_mode(const tm_scan* plan);
/* Bound of every data wait inside the plan's tensor-core kernels, in mbarrier polls
 * (0 restores the default of 4,194,304, on the order of a second). A wait that runs out
 * makes its kernel stop early; the next tm_scan_check then returns TM_E_TIMEOUT and the
 * results of that run are invalid. The waits that keep tensor memory and shared memory
 * alive until in-flight MMAs finish always use the default. No counterpart in the
 * reference, which has no device waits; it plays the role of the reference's error
 * surfacing in device_memory_handler (tme/matching_exhaustive.py:122-141). */
int tm_scan_set_wait_budget(tm_scan* plan, uint32_t iters);
/* Synchronise `stream`; TM_E_TIMEOUT if a bounded wait inside a tensor-core kernel of
 * this plan gave up since the last check (the results of that run are invalid). */
int tm_scan_check(tm_scan* plan, void* stream);

/* Scores n rotations given as row-major 4x4 float32 pull matrices on the device
 * (NumpyFFTWBackend._rigid_transform_matrix of each rotation about the template
 * centre) and folds them into the running state: max_scores (fast_shape float32)
 * and argmax (fast_shape int32), updated where score > max_scores (strict), with
 * rotation i recorded as first_index + i. */
int tm_scan_run(tm_scan* plan, const float* matrices, int n, int32_t first_index,
                float* max_scores, int32_t* argmax, void* stream);

/* Per-stage timing of the fused path: when enabled, each stage of tm_scan_run is
 * bracketed by CUDA events on the launching stream (and the host waits for each
 * stage, so enable it only to measure). Stages: */
#define TM_STAGE_PREPARE 0  /* rotation, template filter, normalisation */
#define TM_STAGE_TEMPLATE 1 /* template transform along axes 2 and 1 */
#define TM_STAGE_XPASS 2    /* axis-0 forward FFT, target product, axis-0 inverse FFT */
#define TM_STAGE_YPASS 3    /* axis-1 inverse FFT */
#define TM_STAGE_ZPASS 4    /* axis-2 c2r, score scaling, max/argmax update */
#define TM_NUM_STAGES 5
int tm_scan_set_timing(tm_scan* plan, int enable); /* also resets the counters */

/* Replay full launch groups of the fused path from one captured CUDA graph (the
 * template preparation and the four passes). The first full group of tm_scan_run
 * captures it for the given max_scores/argmax buffers (a different pair recaptures);
 * later groups copy their matrices and first index into the plan and replay it,
 * ordered on the caller's stream. Ignored by the plain path and while timing. */
int tm_scan_set_graph(tm_scan* plan, int enable);
int tm_scan_get_timing(const tm_scan* plan, double* ms, int64_t* launches); /* TM_NUM_STAGES each */
/* Algorithmic HBM bytes of one launch of `stage` for a group of nb rotations. */
int64_t tm_scan_stage_bytes(const tm_scan* plan, int stage, int nb);

/* ---- peak calling
 * Box maximum filter of edge `size` with SciPy's constant mode (cval 0) and the
 * peak test of NumpyFFTWBackend.max_filter_coordinates
 * (tme/backends/npfftw_backend.py:200-206): mask[v] = (maxfilter(scores)[v] ==
 * scores[v]). tmp_a / tmp_b are caller buffers of n0*n1*n2 floats. */
int tm_max_filter_peaks(const float* scores, int n0, int n1, int n2, int size, float* tmp_a,
                        float* tmp_b, uint8_t* mask, void* stream);

/* Greedy minimum-distance filter of find_candidate_indices
 * (tme/external/bindings.cpp:85-126) for n int64 (x, y, z) coordinates in the
 * order given: point 0 is kept, point i is kept when floor(sqrt(d2)) >
 * min_distance for every kept point. Writes the kept indices to out_idx (device,
 * n int32) and their count to *out_count (device int32). Up to 2048 points run in
 * shared memory; more need `workspace` of tm_find_candidate_indices_workspace(n)
 * bytes of device memory (otherwise NULL). */
int64_t tm_find_candidate_indices_workspace(int n);
int tm_find_candidate_indices(const int64_t* coords, int n, int64_t min_distance,
                              int32_t* out_idx, int32_t* out_count, void* workspace,
                              void* stream);

/* Allocation-free greedy minimum-distance filter. No counterpart in the
 * reference: it is tm_find_candidate_indices for callers that cannot allocate
 * device memory while they run (for example, hosts that own all device memory
 * through their own pool, or that have a fixed memory budget agreed up front).
 * Instead of a caller workspace it uses a fixed scratch array in the library's
 * static device memory, 3 * TM_NOALLOC_MAX_POINTS int64 (1.5 MiB), which every
 * GPU that loads the library holds until the process exits. It allocates nothing:
 * no cudaMalloc, cudaFree or allocating library call. n above
 * TM_NOALLOC_MAX_POINTS returns TM_E_INVALID. The first call on each device looks
 * up the scratch address (cudaGetSymbolAddress) with that device current, and again
 * after the device's context was replaced (cudaDeviceReset); make that first call
 * before any stream capture. All calls share the one scratch
 * array, so calls that overlap on the GPU (different streams, or different host
 * threads on one device) race and must be serialised by the caller. Results are
 * identical to tm_find_candidate_indices. */
#define TM_NOALLOC_MAX_POINTS 65536
int tm_find_candidate_indices_noalloc(const int64_t* coords, int n, int64_t min_distance,
                                      int32_t* out_idx, int32_t* out_count, void* stream);

/* ---- filters built on the device: CTFReconstructed (tme/filters/ctf.py:260-336, 528-655)
 * and WedgeReconstructed with create_continuous_wedge=True (tme/filters/wedge.py:282-374),
 * multiplied in the given order like Compose (tme/filters/compose.py:36-59), written
 * as float32 with the DC term at index 0, in rfft layout (last axis n2//2 + 1) when
 * `rfft` is non-zero. Component parameters are the float64 scalars the reference
 * derives from the filter's arguments:
 *   CTF:   p[0] defocus_x, p[1] 0.5 * aberration, p[2] pi * wavelength, p[3] phase shift,
 *          p[4] atan(A / sqrt(1 - A^2)), p[5] frequency cutoff, p[6] flip phase (0/1);
 *   WEDGE: p[0] start, p[1] stop, p[2] ratio at opening index 0, p[3] opening axis,
 *          p[4] tilt axis, p[5] frequency cutoff (negative: none). */
#define TM_FILTER_CTF 1
#define TM_FILTER_WEDGE 2
#define TM_FILTER_MAX_COMPONENTS 4
typedef struct {
  int kind;
  double p[8];
} tm_filter_component;
int tm_build_filter(const tm_filter_component* components, int n_components,
                    const int* shape, int rfft, float* out, void* stream);

/* LinearWhiteningFilter (tme/filters/whitening.py:23-186) on the device: the inverse
 * square root of the radially averaged power spectrum of the data, normalised to a
 * maximum of 1 and interpolated linearly on the frequency grid of a filter of real shape
 * `shape`, returned like tm_build_filter (float32, DC at index 0, rfft layout when rfft is
 * non-zero). `data_rfft`: complex64 rfft of the data, rfft shape data_ft_shape (the
 * reference's bins are defined on this shape); in the scan path the data is the target
 * padded to the fast shape (tme/matching_exhaustive.py:84-90). n_bins <= 0 selects the
 * reference's default. `factor` (optional, same layout as out) multiplies the filter in
 * float64 before the single rounding to float32, as Compose multiplies a float64
 * whitening array with the product of the other filters. `work`: device scratch of
 * 3 * tm_whitening_bins(data_ft_shape, n_bins) doubles. */
int tm_whitening_bins(const int* data_ft_shape, int n_bins);
int tm_whitening_filter(const void* data_rfft, const int* data_ft_shape, int n_bins,
                        const int* shape, int rfft, double* work, const float* factor,
                        float* out, void* stream);

/* ---- local refinement of candidate peaks: the FLC of flc_scoring
 * (tme/matching_scores.py:629-759) at one pose per peak and its adjoint. This
 * replaces the derivative-free score of tme/matching_optimization.py:54-277 and
 * 488-548, whose optimize_match (:1143-1312) drives scipy.optimize.
 *
 * Peak p: box corner corners[3p..] (target voxel of template voxel 0), rotation
 * rot[9p..] (row-major R, the matrix of the scan's rotation set) about the template
 * centre (t-1)/2, shift shifts[3p..] in voxels in the target frame. Template voxel o
 * samples the template and mask at R^T (o - c - s) + c (order 1, zero unless every
 * coordinate is inside [0, t-1]). The score is computed from the filtered template
 * when tmpl_filtered (n_peaks x t^3, from tm_refine_rotate + tm_fft_filter) is
 * given, else from the rotated template directly; eps is norm_scores' epsilon
 * (tme/backends/npfftw_backend.py:537-587). Sums (n_peaks x 6 doubles: sum M,
 * M T, M T^2, M T f, M f, M f^2) are what the backward pass needs. */
typedef struct {
  const float* tmpl;     /* t^3 template (not reversed) */
  const float* mask;     /* t^3 mask */
  int template_shape[3];
  const float* target;   /* target volume (already filtered) */
  int target_shape[3];
  float target_outside;  /* value of the target outside its bounds (0 for the raw
                            target; minus the subtracted mean for a centred one) */
  const float* rot;      /* n_peaks x 9 */
  const float* shifts;   /* n_peaks x 3 */
  const int32_t* corners;/* n_peaks x 3 */
  int n_peaks;
  double eps;
} tm_refine_desc;

/* R = Rz(a2) Ry(a1) Rz(a0) from zyz angles in degrees (euler_to_rotationmatrix,
 * tme/rotations.py:171-196, SciPy's extrinsic "zyz"), and when drot is not NULL
 * dR/da_k per degree (n x 3 x 9). */
int tm_euler_zyz(const float* angles, int n, float* rot, float* drot, void* stream);
/* Rotated template for every peak (n_peaks x t^3), the input of tm_fft_filter. */
int tm_refine_rotate(const tm_refine_desc* d, float* tmpl_rot, void* stream);
int tm_refine_forward(const tm_refine_desc* d, const float* tmpl_filtered, double* sums,
                      float* scores, void* stream);
/* Filtered path, first half of the backward: dS/d(filtered template), n_peaks x t^3.
 * tm_fft_filter of it (the filter is self-adjoint) gives grad_rotated below. */
int tm_refine_grad_filtered(const tm_refine_desc* d, const float* tmpl_filtered,
                            const double* sums, const float* grad_scores,
                            float* grad_filtered, void* stream);
/* Pose and template gradients of sum_p grad_scores[p] * S_p. tmpl_filtered and
 * grad_rotated are both NULL (unfiltered) or both given. Outputs may be NULL:
 * grad_rot n x 9, grad_shift n x 3, grad_angles n x 3 (needs drot), grad_tmpl t^3 is
 * ACCUMULATED into (zero it first). */
int tm_refine_backward(const tm_refine_desc* d, const float* tmpl_filtered,
                       const float* grad_rotated, const double* sums, const float* grad_scores,
                       const float* drot, double* grad_rot, double* grad_shift,
                       double* grad_angles, float* grad_tmpl, void* stream);

#ifdef __cplusplus
}
#endif

#endif /* PYTME_B200_H */
