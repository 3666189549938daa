// Device kernels behind the MatchingBackend method surface: order-1 rigid
// transforms, masked template normalisation, score normalisation, the running
// max/argmax over rotations, and the elementwise helpers of the plain
// (one-rotation-at-a-time) scan.
#include "common.cuh"
#include "ops.cuh"

#include <algorithm>
#include <cmath>
#include <mutex>
#include <atomic>
#include <string>

namespace tmb {

static thread_local std::string g_last_error;

void set_error(const char* fmt, ...) {
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

const char* last_error() { return g_last_error.c_str(); }

// Process-wide cap on the device memory a plan may hold (0: none), see
// tm_set_device_memory_limit.
static std::atomic<int64_t> g_memory_limit{0};
void set_device_memory_limit(int64_t bytes) { g_memory_limit.store(bytes > 0 ? bytes : 0); }
int64_t device_memory_limit() { return g_memory_limit.load(); }

// --------------------------------------------------------------- rigid transform
// Pull-interpolation out[o] = interp(in, M[:3,:3] o + M[:3,3]) with SciPy's
// order-1, mode="constant" semantics (cval 0): a sample whose coordinate lies
// below 0 or above n-1 on any axis is 0, otherwise trilinear. Coordinates and
// weights are formed in double precision from the float32 matrix, as
// scipy.ndimage.affine_transform does; products of a float32 entry and an
// integer index are exact in double, and the sums are kept free of FMA
// contraction so the bound tests see the same coordinate SciPy sees.
__device__ __forceinline__ double coord(const float* m, int row, int o0, int o1, int o2) {
  double c = __dmul_rn((double)m[row * 4 + 0], (double)o0);
  c = __dadd_rn(c, __dmul_rn((double)m[row * 4 + 1], (double)o1));
  c = __dadd_rn(c, __dmul_rn((double)m[row * 4 + 2], (double)o2));
  c = __dadd_rn(c, (double)m[row * 4 + 3]);
  return c;
}

struct Trilinear {
  int64_t idx[8];
  double w[8];
  bool inside;
};

__device__ __forceinline__ Trilinear trilinear_setup(const float* m, int o0, int o1, int o2,
                                                     int d0, int d1, int d2) {
  Trilinear t;
  double c[3] = {coord(m, 0, o0, o1, o2), coord(m, 1, o0, o1, o2), coord(m, 2, o0, o1, o2)};
  int n[3] = {d0, d1, d2};
  int lo[3], hi[3];
  double f[3];
  t.inside = true;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (!(c[a] >= 0.0) || c[a] > (double)(n[a] - 1)) t.inside = false;
    double fl = floor(c[a]);
    lo[a] = (int)fl;
    f[a] = c[a] - fl;
    hi[a] = min(lo[a] + 1, n[a] - 1);
    lo[a] = max(min(lo[a], n[a] - 1), 0);
  }
  if (!t.inside) return t;
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    int i0 = (q & 4) ? hi[0] : lo[0];
    int i1 = (q & 2) ? hi[1] : lo[1];
    int i2 = (q & 1) ? hi[2] : lo[2];
    double w0 = (q & 4) ? f[0] : 1.0 - f[0];
    double w1 = (q & 2) ? f[1] : 1.0 - f[1];
    double w2 = (q & 1) ? f[2] : 1.0 - f[2];
    t.idx[q] = ((int64_t)i0 * d1 + i1) * d2 + i2;
    t.w[q] = w0 * w1 * w2;
  }
  return t;
}

__device__ __forceinline__ float trilinear_eval(const Trilinear& t, const float* __restrict__ d) {
  if (!t.inside) return 0.f;
  double acc = 0.0;
#pragma unroll
  for (int q = 0; q < 8; ++q) acc += t.w[q] * (double)__ldg(d + t.idx[q]);
  return (float)acc;
}

__global__ void rigid_transform_kernel(const float* __restrict__ data, const float* __restrict__ mask,
                                       int d0, int d1, int d2, const float* __restrict__ matrices,
                                       float* __restrict__ out, float* __restrict__ out_mask,
                                       int o1, int o2, int64_t out_stride) {
  __shared__ float m[16];
  const int b = blockIdx.y;
  if (threadIdx.x < 16) m[threadIdx.x] = matrices[b * 16 + threadIdx.x];
  __syncthreads();
  const int64_t nvox = (int64_t)d0 * d1 * d2;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nvox;
       v += (int64_t)gridDim.x * blockDim.x) {
    int i2 = (int)(v % d2);
    int64_t r = v / d2;
    int i1 = (int)(r % d1);
    int i0 = (int)(r / d1);
    Trilinear t = trilinear_setup(m, i0, i1, i2, d0, d1, d2);
    int64_t oi = b * out_stride + ((int64_t)i0 * o1 + i1) * o2 + i2;
    out[oi] = trilinear_eval(t, data);
    if (out_mask) out_mask[oi] = trilinear_eval(t, mask);
  }
}

int rigid_transform(const float* data, const float* mask, int d0, int d1, int d2,
                    const float* matrices, int n_mat, float* out, float* out_mask, int o0,
                    int o1, int o2, cudaStream_t stream) {
  TM_REQUIRE(data && matrices && out, "rigid_transform: null pointer");
  TM_REQUIRE(!out_mask || mask, "rigid_transform: out_mask given without mask");
  TM_REQUIRE(d0 > 0 && d1 > 0 && d2 > 0 && n_mat > 0, "rigid_transform: empty input");
  TM_REQUIRE(o0 >= d0 && o1 >= d1 && o2 >= d2,
             "rigid_transform: output box (%d,%d,%d) smaller than input (%d,%d,%d)", o0, o1,
             o2, d0, d1, d2);
  int64_t nvox = (int64_t)d0 * d1 * d2;
  int threads = 256;
  int64_t blocks = ceil_div(nvox, threads);
  if (blocks > 4096) blocks = 4096;
  dim3 grid((unsigned)blocks, (unsigned)n_mat);
  rigid_transform_kernel<<<grid, threads, 0, stream>>>(data, mask, d0, d1, d2, matrices, out,
                                                       out_mask, o1, o2,
                                                       (int64_t)o0 * o1 * o2);
  return check_launch("rigid_transform_kernel");
}

// --------------------------------------------------------------- cubic B-spline (order 3)
// SciPy's order-3 path (affine_transform with prefilter=True calls spline_filter, then
// evaluates the spline): interpolation coefficients by the recursive filter of Unser,
// Aldroubi and Eden ("B-spline signal processing", IEEE Trans. Signal Process. 41, 1993)
// with the single pole z = sqrt(3) - 2, gain (1 - z)(1 - 1/z) = 6, and mirror-symmetric
// boundaries (x[-k] = x[k], x[n-1+k] = x[n-1-k]): exact causal initialisation over the
// mirrored period 2n - 2 and the closed-form anticausal start
// c[n-1] = z/(z^2 - 1) * (c+[n-1] + z c+[n-2]) (Thevenaz, Blu and Unser, "Interpolation
// revisited", IEEE Trans. Med. Imaging 19, 2000). Axes are filtered 0, 1, 2 in double.
__global__ void spline_prefilter_kernel(const float* __restrict__ in, double* __restrict__ c,
                                        int d0, int d1, int d2, int axis, int batch) {
  const int n = axis == 0 ? d0 : (axis == 1 ? d1 : d2);
  const int64_t stride = axis == 0 ? (int64_t)d1 * d2 : (axis == 1 ? d2 : 1);
  const int64_t lines_per_item = (int64_t)d0 * d1 * d2 / n;
  const int64_t nvox = (int64_t)d0 * d1 * d2;
  for (int64_t l = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; l < lines_per_item * batch;
       l += (int64_t)gridDim.x * blockDim.x) {
    const int64_t b = l / lines_per_item, r = l % lines_per_item;
    int64_t start;
    if (axis == 0) start = r;                               // r = i1 * d2 + i2
    else if (axis == 1) start = (r / d2) * d1 * d2 + r % d2;  // r = i0 * d2 + i2
    else start = r * d2;                                    // r = i0 * d1 + i1
    double* x = c + b * nvox + start;
    const float* xi = in ? in + b * nvox + start : nullptr;
    if (xi)
      for (int i = 0; i < n; ++i) x[i * stride] = (double)xi[i * stride];
    if (n == 1) continue;
    const double z = sqrt(3.0) - 2.0, gain = (1.0 - z) * (1.0 - 1.0 / z);
    for (int i = 0; i < n; ++i) x[i * stride] *= gain;
    // causal initialisation over the mirrored signal
    double zn = 1.0;
    for (int i = 0; i < n - 1; ++i) zn *= z;  // z^(n-1)
    double acc = x[0] + zn * x[(n - 1) * stride];
    double zi = z;
    for (int i = 1; i < n - 1; ++i) {
      acc += zi * (x[i * stride] + zn * x[(n - 1 - i) * stride]);
      zi *= z;
    }
    x[0] = acc / (1.0 - zn * zn);
    for (int i = 1; i < n; ++i) x[i * stride] += z * x[(i - 1) * stride];
    x[(n - 1) * stride] = z / (z * z - 1.0) * (z * x[(n - 2) * stride] + x[(n - 1) * stride]);
    for (int i = n - 2; i >= 0; --i) x[i * stride] = z * (x[(i + 1) * stride] - x[i * stride]);
  }
}

int spline_prefilter(const float* in, double* coef, int d0, int d1, int d2, int batch,
                     cudaStream_t stream) {
  TM_REQUIRE(coef, "spline_prefilter: null output");
  TM_REQUIRE(d0 > 0 && d1 > 0 && d2 > 0 && batch > 0, "spline_prefilter: empty input");
  const int dims[3] = {d0, d1, d2};
  for (int axis = 0; axis < 3; ++axis) {
    const int64_t lines = (int64_t)d0 * d1 * d2 / dims[axis] * batch;
    const int64_t blocks = std::min<int64_t>(ceil_div(lines, 128), 148 * 8);
    spline_prefilter_kernel<<<(unsigned)blocks, 128, 0, stream>>>(axis == 0 ? in : nullptr,
                                                                 coef, d0, d1, d2, axis, batch);
    TM_TRY(check_launch("spline_prefilter_kernel"));
  }
  return TM_OK;
}

__global__ void to_double_kernel(const float* __restrict__ in, double* __restrict__ out,
                                 int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = (double)in[i];
}

int to_double(const float* in, double* out, int64_t n, cudaStream_t stream) {
  if (n <= 0) return TM_OK;
  const int64_t blocks = std::min<int64_t>(ceil_div(n, 256), 148 * 8);
  to_double_kernel<<<(unsigned)blocks, 256, 0, stream>>>(in, out, n);
  return check_launch("to_double_kernel");
}

// Cubic B-spline basis values at the four samples floor(x) - 1 .. floor(x) + 2 for the
// fractional part t of x.
__device__ __forceinline__ void bspline3_weights(double t, double w[4]) {
  const double t2 = t * t, t3 = t2 * t, s = 1.0 - t;
  w[0] = s * s * s / 6.0;
  w[1] = (3.0 * t3 - 6.0 * t2 + 4.0) / 6.0;
  w[2] = (-3.0 * t3 + 3.0 * t2 + 3.0 * t + 1.0) / 6.0;
  w[3] = t3 / 6.0;
}

// Whole-sample mirror of an index into [0, n-1] (period 2n - 2).
__device__ __forceinline__ int mirror_index(int i, int n) {
  if (n == 1) return 0;
  const int p = 2 * n - 2;
  i = abs(i) % p;
  return i < n ? i : p - i;
}

// Order-3 pull interpolation from coefficient arrays with SciPy's constant mode: a
// sample whose coordinate is below 0 or above n-1 on any axis is 0; otherwise the
// 4 x 4 x 4 spline support reads mirrored coefficients at the edges. Coordinates in
// double from the float32 matrix, exactly as the order-1 kernel forms them.
__global__ void rigid_transform_cubic_kernel(const double* __restrict__ coef,
                                             const double* __restrict__ mcoef, int d0, int d1,
                                             int d2, const float* __restrict__ matrices,
                                             float* __restrict__ out, float* __restrict__ out_mask,
                                             int o1, int o2, int64_t out_stride) {
  __shared__ float m[16];
  const int b = blockIdx.y;
  if (threadIdx.x < 16) m[threadIdx.x] = matrices[b * 16 + threadIdx.x];
  __syncthreads();
  const int64_t nvox = (int64_t)d0 * d1 * d2;
  const int n[3] = {d0, d1, d2};
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < nvox;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int i2 = (int)(v % d2);
    const int64_t r = v / d2;
    const int i1 = (int)(r % d1);
    const int i0 = (int)(r / d1);
    const double c[3] = {coord(m, 0, i0, i1, i2), coord(m, 1, i0, i1, i2),
                         coord(m, 2, i0, i1, i2)};
    bool inside = true;
    double w[3][4];
    int idx[3][4];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      if (!(c[a] >= 0.0) || c[a] > (double)(n[a] - 1)) inside = false;
      const double fl = floor(c[a]);
      bspline3_weights(c[a] - fl, w[a]);
#pragma unroll
      for (int k = 0; k < 4; ++k) idx[a][k] = mirror_index((int)fl - 1 + k, n[a]);
    }
    const int64_t oi = b * out_stride + ((int64_t)i0 * o1 + i1) * o2 + i2;
    double acc = 0.0, accm = 0.0;
    if (inside) {
      for (int i = 0; i < 4; ++i) {
        double ai = 0.0, am = 0.0;
        for (int j = 0; j < 4; ++j) {
          const int64_t row = ((int64_t)idx[0][i] * d1 + idx[1][j]) * d2;
          double aj = 0.0, amj = 0.0;
#pragma unroll
          for (int k = 0; k < 4; ++k) {
            aj += w[2][k] * __ldg(coef + row + idx[2][k]);
            if (mcoef) amj += w[2][k] * __ldg(mcoef + row + idx[2][k]);
          }
          ai += w[1][j] * aj;
          am += w[1][j] * amj;
        }
        acc += w[0][i] * ai;
        accm += w[0][i] * am;
      }
    }
    out[oi] = (float)acc;
    if (out_mask) out_mask[oi] = (float)accm;
  }
}

int rigid_transform_cubic(const double* coef, const double* mcoef, int d0, int d1, int d2,
                          const float* matrices, int n_mat, float* out, float* out_mask, int o0,
                          int o1, int o2, cudaStream_t stream) {
  TM_REQUIRE(coef && matrices && out, "rigid_transform_cubic: null pointer");
  TM_REQUIRE(!out_mask || mcoef, "rigid_transform_cubic: out_mask given without mask");
  TM_REQUIRE(d0 > 0 && d1 > 0 && d2 > 0 && n_mat > 0, "rigid_transform_cubic: empty input");
  TM_REQUIRE(o0 >= d0 && o1 >= d1 && o2 >= d2,
             "rigid_transform_cubic: output box (%d,%d,%d) smaller than input (%d,%d,%d)", o0,
             o1, o2, d0, d1, d2);
  const int64_t nvox = (int64_t)d0 * d1 * d2;
  int64_t blocks = std::min<int64_t>(ceil_div(nvox, 256), 4096);
  dim3 grid((unsigned)blocks, (unsigned)n_mat);
  rigid_transform_cubic_kernel<<<grid, 256, 0, stream>>>(coef, out_mask ? mcoef : nullptr, d0,
                                                         d1, d2, matrices, out, out_mask, o1,
                                                         o2, (int64_t)o0 * o1 * o2);
  return check_launch("rigid_transform_cubic_kernel");
}

// --------------------------------------------------------------- template statistics
// Per batch item: S[0] = sum(x*m), S[1] = sum(x*x*m), S[2] = sum(m), accumulated in
// double by a fixed-shape tree (block partials, then one block per item), so
// repeated runs are bit-identical.
constexpr int kStatThreads = 256;

__device__ __forceinline__ double block_sum(double v, double* sh) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0) sh[warp] = v;
  __syncthreads();
  double s = 0.0;
  if (threadIdx.x == 0)
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sh[w];
  return s;
}

// Partial sums over a strided view: item b covers elements [b*stride, b*stride+n)
// of a box of shape (e0, e1, e2) embedded in rows of (o1, o2).
__global__ void stats_partial_kernel(const float* __restrict__ x, const float* __restrict__ m,
                                     int64_t m_item_stride, int e0, int e1, int e2, int o1,
                                     int o2, int64_t item_stride, double* __restrict__ partial,
                                     int nchunks) {
  __shared__ double sh[32];
  const int b = blockIdx.y;
  const int64_t n = (int64_t)e0 * e1 * e2;
  double s0 = 0, s1 = 0, s2 = 0;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (int64_t)gridDim.x * blockDim.x) {
    int i2 = (int)(v % e2);
    int64_t r = v / e2;
    int i1 = (int)(r % e1);
    int i0 = (int)(r / e1);
    int64_t off = ((int64_t)i0 * o1 + i1) * o2 + i2;
    double xv = x[b * item_stride + off];
    double mv = m[b * m_item_stride + off];
    s0 += xv * mv;
    s1 += xv * xv * mv;
    s2 += mv;
  }
  double t0 = block_sum(s0, sh);
  double t1 = block_sum(s1, sh);
  double t2 = block_sum(s2, sh);
  if (threadIdx.x == 0) {
    double* p = partial + ((int64_t)b * nchunks + blockIdx.x) * 3;
    p[0] = t0;
    p[1] = t1;
    p[2] = t2;
  }
}

// mean/std per item following normalize_template (tme/matching_utils.py:61-99):
// mean = S0/n, std = sqrt(max(S1/n - mean^2, 0)); n is the given n_obs or S2.
__global__ void stats_finalize_kernel(const double* __restrict__ partial, int nchunks,
                                      double n_obs, double* __restrict__ stats) {
  __shared__ double sh[32];
  const int b = blockIdx.x;
  double s0 = 0, s1 = 0, s2 = 0;
  for (int c = threadIdx.x; c < nchunks; c += blockDim.x) {
    const double* p = partial + ((int64_t)b * nchunks + c) * 3;
    s0 += p[0];
    s1 += p[1];
    s2 += p[2];
  }
  double t0 = block_sum(s0, sh);
  double t1 = block_sum(s1, sh);
  double t2 = block_sum(s2, sh);
  if (threadIdx.x == 0) {
    double n = n_obs > 0 ? n_obs : t2;
    double mean = t0 / n;
    double var = t1 / n - mean * mean;
    double sd = sqrt(var > 0 ? var : 0.0);
    stats[b * 4 + 0] = mean;
    stats[b * 4 + 1] = sd;
    stats[b * 4 + 2] = n;
    stats[b * 4 + 3] = 0.0;
  }
}

__global__ void normalize_apply_kernel(float* __restrict__ x, const float* __restrict__ m,
                                       int64_t m_item_stride, int e0, int e1, int e2, int o1,
                                       int o2, int64_t item_stride,
                                       const double* __restrict__ stats) {
  const int b = blockIdx.y;
  const double mean = stats[b * 4 + 0], sd = stats[b * 4 + 1];
  const int64_t n = (int64_t)e0 * e1 * e2;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (int64_t)gridDim.x * blockDim.x) {
    int i2 = (int)(v % e2);
    int64_t r = v / e2;
    int i1 = (int)(r % e1);
    int i0 = (int)(r / e1);
    int64_t off = ((int64_t)i0 * o1 + i1) * o2 + i2;
    float mv = m[b * m_item_stride + off];
    float xv = x[b * item_stride + off];
    x[b * item_stride + off] = (float)(((double)xv - mean) / sd) * mv;
  }
}

int64_t stats_workspace_bytes(int batch) {
  return (int64_t)batch * kStatChunks * 3 * sizeof(double) + (int64_t)batch * 4 * sizeof(double);
}

int template_stats(const float* x, const float* m, int64_t m_item_stride, int e0, int e1, int e2,
                   int o1, int o2, int64_t item_stride, int batch, double n_obs, double* ws,
                   cudaStream_t stream) {
  double* partial = ws;
  double* stats = ws + (int64_t)batch * kStatChunks * 3;
  dim3 grid(kStatChunks, batch);
  stats_partial_kernel<<<grid, kStatThreads, 0, stream>>>(x, m, m_item_stride, e0, e1, e2, o1,
                                                          o2, item_stride, partial, kStatChunks);
  TM_TRY(check_launch("stats_partial_kernel"));
  stats_finalize_kernel<<<batch, kStatThreads, 0, stream>>>(partial, kStatChunks, n_obs, stats);
  return check_launch("stats_finalize_kernel");
}

int normalize_template(float* x, const float* m, int64_t m_item_stride, int e0, int e1, int e2,
                       int o1, int o2, int64_t item_stride, int batch, double n_obs, double* ws,
                       cudaStream_t stream) {
  TM_TRY(template_stats(x, m, m_item_stride, e0, e1, e2, o1, o2, item_stride, batch, n_obs, ws,
                        stream));
  const double* stats = ws + (int64_t)batch * kStatChunks * 3;
  dim3 grid(kStatChunks, batch);
  normalize_apply_kernel<<<grid, kStatThreads, 0, stream>>>(x, m, m_item_stride, e0, e1, e2, o1,
                                                            o2, item_stride, stats);
  return check_launch("normalize_apply_kernel");
}

// --------------------------------------------------------------- norm_scores
// NumpyFFTWBackend.norm_scores (tme/backends/npfftw_backend.py:537-587), evaluated in
// double: sd = sqrt(max(exp_sq/n - (sq_exp/n)^2, 0)); sd < eps -> 1; out = arr/(sd*n).
// arr == nullptr stands for the scalar 1 the FLCSphericalMask setup passes.
__global__ void norm_scores_kernel(const float* __restrict__ arr, const float* __restrict__ exp_sq,
                                   const float* __restrict__ sq_exp, double n_obs,
                                   const float* __restrict__ n_obs_dev, double eps,
                                   float* __restrict__ out, int64_t n) {
  const double nobs = n_obs_dev ? (double)*n_obs_dev : n_obs;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double e = (double)sq_exp[i] / nobs;
    double e2 = (double)exp_sq[i] / nobs;
    double var = e2 - e * e;
    double sd = sqrt(var > 0 ? var : 0.0);
    if (sd < eps) sd = 1.0;
    double a = arr ? (double)arr[i] : 1.0;
    out[i] = (float)(a / (sd * nobs));
  }
}

int norm_scores(const float* arr, const float* exp_sq, const float* sq_exp, double n_obs,
                const float* n_obs_dev, double eps, float* out, int64_t n, cudaStream_t stream) {
  TM_REQUIRE(exp_sq && sq_exp && out, "norm_scores: null pointer");
  if (n <= 0) return TM_OK;
  int64_t blocks = ceil_div(n, 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  norm_scores_kernel<<<(unsigned)blocks, 256, 0, stream>>>(arr, exp_sq, sq_exp, n_obs, n_obs_dev,
                                                          eps, out, n);
  return check_launch("norm_scores_kernel");
}

// --------------------------------------------------------------- max over rotations
// max_score_over_rotations (tme/backends/npfftw_backend.py:503-535): strict >, so
// the earliest rotation wins ties.
__global__ void max_update_kernel(const float* __restrict__ s, float* __restrict__ mx,
                                  int32_t* __restrict__ rot, int32_t index, int64_t n) {
  int64_t n4 = n / 4;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n4;
       i += (int64_t)gridDim.x * blockDim.x) {
    float4 a = reinterpret_cast<const float4*>(s)[i];
    float4 b = reinterpret_cast<float4*>(mx)[i];
    int4 r = reinterpret_cast<int4*>(rot)[i];
    bool u0 = a.x > b.x, u1 = a.y > b.y, u2 = a.z > b.z, u3 = a.w > b.w;
    if (u0 | u1 | u2 | u3) {
      if (u0) { b.x = a.x; r.x = index; }
      if (u1) { b.y = a.y; r.y = index; }
      if (u2) { b.z = a.z; r.z = index; }
      if (u3) { b.w = a.w; r.w = index; }
      reinterpret_cast<float4*>(mx)[i] = b;
      reinterpret_cast<int4*>(rot)[i] = r;
    }
  }
  for (int64_t i = n4 * 4 + (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    if (s[i] > mx[i]) {
      mx[i] = s[i];
      rot[i] = index;
    }
  }
}

int max_score_over_rotations(const float* scores, float* max_scores, int32_t* rotations,
                             int32_t index, int64_t n, cudaStream_t stream) {
  TM_REQUIRE(scores && max_scores && rotations, "max_score_over_rotations: null pointer");
  TM_REQUIRE(((uintptr_t)scores | (uintptr_t)max_scores | (uintptr_t)rotations) % 16 == 0,
             "max_score_over_rotations: buffers must be 16-byte aligned");
  if (n <= 0) return TM_OK;
  int64_t blocks = ceil_div(n / 4 + 1, 256);
  if (blocks > 148 * 8) blocks = 148 * 8;
  max_update_kernel<<<(unsigned)blocks, 256, 0, stream>>>(scores, max_scores, rotations, index, n);
  return check_launch("max_update_kernel");
}

// --------------------------------------------------------------- plain-path helpers
// out = a * b (complex), optionally times a real filter f (same layout as a).
__global__ void cmul_kernel(const float2* __restrict__ a, const float2* __restrict__ b,
                            float2* __restrict__ out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float2 x = a[i], y = b[i];
    out[i] = make_float2(x.x * y.x - x.y * y.y, x.x * y.y + x.y * y.x);
  }
}

int complex_multiply(const void* a, const void* b, void* out, int64_t n, cudaStream_t stream) {
  if (n <= 0) return TM_OK;
  int64_t blocks = ceil_div(n, 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  cmul_kernel<<<(unsigned)blocks, 256, 0, stream>>>((const float2*)a, (const float2*)b,
                                                   (float2*)out, n);
  return check_launch("cmul_kernel");
}

// spectrum *= real filter, broadcast over a batch of spectra
__global__ void filter_kernel(float2* __restrict__ x, const float* __restrict__ f, int64_t n,
                              int batch) {
  const int64_t total = n * batch;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (int64_t)gridDim.x * blockDim.x) {
    float w = f[i % n];
    float2 v = x[i];
    x[i] = make_float2(v.x * w, v.y * w);
  }
}

int apply_real_filter(void* spectra, const float* filt, int64_t n, int batch, cudaStream_t stream) {
  if (n <= 0 || batch <= 0) return TM_OK;
  int64_t blocks = ceil_div(n * batch, 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  filter_kernel<<<(unsigned)blocks, 256, 0, stream>>>((float2*)spectra, filt, n, batch);
  return check_launch("filter_kernel");
}

// x *= s
__global__ void scale_kernel(float* __restrict__ x, float s, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    x[i] *= s;
}

int scale_real(float* x, float s, int64_t n, cudaStream_t stream) {
  if (n <= 0) return TM_OK;
  int64_t blocks = ceil_div(n, 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  scale_kernel<<<(unsigned)blocks, 256, 0, stream>>>(x, s, n);
  return check_launch("scale_kernel");
}

// Epilogue of the plain path: score = x * scale * (inv_den ? inv_den : 1), optionally
// through FLC normalisation with the CC(f,m) / CC(f^2,m) maps, then the strict-> update.
__global__ void plain_epilogue_kernel(const float* __restrict__ x, const float* __restrict__ inv_den,
                                      const float* __restrict__ cc_m, const float* __restrict__ cc_m2,
                                      const double* __restrict__ stats, double eps, float scale,
                                      float* __restrict__ mx, int32_t* __restrict__ rot,
                                      int32_t index, int64_t n) {
  double nobs = 0.0;
  if (cc_m) nobs = stats[2];
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float s;
    if (cc_m) {
      double e = (double)cc_m[i] * (double)scale / nobs;
      double e2 = (double)cc_m2[i] * (double)scale / nobs;
      double var = e2 - e * e;
      double sd = sqrt(var > 0 ? var : 0.0);
      if (sd < eps) sd = 1.0;
      s = (float)((double)x[i] * (double)scale / (sd * nobs));
    } else {
      s = x[i] * scale;
      if (inv_den) s *= inv_den[i];
    }
    if (s > mx[i]) {
      mx[i] = s;
      rot[i] = index;
    }
  }
}

int plain_epilogue(const float* x, const float* inv_den, const float* cc_m, const float* cc_m2,
                   const double* stats, double eps, float scale, float* mx, int32_t* rot,
                   int32_t index, int64_t n, cudaStream_t stream) {
  int64_t blocks = ceil_div(n, 256);
  if (blocks > 148 * 16) blocks = 148 * 16;
  plain_epilogue_kernel<<<(unsigned)blocks, 256, 0, stream>>>(x, inv_den, cc_m, cc_m2, stats, eps,
                                                             scale, mx, rot, index, n);
  return check_launch("plain_epilogue_kernel");
}

// copy a (t0,t1,t2) box into the top-left of a zeroed (n0,n1,n2) array
__global__ void pad_box_kernel(const float* __restrict__ src, int t0, int t1, int t2,
                               float* __restrict__ dst, int n1, int n2) {
  const int64_t n = (int64_t)t0 * t1 * t2;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (int64_t)gridDim.x * blockDim.x) {
    int i2 = (int)(v % t2);
    int64_t r = v / t2;
    int i1 = (int)(r % t1);
    int i0 = (int)(r / t1);
    dst[((int64_t)i0 * n1 + i1) * n2 + i2] = src[v];
  }
}

int pad_box(const float* src, int t0, int t1, int t2, float* dst, int n1, int n2,
            cudaStream_t stream) {
  int64_t n = (int64_t)t0 * t1 * t2;
  int64_t blocks = ceil_div(n, 256);
  if (blocks > 4096) blocks = 4096;
  pad_box_kernel<<<(unsigned)blocks, 256, 0, stream>>>(src, t0, t1, t2, dst, n1, n2);
  return check_launch("pad_box_kernel");
}

}  // namespace tmb
