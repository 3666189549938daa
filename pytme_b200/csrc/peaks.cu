// Peak calling on the device: the box maximum filter of
// NumpyFFTWBackend.max_filter_coordinates (tme/backends/npfftw_backend.py:200-206,
// scipy.ndimage.maximum_filter with mode="constant", cval=0) and the greedy
// minimum-distance filter of find_candidate_indices
// (tme/external/bindings.cpp:85-126).
#include "common.cuh"
#include "peaks.cuh"

namespace tmb {

// 1D running maximum along one axis of a (n0, n1, n2) volume. The window of
// output i covers inputs [i - size/2, i - size/2 + size - 1] (SciPy's origin-0
// placement); positions outside the axis contribute the constant 0.
__global__ void max_filter_axis_kernel(const float* __restrict__ in, float* __restrict__ out,
                                       int n0, int n1, int n2, int axis, int size) {
  const int64_t total = (int64_t)n0 * n1 * n2;
  const int len = axis == 0 ? n0 : (axis == 1 ? n1 : n2);
  const int64_t stride = axis == 0 ? (int64_t)n1 * n2 : (axis == 1 ? n2 : 1);
  const int lo = size / 2;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < total;
       v += (int64_t)gridDim.x * blockDim.x) {
    int pos;
    if (axis == 2) pos = (int)(v % n2);
    else if (axis == 1) pos = (int)((v / n2) % n1);
    else pos = (int)(v / ((int64_t)n1 * n2));
    const int a = pos - lo, b = a + size - 1;
    float m = (a < 0 || b >= len) ? 0.f : -INFINITY;
    const int s = max(a, 0), e = min(b, len - 1);
    const float* base = in + (v - (int64_t)pos * stride);
    for (int j = s; j <= e; ++j) m = fmaxf(m, __ldg(base + (int64_t)j * stride));
    out[v] = m;
  }
}

// mask[v] = (filtered[v] == scores[v])
__global__ void peak_mask_kernel(const float* __restrict__ f, const float* __restrict__ s,
                                 uint8_t* __restrict__ mask, int64_t n) {
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (int64_t)gridDim.x * blockDim.x)
    mask[v] = f[v] == s[v];
}

int max_filter_peaks(const float* scores, int n0, int n1, int n2, int size, float* tmp_a,
                     float* tmp_b, uint8_t* mask, cudaStream_t stream) {
  TM_REQUIRE(scores && tmp_a && tmp_b && mask, "max_filter_peaks: null pointer");
  TM_REQUIRE(n0 > 0 && n1 > 0 && n2 > 0 && size >= 1, "max_filter_peaks: bad shape/size");
  const int64_t n = (int64_t)n0 * n1 * n2;
  int64_t blocks = ceil_div(n, 256);
  if (blocks > 148 * 32) blocks = 148 * 32;
  max_filter_axis_kernel<<<(unsigned)blocks, 256, 0, stream>>>(scores, tmp_a, n0, n1, n2, 2, size);
  max_filter_axis_kernel<<<(unsigned)blocks, 256, 0, stream>>>(tmp_a, tmp_b, n0, n1, n2, 1, size);
  max_filter_axis_kernel<<<(unsigned)blocks, 256, 0, stream>>>(tmp_b, tmp_a, n0, n1, n2, 0, size);
  peak_mask_kernel<<<(unsigned)blocks, 256, 0, stream>>>(tmp_a, scores, mask, n);
  return check_launch("max_filter_peaks");
}

// Greedy filter: point 0 is kept; point i is kept when, for every kept point j,
// floor(sqrt(|c_i - c_j|^2)) > min_distance — the integer arithmetic of the int64
// overload the reference's peak callers reach. One CTA walks the points in order;
// the kept coordinates live in `kept` (shared memory when they fit, else the
// caller's workspace), and every thread tests a strided share of them.
constexpr int kNmsThreads = 1024;

__device__ __forceinline__ bool too_close(int64_t dx, int64_t dy, int64_t dz, int64_t md) {
  // floor(sqrt(d2)) <= md is never true for md < 0 (every point is kept) and always
  // true once (md + 1)^2 exceeds any squared distance of 32-bit coordinates
  if (md < 0) return false;
  if (md >= (int64_t)3037000499LL) return true;
  int64_t d2 = dx * dx + dy * dy + dz * dz;
  // floor(sqrt(d2)) <= md  <=>  d2 < (md + 1)^2 for non-negative integers
  return d2 < (md + 1) * (md + 1);
}

__global__ void __launch_bounds__(kNmsThreads)
greedy_nms_kernel(const int64_t* __restrict__ coords, int n, int64_t min_distance,
                  int32_t* __restrict__ out_idx, int32_t* __restrict__ out_count,
                  int64_t* __restrict__ kept_global, int smem_cap) {
  extern __shared__ int64_t kept_smem[];
  int64_t* kept = (n <= smem_cap) ? kept_smem : kept_global;
  __shared__ int count;
  if (threadIdx.x == 0) {
    count = 0;
    if (n > 0) {
      kept[0] = coords[0];
      kept[1] = coords[1];
      kept[2] = coords[2];
      out_idx[0] = 0;
      count = 1;
    }
  }
  __syncthreads();
  for (int i = 1; i < n; ++i) {
    const int64_t x = coords[3 * (int64_t)i], y = coords[3 * (int64_t)i + 1],
                  z = coords[3 * (int64_t)i + 2];
    const int c = count;
    int reject = 0;
    for (int j = threadIdx.x; j < c; j += blockDim.x) {
      if (too_close(x - kept[3 * j], y - kept[3 * j + 1], z - kept[3 * j + 2], min_distance)) {
        reject = 1;
        break;
      }
    }
    reject = __syncthreads_or(reject);
    if (!reject && threadIdx.x == 0) {
      kept[3 * c] = x;
      kept[3 * c + 1] = y;
      kept[3 * c + 2] = z;
      out_idx[c] = i;
      count = c + 1;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0) *out_count = count;
}

int64_t nms_workspace_bytes(int n) { return (int64_t)(n > 0 ? n : 1) * 3 * sizeof(int64_t); }

int greedy_nms(const int64_t* coords, int n, int64_t min_distance, int32_t* out_idx,
               int32_t* out_count, void* workspace, cudaStream_t stream) {
  TM_REQUIRE(n >= 0, "greedy_nms: negative point count");
  TM_REQUIRE(out_idx && out_count, "greedy_nms: null output");
  TM_REQUIRE(n == 0 || coords, "greedy_nms: null coordinates");
  const int smem_cap = 48 * 1024 / (3 * (int)sizeof(int64_t));
  TM_REQUIRE(n <= smem_cap || workspace,
             "greedy_nms: %d points need a workspace of %lld bytes", n,
             (long long)nms_workspace_bytes(n));
  const size_t smem = (size_t)(n <= smem_cap ? (n > 0 ? n : 1) : 1) * 3 * sizeof(int64_t);
  greedy_nms_kernel<<<1, kNmsThreads, smem, stream>>>(coords, n, min_distance, out_idx,
                                                     out_count,
                                                     static_cast<int64_t*>(workspace), smem_cap);
  return check_launch("greedy_nms_kernel");
}

}  // namespace tmb
