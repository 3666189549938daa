// Fourier filters built on the device: the CTF of a reconstructed volume and the
// continuous missing wedge, multiplied together in the order given, written directly
// in rfft (or full) layout with the DC term at index 0.
//
// Each voxel reproduces the reference's array arithmetic step for step, with the same
// float32 / float64 types (tme/filters/ctf.py:260-336 and 528-655,
// tme/filters/wedge.py:282-374, tme/filters/_utils.py:146-202, compose.py:36-59):
// * the frequency grid of fftfreqn is float32((i - n//2) / n) per axis, its Euclidean
//   norm the float32 sum of float32 squares, square-rooted in float32;
// * the CTF phase chi = (df - h k^2) * pi*lambda * k^2 + phase + atan(A/sqrt(1-A^2)) is
//   float64 from the float32 k^2, then sin(-chi) inside the cutoff, negated, optionally
//   made absolute, and cast to float32;
// * the wedge keeps a voxel when its tilt/opening index ratio lies outside the wedge
//   (start <= ratio or stop >= ratio, float64) and its frequency is within the cutoff;
// * the Compose product is float32.
// Scalars that depend only on the filter parameters (wavelength, aberration term,
// wedge bounds) are computed by the caller in float64 the way the reference does.
#include "common.cuh"
#include "ops.cuh"

#include <algorithm>
#include <cmath>

namespace tmb {

namespace {

struct FilterProgram {
  int n;
  tm_filter_component c[TM_FILTER_MAX_COMPONENTS];
};

__device__ __forceinline__ int centred_frequency(int k, int n) {
  // index k of the DC-at-0 layout -> (i - n//2) of the centred grid
  // (shift_fourier rolls by n//2 + n%2, tme/filters/_utils.py:233-246)
  const int shift = n / 2 + n % 2;
  int i = k - shift;
  i %= n;
  if (i < 0) i += n;
  return i - n / 2;
}

__device__ __forceinline__ float grid_norm(const int f[3], const int n[3]) {
  float acc = 0.f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float g = (float)((double)f[a] / (double)n[a]);
    acc = __fadd_rn(acc, __fmul_rn(g, g));
  }
  return __fsqrt_rn(acc);
}

__device__ __forceinline__ float ctf_value(const tm_filter_component& c, float k) {
  // p: 0 defocus_x, 1 h = 0.5 * aberration, 2 pi * lambda, 3 phase shift,
  //    4 amplitude-contrast phase, 5 cutoff, 6 flip phase (0/1)
  const float ksq = __fmul_rn(k, k);
  const double kd = (double)ksq;
  double chi = __dsub_rn(c.p[0], __dmul_rn(c.p[1], kd));
  chi = __dmul_rn(chi, c.p[2]);
  chi = __dmul_rn(chi, kd);
  chi = __dadd_rn(chi, c.p[3]);
  chi = __dadd_rn(chi, c.p[4]);
  double s = sin(-chi);
  s = (k < (float)c.p[5]) ? s : 0.0 * s;
  double v = -s;
  if (c.p[6] != 0.0) v = fabs(v);
  return (float)v;
}

__device__ __forceinline__ float wedge_value(const tm_filter_component& c, const int f[3],
                                             float k) {
  // p: 0 start, 1 stop, 2 ratio used where the opening index is 0, 3 opening axis,
  //    4 tilt axis, 5 frequency cutoff (negative: none)
  const int oa = (int)c.p[3], ta = (int)c.p[4];
  const double ratio = f[oa] == 0 ? c.p[2] : (double)f[ta] / (double)f[oa];
  float v = (c.p[0] <= ratio || c.p[1] >= ratio) ? 1.f : 0.f;
  if (c.p[5] >= 0.0 && !(k <= (float)c.p[5])) v = 0.f;
  return v > 0.f ? 1.f : 0.f;
}

__global__ void build_filter_kernel(FilterProgram prog, int n0, int n1, int n2, int rfft,
                                    float* __restrict__ out) {
  const int m2 = rfft ? n2 / 2 + 1 : n2;
  const int64_t total = (int64_t)n0 * n1 * m2;
  const int n[3] = {n0, n1, n2};
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < total;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int k2 = (int)(v % m2);
    const int64_t r = v / m2;
    const int k1 = (int)(r % n1), k0 = (int)(r / n1);
    const int f[3] = {centred_frequency(k0, n0), centred_frequency(k1, n1),
                      centred_frequency(k2, n2)};
    const float k = grid_norm(f, n);
    float acc = 1.f;
    for (int i = 0; i < prog.n; ++i) {
      const tm_filter_component& c = prog.c[i];
      const float x = c.kind == TM_FILTER_CTF ? ctf_value(c, k) : wedge_value(c, f, k);
      acc = i == 0 ? x : __fmul_rn(x, acc);
    }
    out[v] = acc;
  }
}

// ---------------------------------------------------------------------------------
// Linear whitening (tme/filters/whitening.py:39-186). On the rfft grid of the data
// (shape (m0, m1, h), DC at index 0) the frequency of index k along the first two axes
// is the signed index f = k or k - m (numpy's fftshift order), along the last f = k; the
// grid value is the float32 norm of float32(f / d) with d = (m0 // 2, m1 // 2, h - 1)
// (fftfreqn with sampling rate 0.5 on an rfft shape). A value's bin is
// floor(float32(grid * (n_bins - 1)) + 0.5); the power |X|^2 (float32 magnitude, squared
// in float32) is averaged per bin in float64 (ndimage.mean), then r = 1 / sqrt(mean),
// divided by its maximum. The filter at the requested shape samples r linearly
// (map_coordinates, order 1, zero outside [0, n_bins - 1]) at float32(grid * (n_bins - 1))
// of its own grid, and is returned with the DC term at index 0 (shift_fourier).

__device__ __forceinline__ int signed_index(int k, int n) { return k < n - n / 2 ? k : k - n; }

__device__ __forceinline__ float whitening_grid(int f0, int f1, int f2, int d0, int d1, int d2) {
  const float g0 = (float)((double)f0 / (double)d0);
  const float g1 = (float)((double)f1 / (double)d1);
  const float g2 = (float)((double)f2 / (double)d2);
  float acc = __fmul_rn(g0, g0);
  acc = __fadd_rn(acc, __fmul_rn(g1, g1));
  acc = __fadd_rn(acc, __fmul_rn(g2, g2));
  return __fsqrt_rn(acc);
}

// sums and counts per bin: per-block histograms in shared memory, merged with atomics
__global__ void whitening_hist_kernel(const float2* __restrict__ X, int m0, int m1, int h,
                                      int nb, double* __restrict__ sum,
                                      double* __restrict__ cnt) {
  extern __shared__ double hist[];  // [nb sums | nb counts]
  for (int i = threadIdx.x; i < 2 * nb; i += blockDim.x) hist[i] = 0.0;
  __syncthreads();
  const int d0 = m0 / 2, d1 = m1 / 2, d2 = h - 1;
  const float scl = (float)(nb - 1);
  const int64_t total = (int64_t)m0 * m1 * h;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < total;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int k2 = (int)(v % h);
    const int64_t r = v / h;
    const int k1 = (int)(r % m1), k0 = (int)(r / m1);
    const float g = whitening_grid(signed_index(k0, m0), signed_index(k1, m1), k2, d0, d1, d2);
    const int bin = (int)floorf(__fadd_rn(__fmul_rn(g, scl), 0.5f));
    if (bin < 0 || bin >= nb) continue;
    const float2 x = X[v];
    // |x| correctly rounded to float32 (both squares are exact in double)
    const float mag = (float)sqrt((double)x.x * (double)x.x + (double)x.y * (double)x.y);
    atomicAdd(&hist[bin], (double)__fmul_rn(mag, mag));
    atomicAdd(&hist[nb + bin], 1.0);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nb; i += blockDim.x) {
    if (hist[i] != 0.0) atomicAdd(&sum[i], hist[i]);
    if (hist[nb + i] != 0.0) atomicAdd(&cnt[i], hist[nb + i]);
  }
}

// r = 1 / sqrt(sum / count), divided by max(r); a NaN anywhere (an empty bin) makes every
// value NaN, as numpy's max does
__global__ void whitening_radial_kernel(const double* __restrict__ sum,
                                        const double* __restrict__ cnt, int nb,
                                        double* __restrict__ radial) {
  __shared__ double red[256];
  __shared__ int nan_any;
  if (threadIdx.x == 0) nan_any = 0;
  __syncthreads();
  double m = -INFINITY;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) {
    const double r = 1.0 / sqrt(sum[i] / cnt[i]);
    radial[i] = r;
    if (r != r) nan_any = 1;
    m = fmax(m, r);
  }
  red[threadIdx.x] = m;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
    __syncthreads();
  }
  const double mx = nan_any ? (double)NAN : red[0];
  for (int i = threadIdx.x; i < nb; i += blockDim.x) radial[i] = radial[i] / mx;
}

// the filter on the requested grid, times an optional float32 factor (the product of the
// other filters of a Compose), rounded once to float32
__global__ void whitening_interp_kernel(const double* __restrict__ radial, int nb, int n0, int n1,
                                        int n2, int rfft, const float* __restrict__ factor,
                                        float* __restrict__ out) {
  const int m2 = rfft ? n2 / 2 + 1 : n2;
  const int d0 = n0 / 2, d1 = n1 / 2, d2 = rfft ? m2 - 1 : n2 / 2;
  const float scl = (float)(nb - 1);
  const int64_t total = (int64_t)n0 * n1 * m2;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < total;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int k2 = (int)(v % m2);
    const int64_t r = v / m2;
    const int k1 = (int)(r % n1), k0 = (int)(r / n1);
    const float g = whitening_grid(signed_index(k0, n0), signed_index(k1, n1),
                                   rfft ? k2 : signed_index(k2, n2), d0, d1, d2);
    const double c = (double)__fmul_rn(g, scl);
    double w = 0.0;
    if (c >= 0.0 && c <= (double)(nb - 1)) {
      const int i = (int)floor(c);
      const double t = c - (double)i;
      w = __dmul_rn(1.0 - t, radial[i]);
      if (i + 1 < nb) w = __dadd_rn(w, __dmul_rn(t, radial[i + 1]));
    }
    out[v] = (float)(factor ? __dmul_rn(w, (double)factor[v]) : w);
  }
}

}  // namespace

int whitening_bins(const int* data_ft_shape, int n_bins) {
  const int max_bins = std::max(std::max(data_ft_shape[0], data_ft_shape[1]) / 2 + 1,
                                data_ft_shape[2]);
  return n_bins <= 0 ? max_bins : std::min(n_bins, max_bins);
}

int whitening_filter(const float2* data_rfft, const int* data_ft_shape, int n_bins,
                     const int* shape, int rfft, double* work, const float* factor, float* out,
                     cudaStream_t stream) {
  TM_REQUIRE(data_rfft && data_ft_shape && shape && work && out, "whitening_filter: null pointer");
  const int m0 = data_ft_shape[0], m1 = data_ft_shape[1], h = data_ft_shape[2];
  TM_REQUIRE(m0 >= 2 && m1 >= 2 && h >= 2, "whitening_filter: data spectrum shape %d x %d x %d",
             m0, m1, h);
  TM_REQUIRE(shape[0] >= 2 && shape[1] >= 2 && shape[2] >= 2,
             "whitening_filter: filter shape %d x %d x %d", shape[0], shape[1], shape[2]);
  const int nb = whitening_bins(data_ft_shape, n_bins);
  TM_REQUIRE(nb >= 2 && nb <= 4096, "whitening_filter: %d bins", nb);
  double* sum = work;
  double* cnt = work + nb;
  double* radial = work + 2 * nb;
  TM_TRY(cuda_status(cudaMemsetAsync(work, 0, sizeof(double) * 2 * nb, stream),
                     "whitening_filter: clear"));
  const int64_t total = (int64_t)m0 * m1 * h;
  const int64_t blocks = std::min<int64_t>(ceil_div(total, 256), 148 * 8);
  whitening_hist_kernel<<<(unsigned)blocks, 256, sizeof(double) * 2 * nb, stream>>>(
      data_rfft, m0, m1, h, nb, sum, cnt);
  TM_TRY(check_launch("whitening_hist_kernel"));
  whitening_radial_kernel<<<1, 256, 0, stream>>>(sum, cnt, nb, radial);
  TM_TRY(check_launch("whitening_radial_kernel"));
  const int m2 = rfft ? shape[2] / 2 + 1 : shape[2];
  const int64_t tout = (int64_t)shape[0] * shape[1] * m2;
  const int64_t ob = std::min<int64_t>(ceil_div(tout, 256), 148 * 16);
  whitening_interp_kernel<<<(unsigned)ob, 256, 0, stream>>>(radial, nb, shape[0], shape[1],
                                                            shape[2], rfft, factor, out);
  return check_launch("whitening_interp_kernel");
}

int build_filter(const tm_filter_component* comps, int n_comp, const int* shape, int rfft,
                 float* out, cudaStream_t stream) {
  TM_REQUIRE(comps && shape && out, "build_filter: null pointer");
  TM_REQUIRE(n_comp >= 1 && n_comp <= TM_FILTER_MAX_COMPONENTS,
             "build_filter: 1 to %d components", TM_FILTER_MAX_COMPONENTS);
  TM_REQUIRE(shape[0] > 0 && shape[1] > 0 && shape[2] > 0, "build_filter: empty shape");
  FilterProgram prog;
  prog.n = n_comp;
  for (int i = 0; i < n_comp; ++i) {
    TM_REQUIRE(comps[i].kind == TM_FILTER_CTF || comps[i].kind == TM_FILTER_WEDGE,
               "build_filter: unknown component kind %d", comps[i].kind);
    if (comps[i].kind == TM_FILTER_WEDGE) {
      const int oa = (int)comps[i].p[3], ta = (int)comps[i].p[4];
      TM_REQUIRE(oa >= 0 && oa < 3 && ta >= 0 && ta < 3, "build_filter: wedge axes out of range");
    }
    prog.c[i] = comps[i];
  }
  const int m2 = rfft ? shape[2] / 2 + 1 : shape[2];
  const int64_t total = (int64_t)shape[0] * shape[1] * m2;
  const int64_t blocks = std::min<int64_t>(ceil_div(total, 256), 148 * 16);
  build_filter_kernel<<<(unsigned)blocks, 256, 0, stream>>>(prog, shape[0], shape[1], shape[2],
                                                           rfft, out);
  return check_launch("build_filter_kernel");
}

}  // namespace tmb
