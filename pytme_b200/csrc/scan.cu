// Exhaustive rotation scan: the per-rotation loops of corr_scoring
// (tme/matching_scores.py:600-624; CC and FLCSphericalMask) and flc_scoring
// (tme/matching_scores.py:727-757; FLC), with MaxScoreOverRotations state updates
// (tme/analyzer/aggregation.py:142-189, tme/backends/npfftw_backend.py:503-535).
//
// Two execution paths share one plan object:
//
//  * plain: one rotation at a time with full-size cuFFT r2c/c2r transforms of the
//    zero-padded template and separate product/epilogue kernels. This is the
//    straightforward FP32 GPU port of the reference loop and serves as the
//    "plain" baseline.
//
//  * fused: B rotations per launch group through four kernels of this library.
//      K1 tmpl_zy    template rows: direct real DFT along axis 2 (only t2 of n2
//                    inputs are non-zero) and a zero-padded FFT along axis 1,
//                    producing G[b][x < t0][k1][k2]
//      K2 xpass      per (k1, k2-tile) column block: forward FFT along axis 0 of
//                    the zero-padded G columns, product with the target spectrum
//                    (held in registers for all B rotations), inverse FFT along
//                    axis 0 -> H[b][x'][k1][k2]
//      K3 ypass      inverse FFT along axis 1, in place on H
//      K4 zpass      c2r along axis 2 (half-length complex FFT), score scaling and
//                    the strict-> max/argmax over the B rotations in registers,
//                    merged into the caller's state once per launch group
//    H is complex64 ("fp32") or half2 with a fixed scale ("mixed").
//
// Target-side quantities (target spectra and the FLCSphericalMask denominator)
// are computed once by set_target; the denominator and the target mean are
// evaluated in double precision.
#include "colfft.cuh"
#include "common.cuh"
#include "fft_smem.cuh"
#include "ops.cuh"
#include "scan.cuh"
#include "tc_common.cuh"
#include "xcorr_tc.cuh"
#include "ypass_tc.cuh"
#include "zpass_tc.cuh"

#include <type_traits>

#include <cuda_fp16.h>
#include <cufft.h>

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

namespace tmb {

using fft::LinePlan;

static int cufft_status(cufftResult r, const char* what) {
  if (r == CUFFT_SUCCESS) return TM_OK;
  set_error("%s: cuFFT error %d", what, (int)r);
  return r == CUFFT_ALLOC_FAILED ? TM_E_OOM : TM_E_CUFFT;
}

LinePlan make_line_plan(int n) {
  LinePlan p{};
  p.n = n;
  int m = n, e2 = 0;
  while (m % 2 == 0) { m /= 2; ++e2; }
  int k = 0;
  int eights = e2 / 3, rem = e2 % 3;
  if (rem == 1 && eights > 0) { eights -= 1; p.radix[k++] = 4; p.radix[k++] = 4; }
  else if (rem == 1) { p.radix[k++] = 2; }
  else if (rem == 2) { p.radix[k++] = 4; }
  for (int i = 0; i < eights; ++i) p.radix[k++] = 8;
  for (int q : {3, 5, 7, 11, 13}) {
    while (m % q == 0) { m /= q; p.radix[k++] = q; }
  }
  p.npass = (m == 1) ? k : -1;
  return p;
}

static bool line_supported(int n) {
  if (n < 2 || n > 4096) return false;
  LinePlan p = make_line_plan(n);
  return p.npass > 0 && p.npass <= fft::kMaxPasses && fft::supported_radices(p);
}

static std::vector<float2> twiddle_table(int n) {
  std::vector<float2> t(n);
  for (int i = 0; i < n; ++i) {
    double a = -2.0 * M_PI * (double)i / (double)n;
    t[i] = make_float2((float)cos(a), (float)sin(a));
  }
  return t;
}

// ------------------------------------------------------------------ storage types
template <typename T> struct Store;
template <> struct Store<float2> {
  static __device__ __forceinline__ float2 load(const float2* p) { return *p; }
  static __device__ __forceinline__ void store(float2* p, float2 v) { *p = v; }
};
template <> struct Store<__half2> {
  static __device__ __forceinline__ float2 load(const __half2* p) { return __half22float2(*p); }
  static __device__ __forceinline__ void store(__half2* p, float2 v) { *p = __float22half2_rn(v); }
};

// Asynchronous global -> shared copies (cp.async): the next tile is staged in shared
// memory while the current one is transformed. Each thread later reads back only the
// elements it copied, so a thread-local wait_group suffices.
template <int BYTES>
__device__ __forceinline__ void cp_async(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  if constexpr (BYTES == 4)
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(s), "l"(gmem));
  else
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int PENDING>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(PENDING));
}

constexpr int kThreads = 512;
constexpr int kMaxE = 8;             // complex elements per thread in a line-FFT tile
constexpr int kTile = kThreads * kMaxE;  // elements per tile (4096)

// ------------------------------------------------------------------ K1: template z/y
// grid (ceil(h2/W), t0, B); tile: n1 lines-fast rows x W lines (k2).
__global__ void __launch_bounds__(kThreads, 1)
tmpl_zy_kernel(const float* __restrict__ tmpl, int t0, int t1, int t2, int n1, int n2, int h2,
               int W, LinePlan p1, const float2* __restrict__ tw1_g, const float2* __restrict__ tw2_g,
               float2* __restrict__ G) {
  extern __shared__ float4 smem_raw[];
  float2* tw1 = reinterpret_cast<float2*>(smem_raw);
  float2* tw2 = tw1 + n1;
  float2* buf = tw2 + n2;
  float* plane = reinterpret_cast<float*>(buf + (int64_t)n1 * W);
  const int tid = threadIdx.x;
  const int k2_0 = blockIdx.x * W;
  const int x = blockIdx.y;
  const int b = blockIdx.z;
  for (int i = tid; i < n1; i += kThreads) tw1[i] = tw1_g[i];
  for (int i = tid; i < n2; i += kThreads) tw2[i] = tw2_g[i];
  const float* src = tmpl + ((int64_t)b * t0 + x) * t1 * t2;
  for (int i = tid; i < t1 * t2; i += kThreads) plane[i] = src[i];
  __syncthreads();
  // G1[y][k2] = sum_z plane[y][z] * exp(-2 pi i z k2 / n2), rows y >= t1 are zero
  for (int e = tid; e < n1 * W; e += kThreads) {
    int y = e / W, l = e % W;
    int k2 = k2_0 + l;
    float2 acc = make_float2(0.f, 0.f);
    if (y < t1 && k2 < h2) {
      const float* row = plane + y * t2;
      int idx = 0;
      for (int z = 0; z < t2; ++z) {
        float v = row[z];
        float2 w = tw2[idx];
        acc.x += v * w.x;
        acc.y += v * w.y;
        idx += k2;
        if (idx >= n2) idx -= n2;
      }
    }
    buf[e] = acc;
  }
  __syncthreads();
  fft::fft_lines<-1, kMaxE, true>(buf, p1, W, 1, W, tw1, n1, tid, kThreads);
  float2* dst = G + ((int64_t)b * t0 + x) * n1 * h2;
  for (int e = tid; e < n1 * W; e += kThreads) {
    int k1 = e / W, l = e % W;
    int k2 = k2_0 + l;
    if (k2 < h2) dst[(int64_t)k1 * h2 + k2] = buf[e];
  }
}

// ------------------------------------------------------------------ K2: x pass
// grid (ceil(h2/W), n1); loops over the B rotations of the group.
template <typename HT>
__global__ void __launch_bounds__(kThreads, 1)
xpass_kernel(const float2* __restrict__ G, const float2* __restrict__ Ft, int B, int t0, int n0,
             int n1, int h2, int W, LinePlan p0, const float2* __restrict__ tw0_g, float scale,
             HT* __restrict__ H, int hp) {
  extern __shared__ float4 smem_raw[];
  float2* tw0 = reinterpret_cast<float2*>(smem_raw);
  float2* buf = tw0 + n0;
  const int tid = threadIdx.x;
  const int k2_0 = blockIdx.x * W;
  const int k1 = blockIdx.y;
  for (int i = tid; i < n0; i += kThreads) tw0[i] = tw0_g[i];
  const int tile = n0 * W;
  // target-spectrum tile: re-read through L1 for every rotation of the group
  const float2* ft_col = Ft + (int64_t)k1 * h2 + k2_0;
  const int64_t ft_row = (int64_t)n1 * h2;
  const int64_t S = (int64_t)n0 * n1 * h2;
  const int64_t SH = (int64_t)n0 * n1 * hp;
  for (int b = 0; b < B; ++b) {
    const float2* g = G + (int64_t)b * t0 * n1 * h2;
    for (int e = tid; e < tile; e += kThreads) {
      int x = e / W, l = e % W;
      int k2 = k2_0 + l;
      float2 v = make_float2(0.f, 0.f);
      if (x < t0 && k2 < h2) v = g[((int64_t)x * n1 + k1) * h2 + k2];
      buf[e] = v;
    }
    __syncthreads();
    fft::fft_lines<-1, kMaxE, true>(buf, p0, W, 1, W, tw0, n0, tid, kThreads);
    for (int e = tid; e < tile; e += kThreads) {
      int k0 = e / W, l = e % W;
      float2 f = make_float2(0.f, 0.f);
      if (k2_0 + l < h2) f = __ldg(ft_col + k0 * ft_row + l);
      buf[e] = fft::cmul(buf[e], make_float2(f.x * scale, f.y * scale));
    }
    __syncthreads();
    fft::fft_lines<1, kMaxE, true>(buf, p0, W, 1, W, tw0, n0, tid, kThreads);
    HT* h = H + (int64_t)b * SH;
    for (int e = tid; e < tile; e += kThreads) {
      int x = e / W, l = e % W;
      int k2 = k2_0 + l;
      if (k2 < h2) Store<HT>::store(h + ((int64_t)x * n1 + k1) * hp + k2, buf[e]);
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------ K3: y pass
// grid (ceil(h2/W), n0, B): inverse FFT along axis 1, in place.
template <typename HT>
__global__ void __launch_bounds__(kThreads, 1)
ypass_kernel(HT* __restrict__ H, int n0, int n1, int h2, int W, LinePlan p1,
             const float2* __restrict__ tw1_g, int hp) {
  extern __shared__ float4 smem_raw[];
  float2* tw1 = reinterpret_cast<float2*>(smem_raw);
  float2* buf = tw1 + n1;
  const int tid = threadIdx.x;
  const int k2_0 = blockIdx.x * W;
  const int x = blockIdx.y;
  const int b = blockIdx.z;
  for (int i = tid; i < n1; i += kThreads) tw1[i] = tw1_g[i];
  const int tile = n1 * W;
  HT* h = H + (int64_t)b * n0 * n1 * hp + (int64_t)x * n1 * hp;
  for (int e = tid; e < tile; e += kThreads) {
    int y = e / W, l = e % W;
    int k2 = k2_0 + l;
    buf[e] = (k2 < h2) ? Store<HT>::load(h + (int64_t)y * hp + k2) : make_float2(0.f, 0.f);
  }
  __syncthreads();
  fft::fft_lines<1, kMaxE, true>(buf, p1, W, 1, W, tw1, n1, tid, kThreads);
  for (int e = tid; e < tile; e += kThreads) {
    int y = e / W, l = e % W;
    int k2 = k2_0 + l;
    if (k2 < h2) Store<HT>::store(h + (int64_t)y * hp + k2, buf[e]);
  }
}

// ------------------------------------------------------------------ register-resident passes
// Power-of-two axis lengths use the column codelet of colfft.cuh: T = N/8 threads
// per column, W columns per CTA (thread id = t*W + l, so a warp spans W columns and
// each global row segment of W elements is one contiguous access).

// Stage 0 of the forward DIF when only rows [0, nz) of the column are non-zero and
// nz <= T: the radix-8 DFT of a single non-zero input is that input, so output j is
// x[t] * W_N^(j*t).
template <int N>
__device__ __forceinline__ void stage0_single(float2 (&v)[8], int t, const float2* tw) {
  const float2 w1 = tw[t];
  float2 x = v[0];
  v[0] = x;
#pragma unroll
  for (int j = 1; j < 8; ++j) {
    x = fft::cmul(x, w1);
    v[j] = x;
  }
}

template <int N, int W, int DIR>
__device__ __forceinline__ void dif_rest(float2 (&v)[8], float2* sm, const float2* tw, int l,
                                         int t) {
  constexpr int NS = colfft::num_stages(N);
  colfft::store_stage<N, W, 0>(v, sm, l, t);
  __syncthreads();
  if constexpr (NS > 1) {
    colfft::load_stage<N, W, 1>(v, sm, l, t);
    colfft::dif_stage_regs<N, 1, DIR>(v, t, tw);
  }
  if constexpr (NS > 2) {
    colfft::store_stage<N, W, 1>(v, sm, l, t);
    __syncthreads();
    colfft::load_stage<N, W, 2>(v, sm, l, t);
    colfft::dif_stage_regs<N, 2, DIR>(v, t, tw);
  }
  if constexpr (NS > 3) {
    colfft::store_stage<N, W, 2>(v, sm, l, t);
    __syncthreads();
    colfft::load_stage<N, W, 3>(v, sm, l, t);
    colfft::dif_stage_regs<N, 3, DIR>(v, t, tw);
  }
}

// K1': template rows -> G. grid (ceil(h2/W), t0, B); N = n1.
template <int N, int W, typename GT = float2>
__global__ void __launch_bounds__(N / 8 * W, 1)
tmpl_zy_reg_kernel(const float* __restrict__ tmpl, int t0, int t1, int t2, int n2, int h2,
                   const float2* __restrict__ tw1_g, const float2* __restrict__ tw2_g,
                   GT* __restrict__ G) {
  constexpr int T = N / 8;
  constexpr int NT = T * W;
  extern __shared__ float4 smem_raw[];
  float2* tw1 = reinterpret_cast<float2*>(smem_raw);
  float2* sm = tw1 + N;
  float2* tw2 = sm + colfft::smem_elems<N>(W);
  float* plane = reinterpret_cast<float*>(tw2 + n2);
  const int tid = threadIdx.x, l = tid % W, t = tid / W;
  const int k2 = blockIdx.x * W + l;
  const int x = blockIdx.y, b = blockIdx.z;
  for (int i = tid; i < N; i += NT) tw1[i] = tw1_g[i];
  for (int i = tid; i < n2; i += NT) tw2[i] = tw2_g[i];
  const float* src = tmpl + ((int64_t)b * t0 + x) * t1 * t2;
  for (int i = tid; i < t1 * t2; i += NT) plane[i] = src[i];
  __syncthreads();
  float2 v[8];
#pragma unroll
  for (int r = 0; r < 8; ++r) {
    const int y = t + T * r;
    float2 acc = make_float2(0.f, 0.f);
    if (y < t1 && k2 < h2) {
      const float* row = plane + y * t2;
      int idx = 0;
      for (int z = 0; z < t2; ++z) {
        const float a = row[z];
        const float2 w = tw2[idx];
        acc.x += a * w.x;
        acc.y += a * w.y;
        idx += k2;
        if (idx >= n2) idx -= n2;
      }
    }
    v[r] = acc;
  }
  if (t1 <= T) stage0_single<N>(v, t, tw1);
  else colfft::dif_stage_regs<N, 0, -1>(v, t, tw1);
  dif_rest<N, W, -1>(v, sm, tw1, l, t);
  if (k2 < h2) {
    GT* dst = G + ((int64_t)b * t0 + x) * N * h2;
    constexpr int R = colfft::stage_radix(N, colfft::num_stages(N) - 1);
#pragma unroll
    for (int i = 0; i < 8 / R; ++i)
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int k1 = colfft::out_index<N>(t, i, r);
        Store<GT>::store(dst + (int64_t)k1 * h2 + k2, v[i * R + r]);
      }
  }
}

// K2': x pass. grid (ceil(h2/W), n1); N = n0; loops over the rotations of the group.
template <int N, int W, typename HT>
__global__ void __launch_bounds__(N / 8 * W, 1024 / (N / 8 * W))
xpass_reg_kernel(const float2* __restrict__ G, const float2* __restrict__ Ft, int B, int t0,
                 int n1, int h2, const float2* __restrict__ tw0_g, float scale,
                 HT* __restrict__ H, int hp) {
  constexpr int T = N / 8;
  constexpr int NT = T * W;
  constexpr int R = colfft::stage_radix(N, colfft::num_stages(N) - 1);
  extern __shared__ float4 smem_raw[];
  float2* tw = reinterpret_cast<float2*>(smem_raw);
  float2* sm = tw + N;
  const int tid = threadIdx.x, l = tid % W, t = tid / W;
  const int k2 = blockIdx.x * W + l;
  const int k1 = blockIdx.y;
  const bool valid = k2 < h2;
  for (int i = tid; i < N; i += NT) tw[i] = tw0_g[i];
  // offsets of the target-spectrum values this thread multiplies (through L1, reused
  // by every rotation of the group)
  const int64_t col = (int64_t)k1 * h2 + k2;
  const int64_t row = (int64_t)n1 * h2;
  const float2* fb = Ft + (int64_t)colfft::out_index<N>(t, 0, 0) * row + col;
  __syncthreads();
  const int64_t SH = (int64_t)N * n1 * hp, rowH = (int64_t)n1 * hp;
  const int64_t colH = (int64_t)k1 * hp + k2;
  for (int b = 0; b < B; ++b) {
    const float2* g = G + (int64_t)b * t0 * row + col;
    float2 v[8];
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int x = t + T * r;
      v[r] = (valid && x < t0) ? g[(int64_t)x * row] : make_float2(0.f, 0.f);
    }
    if (t0 <= T) stage0_single<N>(v, t, tw);
    else colfft::dif_stage_regs<N, 0, -1>(v, t, tw);
    dif_rest<N, W, -1>(v, sm, tw, l, t);
#pragma unroll
    for (int i = 0; i < 8 / R; ++i)
#pragma unroll
      for (int r = 0; r < R; ++r) {
        // out_index(t, i, r) = out_index(t, i, 0) + r * N/R; out_index(t, i, 0) - out_index(t, 0, 0)
        // depends on i only through compile-time digits
        const int dk = colfft::out_index<N>(t, i, r) - colfft::out_index<N>(t, 0, 0);
        const float2 f = valid ? __ldg(fb + (int64_t)dk * row) : make_float2(0.f, 0.f);
        v[i * R + r] = fft::cmul(v[i * R + r], make_float2(f.x * scale, f.y * scale));
      }
    colfft::dif_adjoint<N, W>(v, sm, tw, l, t);
    if (valid) {
      HT* h = H + (int64_t)b * SH + colH;
#pragma unroll
      for (int r = 0; r < 8; ++r) Store<HT>::store(h + (int64_t)(t + T * r) * rowH, v[r]);
    }
  }
}

// K3': y pass (inverse FFT along axis 1, in place). grid (ceil(h2/W), ceil(n0/XP), B);
// each CTA walks XP consecutive x planes; the next plane's columns are staged in shared
// memory with cp.async while the current plane is transformed (each thread stages and
// later reads only its own elements, so a stage is reused without a barrier). The pass
// is bound by instruction issue and shared-memory traffic, not by loads in flight:
// three or four staged planes measured slower than two. N = n1.
constexpr int kYPlanes = 8;
constexpr int kYStages = 2;

template <int N, int W, typename HT>
__global__ void __launch_bounds__(N / 8 * W, 1024 / (N / 8 * W))
ypass_reg_kernel(HT* __restrict__ H, int n0, int h2, const float2* __restrict__ tw1_g, int hp,
                 int seg) {
  constexpr int T = N / 8;
  constexpr int NT = T * W;
  constexpr int R = colfft::stage_radix(N, colfft::num_stages(N) - 1);
  extern __shared__ float4 smem_raw[];
  float2* tw = reinterpret_cast<float2*>(smem_raw);
  float2* sm = tw + N;
  HT* stage = reinterpret_cast<HT*>(sm + colfft::smem_elems<N>(W));  // kYStages x N*W staging
  const int tid = threadIdx.x, l = tid % W, t = tid / W;
  const int k2 = blockIdx.x * W + l;
  const int x0 = blockIdx.y * kYPlanes, b = blockIdx.z;
  const int nx = min(kYPlanes, n0 - x0);
  const bool valid = k2 < h2;
  for (int i = tid; i < N; i += NT) tw[i] = tw1_g[i];
  HT* base = H + ((int64_t)b * n0 + x0) * N * hp + k2;
  const int64_t plane = (int64_t)N * hp;
  auto fetch = [&](int xi) {
    if (valid && xi < nx) {
      HT* dst = stage + (xi % kYStages) * N * W;
      const HT* src = base + (int64_t)xi * plane;
#pragma unroll
      for (int r = 0; r < 8; ++r)
        cp_async<sizeof(HT)>(dst + (t + T * r) * W + l, src + (int64_t)(t + T * r) * hp);
    }
    cp_async_commit();  // one group per plane, empty past the last
  };
#pragma unroll
  for (int xi = 0; xi < kYStages - 1; ++xi) fetch(xi);
  __syncthreads();  // twiddles
  for (int xi = 0; xi < nx; ++xi) {
    HT* cur = stage + (xi % kYStages) * N * W;
    fetch(xi + kYStages - 1);
    cp_async_wait<kYStages - 1>();  // plane xi landed
    float2 v[8];
#pragma unroll
    for (int r = 0; r < 8; ++r)
      v[r] = valid ? Store<HT>::load(cur + (t + T * r) * W + l) : make_float2(0.f, 0.f);
    colfft::dif_stage_regs<N, 0, 1>(v, t, tw);
    dif_rest<N, W, 1>(v, sm, tw, l, t);
    if constexpr (std::is_same<HT, __half2>::value) {
      if (seg) {
        // 32-byte segments [Re x 8 | Im x 8] of 8 consecutive k2 (the even/odd tensor-core
        // z pass's input): the 8 lanes holding one row's segment exchange values so each
        // stores one word, (Re, Re) of columns 2q, 2q+1 for q < 4, (Im, Im) after that
        const int q = l & 7, lane = threadIdx.x & 31;
        const int srcA = (lane & ~7) | ((2 * q) & 7);
        const uint32_t sel = q < 4 ? 0x5410u : 0x7632u;
        HT* h = base + (int64_t)xi * plane;
#pragma unroll
        for (int i = 0; i < 8 / R; ++i)
#pragma unroll
          for (int r = 0; r < R; ++r) {
            const int y = colfft::out_index<N>(t, i, r);
            const __half2 hv = __float22half2_rn(v[i * R + r]);
            uint32_t w = *reinterpret_cast<const uint32_t*>(&hv);
            const uint32_t a = __shfl_sync(0xffffffffu, w, srcA);
            const uint32_t b = __shfl_sync(0xffffffffu, w, srcA + 1);
            w = __byte_perm(a, b, sel);
            if (k2 < hp) *reinterpret_cast<uint32_t*>(h + (int64_t)y * hp) = w;
          }
        __syncthreads();  // the next plane's stage-0 stores reuse the exchange buffer
        continue;
      }
    }
    if (valid) {
      HT* h = base + (int64_t)xi * plane;
#pragma unroll
      for (int i = 0; i < 8 / R; ++i)
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int y = colfft::out_index<N>(t, i, r);
          Store<HT>::store(h + (int64_t)y * hp, v[i * R + r]);
        }
    }
    __syncthreads();  // the next plane's stage-0 stores reuse the exchange buffer
  }
}

// K2'' (FLC): x pass with three outputs per rotation. The rotated mask's spectrum is
// transformed once and multiplied by the spectra of f and f^2 (the local mean and
// mean square under the mask, CC(f, m) and CC(f^2, m)); the normalised template's
// spectrum is multiplied by the spectrum of f (the numerator). The two statistics
// outputs are always complex64.
template <int N, int W, typename HT>
__global__ void __launch_bounds__(N / 8 * W, 1)
xpass_flc_reg_kernel(const float2* __restrict__ Gt, const float2* __restrict__ Gm,
                     const float2* __restrict__ Ft, const float2* __restrict__ Ft2, int B, int t0,
                     int n1, int h2, const float2* __restrict__ tw0_g, float scale,
                     HT* __restrict__ Ht, float2* __restrict__ Hm, float2* __restrict__ Hm2,
                     int hp) {
  constexpr int T = N / 8;
  constexpr int NT = T * W;
  constexpr int R = colfft::stage_radix(N, colfft::num_stages(N) - 1);
  extern __shared__ float4 smem_raw[];
  float2* tw = reinterpret_cast<float2*>(smem_raw);
  float2* sm = tw + N;
  const int tid = threadIdx.x, l = tid % W, t = tid / W;
  const int k2 = blockIdx.x * W + l;
  const int k1 = blockIdx.y;
  const bool valid = k2 < h2;
  for (int i = tid; i < N; i += NT) tw[i] = tw0_g[i];
  int64_t foff[8];
#pragma unroll
  for (int i = 0; i < 8 / R; ++i)
#pragma unroll
    for (int r = 0; r < R; ++r) {
      const int k0 = colfft::out_index<N>(t, i, r);
      foff[i * R + r] = ((int64_t)k0 * n1 + k1) * h2 + k2;
    }
  __syncthreads();
  const int64_t row = (int64_t)n1 * h2;
  const int64_t col = (int64_t)k1 * h2 + k2;
  const int64_t S = (int64_t)N * n1 * hp, rowH = (int64_t)n1 * hp;
  const int64_t colH = (int64_t)k1 * hp + k2;
  for (int b = 0; b < B; ++b) {
    // mask spectrum along axis 0
    float2 vm[8], v[8];
    const float2* gm = Gm + (int64_t)b * t0 * row + col;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int x = t + T * r;
      vm[r] = (valid && x < t0) ? gm[(int64_t)x * row] : make_float2(0.f, 0.f);
    }
    if (t0 <= T) stage0_single<N>(vm, t, tw);
    else colfft::dif_stage_regs<N, 0, -1>(vm, t, tw);
    dif_rest<N, W, -1>(vm, sm, tw, l, t);
    // CC(f, m)
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      float2 f = valid ? __ldg(Ft + foff[e]) : make_float2(0.f, 0.f);
      v[e] = fft::cmul(vm[e], make_float2(f.x * scale, f.y * scale));
    }
    colfft::dif_adjoint<N, W>(v, sm, tw, l, t);
    if (valid) {
      float2* h = Hm + (int64_t)b * S + colH;
#pragma unroll
      for (int r = 0; r < 8; ++r) h[(int64_t)(t + T * r) * rowH] = v[r];
    }
    __syncthreads();
    // CC(f^2, m)
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      float2 f = valid ? __ldg(Ft2 + foff[e]) : make_float2(0.f, 0.f);
      v[e] = fft::cmul(vm[e], make_float2(f.x * scale, f.y * scale));
    }
    colfft::dif_adjoint<N, W>(v, sm, tw, l, t);
    if (valid) {
      float2* h = Hm2 + (int64_t)b * S + colH;
#pragma unroll
      for (int r = 0; r < 8; ++r) h[(int64_t)(t + T * r) * rowH] = v[r];
    }
    __syncthreads();
    // numerator CC(f, t)
    const float2* gt = Gt + (int64_t)b * t0 * row + col;
#pragma unroll
    for (int r = 0; r < 8; ++r) {
      const int x = t + T * r;
      v[r] = (valid && x < t0) ? gt[(int64_t)x * row] : make_float2(0.f, 0.f);
    }
    if (t0 <= T) stage0_single<N>(v, t, tw);
    else colfft::dif_stage_regs<N, 0, -1>(v, t, tw);
    dif_rest<N, W, -1>(v, sm, tw, l, t);
#pragma unroll
    for (int e = 0; e < 8; ++e) {
      float2 f = valid ? __ldg(Ft + foff[e]) : make_float2(0.f, 0.f);
      v[e] = fft::cmul(v[e], make_float2(f.x * scale, f.y * scale));
    }
    colfft::dif_adjoint<N, W>(v, sm, tw, l, t);
    if (valid) {
      HT* h = Ht + (int64_t)b * S + colH;
#pragma unroll
      for (int r = 0; r < 8; ++r) Store<HT>::store(h + (int64_t)(t + T * r) * rowH, v[r]);
    }
    __syncthreads();
  }
}

template <int N>
constexpr int reg_lines() { return N >= 512 ? 8 : 16; }

template <int N>
size_t reg_smem_bytes(int n2, int t1, int t2, bool with_plane) {
  size_t b = sizeof(float2) * (N + colfft::smem_elems<N>(reg_lines<N>()));
  if (with_plane) b += sizeof(float2) * n2 + sizeof(float) * t1 * t2;
  return b;
}

template <int N, typename HT>
size_t ypass_smem_bytes() {
  return reg_smem_bytes<N>(0, 0, 0, false) + kYStages * sizeof(HT) * N * reg_lines<N>();
}

static bool reg_supported(int n) {
  return n == 64 || n == 128 || n == 256 || n == 512 || n == 1024;
}

// ------------------------------------------------------------------ K4: z pass + epilogue
// grid (ceil(n0*n1/R)); each CTA owns R consecutive (x', y') rows = R*n2 output voxels.
// c2r of length n2 (even) via a complex inverse FFT of length m = n2/2:
//   E[k] = X[k] + conj(X[m-k]),  O[k] = (X[k] - conj(X[m-k])) * exp(+2 pi i k / n2),
//   z = IDFT_m(E + i O)  ->  x[2j] = Re z[j], x[2j+1] = Im z[j]
// with the imaginary parts of X[0] and X[m] dropped, as numpy/pocketfft's c2r does.
constexpr int kMaxV = 8;   // output voxels per thread

template <typename HT, int M = 0>
__global__ void __launch_bounds__(kThreads, 1)
zpass_kernel(const HT* __restrict__ H, int B, int64_t rows, int n2, int hp, int R, LinePlan pm,
             const float2* __restrict__ tw2_g, float scale, const float* __restrict__ inv_den,
             int32_t first_index, float* __restrict__ state_max, int32_t* __restrict__ state_rot,
             int64_t S, const int32_t* __restrict__ first_dev) {
  if (first_dev) first_index = *first_dev;
  extern __shared__ float4 smem_raw[];
  const int m = n2 / 2;
  float2* tw2 = reinterpret_cast<float2*>(smem_raw);
  float2* raw = tw2 + n2;
  float2* buf = raw + (int64_t)R * hp;
  const int tid = threadIdx.x;
  const int64_t row0 = (int64_t)blockIdx.x * R;
  const int nrows = (int)min((int64_t)R, rows - row0);
  for (int i = tid; i < n2; i += kThreads) tw2[i] = tw2_g[i];
  const int nout = nrows * n2;
  const int64_t vox0 = row0 * n2;
  float den[kMaxV], best[kMaxV];
  int32_t arg[kMaxV];
#pragma unroll
  for (int c = 0; c < kMaxV; ++c) {
    int v = tid + c * kThreads;
    den[c] = (v < nout) ? (inv_den ? inv_den[vox0 + v] : 1.f) * scale : 0.f;
    best[c] = -INFINITY;
    arg[c] = -1;
  }
  for (int b = 0; b < B; ++b) {
    const HT* src = H + (int64_t)b * S + row0 * hp;
    for (int e = tid; e < nrows * hp; e += kThreads) raw[e] = Store<HT>::load(src + e);
    __syncthreads();
    for (int e = tid; e < nrows * m; e += kThreads) {
      int r = e / m, k = e % m;
      const float2* xr = raw + (int64_t)r * hp;
      float2 a = xr[k], c = xr[m - k];
      if (k == 0) { a.y = 0.f; c.y = 0.f; }
      float2 cc = fft::cconj(c);
      float2 E = fft::cadd(a, cc);
      float2 O = fft::cmul(fft::csub(a, cc), fft::cconj(tw2[k]));
      buf[e] = make_float2(E.x - O.y, E.y + O.x);
    }
    __syncthreads();
    if constexpr (M > 0)
      fft::fft_lines_ct<M, 1, kMaxE, false>(buf, nrows, M, 1, tw2, 2 * M, tid, kThreads);
    else
      fft::fft_lines<1, kMaxE, false>(buf, pm, nrows, m, 1, tw2, n2, tid, kThreads);
    const float* outv = reinterpret_cast<const float*>(buf);
#pragma unroll
    for (int c = 0; c < kMaxV; ++c) {
      int v = tid + c * kThreads;
      if (v < nout) {
        float s = outv[v] * den[c];
        if (s > best[c]) {
          best[c] = s;
          arg[c] = first_index + b;
        }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int c = 0; c < kMaxV; ++c) {
    int v = tid + c * kThreads;
    if (v < nout && arg[c] >= 0) {
      int64_t g = vox0 + v;
      if (best[c] > state_max[g]) {
        state_max[g] = best[c];
        state_rot[g] = arg[c];
      }
    }
  }
}

// K4'' (FLC): c2r of the numerator and both statistics rows, then
// norm_scores (tme/backends/npfftw_backend.py:537-587) in double precision with the
// rotation's own n_obs = sum(rotated mask), and the strict-> update.
template <int M, typename RT = float2>
__device__ __forceinline__ void c2r_rows(const RT* raw, float2* buf, const float2* tw2, int nrows,
                                         int n2, int hp, const LinePlan& pm, int tid) {
  const int m = n2 / 2;
  for (int e = tid; e < nrows * m; e += kThreads) {
    int r = e / m, k = e % m;
    const RT* xr = raw + (int64_t)r * hp;
    float2 a = Store<RT>::load(xr + k), c = Store<RT>::load(xr + (m - k));
    if (k == 0) { a.y = 0.f; c.y = 0.f; }
    float2 cc = fft::cconj(c);
    float2 E = fft::cadd(a, cc);
    float2 O = fft::cmul(fft::csub(a, cc), fft::cconj(tw2[k]));
    buf[e] = make_float2(E.x - O.y, E.y + O.x);
  }
  __syncthreads();
  if constexpr (M > 0)
    fft::fft_lines_ct<M, 1, kMaxE, false>(buf, nrows, M, 1, tw2, 2 * M, tid, kThreads);
  else
    fft::fft_lines<1, kMaxE, false>(buf, pm, nrows, m, 1, tw2, n2, tid, kThreads);
}

// The FLC z pass transforms, for every rotation, the local mean (Hm), the local mean
// square (Hm2) and the numerator (H) of a block of R rows as one batch of 3 R lines (one
// set of barriers per rotation). The next rotation's rows are copied (cp.async, 16-byte
// pieces of three contiguous ranges) into the second of two raw buffer sets while the
// current rotation is transformed.
template <typename HT, int M = 0>
__global__ void __launch_bounds__(kThreads, 1)
zpass_flc_kernel(const HT* __restrict__ Ht, const float2* __restrict__ Hm,
                 const float2* __restrict__ Hm2, int B, int64_t rows, int n2, int hp, int R,
                 LinePlan pm, const float2* __restrict__ tw2_g, float scale_t, float scale_m,
                 const double* __restrict__ stats, double eps, int32_t first_index,
                 float* __restrict__ state_max, int32_t* __restrict__ state_rot, int64_t S,
                 const int32_t* __restrict__ first_dev) {
  if (first_dev) first_index = *first_dev;
  extern __shared__ float4 smem_raw[];
  const int m = n2 / 2;
  float2* tw2 = reinterpret_cast<float2*>(smem_raw);
  // raw set q, part k (0 Hm, 1 Hm2, 2 H): R rows of hp values (float2 room for each)
  float2* raw0 = tw2 + (n2 + 1) / 2 * 2;  // 16-byte aligned
  const int64_t part = (int64_t)R * hp;
  float2* buf = raw0 + 6 * part;
  const int tid = threadIdx.x;
  const int64_t row0 = (int64_t)blockIdx.x * R;
  const int nrows = (int)min((int64_t)R, rows - row0);
  for (int i = tid; i < n2; i += kThreads) tw2[i] = tw2_g[i];
  const int nout = nrows * n2;
  const int64_t vox0 = row0 * n2;
  const int set = R * n2;  // floats between the three parts' outputs in buf
  float best[kMaxV];
  int32_t arg[kMaxV];
#pragma unroll
  for (int c = 0; c < kMaxV; ++c) { best[c] = -INFINITY; arg[c] = -1; }
  const float* outv = reinterpret_cast<const float*>(buf);
  auto issue = [&](int b) {
    if (b < B) {
      const uint32_t dst0 = (uint32_t)__cvta_generic_to_shared(raw0 + (b & 1) * 3 * part);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        const char* src = k == 0   ? reinterpret_cast<const char*>(Hm + (int64_t)b * S + row0 * hp)
                          : k == 1 ? reinterpret_cast<const char*>(Hm2 + (int64_t)b * S + row0 * hp)
                                   : reinterpret_cast<const char*>(Ht + (int64_t)b * S + row0 * hp);
        const int nbytes = nrows * hp * (k == 2 ? (int)sizeof(HT) : (int)sizeof(float2));
        const uint32_t dst = dst0 + (uint32_t)(k * part * (int64_t)sizeof(float2));
        for (int o = tid * 16; o < nbytes; o += kThreads * 16)
          tc::cp_async16(dst + (uint32_t)o, src + o, 16u);
      }
    }
    cp_async_commit();
  };
  // line l = k R + r of buf: the even/odd-combined half spectrum of part k, row r
  auto build = [&](const float2* src_f, const HT* src_h, int k) {
    for (int e = tid; e < nrows * m; e += kThreads) {
      const int r = e / m, j = e - r * m;
      float2 a, c;
      if (k == 2) {
        const HT* xr = src_h + (int64_t)r * hp;
        a = Store<HT>::load(xr + j);
        c = Store<HT>::load(xr + (m - j));
      } else {
        const float2* xr = src_f + (int64_t)r * hp;
        a = xr[j];
        c = xr[m - j];
      }
      if (j == 0) { a.y = 0.f; c.y = 0.f; }
      const float2 cc = fft::cconj(c);
      const float2 E = fft::cadd(a, cc);
      const float2 O = fft::cmul(fft::csub(a, cc), fft::cconj(tw2[j]));
      buf[(int64_t)(k * R + r) * m + j] = make_float2(E.x - O.y, E.y + O.x);
    }
  };
  issue(0);
  for (int b = 0; b < B; ++b) {
    // the other buffer set was last read by rotation b - 1, which ended with a barrier
    issue(b + 1);
    cp_async_wait<1>();
    __syncthreads();  // rotation b's rows landed for every thread
    const float2* rs = raw0 + (b & 1) * 3 * part;
    build(rs, nullptr, 0);
    build(rs + part, nullptr, 1);
    build(nullptr, reinterpret_cast<const HT*>(rs + 2 * part), 2);
    __syncthreads();
    if constexpr (M > 0)
      fft::fft_lines_ct<M, 1, kMaxE, false>(buf, 3 * R, M, 1, tw2, 2 * M, tid, kThreads);
    else
      fft::fft_lines<1, kMaxE, false>(buf, pm, 3 * R, m, 1, tw2, n2, tid, kThreads);
    const double nobs = stats[b * 4 + 2];
#pragma unroll
    for (int c = 0; c < kMaxV; ++c) {
      const int v = tid + c * kThreads;
      if (v < nout) {
        const double e1 = (double)outv[v] * (double)scale_m / nobs;
        const double e2 = (double)outv[set + v] * (double)scale_m / nobs;
        const double var = e2 - e1 * e1;
        double sd = sqrt(var > 0 ? var : 0.0);
        if (sd < eps) sd = 1.0;
        const float sc = (float)((double)outv[2 * set + v] * (double)scale_t / (sd * nobs));
        if (sc > best[c]) { best[c] = sc; arg[c] = first_index + b; }
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int c = 0; c < kMaxV; ++c) {
    int v = tid + c * kThreads;
    if (v < nout && arg[c] >= 0) {
      int64_t g = vox0 + v;
      if (best[c] > state_max[g]) { state_max[g] = best[c]; state_rot[g] = arg[c]; }
    }
  }
}

// K4' (four-step): c2r along axis 2 for m = n2/2 = M1*M2 (M2 a multiple of M1).
// Thread (row, j) of a row's M1 threads builds Z[k] = E + iO for k = j + M1*k2 straight
// from global memory (the half-length c2r pre-twiddle), runs an inverse DFT of size M2
// over k2 in registers, applies exp(+2 pi i n2 j / m), exchanges through padded shared
// memory, and runs C = M2/M1 inverse DFTs of size M1, ending with the outputs
// z[n2 + M2*n1] = x[2(n2 + M2 n1)] + i x[2(n2 + M2 n1) + 1]. Each thread keeps the
// running max/argmax of its 2*M2 voxels in registers; the voxel pairs of a row's
// threads are contiguous, so the state merge is coalesced.
template <typename HT, int M1, int M2>
__global__ void __launch_bounds__(M1 * (256 / M1), 2)
zpass4_kernel(const HT* __restrict__ H, int B, int64_t rows, int hp,
              const float2* __restrict__ tw2_g, float scale, const float* __restrict__ inv_den,
              int32_t first_index, float* __restrict__ state_max,
              int32_t* __restrict__ state_rot, int64_t S, const int32_t* __restrict__ first_dev) {
  if (first_dev) first_index = *first_dev;
  constexpr int M = M1 * M2;
  constexpr int N2 = 2 * M;
  constexpr int C = M2 / M1;
  constexpr int RW = 256 / M1;
  constexpr int NT = M1 * RW;
  constexpr int PITCH = M2 * (M1 + 1);
  constexpr int V = 2 * M2;  // voxels per thread
  extern __shared__ float4 smem_raw[];
  float2* tw = reinterpret_cast<float2*>(smem_raw);
  float2* sx = tw + N2;
  HT* stage = reinterpret_cast<HT*>(sx + RW * PITCH);  // 2 x RW*hp staged rows
  const int tid = threadIdx.x;
  const int rho = tid / M1, j = tid % M1;
  for (int i = tid; i < N2; i += NT) tw[i] = tw2_g[i];
  const int64_t row0 = (int64_t)blockIdx.x * RW;
  const int nrows = (int)min((int64_t)RW, rows - row0);
  const int64_t row = row0 + rho;
  const bool active = rho < RW && rho < nrows;
  const int nel = nrows * hp;
  // rows of this CTA are contiguous in every rotation's H: stage them with cp.async,
  // one rotation ahead of the transform
  auto stage_copy = [&](int bb) {
    const HT* src = H + (int64_t)bb * S + row0 * hp;
    HT* dst = stage + (bb & 1) * RW * hp;
    for (int e = tid; e < nel; e += NT) cp_async<sizeof(HT)>(dst + e, src + e);
    cp_async_commit();
  };
  float best[V];
  int32_t arg[V];
#pragma unroll
  for (int v = 0; v < V; ++v) { best[v] = -INFINITY; arg[v] = -1; }
  // voxel of output slot (c, n1, part): 2*(n2 + M2*n1) + part with n2 = j + M1*c
  const int64_t vrow = row * N2;
  float2* srow = sx + rho * PITCH;
  if (B > 0) stage_copy(0);
  for (int b = 0; b < B; ++b) {
    if (b + 1 < B) {
      stage_copy(b + 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    float2 a[M2];
    if (active) {
      const HT* x = stage + (b & 1) * RW * hp + rho * hp;
#pragma unroll
      for (int k2 = 0; k2 < M2; ++k2) {
        const int k = j + M1 * k2;
        float2 xa = Store<HT>::load(x + k), xc = Store<HT>::load(x + (M - k));
        if (k == 0) { xa.y = 0.f; xc.y = 0.f; }
        const float2 cc = fft::cconj(xc);
        const float2 E = fft::cadd(xa, cc);
        const float2 O = fft::cmul(fft::csub(xa, cc), fft::cconj(tw[k]));
        a[k2] = make_float2(E.x - O.y, E.y + O.x);
      }
      fft::dft_small<M2, 1>(a);
#pragma unroll
      for (int n2 = 1; n2 < M2; ++n2) a[n2] = fft::cmul(a[n2], fft::cconj(tw[(2 * n2 * j) % N2]));
#pragma unroll
      for (int n2 = 0; n2 < M2; ++n2) srow[n2 * (M1 + 1) + j] = a[n2];
    }
    __syncthreads();
    if (active) {
#pragma unroll
      for (int c = 0; c < C; ++c) {
        const int n2 = j + M1 * c;
        float2 z[M1];
#pragma unroll
        for (int k1 = 0; k1 < M1; ++k1) z[k1] = srow[n2 * (M1 + 1) + k1];
        fft::dft_small<M1, 1>(z);
#pragma unroll
        for (int n1 = 0; n1 < M1; ++n1) {
          const int64_t vox = vrow + 2 * (n2 + M2 * n1);
          const float d0 = inv_den ? __ldg(inv_den + vox) : 1.f;
          const float d1 = inv_den ? __ldg(inv_den + vox + 1) : 1.f;
          const float s0 = z[n1].x * scale * d0, s1 = z[n1].y * scale * d1;
          const int slot = (c * M1 + n1) * 2;
          if (s0 > best[slot]) { best[slot] = s0; arg[slot] = first_index + b; }
          if (s1 > best[slot + 1]) { best[slot + 1] = s1; arg[slot + 1] = first_index + b; }
        }
      }
    }
    __syncthreads();
  }
  if (!active) return;
#pragma unroll
  for (int c = 0; c < C; ++c)
#pragma unroll
    for (int n1 = 0; n1 < M1; ++n1)
#pragma unroll
      for (int part = 0; part < 2; ++part) {
        const int slot = (c * M1 + n1) * 2 + part;
        const int64_t g = vrow + 2 * (j + M1 * c + M2 * n1) + part;
        if (arg[slot] >= 0 && best[slot] > state_max[g]) {
          state_max[g] = best[slot];
          state_rot[g] = arg[slot];
        }
      }
}

template <int M1, int M2, typename HT = float2>
size_t zpass4_smem(int hp) {
  // twiddles + exchange + two staged row blocks of pitch hp (>= M1*M2 + 1)
  return sizeof(float2) * (2 * M1 * M2 + (256 / M1) * M2 * (M1 + 1)) +
         2 * sizeof(HT) * (256 / M1) * (size_t)hp;
}

// ------------------------------------------------------------------ helpers
__global__ void sum_double_kernel(const float* __restrict__ x, int64_t n, double* __restrict__ out) {
  __shared__ double sh[32];
  double s = 0.0;
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    s += (double)x[i];
  for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
  int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) sh[warp] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += sh[w];
    out[blockIdx.x] = t;
  }
}

__global__ void center_kernel(const float* __restrict__ x, const double* __restrict__ partial,
                              int nparts, int64_t n, float* __restrict__ out_c,
                              double* __restrict__ out_d, double* __restrict__ out_d2) {
  __shared__ double mean;
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int i = 0; i < nparts; ++i) s += partial[i];
    mean = s / (double)n;
  }
  __syncthreads();
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double v = (double)x[i] - mean;
    if (out_c) out_c[i] = (float)v;
    if (out_d) out_d[i] = v;
    if (out_d2) out_d2[i] = v * v;
  }
}

__global__ void square_kernel(const float* __restrict__ x, float* __restrict__ y, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    float v = x[i];
    y[i] = v * v;
  }
}

__global__ void zmul_kernel(const double2* __restrict__ a, const double2* __restrict__ b,
                            double2* __restrict__ out, int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double2 x = a[i], y = b[i];
    out[i] = make_double2(x.x * y.x - x.y * y.y, x.x * y.y + x.y * y.x);
  }
}

__global__ void pad_double_kernel(const float* __restrict__ src, int t0, int t1, int t2,
                                  double* __restrict__ dst, int n1, int n2) {
  const int64_t n = (int64_t)t0 * t1 * t2;
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n;
       v += (int64_t)gridDim.x * blockDim.x) {
    int i2 = (int)(v % t2);
    int64_t r = v / t2;
    int i1 = (int)(r % t1);
    int i0 = (int)(r / t1);
    dst[((int64_t)i0 * n1 + i1) * n2 + i2] = (double)src[v];
  }
}

// inverse denominator 1 / (n_obs * sd) from unnormalised double inverse transforms
__global__ void inv_den_kernel(const double* __restrict__ cc1, const double* __restrict__ cc2,
                               double invN, double n_obs, double eps, float* __restrict__ out,
                               int64_t n) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double e = cc1[i] * invN / n_obs;
    double e2 = cc2[i] * invN / n_obs;
    double var = e2 - e * e;
    double sd = sqrt(var > 0 ? var : 0.0);
    if (sd < eps) sd = 1.0;
    out[i] = (float)(1.0 / (sd * n_obs));
  }
}

// The dynamic shared-memory limit is a property of each kernel function, shared by every
// plan, so it is raised once to the device's opt-in maximum (launches still request only
// their own tile size).
static int smem_optin_max() {
  static int v = -1;
  if (v < 0) {
    int dev = 0, val = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&val, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    v = val > 0 ? val : 48 * 1024;
  }
  return v;
}

static unsigned grid_for(int64_t n, int threads = 256, int64_t cap = 148 * 16) {
  int64_t b = ceil_div(n, threads);
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return (unsigned)b;
}

// ------------------------------------------------------------------ plan
struct Scan {
  tm_scan_desc d{};
  int n0 = 0, n1 = 0, n2 = 0, h2 = 0, t0 = 0, t1 = 0, t2 = 0, th2 = 0;
  // row pitch of the fused path's intermediate spectra H (and Hm, Hm2): h2 rounded up
  // to 8 elements so rows start on 32-byte sector boundaries
  int hp = 0;
  int64_t SH = 0;
  int64_t N = 0, S = 0, T = 0, TS = 0;
  bool fused = false, half = false;
  int B = 1;
  double mask_sum = 0.0, target_mean = 0.0;
  bool target_ready = false, template_ready = false;
  // persistent buffers
  void* base = nullptr;
  size_t bytes = 0;
  float2* ft_target = nullptr;
  float2* ft_target2 = nullptr;
  float* inv_den = nullptr;
  float* tmpl = nullptr;
  float* mask = nullptr;
  float* tfilter = nullptr;
  float* mat = nullptr;  // B x 16 matrices for the current group (device copy)
  // interpolation order of the template rotation (1 trilinear, 3 cubic B-spline); for
  // order 3 the template's spline coefficients and the mask in double
  int order = 1;
  double* coef = nullptr;
  double* mcoef = nullptr;
  // tensor-core x pass (CC / FLCSphericalMask): per-column correlation kernels of the
  // target, the launch configuration and a device error flag for its bounded waits
  bool xtc_avail = false, xtc = false;
  XcorrTcConfig xcfg{};
  float2* ctarget = nullptr;
  int* tc_err = nullptr;
  // tensor-core z pass (CC / FLCSphericalMask, half-precision H): c2r operator table
  bool ztc_avail = false, ztc = false;
  ZpassTcConfig zcfg{};
  uint16_t* ztable = nullptr;
  // tensor-core y pass (CC / FLCSphericalMask, half-precision H, n1 in {256, 512}): the
  // two DFT operators
  bool ytc_avail = false, ytc = false;
  bool ys1 = false;  // radix-16 stage on the tensor cores too (tm_scan_set_ypass mode 3)
  bool yinplace = false;  // tensor-core y pass in place on row-major H (mode 4)
  // y pass output (row-major) when the x pass writes H x'-inner; allocated where that
  // form is possible
  void* H2 = nullptr;
  YpassTcConfig ycfg{};
  uint16_t* ytable = nullptr;
  // polls of every data wait of the tensor-core kernels before they give up
  uint32_t wait_iters = tc_wait_iters_default();
  // per-group scratch
  float* rot_t = nullptr;
  float* rot_m = nullptr;
  double* stats_ws = nullptr;
  float2* tspec = nullptr;   // template-shape spectra (filter)
  float* arr = nullptr;      // plain: fast real buffers
  float* arr_m = nullptr;
  float* cc_m = nullptr;
  float* cc_m2 = nullptr;
  float2* spec = nullptr;
  float2* spec_m = nullptr;
  float2* G = nullptr;
  void* H = nullptr;
  float2* Gm = nullptr;   // FLC: rotated-mask rows
  float2* Hm = nullptr;   // FLC: CC(f, m) spectra (complex64)
  float2* Hm2 = nullptr;  // FLC: CC(f^2, m) spectra (complex64)
  float2* tw0 = nullptr;
  float2* tw1 = nullptr;
  float2* tw2 = nullptr;
  LinePlan p0{}, p1{}, pm{};
  bool reg0 = false, reg1 = false;  // register-resident column kernels for n0 / n1
  int W1 = 1, W2 = 1, W3 = 1, R4 = 1;
  int R4f = 1;  // rows per block of the FLC z pass (three parts per row)
  size_t smem4f = 0;
  size_t smem1 = 0, smem2 = 0, smem3 = 0, smem4 = 0;
  cufftHandle fwd = 0, inv = 0, tfwd = 0, tinv = 0;
  bool have_fwd = false, have_tfwd = false;
  // CUDA-graph replay of a full launch group (see scan_set_graph)
  bool use_graph = false;
  cudaGraphExec_t gexec = nullptr;
  cudaStream_t gstream = nullptr;
  cudaEvent_t gev_in = nullptr, gev_out = nullptr;
  float* gkey_max = nullptr;
  int32_t* gkey_rot = nullptr;
  int32_t* first_dev = nullptr;     // group's first rotation index, read by the z pass
  int32_t* graph_first = nullptr;   // == first_dev while capturing/replaying, else null
  // optional per-stage timing with CUDA events on the launching stream
  bool timing = false;
  double stage_ms[TM_NUM_STAGES] = {0};
  int64_t stage_launches[TM_NUM_STAGES] = {0};
  cudaEvent_t ev[TM_NUM_STAGES + 1] = {};
  bool have_events = false;
};

// The y pass hands H to the even/odd tensor-core z pass as 32-byte segments
// [Re x 8 | Im x 8] per row and 8 consecutive k2, which its loaders copy straight into
// the operand; the FFT z passes read interleaved complex values. (The generic
// shared-memory y pass for lengths without a register kernel writes interleaved values,
// so it is paired with them only.)
static bool seg_layout(const Scan* s) {
  return s->half && s->ztc && s->zcfg.eo && (s->ytc || s->reg1);
}

// Whether the warp-specialised tensor-core x pass runs every launch group: it can then read
// the template spectra G as FP16 and store H rows as segments in the y pass's stage-1
// order.
static bool x_writes_stage1(const Scan* s) {
  return s->half && s->xtc && s->xcfg.ws && s->B <= s->xcfg.ws_NB && s->hp % 8 == 0 &&
         s->d.score != TM_SCORE_FLC;
}
// The tensor-core y pass runs its radix-16 stage on the tensor cores too (opt-in: measured
// slower than the radix-16 stage on the CUDA cores).
static bool y_stage1_tc(const Scan* s) { return s->ytc && s->ys1 && x_writes_stage1(s); }
// Whether the warp-specialised x pass writes H x'-inner, [b][k1][k2 / 8][x'][8], and the
// tensor-core y pass reads it from there and writes row-major rows into H2 for the z pass.
// A warp of the x pass's epilogue then stores, per rotation, 32 consecutive x' rows of one
// 8-column segment as 1 KB of whole cache lines instead of 32 sectors one plane apart.
static bool x_inner(const Scan* s) {
  return s->H2 && s->ytc && !s->yinplace && !y_stage1_tc(s) && x_writes_stage1(s);
}

// Stage timing: record an event before a stage and accumulate after it.
struct StageTimer {
  Scan* s;
  cudaStream_t st;
  StageTimer(Scan* s_, cudaStream_t st_) : s(s_), st(st_) {}
  void begin() { if (s->timing) cudaEventRecord(s->ev[0], st); }
  void end(int stage) {
    if (!s->timing) return;
    cudaEventRecord(s->ev[1], st);
    cudaEventSynchronize(s->ev[1]);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, s->ev[0], s->ev[1]);
    s->stage_ms[stage] += ms;
    s->stage_launches[stage] += 1;
  }
};

// ---- z pass dispatch: compile-time half-lengths for the common sizes
#define TM_DISPATCH_M(m, CALL)                                   \
  switch (m) {                                                   \
    case 32: { constexpr int MM = 32; CALL; } break;             \
    case 50: { constexpr int MM = 50; CALL; } break;             \
    case 64: { constexpr int MM = 64; CALL; } break;             \
    case 80: { constexpr int MM = 80; CALL; } break;             \
    case 100: { constexpr int MM = 100; CALL; } break;           \
    case 128: { constexpr int MM = 128; CALL; } break;           \
    case 160: { constexpr int MM = 160; CALL; } break;           \
    default: { constexpr int MM = 0; CALL; } break;              \
  }

template <typename HT>
static void launch_zpass_flc(Scan* s, HT* H, int nb, int64_t rows, float out_scale,
                             int32_t first, float* state_max, int32_t* state_rot,
                             cudaStream_t st) {
  const double* stats = s->stats_ws + (int64_t)nb * kStatChunks * 3;
  dim3 g4f(ceil_div(rows, s->R4f));
  TM_DISPATCH_M(s->n2 / 2, (zpass_flc_kernel<HT, MM><<<g4f, kThreads, s->smem4f, st>>>(
                               H, s->Hm, s->Hm2, nb, rows, s->n2, s->hp, s->R4f, s->pm, s->tw2,
                               out_scale, out_scale, stats, 1.1920928955078125e-07, first,
                               state_max, state_rot, s->SH, s->graph_first)));
}

static void set_zpass_attrs(int m, int smem) {
  (void)smem;
  TM_DISPATCH_M(m, (cudaFuncSetAttribute(zpass_flc_kernel<float2, MM>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin_max()),
                    cudaFuncSetAttribute(zpass_flc_kernel<__half2, MM>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin_max())));
  TM_DISPATCH_M(m, (cudaFuncSetAttribute(zpass_kernel<float2, MM>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin_max()),
                    cudaFuncSetAttribute(zpass_kernel<__half2, MM>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin_max())));
}

#define TM_DISPATCH_4STEP(m, CALL)                                  \
  switch (m) {                                                      \
    case 32: { constexpr int A1 = 4, A2 = 8; CALL; } break;         \
    case 50: { constexpr int A1 = 5, A2 = 10; CALL; } break;        \
    case 64: { constexpr int A1 = 8, A2 = 8; CALL; } break;         \
    case 80: { constexpr int A1 = 4, A2 = 20; CALL; } break;        \
    case 100: { constexpr int A1 = 10, A2 = 10; CALL; } break;      \
    case 128: { constexpr int A1 = 8, A2 = 16; CALL; } break;       \
    case 200: { constexpr int A1 = 10, A2 = 20; CALL; } break;      \
    case 256: { constexpr int A1 = 16, A2 = 16; CALL; } break;      \
    default: break;                                                 \
  }

static bool zpass4_supported(int m) {
  return m == 32 || m == 50 || m == 64 || m == 80 || m == 100 || m == 128 || m == 200 ||
         m == 256;
}

template <typename HT>
static void launch_zpass4(Scan* s, HT* H, int nb, int64_t rows, float out_scale, int32_t first,
                          float* state_max, int32_t* state_rot, cudaStream_t st) {
  TM_DISPATCH_4STEP(s->n2 / 2, ({
    constexpr int RW = 256 / A1;
    dim3 g(ceil_div(rows, RW));
    zpass4_kernel<HT, A1, A2><<<g, A1 * RW, zpass4_smem<A1, A2, HT>(s->hp), st>>>(
        H, nb, rows, s->hp, s->tw2, out_scale, s->inv_den, first, state_max, state_rot, s->SH,
        s->graph_first);
  }));
}

static void set_zpass4_attrs(int m) {
  TM_DISPATCH_4STEP(m, ({
    cudaFuncSetAttribute(zpass4_kernel<float2, A1, A2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin_max());
    cudaFuncSetAttribute(zpass4_kernel<__half2, A1, A2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin_max());
  }));
}

template <typename HT>
static void launch_zpass(Scan* s, dim3 g4, HT* H, int nb, int64_t rows, float out_scale,
                         int32_t first, float* state_max, int32_t* state_rot, cudaStream_t st) {
  if (s->ztc && std::is_same<HT, __half2>::value) {
    zpass_tc_run(s->zcfg, H, nb, rows, s->n2, s->h2, s->hp, s->ztable, out_scale, s->inv_den,
                 first, state_max, state_rot, s->SH, s->graph_first, s->tc_err, st,
                 s->wait_iters, seg_layout(s));
    return;
  }
  if (zpass4_supported(s->n2 / 2) && !getenv("PYTME_B200_GENERIC_FFT")) {
    launch_zpass4<HT>(s, H, nb, rows, out_scale, first, state_max, state_rot, st);
    return;
  }
  TM_DISPATCH_M(s->n2 / 2, (zpass_kernel<HT, MM><<<g4, kThreads, s->smem4, st>>>(
                               H, nb, rows, s->n2, s->hp, s->R4, s->pm, s->tw2, out_scale,
                               s->inv_den, first, state_max, state_rot, s->SH, s->graph_first)));
}

// ---- launch helpers for the register-resident kernels
template <int N>
static void set_reg_attrs(size_t zy_smem) {
  constexpr int W = reg_lines<N>();
  const int sm = (int)reg_smem_bytes<N>(0, 0, 0, false);
  cudaFuncSetAttribute(xpass_reg_kernel<N, W, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin_max());
  cudaFuncSetAttribute(xpass_reg_kernel<N, W, __half2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin_max());
  cudaFuncSetAttribute(ypass_reg_kernel<N, W, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin_max());
  cudaFuncSetAttribute(ypass_reg_kernel<N, W, __half2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin_max());
  cudaFuncSetAttribute(tmpl_zy_reg_kernel<N, W>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin_max());
  cudaFuncSetAttribute(tmpl_zy_reg_kernel<N, W, __half2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin_max());
  cudaFuncSetAttribute(xpass_flc_reg_kernel<N, W, float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin_max());
  cudaFuncSetAttribute(xpass_flc_reg_kernel<N, W, __half2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin_max());
}

static void set_reg_attrs_n(int n, size_t zy_smem) {
  switch (n) {
    case 64: set_reg_attrs<64>(zy_smem); break;
    case 128: set_reg_attrs<128>(zy_smem); break;
    case 256: set_reg_attrs<256>(zy_smem); break;
    case 512: set_reg_attrs<512>(zy_smem); break;
    case 1024: set_reg_attrs<1024>(zy_smem); break;
    default: break;
  }
}

template <int N>
static void launch_tmpl_reg(Scan* s, int nb, cudaStream_t st, const float* in = nullptr,
                            float2* out = nullptr, bool half_g = false) {
  constexpr int W = reg_lines<N>();
  dim3 g(ceil_div(s->h2, W), s->t0, nb);
  size_t smem = reg_smem_bytes<N>(s->n2, s->t1, s->t2, true);
  if (half_g)
    tmpl_zy_reg_kernel<N, W, __half2><<<g, N / 8 * W, smem, st>>>(
        in ? in : s->rot_t, s->t0, s->t1, s->t2, s->n2, s->h2, s->tw1, s->tw2,
        reinterpret_cast<__half2*>(out ? out : s->G));
  else
    tmpl_zy_reg_kernel<N, W><<<g, N / 8 * W, smem, st>>>(in ? in : s->rot_t, s->t0, s->t1, s->t2,
                                                         s->n2, s->h2, s->tw1, s->tw2,
                                                         out ? out : s->G);
}

template <int N, typename HT>
static void launch_xpass_flc_reg(Scan* s, int nb, float hs, HT* H, cudaStream_t st) {
  constexpr int W = reg_lines<N>();
  dim3 g(ceil_div(s->h2, W), s->n1);
  xpass_flc_reg_kernel<N, W, HT><<<g, N / 8 * W, reg_smem_bytes<N>(0, 0, 0, false), st>>>(
      s->G, s->Gm, s->ft_target, s->ft_target2, nb, s->t0, s->n1, s->h2, s->tw0, hs, H, s->Hm,
      s->Hm2, s->hp);
}

template <int N, typename HT>
static void launch_xpass_reg(Scan* s, int nb, float hs, HT* H, cudaStream_t st) {
  constexpr int W = reg_lines<N>();
  dim3 g(ceil_div(s->h2, W), s->n1);
  xpass_reg_kernel<N, W, HT><<<g, N / 8 * W, reg_smem_bytes<N>(0, 0, 0, false), st>>>(
      s->G, s->ft_target, nb, s->t0, s->n1, s->h2, s->tw0, hs, H, s->hp);
}

template <int N, typename HT>
static void launch_ypass_reg(Scan* s, int nb, HT* H, cudaStream_t st, bool seg = false) {
  constexpr int W = reg_lines<N>();
  dim3 g(ceil_div(s->h2, W), ceil_div(s->n0, kYPlanes), nb);
  ypass_reg_kernel<N, W, HT><<<g, N / 8 * W, ypass_smem_bytes<N, HT>(), st>>>(
      H, s->n0, s->h2, s->tw1, s->hp, seg ? 1 : 0);
}

#define TM_DISPATCH_N(n, CALL)      \
  switch (n) {                      \
    case 64: { constexpr int NN = 64; CALL; } break;    \
    case 128: { constexpr int NN = 128; CALL; } break;  \
    case 256: { constexpr int NN = 256; CALL; } break;  \
    case 512: { constexpr int NN = 512; CALL; } break;  \
    case 1024: { constexpr int NN = 1024; CALL; } break; \
    default: break;                 \
  }

template <typename HT>
static int launch_template_x_y(Scan* s, int nb, float hs, HT* H, StageTimer& tmr,
                               cudaStream_t stream) {
  const bool flc = s->d.score == TM_SCORE_FLC;
  // the warp-specialised tensor-core x pass reads the template spectra G as FP16 (it
  // rounds them to FP16 for its MMAs anyway), so the template pass writes them so
  const bool half_g = s->reg1 && x_writes_stage1(s);
  tmr.begin();
  if (s->reg1) {
    TM_DISPATCH_N(s->n1, (launch_tmpl_reg<NN>(s, nb, stream, nullptr, nullptr, half_g)));
    if (flc) TM_DISPATCH_N(s->n1, (launch_tmpl_reg<NN>(s, nb, stream, s->rot_m, s->Gm)));
  } else {
    dim3 g1(ceil_div(s->h2, s->W1), s->t0, nb);
    tmpl_zy_kernel<<<g1, kThreads, s->smem1, stream>>>(s->rot_t, s->t0, s->t1, s->t2, s->n1,
                                                       s->n2, s->h2, s->W1, s->p1, s->tw1,
                                                       s->tw2, s->G);
  }
  TM_TRY(check_launch("template pass"));
  tmr.end(TM_STAGE_TEMPLATE);
  tmr.begin();
  if (flc) {
    TM_DISPATCH_N(s->n0, (launch_xpass_flc_reg<NN, HT>(s, nb, hs, H, stream)));
  } else if (s->xtc) {
    const bool s1 = y_stage1_tc(s);
    TM_TRY(xcorr_tc_run(s->xcfg, s->G, s->ctarget, nb, s->t0, s->n0, s->n1, s->h2, s->hp, hs,
                        H, std::is_same<HT, __half2>::value, s->tc_err, stream,
                        s->wait_iters, s1, s1 ? s->n1 / 16 : 0, half_g, x_inner(s)));
  } else if (s->reg0) {
    TM_DISPATCH_N(s->n0, (launch_xpass_reg<NN, HT>(s, nb, hs, H, stream)));
  } else {
    dim3 g2(ceil_div(s->h2, s->W2), s->n1);
    xpass_kernel<HT><<<g2, kThreads, s->smem2, stream>>>(s->G, s->ft_target, nb, s->t0, s->n0,
                                                        s->n1, s->h2, s->W2, s->p0, s->tw0, hs, H,
                                                        s->hp);
  }
  TM_TRY(check_launch("x pass"));
  tmr.end(TM_STAGE_XPASS);
  tmr.begin();
  if (s->ytc && std::is_same<HT, __half2>::value) {
    TM_TRY(ypass_tc_run(s->ycfg, H, nb, s->n0, s->hp, s->h2, s->ytable, s->wait_iters, s->tc_err,
                        stream, seg_layout(s), y_stage1_tc(s), x_inner(s) ? s->H2 : nullptr,
                        x_inner(s)));
  } else if (s->reg1) {
    TM_DISPATCH_N(s->n1, (launch_ypass_reg<NN, HT>(s, nb, H, stream, seg_layout(s))));
    if (flc) {
      TM_DISPATCH_N(s->n1, (launch_ypass_reg<NN, float2>(s, nb, s->Hm, stream)));
      TM_DISPATCH_N(s->n1, (launch_ypass_reg<NN, float2>(s, nb, s->Hm2, stream)));
    }
  } else {
    dim3 g3(ceil_div(s->h2, s->W3), s->n0, nb);
    ypass_kernel<HT><<<g3, kThreads, s->smem3, stream>>>(H, s->n0, s->n1, s->h2, s->W3, s->p1,
                                                        s->tw1, s->hp);
  }
  TM_TRY(check_launch("y pass"));
  tmr.end(TM_STAGE_YPASS);
  return TM_OK;
}

static size_t align_up(size_t x) { return (x + 255) & ~(size_t)255; }

static void destroy(Scan* s) {
  if (!s) return;
  if (s->gexec) cudaGraphExecDestroy(s->gexec);
  if (s->gstream) cudaStreamDestroy(s->gstream);
  if (s->gev_in) cudaEventDestroy(s->gev_in);
  if (s->gev_out) cudaEventDestroy(s->gev_out);
  if (s->have_events)
    for (auto& e : s->ev) cudaEventDestroy(e);
  if (s->have_fwd) { cufftDestroy(s->fwd); cufftDestroy(s->inv); }
  if (s->have_tfwd) { cufftDestroy(s->tfwd); cufftDestroy(s->tinv); }
  if (s->base) cudaFree(s->base);
  if (s->coef) cudaFree(s->coef);
  if (s->mcoef) cudaFree(s->mcoef);
  delete s;
}

int scan_destroy(Scan* s) {
  destroy(s);
  return TM_OK;
}

int scan_create(const tm_scan_desc* desc, Scan** out) {
  TM_REQUIRE(desc && out, "scan_create: null pointer");
  *out = nullptr;
  const tm_scan_desc& d = *desc;
  TM_REQUIRE(d.score == TM_SCORE_CC || d.score == TM_SCORE_FLC || d.score == TM_SCORE_FLCSM,
             "scan_create: unknown score %d", d.score);
  TM_REQUIRE(d.precision == TM_PREC_FP32 || d.precision == TM_PREC_MIXED,
             "scan_create: unknown precision %d", d.precision);
  for (int a = 0; a < 3; ++a) {
    TM_REQUIRE(d.fast_shape[a] > 0 && d.template_shape[a] > 0,
               "scan_create: shapes must be positive");
    TM_REQUIRE(d.template_shape[a] <= d.fast_shape[a],
               "scan_create: template axis %d (%d) exceeds the transform length (%d)", a,
               d.template_shape[a], d.fast_shape[a]);
  }
  TM_REQUIRE(d.batch >= 1 && d.batch <= 4096, "scan_create: batch must be in [1, 4096]");
  Scan* s = new Scan();
  s->d = d;
  s->n0 = d.fast_shape[0]; s->n1 = d.fast_shape[1]; s->n2 = d.fast_shape[2];
  s->h2 = s->n2 / 2 + 1;
  s->hp = (s->h2 + 7) / 8 * 8;
  s->t0 = d.template_shape[0]; s->t1 = d.template_shape[1]; s->t2 = d.template_shape[2];
  s->th2 = s->t2 / 2 + 1;
  s->N = (int64_t)s->n0 * s->n1 * s->n2;
  s->S = (int64_t)s->n0 * s->n1 * s->h2;
  s->T = (int64_t)s->t0 * s->t1 * s->t2;
  s->TS = (int64_t)s->t0 * s->t1 * s->th2;
  s->SH = (int64_t)s->n0 * s->n1 * s->hp;
  s->fused = !d.plain;
  s->half = d.precision == TM_PREC_MIXED;
  s->B = s->fused ? d.batch : 1;
  if (s->fused) {
    bool ok = line_supported(s->n0) && line_supported(s->n1) && (s->n2 % 2 == 0) &&
              line_supported(s->n2 / 2) && s->n0 <= kTile && s->n1 <= kTile &&
              s->n2 <= kThreads * kMaxV &&
              (d.score != TM_SCORE_FLC || (reg_supported(s->n0) && reg_supported(s->n1)));
    if (!ok) {
      set_error("scan_create: fused path does not support shape (%d,%d,%d) / score %d",
                s->n0, s->n1, s->n2, d.score);
      delete s;
      return TM_E_UNSUPPORTED;
    }
  } else {
    TM_REQUIRE(!s->half, "scan_create: the plain path is FP32 only");
  }

  // ---- memory layout
  const int B = s->B;
  size_t off = 0;
  auto take = [&](size_t nbytes) { size_t o = off; off = align_up(off + nbytes); return o; };
  size_t o_ft = take(sizeof(float2) * s->S);
  size_t o_ft2 = d.score == TM_SCORE_FLC ? take(sizeof(float2) * s->S) : 0;
  size_t o_den = d.score == TM_SCORE_FLCSM ? take(sizeof(float) * s->N) : 0;
  size_t o_tm = take(sizeof(float) * s->T);
  size_t o_mk = take(sizeof(float) * s->T);
  size_t o_tf = take(sizeof(float) * s->TS);
  size_t o_mat = take(sizeof(float) * 16 * B);
  size_t o_first = take(sizeof(int32_t) * 4);
  size_t o_rt = take(sizeof(float) * s->T * B);
  size_t o_rm = take(sizeof(float) * s->T * B);
  size_t o_st = take(stats_workspace_bytes(B));
  size_t o_ts = take(sizeof(float2) * s->TS * B);
  size_t o_arr = 0, o_arrm = 0, o_ccm = 0, o_ccm2 = 0, o_spec = 0, o_specm = 0, o_G = 0, o_H = 0;
  size_t o_tw0 = 0, o_tw1 = 0, o_tw2 = 0, o_Gm = 0, o_Hm = 0, o_Hm2 = 0;
  if (!s->fused) {
    o_arr = take(sizeof(float) * s->N);
    o_spec = take(sizeof(float2) * s->S);
    if (d.score == TM_SCORE_FLC) {
      o_arrm = take(sizeof(float) * s->N);
      o_ccm = take(sizeof(float) * s->N);
      o_ccm2 = take(sizeof(float) * s->N);
      o_specm = take(sizeof(float2) * s->S);
    }
  } else {
    o_G = take(sizeof(float2) * (size_t)B * s->t0 * s->n1 * s->h2);
    o_H = take((s->half ? sizeof(__half2) : sizeof(float2)) * (size_t)B * s->SH);
    if (d.score == TM_SCORE_FLC) {
      o_Gm = take(sizeof(float2) * (size_t)B * s->t0 * s->n1 * s->h2);
      o_Hm = take(sizeof(float2) * (size_t)B * s->SH);
      o_Hm2 = take(sizeof(float2) * (size_t)B * s->SH);
    }
    o_tw0 = take(sizeof(float2) * s->n0);
    o_tw1 = take(sizeof(float2) * s->n1);
    o_tw2 = take(sizeof(float2) * s->n2);
  }
  size_t o_ct = 0, o_err = 0, o_zt = 0, o_yt = 0;
  if (s->fused && d.score != TM_SCORE_FLC && s->half) {
    TM_TRY(zpass_tc_config(s->n2, s->h2, s->hp, B, &s->zcfg));
    s->ztc_avail = s->zcfg.ok;
    s->ztc = s->ztc_avail;
    if (s->ztc_avail) o_zt = take(zpass_tc_table_bytes(s->zcfg));
    TM_TRY(ypass_tc_config(s->n1, s->hp, &s->ycfg));
    s->ytc_avail = s->ycfg.ok;
    s->ytc = s->ytc_avail;
    if (s->ytc_avail) o_yt = take(ypass_tc_table_bytes(s->ycfg));
  }
  if (s->fused && d.score != TM_SCORE_FLC) {
    TM_TRY(xcorr_tc_config(s->n0, s->t0, B, &s->xcfg));
    s->xtc_avail = s->xcfg.ok || (s->half && s->xcfg.ws);
    // default: tensor cores for half-precision spectra (the FP16 Hankel kernels), FFTs
    // otherwise; tm_scan_set_xpass overrides
    s->xtc = s->xtc_avail && s->half && (s->xcfg.hk || s->xcfg.ws);
  }
  if (s->xtc_avail) o_ct = take(sizeof(float2) * s->S);
  // the y pass's row-major output where the x pass can write H x'-inner (see x_inner)
  size_t o_H2 = 0;
  const bool h2_buf = s->fused && s->half && d.score != TM_SCORE_FLC && s->ytc_avail &&
                      s->xtc_avail && s->xcfg.ws && B <= s->xcfg.ws_NB && s->hp % 8 == 0;
  if (h2_buf) o_H2 = take(sizeof(__half2) * (size_t)B * s->SH);
  if (s->xtc_avail || s->ztc_avail || s->ytc_avail) o_err = take(sizeof(int) * 4);
  s->bytes = off;
  const int64_t cap = device_memory_limit();
  if (cap > 0 && (int64_t)s->bytes > cap) {
    set_error("scan_create: the plan needs %zu bytes of device memory, above the limit of %lld "
              "bytes set by tm_set_device_memory_limit", s->bytes, (long long)cap);
    delete s;
    return TM_E_OOM;
  }
  cudaError_t e = cudaMalloc(&s->base, s->bytes);
  if (e != cudaSuccess) {
    set_error("scan_create: cudaMalloc of %zu bytes failed: %s", s->bytes, cudaGetErrorString(e));
    delete s;
    return TM_E_OOM;
  }
  char* b8 = static_cast<char*>(s->base);
  s->ft_target = reinterpret_cast<float2*>(b8 + o_ft);
  if (d.score == TM_SCORE_FLC) s->ft_target2 = reinterpret_cast<float2*>(b8 + o_ft2);
  if (d.score == TM_SCORE_FLCSM) s->inv_den = reinterpret_cast<float*>(b8 + o_den);
  s->tmpl = reinterpret_cast<float*>(b8 + o_tm);
  s->mask = reinterpret_cast<float*>(b8 + o_mk);
  s->tfilter = reinterpret_cast<float*>(b8 + o_tf);
  s->mat = reinterpret_cast<float*>(b8 + o_mat);
  s->first_dev = reinterpret_cast<int32_t*>(b8 + o_first);
  s->rot_t = reinterpret_cast<float*>(b8 + o_rt);
  s->rot_m = reinterpret_cast<float*>(b8 + o_rm);
  s->stats_ws = reinterpret_cast<double*>(b8 + o_st);
  s->tspec = reinterpret_cast<float2*>(b8 + o_ts);
  if (!s->fused) {
    s->arr = reinterpret_cast<float*>(b8 + o_arr);
    s->spec = reinterpret_cast<float2*>(b8 + o_spec);
    if (d.score == TM_SCORE_FLC) {
      s->arr_m = reinterpret_cast<float*>(b8 + o_arrm);
      s->cc_m = reinterpret_cast<float*>(b8 + o_ccm);
      s->cc_m2 = reinterpret_cast<float*>(b8 + o_ccm2);
      s->spec_m = reinterpret_cast<float2*>(b8 + o_specm);
    }
  } else {
    s->G = reinterpret_cast<float2*>(b8 + o_G);
    s->H = b8 + o_H;
    if (h2_buf) s->H2 = b8 + o_H2;
    if (d.score == TM_SCORE_FLC) {
      s->Gm = reinterpret_cast<float2*>(b8 + o_Gm);
      s->Hm = reinterpret_cast<float2*>(b8 + o_Hm);
      s->Hm2 = reinterpret_cast<float2*>(b8 + o_Hm2);
    }
    s->tw0 = reinterpret_cast<float2*>(b8 + o_tw0);
    if (s->xtc_avail) s->ctarget = reinterpret_cast<float2*>(b8 + o_ct);
    if (s->xtc_avail || s->ztc_avail || s->ytc_avail) {
      s->tc_err = reinterpret_cast<int*>(b8 + o_err);
      cudaMemset(s->tc_err, 0, sizeof(int));
    }
    if (s->ytc_avail) {
      s->ytable = reinterpret_cast<uint16_t*>(b8 + o_yt);
      int st = ypass_tc_prepare(s->ycfg, s->ytable, 0);
      if (st == TM_OK) st = cuda_status(cudaDeviceSynchronize(), "scan_create: y operators");
      if (st != TM_OK) { destroy(s); return st; }
    }
    if (s->ztc_avail) {
      s->ztable = reinterpret_cast<uint16_t*>(b8 + o_zt);
      int st = zpass_tc_prepare(s->zcfg, s->ztable, s->n2, s->h2, 0);
      if (st == TM_OK) st = cuda_status(cudaDeviceSynchronize(), "scan_create: z operator");
      if (st != TM_OK) { destroy(s); return st; }
    }
    s->tw1 = reinterpret_cast<float2*>(b8 + o_tw1);
    s->tw2 = reinterpret_cast<float2*>(b8 + o_tw2);
    auto t0v = twiddle_table(s->n0), t1v = twiddle_table(s->n1), t2v = twiddle_table(s->n2);
    cudaMemcpy(s->tw0, t0v.data(), sizeof(float2) * s->n0, cudaMemcpyHostToDevice);
    cudaMemcpy(s->tw1, t1v.data(), sizeof(float2) * s->n1, cudaMemcpyHostToDevice);
    e = cudaMemcpy(s->tw2, t2v.data(), sizeof(float2) * s->n2, cudaMemcpyHostToDevice);
    if (e != cudaSuccess) { int st = cuda_status(e, "scan_create: twiddles"); destroy(s); return st; }
    s->p0 = make_line_plan(s->n0);
    s->p1 = make_line_plan(s->n1);
    s->pm = make_line_plan(s->n2 / 2);
    s->W1 = std::max(1, std::min(s->h2, kTile / s->n1));
    s->W2 = std::max(1, std::min(s->h2, kTile / s->n0));
    s->W3 = s->W1;
    s->R4 = std::max(1, std::min(kTile / std::max(1, s->n2 / 2), (kThreads * kMaxV) / s->n2));
    s->R4f = std::max(1, std::min(kTile / std::max(1, 3 * (s->n2 / 2)),
                                  (kThreads * kMaxV) / s->n2));
    s->smem1 = sizeof(float2) * (s->n1 + s->n2 + (size_t)s->n1 * s->W1) + sizeof(float) * s->t1 * s->t2;
    s->smem2 = sizeof(float2) * (s->n0 + (size_t)s->n0 * s->W2);
    s->smem3 = sizeof(float2) * (s->n1 + (size_t)s->n1 * s->W3);
    // twiddles (padded to 16 bytes), two raw row buffers, the c2r buffer
    s->smem4 = sizeof(float2) * ((s->n2 + 1) / 2 * 2 + 2 * (size_t)s->R4 * s->hp +
                                 (size_t)s->R4 * (s->n2 / 2));
    // FLC z pass: twiddles, two raw sets of three parts, the c2r buffer of 3 R4f lines
    s->smem4f = sizeof(float2) * ((s->n2 + 1) / 2 * 2 + 6 * (size_t)s->R4f * s->hp +
                                  3 * (size_t)s->R4f * (s->n2 / 2));
    size_t mx = std::max(std::max(s->smem1, s->smem2), std::max(s->smem3, s->smem4));
    if (d.score == TM_SCORE_FLC) mx = std::max(mx, s->smem4f);
    if (mx > 200 * 1024) {
      set_error("scan_create: shared-memory tile of %zu bytes exceeds the limit", mx);
      destroy(s);
      return TM_E_UNSUPPORTED;
    }
    cudaFuncSetAttribute(tmpl_zy_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin_max());
    cudaFuncSetAttribute(xpass_kernel<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin_max());
    cudaFuncSetAttribute(xpass_kernel<__half2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin_max());
    cudaFuncSetAttribute(ypass_kernel<float2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin_max());
    cudaFuncSetAttribute(ypass_kernel<__half2>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin_max());
    set_zpass_attrs(s->n2 / 2, (int)s->smem4);
    set_zpass4_attrs(s->n2 / 2);
    s->reg0 = reg_supported(s->n0) && !getenv("PYTME_B200_GENERIC_FFT");
    s->reg1 = reg_supported(s->n1) && !getenv("PYTME_B200_GENERIC_FFT");
    size_t zy = 0;
    if (s->reg1) {
      TM_DISPATCH_N(s->n1, (zy = reg_smem_bytes<NN>(s->n2, s->t1, s->t2, true)));
      if (zy > 200 * 1024) s->reg1 = false;
    }
    if (s->reg0) set_reg_attrs_n(s->n0, 0);
    if (s->reg1) set_reg_attrs_n(s->n1, zy);
  }
  // ---- cuFFT plans: fast-shape r2c/c2r (setup and plain path), template-shape (filter)
  int r;
  r = cufftPlan3d(&s->fwd, s->n0, s->n1, s->n2, CUFFT_R2C);
  if (r == CUFFT_SUCCESS) r = cufftPlan3d(&s->inv, s->n0, s->n1, s->n2, CUFFT_C2R);
  if (r != CUFFT_SUCCESS) { int st = cufft_status((cufftResult)r, "scan_create: fast plans"); destroy(s); return st; }
  s->have_fwd = true;
  int ts[3] = {s->t0, s->t1, s->t2};
  r = cufftPlanMany(&s->tfwd, 3, ts, nullptr, 1, 0, nullptr, 1, 0, CUFFT_R2C, B);
  if (r == CUFFT_SUCCESS)
    r = cufftPlanMany(&s->tinv, 3, ts, nullptr, 1, 0, nullptr, 1, 0, CUFFT_C2R, B);
  if (r != CUFFT_SUCCESS) { int st = cufft_status((cufftResult)r, "scan_create: template plans"); destroy(s); return st; }
  s->have_tfwd = true;
  *out = s;
  return TM_OK;
}

int64_t scan_device_bytes(const Scan* s) { return (int64_t)s->bytes; }

// target: fast-shaped (top-left padded, already filtered) float32 device array.
int scan_set_target(Scan* s, const float* target, cudaStream_t stream) {
  TM_REQUIRE(s && target, "scan_set_target: null pointer");
  TM_TRY(cuda_status(cudaStreamSynchronize(stream), "scan_set_target: sync"));
  cufftSetStream(s->fwd, stream);
  cufftSetStream(s->inv, stream);
  const int64_t N = s->N, S = s->S;
  if (s->d.score == TM_SCORE_CC) {
    // CC correlates the raw target (cc_setup, tme/matching_scores.py:153-189)
    float* tmp = nullptr;
    TM_TRY(cuda_status(cudaMallocAsync((void**)&tmp, sizeof(float) * N, stream), "scan_set_target: alloc"));
    cudaMemcpyAsync(tmp, target, sizeof(float) * N, cudaMemcpyDeviceToDevice, stream);
    int r = cufftExecR2C(s->fwd, tmp, (cufftComplex*)s->ft_target);
    cudaFreeAsync(tmp, stream);
    TM_TRY(cufft_status((cufftResult)r, "scan_set_target: r2c"));
    if (s->xtc_avail)
      TM_TRY(xcorr_tc_prepare(s->ft_target, s->ctarget, s->n0, s->n1, s->h2, stream));
    s->target_ready = true;
    return check_launch("scan_set_target");
  }
  // mean in double; the normalised scores are invariant to a constant target offset
  // because the normalised template sums to zero, so the spectra are taken of the
  // centred target, which keeps E[x^2] - E[x]^2 well conditioned.
  const int nparts = 592;
  double* partial = nullptr;
  float* centred = nullptr;
  TM_TRY(cuda_status(cudaMallocAsync((void**)&partial, sizeof(double) * nparts, stream), "alloc"));
  TM_TRY(cuda_status(cudaMallocAsync((void**)&centred, sizeof(float) * N, stream), "alloc"));
  sum_double_kernel<<<nparts, 256, 0, stream>>>(target, N, partial);
  center_kernel<<<grid_for(N), 256, 0, stream>>>(target, partial, nparts, N, centred, nullptr, nullptr);
  TM_TRY(check_launch("scan_set_target: centre"));
  std::vector<double> hp(nparts);
  cudaMemcpyAsync(hp.data(), partial, sizeof(double) * nparts, cudaMemcpyDeviceToHost, stream);
  TM_TRY(cuda_status(cudaStreamSynchronize(stream), "scan_set_target: mean"));
  double tot = 0.0;
  for (double v : hp) tot += v;
  s->target_mean = tot / (double)N;
  int r;
  if (s->d.score == TM_SCORE_FLC) {
    // flc_setup (tme/matching_scores.py:357-387): spectra of f and f^2
    float* sq = nullptr;
    TM_TRY(cuda_status(cudaMallocAsync((void**)&sq, sizeof(float) * N, stream), "alloc"));
    square_kernel<<<grid_for(N), 256, 0, stream>>>(centred, sq, N);
    r = cufftExecR2C(s->fwd, centred, (cufftComplex*)s->ft_target);
    if (r == CUFFT_SUCCESS) r = cufftExecR2C(s->fwd, sq, (cufftComplex*)s->ft_target2);
    cudaFreeAsync(sq, stream);
  } else {
    // flcSphericalMask_setup (tme/matching_scores.py:390-450): the local-variance
    // denominator from CC(f^2, m) and CC(f, m), here in double precision.
    TM_REQUIRE(s->template_ready, "scan_set_target: FLCSphericalMask needs the template mask first");
    cufftHandle dfwd, dinv;
    r = cufftPlan3d(&dfwd, s->n0, s->n1, s->n2, CUFFT_D2Z);
    if (r != CUFFT_SUCCESS) { cudaFreeAsync(centred, stream); cudaFreeAsync(partial, stream); return cufft_status((cufftResult)r, "scan_set_target: D2Z plan"); }
    r = cufftPlan3d(&dinv, s->n0, s->n1, s->n2, CUFFT_Z2D);
    if (r != CUFFT_SUCCESS) { cufftDestroy(dfwd); cudaFreeAsync(centred, stream); cudaFreeAsync(partial, stream); return cufft_status((cufftResult)r, "scan_set_target: Z2D plan"); }
    cufftSetStream(dfwd, stream);
    cufftSetStream(dinv, stream);
    double *f = nullptr, *f2 = nullptr;
    double2 *Ff = nullptr, *Ff2 = nullptr, *Fm = nullptr;
    cudaError_t e = cudaMallocAsync((void**)&f, sizeof(double) * N, stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&f2, sizeof(double) * N, stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&Ff, sizeof(double2) * S, stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&Ff2, sizeof(double2) * S, stream);
    if (e == cudaSuccess) e = cudaMallocAsync((void**)&Fm, sizeof(double2) * S, stream);
    if (e != cudaSuccess) {
      cufftDestroy(dfwd); cufftDestroy(dinv);
      return cuda_status(e, "scan_set_target: FP64 buffers");
    }
    center_kernel<<<grid_for(N), 256, 0, stream>>>(target, partial, nparts, N, nullptr, f, f2);
    r = cufftExecD2Z(dfwd, f, Ff);
    if (r == CUFFT_SUCCESS) r = cufftExecD2Z(dfwd, f2, Ff2);
    // mask: top-left padded into f (reused)
    cudaMemsetAsync(f, 0, sizeof(double) * N, stream);
    pad_double_kernel<<<grid_for(s->T), 256, 0, stream>>>(s->mask, s->t0, s->t1, s->t2, f, s->n1, s->n2);
    if (r == CUFFT_SUCCESS) r = cufftExecD2Z(dfwd, f, Fm);
    zmul_kernel<<<grid_for(S), 256, 0, stream>>>(Ff, Fm, Ff, S);
    zmul_kernel<<<grid_for(S), 256, 0, stream>>>(Ff2, Fm, Ff2, S);
    if (r == CUFFT_SUCCESS) r = cufftExecZ2D(dinv, Ff, f);
    if (r == CUFFT_SUCCESS) r = cufftExecZ2D(dinv, Ff2, f2);
    inv_den_kernel<<<grid_for(N), 256, 0, stream>>>(f, f2, 1.0 / (double)N, s->mask_sum,
                                                   (double)1.1920928955078125e-07, s->inv_den, N);
    if (r == CUFFT_SUCCESS) r = cufftExecR2C(s->fwd, centred, (cufftComplex*)s->ft_target);
    cudaFreeAsync(f, stream); cudaFreeAsync(f2, stream);
    cudaFreeAsync(Ff, stream); cudaFreeAsync(Ff2, stream); cudaFreeAsync(Fm, stream);
    cudaStreamSynchronize(stream);
    cufftDestroy(dfwd);
    cufftDestroy(dinv);
  }
  cudaFreeAsync(centred, stream);
  cudaFreeAsync(partial, stream);
  TM_TRY(cufft_status((cufftResult)r, "scan_set_target: transforms"));
  if (s->xtc_avail)
    TM_TRY(xcorr_tc_prepare(s->ft_target, s->ctarget, s->n0, s->n1, s->h2, stream));
  s->target_ready = true;
  return check_launch("scan_set_target");
}

// x pass on the tensor cores (mode 0, the default where supported) or as FFTs on the
// CUDA cores (mode 1). A captured launch-group graph is dropped.
int scan_set_xpass(Scan* s, int mode) {
  TM_REQUIRE(s, "scan_set_xpass: null plan");
  TM_REQUIRE(mode >= 0 && mode <= 2,
             "scan_set_xpass: mode must be 0 (tensor cores), 1 (FFT) or 2 (default)");
  const bool want =
      mode == 2 ? (s->xtc_avail && s->half && (s->xcfg.hk || s->xcfg.ws)) : mode == 0;
  if (want && !s->xtc_avail) {
    set_error("scan_set_xpass: the tensor-core x pass does not support this plan");
    return TM_E_UNSUPPORTED;
  }
  if (want != s->xtc && s->gexec) { cudaGraphExecDestroy(s->gexec); s->gexec = nullptr; }
  s->xtc = want;
  return TM_OK;
}

int scan_xpass_mode(const Scan* s) { return s && s->xtc ? 0 : 1; }

// z pass on the tensor cores (mode 0, the default where supported: half-precision
// CC / FLCSphericalMask plans with n2 <= 256) or as FFTs on the CUDA cores (mode 1).
int scan_set_zpass(Scan* s, int mode) {
  TM_REQUIRE(s, "scan_set_zpass: null plan");
  TM_REQUIRE(mode >= 0 && mode <= 2,
             "scan_set_zpass: mode must be 0 (tensor cores), 1 (FFT) or 2 (default)");
  const bool want = mode == 1 ? false : (mode == 0 || s->ztc_avail);
  if (want && !s->ztc_avail) {
    set_error("scan_set_zpass: the tensor-core z pass does not support this plan");
    return TM_E_UNSUPPORTED;
  }
  if (want != s->ztc && s->gexec) { cudaGraphExecDestroy(s->gexec); s->gexec = nullptr; }
  s->ztc = want;
  return TM_OK;
}

int scan_zpass_mode(const Scan* s) { return s && s->ztc ? 0 : 1; }

// y pass on the tensor cores (mode 0: radix 16 in FP32 registers, radix n1/16 as an FP16
// GEMM; half-precision CC / FLCSphericalMask plans with n1 in {256, 512}; the default
// where available), as FFTs on the CUDA cores (mode 1), the default (mode 2), or with both
// DFT stages on the tensor cores (mode 3: needs the warp-specialised tensor-core x pass,
// which then writes the y pass's stage-1 layout), or as mode 0 but in place on row-major H
// (mode 4; mode 0 reads the x'-inner H the warp-specialised x pass writes, see x_inner).
int scan_set_ypass(Scan* s, int mode) {
  TM_REQUIRE(s, "scan_set_ypass: null plan");
  TM_REQUIRE(mode >= 0 && mode <= 4,
             "scan_set_ypass: mode must be 0 (tensor cores), 1 (FFT), 2 (default), 3 "
             "(both DFT stages on the tensor cores) or 4 (tensor cores, in place)");
  if (mode == 3 && !(s->ytc_avail && x_writes_stage1(s))) {
    set_error("scan_set_ypass: both y stages on the tensor cores need the tensor-core y pass "
              "and the warp-specialised tensor-core x pass");
    return TM_E_UNSUPPORTED;
  }
  const bool want = mode == 0 || mode == 3 || mode == 4 || (mode == 2 && s->ytc_avail);
  const bool s1 = mode == 3, inplace = mode == 4;
  if ((s1 != s->ys1 || inplace != s->yinplace) && s->gexec) {
    cudaGraphExecDestroy(s->gexec);
    s->gexec = nullptr;
  }
  s->ys1 = s1;
  s->yinplace = inplace;
  if (want && !s->ytc_avail) {
    set_error("scan_set_ypass: the tensor-core y pass does not support this plan");
    return TM_E_UNSUPPORTED;
  }
  if (want != s->ytc && s->gexec) { cudaGraphExecDestroy(s->gexec); s->gexec = nullptr; }
  s->ytc = want;
  return TM_OK;
}

int scan_ypass_mode(const Scan* s) {
  if (!s || !s->ytc) return 1;
  return y_stage1_tc(s) ? 3 : s->yinplace ? 4 : 0;
}

// Polls of every data wait in the plan's tensor-core kernels (0 restores the default).
int scan_set_wait_budget(Scan* s, uint32_t iters) {
  TM_REQUIRE(s, "scan_set_wait_budget: null plan");
  const uint32_t v = iters ? iters : tc_wait_iters_default();
  if (v != s->wait_iters && s->gexec) { cudaGraphExecDestroy(s->gexec); s->gexec = nullptr; }
  s->wait_iters = v;
  return TM_OK;
}

uint32_t tc_wait_iters_default() { return tc::kWaitIters; }

// Synchronise `stream` and report a timed-out wait of the tensor-core passes.
int scan_check(Scan* s, cudaStream_t stream) {
  TM_REQUIRE(s, "scan_check: null plan");
  TM_TRY(cuda_status(cudaStreamSynchronize(stream), "scan_check"));
  if (!s->tc_err) return TM_OK;
  int h = 0;
  TM_TRY(cuda_status(cudaMemcpy(&h, s->tc_err, sizeof(int), cudaMemcpyDeviceToHost), "scan_check"));
  if (h) {
    cudaMemset(s->tc_err, 0, sizeof(int));
    set_error("scan_check: a tensor-core wait timed out");
    return TM_E_TIMEOUT;
  }
  return TM_OK;
}

static int make_coefficients(Scan* s, cudaStream_t stream) {
  TM_TRY(spline_prefilter(s->tmpl, s->coef, s->t0, s->t1, s->t2, 1, stream));
  if (s->d.score == TM_SCORE_FLC) TM_TRY(to_double(s->mask, s->mcoef, s->T, stream));
  return TM_OK;
}

// template/mask: reversed (t0,t1,t2) float32 device arrays; filter: (t0,t1,t2//2+1) or null.
int scan_set_template(Scan* s, const float* tmpl, const float* mask, const float* filt,
                      cudaStream_t stream) {
  TM_REQUIRE(s && tmpl, "scan_set_template: null template");
  TM_REQUIRE(s->d.score == TM_SCORE_CC || mask, "scan_set_template: this score needs a mask");
  cudaMemcpyAsync(s->tmpl, tmpl, sizeof(float) * s->T, cudaMemcpyDeviceToDevice, stream);
  if (mask) cudaMemcpyAsync(s->mask, mask, sizeof(float) * s->T, cudaMemcpyDeviceToDevice, stream);
  s->d.has_template_filter = filt != nullptr;
  if (filt) cudaMemcpyAsync(s->tfilter, filt, sizeof(float) * s->TS, cudaMemcpyDeviceToDevice, stream);
  if (mask) {
    // n_obs = sum(mask) in the backend float dtype (corr_scoring, matching_scores.py:573-576)
    double* partial = nullptr;
    const int nparts = 64;
    TM_TRY(cuda_status(cudaMallocAsync((void**)&partial, sizeof(double) * nparts, stream), "alloc"));
    sum_double_kernel<<<nparts, 256, 0, stream>>>(s->mask, s->T, partial);
    std::vector<double> hp(nparts);
    cudaMemcpyAsync(hp.data(), partial, sizeof(double) * nparts, cudaMemcpyDeviceToHost, stream);
    cudaFreeAsync(partial, stream);
    TM_TRY(cuda_status(cudaStreamSynchronize(stream), "scan_set_template: mask sum"));
    double tot = 0.0;
    for (double v : hp) tot += v;
    s->mask_sum = tot;
  }
  s->template_ready = true;
  if (s->order == 3) TM_TRY(make_coefficients(s, stream));
  return check_launch("scan_set_template");
}

// interpolation_order of corr_scoring / flc_scoring (tme/matching_scores.py:600-608,
// 731-740), passed on to rigid_transform (tme/backends/npfftw_backend.py:390-449): the
// template is prefiltered, the mask is not. A captured launch-group graph is dropped
// because it holds the other rotation kernel.
int scan_set_interpolation(Scan* s, int order, cudaStream_t stream) {
  TM_REQUIRE(s, "scan_set_interpolation: null plan");
  if (order == 0) order = 1;
  if (order != 1 && order != 3) {
    set_error("scan_set_interpolation: interpolation order %d is not supported (1 and 3 are)",
              order);
    return TM_E_UNSUPPORTED;
  }
  if (order == s->order) return TM_OK;
  if (s->gexec) { cudaGraphExecDestroy(s->gexec); s->gexec = nullptr; }
  s->order = order;
  if (order == 3) {
    if (!s->coef) {
      TM_TRY(cuda_status(cudaMalloc((void**)&s->coef, sizeof(double) * s->T), "coefficients"));
      TM_TRY(cuda_status(cudaMalloc((void**)&s->mcoef, sizeof(double) * s->T), "coefficients"));
    }
    if (s->template_ready) TM_TRY(make_coefficients(s, stream));
  }
  return TM_OK;
}

// rotate, filter and normalise B templates of the current group into rot_t (and rot_m for FLC)
static int prepare_templates(Scan* s, int nb, cudaStream_t stream) {
  const bool flc = s->d.score == TM_SCORE_FLC;
  if (s->order == 3)
    TM_TRY(rigid_transform_cubic(s->coef, flc ? s->mcoef : nullptr, s->t0, s->t1, s->t2, s->mat,
                                 nb, s->rot_t, flc ? s->rot_m : nullptr, s->t0, s->t1, s->t2,
                                 stream));
  else
    TM_TRY(rigid_transform(s->tmpl, flc ? s->mask : nullptr, s->t0, s->t1, s->t2, s->mat, nb,
                           s->rot_t, flc ? s->rot_m : nullptr, s->t0, s->t1, s->t2, stream));
  if (s->d.has_template_filter) {
    // _apply_filter_subset (tme/matching_scores.py:125-135): rfftn -> * filter -> irfftn
    cufftSetStream(s->tfwd, stream);
    cufftSetStream(s->tinv, stream);
    TM_TRY(cufft_status(cufftExecR2C(s->tfwd, s->rot_t, (cufftComplex*)s->tspec), "filter r2c"));
    TM_TRY(apply_real_filter(s->tspec, s->tfilter, s->TS, s->B, stream));
    TM_TRY(cufft_status(cufftExecC2R(s->tinv, (cufftComplex*)s->tspec, s->rot_t), "filter c2r"));
    TM_TRY(scale_real(s->rot_t, (float)(1.0 / (double)s->T), s->T * s->B, stream));
  }
  if (s->d.score == TM_SCORE_FLCSM) {
    TM_TRY(normalize_template(s->rot_t, s->mask, 0, s->t0, s->t1, s->t2, s->t1, s->t2, s->T, nb,
                              s->mask_sum, s->stats_ws, stream));
  } else if (flc) {
    TM_TRY(normalize_template(s->rot_t, s->rot_m, s->T, s->t0, s->t1, s->t2, s->t1, s->t2, s->T,
                              nb, 0.0, s->stats_ws, stream));
  }
  return TM_OK;
}

static int run_plain(Scan* s, int n, int32_t first_index, float* state_max, int32_t* state_rot,
                     const float* matrices, cudaStream_t stream) {
  const int64_t N = s->N, S = s->S;
  const float scale = (float)(1.0 / (double)N);
  const double eps = 1.1920928955078125e-07;
  const bool flc = s->d.score == TM_SCORE_FLC;
  cufftSetStream(s->fwd, stream);
  cufftSetStream(s->inv, stream);
  for (int i = 0; i < n; ++i) {
    cudaMemcpyAsync(s->mat, matrices + (int64_t)i * 16, sizeof(float) * 16,
                    cudaMemcpyDeviceToDevice, stream);
    TM_TRY(prepare_templates(s, 1, stream));
    cudaMemsetAsync(s->arr, 0, sizeof(float) * N, stream);
    TM_TRY(pad_box(s->rot_t, s->t0, s->t1, s->t2, s->arr, s->n1, s->n2, stream));
    if (flc) {
      cudaMemsetAsync(s->arr_m, 0, sizeof(float) * N, stream);
      TM_TRY(pad_box(s->rot_m, s->t0, s->t1, s->t2, s->arr_m, s->n1, s->n2, stream));
      TM_TRY(cufft_status(cufftExecR2C(s->fwd, s->arr_m, (cufftComplex*)s->spec_m), "r2c mask"));
      TM_TRY(complex_multiply(s->ft_target, s->spec_m, s->spec, S, stream));
      TM_TRY(cufft_status(cufftExecC2R(s->inv, (cufftComplex*)s->spec, s->cc_m), "c2r"));
      TM_TRY(complex_multiply(s->ft_target2, s->spec_m, s->spec, S, stream));
      TM_TRY(cufft_status(cufftExecC2R(s->inv, (cufftComplex*)s->spec, s->cc_m2), "c2r"));
    }
    TM_TRY(cufft_status(cufftExecR2C(s->fwd, s->arr, (cufftComplex*)s->spec), "r2c"));
    TM_TRY(complex_multiply(s->ft_target, s->spec, s->spec, S, stream));
    TM_TRY(cufft_status(cufftExecC2R(s->inv, (cufftComplex*)s->spec, s->arr), "c2r"));
    const double* stats = s->stats_ws + (int64_t)1 * kStatChunks * 3;
    TM_TRY(plain_epilogue(s->arr, s->inv_den, flc ? s->cc_m : nullptr, flc ? s->cc_m2 : nullptr,
                          stats, eps, scale, state_max, state_rot, first_index + i, N, stream));
  }
  return TM_OK;
}

__global__ void set_first_kernel(int32_t* p, int32_t v) { *p = v; }

// One launch group: template preparation and the four passes for nb rotations whose
// matrices are already in s->mat.
static int launch_group(Scan* s, int nb, double hs, float out_scale, int32_t first,
                        float* state_max, int32_t* state_rot, cudaStream_t stream) {
  StageTimer tmr(s, stream);
  tmr.begin();
  TM_TRY(prepare_templates(s, nb, stream));
  tmr.end(TM_STAGE_PREPARE);
  const int64_t rows = (int64_t)s->n0 * s->n1;
  dim3 g4(ceil_div(rows, s->R4));
  if (s->half) {
    __half2* H = static_cast<__half2*>(s->H);
    TM_TRY(launch_template_x_y<__half2>(s, nb, (float)hs, H, tmr, stream));
    tmr.begin();
    if (s->d.score == TM_SCORE_FLC)
      launch_zpass_flc<__half2>(s, H, nb, rows, out_scale, first, state_max, state_rot, stream);
    else
      launch_zpass<__half2>(s, g4, x_inner(s) ? static_cast<__half2*>(s->H2) : H, nb, rows,
                            out_scale, first, state_max, state_rot, stream);
    TM_TRY(check_launch("z pass"));
    tmr.end(TM_STAGE_ZPASS);
  } else {
    float2* H = static_cast<float2*>(s->H);
    TM_TRY(launch_template_x_y<float2>(s, nb, (float)hs, H, tmr, stream));
    tmr.begin();
    if (s->d.score == TM_SCORE_FLC)
      launch_zpass_flc<float2>(s, H, nb, rows, out_scale, first, state_max, state_rot, stream);
    else
      launch_zpass<float2>(s, g4, H, nb, rows, out_scale, first, state_max, state_rot, stream);
    TM_TRY(check_launch("z pass"));
    tmr.end(TM_STAGE_ZPASS);
  }
  return TM_OK;
}

// Full groups replay one captured graph: the group's matrices are copied into s->mat
// and its first rotation index into s->first_dev before each replay, on the caller's
// stream; the graph runs on a plan-owned stream ordered after and before the caller's.
static int replay_group(Scan* s, double hs, float out_scale, int32_t first, float* state_max,
                        int32_t* state_rot, cudaStream_t stream) {
  set_first_kernel<<<1, 1, 0, stream>>>(s->first_dev, first);
  TM_TRY(check_launch("set_first_kernel"));
  if (!s->gstream) {
    TM_TRY(cuda_status(cudaStreamCreateWithFlags(&s->gstream, cudaStreamNonBlocking), "graph stream"));
    TM_TRY(cuda_status(cudaEventCreateWithFlags(&s->gev_in, cudaEventDisableTiming), "graph event"));
    TM_TRY(cuda_status(cudaEventCreateWithFlags(&s->gev_out, cudaEventDisableTiming), "graph event"));
  }
  TM_TRY(cuda_status(cudaEventRecord(s->gev_in, stream), "graph event"));
  TM_TRY(cuda_status(cudaStreamWaitEvent(s->gstream, s->gev_in, 0), "graph wait"));
  if (!s->gexec || s->gkey_max != state_max || s->gkey_rot != state_rot) {
    if (s->gexec) { cudaGraphExecDestroy(s->gexec); s->gexec = nullptr; }
    cudaGraph_t graph = nullptr;
    s->graph_first = s->first_dev;
    const bool timing = s->timing;
    s->timing = false;
    TM_TRY(cuda_status(cudaStreamBeginCapture(s->gstream, cudaStreamCaptureModeThreadLocal),
                       "begin capture"));
    int st = launch_group(s, s->B, hs, out_scale, first, state_max, state_rot, s->gstream);
    cudaError_t e = cudaStreamEndCapture(s->gstream, &graph);
    s->timing = timing;
    s->graph_first = nullptr;
    if (st != TM_OK) { if (graph) cudaGraphDestroy(graph); return st; }
    TM_TRY(cuda_status(e, "end capture"));
    e = cudaGraphInstantiate(&s->gexec, graph, 0);
    cudaGraphDestroy(graph);
    TM_TRY(cuda_status(e, "graph instantiate"));
    s->gkey_max = state_max;
    s->gkey_rot = state_rot;
  }
  TM_TRY(cuda_status(cudaGraphLaunch(s->gexec, s->gstream), "graph launch"));
  TM_TRY(cuda_status(cudaEventRecord(s->gev_out, s->gstream), "graph event"));
  return cuda_status(cudaStreamWaitEvent(stream, s->gev_out, 0), "graph wait");
}

static int run_fused(Scan* s, int n, int32_t first_index, float* state_max, int32_t* state_rot,
                     const float* matrices, cudaStream_t stream) {
  const double Nd = (double)s->N;
  // H holds the product after two inverse passes scaled by hs; the z pass divides by
  // N * hs. hs keeps half2 storage in range.
  double hs = 1.0;
  if (s->half) hs = 1.0 / (sqrt(Nd) * sqrt((double)s->n0) * sqrt(std::max(1.0, s->mask_sum)));
  const float out_scale = (float)(1.0 / (Nd * hs));
  for (int g0 = 0; g0 < n; g0 += s->B) {
    const int nb = std::min(s->B, n - g0);
    cudaMemcpyAsync(s->mat, matrices + (int64_t)g0 * 16, sizeof(float) * 16 * nb,
                    cudaMemcpyDeviceToDevice, stream);
    if (s->use_graph && nb == s->B && !s->timing) {
      TM_TRY(replay_group(s, hs, out_scale, first_index + g0, state_max, state_rot, stream));
    } else {
      TM_TRY(launch_group(s, nb, hs, out_scale, first_index + g0, state_max, state_rot, stream));
    }
  }
  return TM_OK;
}

int scan_set_graph(Scan* s, int enable) {
  TM_REQUIRE(s, "scan_set_graph: null plan");
  if (!s->fused) enable = 0;  // the plain path is one rotation at a time by design
  s->use_graph = enable != 0;
  if (!s->use_graph && s->gexec) { cudaGraphExecDestroy(s->gexec); s->gexec = nullptr; }
  return TM_OK;
}

int scan_set_timing(Scan* s, int enable) {
  TM_REQUIRE(s, "scan_set_timing: null plan");
  if (enable && !s->have_events) {
    for (auto& e : s->ev) TM_TRY(cuda_status(cudaEventCreate(&e), "scan_set_timing: event"));
    s->have_events = true;
  }
  s->timing = enable != 0;
  for (int i = 0; i < TM_NUM_STAGES; ++i) { s->stage_ms[i] = 0.0; s->stage_launches[i] = 0; }
  return TM_OK;
}

int scan_get_timing(const Scan* s, double* ms, int64_t* launches) {
  TM_REQUIRE(s && ms && launches, "scan_get_timing: null pointer");
  for (int i = 0; i < TM_NUM_STAGES; ++i) { ms[i] = s->stage_ms[i]; launches[i] = s->stage_launches[i]; }
  return TM_OK;
}

int64_t scan_stage_bytes(const Scan* s, int stage, int nb) {
  // Algorithmic HBM bytes of one launch of a stage for a group of nb rotations:
  // every array the stage must read or write once, at its storage width. FLC
  // carries two extra complex64 statistics spectra per rotation.
  const int64_t e = s->half ? 4 : 8;
  const bool flc = s->d.score == TM_SCORE_FLC;
  const int64_t G = (int64_t)nb * s->t0 * s->n1 * s->h2 * 8;
  const int64_t H = (int64_t)nb * s->S * e;
  const int64_t Hs = flc ? 2 * (int64_t)nb * s->S * 8 : 0;
  switch (stage) {
    case TM_STAGE_TEMPLATE: return (flc ? 2 : 1) * ((int64_t)nb * s->T * 4 + G);
    case TM_STAGE_XPASS: return (flc ? 2 : 1) * (G + s->S * 8) + H + Hs;
    case TM_STAGE_YPASS: return 2 * (H + Hs);
    case TM_STAGE_ZPASS: return H + Hs + s->N * (s->inv_den ? 4 : 0) + s->N * 16;
    default: return 0;
  }
}

int scan_run(Scan* s, const float* matrices, int n, int32_t first_index, float* state_max,
             int32_t* state_rot, cudaStream_t stream) {
  TM_REQUIRE(s && state_max && state_rot, "scan_run: null pointer");
  TM_REQUIRE(n == 0 || matrices, "scan_run: null matrices");
  TM_REQUIRE(s->target_ready && s->template_ready, "scan_run: target and template must be set");
  TM_REQUIRE(n >= 0, "scan_run: negative rotation count");
  if (n == 0) return TM_OK;
  return s->fused ? run_fused(s, n, first_index, state_max, state_rot, matrices, stream)
                  : run_plain(s, n, first_index, state_max, state_rot, matrices, stream);
}

// Line-FFT self test: y[l][:] = FFT_dir(x[l][:]) for `lines` lines of length n
// (interleaved smem tile), used by the test-suite to check the device FFT code.
__global__ void line_fft_test_kernel(const float2* x, float2* y, int n, int lines, LinePlan p,
                                     const float2* tw_g, int dir) {
  extern __shared__ float4 smem_raw[];
  float2* tw = reinterpret_cast<float2*>(smem_raw);
  float2* buf = tw + n;
  for (int i = threadIdx.x; i < n; i += kThreads) tw[i] = tw_g[i];
  for (int e = threadIdx.x; e < n * lines; e += kThreads) {
    int i = e / lines, l = e % lines;
    buf[e] = x[(int64_t)l * n + i];
  }
  __syncthreads();
  if (dir < 0) fft::fft_lines<-1, kMaxE, true>(buf, p, lines, 1, lines, tw, n, threadIdx.x, kThreads);
  else fft::fft_lines<1, kMaxE, true>(buf, p, lines, 1, lines, tw, n, threadIdx.x, kThreads);
  for (int e = threadIdx.x; e < n * lines; e += kThreads) {
    int i = e / lines, l = e % lines;
    y[(int64_t)l * n + i] = buf[e];
  }
}

int line_fft_test(const void* x, void* y, int n, int lines, int dir, cudaStream_t stream) {
  TM_REQUIRE(line_supported(n), "line_fft_test: length %d not supported", n);
  TM_REQUIRE(lines >= 1 && (int64_t)n * lines <= kTile, "line_fft_test: tile too large");
  LinePlan p = make_line_plan(n);
  auto tv = twiddle_table(n);
  float2* tw = nullptr;
  TM_TRY(cuda_status(cudaMalloc(&tw, sizeof(float2) * n), "line_fft_test: alloc"));
  cudaMemcpy(tw, tv.data(), sizeof(float2) * n, cudaMemcpyHostToDevice);
  size_t smem = sizeof(float2) * (n + (size_t)n * lines);
  cudaFuncSetAttribute(line_fft_test_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_optin_max());
  line_fft_test_kernel<<<1, kThreads, smem, stream>>>((const float2*)x, (float2*)y, n, lines, p, tw, dir);
  int st = check_launch("line_fft_test_kernel");
  cudaStreamSynchronize(stream);
  cudaFree(tw);
  return st;
}

}  // namespace tmb
