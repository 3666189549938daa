// x pass of the fused FLCSphericalMask / CC scan on the 5th-generation tensor cores.
//
// For one spectrum column (k1, k2) the x pass turns the template's (y, z)-transformed
// rows g_b[x] (x < t0, zero beyond) into
//     H_b[x'] = sum_k e^{+2 pi i k x'/n0} s F[k] sum_x e^{-2 pi i k x/n0} g_b[x]
//             = sum_{x < t0} c[(x' - x) mod n0] g_b[x],
// c = s * (unnormalised inverse DFT along x of the target spectrum column): a circular
// correlation, i.e. a (n0 x t0) Toeplitz matrix times the (t0 x B) matrix of the group's
// rotations. This kernel evaluates it as a GEMM with tcgen05.mma (kind::tf32, FP32
// accumulators in tensor memory) instead of a forward and an inverse FFT per column and
// rotation.
//
// Complex arithmetic in real form: rows interleave (Re, Im) of x', the K dimension holds
// (Re g[x], Im g[x]):   [Re H; Im H] = [[Re c, -Im c], [Im c, Re c]] [Re g; Im g].
// Precision: every operand is split into a TF32 head (low 13 mantissa bits cleared) and
// the FP32 remainder, and hi*hi + hi*lo + lo*hi are accumulated (three MMAs), which
// keeps the products to about 2^-20 relative: the FP32 path's accuracy.
//
// A CTA owns W consecutive k2 columns of one k1 row and every rotation of the group. It
// stages c for its columns and the split G operands in shared memory once, then for each
// 64-row block of x' builds the Toeplitz operand of each column in shared memory
// (canonical K-major layout without swizzle: 8-row x 16-byte core matrices), one thread
// issues the MMAs, tcgen05.commit signals an mbarrier, and all warps read the
// accumulators back with tcgen05.ld and store H rows of W consecutive k2.
// Every wait is bounded; on a timeout the kernel records an error, frees its tensor
// memory and returns.
#include "common.cuh"
#include "xcorr_tc.cuh"

#include <cuda_fp16.h>
#include <cufft.h>

#include <algorithm>

namespace tmb {

namespace {

constexpr int kTcThreads = 256;
constexpr int kTileRows = 128;          // MMA M: 64 values of x' as (Re, Im) row pairs
constexpr int kTmemCols = 128;          // W * NB accumulator columns (fp32)
constexpr uint32_t kWaitIters = 1u << 22;

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ float tf32_head(float v) {
  return __uint_as_float(__float_as_uint(v) & 0xffffe000u);
}

// Canonical K-major, no-swizzle operand: element (r, k) of a rows x K tile.
__device__ __forceinline__ int kmajor_index(int r, int k, int K) {
  return (r >> 3) * (K * 8) + (k >> 2) * 32 + (r & 7) * 4 + (k & 3);
}

__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3fffu);
  d |= (uint64_t)((lbo >> 4) & 0x3fffu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3fffu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, no swizzle
}

__device__ __forceinline__ void mma_tf32(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :
               : "r"(mbar)
               : "memory");
}

__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t phase) {
  for (uint32_t i = 0; i < kWaitIters; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tmem_ld8(uint32_t addr, float (&v)[8]) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                 "=r"(r[6]), "=r"(r[7])
               : "r"(addr));
#pragma unroll
  for (int i = 0; i < 8; ++i) v[i] = __uint_as_float(r[i]);
}

template <typename HT>
struct StoreH;
template <>
struct StoreH<float2> {
  static __device__ __forceinline__ void put(float2* p, float re, float im) {
    *p = make_float2(re, im);
  }
};
template <>
struct StoreH<__half2> {
  static __device__ __forceinline__ void put(__half2* p, float re, float im) {
    *p = __floats2half2_rn(re, im);
  }
};

template <typename HT>
__global__ void __launch_bounds__(kTcThreads, 1)
xcorr_tc_kernel(const float2* __restrict__ G, const float2* __restrict__ C, int nb, int NB,
                int W, int t0, int t0p, int n0, int n1, int h2, float scale,
                HT* __restrict__ H, int* __restrict__ err) {
  extern __shared__ __align__(128) float smem_f[];
  const int K = 2 * t0p;
  float* a_hi = smem_f;
  float* a_lo = a_hi + kTileRows * K;
  float* b_all = a_lo + kTileRows * K;      // [w][hi|lo][NB x K]
  float2* cwin = reinterpret_cast<float2*>(b_all + W * 2 * NB * K);  // [w][n0]
  uint64_t* mbar = reinterpret_cast<uint64_t*>(cwin + W * n0);
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + 1);
  int* fail = reinterpret_cast<int*>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int k1 = blockIdx.y, k20 = blockIdx.x * W;
  const int64_t row = (int64_t)n1 * h2;
  const int64_t col0 = (int64_t)k1 * h2 + k20;
  const int64_t S = (int64_t)n0 * row;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_u32(tmem_slot)), "r"(kTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" : : "r"(smem_u32(mbar)));
    asm volatile("fence.mbarrier_init.release.cluster;");
    *fail = 0;
  }
  // target correlation kernels of the CTA's columns
  for (int i = tid; i < W * n0; i += kTcThreads) {
    const int w = i / n0, m = i - w * n0;
    cwin[i] = (k20 + w < h2) ? C[(int64_t)m * row + col0 + w] : make_float2(0.f, 0.f);
  }
  // split rotation operands: B_w[n][k] = (Re g_n[k], Im g_n[k - t0p]), K-major
  for (int i = tid; i < W * NB * t0p; i += kTcThreads) {
    const int w = i % W;
    const int rest = i / W;
    const int x = rest % t0p, n = rest / t0p;
    float2 g = make_float2(0.f, 0.f);
    if (x < t0 && n < nb && k20 + w < h2) g = G[((int64_t)n * t0 + x) * row + col0 + w];
    float* bh = b_all + (size_t)w * 2 * NB * K;
    float* bl = bh + NB * K;
    const float rh = tf32_head(g.x), ih = tf32_head(g.y);
    bh[kmajor_index(n, x, K)] = rh;
    bl[kmajor_index(n, x, K)] = g.x - rh;
    bh[kmajor_index(n, x + t0p, K)] = ih;
    bl[kmajor_index(n, x + t0p, K)] = g.y - ih;
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;
  const uint32_t mbar_a = smem_u32(mbar);
  // instruction descriptor: F32 accumulate, TF32 A and B, both K-major, M = 128, N = NB
  const uint32_t idesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(NB >> 3) << 17) |
                         ((uint32_t)(kTileRows >> 4) << 24);
  const uint32_t sbo_a = (uint32_t)K * 32u;  // bytes between 8-row core-matrix groups
  const uint32_t lbo = 128u;                 // bytes between K-adjacent core matrices
  uint32_t phase = 0;
  const int quarter = warp & 3, half = warp >> 2;
  bool ok = true;

  for (int x0 = 0; x0 < n0 && ok; x0 += kTileRows / 2) {
    for (int w = 0; w < W && ok; ++w) {
      // Toeplitz operand of column w for rows x' in [x0, x0 + 64)
      const float2* cw = cwin + w * n0;
      for (int i = tid; i < kTileRows * t0p; i += kTcThreads) {
        const int r = i % kTileRows, x = i / kTileRows;
        const int j = r >> 1, im = r & 1;
        float v0 = 0.f, v1 = 0.f;  // coefficients of Re g[x] and Im g[x]
        if (x < t0) {
          int d = x0 + j - x;
          d += (d < 0) ? n0 : 0;
          const float2 c = cw[d];
          v0 = scale * (im ? c.y : c.x);
          v1 = scale * (im ? c.x : -c.y);
        }
        const float h0 = tf32_head(v0), h1 = tf32_head(v1);
        a_hi[kmajor_index(r, x, K)] = h0;
        a_lo[kmajor_index(r, x, K)] = v0 - h0;
        a_hi[kmajor_index(r, x + t0p, K)] = h1;
        a_lo[kmajor_index(r, x + t0p, K)] = v1 - h1;
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncthreads();
      if (tid == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;");
        const float* bh = b_all + (size_t)w * 2 * NB * K;
        const float* bl = bh + NB * K;
        const uint32_t ah = smem_u32(a_hi), al = smem_u32(a_lo);
        const uint32_t bhh = smem_u32(bh), bll = smem_u32(bl);
        const uint32_t sbo_b = (uint32_t)K * 32u;
        const uint32_t d = tmem + (uint32_t)(w * NB);
        uint32_t acc = 0;
        for (int s = 0; s < K / 8; ++s) {
          const uint32_t off = (uint32_t)s * 256u;  // two core matrices along K
          mma_tf32(d, smem_desc(ah + off, lbo, sbo_a), smem_desc(bhh + off, lbo, sbo_b), idesc,
                   acc);
          acc = 1;
          mma_tf32(d, smem_desc(ah + off, lbo, sbo_a), smem_desc(bll + off, lbo, sbo_b), idesc,
                   1);
          mma_tf32(d, smem_desc(al + off, lbo, sbo_a), smem_desc(bhh + off, lbo, sbo_b), idesc,
                   1);
        }
        mma_commit(mbar_a);
        if (!mbar_wait(mbar_a, phase)) *fail = 1;
        asm volatile("tcgen05.fence::before_thread_sync;");
      }
      phase ^= 1u;
      __syncthreads();
      asm volatile("tcgen05.fence::after_thread_sync;");
      if (*fail) ok = false;
    }
    if (!ok) break;
    // accumulators of the W columns -> H rows x' in [x0, x0 + 64)
    const int rlane = quarter * 32 + lane;          // accumulator row of this thread
    const int xp = x0 + (rlane >> 1);
    for (int b0 = half * 8; b0 < NB; b0 += 16) {
      float v[4][8], u[4][8];
#pragma unroll
      for (int w = 0; w < 4; ++w)
        if (w < W)
          tmem_ld8(tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(w * NB + b0), v[w]);
      asm volatile("tcgen05.wait::ld.sync.aligned;");
      // rows come in (Re, Im) pairs on neighbouring lanes: even lanes take the odd
      // neighbour's value as the imaginary part and store
#pragma unroll
      for (int w = 0; w < 4; ++w)
#pragma unroll
        for (int q = 0; q < 8; ++q) u[w][q] = __shfl_down_sync(0xffffffffu, v[w][q], 1);
      if (!(lane & 1)) {
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int b = b0 + q;
          if (b >= nb) break;
          HT* h = H + (int64_t)b * S + (int64_t)xp * row + col0;
#pragma unroll
          for (int w = 0; w < 4; ++w)
            if (w < W && k20 + w < h2) StoreH<HT>::put(h + w, v[w][q], u[w][q]);
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
  }
  if (!ok && tid == 0) {
    // the MMAs of the failed wait may still be running: give them a second bounded wait
    mbar_wait(mbar_a, phase ^ 1u);
  }
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :
                 : "r"(tmem), "r"(kTmemCols));
  if (tid == 0 && !ok) atomicExch(err, 1);
}

}  // namespace

int xcorr_tc_config(int n0, int t0, int nb, XcorrTcConfig* cfg) {
  cfg->ok = false;
  if (n0 % 64 != 0 || nb < 1) return TM_OK;
  cfg->t0p = (t0 + 3) / 4 * 4;
  cfg->K = 2 * cfg->t0p;
  cfg->NB = (nb + 7) / 8 * 8;
  if (cfg->NB > 64) return TM_OK;
  cfg->W = cfg->NB <= 32 ? 4 : 2;
  cfg->smem = (size_t)(2 * kTileRows * cfg->K + cfg->W * 2 * cfg->NB * cfg->K) * sizeof(float) +
              (size_t)cfg->W * n0 * sizeof(float2) + 16;
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaGetLastError();
  cfg->ok = cfg->smem <= (size_t)optin;
  if (cfg->ok) {
    // set once per configuration, outside any stream capture
    TM_TRY(cuda_status(cudaFuncSetAttribute(xcorr_tc_kernel<float2>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, optin),
                       "xcorr_tc: shared memory attribute"));
    TM_TRY(cuda_status(cudaFuncSetAttribute(xcorr_tc_kernel<__half2>,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, optin),
                       "xcorr_tc: shared memory attribute"));
  }
  return TM_OK;
}

int xcorr_tc_prepare(const float2* F, float2* C, int n0, int n1, int h2, cudaStream_t stream) {
  TM_REQUIRE(F && C, "xcorr_tc_prepare: null pointer");
  cufftHandle plan;
  int n[1] = {n0};
  const int dist = 1, stride = n1 * h2;
  cufftResult r = cufftPlanMany(&plan, 1, n, n, stride, dist, n, stride, dist, CUFFT_C2C,
                                n1 * h2);
  if (r != CUFFT_SUCCESS) {
    set_error("xcorr_tc_prepare: cuFFT plan error %d", (int)r);
    return r == CUFFT_ALLOC_FAILED ? TM_E_OOM : TM_E_CUFFT;
  }
  cufftSetStream(plan, stream);
  r = cufftExecC2C(plan, (cufftComplex*)const_cast<float2*>(F), (cufftComplex*)C, CUFFT_INVERSE);
  cufftDestroy(plan);
  if (r != CUFFT_SUCCESS) {
    set_error("xcorr_tc_prepare: cuFFT error %d", (int)r);
    return TM_E_CUFFT;
  }
  return check_launch("xcorr_tc_prepare");
}

template <typename HT>
static int launch_xcorr(const XcorrTcConfig& cfg, const float2* G, const float2* C, int nb,
                        int t0, int n0, int n1, int h2, float scale, HT* H, int* err,
                        cudaStream_t stream) {
  dim3 g((unsigned)ceil_div(h2, cfg.W), (unsigned)n1);
  xcorr_tc_kernel<HT><<<g, kTcThreads, cfg.smem, stream>>>(G, C, nb, cfg.NB, cfg.W, t0, cfg.t0p,
                                                          n0, n1, h2, scale, H, err);
  return check_launch("xcorr_tc_kernel");
}

int xcorr_tc_run(const XcorrTcConfig& cfg, const float2* G, const float2* C, int nb, int t0,
                 int n0, int n1, int h2, float scale, void* H, bool half, int* err,
                 cudaStream_t stream) {
  TM_REQUIRE(cfg.ok, "xcorr_tc_run: unsupported configuration");
  TM_REQUIRE(nb <= cfg.NB, "xcorr_tc_run: %d rotations exceed the configured %d", nb, cfg.NB);
  if (half)
    return launch_xcorr<__half2>(cfg, G, C, nb, t0, n0, n1, h2, scale,
                                 static_cast<__half2*>(H), err, stream);
  return launch_xcorr<float2>(cfg, G, C, nb, t0, n0, n1, h2, scale, static_cast<float2*>(H),
                              err, stream);
}

}  // namespace tmb
