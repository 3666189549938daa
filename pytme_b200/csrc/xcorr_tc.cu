// x pass of the fused FLCSphericalMask / CC scan on the 5th-generation tensor cores.
//
// For one spectrum column (k1, k2) the x pass turns the template's (y, z)-transformed
// rows g_b[x] (x < t0, zero beyond) into
//     H_b[x'] = sum_k e^{+2 pi i k x'/n0} s F[k] sum_x e^{-2 pi i k x/n0} g_b[x]
//             = sum_{x < t0} c[(x' - x) mod n0] g_b[x],
// c = s * (unnormalised inverse DFT along x of the target spectrum column): a circular
// correlation, i.e. a (n0 x t0) Toeplitz matrix times the (t0 x B) matrix of the group's
// rotations. This kernel evaluates it as a GEMM with tcgen05.mma (kind::f16 with BF16
// operands, FP32 accumulators in tensor memory) instead of a forward and an inverse FFT
// per column and rotation.
//
// Complex arithmetic in real form: rows interleave (Re, Im) of x', the K dimension holds
// (Re g[x], Im g[x]):   [Re H; Im H] = [[Re c, -Im c], [Im c, Re c]] [Re g; Im g].
// Precision: every operand is split into a BF16 head and a BF16 tail (the rounded
// remainder), and hi*hi + hi*lo + lo*hi are accumulated (three MMAs): products carry
// about 16 significant bits, errors of a few 1e-6 relative to the largest term.
//
// A CTA owns W consecutive k2 columns of one k1 row and every rotation of the group. It
// stages c (scaled, split) for its columns and the split G operands in shared memory
// once, then for each 64-row block of x' builds the Toeplitz operand of each column in
// shared memory (canonical K-major layout without swizzle: 8-row x 16-byte core
// matrices, 16-byte stores laid out so a quarter warp covers one core-matrix row set),
// double-buffered so that building column w + 1 overlaps the MMAs of column w. One
// thread issues the MMAs, tcgen05.commit signals the buffer's mbarrier, and at the end
// of a row block all warps read the accumulators back with tcgen05.ld and store H rows
// of W consecutive k2 (accumulators alternate between two tensor-memory halves).
// Every wait is bounded; on a timeout the kernel records an error, frees its tensor
// memory and returns.
#include "common.cuh"
#include "tc_common.cuh"
#include "xcorr_tc.cuh"

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cufft.h>

#include <algorithm>

namespace tmb {

namespace {

constexpr int kTcThreads = 256;
constexpr int kTileRows = 128;          // MMA M: 64 values of x' as (Re, Im) row pairs
using tc::kmajor16;
using tc::kWaitIters;
using tc::mbar_wait;
using tc::mma_commit;
using tc::smem_desc;
using tc::smem_u32;

__device__ __forceinline__ void mma_bf16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
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

__device__ __forceinline__ void tmem_ld4(uint32_t addr, float (&v)[4]) {
  uint32_t r[4];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(addr));
#pragma unroll
  for (int i = 0; i < 4; ++i) v[i] = __uint_as_float(r[i]);
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
                int W, int t0, int t0p, int n0, int n1, int h2, int hp, float scale,
                HT* __restrict__ H, int* __restrict__ err) {
  extern __shared__ __align__(128) uint16_t smem_h[];
  const int K = 2 * t0p;              // multiple of 16
  const int E = n0 + t0p + 8;         // extended length of the correlation kernels
  const int PAD = t0p + 8;
  uint16_t* a_buf = smem_h;                               // [2 buffers][hi|lo][128 x K]
  uint16_t* b_all = a_buf + 4 * kTileRows * K;            // [w][hi|lo][NB x K]
  uint16_t* comps = b_all + W * 2 * NB * K;               // [w][6][E]
  uint64_t* mbar = reinterpret_cast<uint64_t*>(comps + ((W * 6 * E + 7) & ~7));
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + 2);
  int* fail = reinterpret_cast<int*>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int k1 = blockIdx.y, k20 = blockIdx.x * W;
  const int64_t row = (int64_t)n1 * h2;
  const int64_t col0 = (int64_t)k1 * h2 + k20;
  const int64_t rowH = (int64_t)n1 * hp, colH = (int64_t)k1 * hp + k20;
  const int64_t SH = (int64_t)n0 * rowH;

  // two row blocks of W * NB fp32 accumulator columns, rounded up to a power of two
  uint32_t tmem_cols = 32;
  while (tmem_cols < (uint32_t)(2 * W * NB)) tmem_cols <<= 1;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_u32(tmem_slot)), "r"(tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" : : "r"(smem_u32(mbar)));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" : : "r"(smem_u32(mbar + 1)));
    asm volatile("fence.mbarrier_init.release.cluster;");
    *fail = 0;
  }
  // correlation kernels of the CTA's columns, scaled and split into BF16 head and tail:
  // comps[w][0..5] = (Re hi, Re lo, Im hi, Im lo, -Im hi, -Im lo), index d + PAD for
  // d in [-PAD, n0) (circular)
  for (int i = tid; i < W * E; i += kTcThreads) {
    const int w = i / E, e = i - w * E;
    int m = e - PAD;
    m += (m < 0) ? n0 : 0;
    float2 c = make_float2(0.f, 0.f);
    if (k20 + w < h2) c = C[(int64_t)m * row + col0 + w];
    c.x *= scale;
    c.y *= scale;
    uint16_t* cp = comps + (size_t)w * 6 * E + e;
    const __nv_bfloat16 rh = __float2bfloat16_rn(c.x), ih = __float2bfloat16_rn(c.y);
    const __nv_bfloat16 rl = __float2bfloat16_rn(c.x - __bfloat162float(rh));
    const __nv_bfloat16 il = __float2bfloat16_rn(c.y - __bfloat162float(ih));
    cp[0 * E] = __bfloat16_as_ushort(rh);
    cp[1 * E] = __bfloat16_as_ushort(rl);
    cp[2 * E] = __bfloat16_as_ushort(ih);
    cp[3 * E] = __bfloat16_as_ushort(il);
    cp[4 * E] = __bfloat16_as_ushort(__hneg(ih));
    cp[5 * E] = __bfloat16_as_ushort(__hneg(il));
  }
  // rotation operands B_w[n][k] = (Re g_n[k], Im g_n[k - t0p]), K-major, head and tail
  for (int i = tid; i < W * NB * t0p; i += kTcThreads) {
    const int w = i % W;
    const int rest = i / W;
    const int x = rest % t0p, n = rest / t0p;
    float2 g = make_float2(0.f, 0.f);
    if (x < t0 && n < nb && k20 + w < h2) g = G[((int64_t)n * t0 + x) * row + col0 + w];
    uint16_t* bh = b_all + (size_t)w * 2 * NB * K;
    uint16_t* bl = bh + NB * K;
    const __nv_bfloat16 rh = __float2bfloat16_rn(g.x), ih = __float2bfloat16_rn(g.y);
    bh[kmajor16(n, x, K)] = __bfloat16_as_ushort(rh);
    bl[kmajor16(n, x, K)] = __bfloat16_as_ushort(__float2bfloat16_rn(g.x - __bfloat162float(rh)));
    bh[kmajor16(n, x + t0p, K)] = __bfloat16_as_ushort(ih);
    bl[kmajor16(n, x + t0p, K)] = __bfloat16_as_ushort(__float2bfloat16_rn(g.y - __bfloat162float(ih)));
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;
  // instruction descriptor: F32 accumulate, BF16 A and B, both K-major, M = 128, N = NB
  const uint32_t idesc = (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(NB >> 3) << 17) |
                         ((uint32_t)(kTileRows >> 4) << 24);
  const uint32_t sbo = (uint32_t)K * 16u;  // bytes between 8-row core-matrix groups
  const uint32_t lbo = 128u;               // bytes between K-adjacent core matrices
  uint32_t phase[2] = {0u, 0u};
  bool pending[2] = {false, false};  // a commit on this buffer's barrier not yet waited for
  const int quarter = warp & 3, half = warp >> 2;
  const int nkc = K / 8;
  // build tasks: (head/tail, 8-column chunk kc) groups of 8 lanes; lane = (row parity s,
  // row phase ph), so the 8 lanes of a quarter warp store 8 distinct rows of a core matrix
  const int ph = tid & 3, s = (tid >> 2) & 1;
  bool ok = true;
  const int ntile = n0 / (kTileRows / 2);
  const int iters = ntile * W;

  for (int it = 0; it < iters && ok; ++it) {
    const int tile = it / W, w = it - tile * W;
    const int x0 = tile * (kTileRows / 2);
    const int bi = it & 1;
    uint16_t* a_hi = a_buf + (size_t)bi * 2 * kTileRows * K;
    uint16_t* a_lo = a_hi + kTileRows * K;
    if (pending[bi]) {
      // the MMAs of iteration it - 2 read this buffer
      if (tid == 0 && !mbar_wait(smem_u32(mbar + bi), phase[bi])) *fail = 1;
      phase[bi] ^= 1u;
      pending[bi] = false;
      __syncthreads();
      if (*fail) { ok = false; break; }
    }
    for (int tg = tid >> 3; tg < 2 * nkc; tg += kTcThreads / 8) {
      const int kc = tg % nkc, tail = tg / nkc;
      const int kx = kc * 8;
      const int part = kx < t0p ? 0 : 1;     // 0: multiplies Re g, 1: multiplies Im g
      const int xs = part ? kx - t0p : kx;   // first x of the chunk
      // component: part 0 -> (s ? Im : Re), part 1 -> (s ? Re : -Im)
      const int comp = (part == 0 ? (s ? 2 : 0) : (s ? 0 : 4)) + tail;
      const uint16_t* cp = comps + ((size_t)w * 6 + comp) * E + PAD;
      uint16_t* dst = tail ? a_lo : a_hi;
#pragma unroll 4
      for (int j = ph; j < kTileRows / 2; j += 4) {
        const int d0 = x0 + j - xs;  // kernel index of the chunk's first x
        uint32_t pk[4];
#pragma unroll
        for (int q = 0; q < 8; q += 2) {
          const uint32_t lo = (xs + q < t0) ? cp[d0 - q] : 0u;
          const uint32_t hi = (xs + q + 1 < t0) ? cp[d0 - q - 1] : 0u;
          pk[q >> 1] = lo | (hi << 16);
        }
        const int r = 2 * j + s;
        *reinterpret_cast<uint4*>(dst + kmajor16(r, kx, K)) = make_uint4(pk[0], pk[1], pk[2], pk[3]);
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint16_t* bh = b_all + (size_t)w * 2 * NB * K;
      const uint16_t* bl = bh + NB * K;
      const uint32_t ah = smem_u32(a_hi), al = smem_u32(a_lo);
      const uint32_t bhh = smem_u32(bh), bll = smem_u32(bl);
      const uint32_t d = tmem + (uint32_t)((tile & 1) * W * NB + w * NB);
      for (int st = 0; st < K / 16; ++st) {
        const uint32_t off = (uint32_t)st * 256u;  // two core matrices along K
        mma_bf16(d, smem_desc(ah + off, lbo, sbo), smem_desc(bhh + off, lbo, sbo), idesc,
                 st > 0);
        mma_bf16(d, smem_desc(ah + off, lbo, sbo), smem_desc(bll + off, lbo, sbo), idesc, 1);
        mma_bf16(d, smem_desc(al + off, lbo, sbo), smem_desc(bhh + off, lbo, sbo), idesc, 1);
      }
      mma_commit(smem_u32(mbar + bi));
    }
    pending[bi] = true;
    if (w == W - 1) {
      // drain the tile: wait for every outstanding commit
#pragma unroll
      for (int q = 0; q < 2; ++q)
        if (pending[q]) {
          if (tid == 0 && !mbar_wait(smem_u32(mbar + q), phase[q])) *fail = 1;
          phase[q] ^= 1u;
          pending[q] = false;
        }
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncthreads();
      asm volatile("tcgen05.fence::after_thread_sync;");
      if (*fail) { ok = false; break; }
      const uint32_t tbase = tmem + ((uint32_t)(quarter * 32) << 16) +
                             (uint32_t)((tile & 1) * W * NB);
      const int xp = x0 + ((quarter * 32 + lane) >> 1);
      for (int b0 = half * 8; b0 < NB; b0 += 16) {
        float v[4][8], u[4][8];
#pragma unroll
        for (int ww = 0; ww < 4; ++ww)
          if (ww < W) tmem_ld8(tbase + (uint32_t)(ww * NB + b0), v[ww]);
        asm volatile("tcgen05.wait::ld.sync.aligned;");
#pragma unroll
        for (int ww = 0; ww < 4; ++ww)
#pragma unroll
          for (int q = 0; q < 8; ++q) u[ww][q] = __shfl_down_sync(0xffffffffu, v[ww][q], 1);
        if (!(lane & 1)) {
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const int b = b0 + q;
            if (b >= nb) break;
            HT* h = H + (int64_t)b * SH + (int64_t)xp * rowH + colH;
#pragma unroll
            for (int ww = 0; ww < 4; ++ww)
              if (ww < W && k20 + ww < h2) StoreH<HT>::put(h + ww, v[ww][q], u[ww][q]);
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;");
      // the next MMAs go to the other accumulator half; its reads finished above
    }
  }
  if (!ok && tid == 0) {
    // MMAs of a failed wait may still be running: one more bounded wait per buffer
    for (int q = 0; q < 2; ++q)
      if (pending[q]) mbar_wait(smem_u32(mbar + q), phase[q]);
  }
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :
                 : "r"(tmem), "r"(tmem_cols));
  if (tid == 0 && !ok) atomicExch(err, 1);
}

// ---------------------------------------------------------------------------------
// Mixed-precision variant: one FP16 product per term (the rotation spectra are stored in
// half precision by this path anyway), and the correlation operand as a Hankel matrix
// addressed in place. With the rows of a 128-row block in reverse order of x'
// (row r <-> x' = x0 + 127 - r) the operand is A[r][x] = c[x0 + 127 - r - x], a function
// of r + x. Writing e[i] = c[(n0 - 1 - i) mod n0] and Z block u = the 8 x 8 matrix with
// row p = e[8u + p .. 8u + p + 7], the canonical core matrix (row group g, K chunk kc)
// of the block at x0 is Z block (n0 - 128 - x0)/8 + g + kc: a descriptor with both
// strides 128 bytes reads every row block from one Z array per component, built once
// per column. Re and Im of H accumulate separately:
//   Re H = Re c * Re g - Im c * Im g,   Im H = Im c * Re g + Re c * Im g,
// the minus through the instruction descriptor's A-negate bit.
__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

constexpr float kHankelPrescale = 256.f;  // keeps the scaled kernel values in FP16's normal range
constexpr int kHkThreads = 512;

__global__ void __launch_bounds__(kHkThreads, 1)
xcorr_hankel_kernel(const float2* __restrict__ G, const float2* __restrict__ C, int nb, int NB,
                    int W, int t0, int t0p, int n0, int n1, int h2, int hp, float scale,
                    __half2* __restrict__ H, int* __restrict__ err) {
  extern __shared__ __align__(128) uint16_t smem_h[];
  const int K = 2 * t0p;                  // multiple of 16
  const int nZ = (n0 + t0p) / 8 + 2;      // Z blocks per component
  const int zsz = nZ * 64;                // halves per Z array
  uint16_t* zs = smem_h;                                  // [w][re|im][nZ x 64]
  uint16_t* bs = zs + (size_t)W * 2 * zsz;                // [w][NB x K]
  // the kernels' diagonal arrays e (FP16, [w][re|im][E2]) after the rotation operands
  const int E2 = 8 * nZ + 8;
  uint16_t* eh = bs + (size_t)W * NB * K;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(eh + (((size_t)W * 2 * E2 + 7) & ~(size_t)7));
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mbar + 2);
  int* fail = reinterpret_cast<int*>(tmem_slot + 1);

  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int k1 = blockIdx.y, k20 = blockIdx.x * W;
  const int64_t row = (int64_t)n1 * h2;
  const int64_t col0 = (int64_t)k1 * h2 + k20;
  const int64_t rowH = (int64_t)n1 * hp, colH = (int64_t)k1 * hp + k20;
  const int64_t SH = (int64_t)n0 * rowH;
  const int blk_cols = 2 * W * NB;        // accumulator columns of one row block (<= 512)
  uint32_t tmem_cols = 32;
  while (tmem_cols < (uint32_t)blk_cols) tmem_cols <<= 1;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_u32(tmem_slot)), "r"(tmem_cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" : : "r"(smem_u32(mbar)));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" : : "r"(smem_u32(mbar + 1)));
    asm volatile("fence.mbarrier_init.release.cluster;");
    *fail = 0;
  }
  // the global loads of the rotation operands and of the kernel columns are independent:
  // both loops run before the first barrier so their latencies overlap
  // rotation operands: B_w[n][k] = (Re g_n[k], Im g_n[k - t0p]) in FP16, K-major; one
  // task = 8 consecutive x of one rotation, stored as two 16-byte rows
  const int nxc = t0p / 8;
#pragma unroll 3
  for (int i = tid; i < W * NB * nxc; i += kHkThreads) {
    const int w = i % W;
    const int rest = i / W;
    const int xc = rest % nxc, n = rest / nxc;
    uint32_t re[4], im[4];
#pragma unroll
    for (int q = 0; q < 8; q += 2) {
      const int x = xc * 8 + q;
      float2 a = make_float2(0.f, 0.f), b = make_float2(0.f, 0.f);
      if (n < nb && k20 + w < h2) {
        if (x < t0) a = G[((int64_t)n * t0 + x) * row + col0 + w];
        if (x + 1 < t0) b = G[((int64_t)n * t0 + x + 1) * row + col0 + w];
      }
      re[q >> 1] = (uint32_t)__half_as_ushort(__float2half_rn(a.x)) |
                   ((uint32_t)__half_as_ushort(__float2half_rn(b.x)) << 16);
      im[q >> 1] = (uint32_t)__half_as_ushort(__float2half_rn(a.y)) |
                   ((uint32_t)__half_as_ushort(__float2half_rn(b.y)) << 16);
    }
    uint16_t* bw = bs + (size_t)w * NB * K;
    *reinterpret_cast<uint4*>(bw + kmajor16(n, xc * 8, K)) = make_uint4(re[0], re[1], re[2], re[3]);
    *reinterpret_cast<uint4*>(bw + kmajor16(n, t0p + xc * 8, K)) =
        make_uint4(im[0], im[1], im[2], im[3]);
  }
  // diagonal arrays e[i] = s * c[(n0 - 1 - i) mod n0] in FP16, read from the kernel columns
  const float cs = scale * kHankelPrescale;
#pragma unroll 4
  for (int i = tid; i < W * E2; i += kHkThreads) {
    const int w = i / E2, e = i - w * E2;
    int m = n0 - 1 - e;
    m += (m < 0) ? n0 : 0;
    const float2 c = (k20 + w < h2) ? C[(int64_t)m * row + col0 + w] : make_float2(0.f, 0.f);
    eh[(size_t)(2 * w) * E2 + e] = __half_as_ushort(__float2half_rn(c.x * cs));
    eh[(size_t)(2 * w + 1) * E2 + e] = __half_as_ushort(__float2half_rn(c.y * cs));
  }
  __syncthreads();
  // Z arrays: block u, row p = e[8u + p + q], q = 0..7
  for (int i = tid; i < W * 2 * nZ * 8; i += kHkThreads) {
    const int p = i & 7;
    const int rest = i >> 3;
    const int u = rest % nZ;
    const int wc = rest / nZ;            // w * 2 + component
    const uint16_t* ew = eh + (size_t)wc * E2 + 8 * u + p;
    uint32_t pk[4];
#pragma unroll
    for (int q = 0; q < 8; q += 2) pk[q >> 1] = (uint32_t)ew[q] | ((uint32_t)ew[q + 1] << 16);
    *reinterpret_cast<uint4*>(zs + (size_t)wc * zsz + (size_t)(u * 8 + p) * 8) =
        make_uint4(pk[0], pk[1], pk[2], pk[3]);
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;
  // F32 accumulate, F16 A and B, both K-major, M = 128, N = NB
  const uint32_t idesc = (1u << 4) | ((uint32_t)(NB >> 3) << 17) | ((uint32_t)(kTileRows >> 4) << 24);
  const uint32_t idesc_neg = idesc | (1u << 13);
  const uint32_t sbo_b = (uint32_t)K * 16u;
  const int ntile = n0 / kTileRows;
  uint32_t phase[2] = {0u, 0u};

  auto issue = [&](int t) {
    if (tid != 0) return;
    asm volatile("tcgen05.fence::after_thread_sync;");
    const int u0 = (n0 - kTileRows - t * kTileRows) / 8;
    const uint32_t dbase = tmem;
    for (int w = 0; w < W; ++w) {
      const uint32_t zr = smem_u32(zs + (size_t)(2 * w) * zsz);
      const uint32_t zi = smem_u32(zs + (size_t)(2 * w + 1) * zsz);
      const uint32_t bw = smem_u32(bs + (size_t)w * NB * K);
      const uint32_t d_re = dbase + (uint32_t)(w * 2 * NB), d_im = d_re + (uint32_t)NB;
      for (int s = 0; s < K / 16; ++s) {
        const int kc = 2 * s;                       // first 8-column chunk of the step
        const bool imag_g = kc * 8 >= t0p;
        const int kcl = imag_g ? kc - t0p / 8 : kc;  // chunk within its half
        const uint32_t za = (uint32_t)(u0 + kcl) * 128u;
        const uint64_t bd = smem_desc(bw + (uint32_t)s * 256u, 128u, sbo_b);
        const uint64_t ar = smem_desc(zr + za, 128u, 128u);
        const uint64_t ai = smem_desc(zi + za, 128u, 128u);
        // Re H: Re c * Re g - Im c * Im g;  Im H: Im c * Re g + Re c * Im g
        mma_f16(d_re, imag_g ? ai : ar, bd, imag_g ? idesc_neg : idesc, s > 0);
        mma_f16(d_im, imag_g ? ar : ai, bd, idesc, s > 0);
      }
    }
    mma_commit(smem_u32(mbar));
  };

  bool ok = true;
  // warps w and w + 4k share the accumulator lanes 32 (w mod 4) ..; the groups k split
  // the rotations
  const int quarter = warp & 3, grp = warp >> 2, ngrp = kHkThreads / 128;
  const float inv = 1.f / kHankelPrescale;
  // 32-byte row segments need 8 columns per CTA and a row pitch of a multiple of 8
  const bool vec = (W == 8 || W == 4) && (hp % 8 == 0);
  for (int t = 0; t < ntile && ok; ++t) {
    issue(t);
    if (tid == 0 && !mbar_wait(smem_u32(mbar), phase[0])) *fail = 1;
    phase[0] ^= 1u;
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (*fail) { ok = false; break; }
    const int r = quarter * 32 + lane;
    const int xp = t * kTileRows + kTileRows - 1 - r;
    const uint32_t tb = tmem + ((uint32_t)(quarter * 32) << 16);
    for (int b0 = grp * 4; b0 < NB; b0 += 4 * ngrp) {
      float vr[8][4], vi[8][4];
#pragma unroll
      for (int w = 0; w < 8; ++w)
        if (w < W) {
          tmem_ld4(tb + (uint32_t)(w * 2 * NB + b0), vr[w]);
          tmem_ld4(tb + (uint32_t)(w * 2 * NB + NB + b0), vi[w]);
        }
      asm volatile("tcgen05.wait::ld.sync.aligned;");
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const int b = b0 + q;
        if (b >= nb) break;
        __half2* h = H + (int64_t)b * SH + (int64_t)xp * rowH + colH;
        if (vec) {
          // W consecutive k2 of a row (padding columns included): aligned 16-byte stores
          uint32_t pk[8];
#pragma unroll
          for (int w = 0; w < 8; ++w) {
            const __half2 hv = __floats2half2_rn(vr[w][q] * inv, vi[w][q] * inv);
            pk[w] = *reinterpret_cast<const uint32_t*>(&hv);
          }
          uint4* dst = reinterpret_cast<uint4*>(h);
          dst[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
          if (W == 8) dst[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
        } else {
#pragma unroll
          for (int w = 0; w < 8; ++w)
            if (w < W && k20 + w < h2) h[w] = __floats2half2_rn(vr[w][q] * inv, vi[w][q] * inv);
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();  // accumulators are free for the next row block
  }
  if (!ok && tid == 0) mbar_wait(smem_u32(mbar), phase[0]);
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :
                 : "r"(tmem), "r"(tmem_cols));
  if (tid == 0 && !ok) atomicExch(err, 1);
}

}  // namespace

int xcorr_tc_config(int n0, int t0, int nb, XcorrTcConfig* cfg) {
  cfg->ok = false;
  cfg->hk = false;
  TM_TRY(xcorr_ws_config(n0, t0, nb, cfg));
  if (n0 % 64 != 0 || nb < 1) return TM_OK;
  cfg->t0p = (t0 + 7) / 8 * 8;
  cfg->K = 2 * cfg->t0p;
  // with M = 128, kind::f16 takes N in steps of 16
  cfg->NB = (nb + 15) / 16 * 16;
  if (cfg->NB > 128) return TM_OK;
  // W * NB accumulator columns per row block, two blocks in the 512 tensor-memory columns
  cfg->W = cfg->NB <= 32 ? 4 : 2;
  const int E = n0 + cfg->t0p + 8;
  cfg->smem = (size_t)(4 * kTileRows * cfg->K + cfg->W * 2 * cfg->NB * cfg->K) * 2 +
              (size_t)((cfg->W * 6 * E + 7) & ~7) * 2 + 32;
  int dev = 0, optin = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaGetLastError();
  cfg->ok = cfg->smem <= (size_t)optin;
  // Hankel variant: 128-row blocks, K steps that never straddle the Re / Im halves
  cfg->hk = false;
  cfg->hk_t0p = (t0 + 15) / 16 * 16;
  // 2 * W * NB accumulator columns: (8, 32), (4, 64) or (2, 128)
  cfg->hk_W = cfg->NB <= 32 ? 8 : (cfg->NB <= 64 ? 4 : 2);
  {
    const int K = 2 * cfg->hk_t0p;
    const int nZ = (n0 + cfg->hk_t0p) / 8 + 2;
    const size_t ereg = (((size_t)cfg->hk_W * 2 * (8 * nZ + 8) + 7) & ~(size_t)7) * 2;
    cfg->hk_smem = (size_t)cfg->hk_W * 2 * nZ * 64 * 2 + (size_t)cfg->hk_W * cfg->NB * K * 2 +
                   ereg + 32;
    cfg->hk = n0 % kTileRows == 0 && cfg->hk_smem <= (size_t)optin;
  }
  if (cfg->hk)
    TM_TRY(cuda_status(cudaFuncSetAttribute(xcorr_hankel_kernel,
                                            cudaFuncAttributeMaxDynamicSharedMemorySize, optin),
                       "xcorr_hankel: shared memory attribute"));
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
                        int t0, int n0, int n1, int h2, int hp, float scale, HT* H, int* err,
                        cudaStream_t stream) {
  dim3 g((unsigned)ceil_div(h2, cfg.W), (unsigned)n1);
  xcorr_tc_kernel<HT><<<g, kTcThreads, cfg.smem, stream>>>(G, C, nb, cfg.NB, cfg.W, t0, cfg.t0p,
                                                          n0, n1, h2, hp, scale, H, err);
  return check_launch("xcorr_tc_kernel");
}

int xcorr_tc_run(const XcorrTcConfig& cfg, const float2* G, const float2* C, int nb, int t0,
                 int n0, int n1, int h2, int hp, float scale, void* H, bool half, int* err,
                 cudaStream_t stream, uint32_t wait_iters, bool seg, int rowq, bool g_half,
                 bool xin) {
  if (half && cfg.ws && nb <= cfg.ws_NB && hp % 8 == 0)
    return xcorr_ws_run(cfg, G, C, nb, t0, n0, n1, h2, hp, scale, static_cast<__half2*>(H), err,
                        stream, wait_iters, seg, rowq, g_half, xin);
  TM_REQUIRE(!seg && rowq == 0 && !g_half && !xin,
             "xcorr_tc_run: segment-layout output needs the warp-specialised kernel");
  TM_REQUIRE(cfg.ok, "xcorr_tc_run: unsupported configuration");
  TM_REQUIRE(nb <= cfg.NB, "xcorr_tc_run: %d rotations exceed the configured %d", nb, cfg.NB);
  if (half && cfg.hk) {
    dim3 g((unsigned)ceil_div(h2, cfg.hk_W), (unsigned)n1);
    xcorr_hankel_kernel<<<g, kHkThreads, cfg.hk_smem, stream>>>(
        G, C, nb, cfg.NB, cfg.hk_W, t0, cfg.hk_t0p, n0, n1, h2, hp, scale,
        static_cast<__half2*>(H), err);
    return check_launch("xcorr_hankel_kernel");
  }
  if (half)
    return launch_xcorr<__half2>(cfg, G, C, nb, t0, n0, n1, h2, hp, scale,
                                 static_cast<__half2*>(H), err, stream);
  return launch_xcorr<float2>(cfg, G, C, nb, t0, n0, n1, h2, hp, scale, static_cast<float2*>(H),
                              err, stream);
}

}  // namespace tmb
