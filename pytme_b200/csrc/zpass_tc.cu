// z pass of the fused CC / FLCSphericalMask scan on the tensor cores.
//
// The z pass turns each row of the intermediate spectra, H_b[x'][y'][k2] (k2 < h2, FP16
// complex, row pitch hp), into n2 real scores by an unnormalised c2r along z,
//     x[z] = Re X[0] + Re X[m] (-1)^z + 2 sum_{0<k<m} (Re X[k] cos(2 pi k z/n2)
//                                                    - Im X[k] sin(2 pi k z/n2)),
// m = n2/2 (the imaginary parts of X[0] and X[m] are dropped as numpy's irfft does), then
// scales by the score normalisation and keeps the strict maximum over the group's
// rotations. Written as a GEMM, a block of rows and rotations is
//     D[z][(row, b)] = sum_K A[z][K] B[K][(row, b)],   K = 2k + (0: Re, 1: Im),
// with A the fixed c2r operator (built once per plan as an FP16 head plus the FP16
// rounded remainder, two MMAs per step, so the products keep about 22 significant bits
// and the only rounding left is that of the FP16 spectra) and B the H rows themselves:
// a row's 2*hp halves are exactly one K-contiguous operand column, so cp.async copies
// 16-byte pieces of H straight into the canonical K-major layout. A CTA takes 2 rows x
// 32 rotations (N = 64) per step, two M = 128 tiles cover z < 256, tcgen05.mma
// accumulates in FP32 in tensor memory; operand buffers and accumulators are double
// buffered so a block's MMAs run while the previous block's epilogue executes and the
// next block's operands are in flight. The epilogue reads each
// (z, row) accumulator run over the rotations with tcgen05.ld, takes the first maximum
// over the rotations, applies the denominator and merges into the running state.
// Persistent CTAs loop over row blocks; every wait is bounded.
#include "common.cuh"
#include "tc_common.cuh"
#include "zpass_tc.cuh"

#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>

namespace tmb {

namespace {

using namespace tc;

constexpr int kZThreads = 512;
constexpr int kZRows = 2;     // H rows per block
constexpr int kZRot = 32;     // rotations per block
constexpr int kZN = kZRows * kZRot;  // MMA N
constexpr int kZM = 256;      // z extent of the two M = 128 tiles

// Rows of the stored operator: z < n2 rounded up to a core-matrix group. The second
// M tile's rows past them read the memory that follows (the tail operator, then the
// rotation operands); those accumulator rows (z >= n2) are never used.
__host__ __device__ inline int zrows(int n2) { return (n2 + 7) / 8 * 8; }

// c2r operator A[z][K] = head + tail, both FP16 (head = A rounded, tail = the rounded
// remainder), canonical K-major layout: [head | tail], zrows(n2) x K each.
__global__ void zdft_table_kernel(uint16_t* __restrict__ A, int n2, int h2, int K) {
  const int zr = zrows(n2);
  const int total = zr * K;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const int z = i / K, kk = i - z * K;
    const int k = kk >> 1, part = kk & 1;
    float v = 0.f;
    if (z < n2 && k < h2) {
      const bool edge = (k == 0) || ((n2 % 2 == 0) && (2 * k == n2));
      if (!(edge && part == 1)) {
        const double c = edge ? 1.0 : 2.0;
        const long long kz = ((long long)k * z) % n2;
        double sn, cs;
        sincospi(2.0 * (double)kz / (double)n2, &sn, &cs);
        v = (float)(part == 0 ? c * cs : -c * sn);
      }
    }
    const __half hi = __float2half_rn(v);
    const __half lo = __float2half_rn(v - __half2float(hi));
    A[kmajor16(z, kk, K)] = __half_as_ushort(hi);
    A[(size_t)zr * K + kmajor16(z, kk, K)] = __half_as_ushort(lo);
  }
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" : : "r"(smem_u32(bar)) : "memory");
}
// arrival once this thread's earlier cp.async copies have landed
__device__ __forceinline__ void mbar_arrive_cp_async(uint64_t* bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" : : "r"(smem_u32(bar))
               : "memory");
}

// Warp roles: warp 0 lane 0 issues the MMAs; warps 4-7 and 12-15 (two groups with one
// warp per tensor-memory lane quarter) run the epilogue; warps 1-3 and 8-11 load
// operands, state and denominators. Blocks
// alternate between two operand buffers and two accumulator halves; mbarriers pass
// them between the roles (no block-wide barrier inside the loop):
//   bfull[s]  loads of the block landed               (count: loader threads)
//   tfull[s]  MMAs of the block done                   (tcgen05.commit)
//   tempty[s] epilogue done with the block's accumulators and prefetched state, so the
//             accumulator half and the buffers of parity s are free (count: epilogue
//             threads)
// Block j uses s = j % 2, and the u-th use of a barrier (u = j / 2) completes phase u.
constexpr int kZLoaders = 224, kZEpi = 256;
__device__ __forceinline__ bool zp_epilogue_warp(int w) { return (w & 4) != 0; }
__device__ __forceinline__ int zp_loader_index(int tid) {
  // warps 1-3 -> 0..95, warps 8-11 -> 96..223
  const int w = tid >> 5;
  return w < 4 ? tid - 32 : tid - 256 + 96;
}

__global__ void __launch_bounds__(kZThreads, 1)
zpass_tc_kernel(const __half2* __restrict__ H, int nb, int64_t rows, int n2, int h2, int hp,
                const uint16_t* __restrict__ Ag, float scale, const float* __restrict__ inv_den,
                int32_t first_index, float* __restrict__ state_max,
                int32_t* __restrict__ state_rot, int64_t SH, const int32_t* __restrict__ first_dev,
                int* __restrict__ err, uint32_t wait_iters) {
  if (first_dev) first_index = *first_dev;
  const uint32_t wi = wait_iters ? wait_iters : kWaitIters;  // data waits
  extern __shared__ __align__(128) uint16_t smem_z[];
  const int K = 2 * hp;  // multiple of 16
  const int zr = zrows(n2);
  uint16_t* As = smem_z;                         // [head | tail] x [zr x K]
  uint16_t* Bs = As + (size_t)2 * zr * K;        // 2 buffers x [kZN x K]
  float* sst = reinterpret_cast<float*>(Bs + (size_t)2 * kZN * K);  // 2 x [kZRows x n2]
  float* sden = sst + 2 * kZRows * n2;                              // 2 x [kZRows x n2]
  uint64_t* bar = reinterpret_cast<uint64_t*>(sden + 2 * kZRows * n2);
  uint64_t* bfull = bar;
  uint64_t* tfull = bar + 2;
  uint64_t* tempty = bar + 4;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 8);
  int* fail = reinterpret_cast<int*>(tmem_slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_u32(tmem_slot)), "r"(4 * kZN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int q = 0; q < 2; ++q) {
      mbar_init(bfull + q, kZLoaders);
      mbar_init(tfull + q, 1);
      mbar_init(tempty + q, kZEpi);
    }
    asm volatile("fence.mbarrier_init.release.cluster;");
    *fail = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;

  const int64_t nblk = (rows + kZRows - 1) / kZRows;
  const int64_t mine = nblk > blockIdx.x ? (nblk - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const int kcn = K / 8;  // 16-byte pieces per H row (4 complex values each)
  const uint32_t as = smem_u32(As);
  const uint32_t bsa = smem_u32(Bs);
  const uint32_t bbytes = (uint32_t)kZN * (uint32_t)K * 2u;

  if (warp != 0 && !zp_epilogue_warp(warp)) {
    // ---------------------------------------------------------------- loaders
    const int lt = zp_loader_index(tid);
    const int npa = 2 * zr * K / 8;  // the operator, with block 0
    for (int i = lt; i < npa; i += kZLoaders) cp_async16(as + 16u * i, Ag + 8 * (size_t)i, 16);
    for (int64_t j = 0; j < mine; ++j) {
      const int sidx = (int)(j & 1);
      const uint32_t u = (uint32_t)(j >> 1);
      if (j >= 2 && !mbar_wait_n(smem_u32(tempty + sidx), (u - 1) & 1u, wi)) { *fail = 1; break; }
      if (*fail) break;
      const int64_t row0 = ((int64_t)blockIdx.x + j * gridDim.x) * kZRows;
      const uint32_t dst = bsa + (uint32_t)sidx * bbytes;
      for (int i = lt; i < kZN * kcn; i += kZLoaders) {
        const int n = i / kcn, kc = i - n * kcn;
        const int r = n >> 5, b = n & (kZRot - 1);
        const int64_t row = row0 + r;
        int bytes = 0;
        if (b < nb && row < rows) bytes = max(0, min(4, h2 - 4 * kc)) * 4;
        const __half2* src = bytes ? H + (int64_t)b * SH + row * hp + 4 * kc : H;
        cp_async16(dst + 2u * (uint32_t)kmajor16(n, 8 * kc, K), src, (uint32_t)bytes);
      }
      const int nq = kZRows * n2 / 4;
      const int64_t g0 = row0 * n2;
      const uint32_t sd = smem_u32(sst + sidx * kZRows * n2);
      const uint32_t dd = smem_u32(sden + sidx * kZRows * n2);
      for (int i = lt; i < 2 * nq; i += kZLoaders) {
        const int q = i % nq;
        const int64_t g = g0 + 4 * q;
        const int64_t nvalid = rows * n2 - g;
        const uint32_t bytes = nvalid >= 4 ? 16u : (nvalid > 0 ? (uint32_t)nvalid * 4u : 0u);
        if (i < nq) {
          cp_async16(sd + 16u * q, bytes ? state_max + g : state_max, bytes);
        } else {
          const uint32_t db = inv_den ? bytes : 0u;
          cp_async16(dd + 16u * q, db ? inv_den + g : state_max, db);
        }
      }
      mbar_arrive_cp_async(bfull + sidx);
    }
  } else if (warp == 0) {
    // ---------------------------------------------------------------- MMA issuer
    if (lane == 0) {
      const uint32_t idesc = idesc_f16(128, kZN);
      const uint32_t sbo = (uint32_t)K * 16u;
      const uint32_t tail = (uint32_t)zr * (uint32_t)K * 2u;
      for (int64_t j = 0; j < mine; ++j) {
        const int sidx = (int)(j & 1);
        const uint32_t u = (uint32_t)(j >> 1);
        if (!mbar_wait_n(smem_u32(bfull + sidx), u & 1u, wi)) { *fail = 1; break; }
        if (j >= 2 && !mbar_wait_n(smem_u32(tempty + sidx), (u - 1) & 1u, wi)) { *fail = 1; break; }
        if (*fail) break;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t bj = bsa + (uint32_t)sidx * bbytes;
        for (int m = 0; m < 2; ++m) {
          const uint32_t am = as + (uint32_t)(m * 128) * (uint32_t)K * 2u;
          const uint32_t d = tmem + (uint32_t)(sidx * 2 * kZN + m * kZN);
          for (int st = 0; st < K / 16; ++st) {
            const uint32_t off = (uint32_t)st * 256u;
            const uint64_t bd = smem_desc(bj + off, 128u, sbo);
            mma_f16(d, smem_desc(am + off, 128u, sbo), bd, idesc, st > 0);
            mma_f16(d, smem_desc(am + tail + off, 128u, sbo), bd, idesc, 1);
          }
        }
        mma_commit(smem_u32(tfull + sidx));
      }
    }
  } else if (zp_epilogue_warp(warp)) {
    // ---------------------------------------------------------------- epilogue
    const int quarter = warp & 3, egrp = warp >> 3;
    for (int64_t j = 0; j < mine; ++j) {
      const int sidx = (int)(j & 1);
      const uint32_t u = (uint32_t)(j >> 1);
      if (!mbar_wait_n(smem_u32(tfull + sidx), u & 1u, wi)) { *fail = 1; break; }
      if (*fail) break;
      asm volatile("tcgen05.fence::after_thread_sync;");
      const int64_t row0 = ((int64_t)blockIdx.x + j * gridDim.x) * kZRows;
      const uint32_t tb = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(sidx * 2 * kZN);
      const float* st = sst + sidx * kZRows * n2;
      const float* dn = sden + sidx * kZRows * n2;
#pragma unroll
      for (int pr = egrp; pr < 2 * kZRows; pr += 2) {
        const int m = pr / kZRows, r = pr % kZRows;
        float v[32];
        tmem_ld32(tb + (uint32_t)(m * kZN + r * kZRot), v);
        asm volatile("tcgen05.wait::ld.sync.aligned;");
        const int z = m * 128 + quarter * 32 + lane;
        const int64_t row = row0 + r;
        float best = -INFINITY;
        int arg = -1;
#pragma unroll
        for (int b = 0; b < kZRot; ++b)
          if (b < nb && v[b] > best) { best = v[b]; arg = b; }
        if (z < n2 && row < rows && arg >= 0) {
          const int64_t g = row * n2 + z;
          const int e = r * n2 + z;
          const float sc = best * scale * (inv_den ? dn[e] : 1.f);
          if (sc > st[e]) {
            state_max[g] = sc;
            state_rot[g] = first_index + arg;
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;");
      mbar_arrive(tempty + sidx);
    }
  }
  asm volatile("cp.async.wait_all;\n" ::);
  __syncthreads();
  if (*fail && tid == 0) {
    // MMAs of a failed block may still be running: one bounded wait on each commit
    for (int q = 0; q < 2; ++q) mbar_wait(smem_u32(tfull + q), 0u);
  }
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :
                 : "r"(tmem), "r"(4 * kZN));
  if (tid == 0 && *fail) atomicExch(err, 1);
}


// ---------------------------------------------------------------------------------
// Even/odd variant. With E[z] = sum_k w_k Re X[k] cos(2 pi k z/n2) and
// O[z] = -sum_k w_k Im X[k] sin(2 pi k z/n2) (w_k = 1 for k = 0 and k = n2/2, else 2),
//     x[z] = E[z] + O[z],   x[n2 - z] = E[z] - O[z],
// so z <= n2/2 (one M = 128 tile, n2/2 + 1 <= 128) and K' = h2 rounded up to 16 per GEMM
// give all n2 outputs: two GEMMs with half the K of the interleaved operator, a quarter
// of the MMAs of the two-tile form for the same outputs. The rotation operand holds each
// H row de-interleaved, [Re X[0..K') | Im X[0..K')] (the loaders split the FP16 complex
// values in registers). Blocks are 2 rows x 32 rotations (N = 64) in a ring of 4 stages
// (operand buffer, E and O accumulators in 128 tensor-memory columns, state); two loader
// groups take alternate blocks, so the loads of two blocks are in flight while earlier
// ones are multiplied. A loader that waits for its loads before storing them holds one
// block in flight: with one group, the DRAM round trip set the pace.
constexpr int kEoRows = 2;
constexpr int kEoN = kEoRows * kZRot;  // 64
constexpr int kEoS = 4;                // stages: operand buffers, accumulator pairs, state

__host__ __device__ inline int eo_rows(int n2) { return (n2 / 2 + 1 + 7) / 8 * 8; }

// [C head | C tail | S head | S tail], each zr x K' in the canonical K-major layout:
// C[z][k] = w_k cos(2 pi k z/n2), S[z][k] = -w_k sin(2 pi k z/n2) for z <= n2/2, k < h2.
__global__ void eo_table_kernel(uint16_t* __restrict__ A, int n2, int h2, int Kp) {
  const int zr = eo_rows(n2);
  const int total = zr * Kp;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const int z = i / Kp, k = i - z * Kp;
    float c = 0.f, s = 0.f;
    if (z <= n2 / 2 && k < h2) {
      const double w = (k == 0 || 2 * k == n2) ? 1.0 : 2.0;
      const long long kz = ((long long)k * z) % n2;
      double sn, cs;
      sincospi(2.0 * (double)kz / (double)n2, &sn, &cs);
      c = (float)(w * cs);
      s = (float)(-w * sn);
    }
    const size_t tab = (size_t)zr * Kp;
    const int o = kmajor16(z, k, Kp);
    const __half ch = __float2half_rn(c), sh = __float2half_rn(s);
    A[o] = __half_as_ushort(ch);
    A[tab + o] = __half_as_ushort(__float2half_rn(c - __half2float(ch)));
    A[2 * tab + o] = __half_as_ushort(sh);
    A[3 * tab + o] = __half_as_ushort(__float2half_rn(s - __half2float(sh)));
  }
}

// tcgen05.mma with the shared-memory descriptors given as (low, high) words: the low
// word holds the start address >> 4 and the leading byte offset, so operands are
// advanced by adding byte offsets >> 4 to it (addresses stay below 256 KB)
__device__ __forceinline__ void mma_f16_w(uint32_t tmem_d, uint32_t alo, uint32_t ahi,
                                          uint32_t blo, uint32_t bhi, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t.reg .b64 a, b;\n\t"
      "setp.ne.b32 p, %6, 0;\n\t"
      "mov.b64 a, {%1, %2};\n\t"
      "mov.b64 b, {%3, %4};\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], a, b, %5, p;\n\t}\n"
      :
      : "r"(tmem_d), "r"(alo), "r"(ahi), "r"(blo), "r"(bhi), "r"(idesc), "r"(accumulate));
}
// max of three (NaN operands are skipped, as fmaxf skips them)
__device__ __forceinline__ float fmax3(float a, float b, float c) {
  float d;
  asm("max.f32 %0, %1, %2, %3;" : "=f"(d) : "f"(a), "f"(b), "f"(c));
  return d;
}
// the barrier's phase also waits for this thread's earlier cp.async copies (net zero on
// the expected count: the thread arrives separately)
__device__ __forceinline__ void mbar_track_cp_async(uint64_t* bar) {
  asm volatile("cp.async.mbarrier.arrive.shared::cta.b64 [%0];" : : "r"(smem_u32(bar))
               : "memory");
}

// Roles as in zpass_tc_kernel. Barriers per buffer s:
//   bfull[s]   operands of the block stored, its state and denominators landed
//              (count: loader threads; their cp.async completion tracked as well)
//   bempty[s]  MMAs of the block done: its rotation-operand buffer is free (commit)
//   tfull[s]   accumulators of the block written (commit)
//   tempty[s]  epilogue done: accumulators and state buffers free (count: epilogue)
// Roles: warp 0 issues the MMAs; warps 4-7 run the epilogue (one per tensor-memory lane
// quarter, every row of a block); the loaders form two groups, warps 1-3 and 8-10
// (192 threads) for the blocks of even index and warps 11-15 (160 threads) for the odd
// ones, so each group has two block periods for the DRAM round trip of its loads. With
// an even number of stages a stage always belongs to the same group.
constexpr int kEoEpi = 128;
constexpr int kEoGroup0 = 192, kEoGroup1 = 160;
// 16-byte pieces per loader thread of the segment-layout path: kEoN rows x 2 halves x at
// most 16 segments (h2 <= 128) over the smaller group
constexpr int kEoSegPieces = (kEoN * 2 * 16 + kEoGroup1 - 1) / kEoGroup1;
static_assert(kEoS % 2 == 0, "stages alternate between the two loader groups");
__device__ __forceinline__ bool eo_epilogue_warp(int w) { return w >= 4 && w < 8; }
__device__ __forceinline__ int eo_loader_group(int w) { return w <= 10 ? 0 : 1; }
__device__ __forceinline__ int eo_loader_index(int tid) {
  const int w = tid >> 5;
  if (w < 4) return tid - 32;           // warps 1-3: 0..95
  if (w <= 10) return tid - 256 + 96;   // warps 8-10: 96..191
  return tid - 352;                     // warps 11-15: 0..159
}

// MT: loader tasks per thread of the smaller group, ceil(256 * ceil(ceil(h2/4)/4) / 160).
// SEG: H rows hold 32-byte segments [Re x 8 | Im x 8] of 8 consecutive k2 (the layout the
// tensor-core y pass writes for this kernel) instead of interleaved complex values; the
// loaders then copy each 16-byte half straight into the operand with cp.async.
template <int MT, bool SEG>
__global__ void __launch_bounds__(kZThreads, 1)
zpass_eo_kernel(const __half2* __restrict__ H, int nb, int64_t rows, int n2, int h2, int hp,
                int Kp, const uint16_t* __restrict__ Ag, float scale,
                const float* __restrict__ inv_den, int32_t first_index,
                float* __restrict__ state_max, int32_t* __restrict__ state_rot, int64_t SH,
                const int32_t* __restrict__ first_dev, int* __restrict__ err,
                uint32_t wait_iters) {
  if (first_dev) first_index = *first_dev;
  const uint32_t wi = wait_iters ? wait_iters : kWaitIters;  // data waits
  extern __shared__ __align__(128) uint16_t smem_e[];
  const int zr = eo_rows(n2);
  const int K2 = 2 * Kp;                          // rotation-operand K: Re block, Im block
  const size_t tab = (size_t)zr * Kp;             // halves per operator table
  uint16_t* As = smem_e;                          // 4 tables
  uint16_t* Bs = As + 4 * tab;                    // kEoS buffers x [kEoN x K2]
  float* sst = reinterpret_cast<float*>(Bs + (size_t)kEoS * kEoN * K2);  // kEoS x [kEoRows x n2]
  float* sden = sst + kEoS * kEoRows * n2;                               // kEoS x [kEoRows x n2]
  uint64_t* bar = reinterpret_cast<uint64_t*>(sden + kEoS * kEoRows * n2);
  uint64_t* bfull = bar;
  uint64_t* bempty = bar + kEoS;
  uint64_t* tfull = bar + 2 * kEoS;
  uint64_t* tempty = bar + 3 * kEoS;
  uint64_t* mdone = bar + 4 * kEoS;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 4 * kEoS + 1);
  int* fail = reinterpret_cast<int*>(tmem_slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_u32(tmem_slot)), "r"(2 * kEoS * kEoN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  // zero the rotation-operand buffers once: K positions past h2, rotations past nb and
  // rows past the end are never written and must hold finite values
  for (int i = tid; i < kEoS * kEoN * K2 / 4; i += kZThreads)
    reinterpret_cast<uint2*>(Bs)[i] = make_uint2(0u, 0u);
  if (tid == 0) {
    for (int q = 0; q < kEoS; ++q) {
      mbar_init(bfull + q, (q & 1) ? kEoGroup1 : kEoGroup0);
      mbar_init(bempty + q, 1);
      mbar_init(tfull + q, 1);
      mbar_init(tempty + q, kEoEpi);
    }
    mbar_init(mdone, 1);
    asm volatile("fence.mbarrier_init.release.cluster;");
    *fail = 0;
  }
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;

  const int64_t nblk = (rows + kEoRows - 1) / kEoRows;
  const int64_t mine = nblk > blockIdx.x ? (nblk - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const int zmax = n2 / 2;              // rows z <= zmax of the tile are outputs
  const int zodd = (n2 + 1) / 2 - 1;    // z in [1, zodd] also gives x[n2 - z]

  if (warp != 0 && !eo_epilogue_warp(warp)) {
    // ---------------------------------------------------------------- loaders
    const int grp = eo_loader_group(warp);
    const int gsz = grp ? kEoGroup1 : kEoGroup0;
    const int lt = eo_loader_index(tid);
    // the operator tables, tracked by block 0's barrier (group 0)
    if (grp == 0)
      for (int i = lt; i < (int)(4 * tab / 8); i += kEoGroup0)
        cp_async16(smem_u32(As) + 16u * i, Ag + 8 * (size_t)i, 16);
    if constexpr (SEG) {
      // piece i -> (operand row n = i / (2 nseg), segment c, half part = Re/Im): the
      // lanes of a warp take 16 consecutive 16-byte pieces of one H row. The mapping is
      // the same for every block, so each thread packs its pieces once: bits 0-10 operand
      // offset (16-byte units), 11-15 rotation, 16 row in the block, 17-23 word offset
      // 8 c + 4 part in the H row, 24-27 values k < h2 in the half, 28 present.
      const int nseg = hp / 8;
      const int npiece = kEoN * nseg * 2;
      uint32_t pd[kEoSegPieces];
#pragma unroll
      for (int m = 0; m < kEoSegPieces; ++m) {
        const int i = lt + m * gsz;
        uint32_t d = 0u;
        if (i < npiece) {
          const int part = i & 1, rest = i >> 1;
          const int c = rest % nseg, n = rest / nseg;
          const int valid = min(8, max(0, h2 - 8 * c));
          d = ((uint32_t)kmajor16(n, part * Kp + 8 * c, K2) >> 3) |
              ((uint32_t)(n & (kZRot - 1)) << 11) | ((uint32_t)(n >> 5) << 16) |
              ((uint32_t)(8 * c + 4 * part) << 17) | ((uint32_t)valid << 24) | (1u << 28);
        }
        pd[m] = d;
      }
      for (int64_t j = grp; j < mine; j += 2) {
        const int sidx = (int)(j % kEoS);
        const uint32_t u = (uint32_t)(j / kEoS);
        if (j >= kEoS && !mbar_wait_n(smem_u32(bempty + sidx), (u - 1) & 1u, wi)) {
          *fail = 1;
          break;
        }
        if (*fail) break;
        const int64_t row0 = ((int64_t)blockIdx.x + j * gridDim.x) * kEoRows;
        const uint32_t bj = smem_u32(Bs + (size_t)sidx * kEoN * K2);
#pragma unroll
        for (int m = 0; m < kEoSegPieces; ++m) {
          const uint32_t d = pd[m];
          if (!(d >> 28)) continue;
          const int b = (int)((d >> 11) & 31u);
          const int64_t row = row0 + (int64_t)((d >> 16) & 1u);
          const uint32_t valid = (d >> 24) & 15u;  // values k < h2 in the half
          const bool live = b < nb && row < rows && valid > 0;
          const __half2* src =
              live ? H + (int64_t)b * SH + row * hp + (int64_t)((d >> 17) & 127u) : H;
          cp_async16(bj + 16u * (d & 2047u), src, live ? 2u * valid : 0u);
        }
        if (j >= kEoS && !mbar_wait_n(smem_u32(tempty + sidx), (u - 1) & 1u, wi)) {
          *fail = 1;
          break;
        }
        const int nqs = kEoRows * n2 / 4;
        const int64_t g0 = row0 * n2;
        const int64_t gend = rows * n2;
        const uint32_t sd = smem_u32(sst + sidx * kEoRows * n2);
        const uint32_t dd = smem_u32(sden + sidx * kEoRows * n2);
        for (int q = lt; q < nqs; q += gsz) {
          const int64_t g = g0 + 4 * q;
          const uint32_t bytes = g + 4 <= gend ? 16u : (g < gend ? (uint32_t)(gend - g) * 4u : 0u);
          cp_async16(sd + 16u * q, bytes ? state_max + g : state_max, bytes);
          if (inv_den) cp_async16(dd + 16u * q, bytes ? inv_den + g : state_max, bytes);
        }
        mbar_track_cp_async(bfull + sidx);
        mbar_arrive(bfull + sidx);
      }
    } else {
    // task i = (quad of 4-value chunks i >> 8, 8-row group (i >> 5) & 7, lane i & 31):
    // lanes 0-7 take rows 0-7 of chunk 4q, lanes 8-15 chunk 4q + 1, ...: 64 contiguous
    // bytes per H row per warp access, and 8-byte shared stores that fill two core
    // matrices without conflicts
    static_assert(kEoN == 64, "task decomposition: 8 row groups of 8");
    const int nq = (h2 + 3) / 4;        // 4-value chunks holding values k < h2
    const int nquad = (nq + 3) / 4;
    const int ntask = nquad * 256;
    // per-thread tasks, the same for every block: bits 0-15 shared-memory offset of the
    // Re values (halves; Im at + 8 K'), 16-20 chunk, 21-25 rotation, 26-27 row in the
    // block, 28 live (a task of this launch, chunk holding values k < h2, rotation < nb)
    uint32_t task[MT];
#pragma unroll
    for (int m = 0; m < MT; ++m) {
      const int i = lt + m * gsz;
      const int ln = i & 31, ng = (i >> 5) & 7;
      const int n = ng * 8 + (ln & 7), kq = (i >> 8) * 4 + (ln >> 3);
      const int r = n >> 5, b = n & (kZRot - 1);
      const bool live = i < ntask && kq < nq && b < nb;
      task[m] = (uint32_t)kmajor16(n, 4 * (kq & 31), K2) | ((uint32_t)(kq & 31) << 16) |
                ((uint32_t)b << 21) | ((uint32_t)r << 26) | (live ? 1u << 28 : 0u);
    }
    for (int64_t j = grp; j < mine; j += 2) {
      const int sidx = (int)(j % kEoS);
      const uint32_t u = (uint32_t)(j / kEoS);
      if (j >= kEoS && !mbar_wait_n(smem_u32(bempty + sidx), (u - 1) & 1u, wi)) { *fail = 1; break; }
      if (*fail) break;
      const int64_t row0 = ((int64_t)blockIdx.x + j * gridDim.x) * kEoRows;
      const int64_t left = rows - row0;
      const int rlive = left < kEoRows ? (int)left : kEoRows;  // rows in the block
      uint4 val[MT];
#pragma unroll
      for (int m = 0; m < MT; ++m) {
        const uint32_t tk = task[m];
        const int kq = (tk >> 16) & 31, b = (tk >> 21) & 31, r = (tk >> 26) & 3;
        val[m] = make_uint4(0u, 0u, 0u, 0u);
        if ((tk >> 28) && r < rlive)
          val[m] = __ldg(reinterpret_cast<const uint4*>(H + (int64_t)b * SH + (row0 + r) * hp) + kq);
      }
      if (j >= kEoS && !mbar_wait_n(smem_u32(tempty + sidx), (u - 1) & 1u, wi)) { *fail = 1; break; }
      // state and denominators of the block's rows
      const int nqs = kEoRows * n2 / 4;
      const int64_t g0 = row0 * n2;
      const int64_t gend = rows * n2;
      const uint32_t sd = smem_u32(sst + sidx * kEoRows * n2);
      const uint32_t dd = smem_u32(sden + sidx * kEoRows * n2);
      for (int q = lt; q < nqs; q += gsz) {
        const int64_t g = g0 + 4 * q;
        const uint32_t bytes = g + 4 <= gend ? 16u : (g < gend ? (uint32_t)(gend - g) * 4u : 0u);
        cp_async16(sd + 16u * q, bytes ? state_max + g : state_max, bytes);
      }
      if (inv_den) {
        for (int q = lt; q < nqs; q += gsz) {
          const int64_t g = g0 + 4 * q;
          const uint32_t bytes = g + 4 <= gend ? 16u : (g < gend ? (uint32_t)(gend - g) * 4u : 0u);
          cp_async16(dd + 16u * q, bytes ? inv_den + g : state_max, bytes);
        }
      }
      mbar_track_cp_async(bfull + sidx);
      uint16_t* bj = Bs + (size_t)sidx * kEoN * K2;
#pragma unroll
      for (int m = 0; m < MT; ++m) {
        const uint32_t tk = task[m];
        const int kq = (tk >> 16) & 31, r = (tk >> 26) & 3;
        if ((tk >> 28) && r < rlive) {
          uint4 v = val[m];
          // values k >= h2 of the last chunk are zero in the operand
          const int live = h2 - 4 * kq;
          if (live < 4) v.w = 0u;
          if (live < 3) v.z = 0u;
          if (live < 2) v.y = 0u;
          const uint2 re = make_uint2(__byte_perm(v.x, v.y, 0x5410), __byte_perm(v.z, v.w, 0x5410));
          const uint2 im = make_uint2(__byte_perm(v.x, v.y, 0x7632), __byte_perm(v.z, v.w, 0x7632));
          uint16_t* dst = bj + (tk & 0xffffu);
          *reinterpret_cast<uint2*>(dst) = re;
          *reinterpret_cast<uint2*>(dst + 8 * Kp) = im;  // K' further on: chunk K'/8 later
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(bfull + sidx);
    }
    }  // register-path loaders
  } else if (warp == 0) {
    // ---------------------------------------------------------------- MMA issuer
    if (lane == 0) {
      const uint32_t idesc = idesc_f16(128, kEoN);
      const uint64_t ad = smem_desc(smem_u32(As), 128u, (uint32_t)Kp * 16u);
      const uint64_t bd = smem_desc(smem_u32(Bs), 128u, (uint32_t)K2 * 16u);
      const uint32_t alo = (uint32_t)ad, ahi = (uint32_t)(ad >> 32);
      const uint32_t blo = (uint32_t)bd, bhi = (uint32_t)(bd >> 32);
      const uint32_t tab16 = (uint32_t)(tab * 2 >> 4);            // one table, >> 4
      const uint32_t bbuf16 = (uint32_t)((size_t)kEoN * K2 * 2 >> 4);
      const uint32_t im16 = (uint32_t)Kp;                         // Im block: K' * 16 bytes
      const int steps = Kp / 16;
      bool ok = true;
      for (int64_t j = 0; j < mine; ++j) {
        const int sidx = (int)(j % kEoS);
        const uint32_t u = (uint32_t)(j / kEoS);
        if (!mbar_wait_n(smem_u32(bfull + sidx), u & 1u, wi)) { ok = false; break; }
        if (j >= kEoS && !mbar_wait_n(smem_u32(tempty + sidx), (u - 1) & 1u, wi)) { ok = false; break; }
        if (*fail) { ok = false; break; }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t bj = blo + (uint32_t)sidx * bbuf16;
        const uint32_t dE = tmem + (uint32_t)(sidx * 2 * kEoN), dO = dE + (uint32_t)kEoN;
        for (int s = 0; s < steps; ++s) {
          const uint32_t o = 16u * (uint32_t)s;  // 256 bytes per 16 K values
          mma_f16_w(dE, alo + o, ahi, bj + o, bhi, idesc, s > 0);
          mma_f16_w(dE, alo + tab16 + o, ahi, bj + o, bhi, idesc, 1);
          mma_f16_w(dO, alo + 2 * tab16 + o, ahi, bj + im16 + o, bhi, idesc, s > 0);
          mma_f16_w(dO, alo + 3 * tab16 + o, ahi, bj + im16 + o, bhi, idesc, 1);
        }
        mma_commit(smem_u32(tfull + sidx));
        mma_commit(smem_u32(bempty + sidx));
      }
      if (!ok) *fail = 1;
      // nothing may free tensor memory or shared memory under a running MMA
      mma_commit(smem_u32(mdone));
      if (!mbar_wait(smem_u32(mdone), 0u)) *fail = 1;
    }
  } else {
    // ---------------------------------------------------------------- epilogue
    const int quarter = warp & 3;
    const int z = quarter * 32 + lane;
    bool ok = true;
    for (int64_t j = 0; j < mine && ok; ++j) {
      const int sidx = (int)(j % kEoS);
      const uint32_t u = (uint32_t)(j / kEoS);
      const bool got = mbar_wait_n(smem_u32(tfull + sidx), u & 1u, wi);
      __syncwarp();  // tcgen05.ld needs the whole warp, converged
      if (!__all_sync(0xffffffffu, got)) { *fail = 1; ok = false; break; }
      asm volatile("tcgen05.fence::after_thread_sync;");
      const int64_t row0 = ((int64_t)blockIdx.x + j * gridDim.x) * kEoRows;
      const uint32_t tb = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)(sidx * 2 * kEoN);
      const float* st = sst + sidx * kEoRows * n2;
      const float* dn = sden + sidx * kEoRows * n2;
#pragma unroll 1
      for (int r = 0; r < kEoRows; ++r) {
        float ev[32], ov[32];
        tmem_ld32(tb + (uint32_t)(r * kZRot), ev);
        tmem_ld32(tb + (uint32_t)(kEoN + r * kZRot), ov);
        asm volatile("tcgen05.wait::ld.sync.aligned;");
        const int64_t row = row0 + r;
        if (z <= zmax && row < rows) {
          // maxima of x[z] = E + O and x[n2 - z] = E - O over the rotations (fmaxf skips
          // NaN as the strict comparison does); the first rotation reaching a maximum is
          // looked up only when the scaled maximum beats the running state
          float b1 = -INFINITY, b2 = -INFINITY;
          if (nb == kZRot) {
            // three-input max: two rotations per instruction
#pragma unroll
            for (int b = 0; b < kZRot; b += 2) {
              b1 = fmax3(b1, ev[b] + ov[b], ev[b + 1] + ov[b + 1]);
              b2 = fmax3(b2, ev[b] - ov[b], ev[b + 1] - ov[b + 1]);
            }
          } else {
#pragma unroll
            for (int b = 0; b < kZRot; ++b)
              if (b < nb) {
                b1 = fmaxf(b1, ev[b] + ov[b]);
                b2 = fmaxf(b2, ev[b] - ov[b]);
              }
          }
          const int64_t g = row * n2;
          const int e1 = r * n2 + z;
          const float s1 = b1 * scale * (inv_den ? dn[e1] : 1.f);
          if (b1 > -INFINITY && s1 > st[e1]) {
            int a1 = 0;
#pragma unroll
            for (int b = kZRot - 1; b >= 0; --b)
              if (b < nb && ev[b] + ov[b] == b1) a1 = b;
            state_max[g + z] = s1;
            state_rot[g + z] = first_index + a1;
          }
          if (z >= 1 && z <= zodd) {
            const int e2 = r * n2 + (n2 - z);
            const float s2 = b2 * scale * (inv_den ? dn[e2] : 1.f);
            if (b2 > -INFINITY && s2 > st[e2]) {
              int a2 = 0;
#pragma unroll
              for (int b = kZRot - 1; b >= 0; --b)
                if (b < nb && ev[b] - ov[b] == b2) a2 = b;
              state_max[g + n2 - z] = s2;
              state_rot[g + n2 - z] = first_index + a2;
            }
          }
        }
      }
      asm volatile("tcgen05.fence::before_thread_sync;");
      mbar_arrive(tempty + sidx);
    }
  }
  asm volatile("cp.async.wait_all;\n" ::);
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == 0) {
    __syncwarp();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :
                 : "r"(tmem), "r"(2 * kEoS * kEoN));
  }
  if (tid == 0 && *fail) atomicExch(err, 1);
}

}  // namespace

// loader tasks per thread of the even/odd kernel
static int eo_tasks(int h2) {
  const int nquad = ((h2 + 3) / 4 + 3) / 4;
  return (nquad * 256 + kEoGroup1 - 1) / kEoGroup1;
}

int zpass_tc_config(int n2, int h2, int hp, int nb, ZpassTcConfig* cfg) {
  cfg->ok = false;
  cfg->eo = false;
  cfg->Kp = (h2 + 15) / 16 * 16;
  cfg->zr = eo_rows(n2);
  cfg->eo_smem = ((size_t)4 * cfg->zr * cfg->Kp + (size_t)kEoS * kEoN * 2 * cfg->Kp) * 2 +
                 (size_t)2 * kEoS * kEoRows * n2 * sizeof(float) + (4 * kEoS + 1) * 8 + 16;
  cfg->K = 2 * hp;
  cfg->n2 = n2;
  cfg->smem = (size_t)(2 * zrows(n2) + 2 * kZN) * cfg->K * 2 +
              (size_t)4 * kZRows * n2 * sizeof(float) + 8 * 8 + 16;
  // z < 256 in two M = 128 tiles; the second tile's reads past the tail stay inside the
  // operand buffers when zrows(n2) >= 64
  if (hp % 8 != 0 || nb < 1 || nb > kZRot || h2 > hp || h2 != n2 / 2 + 1) return TM_OK;
  int dev = 0, optin = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaGetLastError();
  cfg->sms = sms;
  // even/odd form: z <= n2/2 in one M = 128 tile
  if (n2 >= 16 && n2 / 2 + 1 <= 128 && eo_tasks(h2) <= 13 && cfg->eo_smem <= (size_t)optin) {
    for (auto fn : {zpass_eo_kernel<12, false>, zpass_eo_kernel<13, false>,
                    zpass_eo_kernel<12, true>, zpass_eo_kernel<13, true>})
      TM_TRY(cuda_status(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              optin),
                         "zpass_tc: shared memory attribute"));
    cfg->eo = true;
    cfg->ok = true;
    return TM_OK;
  }
  // two-tile form: z < 256 in two M = 128 tiles, the operator interleaved like H
  if (n2 > kZM || n2 < 128 || n2 % 4 != 0) return TM_OK;
  if (cfg->smem > (size_t)optin) return TM_OK;
  TM_TRY(cuda_status(cudaFuncSetAttribute(zpass_tc_kernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, optin),
                     "zpass_tc: shared memory attribute"));
  cfg->ok = true;
  return TM_OK;
}

size_t zpass_tc_table_bytes(const ZpassTcConfig& cfg) {
  if (cfg.eo) return (size_t)4 * cfg.zr * cfg.Kp * 2;
  return (size_t)2 * zrows(cfg.n2) * cfg.K * 2;
}

int zpass_tc_prepare(const ZpassTcConfig& cfg, uint16_t* table, int n2, int h2,
                     cudaStream_t stream) {
  TM_REQUIRE(cfg.ok && table, "zpass_tc_prepare: unsupported configuration");
  if (cfg.eo) {
    eo_table_kernel<<<64, 256, 0, stream>>>(table, n2, h2, cfg.Kp);
    return check_launch("eo_table_kernel");
  }
  zdft_table_kernel<<<64, 256, 0, stream>>>(table, n2, h2, cfg.K);
  return check_launch("zdft_table_kernel");
}

int zpass_tc_run(const ZpassTcConfig& cfg, const void* H, int nb, int64_t rows, int n2, int h2,
                 int hp, const uint16_t* table, float scale, const float* inv_den,
                 int32_t first_index, float* state_max, int32_t* state_rot, int64_t SH,
                 const int32_t* first_dev, int* err, cudaStream_t stream, uint32_t wait_iters,
                 bool seg) {
  TM_REQUIRE(cfg.ok, "zpass_tc_run: unsupported configuration");
  TM_REQUIRE(!seg || cfg.eo, "zpass_tc_run: segment-layout rows need the even/odd kernel");
  TM_REQUIRE(nb >= 1 && nb <= kZRot, "zpass_tc_run: %d rotations per group (1..%d)", nb, kZRot);
  if (cfg.eo) {
    const int64_t nblk = (rows + kEoRows - 1) / kEoRows;
    const int grid = (int)std::min<int64_t>(nblk, cfg.sms);
    auto fn = eo_tasks(h2) <= 12 ? (seg ? zpass_eo_kernel<12, true> : zpass_eo_kernel<12, false>)
                                 : (seg ? zpass_eo_kernel<13, true> : zpass_eo_kernel<13, false>);
    fn<<<grid, kZThreads, cfg.eo_smem, stream>>>(
        static_cast<const __half2*>(H), nb, rows, n2, h2, hp, cfg.Kp, table, scale, inv_den,
        first_index, state_max, state_rot, SH, first_dev, err, wait_iters);
    return check_launch("zpass_eo_kernel");
  }
  const int64_t nblk = (rows + kZRows - 1) / kZRows;
  const int grid = (int)std::min<int64_t>(nblk, cfg.sms);
  zpass_tc_kernel<<<grid, kZThreads, cfg.smem, stream>>>(
      static_cast<const __half2*>(H), nb, rows, n2, h2, hp, table, scale, inv_den, first_index,
      state_max, state_rot, SH, first_dev, err, wait_iters);
  return check_launch("zpass_tc_kernel");
}

}  // namespace tmb
