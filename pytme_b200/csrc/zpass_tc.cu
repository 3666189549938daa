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
                int* __restrict__ err) {
  if (first_dev) first_index = *first_dev;
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
      if (j >= 2 && !mbar_wait(smem_u32(tempty + sidx), (u - 1) & 1u)) { *fail = 1; break; }
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
        if (!mbar_wait(smem_u32(bfull + sidx), u & 1u)) { *fail = 1; break; }
        if (j >= 2 && !mbar_wait(smem_u32(tempty + sidx), (u - 1) & 1u)) { *fail = 1; break; }
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
      if (!mbar_wait(smem_u32(tfull + sidx), u & 1u)) { *fail = 1; break; }
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

}  // namespace

int zpass_tc_config(int n2, int h2, int hp, int nb, ZpassTcConfig* cfg) {
  cfg->ok = false;
  cfg->K = 2 * hp;
  cfg->n2 = n2;
  cfg->smem = (size_t)(2 * zrows(n2) + 2 * kZN) * cfg->K * 2 +
              (size_t)4 * kZRows * n2 * sizeof(float) + 8 * 8 + 16;
  // z < 256 in two M = 128 tiles; the second tile's reads past the tail stay inside the
  // operand buffers when zrows(n2) >= 64
  if (n2 > kZM || n2 < 128 || n2 % 4 != 0 || hp % 8 != 0 || nb < 1 || nb > kZRot || h2 > hp)
    return TM_OK;
  int dev = 0, optin = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaGetLastError();
  cfg->sms = sms;
  if (cfg->smem > (size_t)optin) return TM_OK;
  TM_TRY(cuda_status(cudaFuncSetAttribute(zpass_tc_kernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, optin),
                     "zpass_tc: shared memory attribute"));
  cfg->ok = true;
  return TM_OK;
}

size_t zpass_tc_table_bytes(const ZpassTcConfig& cfg) {
  return (size_t)2 * zrows(cfg.n2) * cfg.K * 2;
}

int zpass_tc_prepare(const ZpassTcConfig& cfg, uint16_t* table, int n2, int h2,
                     cudaStream_t stream) {
  TM_REQUIRE(cfg.ok && table, "zpass_tc_prepare: unsupported configuration");
  zdft_table_kernel<<<64, 256, 0, stream>>>(table, n2, h2, cfg.K);
  return check_launch("zdft_table_kernel");
}

int zpass_tc_run(const ZpassTcConfig& cfg, const void* H, int nb, int64_t rows, int n2, int h2,
                 int hp, const uint16_t* table, float scale, const float* inv_den,
                 int32_t first_index, float* state_max, int32_t* state_rot, int64_t SH,
                 const int32_t* first_dev, int* err, cudaStream_t stream) {
  TM_REQUIRE(cfg.ok, "zpass_tc_run: unsupported configuration");
  TM_REQUIRE(nb >= 1 && nb <= kZRot, "zpass_tc_run: %d rotations per group (1..%d)", nb, kZRot);
  const int64_t nblk = (rows + kZRows - 1) / kZRows;
  const int grid = (int)std::min<int64_t>(nblk, cfg.sms);
  zpass_tc_kernel<<<grid, kZThreads, cfg.smem, stream>>>(
      static_cast<const __half2*>(H), nb, rows, n2, h2, hp, table, scale, inv_den, first_index,
      state_max, state_rot, SH, first_dev, err);
  return check_launch("zpass_tc_kernel");
}

}  // namespace tmb
