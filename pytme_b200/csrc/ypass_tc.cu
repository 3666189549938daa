// y pass of the fused CC / FLCSphericalMask scan on the tensor cores.
//
// For every rotation, x' plane and k2 column of the half-precision intermediate spectra
// H[b][x'][k1][k2] (row pitch hp), the unnormalised inverse DFT along y,
//     Y[y'] = sum_{k1 < n1} X[k1] w^(k1 y'),   w = exp(+2 pi i / n1),  n1 = 16 Q,
// runs as two GEMM stages with k1 = Q a + c and y' = y1 + 16 y2 (a, y1 < 16; c, y2 < Q):
//     Z[y1][c]      = sum_{a < 16} X[Q a + c] w16^(a y1)       (stage 1, radix 16)
//     Z'[y1][c]     = Z[y1][c] w^(c y1)                        (twiddle, CUDA cores)
//     Y[y1 + 16 y2] = sum_{c < Q} Z'[y1][c] wQ^(c y2)          (stage 2, radix Q)
// Complex products are real GEMMs over interleaved (Re, Im) K positions: the data are the
// M operand (rows = independent transforms), a fixed DFT operator the N operand, with
// output columns [Re | Im] of the operator's FP16 head and then of its FP16 rounded
// remainder (the tail), so one MMA pass gives head and tail products side by side and the
// epilogue adds them (the operators keep about 22 significant bits). The only added
// rounding is that of Z' to FP16 between the stages.
//
// A work item is one rotation, one x' plane and 8 consecutive k2 columns: n1 rows of
// 32 bytes (one sector each), read and written in place. Roles of the persistent
// 512-thread CTA:
//   warp 0        one thread issues the MMAs of both stages;
//   warps 1-3     load items straight into the stage-1 operand with 4-byte cp.async
//                 (the gather k1 = Q a + c -> row (c, k2), K position 2a is done by the
//                 copies' addresses), kYS1 items in flight;
//   warps 4-11    stage-1 epilogue: tensor memory -> head + tail -> twiddle -> FP16 ->
//                 the stage-2 operand (rows (y1, k2), K position 2c);
//   warps 12-15   stage-2 epilogue: tensor memory -> head + tail -> FP16 -> H, either as
//                 interleaved complex values or, for the tensor-core z pass, as 32-byte
//                 segments [Re x 8 | Im x 8] per row and item (full-sector stores both).
// mbarriers hand every buffer between the roles; every wait is bounded by the plan's
// wait budget, and a wait that runs out sets the error flag, after which all roles
// leave, the MMAs in flight are waited for and the tensor memory is freed.
#include "common.cuh"
#include "tc_common.cuh"
#include "ypass_tc.cuh"

#include <cuda_fp16.h>

#include <algorithm>

namespace tmb {

namespace {

using namespace tc;

constexpr int kYThreads = 512;
constexpr int kYS1 = 4;         // stage-1 operand buffers (items whose loads are in flight)
constexpr int kYLoaders = 96;   // warps 1-3

// Operator tables, canonical K-major FP16 (head rows, then tail rows):
//   T1: 64 rows x 32 K, rows [Re Z | Im Z] x 16 outputs, K = 2a + (0: Re X, 1: Im X);
//   T2: 4Q rows x 2Q K, rows [Re Y | Im Y] x Q outputs, K = 2c + (0: Re Z', 1: Im Z').
__host__ __device__ constexpr int t1_halves() { return 64 * 32; }
__host__ __device__ constexpr int t2_halves(int Q) { return 4 * Q * 2 * Q; }

__global__ void ydft_table_kernel(uint16_t* __restrict__ T, int Q) {
  const int n1 = t1_halves(), total = n1 + t2_halves(Q);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const int R = i < n1 ? 16 : Q;            // radix of the stage
    const int K = 2 * R;
    const int idx = i < n1 ? i : i - n1;
    const int n = idx / K, k = idx - n * K;
    const int part = n / (2 * R), comp = (n / R) & 1, o = n % R;
    const int a = k >> 1, ri = k & 1;
    double sn, cs;
    sincospi(2.0 * (double)((a * o) % R) / (double)R, &sn, &cs);
    // (Re, Im) of X w^(a o): Re = Re X cos - Im X sin, Im = Re X sin + Im X cos
    const double v = comp == 0 ? (ri == 0 ? cs : -sn) : (ri == 0 ? sn : cs);
    const float vf = (float)v;
    const __half hd = __float2half_rn(vf);
    const __half tl = __float2half_rn(vf - __half2float(hd));
    const int rows = 2 * R;  // rows per part
    const int nn = comp * R + o;
    const int base = i < n1 ? 0 : n1;
    T[base + kmajor16(part * rows + nn, k, K)] = __half_as_ushort(part == 0 ? hd : tl);
  }
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" : : "r"(smem_u32(bar)) : "memory");
}
// arrival once this thread's earlier cp.async copies have landed (counted in the
// barrier's expected arrivals)
__device__ __forceinline__ void mbar_arrive_cp_async(uint64_t* bar) {
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];" : : "r"(smem_u32(bar))
               : "memory");
}
__device__ __forceinline__ void cp_async4(uint32_t smem, const void* gmem) {
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(smem), "l"(gmem));
}
__device__ __forceinline__ void tmem_ld16(uint32_t addr, float (&v)[16]) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(addr));
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ uint32_t pack_half2(float re, float im) {
  const __half2 h = __floats2half2_rn(re, im);
  return *reinterpret_cast<const uint32_t*>(&h);
}

template <int Q>
struct YLayout {
  static constexpr int N1 = 16 * Q;        // transform length
  static constexpr int R1 = 8 * Q;         // stage-1 rows (c, k2)
  static constexpr int NT1 = R1 / 128;     // stage-1 M tiles
  static constexpr int K1 = 32;            // stage-1 K: 16 complex inputs
  static constexpr int NC1 = 64;           // stage-1 N: [Re | Im] x 16, head then tail
  static constexpr int K2 = 2 * Q;         // stage-2 K: Q complex inputs
  static constexpr int NC2 = 4 * Q;        // stage-2 N: [Re | Im] x Q, head then tail
  static constexpr int A1 = R1 * K1;       // halves per stage-1 operand buffer
  static constexpr int A2 = 128 * K2;      // halves per stage-2 operand buffer
  static constexpr int EPI1 = 128 * NT1;   // stage-1 epilogue threads
  static constexpr int EPI2 = 128;
  static constexpr size_t smem_bytes() {
    return (size_t)(t1_halves() + t2_halves(Q) + kYS1 * A1 + 2 * A2) * 2 +
           (size_t)(2 * kYS1 + 9) * 8 + 16;
  }
};

template <int Q>
__global__ void __launch_bounds__(kYThreads, 1)
ypass_tc_kernel(__half2* __restrict__ H, int64_t nitems, int hp,
                const uint16_t* __restrict__ Tg, uint32_t wait_iters, int* __restrict__ err,
                int seg) {
  using L = YLayout<Q>;
  extern __shared__ __align__(128) uint16_t smem_y[];
  uint16_t* T1s = smem_y;
  uint16_t* T2s = T1s + t1_halves();
  uint16_t* A1s = T2s + t2_halves(Q);
  uint16_t* A2s = A1s + kYS1 * L::A1;
  uint64_t* bar = reinterpret_cast<uint64_t*>(A2s + 2 * L::A2);
  uint64_t* a1full = bar;              // [kYS1] item loaded (loader threads, async)
  uint64_t* a1empty = bar + kYS1;      // [kYS1] stage-1 MMAs done with the operand (commit)
  uint64_t* d1full = bar + 2 * kYS1;   // [2] stage-1 accumulators written (commit)
  uint64_t* e1done = d1full + 2;       // [2] stage-1 epilogue: D1 read, A2 written
  uint64_t* s2done = e1done + 2;       // [2] stage-2 MMAs done: A2 free, D2 written (commit)
  uint64_t* d2empty = s2done + 2;      // [2] stage-2 epilogue read D2
  uint64_t* mdone = d2empty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mdone + 1);
  volatile int* fail = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_u32(tmem_slot)), "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int s = 0; s < kYS1; ++s) {
      mbar_init(a1full + s, kYLoaders);
      mbar_init(a1empty + s, 1);
    }
    for (int p = 0; p < 2; ++p) {
      mbar_init(d1full + p, 1);
      mbar_init(e1done + p, L::EPI1);
      mbar_init(s2done + p, 1);
      mbar_init(d2empty + p, L::EPI2);
    }
    mbar_init(mdone, 1);
    asm volatile("fence.mbarrier_init.release.cluster;");
    *fail = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;
  // tensor memory: D1 (stage-1 accumulators) in columns [0, 256), two buffers of 128;
  // D2 in [256, 512), two buffers of 128
  const int64_t mine = nitems > blockIdx.x ? (nitems - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const int nc = hp / 8;  // items per (rotation, x') plane
  auto item_base = [&](int64_t j) -> int64_t {
    const int64_t id = (int64_t)blockIdx.x + j * gridDim.x;
    return (id / nc) * (int64_t)L::N1 * hp + (id % nc) * 8;
  };

  if (warp >= 1 && warp <= 3) {
    // ---------------------------------------------------------------- loaders
    const int lt = tid - 32;
    constexpr int tpieces = (t1_halves() + t2_halves(Q)) / 8;
    for (int i = lt; i < tpieces; i += kYLoaders)
      cp_async16(smem_u32(T1s) + 16u * i, Tg + 8 * (size_t)i, 16);
    // lane -> (j4 = lane >> 3, k2 = lane & 7); warp task t -> (am = t & 3, c = t >> 2),
    // a = 4 am + j4: element X[Q a + c][k2] goes to row 8c + k2, K position 2a, i.e. byte
    // 512 c + 128 am + 16 k2 + 4 j4 of the operand (32 distinct banks per warp access)
    const int wl = warp - 1, j4 = lane >> 3, k2 = lane & 7;
    for (int64_t j = 0; j < mine; ++j) {
      const int s = (int)(j % kYS1);
      const uint32_t u = (uint32_t)(j / kYS1);
      if (j >= kYS1 && !mbar_wait_n(smem_u32(a1empty + s), (u - 1) & 1u, wait_iters)) {
        *fail = 1;
        break;
      }
      if (*fail) break;
      const __half2* src0 = H + item_base(j) + k2;
      const uint32_t dst0 = smem_u32(A1s + (size_t)s * L::A1) + 16u * k2 + 4u * j4;
#pragma unroll 4
      for (int t = wl; t < 4 * Q; t += 3) {
        const int am = t & 3, c = t >> 2;
        cp_async4(dst0 + 512u * c + 128u * am, src0 + (int64_t)(Q * (4 * am + j4) + c) * hp);
      }
      mbar_arrive_cp_async(a1full + s);
    }
  } else if (warp == 0) {
    // ---------------------------------------------------------------- MMA issuer
    if (lane == 0) {
      const uint32_t id1 = idesc_f16(128, L::NC1), id2 = idesc_f16(128, L::NC2);
      const uint32_t t1 = smem_u32(T1s), t2 = smem_u32(T2s);
      const uint32_t a1 = smem_u32(A1s), a2 = smem_u32(A2s);
      bool ok = true;
      for (int64_t j = 0; j <= mine && ok; ++j) {
        if (j < mine) {
          // stage 1 of item j into D1[j & 1]
          const int s = (int)(j % kYS1), p = (int)(j & 1);
          const uint32_t u = (uint32_t)(j / kYS1);
          if (!mbar_wait_n(smem_u32(a1full + s), u & 1u, wait_iters)) { ok = false; break; }
          if (j >= 2 &&
              !mbar_wait_n(smem_u32(e1done + p), (uint32_t)((j - 2) >> 1) & 1u, wait_iters)) {
            ok = false;
            break;
          }
          if (*fail) { ok = false; break; }
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          asm volatile("tcgen05.fence::after_thread_sync;");
          const uint32_t ab = a1 + (uint32_t)s * (uint32_t)L::A1 * 2u;
#pragma unroll
          for (int m = 0; m < L::NT1; ++m)
#pragma unroll
            for (int st = 0; st < L::K1 / 16; ++st)
              mma_f16(tmem + (uint32_t)(p * 128 + m * 64),
                      smem_desc(ab + (uint32_t)(m * 128 * L::K1 * 2 + st * 256), 128u,
                                (uint32_t)L::K1 * 16u),
                      smem_desc(t1 + (uint32_t)(st * 256), 128u, (uint32_t)L::K1 * 16u), id1,
                      st > 0);
          mma_commit(smem_u32(a1empty + s));
          mma_commit(smem_u32(d1full + p));
        }
        if (j >= 1) {
          // stage 2 of item j - 1 into D2[(j - 1) & 1]
          const int64_t jj = j - 1;
          const int p = (int)(jj & 1);
          if (!mbar_wait_n(smem_u32(e1done + p), (uint32_t)(jj >> 1) & 1u, wait_iters)) {
            ok = false;
            break;
          }
          if (jj >= 2 &&
              !mbar_wait_n(smem_u32(d2empty + p), (uint32_t)((jj - 2) >> 1) & 1u, wait_iters)) {
            ok = false;
            break;
          }
          if (*fail) { ok = false; break; }
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          asm volatile("tcgen05.fence::after_thread_sync;");
          const uint32_t ab = a2 + (uint32_t)p * (uint32_t)L::A2 * 2u;
#pragma unroll
          for (int st = 0; st < L::K2 / 16; ++st)
            mma_f16(tmem + 256u + (uint32_t)(p * 128),
                    smem_desc(ab + (uint32_t)(st * 256), 128u, (uint32_t)L::K2 * 16u),
                    smem_desc(t2 + (uint32_t)(st * 256), 128u, (uint32_t)L::K2 * 16u), id2,
                    st > 0);
          mma_commit(smem_u32(s2done + p));
        }
      }
      if (!ok) *fail = 1;
      // nothing may free tensor memory or shared memory under a running MMA: this wait
      // keeps the full default budget whatever the plan's wait budget is
      mma_commit(smem_u32(mdone));
      if (!mbar_wait(smem_u32(mdone), 0u)) *fail = 1;
    }
  } else if (warp < 4 + 4 * L::NT1) {
    // ---------------------------------------------------------------- stage-1 epilogue
    const int m = (warp - 4) >> 2, q = warp & 3;
    const int c = 16 * m + 4 * q + (lane >> 3), k2 = lane & 7;
    float wr[16], wi[16];
#pragma unroll
    for (int y1 = 0; y1 < 16; ++y1) sincospif(2.0f * (float)(c * y1) / (float)L::N1, &wi[y1], &wr[y1]);
    const uint32_t tl = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(m * 64);
    // row (y1, k2), K position 2c of the stage-2 operand: byte
    // y1 * 32Q + 128 (c >> 2) + 16 k2 + 4 (c & 3)
    const uint32_t a2t = smem_u32(A2s) + 128u * (uint32_t)(c >> 2) + 16u * (uint32_t)k2 +
                         4u * (uint32_t)(c & 3);
    for (int64_t j = 0; j < mine; ++j) {
      const int p = (int)(j & 1);
      const uint32_t u = (uint32_t)(j >> 1);
      bool got = mbar_wait_n(smem_u32(d1full + p), u & 1u, wait_iters);
      if (got && j >= 2) got = mbar_wait_n(smem_u32(s2done + p), (u - 1) & 1u, wait_iters);
      __syncwarp();
      if (!__all_sync(0xffffffffu, got)) { *fail = 1; break; }
      if (__any_sync(0xffffffffu, *fail)) break;
      asm volatile("tcgen05.fence::after_thread_sync;");
      float re[16], im[16];
      {
        float hr[16], hi[16];
        tmem_ld16(tl + (uint32_t)(p * 128), hr);
        tmem_ld16(tl + (uint32_t)(p * 128 + 32), re);
        tmem_ld16(tl + (uint32_t)(p * 128 + 16), hi);
        tmem_ld16(tl + (uint32_t)(p * 128 + 48), im);
        asm volatile("tcgen05.wait::ld.sync.aligned;");
#pragma unroll
        for (int y1 = 0; y1 < 16; ++y1) {
          re[y1] += hr[y1];
          im[y1] += hi[y1];
        }
      }
      const uint32_t dst = a2t + (uint32_t)p * (uint32_t)L::A2 * 2u;
#pragma unroll
      for (int y1 = 0; y1 < 16; ++y1) {
        const float orr = re[y1] * wr[y1] - im[y1] * wi[y1];
        const float oi = re[y1] * wi[y1] + im[y1] * wr[y1];
        asm volatile("st.shared.b32 [%0], %1;" ::"r"(dst + (uint32_t)(y1 * 32 * Q)),
                     "r"(pack_half2(orr, oi))
                     : "memory");
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;");
      mbar_arrive(e1done + p);
    }
  } else if (warp >= 12) {
    // ---------------------------------------------------------------- stage-2 epilogue
    const int q = warp & 3;
    const int y1 = 4 * q + (lane >> 3), k2 = lane & 7;
    const uint32_t tl = tmem + ((uint32_t)(q * 32) << 16) + 256u;
    // segment layout: word k2 of a row's 32-byte segment is (Re, Re) of columns 2k2, 2k2+1
    // for k2 < 4 and (Im, Im) of columns 2(k2-4), 2(k2-4)+1 otherwise, gathered from the
    // lanes of the same row
    const int srcA = (lane & ~7) | ((2 * k2) & 7);
    const uint32_t sel = k2 < 4 ? 0x5410u : 0x7632u;
    for (int64_t j = 0; j < mine; ++j) {
      const int p = (int)(j & 1);
      const uint32_t u = (uint32_t)(j >> 1);
      const bool got = mbar_wait_n(smem_u32(s2done + p), u & 1u, wait_iters);
      __syncwarp();
      if (!__all_sync(0xffffffffu, got)) { *fail = 1; break; }
      if (__any_sync(0xffffffffu, *fail)) break;
      asm volatile("tcgen05.fence::after_thread_sync;");
      __half2* dst = H + item_base(j) + k2 + (int64_t)y1 * hp;
      const uint32_t tb = tl + (uint32_t)(p * 128);
      // D2 columns [Re head | Im head | Re tail | Im tail], Q each
#pragma unroll
      for (int g = 0; g < Q / 16; ++g) {
        float re[16], im[16], tr[16], ti[16];
        tmem_ld16(tb + (uint32_t)(g * 16), re);
        tmem_ld16(tb + (uint32_t)(Q + g * 16), im);
        tmem_ld16(tb + (uint32_t)(2 * Q + g * 16), tr);
        tmem_ld16(tb + (uint32_t)(3 * Q + g * 16), ti);
        asm volatile("tcgen05.wait::ld.sync.aligned;");
        if (g == Q / 16 - 1) {
          asm volatile("tcgen05.fence::before_thread_sync;");
          mbar_arrive(d2empty + p);
        }
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const int y2 = g * 16 + i;
          uint32_t v = pack_half2(re[i] + tr[i], im[i] + ti[i]);
          if (seg) {
            const uint32_t a = __shfl_sync(0xffffffffu, v, srcA);
            const uint32_t b = __shfl_sync(0xffffffffu, v, srcA + 1);
            v = __byte_perm(a, b, sel);
          }
          *reinterpret_cast<uint32_t*>(dst + (int64_t)(16 * y2) * hp) = v;
        }
      }
    }
  }
  asm volatile("cp.async.wait_all;\n" ::);
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == 0) {
    __syncwarp();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" : : "r"(tmem), "r"(512));
  }
  if (tid == 0 && *fail) atomicExch(err, 1);
}

template <int Q>
int set_attrs(int optin) {
  return cuda_status(cudaFuncSetAttribute(ypass_tc_kernel<Q>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, optin),
                     "ypass_tc: shared memory attribute");
}

}  // namespace

int ypass_tc_config(int n1, int hp, YpassTcConfig* cfg) {
  cfg->ok = false;
  cfg->n1 = n1;
  cfg->Q = n1 / 16;
  if ((n1 != 256 && n1 != 512) || hp % 8 != 0 || hp <= 0) return TM_OK;
  int dev = 0, optin = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaGetLastError();
  cfg->sms = sms;
  cfg->smem = cfg->Q == 32 ? YLayout<32>::smem_bytes() : YLayout<16>::smem_bytes();
  if (cfg->smem > (size_t)optin) return TM_OK;
  TM_TRY(cfg->Q == 32 ? set_attrs<32>(optin) : set_attrs<16>(optin));
  cfg->ok = true;
  return TM_OK;
}

size_t ypass_tc_table_bytes(const YpassTcConfig& cfg) {
  return (size_t)(t1_halves() + t2_halves(cfg.Q)) * 2;
}

int ypass_tc_prepare(const YpassTcConfig& cfg, uint16_t* table, cudaStream_t stream) {
  TM_REQUIRE(cfg.ok && table, "ypass_tc_prepare: unsupported configuration");
  ydft_table_kernel<<<32, 256, 0, stream>>>(table, cfg.Q);
  return check_launch("ydft_table_kernel");
}

int ypass_tc_run(const YpassTcConfig& cfg, void* H, int nb, int n0, int hp,
                 const uint16_t* table, uint32_t wait_iters, int* err, cudaStream_t stream,
                 bool seg) {
  TM_REQUIRE(cfg.ok, "ypass_tc_run: unsupported configuration");
  TM_REQUIRE(H && table && err && nb >= 1 && n0 >= 1 && hp % 8 == 0,
             "ypass_tc_run: bad arguments");
  const int64_t nitems = (int64_t)nb * n0 * (hp / 8);
  const int grid = (int)std::min<int64_t>(nitems, cfg.sms);
  if (cfg.Q == 32)
    ypass_tc_kernel<32><<<grid, kYThreads, cfg.smem, stream>>>(
        static_cast<__half2*>(H), nitems, hp, table, wait_iters, err, seg ? 1 : 0);
  else
    ypass_tc_kernel<16><<<grid, kYThreads, cfg.smem, stream>>>(
        static_cast<__half2*>(H), nitems, hp, table, wait_iters, err, seg ? 1 : 0);
  return check_launch("ypass_tc_kernel");
}

}  // namespace tmb
