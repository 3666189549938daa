// y pass of the fused CC / FLCSphericalMask scan with its long stage on the tensor cores.
//
// For every rotation, x' plane and k2 column of the half-precision intermediate spectra
// H[b][x'][k1][k2] (row pitch hp), the unnormalised inverse DFT along y,
//     Y[y'] = sum_{k1 < n1} X[k1] w^(k1 y'),   w = exp(+2 pi i / n1),  n1 = 16 Q,
// runs in two stages with k1 = Q a + c and y' = y1 + 16 y2 (a, y1 < 16; c, y2 < Q):
//     Z[y1][c]      = sum_{a < 16} X[Q a + c] w16^(a y1)       (radix 16, CUDA cores)
//     Z'[y1][c]     = Z[y1][c] w^(c y1)                        (twiddle, CUDA cores)
//     Y[y1 + 16 y2] = sum_{c < Q} Z'[y1][c] wQ^(c y2)          (radix Q, tensor cores)
// The radix-16 stage is a 4 x 4 register FFT in FP32 per (c, k2) column; the radix-Q stage
// is a real GEMM over interleaved (Re, Im) K positions: rows (y1, k2) of Z' are the M
// operand, a fixed DFT operator the N operand (output columns [Re | Im]). Both enter as an
// FP16 head plus its FP16 rounded remainder (the tail), and three MMAs per K step
// accumulate Zh Th + Zt Th + Zh Tt in one FP32 accumulator (about 22 significant bits),
// so the only rounding of the pass is that of its FP16 output, as in the FFT y pass.
//
// A work item is one rotation, one x' plane and 8 consecutive k2 columns: n1 rows of
// 32 bytes, read and written in place. The rows of an item move between H and shared
// memory as tiles of the tensor memory accelerator (TMA): H is a 2D tensor of 4-byte
// words (hp columns, nb n0 n1 rows) and an item is n1 / 256 boxes of 8 x 256 words, so
// no thread issues per-row loads or stores. Roles of the persistent 512-thread CTA:
//   warp 0         one thread issues the stage-2 MMAs;
//   warp 1         one thread issues the TMA loads of the items (kYS in flight) and the
//                  bulk copy of the operator;
//   warp 2         one thread issues the TMA stores of the finished items;
//   warps 4-11     stage 1: one thread per (c, k2) column reads its 16 values from the
//                  staging buffer (bank-conflict-free), runs the radix-16 FFT and the
//                  twiddle, and writes Z' (head and tail) into the stage-2 operand;
//   warps 12-15    stage-2 epilogue: tensor memory -> FP16 -> an output staging buffer
//                  holding the item's rows, either as interleaved complex values or, for
//                  the tensor-core z pass, as 32-byte segments [Re x 8 | Im x 8].
// mbarriers hand every buffer between the roles; every wait is bounded by the plan's
// wait budget, and a wait that runs out sets the error flag, after which all roles
// leave, the copies and MMAs in flight are waited for and the tensor memory is freed.
// No load here uses cluster multicast.
#include "common.cuh"
#include "fft_smem.cuh"
#include "tc_common.cuh"
#include "ypass_tc.cuh"

#include "tma.cuh"

#include <cuda_fp16.h>

#include <algorithm>

namespace tmb {

namespace {

using namespace tc;

constexpr int kYThreads = 512;
// Buffer counts of the pipeline. Deeper rings (3 operand and 4 accumulator buffers, or 3
// output staging buffers) measured no faster.
constexpr int kYS = 4;          // input staging buffers (items whose loads are in flight)
constexpr int kNA = 2;          // stage-2 operand buffers
constexpr int kND = 2;          // stage-2 accumulator buffers in tensor memory
constexpr int kNE = 2;          // output staging buffers
constexpr int kBoxRows = 256;   // rows per TMA box (the box-dimension limit)

// Stage-2 operator, canonical K-major FP16, two tables (the FP16 head, then the FP16
// rounded remainder) of 2Q rows [Re Y | Im Y] x Q outputs by 2Q K positions
// 2c + (0: Re Z', 1: Im Z').
__host__ __device__ constexpr int t2_halves(int Q) { return 2 * (2 * Q) * (2 * Q); }

__global__ void ydft_table_kernel(uint16_t* __restrict__ T, int Q) {
  const int K = 2 * Q, total = t2_halves(Q);
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const int part = i / (K * K), e = i - part * K * K;
    const int n = e / K, k = e - n * K;
    const int comp = n / Q, o = n % Q;
    const int c = k >> 1, ri = k & 1;
    double sn, cs;
    sincospi(2.0 * (double)((c * o) % Q) / (double)Q, &sn, &cs);
    // (Re, Im) of Z' wQ^(c o): Re = Re Z' cos - Im Z' sin, Im = Re Z' sin + Im Z' cos
    const double v = comp == 0 ? (ri == 0 ? cs : -sn) : (ri == 0 ? sn : cs);
    const float vf = (float)v;
    const __half hd = __float2half_rn(vf);
    const __half tl = __float2half_rn(vf - __half2float(hd));
    T[part * K * K + kmajor16(n, k, K)] = __half_as_ushort(part == 0 ? hd : tl);
  }
}

// Stage-1 operator (radix 16 on the tensor cores), canonical K-major FP16, two tables (head,
// then the FP16 rounded remainder) of 32 rows [Re Z | Im Z] x 16 outputs y1 by 32 K
// positions 2a + (0: Re X, 1: Im X): the inverse DFT w16^(a y1).
constexpr int kF1Halves = 2 * 32 * 32;

__global__ void ydft16_table_kernel(uint16_t* __restrict__ T) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kF1Halves; i += gridDim.x * blockDim.x) {
    const int part = i / 1024, e = i - part * 1024;
    const int n = e / 32, k = e - n * 32;
    const int comp = n / 16, y1 = n % 16;
    const int a = k >> 1, ri = k & 1;
    double sn, cs;
    sincospi(2.0 * (double)((a * y1) % 16) / 16.0, &sn, &cs);
    const double v = comp == 0 ? (ri == 0 ? cs : -sn) : (ri == 0 ? sn : cs);
    const float vf = (float)v;
    const __half hd = __float2half_rn(vf);
    const __half tl = __float2half_rn(vf - __half2float(hd));
    T[part * 1024 + kmajor16(n, k, 32)] = __half_as_ushort(part == 0 ? hd : tl);
  }
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" : : "r"(smem_u32(bar)) : "memory");
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
// v * w16^k, w16 = exp(+2 pi i / 16), for the products k = a0 y0 (a0, y0 < 4) of the
// radix-16 stage, with the twiddles as constants: cos(pi/8), sin(pi/8), sqrt(1/2).
__device__ __forceinline__ float2 tw16(float2 v, int k) {
  constexpr float c8 = 0.923879532511286756f, s8 = 0.382683432365089772f;
  constexpr float r2 = 0.707106781186547524f;
  switch (k) {
    case 0: return v;
    case 1: return make_float2(v.x * c8 - v.y * s8, v.x * s8 + v.y * c8);
    case 2: return make_float2((v.x - v.y) * r2, (v.x + v.y) * r2);
    case 3: return make_float2(v.x * s8 - v.y * c8, v.x * c8 + v.y * s8);
    case 4: return make_float2(-v.y, v.x);
    case 6: return make_float2(-(v.x + v.y) * r2, (v.x - v.y) * r2);
    default: return make_float2(-v.x * c8 + v.y * s8, -v.x * s8 - v.y * c8);  // 9
  }
}

__device__ __forceinline__ uint32_t pack_half2(float re, float im) {
  const __half2 h = __floats2half2_rn(re, im);
  return *reinterpret_cast<const uint32_t*>(&h);
}

template <int Q>
struct YLayout {
  static constexpr int N1 = 16 * Q;        // transform length
  static constexpr int K2 = 4 * Q;         // stage-2 operand K: Z' head (2Q), Z' tail (2Q)
  static constexpr int KT = 2 * Q;         // operator K: Q complex inputs
  static constexpr int NC2 = 2 * Q;        // stage-2 N: [Re | Im] x Q
  static constexpr int S = N1 * 16;        // halves per item buffer (n1 rows of 32 B)
  static constexpr int A2 = 128 * K2;      // halves per stage-2 operand buffer
  static constexpr int EPI1 = 8 * Q;       // stage-1 threads: one per (c, k2)
  static constexpr int EPI2 = 128;
  static constexpr int NBOX = N1 / kBoxRows;  // TMA boxes per item
  static constexpr uint32_t ITEM_BYTES = (uint32_t)N1 * 32u;
  static constexpr int NBAR = 2 * (kYS + kNA + kND + kNE) + 2 + 4;  // + d1full, d1empty
  // tensor-memory columns: kND accumulators of NC2 columns, allocated as a power of two
  // with stage 1 on the tensor cores, two more buffers of Q/16 tiles x 32 columns (D1)
  static constexpr int D1COLS = (Q / 16) * 32;
  static constexpr int TCOLS = kND * NC2 + 2 * D1COLS;
  static constexpr uint32_t TMEM = TCOLS <= 32 ? 32u : TCOLS <= 64 ? 64u
                                 : TCOLS <= 128 ? 128u : TCOLS <= 256 ? 256u : 512u;
  static constexpr size_t smem_bytes() {
    return (size_t)(t2_halves(Q) + kF1Halves + kYS * S + kNA * A2 + kNE * S) * 2 +
           (size_t)NBAR * 8 + 16;
  }
};
static_assert(YLayout<16>::N1 % kBoxRows == 0 && YLayout<32>::N1 % kBoxRows == 0,
              "items are whole TMA boxes");
static_assert(YLayout<32>::TCOLS <= 512, "accumulators fit in tensor memory");

// Shared-memory descriptor strides of the stage-1 X operand, which is M-major (8 k2 values
// of one row half per 16 bytes): M groups (one c each) 512 bytes apart, K groups (four
// rows a) 128 bytes apart. As for K-major operands, the descriptor's leading-dimension
// offset is the stride between core matrices along K and the stride-dimension offset the
// stride along M (checked against a known product on a B200).
constexpr uint32_t kS1MStride = 512, kS1KStride = 128;

template <int Q, bool S1>
__global__ void __launch_bounds__(kYThreads, 1)
ypass_tc_kernel(const __grid_constant__ CUtensorMap lmap, const __grid_constant__ CUtensorMap smap,
                int64_t nitems, int nc, int n0, int h2, const uint16_t* __restrict__ Tg,
                uint32_t wait_iters, int* __restrict__ err, int seg, int xin) {
  using L = YLayout<Q>;
  extern __shared__ __align__(1024) uint16_t smem_y[];
  uint16_t* T2s = smem_y;
  uint16_t* F1s = T2s + t2_halves(Q);               // stage-1 operator (S1)
  uint16_t* Ss = F1s + kF1Halves;                   // kYS input staging buffers
  uint16_t* A2s = Ss + kYS * L::S;                  // kNA stage-2 operand buffers
  uint16_t* Es = A2s + kNA * L::A2;                 // kNE output staging buffers
  uint64_t* bar = reinterpret_cast<uint64_t*>(Es + kNE * L::S);
  uint64_t* sfull = bar;               // [kYS] item landed (loader arrival + TMA bytes)
  uint64_t* sempty = bar + kYS;        // [kYS] stage 1 read the item (stage-1 threads)
  uint64_t* e1done = bar + 2 * kYS;    // [kNA] stage 1 wrote the operand (stage-1 threads)
  uint64_t* a2free = e1done + kNA;     // [kNA] the MMAs that read the operand are done
  uint64_t* d2full = a2free + kNA;     // [kND] the MMAs that write the accumulator are done
  uint64_t* d2empty = d2full + kND;    // [kND] stage-2 epilogue read the accumulator
  uint64_t* estaged = d2empty + kND;   // [kNE] output rows staged (epilogue threads)
  uint64_t* efree = estaged + kNE;     // [kNE] TMA stores finished reading the staging
  uint64_t* tfull = efree + kNE;       // the operator landed (loader arrival + bytes)
  uint64_t* mdone = tfull + 1;
  uint64_t* d1full = mdone + 1;        // [2] stage-1 MMAs done (S1; commit)
  uint64_t* d1empty = d1full + 2;      // [2] stage-1 accumulators read (S1; stage-1 threads)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(d1empty + 2);
  volatile int* fail = reinterpret_cast<volatile int*>(tmem_slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_u32(tmem_slot)), "r"(L::TMEM));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int s = 0; s < kYS; ++s) {
      mbar_init(sfull + s, 1);
      mbar_init(sempty + s, S1 ? 1 : L::EPI1);
    }
    for (int p = 0; p < kNA; ++p) {
      mbar_init(e1done + p, L::EPI1);
      mbar_init(a2free + p, 1);
    }
    for (int p = 0; p < kND; ++p) {
      mbar_init(d2full + p, 1);
      mbar_init(d2empty + p, L::EPI2);
    }
    for (int p = 0; p < kNE; ++p) {
      mbar_init(estaged + p, L::EPI2);
      mbar_init(efree + p, 1);
    }
    mbar_init(tfull, 1);
    mbar_init(mdone, 1);
    for (int p = 0; p < 2; ++p) {
      mbar_init(d1full + p, 1);
      mbar_init(d1empty + p, L::EPI1);
    }
    asm volatile("fence.mbarrier_init.release.cluster;");
    *fail = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;
  // tensor memory: D2 (stage-2 accumulators) in kND buffers of NC2 columns
  const int64_t mine = nitems > blockIdx.x ? (nitems - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  // item id -> (tensor row of its first row, tensor column of its first word)
  auto item_xy = [&](int64_t j, int& x, int& y) {
    const int64_t id = (int64_t)blockIdx.x + j * gridDim.x;
    x = (int)(id % nc) * 8;
    y = (int)(id / nc) * L::N1;
  };

  if (warp == 1) {
    // ---------------------------------------------------------------- TMA loader
    if (lane == 0) {
      tma::arrive_expect_tx(tfull, (uint32_t)(t2_halves(Q) + kF1Halves) * 2u);
      tma::bulk_load(smem_u32(T2s), Tg, (uint32_t)(t2_halves(Q) + kF1Halves) * 2u, tfull);
      int64_t issued = 0;
      for (int64_t j = 0; j < mine; ++j) {
        const int s = (int)(j % kYS);
        if (j >= kYS &&
            !mbar_wait_s(smem_u32(sempty + s), (uint32_t)(j / kYS - 1) & 1u, wait_iters)) {
          *fail = 1;
          break;
        }
        if (*fail) break;
        int x, y;
        item_xy(j, x, y);
        const uint32_t dst = smem_u32(Ss + (size_t)s * L::S);
        tma::arrive_expect_tx(sfull + s, L::ITEM_BYTES);
        if (xin) {
          // x'-inner input [b][k1][k2 / 8][x'][8]: the item's rows are the k1 of segment
          // x / 8 of plane (b, x')
          const int plane = y / L::N1, xp = plane % n0, z0 = (plane / n0) * L::N1;
#pragma unroll
          for (int b = 0; b < L::NBOX; ++b)
            tma::load_4d(dst + (uint32_t)(b * kBoxRows * 32), &lmap, 0, xp, x >> 3,
                         z0 + b * kBoxRows, sfull + s);
        } else {
#pragma unroll
          for (int b = 0; b < L::NBOX; ++b)
            tma::load_2d(dst + (uint32_t)(b * kBoxRows * 32), &lmap, x, y + b * kBoxRows,
                         sfull + s);
        }
        issued = j + 1;
      }
      // nothing may leave while a load still writes into shared memory: wait (with the
      // full default budget) for the loads of every item stage 1 did not consume
      for (int64_t j = issued > kYS ? issued - kYS : 0; j < issued; ++j)
        mbar_wait(smem_u32(sfull + (int)(j % kYS)), (uint32_t)(j / kYS) & 1u);
      mbar_wait(smem_u32(tfull), 0u);
    }
  } else if (warp == 2) {
    // ---------------------------------------------------------------- TMA storer
    if (lane == 0) {
      for (int64_t j = 0; j < mine; ++j) {
        const int p = (int)(j % kNE);
        if (!mbar_wait_s(smem_u32(estaged + p), (uint32_t)(j / kNE) & 1u, wait_iters)) {
          *fail = 1;
          break;
        }
        if (*fail) break;
        int x, y;
        item_xy(j, x, y);
        const uint32_t src = smem_u32(Es + (size_t)p * L::S);
#pragma unroll
        for (int b = 0; b < L::NBOX; ++b)
          tma::store_2d(&smap, x, y + b * kBoxRows, src + (uint32_t)(b * kBoxRows * 32));
        asm volatile("cp.async.bulk.commit_group;" ::: "memory");
        // the staging buffer is free once the stores have read it
        asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
        mbar_arrive(efree + p);
      }
      asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
    }
  } else if (warp == 0) {
    // ---------------------------------------------------------------- MMA issuer
    if (lane == 0) {
      const uint32_t id2 = idesc_f16(128, L::NC2);
      const uint32_t id1 = idesc_f16(128, 32) | (1u << 15);  // stage 1: X is M-major
      const uint32_t t2 = smem_u32(T2s), a2 = smem_u32(A2s), f1 = smem_u32(F1s);
      const uint32_t d1base = tmem + (uint32_t)(kND * L::NC2);
      // stage 1 of item j (S1): X (staging, rows (c, a)) times the radix-16 operator
      auto stage1 = [&](int64_t j) -> bool {
        const int s = (int)(j % kYS), p1 = (int)(j & 1);
        if (!mbar_wait_n(smem_u32(sfull + s), (uint32_t)(j / kYS) & 1u, wait_iters)) return false;
        if (j >= 2 &&
            !mbar_wait_n(smem_u32(d1empty + p1), (uint32_t)((j - 2) >> 1) & 1u, wait_iters))
          return false;
        if (*fail) return false;
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t xs = smem_u32(Ss + (size_t)s * L::S);
#pragma unroll
        for (int tt = 0; tt < Q / 16; ++tt) {
          const uint32_t d1 = d1base + (uint32_t)(p1 * L::D1COLS + tt * 32);
#pragma unroll
          for (int st = 0; st < 2; ++st) {
            const uint64_t xd = smem_desc(xs + (uint32_t)(tt * 16 * 512 + st * 256), kS1KStride,
                                          kS1MStride);
            const uint64_t fh = smem_desc(f1 + (uint32_t)(st * 256), 128u, 512u);
            const uint64_t ft = smem_desc(f1 + 2048u + (uint32_t)(st * 256), 128u, 512u);
            mma_f16(d1, xd, fh, id1, st > 0);
            mma_f16(d1, xd, ft, id1, 1);
          }
        }
        mma_commit(smem_u32(d1full + p1));
        mma_commit(smem_u32(sempty + s));  // the staging buffer is free once read
        return true;
      };
      // stage 2 of item j: Z' (operand buffer) times the radix-Q operator
      auto stage2 = [&](int64_t j) -> bool {
        const int pa = (int)(j % kNA), pd = (int)(j % kND);
        if (!mbar_wait_n(smem_u32(e1done + pa), (uint32_t)(j / kNA) & 1u, wait_iters))
          return false;
        if (j >= kND &&
            !mbar_wait_n(smem_u32(d2empty + pd), (uint32_t)(j / kND - 1) & 1u, wait_iters))
          return false;
        if (*fail) return false;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t ab = a2 + (uint32_t)pa * (uint32_t)L::A2 * 2u;
        const uint32_t dt = tmem + (uint32_t)(pd * L::NC2);
        // D = Zh Th + Zt Th + Zh Tt, K step by K step (16 positions, 256 bytes)
#pragma unroll
        for (int st = 0; st < L::KT / 16; ++st) {
          const uint64_t zh = smem_desc(ab + (uint32_t)(st * 256), 128u, (uint32_t)L::K2 * 16u);
          const uint64_t zt = smem_desc(ab + (uint32_t)((L::KT / 16 + st) * 256), 128u,
                                        (uint32_t)L::K2 * 16u);
          const uint64_t th = smem_desc(t2 + (uint32_t)(st * 256), 128u, (uint32_t)L::KT * 16u);
          const uint64_t tt = smem_desc(t2 + (uint32_t)(L::KT * L::KT * 2 + st * 256), 128u,
                                        (uint32_t)L::KT * 16u);
          mma_f16(dt, zh, th, id2, st > 0);
          mma_f16(dt, zt, th, id2, 1);
          mma_f16(dt, zh, tt, id2, 1);
        }
        mma_commit(smem_u32(a2free + pa));
        mma_commit(smem_u32(d2full + pd));
        return true;
      };
      bool ok = mbar_wait_n(smem_u32(tfull), 0u, wait_iters);
      if constexpr (S1) {
        // stage 1 of item j runs ahead of stage 2 of item j - 1
        for (int64_t j = 0; j <= mine && ok; ++j) {
          if (j < mine) ok = stage1(j);
          if (ok && j >= 1) ok = stage2(j - 1);
        }
      } else {
        for (int64_t j = 0; j < mine && ok; ++j) ok = stage2(j);
      }
      if (!ok) *fail = 1;
      // nothing may free tensor memory or shared memory under a running MMA: this wait
      // keeps the full default budget whatever the plan's wait budget is
      mma_commit(smem_u32(mdone));
      if (!mbar_wait(smem_u32(mdone), 0u)) *fail = 1;
    }
  } else if (warp >= 4 && warp < 4 + L::EPI1 / 32) {
    // ---------------------------------------------------------------- stage 1
    if constexpr (S1) {
      // radix 16 came from the tensor cores: read Z[y1] of this (c, k2) row from tensor
      // memory, apply the twiddle w^(c y1) and write Z' (head and tail) as below
      const int t = tid - 128;
      const int c = t >> 3, k2 = t & 7;
      float wr[16], wi[16];
#pragma unroll
      for (int y1 = 0; y1 < 16; ++y1)
        sincospif(2.0f * (float)(c * y1) / (float)L::N1, &wi[y1], &wr[y1]);
      const uint32_t a2t = smem_u32(A2s) + 128u * (uint32_t)(c >> 2) + 16u * (uint32_t)k2 +
                           4u * (uint32_t)(c & 3);
      // lanes 32 q .. 32 q + 31 of tile (warp - 4) / 4: rows (c mod 16, k2)
      const uint32_t tl1 = tmem + ((uint32_t)((warp & 3) * 32) << 16) +
                           (uint32_t)(kND * L::NC2 + ((warp - 4) >> 2) * 32);
      for (int64_t j = 0; j < mine; ++j) {
        const int p1 = (int)(j & 1), pa = (int)(j % kNA);
        const bool got = mbar_wait_n(smem_u32(d1full + p1), (uint32_t)(j >> 1) & 1u, wait_iters);
        __syncwarp();  // tcgen05.ld needs the whole warp, converged
        if (!__all_sync(0xffffffffu, got)) { *fail = 1; break; }
        if (__any_sync(0xffffffffu, *fail)) break;
        asm volatile("tcgen05.fence::after_thread_sync;");
        float re[16], im[16];
        tmem_ld16(tl1 + (uint32_t)(p1 * L::D1COLS), re);
        tmem_ld16(tl1 + (uint32_t)(p1 * L::D1COLS + 16), im);
        asm volatile("tcgen05.wait::ld.sync.aligned;");
        asm volatile("tcgen05.fence::before_thread_sync;");
        mbar_arrive(d1empty + p1);
        if (j >= kNA && !mbar_wait_n(smem_u32(a2free + pa), (uint32_t)(j / kNA - 1) & 1u,
                                     wait_iters)) {
          *fail = 1;
          break;
        }
        const uint32_t dst = a2t + (uint32_t)pa * (uint32_t)L::A2 * 2u;
#pragma unroll
        for (int y1 = 0; y1 < 16; ++y1) {
          const float orr = re[y1] * wr[y1] - im[y1] * wi[y1];
          const float oi = re[y1] * wi[y1] + im[y1] * wr[y1];
          const __half2 hd = __floats2half2_rn(orr, oi);
          const float2 hf = __half22float2(hd);
          const uint32_t head = *reinterpret_cast<const uint32_t*>(&hd);
          asm volatile("st.shared.b32 [%0], %1;" ::"r"(dst + (uint32_t)(y1 * 64 * Q)), "r"(head)
                       : "memory");
          asm volatile("st.shared.b32 [%0], %1;" ::"r"(dst + (uint32_t)(y1 * 64 * Q + 32 * Q)),
                       "r"(pack_half2(orr - hf.x, oi - hf.y))
                       : "memory");
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive(e1done + pa);
      }
    } else {
    const int t = tid - 128;
    const int c = t >> 3, k2 = t & 7;
    // twiddles w^(c y1) of the column and w16^k, k <= 9, of the radix-16 FFT
    float wr[16], wi[16];
#pragma unroll
    for (int y1 = 0; y1 < 16; ++y1)
      sincospif(2.0f * (float)(c * y1) / (float)L::N1, &wi[y1], &wr[y1]);
#pragma unroll
    // staging: X[k1][k2] at byte 32 k1 + 4 k2 (banks 8c + k2: conflict-free per warp);
    // operand: row (y1, k2), K position 2c (head) at byte
    // y1 * 64Q + 128 (c >> 2) + 16 k2 + 4 (c & 3), the tail 32Q bytes further
    const uint32_t src0 = 32u * (uint32_t)c + 4u * (uint32_t)k2;
    const uint32_t a2t = smem_u32(A2s) + 128u * (uint32_t)(c >> 2) + 16u * (uint32_t)k2 +
                         4u * (uint32_t)(c & 3);
    for (int64_t j = 0; j < mine; ++j) {
      const int s = (int)(j % kYS), pa = (int)(j % kNA);
      if (!mbar_wait_n(smem_u32(sfull + s), (uint32_t)(j / kYS) & 1u, wait_iters)) {
        *fail = 1;
        break;
      }
      if (*fail) break;
      float2 x[16];
      const uint32_t sb = smem_u32(Ss + (size_t)s * L::S) + src0;
#pragma unroll
      for (int a = 0; a < 16; ++a) {
        uint32_t w;
        asm volatile("ld.shared.b32 %0, [%1];" : "=r"(w) : "r"(sb + (uint32_t)(a * 32 * Q)));
        x[a] = __half22float2(*reinterpret_cast<const __half2*>(&w));
      }
      mbar_arrive(sempty + s);
      // radix 16 = 4 x 4: DFT4 over a1 (a = 4 a1 + a0), twiddle w16^(a0 y0), DFT4 over a0;
      // Z[y0 + 4 y1] ends in v[y0][y1]
      float2 v[4][4];
#pragma unroll
      for (int a0 = 0; a0 < 4; ++a0) {
        float2 u[4] = {x[a0], x[a0 + 4], x[a0 + 8], x[a0 + 12]};
        fft::dft4<1>(u);
#pragma unroll
        for (int y0 = 0; y0 < 4; ++y0) {
          const int k = a0 * y0;
          v[y0][a0] = tw16(u[y0], k);
        }
      }
#pragma unroll
      for (int y0 = 0; y0 < 4; ++y0) fft::dft4<1>(v[y0]);
      if (j >= kNA && !mbar_wait_n(smem_u32(a2free + pa), (uint32_t)(j / kNA - 1) & 1u,
                                   wait_iters)) {
        *fail = 1;
        break;
      }
      const uint32_t dst = a2t + (uint32_t)pa * (uint32_t)L::A2 * 2u;
#pragma unroll
      for (int y1 = 0; y1 < 16; ++y1) {
        const float2 z = v[y1 & 3][y1 >> 2];
        const float orr = z.x * wr[y1] - z.y * wi[y1];
        const float oi = z.x * wi[y1] + z.y * wr[y1];
        const __half2 hd = __floats2half2_rn(orr, oi);
        const float2 hf = __half22float2(hd);
        const uint32_t head = *reinterpret_cast<const uint32_t*>(&hd);
        asm volatile("st.shared.b32 [%0], %1;" ::"r"(dst + (uint32_t)(y1 * 64 * Q)), "r"(head)
                     : "memory");
        asm volatile("st.shared.b32 [%0], %1;" ::"r"(dst + (uint32_t)(y1 * 64 * Q + 32 * Q)),
                     "r"(pack_half2(orr - hf.x, oi - hf.y))
                     : "memory");
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(e1done + pa);
    }
    }
  } else if (warp >= 12) {
    // ---------------------------------------------------------------- stage-2 epilogue
    // tensor memory -> FP16 -> output staging (row y' of 32 bytes, interleaved complex or
    // the segment [Re x 8 | Im x 8]), then handed to the TMA storer
    const int q = warp & 3;
    const int y1 = 4 * q + (lane >> 3), k2 = lane & 7;
    const uint32_t tl = tmem + ((uint32_t)(q * 32) << 16);
    for (int64_t j = 0; j < mine; ++j) {
      const int pd = (int)(j % kND), pe = (int)(j % kNE);
      const bool got = mbar_wait_s(smem_u32(d2full + pd), (uint32_t)(j / kND) & 1u, wait_iters);
      // staging buffer pe is free once the stores of item j - kNE have read it
      const bool freed = got && (j < kNE || mbar_wait_n(smem_u32(efree + pe),
                                                        (uint32_t)(j / kNE - 1) & 1u,
                                                        wait_iters));
      __syncwarp();  // tcgen05.ld needs the whole warp, converged
      if (!__all_sync(0xffffffffu, freed)) { *fail = 1; break; }
      if (__any_sync(0xffffffffu, *fail)) break;
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t tb = tl + (uint32_t)(pd * L::NC2);
      const uint32_t es = smem_u32(Es + (size_t)pe * L::S);
      // columns k2 >= h2 (the row padding) are written as zeros
      int xcol, yrow;
      item_xy(j, xcol, yrow);
      const bool pad = xcol + k2 >= h2;
      // D2 columns [Re | Im], Q each: output y' = y1 + 16 y2
#pragma unroll
      for (int g = 0; g < Q / 16; ++g) {
        float re[16], im[16];
        tmem_ld16(tb + (uint32_t)(g * 16), re);
        tmem_ld16(tb + (uint32_t)(Q + g * 16), im);
        asm volatile("tcgen05.wait::ld.sync.aligned;");
        if (g == Q / 16 - 1) {
          asm volatile("tcgen05.fence::before_thread_sync;");
          mbar_arrive(d2empty + pd);
        }
#pragma unroll
        for (int i = 0; i < 16; ++i) {
          const uint32_t row = es + 32u * (uint32_t)(y1 + 16 * (g * 16 + i));
          const uint32_t v = pad ? 0u : pack_half2(re[i], im[i]);
          if (seg) {
            asm volatile("st.shared.b16 [%0], %1;" ::"r"(row + 2u * k2),
                         "h"((uint16_t)(v & 0xffffu))
                         : "memory");
            asm volatile("st.shared.b16 [%0], %1;" ::"r"(row + 16u + 2u * k2),
                         "h"((uint16_t)(v >> 16))
                         : "memory");
          } else {
            asm volatile("st.shared.b32 [%0], %1;" ::"r"(row + 4u * k2), "r"(v) : "memory");
          }
        }
      }
      // the TMA stores read the staging through the async proxy
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(estaged + pe);
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == 0) {
    __syncwarp();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" : : "r"(tmem), "r"(L::TMEM));
  }
  if (tid == 0 && *fail) atomicExch(err, 1);
}

template <int Q>
int set_attrs(int optin) {
  TM_TRY(cuda_status(cudaFuncSetAttribute(ypass_tc_kernel<Q, false>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, optin),
                     "ypass_tc: shared memory attribute"));
  return cuda_status(cudaFuncSetAttribute(ypass_tc_kernel<Q, true>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, optin),
                     "ypass_tc: shared memory attribute");
}

}  // namespace

int ypass_tc_config(int n1, int hp, YpassTcConfig* cfg) {
  cfg->ok = false;
  cfg->n1 = n1;
  cfg->Q = n1 / 16;
  if ((n1 != 256 && n1 != 512) || hp % 8 != 0 || hp <= 0) return TM_OK;
  if (!tensor_maps_available()) return TM_OK;
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
  return (size_t)(t2_halves(cfg.Q) + kF1Halves) * 2;
}

int ypass_tc_prepare(const YpassTcConfig& cfg, uint16_t* table, cudaStream_t stream) {
  TM_REQUIRE(cfg.ok && table, "ypass_tc_prepare: unsupported configuration");
  ydft_table_kernel<<<32, 256, 0, stream>>>(table, cfg.Q);
  TM_TRY(check_launch("ydft_table_kernel"));
  ydft16_table_kernel<<<8, 256, 0, stream>>>(table + t2_halves(cfg.Q));
  return check_launch("ydft16_table_kernel");
}

int ypass_tc_run(const YpassTcConfig& cfg, void* H, int nb, int n0, int hp, int h2,
                 const uint16_t* table, uint32_t wait_iters, int* err, cudaStream_t stream,
                 bool seg, bool s1, void* Hout, bool xin) {
  TM_REQUIRE(cfg.ok, "ypass_tc_run: unsupported configuration");
  TM_REQUIRE(H && table && err && nb >= 1 && n0 >= 1 && hp % 8 == 0 && h2 >= 1 && h2 <= hp &&
                 wait_iters > 0,
             "ypass_tc_run: bad arguments");
  if (!Hout) Hout = H;
  // an x'-inner input cannot be overwritten item by item with row-major output
  TM_REQUIRE(!xin || Hout != H, "ypass_tc_run: an x'-inner input needs a separate output");
  TM_REQUIRE(reinterpret_cast<uintptr_t>(H) % 16 == 0 &&
                 reinterpret_cast<uintptr_t>(Hout) % 16 == 0 &&
                 reinterpret_cast<uintptr_t>(table) % 16 == 0,
             "ypass_tc_run: H, the output and the operator table must be 16-byte aligned");
  const int64_t rows = (int64_t)nb * n0 * cfg.n1;
  TM_REQUIRE(rows < ((int64_t)1 << 31), "ypass_tc_run: more than 2^31 rows");
  // the output as a 2D tensor of 4-byte words: hp columns, rows rows; boxes of 8 x 256
  // words. The input likewise, or, x'-inner, as a 4D tensor (8 words, n0 x', hp / 8
  // segments, nb n1 (b, k1) rows) with boxes of 8 x 1 x 1 x 256 words, which land in the
  // same shared layout.
  CUtensorMap lmap, smap;
  const uint64_t dims[2] = {(uint64_t)hp, (uint64_t)rows};
  const uint64_t strides[1] = {(uint64_t)hp * 4u};
  const uint32_t box[2] = {8u, (uint32_t)kBoxRows};
  TM_TRY(encode_tensor_map_u32(&smap, Hout, 2, dims, strides, box));
  if (xin) {
    const uint64_t dims4[4] = {8u, (uint64_t)n0, (uint64_t)hp / 8u, (uint64_t)nb * cfg.n1};
    const uint64_t strides4[3] = {32u, (uint64_t)n0 * 32u, (uint64_t)n0 * hp * 4u};
    const uint32_t box4[4] = {8u, 1u, 1u, (uint32_t)kBoxRows};
    TM_TRY(encode_tensor_map_u32(&lmap, H, 4, dims4, strides4, box4));
  } else {
    TM_TRY(encode_tensor_map_u32(&lmap, H, 2, dims, strides, box));
  }
  const int64_t nitems = (int64_t)nb * n0 * (hp / 8);
  const int grid = (int)std::min<int64_t>(nitems, cfg.sms);
  auto fn = cfg.Q == 32 ? (s1 ? ypass_tc_kernel<32, true> : ypass_tc_kernel<32, false>)
                        : (s1 ? ypass_tc_kernel<16, true> : ypass_tc_kernel<16, false>);
  fn<<<grid, kYThreads, cfg.smem, stream>>>(lmap, smap, nitems, hp / 8, n0, h2, table,
                                            wait_iters, err, seg ? 1 : 0, xin ? 1 : 0);
  return check_launch("ypass_tc_kernel");
}

}  // namespace tmb
