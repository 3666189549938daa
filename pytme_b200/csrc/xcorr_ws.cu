// x pass of the fused FLCSphericalMask / CC scan on the tensor cores, persistent and
// warp-specialised (mixed precision: FP16 operands, FP32 accumulation, FP16 output).
//
// Per spectrum column (k1, k2) the x pass is the circular correlation
//     H_b[x'] = sum_{x < t0} c[(x' - x) mod n0] g_b[x],
// c = s * (unnormalised inverse DFT along x of the target spectrum column), a Toeplitz
// (n0 x t0) by (t0 x B) complex product (the derivation is in xcorr_tc.cu). With the rows
// of a 128-row tile in reverse order of x' (row r <-> x' = 128 t + 127 - r) the operand is
// a Hankel matrix, A[r][x] = e[8 u0 + r + x] with e[i] = c[(n0 - 1 - i) mod n0] and
// u0 = (n0 - 128 (t + 1)) / 8. Its canonical K-major core matrix (row group g, K chunk kc)
// is the 8 x 8 block Z[g + kc] with row p = e[8 (u0 + g + kc) + p .. + 7]: one array of
// NZB = t0p/8 + 15 such blocks per tile and component, read by a shared-memory
// descriptor whose two strides are both 128 bytes.
//
// Work item = 8 consecutive k2 columns of one k1 and the group's rotations; a CTA runs
// items blockIdx.x, blockIdx.x + gridDim.x, ... and each item's n0/128 row tiles. Roles:
//   warp 0, lane 0   issues the MMAs (per tile and 16 rotations, one accumulator buffer:
//                    Re and Im of H for the 8 columns, N = 16, K = (Re g | Im g) in
//                    16-steps; the -Im c * Im g term through the A-negate bit) and commits
//                    them; the two buffers alternate;
//   warps 1-3        load the item's rotation operands (G, FP32 complex) and store them as
//                    FP16 in the K-major layout (double-buffered per item);
//   warps 4-7        stage the kernel values e of a tile (FP16, prescaled) and expand them
//                    into the Z blocks (double-buffered per tile);
//   warps 8-15       read the accumulators (tcgen05.ld), convert to FP16 complex and store
//                    each (rotation, x') row segment of 8 consecutive k2 as one aligned
//                    32-byte store: a sector written in parts by separate stores made the
//                    L2 fetch it from DRAM first.
// mbarriers hand the buffers between the roles; there is no block-wide barrier in the
// loop, so the loads of the next item and tile, the MMAs of the next accumulator buffer
// and the stores of the current one overlap. Every wait is bounded: on a timeout the
// role records the failure and leaves its loop, the MMA issuer waits for its last
// commit, and the kernel frees its tensor memory and returns with the error flag set.
#include "common.cuh"
#include "tc_common.cuh"
#include "xcorr_tc.cuh"

#include <cuda_fp16.h>

#include <algorithm>

namespace tmb {

namespace {

using namespace tc;

constexpr int kWsW = 8;          // k2 columns per item
constexpr int kWsRows = 128;     // x' rows per tile (MMA M)
constexpr int kWsGL = 96;        // rotation-operand loader threads (warps 1-3)
constexpr int kWsZB = 128;       // kernel-operand builder threads (warps 4-7)
constexpr int kWsEpi = 256;      // epilogue threads (warps 8-15)
constexpr int kWsThreads = 32 + kWsGL + kWsZB + kWsEpi;
constexpr float kWsPrescale = 256.f;  // keeps the scaled kernel values in FP16's normal range
constexpr uint32_t kWsTmemCols = 512;  // all of tensor memory
// A fill of R rotations (MMA N = R) takes 8 columns x (Re, Im) x R accumulator columns:
// two alternating buffers for R = 16, one for R = 32 (fewer, wider MMAs; each MMA fetches
// its 4 KB Hankel tile from shared memory once, whatever N is)

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" : : "r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" : : "r"(smem_u32(bar)) : "memory");
}
// barrier of the kernel-operand builders (warps 4-7) that returns the OR of `pred` over
// them, so every builder takes the same branch after it
__device__ __forceinline__ bool builders_any(bool pred) {
  uint32_t r;
  asm volatile(
      "{\n\t.reg .pred p, q;\n\t"
      "setp.ne.u32 p, %1, 0;\n\t"
      "bar.red.or.pred q, 1, %2, p;\n\t"
      "selp.u32 %0, 1, 0, q;\n\t}\n"
      : "=r"(r)
      : "r"((uint32_t)pred), "n"(kWsZB)
      : "memory");
  return r != 0;
}
constexpr int kWsMaxT0p = 64;
// kernel values staged per builder thread and tile: 8 columns x En / kWsZB, En <= 8 * (64/8 + 16)
constexpr int kWsMaxE = (kWsW * (8 * (kWsMaxT0p / 8 + 16)) + kWsZB - 1) / kWsZB;
__device__ __forceinline__ void tmem_ld4(uint32_t addr, float (&v)[4]) {
  uint32_t r[4];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0, %1, %2, %3}, [%4];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
               : "r"(addr));
#pragma unroll
  for (int i = 0; i < 4; ++i) v[i] = __uint_as_float(r[i]);
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

// The MMAs of one accumulator fill: for each of the 8 columns, Re H and Im H of R
// rotations over K = (Re g | Im g) in NXC steps of 16 (NXC = t0p / 8; the first half of
// the steps multiplies Re g, the second Im g). zlo: descriptor low word of the fill's
// Z segment; blo: of the rotation operand rows of the fill; nzb8 / bst16: the Z array
// and rotation operand strides >> 4.
template <int NXC, int R>
__device__ __forceinline__ void issue_fill(uint32_t d0, uint32_t zlo, uint32_t blo, uint32_t ahi,
                                           uint32_t bhi, uint32_t nzb8, uint32_t bst16,
                                           uint32_t idesc, uint32_t idesc_neg) {
#pragma unroll
  for (int w = 0; w < kWsW; ++w) {
    const uint32_t zr = zlo + (uint32_t)(2 * w) * nzb8, zi = zr + nzb8;
    const uint32_t bw = blo + (uint32_t)w * bst16;
    const uint32_t d_re = d0 + (uint32_t)(w * 2 * R), d_im = d_re + (uint32_t)R;
#pragma unroll
    for (int s = 0; s < NXC; ++s) {
      const bool imag_g = 2 * s >= NXC;
      const uint32_t kcl = (uint32_t)(imag_g ? 2 * s - NXC : 2 * s);
      const uint32_t ar = zr + 8u * kcl, ai = zi + 8u * kcl;  // Z blocks are 128 bytes
      const uint32_t b = bw + 16u * (uint32_t)s;               // 16 K values are 256 bytes
      // Re H: Re c Re g - Im c Im g;  Im H: Im c Re g + Re c Im g
      mma_f16_w(d_re, imag_g ? ai : ar, ahi, b, bhi, imag_g ? idesc_neg : idesc, s > 0);
      mma_f16_w(d_im, imag_g ? ar : ai, ahi, b, bhi, idesc, s > 0);
    }
  }
}

// one 32-byte store (the address is 32-byte aligned)
__device__ __forceinline__ void st_global_v8(void* p, const uint32_t (&v)[8]) {
  asm volatile("st.global.v8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};"
               :
               : "l"(p), "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]),
                 "r"(v[6]), "r"(v[7])
               : "memory");
}

struct WsLayout {
  int K, nzb, En, E;
  size_t b_stride;  // halves per column's rotation operand (NB x K, plus 16 bytes)
  size_t b_buf, z_buf, e_all, bar_off, total;
};

__host__ __device__ inline WsLayout ws_layout(int t0p, int NB) {
  WsLayout L;
  L.K = 2 * t0p;
  L.nzb = t0p / 8 + 15;
  // kernel values per array: En = 8 NZB + 8; the array stride E has 2 more so that the
  // 16 arrays start in different banks (the staging stores run across the arrays)
  L.En = 8 * L.nzb + 8;
  L.E = L.En + 2;
  L.b_stride = (size_t)NB * L.K + 8;  // the pad spreads the 8 columns' stores over the banks
  L.b_buf = (size_t)kWsW * L.b_stride * 2;           // bytes
  L.z_buf = (size_t)kWsW * 2 * L.nzb * 128;          // bytes
  L.e_all = (size_t)kWsW * 2 * L.E * 2;              // bytes
  L.bar_off = 2 * L.b_buf + 2 * L.z_buf + L.e_all;   // multiple of 16
  L.total = L.bar_off + 14 * 8 + 16;
  return L;
}

template <int NXC, int R>
__global__ void __launch_bounds__(kWsThreads, 1)
xcorr_ws_kernel(const float2* __restrict__ G, const float2* __restrict__ C, int nb, int NB,
                int t0, int n0, int n1, int h2, int hp, float scale,
                __half2* __restrict__ H, int* __restrict__ err, uint32_t wait_iters,
                int seg, int rowq, int ghalf, int xin) {
  constexpr int t0p = 8 * NXC;
  const uint32_t wi = wait_iters ? wait_iters : kWaitIters;  // data waits
  constexpr uint32_t kAccCols = 16u * R;               // one fill
  constexpr int kNbuf = (int)(kWsTmemCols / kAccCols);  // 2 (R = 16) or 1 (R = 32)
  extern __shared__ __align__(128) uint8_t smem_ws[];
  const WsLayout L = ws_layout(t0p, NB);
  const int K = L.K, NZB = L.nzb, En = L.En, E = L.E;
  uint16_t* Bs = reinterpret_cast<uint16_t*>(smem_ws);                         // 2 x [w][NB x K]
  uint16_t* Zs = reinterpret_cast<uint16_t*>(smem_ws + 2 * L.b_buf);           // 2 x [w,c][NZB][64]
  uint16_t* eh = reinterpret_cast<uint16_t*>(smem_ws + 2 * L.b_buf + 2 * L.z_buf);  // [w,c][E]
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_ws + L.bar_off);
  uint64_t* bfull = bar;       // rotation operands of an item stored   (count kWsGL)
  uint64_t* bempty = bar + 2;  // MMAs of an item done                  (commit)
  uint64_t* zfull = bar + 4;   // Z blocks of a tile stored              (count kWsZB)
  uint64_t* zempty = bar + 6;  // MMAs of a tile done                    (commit)
  uint64_t* tfull = bar + 8;   // accumulator buffer written             (commit)
  uint64_t* tempty = bar + 10; // accumulator buffer read                (count kWsEpi)
  uint64_t* mdone = bar + 12;  // every MMA of this CTA complete         (commit)
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(bar + 14);
  int* fail = reinterpret_cast<int*>(tmem_slot + 1);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;

  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :
                 : "r"(smem_u32(tmem_slot)), "r"(kWsTmemCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int q = 0; q < 2; ++q) {
      mbar_init(bfull + q, kWsGL);
      mbar_init(bempty + q, 1);
      mbar_init(zfull + q, kWsZB);
      mbar_init(zempty + q, 1);
      mbar_init(tfull + q, 1);
      mbar_init(tempty + q, kWsEpi);
    }
    mbar_init(mdone, 1);
    asm volatile("fence.mbarrier_init.release.cluster;");
    *fail = 0;
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;

  const int ncg = (h2 + kWsW - 1) / kWsW;
  const int64_t nitems = (int64_t)n1 * ncg;
  const int64_t mine = nitems > blockIdx.x ? (nitems - 1 - blockIdx.x) / gridDim.x + 1 : 0;
  const int ntile = n0 / kWsRows;
  const int64_t row = (int64_t)n1 * h2;  // G and C: [.][x][k1][k2]
  constexpr int nxc = NXC;
  // accumulator fills: f = tile * nh + h for the h-th R rotations of a tile, in buffer
  // f % kNbuf; the u-th fill of a buffer (u = f / kNbuf) completes phase u of its barriers
  const int nh = NB / R;

  if (warp == 0) {
    // ------------------------------------------------------------------ MMA issuer
    if (lane == 0) {
      const uint32_t idesc = idesc_f16(kWsRows, R);
      const uint32_t idesc_neg = idesc | (1u << 13);
      // descriptor words: Z blocks with both strides 128 bytes; rotation operands with
      // K-adjacent core matrices 128 bytes and 8-row groups K * 16 bytes apart
      const uint64_t za = smem_desc(smem_u32(Zs), 128u, 128u);
      const uint64_t bd = smem_desc(smem_u32(Bs), 128u, (uint32_t)K * 16u);
      const uint32_t zlo = (uint32_t)za, ahi = (uint32_t)(za >> 32);
      const uint32_t blo = (uint32_t)bd, bhi = (uint32_t)(bd >> 32);
      const uint32_t nzb8 = (uint32_t)NZB * 8u, zbuf16 = (uint32_t)(L.z_buf >> 4);
      const uint32_t bst16 = (uint32_t)(L.b_stride * 2 >> 4), bbuf16 = (uint32_t)(L.b_buf >> 4);
      bool ok = true;
      for (int64_t j = 0; j < mine && ok; ++j) {
        const int bsl = (int)(j & 1);
        if (!mbar_wait_n(smem_u32(bfull + bsl), (uint32_t)(j >> 1) & 1u, wi)) { ok = false; break; }
        for (int t = 0; t < ntile; ++t) {
          const int64_t tau = j * ntile + t;
          const int zsl = (int)(tau & 1);
          if (!mbar_wait_n(smem_u32(zfull + zsl), (uint32_t)(tau >> 1) & 1u, wi)) { ok = false; break; }
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          for (int h = 0; h < nh; ++h) {
            const int64_t f = tau * nh + h;
            const int buf = (int)(f % kNbuf);
            const uint32_t uf = (uint32_t)(f / kNbuf);
            if (f >= kNbuf && !mbar_wait_n(smem_u32(tempty + buf), (uf - 1) & 1u, wi)) {
              ok = false;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
            // rotations R h.. are row groups (R/8) h.. of the K-major operand
            issue_fill<NXC, R>(tmem + (uint32_t)buf * kAccCols, zlo + (uint32_t)zsl * zbuf16,
                               blo + (uint32_t)bsl * bbuf16 + (uint32_t)(R / 8 * h) * (uint32_t)K,
                               ahi, bhi, nzb8, bst16, idesc, idesc_neg);
            mma_commit(smem_u32(tfull + buf));
          }
          if (!ok) break;
          mma_commit(smem_u32(zempty + zsl));
        }
        if (!ok) break;
        mma_commit(smem_u32(bempty + bsl));
      }
      if (!ok) *fail = 1;
      // nothing may free tensor memory or shared memory under a running MMA
      mma_commit(smem_u32(mdone));
      if (!mbar_wait(smem_u32(mdone), 0u)) *fail = 1;
    }
  } else if (warp <= 3) {
    // ------------------------------------------------------------------ rotation operands
    const int lt = tid - 32;
    const int ntask = kWsW * NB * nxc;
    for (int64_t j = 0; j < mine; ++j) {
      const int bsl = (int)(j & 1);
      if (j >= 2 && !mbar_wait_n(smem_u32(bempty + bsl), (uint32_t)((j >> 1) - 1) & 1u, wi)) {
        *fail = 1;
        break;
      }
      if (*fail) break;
      const int64_t item = (int64_t)blockIdx.x + j * gridDim.x;
      const int k1 = (int)(item / ncg), cg = (int)(item - (int64_t)k1 * ncg);
      const int k20 = cg * kWsW;
      const int64_t col0 = (int64_t)k1 * h2 + k20;
      uint16_t* bb = Bs + (size_t)bsl * (L.b_buf / 2);
      // task = 8 consecutive x of one rotation and column, stored as two 16-byte rows;
      // the 8 lanes of a quarter warp read the 8 columns of one (rotation, x) row
#pragma unroll 4
      for (int i = lt; i < ntask; i += kWsGL) {
        const int w = i & (kWsW - 1);
        const int rest = i >> 3;
        const int xc = rest % nxc, n = rest / nxc;
        const bool live = n < nb && k20 + w < h2;
        uint32_t re[4], im[4];
        if (ghalf) {
          // G already FP16 (Re, Im) words: pair the x and x + 1 halves
          const uint32_t* Gh = reinterpret_cast<const uint32_t*>(G);
#pragma unroll
          for (int q = 0; q < 8; q += 2) {
            const int x = xc * 8 + q;
            uint32_t a = 0u, b = 0u;
            if (live && x < t0) a = __ldg(Gh + ((int64_t)n * t0 + x) * row + col0 + w);
            if (live && x + 1 < t0) b = __ldg(Gh + ((int64_t)n * t0 + x + 1) * row + col0 + w);
            re[q >> 1] = __byte_perm(a, b, 0x5410);
            im[q >> 1] = __byte_perm(a, b, 0x7632);
          }
        } else {
#pragma unroll
          for (int q = 0; q < 8; q += 2) {
            const int x = xc * 8 + q;
            float2 a = make_float2(0.f, 0.f), b = make_float2(0.f, 0.f);
            if (live && x < t0) a = G[((int64_t)n * t0 + x) * row + col0 + w];
            if (live && x + 1 < t0) b = G[((int64_t)n * t0 + x + 1) * row + col0 + w];
            const __half2 r2 = __floats2half2_rn(a.x, b.x);
            const __half2 i2 = __floats2half2_rn(a.y, b.y);
            re[q >> 1] = *reinterpret_cast<const uint32_t*>(&r2);
            im[q >> 1] = *reinterpret_cast<const uint32_t*>(&i2);
          }
        }
        uint16_t* bw = bb + (size_t)w * L.b_stride;
        *reinterpret_cast<uint4*>(bw + kmajor16(n, xc * 8, K)) =
            make_uint4(re[0], re[1], re[2], re[3]);
        *reinterpret_cast<uint4*>(bw + kmajor16(n, t0p + xc * 8, K)) =
            make_uint4(im[0], im[1], im[2], im[3]);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      mbar_arrive(bfull + bsl);
    }
  } else if (warp <= 7) {
    // ------------------------------------------------------------------ kernel operand
    const int lz = tid - 32 - kWsGL;
    const float cs = scale * kWsPrescale;
    // the kernel values of tile (j, t) for this thread, e[i] for i in [e0, e0 + En) with
    // e0 = 8 u0; the 8 lanes of a quarter warp read the 8 columns of one x
    float2 c[kWsMaxE];
    auto fetch = [&](int64_t j, int t) {
      const int64_t item = (int64_t)blockIdx.x + j * gridDim.x;
      const int k1 = (int)(item / ncg), cg = (int)(item - (int64_t)k1 * ncg);
      const int k20 = cg * kWsW;
      const int64_t col0 = (int64_t)k1 * h2 + k20;
      const int e0 = n0 - kWsRows * (t + 1);
#pragma unroll
      for (int k = 0; k < kWsMaxE; ++k) {
        const int idx = lz + k * kWsZB;
        const int w = idx & (kWsW - 1), i = idx >> 3;
        int m = n0 - 1 - (e0 + i);
        m += (m < 0) ? n0 : 0;
        c[k] = (idx < kWsW * En && k20 + w < h2) ? C[(int64_t)m * row + col0 + w]
                                                : make_float2(0.f, 0.f);
      }
    };
    if (mine > 0) fetch(0, 0);
    for (int64_t j = 0; j < mine; ++j) {
      bool stop = false;
      for (int t = 0; t < ntile; ++t) {
        const int64_t tau = j * ntile + t;
        const int zsl = (int)(tau & 1);
        // every builder is done reading the previous tile's e
        if (builders_any(*fail != 0)) { stop = true; break; }
#pragma unroll
        for (int k = 0; k < kWsMaxE; ++k) {
          const int idx = lz + k * kWsZB;
          if (idx < kWsW * En) {
            const int w = idx & (kWsW - 1), i = idx >> 3;
            eh[(size_t)(2 * w) * E + i] = __half_as_ushort(__float2half_rn(c[k].x * cs));
            eh[(size_t)(2 * w + 1) * E + i] = __half_as_ushort(__float2half_rn(c[k].y * cs));
          }
        }
        // the next tile's loads run while this tile's blocks are built
        if (t + 1 < ntile) fetch(j, t + 1);
        else if (j + 1 < mine) fetch(j + 1, 0);
        bool bad = false;
        if (tau >= 2) bad = !mbar_wait_n(smem_u32(zempty + zsl), (uint32_t)((tau >> 1) - 1) & 1u, wi);
        if (builders_any(bad)) {  // also: e of this tile complete
          *fail = 1;
          stop = true;
          break;
        }
        uint16_t* zz = Zs + (size_t)zsl * (L.z_buf / 2);
        // Z block u of array (w, c): row p = e[8u + p .. 8u + p + 7]
        for (int r = lz; r < kWsW * 2 * NZB * 8; r += kWsZB) {
          const int p = r & 7;
          const int rest = r >> 3;
          const int u = rest % NZB, wc = rest / NZB;
          const int s0 = 8 * u + p;
          const uint32_t* e32 = reinterpret_cast<const uint32_t*>(eh + (size_t)wc * E) + (s0 >> 1);
          const uint32_t sh = (uint32_t)(s0 & 1) * 16u;
          const uint32_t a0 = e32[0], a1 = e32[1], a2 = e32[2], a3 = e32[3], a4 = e32[4];
          *reinterpret_cast<uint4*>(zz + ((size_t)wc * NZB + u) * 64 + p * 8) =
              make_uint4(__funnelshift_r(a0, a1, sh), __funnelshift_r(a1, a2, sh),
                         __funnelshift_r(a2, a3, sh), __funnelshift_r(a3, a4, sh));
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        mbar_arrive(zfull + zsl);
      }
      if (stop) break;
    }
  } else {
    // ------------------------------------------------------------------ epilogue
    const int quarter = warp & 3, eg = (warp - 8) >> 2;  // eg: rotations (R/2) eg .. of a fill
    const float inv = 1.f / kWsPrescale;
    // H element strides of x', k1 and the 8-column segment: row-major [b][x'][k1][k2], or
    // x'-inner [b][k1][k2 / 8][x'][8], where the 32 consecutive x' rows a warp stores for
    // one rotation form 1 KB of whole cache lines
    const int64_t SH = (int64_t)n0 * n1 * hp;
    const int64_t xstr = xin ? 8 : (int64_t)n1 * hp;
    const int64_t kstr = xin ? (int64_t)n0 * hp : (int64_t)hp;
    const int64_t cstr = xin ? (int64_t)n0 * 8 : 8;
    const int r = quarter * 32 + lane;
    bool ok = true;
    for (int64_t j = 0; j < mine && ok; ++j) {
      const int64_t item = (int64_t)blockIdx.x + j * gridDim.x;
      const int k1 = (int)(item / ncg), cg = (int)(item - (int64_t)k1 * ncg);
      // row k1 = rowq a + c goes to position 16 c + a when rowq > 0 (the y pass's stage-1
      // order), to position k1 otherwise
      const int krow = rowq > 0 ? (k1 % rowq) * 16 + k1 / rowq : k1;
      const int64_t colH = (int64_t)krow * kstr + (int64_t)cg * cstr;
      for (int t = 0; t < ntile && ok; ++t) {
        const int64_t tau = j * ntile + t;
        const int xp = t * kWsRows + kWsRows - 1 - r;
        __half2* hrow = H + (int64_t)xp * xstr + colH;
        for (int h = 0; h < nh; ++h) {
          const int64_t f = tau * nh + h;
          const int buf = (int)(f % kNbuf);
          const bool got = mbar_wait_n(smem_u32(tfull + buf), (uint32_t)(f / kNbuf) & 1u, wi);
          __syncwarp();  // tcgen05.ld needs the whole warp, converged
          if (!__all_sync(0xffffffffu, got)) {
            *fail = 1;
            ok = false;
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;");
          const uint32_t tb = tmem + ((uint32_t)(quarter * 32) << 16) + (uint32_t)buf * kAccCols;
#pragma unroll
          for (int rr = 0; rr < R / 8; ++rr) {
            const int bl = R / 2 * eg + 4 * rr;  // rotation within the fill
            float v[2 * kWsW][4];            // [column * 2 + component][rotation]
#pragma unroll
            for (int wc = 0; wc < 2 * kWsW; ++wc)
              tmem_ld4(tb + (uint32_t)((wc >> 1) * 2 * R + (wc & 1) * R + bl), v[wc]);
            asm volatile("tcgen05.wait::ld.sync.aligned;");
#pragma unroll
            for (int q = 0; q < 4; ++q) {
              const int b = R * h + bl + q;
              if (b >= nb) break;
              uint32_t pk[kWsW];
              if (seg) {
                // segment [Re x 8 | Im x 8]: words 0-3 Re of column pairs, 4-7 Im
#pragma unroll
                for (int w = 0; w < kWsW / 2; ++w) {
                  const __half2 re = __floats2half2_rn(v[4 * w][q] * inv, v[4 * w + 2][q] * inv);
                  const __half2 im =
                      __floats2half2_rn(v[4 * w + 1][q] * inv, v[4 * w + 3][q] * inv);
                  pk[w] = *reinterpret_cast<const uint32_t*>(&re);
                  pk[kWsW / 2 + w] = *reinterpret_cast<const uint32_t*>(&im);
                }
              } else {
#pragma unroll
                for (int w = 0; w < kWsW; ++w) {
                  const __half2 hv =
                      __floats2half2_rn(v[2 * w][q] * inv, v[2 * w + 1][q] * inv);
                  pk[w] = *reinterpret_cast<const uint32_t*>(&hv);
                }
              }
              st_global_v8(hrow + (int64_t)b * SH, pk);
            }
          }
          asm volatile("tcgen05.fence::before_thread_sync;");
          mbar_arrive(tempty + buf);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == 0) {
    __syncwarp();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :
                 : "r"(tmem), "r"(kWsTmemCols));
  }
  if (tid == 0 && *fail) atomicExch(err, 1);
}

}  // namespace

int xcorr_ws_config(int n0, int t0, int nb, XcorrTcConfig* cfg) {
  cfg->ws = false;
  cfg->ws_t0p = (t0 + 15) / 16 * 16;
  cfg->ws_NB = (nb + 15) / 16 * 16;
  cfg->ws_smem = ws_layout(cfg->ws_t0p, cfg->ws_NB).total;
  // groups of 16 rotations, each in one of two 256-column accumulator buffers
  if (n0 % kWsRows != 0 || nb < 1 || cfg->ws_NB > 32 || cfg->ws_t0p > kWsMaxT0p) return TM_OK;
  int dev = 0, optin = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cudaGetLastError();
  cfg->sms = sms;
  if (cfg->ws_smem > (size_t)optin) return TM_OK;
  for (auto fn : {xcorr_ws_kernel<2, 16>, xcorr_ws_kernel<4, 16>, xcorr_ws_kernel<6, 16>,
                  xcorr_ws_kernel<8, 16>, xcorr_ws_kernel<2, 32>, xcorr_ws_kernel<4, 32>,
                  xcorr_ws_kernel<6, 32>, xcorr_ws_kernel<8, 32>})
    TM_TRY(cuda_status(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            optin),
                       "xcorr_ws: shared memory attribute"));
  cfg->ws = true;
  return TM_OK;
}

int xcorr_ws_run(const XcorrTcConfig& cfg, const float2* G, const float2* C, int nb, int t0,
                 int n0, int n1, int h2, int hp, float scale, __half2* H, int* err,
                 cudaStream_t stream, uint32_t wait_iters, bool seg, int rowq, bool g_half,
                 bool xin) {
  // 32-byte row segments: pitch a multiple of 8 complex values, aligned base
  TM_REQUIRE(cfg.ws && nb <= cfg.ws_NB && hp % 8 == 0 && hp >= h2 &&
                 reinterpret_cast<uintptr_t>(H) % 32 == 0 &&
                 (rowq == 0 || (rowq > 0 && n1 == 16 * rowq)),
             "xcorr_ws_run: unsupported configuration");
  const int64_t nitems = (int64_t)n1 * ((h2 + kWsW - 1) / kWsW);
  const int grid = (int)std::min<int64_t>(nitems, cfg.sms);
  // one fill of all 32 rotations (single buffer) or two alternating fills of 16
  const bool wide = cfg.ws_NB == 32;
  auto fn = wide ? xcorr_ws_kernel<6, 32> : xcorr_ws_kernel<6, 16>;
  switch (cfg.ws_t0p) {
    case 16: fn = wide ? xcorr_ws_kernel<2, 32> : xcorr_ws_kernel<2, 16>; break;
    case 32: fn = wide ? xcorr_ws_kernel<4, 32> : xcorr_ws_kernel<4, 16>; break;
    case 48: break;
    case 64: fn = wide ? xcorr_ws_kernel<8, 32> : xcorr_ws_kernel<8, 16>; break;
    default: TM_REQUIRE(false, "xcorr_ws_run: t0p %d", cfg.ws_t0p);
  }
  fn<<<grid, kWsThreads, cfg.ws_smem, stream>>>(G, C, nb, cfg.ws_NB, t0, n0, n1, h2, hp, scale,
                                               H, err, wait_iters, seg ? 1 : 0, rowq,
                                               g_half ? 1 : 0, xin ? 1 : 0);
  return check_launch("xcorr_ws_kernel");
}

}  // namespace tmb
