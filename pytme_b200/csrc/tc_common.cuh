// Shared helpers of the tensor-core kernels (tcgen05 on sm_100a): shared-memory matrix
// descriptors for the canonical K-major layout without swizzle, MMA issue and commit,
// bounded mbarrier waits and tensor-memory loads.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace tmb {
namespace tc {

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Canonical K-major, no-swizzle 16-bit operand: element (r, k) of a rows x K tile, in
// 8-row x 16-byte core matrices (K-adjacent core matrices 128 bytes apart, 8-row groups
// K*16 bytes apart).
__device__ __forceinline__ int kmajor16(int r, int k, int K) {
  return (r >> 3) * (K * 8) + (k >> 3) * 64 + (r & 7) * 8 + (k & 7);
}

// Shared-memory matrix descriptor: start address, leading- and stride-dimension byte
// offsets, descriptor version 1 (sm_100), base offset 0, no swizzle.
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  uint64_t d = 0;
  d |= (uint64_t)((addr >> 4) & 0x3fffu);
  d |= (uint64_t)((lbo >> 4) & 0x3fffu) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3fffu) << 32;
  d |= (uint64_t)1 << 46;
  return d;
}

// Instruction descriptor of kind::f16 with FP16 operands, FP32 accumulation, both
// operands K-major, M x N.
__host__ __device__ constexpr uint32_t idesc_f16(int M, int N) {
  return (1u << 4) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mma_f16(uint32_t tmem_d, uint64_t a, uint64_t b, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}\n"
      :
      : "r"(tmem_d), "l"(a), "l"(b), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void mma_commit(uint32_t mbar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :
               : "r"(mbar)
               : "memory");
}

constexpr uint32_t kWaitIters = 1u << 22;

// Wait for the completion of the mbarrier phase with the given parity, polling at most
// `iters` times; false when it did not complete.
__device__ __forceinline__ bool mbar_wait_n(uint32_t mbar, uint32_t phase, uint32_t iters) {
  for (uint32_t i = 0; i < iters; ++i) {
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

// The same for waits off the critical path: each poll lets the thread sleep until the
// phase completes or up to kSuspendNs have passed (the try_wait suspend-time hint), so a
// waiting warp takes fewer issue slots from the warps that work; the poll count is cut by
// kSuspendDiv so that the bound stays near that of mbar_wait_n.
constexpr uint32_t kSuspendNs = 1000, kSuspendDiv = 4;
__device__ __forceinline__ bool mbar_wait_s(uint32_t mbar, uint32_t phase, uint32_t iters) {
  const uint32_t n = iters / kSuspendDiv > 0 ? iters / kSuspendDiv : 1;
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}\n"
        : "=r"(done)
        : "r"(mbar), "r"(phase), "n"(kSuspendNs)
        : "memory");
    if (done) return true;
  }
  return false;
}

// Bounded wait for the completion of the mbarrier phase with the given parity.
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

__device__ __forceinline__ void tmem_ld32(uint32_t addr, float (&v)[32]) {
  uint32_t r[32];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, "
      "%11, %12, %13, %14, %15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, "
      "%28, %29, %30, %31}, [%32];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]),
        "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]),
        "=r"(r[13]), "=r"(r[14]), "=r"(r[15]), "=r"(r[16]), "=r"(r[17]), "=r"(r[18]),
        "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]), "=r"(r[24]),
        "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]),
        "=r"(r[31])
      : "r"(addr));
#pragma unroll
  for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// 16-byte asynchronous copy global -> shared; src_bytes < 16 zero-fills the rest.
__device__ __forceinline__ void cp_async16(uint32_t smem, const void* gmem, uint32_t src_bytes) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem), "l"(gmem),
               "r"(src_bytes));
}

}  // namespace tc
}  // namespace tmb
