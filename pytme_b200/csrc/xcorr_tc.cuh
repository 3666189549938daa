// Tensor-core x pass of the fused FLCSphericalMask / CC scan (xcorr_tc.cu).
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

namespace tmb {

struct XcorrTcConfig {
  bool ok;
  int t0p, K, NB, W;
  size_t smem;
  // FP16 Hankel-operand variant for half-precision outputs (n0 a multiple of 128)
  bool hk;
  int hk_t0p, hk_W;
  size_t hk_smem;
  // persistent warp-specialised FP16 variant (xcorr_ws.cu): at most 32 rotations per
  // group, t0 <= 64, n0 a multiple of 128, output row pitch a multiple of 8
  bool ws;
  int ws_t0p, ws_NB, sms;
  size_t ws_smem;
};

// Whether the tensor-core x pass handles n0 / t0 / nb, with its launch shape.
int xcorr_tc_config(int n0, int t0, int nb, XcorrTcConfig* cfg);
// Fills the ws fields of cfg (called by xcorr_tc_config).
int xcorr_ws_config(int n0, int t0, int nb, XcorrTcConfig* cfg);
// wait_iters bounds every data wait of the persistent kernel (0: the default budget).
// seg: write each row's 8-column segment as [Re x 8 | Im x 8] instead of interleaved
// complex values; rowq > 0 (n1 = 16 rowq): store row k1 = rowq a + c of each plane at
// position 16 c + a. Both together give the input layout of the tensor-core y pass with
// its radix-16 stage on the tensor cores. g_half: G holds FP16 complex values (__half2)
// instead of float2, at the same element offsets. xin: H is laid out x'-inner,
// [b][k1][k2 / 8][x'][8] (hp a multiple of 8), so that the 32-byte segments a warp stores
// for 32 consecutive x' form whole cache lines instead of 32 lines one plane apart.
int xcorr_ws_run(const XcorrTcConfig& cfg, const float2* G, const float2* C, int nb, int t0,
                 int n0, int n1, int h2, int hp, float scale, __half2* H, int* err,
                 cudaStream_t stream, uint32_t wait_iters = 0, bool seg = false, int rowq = 0,
                 bool g_half = false, bool xin = false);
// C = unnormalised inverse DFT along x (axis 0) of the target spectrum F [n0][n1][h2].
int xcorr_tc_prepare(const float2* F, float2* C, int n0, int n1, int h2, cudaStream_t stream);
// H[b][x'][k1][k2] = sum_{x<t0} scale * C[(x'-x) mod n0][k1][k2] * G[b][x][k1][k2];
// G and C have row pitch h2, H has row pitch hp >= h2.
int xcorr_tc_run(const XcorrTcConfig& cfg, const float2* G, const float2* C, int nb, int t0,
                 int n0, int n1, int h2, int hp, float scale, void* H, bool half, int* err,
                 cudaStream_t stream, uint32_t wait_iters = 0, bool seg = false,
                 int rowq = 0, bool g_half = false, bool xin = false);

}  // namespace tmb
