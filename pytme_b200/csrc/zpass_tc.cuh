// Tensor-core z pass of the fused CC / FLCSphericalMask scan (zpass_tc.cu).
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

namespace tmb {

struct ZpassTcConfig {
  bool ok;
  int K;        // 2 * row pitch (FP16 halves per H row)
  int n2;
  int sms;      // persistent grid size
  size_t smem;
  // even/odd variant (n2/2 + 1 <= 128): cosine and sine operators over z <= n2/2,
  // K' = h2 rounded up to 16 per component
  bool eo;
  int Kp, zr;
  size_t eo_smem;
};

// Whether the tensor-core z pass handles n2 / h2 / row pitch hp / nb rotations per group.
int zpass_tc_config(int n2, int h2, int hp, int nb, ZpassTcConfig* cfg);
size_t zpass_tc_table_bytes(const ZpassTcConfig& cfg);
// The c2r operator table (FP16, device memory of zpass_tc_table_bytes).
int zpass_tc_prepare(const ZpassTcConfig& cfg, uint16_t* table, int n2, int h2,
                     cudaStream_t stream);
// c2r of the half-precision rows of H (pitch hp) for nb rotations, scaled by
// scale * inv_den (inv_den may be null), strict running max / argmax into the state.
// wait_iters bounds every data wait (0: the default budget). seg: rows of H hold 32-byte
// segments [Re x 8 | Im x 8] of 8 consecutive k2 (even/odd kernel only).
int zpass_tc_run(const ZpassTcConfig& cfg, const void* H, int nb, int64_t rows, int n2, int h2,
                 int hp, const uint16_t* table, float scale, const float* inv_den,
                 int32_t first_index, float* state_max, int32_t* state_rot, int64_t SH,
                 const int32_t* first_dev, int* err, cudaStream_t stream,
                 uint32_t wait_iters = 0, bool seg = false);

}  // namespace tmb
