// Tensor-core y pass of the fused CC / FLCSphericalMask scan (ypass_tc.cu).
#pragma once

#include <cuda_runtime.h>
#include <cstddef>
#include <cstdint>

namespace tmb {

struct YpassTcConfig {
  bool ok;
  int n1;      // transform length along y: 16 * Q, Q in {16, 32}
  int Q;
  int sms;     // persistent grid size
  size_t smem;
};

// Whether the tensor-core y pass handles n1 (and the row pitch hp of H).
int ypass_tc_config(int n1, int hp, YpassTcConfig* cfg);
size_t ypass_tc_table_bytes(const YpassTcConfig& cfg);
// The two DFT operators (FP16 head and rounded remainder), device memory of
// ypass_tc_table_bytes.
int ypass_tc_prepare(const YpassTcConfig& cfg, uint16_t* table, cudaStream_t stream);
// Unnormalised inverse DFT along axis 1 of the half-precision spectra
// H[nb][n0][n1][hp], in place, or into Hout (same shape and layout) when Hout is given;
// columns h2 .. hp - 1 of every row are written as zeros.
// wait_iters bounds every mbarrier wait; a wait that runs out sets *err and the kernel
// returns early (its output is then invalid).
// seg: write each row's 8-column item as a segment [Re x 8 | Im x 8] (the layout the
// even/odd tensor-core z pass reads with plain 16-byte copies) instead of interleaved.
// s1: the input rows are segments too, stored in the stage-1 order (row k1 = Q a + c of
// a plane at position 16 c + a, the order the tensor-core x pass writes with rowq = Q), and
// the radix-16 stage runs on the tensor cores; the output rows are in natural order.
// xin: the input is laid out x'-inner, H[nb][n1][hp / 8][n0][8] (the tensor-core x pass's
// xin layout); the output is row-major in Hout, which must then be a separate buffer.
int ypass_tc_run(const YpassTcConfig& cfg, void* H, int nb, int n0, int hp, int h2,
                 const uint16_t* table, uint32_t wait_iters, int* err, cudaStream_t stream,
                 bool seg = false, bool s1 = false, void* Hout = nullptr, bool xin = false);

}  // namespace tmb
