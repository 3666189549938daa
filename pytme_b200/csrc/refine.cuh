// Internal interfaces of the local-refinement kernels (refine.cu).
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace tmb {

// Shared arguments: template and mask (t^3), per-peak rotation (9, row-major),
// sub-voxel shift (3, target frame) and box corner (3), target (n^3), the value the
// target takes outside its bounds, and the norm_scores epsilon.
struct RefineArgs {
  const float* tmpl;
  const float* mask;
  int t[3];
  const float* rot;
  const float* shifts;
  const int32_t* corners;
  int P;
  const float* target;
  int n[3];
  float outside;  // target value outside its bounds
  double eps;
};

int euler_zyz(const float* angles, int P, float* R, float* dR, cudaStream_t st);
int refine_rotate(const RefineArgs& a, float* Tr, cudaStream_t st);
int refine_forward(const RefineArgs& a, const float* Tf, double* sums, float* scores,
                   cudaStream_t st);
int refine_grad_filtered(const RefineArgs& a, const float* Tf, const double* sums,
                         const float* grad_scores, float* gTf, cudaStream_t st);
int refine_backward(const RefineArgs& a, const float* Tf, const float* gTr, const double* sums,
                    const float* grad_scores, const float* dR, double* grad_rot,
                    double* grad_shift, double* grad_angles, float* grad_tmpl,
                    cudaStream_t st);

}  // namespace tmb
