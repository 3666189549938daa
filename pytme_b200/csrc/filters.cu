// Fourier filters built on the device: the CTF of a reconstructed volume and the
// continuous missing wedge, multiplied together in the order given, written directly
// in rfft (or full) layout with the DC term at index 0.
//
// Each voxel reproduces the reference's array arithmetic step for step, with the same
// float32 / float64 types (tme/filters/ctf.py:260-336 and 528-655,
// tme/filters/wedge.py:282-374, tme/filters/_utils.py:146-202, compose.py:36-59):
// * the frequency grid of fftfreqn is float32((i - n//2) / n) per axis, its Euclidean
//   norm the float32 sum of float32 squares, square-rooted in float32;
// * the CTF phase chi = (df - h k^2) * pi*lambda * k^2 + phase + atan(A/sqrt(1-A^2)) is
//   float64 from the float32 k^2, then sin(-chi) inside the cutoff, negated, optionally
//   made absolute, and cast to float32;
// * the wedge keeps a voxel when its tilt/opening index ratio lies outside the wedge
//   (start <= ratio or stop >= ratio, float64) and its frequency is within the cutoff;
// * the Compose product is float32.
// Scalars that depend only on the filter parameters (wavelength, aberration term,
// wedge bounds) are computed by the caller in float64 the way the reference does.
#include "common.cuh"
#include "ops.cuh"

#include <algorithm>
#include <cmath>

namespace tmb {

namespace {

struct FilterProgram {
  int n;
  tm_filter_component c[TM_FILTER_MAX_COMPONENTS];
};

__device__ __forceinline__ int centred_frequency(int k, int n) {
  // index k of the DC-at-0 layout -> (i - n//2) of the centred grid
  // (shift_fourier rolls by n//2 + n%2, tme/filters/_utils.py:233-246)
  const int shift = n / 2 + n % 2;
  int i = k - shift;
  i %= n;
  if (i < 0) i += n;
  return i - n / 2;
}

__device__ __forceinline__ float grid_norm(const int f[3], const int n[3]) {
  float acc = 0.f;
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    const float g = (float)((double)f[a] / (double)n[a]);
    acc = __fadd_rn(acc, __fmul_rn(g, g));
  }
  return __fsqrt_rn(acc);
}

__device__ __forceinline__ float ctf_value(const tm_filter_component& c, float k) {
  // p: 0 defocus_x, 1 h = 0.5 * aberration, 2 pi * lambda, 3 phase shift,
  //    4 amplitude-contrast phase, 5 cutoff, 6 flip phase (0/1)
  const float ksq = __fmul_rn(k, k);
  const double kd = (double)ksq;
  double chi = __dsub_rn(c.p[0], __dmul_rn(c.p[1], kd));
  chi = __dmul_rn(chi, c.p[2]);
  chi = __dmul_rn(chi, kd);
  chi = __dadd_rn(chi, c.p[3]);
  chi = __dadd_rn(chi, c.p[4]);
  double s = sin(-chi);
  s = (k < (float)c.p[5]) ? s : 0.0 * s;
  double v = -s;
  if (c.p[6] != 0.0) v = fabs(v);
  return (float)v;
}

__device__ __forceinline__ float wedge_value(const tm_filter_component& c, const int f[3],
                                             float k) {
  // p: 0 start, 1 stop, 2 ratio used where the opening index is 0, 3 opening axis,
  //    4 tilt axis, 5 frequency cutoff (negative: none)
  const int oa = (int)c.p[3], ta = (int)c.p[4];
  const double ratio = f[oa] == 0 ? c.p[2] : (double)f[ta] / (double)f[oa];
  float v = (c.p[0] <= ratio || c.p[1] >= ratio) ? 1.f : 0.f;
  if (c.p[5] >= 0.0 && !(k <= (float)c.p[5])) v = 0.f;
  return v > 0.f ? 1.f : 0.f;
}

__global__ void build_filter_kernel(FilterProgram prog, int n0, int n1, int n2, int rfft,
                                    float* __restrict__ out) {
  const int m2 = rfft ? n2 / 2 + 1 : n2;
  const int64_t total = (int64_t)n0 * n1 * m2;
  const int n[3] = {n0, n1, n2};
  for (int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; v < total;
       v += (int64_t)gridDim.x * blockDim.x) {
    const int k2 = (int)(v % m2);
    const int64_t r = v / m2;
    const int k1 = (int)(r % n1), k0 = (int)(r / n1);
    const int f[3] = {centred_frequency(k0, n0), centred_frequency(k1, n1),
                      centred_frequency(k2, n2)};
    const float k = grid_norm(f, n);
    float acc = 1.f;
    for (int i = 0; i < prog.n; ++i) {
      const tm_filter_component& c = prog.c[i];
      const float x = c.kind == TM_FILTER_CTF ? ctf_value(c, k) : wedge_value(c, f, k);
      acc = i == 0 ? x : __fmul_rn(x, acc);
    }
    out[v] = acc;
  }
}

}  // namespace

int build_filter(const tm_filter_component* comps, int n_comp, const int* shape, int rfft,
                 float* out, cudaStream_t stream) {
  TM_REQUIRE(comps && shape && out, "build_filter: null pointer");
  TM_REQUIRE(n_comp >= 1 && n_comp <= TM_FILTER_MAX_COMPONENTS,
             "build_filter: 1 to %d components", TM_FILTER_MAX_COMPONENTS);
  TM_REQUIRE(shape[0] > 0 && shape[1] > 0 && shape[2] > 0, "build_filter: empty shape");
  FilterProgram prog;
  prog.n = n_comp;
  for (int i = 0; i < n_comp; ++i) {
    TM_REQUIRE(comps[i].kind == TM_FILTER_CTF || comps[i].kind == TM_FILTER_WEDGE,
               "build_filter: unknown component kind %d", comps[i].kind);
    if (comps[i].kind == TM_FILTER_WEDGE) {
      const int oa = (int)comps[i].p[3], ta = (int)comps[i].p[4];
      TM_REQUIRE(oa >= 0 && oa < 3 && ta >= 0 && ta < 3, "build_filter: wedge axes out of range");
    }
    prog.c[i] = comps[i];
  }
  const int m2 = rfft ? shape[2] / 2 + 1 : shape[2];
  const int64_t total = (int64_t)shape[0] * shape[1] * m2;
  const int64_t blocks = std::min<int64_t>(ceil_div(total, 256), 148 * 16);
  build_filter_kernel<<<(unsigned)blocks, 256, 0, stream>>>(prog, shape[0], shape[1], shape[2],
                                                           rfft, out);
  return check_launch("build_filter_kernel");
}

}  // namespace tmb
