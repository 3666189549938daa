// Local refinement of candidate peaks: the FLC score of the exhaustive scan at one
// pose per peak, and its hand-written adjoint.
//
// Peak p has a box corner k_p (target voxel of template voxel 0), a rotation R_p about
// the template centre c = (t - 1)/2 and a sub-voxel shift s_p in the target frame.
// Template voxel o samples the template and mask at
//     u(o) = R_p^T (o - c - s_p) + c
// by order-1 interpolation with SciPy's constant-mode bounds (0 unless every
// coordinate lies in [0, n - 1]), giving T_r(o) and M_r(o). With T_f = L T_r (the
// template filter, a real multiplier on the rfft spectrum applied by the host between
// kernels; L is self-adjoint) and f(o) = target[k_p + o] (a given constant outside the
// target, 0 for the raw target):
//     A = sum M_r, B = sum M_r T_f, C = sum M_r T_f^2, D = sum M_r T_f f,
//     E = sum M_r f, F = sum M_r f^2,
//     mu = B/A, v_t = C/A - mu^2, v_f = F/A - (E/A)^2,
//     S = (D - mu E) / (sqrt(v_t) A sigma_f),  sigma_f = sqrt(v_f), or 1 if below eps,
// which is flc_scoring (tme/matching_scores.py:629-759) at one translation:
// normalize_template (tme/matching_utils.py:61-99) of the filtered rotated template
// under the rotated mask, and norm_scores (tme/backends/npfftw_backend.py:537-587).
//
// Forward: one pass per peak over its t^3 voxels accumulating A..F in double.
// Backward: the rotation is recomputed (checkpointed, never stored across the
// pass); per voxel dS/dT_f = M_r (gB + 2 gC T_f + gD f) and
// dS/dM_r = gA + gB T_f + gC T_f^2 + gD T_f f + gE f + gF f^2 are chained through the
// trilinear weights into dS/du, then into dS/dR, dS/ds, dS/d(angles) and the template
// density gradient (summed over peaks, in shared memory when t^3 floats fit).
#include "common.cuh"
#include "refine.cuh"

#include <algorithm>
#include <cmath>

namespace tmb {

namespace {

constexpr int kRefThreads = 256;
constexpr int kRefBackSmemThreads = 512;       // one CTA per SM holds the gradient
constexpr int kSmemGradMaxVoxels = 48 * 1024;  // 192 KiB of float template gradient

struct Box {
  int t0, t1, t2;
  float c0, c1, c2;
  int nv;
};

__device__ __forceinline__ Box make_box(int t0, int t1, int t2) {
  Box b;
  b.t0 = t0; b.t1 = t1; b.t2 = t2;
  b.c0 = 0.5f * (t0 - 1); b.c1 = 0.5f * (t1 - 1); b.c2 = 0.5f * (t2 - 1);
  b.nv = t0 * t1 * t2;
  return b;
}

// Template voxel (o0, o1, o2) of v = start, start + stride, ...: one division set at
// the start, then carries instead of a division per voxel.
struct Walker {
  int o0, o1, o2, d0, d1, d2;
  __device__ __forceinline__ void init(const Box& b, int v, int stride) {
    o2 = v % b.t2;
    o1 = (v / b.t2) % b.t1;
    o0 = v / (b.t1 * b.t2);
    d2 = stride % b.t2;
    d1 = (stride / b.t2) % b.t1;
    d0 = stride / (b.t1 * b.t2);
  }
  __device__ __forceinline__ void next(const Box& b) {
    o2 += d2;
    int c = o2 >= b.t2 ? 1 : 0;
    o2 -= c * b.t2;
    o1 += d1 + c;
    c = o1 >= b.t1 ? 1 : 0;
    o1 -= c * b.t1;
    o0 += d0 + c;
  }
};

// d = o - c - s and u = R^T d + c; R row-major.
__device__ __forceinline__ void pose_coords(const Box& b, const float* R, const float* s,
                                            const Walker& w, float d[3], float u[3]) {
  d[0] = (float)w.o0 - b.c0 - s[0];
  d[1] = (float)w.o1 - b.c1 - s[1];
  d[2] = (float)w.o2 - b.c2 - s[2];
  u[0] = fmaf(R[0], d[0], fmaf(R[3], d[1], fmaf(R[6], d[2], b.c0)));
  u[1] = fmaf(R[1], d[0], fmaf(R[4], d[1], fmaf(R[7], d[2], b.c1)));
  u[2] = fmaf(R[2], d[0], fmaf(R[5], d[1], fmaf(R[8], d[2], b.c2)));
}

// Trilinear stencil: base index, per-axis steps (0 at the upper edge) and fractions.
struct Stencil {
  int base, s0, s1, s2;
  float f0, f1, f2;
};

__device__ __forceinline__ bool stencil(const Box& b, const float u[3], Stencil& st) {
  const int n[3] = {b.t0, b.t1, b.t2};
  int lo[3], step[3];
  float f[3];
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    if (!(u[a] >= 0.f) || u[a] > (float)(n[a] - 1)) return false;
    const float fl = floorf(u[a]);
    lo[a] = (int)fl;
    f[a] = u[a] - fl;
    step[a] = lo[a] + 1 < n[a] ? 1 : 0;
  }
  st.base = (lo[0] * b.t1 + lo[1]) * b.t2 + lo[2];
  st.s0 = step[0] * b.t1 * b.t2;
  st.s1 = step[1] * b.t2;
  st.s2 = step[2];
  st.f0 = f[0]; st.f1 = f[1]; st.f2 = f[2];
  return true;
}

// Corner values c[4*b0 + 2*b1 + b2] (b_a = 1: upper neighbour on axis a).
__device__ __forceinline__ void corners8(const float* __restrict__ a, const Stencil& st,
                                         float c[8]) {
  const float* p = a + st.base;
  const int s12 = st.s1 + st.s2;
  c[0] = __ldg(p);
  c[1] = __ldg(p + st.s2);
  c[2] = __ldg(p + st.s1);
  c[3] = __ldg(p + s12);
  p += st.s0;
  c[4] = __ldg(p);
  c[5] = __ldg(p + st.s2);
  c[6] = __ldg(p + st.s1);
  c[7] = __ldg(p + s12);
}

// Trilinear value as nested linear interpolations (axis 2, then 1, then 0).
__device__ __forceinline__ float lerp8(const float c[8], const Stencil& st) {
  const float l00 = fmaf(st.f2, c[1] - c[0], c[0]);
  const float l01 = fmaf(st.f2, c[3] - c[2], c[2]);
  const float l10 = fmaf(st.f2, c[5] - c[4], c[4]);
  const float l11 = fmaf(st.f2, c[7] - c[6], c[6]);
  const float l0 = fmaf(st.f1, l01 - l00, l00);
  const float l1 = fmaf(st.f1, l11 - l10, l10);
  return fmaf(st.f0, l1 - l0, l0);
}

// Gradient of lerp8 with respect to the fractions (= the sample coordinates).
__device__ __forceinline__ void lerp8_grad(const float e[8], const Stencil& st, float du[3]) {
  const float a00 = e[1] - e[0], a01 = e[3] - e[2], a10 = e[5] - e[4], a11 = e[7] - e[6];
  const float l00 = fmaf(st.f2, a00, e[0]), l01 = fmaf(st.f2, a01, e[2]);
  const float l10 = fmaf(st.f2, a10, e[4]), l11 = fmaf(st.f2, a11, e[6]);
  const float b0 = fmaf(st.f1, a01 - a00, a00), b1 = fmaf(st.f1, a11 - a10, a10);
  du[2] = fmaf(st.f0, b1 - b0, b0);
  const float c0 = l01 - l00, c1 = l11 - l10;
  du[1] = fmaf(st.f0, c1 - c0, c0);
  du[0] = fmaf(st.f1, l11 - l10, l10) - fmaf(st.f1, l01 - l00, l00);
}

__device__ __forceinline__ float target_at(const float* __restrict__ tg, int n0, int n1, int n2,
                                           float outside, const int k[3], const Walker& w) {
  const int x = k[0] + w.o0, y = k[1] + w.o1, z = k[2] + w.o2;
  if (x < 0 || y < 0 || z < 0 || x >= n0 || y >= n1 || z >= n2) return outside;
  return __ldg(tg + ((int64_t)x * n1 + y) * n2 + z);
}

// Block-wide sums of K doubles; the result is valid in thread 0. sh holds 32*K doubles.
template <int K>
__device__ __forceinline__ void block_sums(double (&v)[K], double* sh) {
#pragma unroll
  for (int k = 0; k < K; ++k)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  __syncthreads();
  if (lane == 0)
#pragma unroll
    for (int k = 0; k < K; ++k) sh[warp * K + k] = v[k];
  __syncthreads();
  if (threadIdx.x == 0) {
#pragma unroll
    for (int k = 0; k < K; ++k) {
      double s = 0.0;
      for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += sh[w * K + k];
      v[k] = s;
    }
  }
}

// Score and its partial derivatives with respect to the six sums, scaled by g.
struct ScoreGrad {
  double S, gA, gB, gC, gD, gE, gF;
  bool valid;
};

__device__ __forceinline__ ScoreGrad score_grad(const double* sums, double eps, double g) {
  ScoreGrad r{0, 0, 0, 0, 0, 0, 0, false};
  const double A = sums[0], B = sums[1], C = sums[2], D = sums[3], E = sums[4], F = sums[5];
  if (!(A > 0.0)) return r;
  const double mu = B / A;
  const double vt = C / A - mu * mu;
  if (!(vt > 0.0)) return r;
  double vf = F / A - (E / A) * (E / A);
  vf = vf > 0.0 ? vf : 0.0;
  double sf = sqrt(vf);
  const bool use_sf = !(sf < eps);
  if (!use_sf) sf = 1.0;
  const double K = 1.0 / (sqrt(vt) * A * sf);
  const double S = (D - mu * E) * K;
  r.S = S;
  r.valid = true;
  r.gD = g * K;
  r.gB = g * (-E * K + S * mu / vt) / A;
  r.gC = g * (-S / (2.0 * vt * A));
  r.gE = g * (-mu * K + (use_sf ? S * E / (vf * A * A) : 0.0));
  r.gF = use_sf ? g * (-S / (2.0 * vf * A)) : 0.0;
  r.gA = g * (-S / A + E * K * mu / A + (S / vt) * (C / (2.0 * A * A) - mu * mu / A) +
              (use_sf ? (S / vf) * (F / (2.0 * A * A) - E * E / (A * A * A)) : 0.0));
  return r;
}

__device__ __forceinline__ void load_pose(const float* rot, const float* shifts,
                                          const int32_t* corners, int p, float* Rs, float* ss,
                                          int* ks) {
  if (threadIdx.x < 9) Rs[threadIdx.x] = rot[p * 9 + threadIdx.x];
  if (threadIdx.x < 3) {
    ss[threadIdx.x] = shifts[p * 3 + threadIdx.x];
    ks[threadIdx.x] = corners[p * 3 + threadIdx.x];
  }
}

// R = Rz(g) Ry(b) Rz(a) for angles (a, b, g) in degrees (SciPy's extrinsic "zyz"),
// and dR/d(angle) per degree.
__global__ void euler_zyz_kernel(const float* __restrict__ angles, int P, float* __restrict__ R,
                                 float* __restrict__ dR) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= P) return;
  const double k = 3.14159265358979323846 / 180.0;
  double ca, sa, cb, sb, cg, sg;
  sincos(k * (double)angles[3 * p + 0], &sa, &ca);
  sincos(k * (double)angles[3 * p + 1], &sb, &cb);
  sincos(k * (double)angles[3 * p + 2], &sg, &cg);
  const double Za[9] = {ca, -sa, 0, sa, ca, 0, 0, 0, 1};
  const double Yb[9] = {cb, 0, sb, 0, 1, 0, -sb, 0, cb};
  const double Zg[9] = {cg, -sg, 0, sg, cg, 0, 0, 0, 1};
  const double dZa[9] = {-sa, -ca, 0, ca, -sa, 0, 0, 0, 0};
  const double dYb[9] = {-sb, 0, cb, 0, 0, 0, -cb, 0, -sb};
  const double dZg[9] = {-sg, -cg, 0, cg, -sg, 0, 0, 0, 0};
  auto mm = [](const double* a, const double* b, double* c) {
    for (int i = 0; i < 3; ++i)
      for (int j = 0; j < 3; ++j)
        c[i * 3 + j] = a[i * 3] * b[j] + a[i * 3 + 1] * b[3 + j] + a[i * 3 + 2] * b[6 + j];
  };
  double t[9], out[9];
  mm(Zg, Yb, t);
  mm(t, Za, out);
  for (int i = 0; i < 9; ++i) R[9 * p + i] = (float)out[i];
  if (!dR) return;
  mm(t, dZa, out);  // d/da
  for (int i = 0; i < 9; ++i) dR[27 * p + i] = (float)(out[i] * k);
  mm(Zg, dYb, t);   // d/db
  mm(t, Za, out);
  for (int i = 0; i < 9; ++i) dR[27 * p + 9 + i] = (float)(out[i] * k);
  mm(dZg, Yb, t);   // d/dg
  mm(t, Za, out);
  for (int i = 0; i < 9; ++i) dR[27 * p + 18 + i] = (float)(out[i] * k);
}

// Rotated template T_r for every peak (the input of the template filter).
__global__ void __launch_bounds__(kRefThreads)
refine_rotate_kernel(const float* __restrict__ T, int t0, int t1, int t2,
                     const float* __restrict__ rot, const float* __restrict__ shifts,
                     float* __restrict__ Tr) {
  const int p = blockIdx.y;
  __shared__ float Rs[9], ss[3];
  if (threadIdx.x < 9) Rs[threadIdx.x] = rot[p * 9 + threadIdx.x];
  if (threadIdx.x < 3) ss[threadIdx.x] = shifts[p * 3 + threadIdx.x];
  __syncthreads();
  const Box b = make_box(t0, t1, t2);
  const int start = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  Walker w;
  w.init(b, start, stride);
  for (int v = start; v < b.nv; v += stride, w.next(b)) {
    float d[3], u[3];
    pose_coords(b, Rs, ss, w, d, u);
    Stencil st;
    float a = 0.f;
    if (stencil(b, u, st)) {
      float c[8];
      corners8(T, st, c);
      a = lerp8(c, st);
    }
    Tr[(int64_t)p * b.nv + v] = a;
  }
}

// Sums A..F and the score of each peak. FILTERED reads T_f from memory, otherwise the
// rotated template is interpolated in place.
template <bool FILTERED>
__global__ void __launch_bounds__(kRefThreads)
refine_forward_kernel(const float* __restrict__ T, const float* __restrict__ M, int t0, int t1,
                      int t2, const float* __restrict__ rot, const float* __restrict__ shifts,
                      const int32_t* __restrict__ corners, int P, const float* __restrict__ Tf,
                      const float* __restrict__ tg, int n0, int n1, int n2, float outside, double eps,
                      double* __restrict__ sums, float* __restrict__ scores) {
  __shared__ double red[32 * 6];
  __shared__ float Rs[9], ss[3];
  __shared__ int ks[3];
  const Box b = make_box(t0, t1, t2);
  for (int p = blockIdx.x; p < P; p += gridDim.x) {
    __syncthreads();
    if (threadIdx.x < 9) Rs[threadIdx.x] = rot[p * 9 + threadIdx.x];
    if (threadIdx.x < 3) {
      ss[threadIdx.x] = shifts[p * 3 + threadIdx.x];
      ks[threadIdx.x] = corners[p * 3 + threadIdx.x];
    }
    __syncthreads();
    double acc[6] = {0, 0, 0, 0, 0, 0};
    Walker w;
    w.init(b, threadIdx.x, blockDim.x);
    for (int v = threadIdx.x; v < b.nv; v += blockDim.x, w.next(b)) {
      float d[3], u[3];
      pose_coords(b, Rs, ss, w, d, u);
      Stencil st;
      if (!stencil(b, u, st)) continue;
      float c[8];
      corners8(M, st, c);
      const float mr = lerp8(c, st);
      if (mr == 0.f) continue;
      float tr;
      if (FILTERED) {
        tr = __ldg(Tf + (int64_t)p * b.nv + v);
      } else {
        corners8(T, st, c);
        tr = lerp8(c, st);
      }
      const double m = mr, tf = tr;
      const double f = target_at(tg, n0, n1, n2, outside, ks, w);
      const double mt = m * tf, mf = m * f;
      acc[0] += m;
      acc[1] += mt;
      acc[2] += mt * tf;
      acc[3] += mt * f;
      acc[4] += mf;
      acc[5] += mf * f;
    }
    block_sums<6>(acc, red);
    if (threadIdx.x == 0) {
#pragma unroll
      for (int k = 0; k < 6; ++k) sums[p * 6 + k] = acc[k];
      scores[p] = (float)score_grad(acc, eps, 0.0).S;
    }
  }
}

// dS/dT_f of every voxel (filtered path), the input of the adjoint filter.
__global__ void __launch_bounds__(kRefThreads)
refine_grad_filtered_kernel(const float* __restrict__ M, int t0, int t1, int t2,
                            const float* __restrict__ rot, const float* __restrict__ shifts,
                            const int32_t* __restrict__ corners, const float* __restrict__ Tf,
                            const float* __restrict__ tg, int n0, int n1, int n2, float outside, double eps,
                            const double* __restrict__ sums, const float* __restrict__ gout,
                            float* __restrict__ gTf) {
  const int p = blockIdx.y;
  __shared__ float Rs[9], ss[3];
  __shared__ int ks[3];
  load_pose(rot, shifts, corners, p, Rs, ss, ks);
  __syncthreads();
  const ScoreGrad sg = score_grad(sums + 6 * p, eps, (double)gout[p]);
  const Box b = make_box(t0, t1, t2);
  const int start = blockIdx.x * blockDim.x + threadIdx.x, stride = gridDim.x * blockDim.x;
  Walker w;
  w.init(b, start, stride);
  for (int v = start; v < b.nv; v += stride, w.next(b)) {
    float g = 0.f;
    if (sg.valid) {
      float d[3], u[3];
      pose_coords(b, Rs, ss, w, d, u);
      Stencil st;
      if (stencil(b, u, st)) {
        float c[8];
        corners8(M, st, c);
        const float mr = lerp8(c, st);
        if (mr != 0.f) {
          const double tf = __ldg(Tf + (int64_t)p * b.nv + v);
          const double f = target_at(tg, n0, n1, n2, outside, ks, w);
          g = (float)((double)mr * (sg.gB + 2.0 * sg.gC * tf + sg.gD * f));
        }
      }
    }
    gTf[(int64_t)p * b.nv + v] = g;
  }
}

// Chain through the interpolation into the pose and template gradients. FILTERED reads
// T_f and dS/dT_r = L^T dS/dT_f from memory; otherwise both come from the in-place
// interpolation. SMEM_GT accumulates the template gradient in shared memory.
template <bool FILTERED, bool SMEM_GT, int THREADS>
__global__ void __launch_bounds__(THREADS)
refine_backward_kernel(const float* __restrict__ T, const float* __restrict__ M, int t0, int t1,
                       int t2, const float* __restrict__ rot, const float* __restrict__ shifts,
                       const int32_t* __restrict__ corners, int P, const float* __restrict__ Tf,
                       const float* __restrict__ gTr_in, const float* __restrict__ tg, int n0,
                       int n1, int n2, float outside, double eps, const double* __restrict__ sums,
                       const float* __restrict__ gout, const float* __restrict__ dR,
                       double* __restrict__ grad_rot, double* __restrict__ grad_shift,
                       double* __restrict__ grad_angles, float* __restrict__ gT) {
  extern __shared__ float gts[];
  __shared__ double red[32 * 12];
  __shared__ float Rs[9], ss[3];
  __shared__ int ks[3];
  const Box b = make_box(t0, t1, t2);
  if (SMEM_GT) {
    for (int v = threadIdx.x; v < b.nv; v += blockDim.x) gts[v] = 0.f;
  }
  for (int p = blockIdx.x; p < P; p += gridDim.x) {
    __syncthreads();
    if (threadIdx.x < 9) Rs[threadIdx.x] = rot[p * 9 + threadIdx.x];
    if (threadIdx.x < 3) {
      ss[threadIdx.x] = shifts[p * 3 + threadIdx.x];
      ks[threadIdx.x] = corners[p * 3 + threadIdx.x];
    }
    __syncthreads();
    const ScoreGrad sg = score_grad(sums + 6 * p, eps, (double)gout[p]);
    // per-voxel gradient terms in float; the coefficients come from the double sums
    const float gA = (float)sg.gA, gB = (float)sg.gB, gC = (float)sg.gC, gD = (float)sg.gD,
                gE = (float)sg.gE, gF = (float)sg.gF;
    // per-thread partial sums in float (a few hundred terms each), combined in double
    float accf[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) accf[k] = 0.f;
    if (sg.valid) {
      Walker w;
      w.init(b, threadIdx.x, blockDim.x);
      for (int v = threadIdx.x; v < b.nv; v += blockDim.x, w.next(b)) {
        float d[3], u[3];
        pose_coords(b, Rs, ss, w, d, u);
        Stencil st;
        if (!stencil(b, u, st)) continue;
        float tq[8], mq[8];
        corners8(T, st, tq);
        corners8(M, st, mq);
        const float mr = lerp8(mq, st);
        const float tf = FILTERED ? __ldg(Tf + (int64_t)p * b.nv + v) : lerp8(tq, st);
        const float f = target_at(tg, n0, n1, n2, outside, ks, w);
        const float gm = fmaf(tf, fmaf(gC, tf, fmaf(gD, f, gB)), fmaf(f, fmaf(gF, f, gE), gA));
        const float gt = FILTERED ? __ldg(gTr_in + (int64_t)p * b.nv + v)
                                  : mr * fmaf(2.f * gC, tf, fmaf(gD, f, gB));
        // dS/du through the trilinear weights of T and M
        float e[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) e[q] = fmaf(gt, tq[q], gm * mq[q]);
        float du[3];
        lerp8_grad(e, st, du);
        if (gT != nullptr && gt != 0.f) {
          const float wx[2] = {1.f - st.f0, st.f0}, wy[2] = {1.f - st.f1, st.f1};
          const float wz[2] = {(1.f - st.f2) * gt, st.f2 * gt};
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const int i = st.base + ((q & 4) ? st.s0 : 0) + ((q & 2) ? st.s1 : 0) +
                          ((q & 1) ? st.s2 : 0);
            const float wq = wx[q >> 2] * wy[(q >> 1) & 1] * wz[q & 1];
            if (SMEM_GT) atomicAdd(gts + i, wq);
            else atomicAdd(gT + i, wq);
          }
        }
        // u_i = sum_j R[j][i] d_j + c_i: dS/dR[j][i] += du_i d_j; dS/ds_j = -sum_i R[j][i] du_i
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
          for (int i = 0; i < 3; ++i) accf[j * 3 + i] = fmaf(du[i], d[j], accf[j * 3 + i]);
        accf[9] += du[0];
        accf[10] += du[1];
        accf[11] += du[2];
      }
    }
    double acc[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) acc[k] = accf[k];
    block_sums<12>(acc, red);
    if (threadIdx.x == 0) {
      if (grad_rot)
        for (int k = 0; k < 9; ++k) grad_rot[p * 9 + k] = acc[k];
      if (grad_shift)
        for (int j = 0; j < 3; ++j)
          grad_shift[p * 3 + j] = -((double)Rs[j * 3 + 0] * acc[9] +
                                    (double)Rs[j * 3 + 1] * acc[10] +
                                    (double)Rs[j * 3 + 2] * acc[11]);
      if (grad_angles && dR)
        for (int a = 0; a < 3; ++a) {
          double s = 0.0;
          for (int k = 0; k < 9; ++k) s += acc[k] * (double)dR[p * 27 + a * 9 + k];
          grad_angles[p * 3 + a] = s;
        }
    }
  }
  if (SMEM_GT && gT != nullptr) {
    __syncthreads();
    for (int v = threadIdx.x; v < b.nv; v += blockDim.x) {
      const float g = gts[v];
      if (g != 0.f) atomicAdd(gT + v, g);
    }
  }
}

int resident_grid(const void* fn, int threads, size_t smem, int P) {
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  cudaGetLastError();
  return std::max(1, std::min(P, sms * per_sm));
}

}  // namespace

int euler_zyz(const float* angles, int P, float* R, float* dR, cudaStream_t st) {
  TM_REQUIRE(angles && R, "euler_zyz: null pointer");
  TM_REQUIRE(P > 0, "euler_zyz: no angles");
  euler_zyz_kernel<<<(unsigned)ceil_div(P, 128), 128, 0, st>>>(angles, P, R, dR);
  return check_launch("euler_zyz_kernel");
}

static int check_refine_args(const RefineArgs& a, const char* what) {
  TM_REQUIRE(a.tmpl && a.mask && a.rot && a.shifts && a.corners && a.target,
             "%s: null pointer", what);
  TM_REQUIRE(a.P > 0, "%s: no peaks", what);
  TM_REQUIRE(a.t[0] > 0 && a.t[1] > 0 && a.t[2] > 0 && a.n[0] > 0 && a.n[1] > 0 && a.n[2] > 0,
             "%s: empty template or target", what);
  TM_REQUIRE((int64_t)a.t[0] * a.t[1] * a.t[2] <= (1LL << 24),
             "%s: template of %d x %d x %d voxels is above 2^24", what, a.t[0], a.t[1], a.t[2]);
  return TM_OK;
}

int refine_rotate(const RefineArgs& a, float* Tr, cudaStream_t st) {
  TM_TRY(check_refine_args(a, "refine_rotate"));
  TM_REQUIRE(Tr, "refine_rotate: null output");
  TM_REQUIRE(a.P <= 65535, "refine_rotate: at most 65535 peaks per call");
  const int nv = a.t[0] * a.t[1] * a.t[2];
  dim3 g((unsigned)std::min<int64_t>(ceil_div(nv, kRefThreads), 512), (unsigned)a.P);
  refine_rotate_kernel<<<g, kRefThreads, 0, st>>>(a.tmpl, a.t[0], a.t[1], a.t[2], a.rot,
                                                  a.shifts, Tr);
  return check_launch("refine_rotate_kernel");
}

int refine_forward(const RefineArgs& a, const float* Tf, double* sums, float* scores,
                   cudaStream_t st) {
  TM_TRY(check_refine_args(a, "refine_forward"));
  TM_REQUIRE(sums && scores, "refine_forward: null output");
  if (Tf) {
    const int g = resident_grid((const void*)refine_forward_kernel<true>, kRefThreads, 0, a.P);
    refine_forward_kernel<true><<<g, kRefThreads, 0, st>>>(
        a.tmpl, a.mask, a.t[0], a.t[1], a.t[2], a.rot, a.shifts, a.corners, a.P, Tf, a.target,
        a.n[0], a.n[1], a.n[2], a.outside, a.eps, sums, scores);
  } else {
    const int g = resident_grid((const void*)refine_forward_kernel<false>, kRefThreads, 0, a.P);
    refine_forward_kernel<false><<<g, kRefThreads, 0, st>>>(
        a.tmpl, a.mask, a.t[0], a.t[1], a.t[2], a.rot, a.shifts, a.corners, a.P, nullptr,
        a.target, a.n[0], a.n[1], a.n[2], a.outside, a.eps, sums, scores);
  }
  return check_launch("refine_forward_kernel");
}

int refine_grad_filtered(const RefineArgs& a, const float* Tf, const double* sums,
                         const float* grad_scores, float* gTf, cudaStream_t st) {
  TM_TRY(check_refine_args(a, "refine_grad_filtered"));
  TM_REQUIRE(Tf && sums && grad_scores && gTf, "refine_grad_filtered: null pointer");
  TM_REQUIRE(a.P <= 65535, "refine_grad_filtered: at most 65535 peaks per call");
  const int nv = a.t[0] * a.t[1] * a.t[2];
  dim3 g((unsigned)std::min<int64_t>(ceil_div(nv, kRefThreads), 512), (unsigned)a.P);
  refine_grad_filtered_kernel<<<g, kRefThreads, 0, st>>>(
      a.mask, a.t[0], a.t[1], a.t[2], a.rot, a.shifts, a.corners, Tf, a.target, a.n[0], a.n[1],
      a.n[2], a.outside, a.eps, sums, grad_scores, gTf);
  return check_launch("refine_grad_filtered_kernel");
}

template <bool FILTERED, bool SMEM>
static int launch_backward(const RefineArgs& a, const float* Tf, const float* gTr,
                           const double* sums, const float* gout, const float* dR, double* gRot,
                           double* gShift, double* gAng, float* gT, cudaStream_t st) {
  constexpr int kThreads = SMEM ? kRefBackSmemThreads : kRefThreads;
  const int nv = a.t[0] * a.t[1] * a.t[2];
  const size_t smem = SMEM ? (size_t)nv * sizeof(float) : 0;
  auto fn = refine_backward_kernel<FILTERED, SMEM, kThreads>;
  if (SMEM)
    TM_TRY(cuda_status(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                            (int)smem),
                       "refine_backward: shared memory attribute"));
  const int g = resident_grid((const void*)fn, kThreads, smem, a.P);
  fn<<<g, kThreads, smem, st>>>(a.tmpl, a.mask, a.t[0], a.t[1], a.t[2], a.rot, a.shifts,
                                   a.corners, a.P, Tf, gTr, a.target, a.n[0], a.n[1], a.n[2],
                                   a.outside, a.eps, sums, gout, dR, gRot, gShift, gAng, gT);
  return check_launch("refine_backward_kernel");
}

int refine_backward(const RefineArgs& a, const float* Tf, const float* gTr, const double* sums,
                    const float* grad_scores, const float* dR, double* grad_rot,
                    double* grad_shift, double* grad_angles, float* grad_tmpl,
                    cudaStream_t st) {
  TM_TRY(check_refine_args(a, "refine_backward"));
  TM_REQUIRE(sums && grad_scores, "refine_backward: null pointer");
  TM_REQUIRE((Tf == nullptr) == (gTr == nullptr),
             "refine_backward: the filtered template and its gradient go together");
  TM_REQUIRE(!grad_angles || dR, "refine_backward: angle gradients need dR");
  const int nv = a.t[0] * a.t[1] * a.t[2];
  const bool smem = grad_tmpl != nullptr && nv <= kSmemGradMaxVoxels;
  if (Tf) {
    if (smem)
      return launch_backward<true, true>(a, Tf, gTr, sums, grad_scores, dR, grad_rot, grad_shift,
                                         grad_angles, grad_tmpl, st);
    return launch_backward<true, false>(a, Tf, gTr, sums, grad_scores, dR, grad_rot, grad_shift,
                                        grad_angles, grad_tmpl, st);
  }
  if (smem)
    return launch_backward<false, true>(a, nullptr, nullptr, sums, grad_scores, dR, grad_rot,
                                        grad_shift, grad_angles, grad_tmpl, st);
  return launch_backward<false, false>(a, nullptr, nullptr, sums, grad_scores, dR, grad_rot,
                                       grad_shift, grad_angles, grad_tmpl, st);
}

}  // namespace tmb
