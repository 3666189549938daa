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

// d = o - c - s and u = R^T d + c for template voxel v; R row-major.
__device__ __forceinline__ void pose_coords(const Box& b, const float* R, const float* s, int v,
                                            int o[3], float d[3], float u[3]) {
  o[2] = v % b.t2;
  o[1] = (v / b.t2) % b.t1;
  o[0] = v / (b.t1 * b.t2);
  d[0] = (float)o[0] - b.c0 - s[0];
  d[1] = (float)o[1] - b.c1 - s[1];
  d[2] = (float)o[2] - b.c2 - s[2];
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

__device__ __forceinline__ int corner_index(const Stencil& st, int q) {
  return st.base + ((q & 4) ? st.s0 : 0) + ((q & 2) ? st.s1 : 0) + ((q & 1) ? st.s2 : 0);
}

__device__ __forceinline__ float corner_weight(const Stencil& st, int q) {
  const float w0 = (q & 4) ? st.f0 : 1.f - st.f0;
  const float w1 = (q & 2) ? st.f1 : 1.f - st.f1;
  const float w2 = (q & 1) ? st.f2 : 1.f - st.f2;
  return w0 * w1 * w2;
}

__device__ __forceinline__ float target_at(const float* __restrict__ tg, int n0, int n1, int n2,
                                           float outside, const int k[3], const int o[3]) {
  const int x = k[0] + o[0], y = k[1] + o[1], z = k[2] + o[2];
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
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < b.nv; v += gridDim.x * blockDim.x) {
    int o[3];
    float d[3], u[3];
    pose_coords(b, Rs, ss, v, o, d, u);
    Stencil st;
    float a = 0.f;
    if (stencil(b, u, st)) {
#pragma unroll
      for (int q = 0; q < 8; ++q) a += corner_weight(st, q) * __ldg(T + corner_index(st, q));
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
    for (int v = threadIdx.x; v < b.nv; v += blockDim.x) {
      int o[3];
      float d[3], u[3];
      pose_coords(b, Rs, ss, v, o, d, u);
      Stencil st;
      if (!stencil(b, u, st)) continue;
      float mr = 0.f, tr = 0.f;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int i = corner_index(st, q);
        const float w = corner_weight(st, q);
        mr += w * __ldg(M + i);
        if (!FILTERED) tr += w * __ldg(T + i);
      }
      if (mr == 0.f) continue;
      const double m = mr;
      const double tf = FILTERED ? (double)__ldg(Tf + (int64_t)p * b.nv + v) : (double)tr;
      const double f = target_at(tg, n0, n1, n2, outside, ks, o);
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
  for (int v = blockIdx.x * blockDim.x + threadIdx.x; v < b.nv; v += gridDim.x * blockDim.x) {
    float g = 0.f;
    if (sg.valid) {
      int o[3];
      float d[3], u[3];
      pose_coords(b, Rs, ss, v, o, d, u);
      Stencil st;
      if (stencil(b, u, st)) {
        float mr = 0.f;
#pragma unroll
        for (int q = 0; q < 8; ++q) mr += corner_weight(st, q) * __ldg(M + corner_index(st, q));
        if (mr != 0.f) {
          const double tf = __ldg(Tf + (int64_t)p * b.nv + v);
          const double f = target_at(tg, n0, n1, n2, outside, ks, o);
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
    double acc[12];
#pragma unroll
    for (int k = 0; k < 12; ++k) acc[k] = 0.0;
    if (sg.valid) {
      for (int v = threadIdx.x; v < b.nv; v += blockDim.x) {
        int o[3];
        float d[3], u[3];
        pose_coords(b, Rs, ss, v, o, d, u);
        Stencil st;
        if (!stencil(b, u, st)) continue;
        float tq[8], mq[8];
        float mr = 0.f, tr = 0.f;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int i = corner_index(st, q);
          const float w = corner_weight(st, q);
          tq[q] = __ldg(T + i);
          mq[q] = __ldg(M + i);
          mr += w * mq[q];
          tr += w * tq[q];
        }
        const double tf = FILTERED ? (double)__ldg(Tf + (int64_t)p * b.nv + v) : (double)tr;
        const double f = target_at(tg, n0, n1, n2, outside, ks, o);
        const float gm = (float)(sg.gA + tf * (sg.gB + sg.gC * tf + sg.gD * f) +
                                 f * (sg.gE + sg.gF * f));
        const float gt = FILTERED
                             ? __ldg(gTr_in + (int64_t)p * b.nv + v)
                             : (float)((double)mr * (sg.gB + 2.0 * sg.gC * tf + sg.gD * f));
        // dS/du through the corner weights; fractional derivative signs per axis
        float e[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) e[q] = gt * tq[q] + gm * mq[q];
        const float f0 = st.f0, f1 = st.f1, f2 = st.f2;
        // differences along axis 2, then bilinear weights on the other two
        const float a00 = e[1] - e[0], a01 = e[3] - e[2], a10 = e[5] - e[4], a11 = e[7] - e[6];
        const float du2 = (1.f - f0) * ((1.f - f1) * a00 + f1 * a01) +
                          f0 * ((1.f - f1) * a10 + f1 * a11);
        const float l00 = e[0] + f2 * (e[1] - e[0]), l01 = e[2] + f2 * (e[3] - e[2]);
        const float l10 = e[4] + f2 * (e[5] - e[4]), l11 = e[6] + f2 * (e[7] - e[6]);
        const float du1 = (1.f - f0) * (l01 - l00) + f0 * (l11 - l10);
        const float du0 = ((1.f - f1) * l10 + f1 * l11) - ((1.f - f1) * l00 + f1 * l01);
        if (gT != nullptr && gt != 0.f) {
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            const float w = corner_weight(st, q) * gt;
            if (SMEM_GT) atomicAdd(gts + corner_index(st, q), w);
            else atomicAdd(gT + corner_index(st, q), w);
          }
        }
        // u_i = sum_j R[j][i] d_j + c_i: dS/dR[j][i] += du_i d_j; dS/ds_j = -sum_i R[j][i] du_i
        const float du[3] = {du0, du1, du2};
#pragma unroll
        for (int j = 0; j < 3; ++j)
#pragma unroll
          for (int i = 0; i < 3; ++i) acc[j * 3 + i] += (double)(du[i] * d[j]);
        acc[9] += du0;
        acc[10] += du1;
        acc[11] += du2;
      }
    }
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
