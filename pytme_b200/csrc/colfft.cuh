// Column FFTs of length N (a power of two, 64..1024) for the fused scan passes.
//
// A CTA transforms W columns (lines) of a tile at once; each line is handled by
// T = N/8 threads that hold 8 complex values each, so a thread's data stay in
// registers between stages and shared memory is only used to exchange them.
//
// The forward transform is an in-place decimation-in-frequency FFT with radix-8
// stages (a final radix-4 or radix-2 stage when N is not a power of 8). Stage s
// works on sub-problems of size L_s (L_0 = N, L_{s+1} = L_s / R_s): butterfly
// (p, q) reads positions p*L + q + (L/R)*r, computes the R-point DFT, multiplies
// output j by W_L^(j*q) and writes it back to position p*L + q + (L/R)*j. The same
// thread reads and writes the same positions, so a stage needs no barrier between
// its loads and stores. After the last stage position `pos` holds frequency
// digitrev(pos) (the mixed-radix digits of pos in reverse order).
//
// The adjoint stages (conjugate twiddles applied before an inverse R-point DFT, in
// reverse stage order) undo this: starting from digit-reversed data they return
// natural order, i.e. an unnormalised inverse DFT. The fused x pass runs
//   stage 0 (loads from global) ... last stage | product | adjoint last ... adjoint 0
// with the product and both last stages in registers; the y pass runs the forward
// stage structure with conjugate twiddles (an inverse DFT with digit-reversed
// output) and stores rows at digitrev(pos).
//
// Shared-memory layout of a tile: element (line l, position pos) sits at
// pos*W + l + W*(pos >> 3). With W lines spanning a warp this keeps every stage's
// warp-wide access to the minimum number of wavefronts.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

#include "fft_smem.cuh"

namespace tmb {
namespace colfft {

using fft::cadd;
using fft::cconj;
using fft::cmul;
using fft::csub;

constexpr int num_stages(int n) {
  int k = 0;
  while (n >= 8) { n /= 8; ++k; }
  return k + (n > 1 ? 1 : 0);
}
constexpr int stage_size(int n, int s) {
  for (int i = 0; i < s; ++i) n /= 8;
  return n;
}
constexpr int stage_radix(int n, int s) {
  int l = stage_size(n, s);
  return l >= 8 ? 8 : l;
}

// frequency index held at position pos after the forward stages
template <int N>
__device__ __forceinline__ int digitrev(int pos) {
  constexpr int S = num_stages(N);
  int k = 0, mul = 1;
#pragma unroll
  for (int s = 0; s < S; ++s) {
    const int R = stage_radix(N, s);
    const int stride = stage_size(N, s) / R;  // N / (R_0 ... R_s)
    const int digit = (pos / stride) % R;
    k += digit * mul;
    mul *= R;
  }
  return k;
}

template <int W>
__device__ __forceinline__ int saddr(int l, int pos) {
  return pos * W + l + W * (pos >> 3);
}

template <int N>
constexpr int smem_elems(int W) {
  return (N + N / 8) * W;
}

template <int R, int DIR>
__device__ __forceinline__ void dftR(float2* v) {
  if constexpr (R == 8) fft::dft8<DIR>(v);
  else if constexpr (R == 4) fft::dft4<DIR>(v);
  else fft::dft2<DIR>(v);
}

// Twiddles w^j (j = 1..R-1) of one butterfly from a single table read: powers by
// repeated complex multiplication (error ~j ulp, far below the FP32 FFT's own).
template <int R>
__device__ __forceinline__ void twiddle_powers(float2 (&w)[R], float2 w1) {
  w[1] = w1;
#pragma unroll
  for (int j = 2; j < R; ++j) w[j] = cmul(w[j - 1], w1);
}

// One forward-structured DIF stage s (DIR -1: forward DFT, +1: inverse DFT with
// conjugate twiddles) on values already in registers; twiddles applied after the
// butterflies. v holds the thread's 8 values in the order (butterfly i, r).
template <int N, int S, int DIR>
__device__ __forceinline__ void dif_stage_regs(float2 (&v)[8], int t, const float2* tw) {
  constexpr int L = stage_size(N, S);
  constexpr int R = stage_radix(N, S);
  constexpr int NB = 8 / R;
  constexpr int LR = L / R;
#pragma unroll
  for (int i = 0; i < NB; ++i) {
    dftR<R, DIR>(&v[i * R]);
    if constexpr (LR > 1) {
      const int b = t * NB + i;
      const int q = b % LR;
      float2 w1 = tw[q * (N / L)];
      if (DIR > 0) w1 = cconj(w1);
      float2 w[R];
      twiddle_powers<R>(w, w1);
#pragma unroll
      for (int j = 1; j < R; ++j) v[i * R + j] = cmul(v[i * R + j], w[j]);
    }
  }
}

// Adjoint of a DIF stage: conjugate twiddles first, then the inverse DFT.
template <int N, int S>
__device__ __forceinline__ void dif_stage_adjoint_regs(float2 (&v)[8], int t, const float2* tw) {
  constexpr int L = stage_size(N, S);
  constexpr int R = stage_radix(N, S);
  constexpr int NB = 8 / R;
  constexpr int LR = L / R;
#pragma unroll
  for (int i = 0; i < NB; ++i) {
    if constexpr (LR > 1) {
      const int b = t * NB + i;
      const int q = b % LR;
      float2 w[R];
      twiddle_powers<R>(w, cconj(tw[q * (N / L)]));
#pragma unroll
      for (int j = 1; j < R; ++j) v[i * R + j] = cmul(v[i * R + j], w[j]);
    }
    dftR<R, 1>(&v[i * R]);
  }
}

// position of value (i, r) of thread t at stage S
template <int N, int S>
__device__ __forceinline__ int stage_pos(int t, int i, int r) {
  constexpr int L = stage_size(N, S);
  constexpr int R = stage_radix(N, S);
  constexpr int NB = 8 / R;
  constexpr int LR = L / R;
  const int b = t * NB + i;
  const int p = b / LR, q = b % LR;
  return p * L + q + LR * r;
}

// Shared-memory address of value (i, r) of thread t at stage S, written as a per-thread
// base plus a compile-time offset: positions p*L + q + LR*r with LR a multiple of 8 (or
// LR = 1 on the last stage, where p*L is a multiple of 8 and q = 0) keep pos >> 3 affine
// in (i, r), so the padded address is affine too.
template <int N, int W, int S>
__device__ __forceinline__ int stage_base(int l, int t) {
  constexpr int L = stage_size(N, S);
  constexpr int R = stage_radix(N, S);
  constexpr int NB = 8 / R;
  constexpr int LR = L / R;
  const int b = t * NB;
  const int pos = (b / LR) * L + (b % LR);
  return saddr<W>(l, pos);
}

template <int N, int W, int S>
__device__ __forceinline__ constexpr int stage_off(int i, int r) {
  constexpr int L = stage_size(N, S);
  constexpr int R = stage_radix(N, S);
  constexpr int LR = L / R;
  if constexpr (LR > 1) {
    // radix-8 stage, one butterfly per thread (q < LR): (q + LR*r) >> 3 equals
    // (q >> 3) + (LR*r >> 3) because LR*r is a multiple of 8 or q + (LR*r mod 8) < 8
    return (LR * r) * W + W * ((LR * r) >> 3);
  } else {
    // LR == 1: positions b*L + r with b = t*NB + i; t*NB*L is a multiple of 8
    const int d = i * L + r;
    return d * W + W * (d >> 3);
  }
}

template <int N, int W, int S>
__device__ __forceinline__ void load_stage(float2 (&v)[8], const float2* sm, int l, int t) {
  constexpr int R = stage_radix(N, S);
  constexpr int NB = 8 / R;
  const float2* base = sm + stage_base<N, W, S>(l, t);
#pragma unroll
  for (int i = 0; i < NB; ++i)
#pragma unroll
    for (int r = 0; r < R; ++r) v[i * R + r] = base[stage_off<N, W, S>(i, r)];
}

template <int N, int W, int S>
__device__ __forceinline__ void store_stage(const float2 (&v)[8], float2* sm, int l, int t) {
  constexpr int R = stage_radix(N, S);
  constexpr int NB = 8 / R;
  float2* base = sm + stage_base<N, W, S>(l, t);
#pragma unroll
  for (int i = 0; i < NB; ++i)
#pragma unroll
    for (int r = 0; r < R; ++r) base[stage_off<N, W, S>(i, r)] = v[i * R + r];
}

// Frequency index of value (i, r) after the last forward stage: the last digit r is the
// most significant frequency digit, so k = digitrev(p*R) + r*(N/R) with p = t*NB + i.
template <int N>
__device__ __forceinline__ int out_index(int t, int i, int r) {
  constexpr int S = num_stages(N) - 1;
  constexpr int R = stage_radix(N, S);
  constexpr int NB = 8 / R;
  return digitrev<N>((t * NB + i) * R) + r * (N / R);
}

// Forward (DIR=-1) or inverse (DIR=+1) DIF transform of the thread's line: v holds
// the natural-order inputs x[t + T*r] on entry and the outputs at the last stage's
// positions on exit (frequency/position digitrev(stage_pos<N, last>(t, i, r))).
// Stage 0 runs on v directly; later stages exchange through shared memory.
template <int N, int W, int DIR>
__device__ __forceinline__ void dif_forward(float2 (&v)[8], float2* sm, const float2* tw, int l,
                                            int t) {
  constexpr int NS = num_stages(N);
  dif_stage_regs<N, 0, DIR>(v, t, tw);
  // stage 0 outputs j sit at positions t + T*j, i.e. stage_pos<N,0>(t, 0, j)
  store_stage<N, W, 0>(v, sm, l, t);
  __syncthreads();
  if constexpr (NS > 1) {
    load_stage<N, W, 1>(v, sm, l, t);
    dif_stage_regs<N, 1, DIR>(v, t, tw);
  }
  if constexpr (NS > 2) {
    store_stage<N, W, 1>(v, sm, l, t);
    __syncthreads();
    load_stage<N, W, 2>(v, sm, l, t);
    dif_stage_regs<N, 2, DIR>(v, t, tw);
  }
  if constexpr (NS > 3) {
    store_stage<N, W, 2>(v, sm, l, t);
    __syncthreads();
    load_stage<N, W, 3>(v, sm, l, t);
    dif_stage_regs<N, 3, DIR>(v, t, tw);
  }
}

// Adjoint of dif_forward<.., -1>: from the last stage's positions back to natural
// order x[t + T*r] (unnormalised inverse DFT). Ends with v in natural order.
template <int N, int W>
__device__ __forceinline__ void dif_adjoint(float2 (&v)[8], float2* sm, const float2* tw, int l,
                                            int t) {
  constexpr int NS = num_stages(N);
  if constexpr (NS > 3) {
    dif_stage_adjoint_regs<N, 3>(v, t, tw);
    store_stage<N, W, 3>(v, sm, l, t);
    __syncthreads();
    load_stage<N, W, 2>(v, sm, l, t);
  }
  if constexpr (NS > 2) {
    dif_stage_adjoint_regs<N, 2>(v, t, tw);
    store_stage<N, W, 2>(v, sm, l, t);
    __syncthreads();
    load_stage<N, W, 1>(v, sm, l, t);
  }
  if constexpr (NS > 1) {
    dif_stage_adjoint_regs<N, 1>(v, t, tw);
    store_stage<N, W, 1>(v, sm, l, t);
    __syncthreads();
    load_stage<N, W, 0>(v, sm, l, t);
  }
  dif_stage_adjoint_regs<N, 0>(v, t, tw);
}

template <int N>
__device__ __forceinline__ int last_pos(int t, int i, int r) {
  return stage_pos<N, num_stages(N) - 1>(t, i, r);
}

}  // namespace colfft
}  // namespace tmb
