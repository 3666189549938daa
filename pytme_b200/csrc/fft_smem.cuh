// Batched 1D complex FFTs of lines held in shared memory (Stockham autosort).
//
// A CTA transforms `nlines` lines of length n in place. Element i of line l
// lives at buf[l * ls + i * es], so both "interleaved" tiles (lines fastest,
// es = nlines, ls = 1) and "row-major" tiles (es = 1) are supported. Each pass
// of radix R loads R elements per butterfly into registers, applies the
// twiddles, runs an R-point DFT and, after a barrier, stores the outputs in
// autosorted order, so one buffer suffices. The number of butterflies per
// thread per pass is bounded at compile time (MAXE / R); launches keep
// n * nlines <= MAXE * nthreads.
//
// Twiddles come from a table tw[i] = exp(-2 pi i * i / N) in shared memory,
// computed on the host in double precision and rounded to float; a line of
// length n with n | N reads it with stride N / n.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>

namespace tmb {
namespace fft {

constexpr int kMaxPasses = 12;

struct LinePlan {
  int n;                    // transform length
  int npass;                // number of radix passes
  int radix[kMaxPasses];    // radices, first pass first
};

__device__ __forceinline__ float2 cadd(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 csub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 cmul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ float2 cconj(float2 a) { return make_float2(a.x, -a.y); }
__device__ __forceinline__ float2 cscale(float2 a, float s) { return make_float2(a.x * s, a.y * s); }

// multiply by -i (forward, DIR=-1) or +i (inverse, DIR=+1)
template <int DIR>
__device__ __forceinline__ float2 rot90(float2 a) {
  return DIR < 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}

template <int DIR>
__device__ __forceinline__ float2 twiddle(const float2* tw, int idx) {
  float2 w = tw[idx];
  return DIR < 0 ? w : cconj(w);
}

// ---- small DFTs in registers; DIR = -1 computes sum_j v_j exp(-2 pi i jk/R)
template <int DIR>
__device__ __forceinline__ void dft2(float2* v) {
  float2 a = v[0], b = v[1];
  v[0] = cadd(a, b);
  v[1] = csub(a, b);
}

template <int DIR>
__device__ __forceinline__ void dft3(float2* v) {
  const float c = -0.5f;
  const float s = (DIR < 0 ? -1.f : 1.f) * 0.86602540378443864676f;
  float2 t1 = cadd(v[1], v[2]);
  float2 t2 = csub(v[1], v[2]);
  float2 m = make_float2(v[0].x + c * t1.x, v[0].y + c * t1.y);
  float2 r = make_float2(-s * t2.y, s * t2.x);  // i * s * t2
  v[0] = cadd(v[0], t1);
  v[1] = cadd(m, r);
  v[2] = csub(m, r);
}

template <int DIR>
__device__ __forceinline__ void dft4(float2* v) {
  float2 a0 = cadd(v[0], v[2]);
  float2 a1 = csub(v[0], v[2]);
  float2 a2 = cadd(v[1], v[3]);
  float2 a3 = rot90<DIR>(csub(v[1], v[3]));
  v[0] = cadd(a0, a2);
  v[2] = csub(a0, a2);
  v[1] = cadd(a1, a3);
  v[3] = csub(a1, a3);
}

template <int DIR>
__device__ __forceinline__ void dft5(float2* v) {
  // Winograd-style 5-point DFT with constants from cos/sin(2 pi / 5), cos/sin(4 pi / 5).
  const float c1 = 0.30901699437494742410f;   // cos(2pi/5)
  const float c2 = -0.80901699437494742410f;  // cos(4pi/5)
  const float sg = DIR < 0 ? -1.f : 1.f;
  const float s1 = sg * 0.95105651629515357212f;  // sin(2pi/5)
  const float s2 = sg * 0.58778525229247312917f;  // sin(4pi/5)
  float2 a1 = cadd(v[1], v[4]), b1 = csub(v[1], v[4]);
  float2 a2 = cadd(v[2], v[3]), b2 = csub(v[2], v[3]);
  float2 x0 = v[0];
  float2 m1 = make_float2(x0.x + c1 * a1.x + c2 * a2.x, x0.y + c1 * a1.y + c2 * a2.y);
  float2 m2 = make_float2(x0.x + c2 * a1.x + c1 * a2.x, x0.y + c2 * a1.y + c1 * a2.y);
  // i * (s1 b1 + s2 b2), i * (s2 b1 - s1 b2)
  float2 n1 = make_float2(-(s1 * b1.y + s2 * b2.y), s1 * b1.x + s2 * b2.x);
  float2 n2 = make_float2(-(s2 * b1.y - s1 * b2.y), s2 * b1.x - s1 * b2.x);
  v[0] = make_float2(x0.x + a1.x + a2.x, x0.y + a1.y + a2.y);
  v[1] = cadd(m1, n1);
  v[4] = csub(m1, n1);
  v[2] = cadd(m2, n2);
  v[3] = csub(m2, n2);
}

template <int DIR>
__device__ __forceinline__ void dft8(float2* v) {
  const float h = 0.70710678118654752440f;
  float2 e[4] = {v[0], v[2], v[4], v[6]};
  float2 o[4] = {v[1], v[3], v[5], v[7]};
  dft4<DIR>(e);
  dft4<DIR>(o);
  // o[k] *= exp(DIR * 2 pi i k / 8)
  o[1] = DIR < 0 ? make_float2(h * (o[1].x + o[1].y), h * (o[1].y - o[1].x))
                 : make_float2(h * (o[1].x - o[1].y), h * (o[1].y + o[1].x));
  o[2] = rot90<DIR>(o[2]);
  o[3] = DIR < 0 ? make_float2(h * (o[3].y - o[3].x), -h * (o[3].x + o[3].y))
                 : make_float2(-h * (o[3].x + o[3].y), h * (o[3].x - o[3].y));
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    v[k] = cadd(e[k], o[k]);
    v[k + 4] = csub(e[k], o[k]);
  }
}

// Generic odd radix (7, 11, 13): direct DFT with roots of unity read from the
// twiddle table; tw_r(k) = exp(-2 pi i k / R) sits at table index k * N / R.
template <int R, int DIR>
__device__ __forceinline__ void dft_generic(float2* v, const float2* tw, int root_stride) {
  float2 out[R];
#pragma unroll
  for (int k = 0; k < R; ++k) {
    float2 acc = v[0];
#pragma unroll
    for (int j = 1; j < R; ++j) {
      int e = (j * k) % R;
      acc = cadd(acc, cmul(v[j], twiddle<DIR>(tw, e * root_stride)));
    }
    out[k] = acc;
  }
#pragma unroll
  for (int k = 0; k < R; ++k) v[k] = out[k];
}

template <int R, int DIR>
__device__ __forceinline__ void dft(float2* v, const float2* tw, int table_n) {
  if constexpr (R == 2) dft2<DIR>(v);
  else if constexpr (R == 3) dft3<DIR>(v);
  else if constexpr (R == 4) dft4<DIR>(v);
  else if constexpr (R == 5) dft5<DIR>(v);
  else if constexpr (R == 8) dft8<DIR>(v);
  else dft_generic<R, DIR>(v, tw, table_n / R);
}

// One Stockham pass of radix R over all lines.
//   Ns: product of the radices of earlier passes.
//   tws: table stride for this line length (table_n / n).
template <int R, int DIR, int MAXE, bool LINES_FAST>
__device__ __forceinline__ void stockham_pass(float2* buf, int n, int Ns, int nlines, int ls,
                                              int es, const float2* tw, int tws, int table_n,
                                              int tid, int nthr) {
  constexpr int MAXB = (MAXE + R - 1) / R;
  const int nb = n / R;
  const int total = nb * nlines;
  const int tstep = (n / (Ns * R)) * tws;
  float2 v[MAXB][R];
#pragma unroll
  for (int c = 0; c < MAXB; ++c) {
    int w = tid + c * nthr;
    if (w < total) {
      int l, j;
      if (LINES_FAST) { l = w % nlines; j = w / nlines; } else { j = w % nb; l = w / nb; }
      const float2* base = buf + l * ls;
#pragma unroll
      for (int r = 0; r < R; ++r) v[c][r] = base[(j + r * nb) * es];
      int k = j % Ns;
      if (k != 0) {
#pragma unroll
        for (int r = 1; r < R; ++r) v[c][r] = cmul(v[c][r], twiddle<DIR>(tw, r * k * tstep));
      }
      dft<R, DIR>(v[c], tw, table_n);
    }
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < MAXB; ++c) {
    int w = tid + c * nthr;
    if (w < total) {
      int l, j;
      if (LINES_FAST) { l = w % nlines; j = w / nlines; } else { j = w % nb; l = w / nb; }
      float2* base = buf + l * ls;
      int k = j % Ns;
      int o = (j / Ns) * Ns * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) base[(o + r * Ns) * es] = v[c][r];
    }
  }
  __syncthreads();
}

// Stockham pass with compile-time length, radix and span.
template <int N, int R, int Ns, int DIR, int MAXE, bool LINES_FAST>
__device__ __forceinline__ void stockham_pass_ct(float2* buf, int nlines, int ls, int es,
                                                 const float2* tw, int tws, int table_n, int tid,
                                                 int nthr) {
  constexpr int MAXB = (MAXE + R - 1) / R;
  constexpr int nb = N / R;
  constexpr int tstep = N / (Ns * R);
  const int total = nb * nlines;
  float2 v[MAXB][R];
#pragma unroll
  for (int c = 0; c < MAXB; ++c) {
    int w = tid + c * nthr;
    if (w < total) {
      int l, j;
      if (LINES_FAST) { l = w % nlines; j = w / nlines; } else { j = w % nb; l = w / nb; }
      const float2* base = buf + l * ls;
#pragma unroll
      for (int r = 0; r < R; ++r) v[c][r] = base[(j + r * nb) * es];
      if constexpr (Ns > 1) {
        const int k = j % Ns;
#pragma unroll
        for (int r = 1; r < R; ++r) v[c][r] = cmul(v[c][r], twiddle<DIR>(tw, r * k * tstep * tws));
      }
      dft<R, DIR>(v[c], tw, table_n);
    }
  }
  __syncthreads();
#pragma unroll
  for (int c = 0; c < MAXB; ++c) {
    int w = tid + c * nthr;
    if (w < total) {
      int l, j;
      if (LINES_FAST) { l = w % nlines; j = w / nlines; } else { j = w % nb; l = w / nb; }
      float2* base = buf + l * ls;
      const int k = j % Ns;
      const int o = (j / Ns) * Ns * R + k;
#pragma unroll
      for (int r = 0; r < R; ++r) base[(o + r * Ns) * es] = v[c][r];
    }
  }
  __syncthreads();
}

// Full transform of all lines: runs the plan's passes. Callers must
// __syncthreads() before (data loaded) — the routine ends synchronised.
// Radices 2, 3, 4, 5 and 8 are compiled in (every 5-smooth length); plans with
// other radices are rejected on the host (supported_radices).
template <int DIR, int MAXE, bool LINES_FAST>
__device__ __forceinline__ void fft_lines(float2* buf, const LinePlan& p, int nlines, int ls, int es,
                          const float2* tw, int table_n, int tid, int nthr) {
  const int tws = table_n / p.n;
  int Ns = 1;
  for (int s = 0; s < p.npass; ++s) {
    const int R = p.radix[s];
    switch (R) {
      case 8: stockham_pass<8, DIR, MAXE, LINES_FAST>(buf, p.n, Ns, nlines, ls, es, tw, tws, table_n, tid, nthr); break;
      case 4: stockham_pass<4, DIR, MAXE, LINES_FAST>(buf, p.n, Ns, nlines, ls, es, tw, tws, table_n, tid, nthr); break;
      case 2: stockham_pass<2, DIR, MAXE, LINES_FAST>(buf, p.n, Ns, nlines, ls, es, tw, tws, table_n, tid, nthr); break;
      case 3: stockham_pass<3, DIR, MAXE, LINES_FAST>(buf, p.n, Ns, nlines, ls, es, tw, tws, table_n, tid, nthr); break;
      case 5: stockham_pass<5, DIR, MAXE, LINES_FAST>(buf, p.n, Ns, nlines, ls, es, tw, tws, table_n, tid, nthr); break;
      default: break;
    }
    Ns *= R;
  }
}

// ---- compile-time length: the radix list and every stride constant-fold.
constexpr int ct_npass(int n) {
  int m = n, e2 = 0, k = 0;
  while (m % 2 == 0) { m /= 2; ++e2; }
  int eights = e2 / 3, rem = e2 % 3;
  if (rem == 1 && eights > 0) { eights -= 1; k += 2; }
  else if (rem == 1) k += 1;
  else if (rem == 2) k += 1;
  k += eights;
  while (m % 3 == 0) { m /= 3; ++k; }
  while (m % 5 == 0) { m /= 5; ++k; }
  return m == 1 ? k : -1;
}

constexpr int ct_radix(int n, int idx) {
  int m = n, e2 = 0, k = 0;
  int r[kMaxPasses] = {};
  while (m % 2 == 0) { m /= 2; ++e2; }
  int eights = e2 / 3, rem = e2 % 3;
  if (rem == 1 && eights > 0) { eights -= 1; r[k++] = 4; r[k++] = 4; }
  else if (rem == 1) r[k++] = 2;
  else if (rem == 2) r[k++] = 4;
  for (int i = 0; i < eights; ++i) r[k++] = 8;
  while (m % 3 == 0) { m /= 3; r[k++] = 3; }
  while (m % 5 == 0) { m /= 5; r[k++] = 5; }
  return r[idx];
}

constexpr int ct_ns(int n, int idx) {
  int ns = 1;
  for (int i = 0; i < idx; ++i) ns *= ct_radix(n, i);
  return ns;
}

template <int N, int P, int DIR, int MAXE, bool LINES_FAST>
__device__ __forceinline__ void ct_passes(float2* buf, int nlines, int ls, int es, const float2* tw,
                                          int table_n, int tid, int nthr) {
  if constexpr (P < ct_npass(N)) {
    constexpr int R = ct_radix(N, P);
    constexpr int Ns = ct_ns(N, P);
    stockham_pass_ct<N, R, Ns, DIR, MAXE, LINES_FAST>(buf, nlines, ls, es, tw, table_n / N,
                                                     table_n, tid, nthr);
    ct_passes<N, P + 1, DIR, MAXE, LINES_FAST>(buf, nlines, ls, es, tw, table_n, tid, nthr);
  }
}

template <int N, int DIR, int MAXE, bool LINES_FAST>
__device__ __forceinline__ void fft_lines_ct(float2* buf, int nlines, int ls, int es,
                                             const float2* tw, int table_n, int tid, int nthr) {
  static_assert(ct_npass(N) > 0, "length must be 5-smooth");
  ct_passes<N, 0, DIR, MAXE, LINES_FAST>(buf, nlines, ls, es, tw, table_n, tid, nthr);
}

// ---- small DFTs of compile-time size in registers (DIR -1 forward, +1 inverse)
// 16 = 4 x 4 Cooley-Tukey with its constant twiddles; 6, 10, 12, 15, 20 = Good-Thomas
// prime-factor forms (coprime factors, no twiddles).
template <int DIR>
__device__ __forceinline__ void dft16(float2* v) {
  const float c1 = 0.92387953251128675613f, s1 = 0.38268343236508977173f;
  const float h = 0.70710678118654752440f;
  const float sg = DIR < 0 ? -1.f : 1.f;
  // w16^j for j = 0..9 (exp(DIR * 2 pi i j / 16))
  const float2 w[10] = {make_float2(1.f, 0.f), make_float2(c1, sg * s1), make_float2(h, sg * h),
                        make_float2(s1, sg * c1), make_float2(0.f, sg * 1.f),
                        make_float2(-s1, sg * c1), make_float2(-h, sg * h),
                        make_float2(-c1, sg * s1), make_float2(-1.f, 0.f),
                        make_float2(-c1, -sg * s1)};
  float2 a[4][4];
#pragma unroll
  for (int n1 = 0; n1 < 4; ++n1) {
#pragma unroll
    for (int n2 = 0; n2 < 4; ++n2) a[n1][n2] = v[4 * n2 + n1];
    dft4<DIR>(a[n1]);
#pragma unroll
    for (int k2 = 1; k2 < 4; ++k2) {
      const int e = n1 * k2;
      if (e) a[n1][k2] = cmul(a[n1][k2], w[e]);
    }
  }
#pragma unroll
  for (int k2 = 0; k2 < 4; ++k2) {
    float2 b[4] = {a[0][k2], a[1][k2], a[2][k2], a[3][k2]};
    dft4<DIR>(b);
#pragma unroll
    for (int k1 = 0; k1 < 4; ++k1) v[k2 + 4 * k1] = b[k1];
  }
}

constexpr int modinv(int a, int m) {
  for (int x = 1; x < m; ++x)
    if ((a * x) % m == 1) return x;
  return 1;
}

template <int R, int DIR>
__device__ __forceinline__ void dft_prime_or_pow2(float2* v) {
  if constexpr (R == 2) dft2<DIR>(v);
  else if constexpr (R == 3) dft3<DIR>(v);
  else if constexpr (R == 4) dft4<DIR>(v);
  else if constexpr (R == 5) dft5<DIR>(v);
  else if constexpr (R == 8) dft8<DIR>(v);
  else dft16<DIR>(v);
}

template <int N1, int N2, int DIR>
__device__ __forceinline__ void dft_pfa(float2* v) {
  constexpr int N = N1 * N2;
  constexpr int K1 = N2 * modinv(N2 % N1, N1);
  constexpr int K2 = N1 * modinv(N1 % N2, N2);
  float2 a[N2][N1];
#pragma unroll
  for (int n2 = 0; n2 < N2; ++n2) {
#pragma unroll
    for (int n1 = 0; n1 < N1; ++n1) a[n2][n1] = v[(N2 * n1 + N1 * n2) % N];
    dft_prime_or_pow2<N1, DIR>(a[n2]);
  }
#pragma unroll
  for (int k1 = 0; k1 < N1; ++k1) {
    float2 b[N2];
#pragma unroll
    for (int n2 = 0; n2 < N2; ++n2) b[n2] = a[n2][k1];
    dft_prime_or_pow2<N2, DIR>(b);
#pragma unroll
    for (int k2 = 0; k2 < N2; ++k2) v[(K1 * k1 + K2 * k2) % N] = b[k2];
  }
}

template <int N, int DIR>
__device__ __forceinline__ void dft_small(float2* v) {
  if constexpr (N == 1) {
  } else if constexpr (N == 2 || N == 3 || N == 4 || N == 5 || N == 8 || N == 16) {
    dft_prime_or_pow2<N, DIR>(v);
  } else if constexpr (N == 6) dft_pfa<2, 3, DIR>(v);
  else if constexpr (N == 10) dft_pfa<2, 5, DIR>(v);
  else if constexpr (N == 12) dft_pfa<4, 3, DIR>(v);
  else if constexpr (N == 15) dft_pfa<3, 5, DIR>(v);
  else if constexpr (N == 20) dft_pfa<4, 5, DIR>(v);
  else static_assert(N == 0, "unsupported small DFT size");
}

inline bool supported_radices(const LinePlan& p) {
  if (p.npass <= 0) return false;
  for (int i = 0; i < p.npass; ++i) {
    int r = p.radix[i];
    if (r != 2 && r != 3 && r != 4 && r != 5 && r != 8) return false;
  }
  return true;
}

}  // namespace fft
}  // namespace tmb
