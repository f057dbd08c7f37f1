// fft.cuh -- in-place mixed-radix FFT stages over lines held in shared memory.
//
// A length-N transform is a sequence of radix stages (N = R1*R2*...*Rm). The forward form is
// decimation in frequency: stage s splits every block of M_{s-1} = R_s*M_s points into R_s
// interleaved sub-blocks, does a radix-R_s DFT on each group {n' + j*M_s}, multiplies output
// k by w_{M_{s-1}}^{n'k} and writes it back to the same places. The result is the spectrum in
// mixed-radix digit-reversed order: frequency k = k1 + R1*k2 + R1*R2*k3 + ... sits at
// position k1*M_1 + k2*M_2 + ... (fft_pos below). The inverse runs the conjugate stages in
// reverse order and returns natural order from digit-reversed input, so a forward transform,
// a pointwise product in digit-reversed order and an inverse need no permutation at all.
// Every butterfly reads and writes the same R slots, so stages run in place; the caller puts
// a __syncthreads() between stages. The inverse is unnormalised (factor N).
#pragma once
#include <cuda_runtime.h>

namespace cdk {

__device__ __forceinline__ float2 c_add(float2 a, float2 b) { return make_float2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ float2 c_sub(float2 a, float2 b) { return make_float2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ float2 c_mul(float2 a, float2 b) {
  return make_float2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
// a * conj(b)
__device__ __forceinline__ float2 c_mulc(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}
// conj(a) * b
__device__ __forceinline__ float2 c_conjmul(float2 a, float2 b) {
  return make_float2(a.x * b.x + a.y * b.y, a.x * b.y - a.y * b.x);
}
// multiply by -i (forward) or +i (inverse): SIGN = -1 forward, +1 inverse
template <int SIGN>
__device__ __forceinline__ float2 c_rot90(float2 a) {
  return SIGN < 0 ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
}

// Radix-R DFT kernels y_k = sum_j x_j exp(SIGN * 2 pi i j k / R), SIGN = -1 forward.
template <int R, int SIGN>
struct Radix;

template <int SIGN>
struct Radix<2, SIGN> {
  __device__ __forceinline__ static void run(float2* v) {
    float2 a = v[0], b = v[1];
    v[0] = c_add(a, b);
    v[1] = c_sub(a, b);
  }
};

template <int SIGN>
struct Radix<3, SIGN> {
  __device__ __forceinline__ static void run(float2* v) {
    const float h = 0.86602540378443864676f;  // sin(2 pi / 3)
    float2 t = c_add(v[1], v[2]);
    float2 d = c_sub(v[1], v[2]);
    float2 m = make_float2(v[0].x - 0.5f * t.x, v[0].y - 0.5f * t.y);
    // y1 = m + SIGN*i*h*d, y2 = m - SIGN*i*h*d
    float2 r = c_rot90<SIGN>(d);
    v[0] = c_add(v[0], t);
    v[1] = make_float2(m.x + h * r.x, m.y + h * r.y);
    v[2] = make_float2(m.x - h * r.x, m.y - h * r.y);
  }
};

template <int SIGN>
struct Radix<4, SIGN> {
  __device__ __forceinline__ static void run(float2* v) {
    float2 s02 = c_add(v[0], v[2]), d02 = c_sub(v[0], v[2]);
    float2 s13 = c_add(v[1], v[3]), d13 = c_rot90<SIGN>(c_sub(v[1], v[3]));
    v[0] = c_add(s02, s13);
    v[2] = c_sub(s02, s13);
    v[1] = c_add(d02, d13);
    v[3] = c_sub(d02, d13);
  }
};

template <int SIGN>
struct Radix<8, SIGN> {
  __device__ __forceinline__ static void run(float2* v) {
    const float r2 = 0.70710678118654752440f;
    // split into even / odd output halves (radix-2 DIF step), then two radix-4 DFTs
    float2 u[4], w[4];
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      u[j] = c_add(v[j], v[j + 4]);
      w[j] = c_sub(v[j], v[j + 4]);
    }
    // w_j *= exp(SIGN * 2 pi i j / 8)
    w[1] = make_float2(r2 * (w[1].x - SIGN * w[1].y), r2 * (w[1].y + SIGN * w[1].x));
    w[2] = c_rot90<SIGN>(w[2]);
    w[3] = make_float2(r2 * (-w[3].x - SIGN * w[3].y), r2 * (-w[3].y + SIGN * w[3].x));
    Radix<4, SIGN>::run(u);
    Radix<4, SIGN>::run(w);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      v[2 * j] = u[j];
      v[2 * j + 1] = w[j];
    }
  }
};

// exp(SIGN * 2 pi i m / R) for the composite radices below (constants from the unit circle:
// cos/sin of multiples of pi/6 and pi/8)
template <int R, int SIGN>
__device__ __forceinline__ float2 unit_root(int m) {
  constexpr float c8 = 0.92387953251128675613f, s8 = 0.38268343236508977173f;
  constexpr float h2 = 0.70710678118654752440f, r3 = 0.86602540378443864676f;
  float c = 1.f, sn = 0.f;
  if (R == 16) {
    const float cs[16] = {1.f, c8, h2, s8, 0.f, -s8, -h2, -c8, -1.f, -c8, -h2, -s8, 0.f, s8, h2, c8};
    const float ss[16] = {0.f, s8, h2, c8, 1.f, c8, h2, s8, 0.f, -s8, -h2, -c8, -1.f, -c8, -h2, -s8};
    c = cs[m & 15];
    sn = ss[m & 15];
  } else if (R == 12) {
    const float cs[12] = {1.f, r3, .5f, 0.f, -.5f, -r3, -1.f, -r3, -.5f, 0.f, .5f, r3};
    const float ss[12] = {0.f, .5f, r3, 1.f, r3, .5f, 0.f, -.5f, -r3, -1.f, -r3, -.5f};
    c = cs[m % 12];
    sn = ss[m % 12];
  }
  return make_float2(c, SIGN * sn);
}

// Composite radix R = A * B in registers: n = B*n1 + n2, k = k1 + A*k2;
// y[k] = sum_n2 w_R^(n2 k1) w_B^(n2 k2) sum_n1 x[B n1 + n2] w_A^(n1 k1)
template <int A, int B, int SIGN>
__device__ __forceinline__ void radix_composite(float2* v) {
  constexpr int R = A * B;
  float2 u[B][A];
#pragma unroll
  for (int n2 = 0; n2 < B; ++n2) {
#pragma unroll
    for (int n1 = 0; n1 < A; ++n1) u[n2][n1] = v[B * n1 + n2];
    Radix<A, SIGN>::run(u[n2]);
#pragma unroll
    for (int k1 = 1; k1 < A; ++k1)
      if (n2 > 0) u[n2][k1] = c_mul(u[n2][k1], unit_root<R, SIGN>(n2 * k1));
  }
#pragma unroll
  for (int k1 = 0; k1 < A; ++k1) {
    float2 w[B];
#pragma unroll
    for (int n2 = 0; n2 < B; ++n2) w[n2] = u[n2][k1];
    Radix<B, SIGN>::run(w);
#pragma unroll
    for (int k2 = 0; k2 < B; ++k2) v[k1 + A * k2] = w[k2];
  }
}

template <int SIGN>
struct Radix<12, SIGN> {
  __device__ __forceinline__ static void run(float2* v) { radix_composite<4, 3, SIGN>(v); }
};

template <int SIGN>
struct Radix<16, SIGN> {
  __device__ __forceinline__ static void run(float2* v) { radix_composite<4, 4, SIGN>(v); }
};

// Radix sequences per transform length (R0 first in the forward transform).
template <int N>
struct FFTPlan;
template <>
struct FFTPlan<32> {
  static constexpr int NS = 2, R0 = 8, R1 = 4, R2 = 1;
};
template <>
struct FFTPlan<64> {
  static constexpr int NS = 2, R0 = 8, R1 = 8, R2 = 1;
};
template <>
struct FFTPlan<96> {
  static constexpr int NS = 2, R0 = 8, R1 = 12, R2 = 1;
};
template <>
struct FFTPlan<128> {
  static constexpr int NS = 2, R0 = 8, R1 = 16, R2 = 1;
};

template <int N>
__host__ __device__ constexpr int fft_radix(int s) {
  return s == 0 ? FFTPlan<N>::R0 : (s == 1 ? FFTPlan<N>::R1 : FFTPlan<N>::R2);
}

// Stride M_s of stage s (1-based): N / (R0 * ... * R(s-1)).
template <int N, int S>
struct StageM {
  static constexpr int value = StageM<N, S - 1>::value / fft_radix<N>(S - 1);
};
template <int N>
struct StageM<N, 0> {
  static constexpr int value = N;
};

// Position of natural frequency k in the digit-reversed layout.
template <int N>
__host__ __device__ __forceinline__ int fft_pos(int k) {
  int pos = 0, m = N;
#pragma unroll
  for (int s = 0; s < FFTPlan<N>::NS; ++s) {
    const int r = fft_radix<N>(s);
    m /= r;
    pos += (k % r) * m;
    k /= r;
  }
  return pos;
}

// One stage over `nlines` lines; element e of line l is buf[l*ls + e*es].
// tw[j] = exp(-2 pi i j / N), j < N (shared memory).
// Work items run line-fastest so that a warp touches consecutive lines.
template <int N, int R, int M, bool INV>
__device__ __forceinline__ void fft_stage(float2* buf, int nlines, int ls, int es,
                                          const float2* __restrict__ tw, int tid, int nthr) {
  constexpr int NB = N / R;
  constexpr int TWM = N / (R * M);
  const int total = nlines * NB;
  for (int w = tid; w < total; w += nthr) {
    const int b = w / nlines;
    const int l = w - b * nlines;
    const int blk = b / M;
    const int np = b - blk * M;
    float2* p = buf + l * ls + (blk * R * M + np) * es;
    float2 v[R];
#pragma unroll
    for (int j = 0; j < R; ++j) v[j] = p[j * M * es];
    if (!INV) {
      Radix<R, -1>::run(v);
      if (M > 1) {
#pragma unroll
        for (int k = 1; k < R; ++k) v[k] = c_mul(v[k], tw[np * k * TWM]);
      }
    } else {
      if (M > 1) {
#pragma unroll
        for (int k = 1; k < R; ++k) v[k] = c_mulc(v[k], tw[np * k * TWM]);
      }
      Radix<R, +1>::run(v);
    }
#pragma unroll
    for (int j = 0; j < R; ++j) p[j * M * es] = v[j];
  }
}

// fft_stage with a compile-time line count bound SLOTS >= nlines: work item w is line w % SLOTS
// of butterfly block w / SLOTS (no division by a run-time count), lines >= nlines idle.
template <int N, int R, int M, bool INV, int SLOTS>
__device__ __forceinline__ void fft_stage_slots(float2* buf, int nlines, int ls, int es,
                                                const float2* __restrict__ tw, int tid, int nthr) {
  constexpr int NB = N / R;
  constexpr int TWM = N / (R * M);
  for (int w = tid; w < SLOTS * NB; w += nthr) {
    const int l = w % SLOTS;
    if (l >= nlines) continue;
    const int b = w / SLOTS;
    const int blk = b / M;
    const int np = b - blk * M;
    float2* p = buf + l * ls + (blk * R * M + np) * es;
    float2 v[R];
#pragma unroll
    for (int j = 0; j < R; ++j) v[j] = p[j * M * es];
    if (!INV) {
      Radix<R, -1>::run(v);
      if (M > 1) {
#pragma unroll
        for (int k = 1; k < R; ++k) v[k] = c_mul(v[k], tw[np * k * TWM]);
      }
    } else {
      if (M > 1) {
#pragma unroll
        for (int k = 1; k < R; ++k) v[k] = c_mulc(v[k], tw[np * k * TWM]);
      }
      Radix<R, +1>::run(v);
    }
#pragma unroll
    for (int j = 0; j < R; ++j) p[j * M * es] = v[j];
  }
}

// Inverse transform of at most SLOTS lines (two-stage plans), without run-time divisions.
template <int N, int SLOTS>
__device__ __forceinline__ void ifft_lines_slots(float2* buf, int nlines, int ls, int es,
                                                 const float2* __restrict__ tw, int tid, int nthr) {
  using P = FFTPlan<N>;
  static_assert(P::NS == 2, "two-stage plans only");
  fft_stage_slots<N, P::R1, StageM<N, 2>::value, true, SLOTS>(buf, nlines, ls, es, tw, tid, nthr);
  __syncthreads();
  fft_stage_slots<N, P::R0, StageM<N, 1>::value, true, SLOTS>(buf, nlines, ls, es, tw, tid, nthr);
  __syncthreads();
}

// Full forward (DIF, natural -> digit-reversed) or inverse (DIT, digit-reversed -> natural)
// transform of `nlines` lines. Contains the __syncthreads() between stages and one at the end.
template <int N, bool INV>
__device__ __forceinline__ void fft_lines(float2* buf, int nlines, int ls, int es,
                                          const float2* __restrict__ tw, int tid, int nthr) {
  using P = FFTPlan<N>;
  if (!INV) {
    fft_stage<N, P::R0, StageM<N, 1>::value, false>(buf, nlines, ls, es, tw, tid, nthr);
    __syncthreads();
    fft_stage<N, P::R1, StageM<N, 2>::value, false>(buf, nlines, ls, es, tw, tid, nthr);
    __syncthreads();
    if constexpr (P::NS == 3) {
      fft_stage<N, P::R2, StageM<N, 3>::value, false>(buf, nlines, ls, es, tw, tid, nthr);
      __syncthreads();
    }
  } else {
    if constexpr (P::NS == 3) {
      fft_stage<N, P::R2, StageM<N, 3>::value, true>(buf, nlines, ls, es, tw, tid, nthr);
      __syncthreads();
    }
    fft_stage<N, P::R1, StageM<N, 2>::value, true>(buf, nlines, ls, es, tw, tid, nthr);
    __syncthreads();
    fft_stage<N, P::R0, StageM<N, 1>::value, true>(buf, nlines, ls, es, tw, tid, nthr);
    __syncthreads();
  }
}

}  // namespace cdk
