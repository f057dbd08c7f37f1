// tc_xpass.cu -- the x pass of the precision form on the tensor cores, split BF16.
//
// Along x, the FP32 form runs forward DFT -> conj product with the receptor spectrum ->
// inverse DFT. By the convolution theorem that chain is one circulant matrix per receptor
// channel and (ky,kz) column: with P~_k(m, col) = sum_kx P^_k(kx, col) w^(-kx m) (the receptor
// grid transformed over y and z only, times n),
//     B_r(x', col) = sum_k sum_x P~_k((x + x') mod n, col) * conj(A_{r,k}(x, col)).
// This kernel applies that operator as a dense contraction on the tensor cores:
//     out[x'][r] = sum_{(k, part, x)} T[x'][(k, part, x)] * L[(k, part, x)][r]
// with T the (Toeplitz) real-ified receptor operator and L the real-ified ligand data, two
// output columns (re, im) per rotation:
//     Br = sum Tr*ar + Ti*ai,    Bi = sum Ti*ar - Tr*ai.
// Each operand is split into BF16 hi + lo (x = hi + lo, |lo| <= 2^-9 |x|), and the product
// keeps hi*hi + hi*lo + lo*hi with FP32 accumulation (mma.sync m16n8k16, row.col): relative
// error of each product about 2^-16.
//
// A fragments come straight from a "pair array" per (column, channel, part, hi/lo):
// q[j] = (p[j mod n], p[(j+1) mod n]) as one 32-bit word, so the (x, x+1) element pair of any
// Toeplitz row is one aligned load: the Toeplitz matrix is never materialised.
//
// CTA = CT (4) spectral columns x a chunk of rotations, handled 16 rotations at a time;
// warp w owns column w/2 and x' rows [32*(w&1), 32*(w&1) + 32) (2 m-tiles per 64 rows; for other
// n, MT/2 m-tiles), all 4 n-tiles (16 rotations x re/im).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include "cdk_internal.h"

namespace cdk {
namespace {

constexpr int TC_CT = 4;    // spectral columns per CTA (one 32-byte sector of A per x row)
constexpr int TC_R = 16;    // rotations per MMA group (4 n-tiles of 8: re/im per rotation)
constexpr int TC_WARPS = 2 * TC_CT;

__device__ __forceinline__ void split_bf16(float v, __nv_bfloat16& hi, __nv_bfloat16& lo) {
  hi = __float2bfloat16_rn(v);
  lo = __float2bfloat16_rn(v - __bfloat162float(hi));
}

__device__ __forceinline__ unsigned int pack2(__nv_bfloat16 lo16, __nv_bfloat16 hi16) {
  return (unsigned int)__bfloat16_as_ushort(lo16) |
         ((unsigned int)__bfloat16_as_ushort(hi16) << 16);
}

__device__ __forceinline__ void mma_bf16(float* c, unsigned a0, unsigned a1, unsigned a2,
                                         unsigned a3, unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 "
      "{%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

// P~ (resident, [col][k][m] complex) from the receptor's (y,z) transform scratch
// [k][m][col] (unnormalised); the factor n makes it the unnormalised inverse along x.
__global__ void k_ptilde(const float2* __restrict__ yz, float2* __restrict__ pt, int n, int K,
                         int ncol) {
  const long total = (long)ncol * K * n;
  for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < total;
       i += (long)gridDim.x * blockDim.x) {
    const int m = (int)(i % n);
    const int k = (int)((i / n) % K);
    const int col = (int)(i / ((long)n * K));
    const float2 v = yz[((size_t)k * n + m) * ncol + col];
    pt[i] = make_float2(v.x * n, v.y * n);
  }
}

template <int N>
__global__ void __launch_bounds__(256, 2) k_xpass_tc(WaveArgs a, const float2* __restrict__ pt,
                                                     int Lp, int rot_per_cta) {
  constexpr int NZH = N / 2 + 1;
  constexpr int NCOL = N * NZH;
  constexpr int MT = N / 16;       // m-tiles over x'
  constexpr int MTW = MT / 2;      // m-tiles per warp
  static_assert(NCOL % TC_CT == 0, "column tiles must divide the half spectrum");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int K = a.K;
  const int QL = N + Lp;           // pair-array length
  const int KS = 2 * Lp + 8;       // B-operand row stride (bf16), +8 keeps banks apart
  // pair arrays: [c][k][part][hl][QL] words
  unsigned int* q = reinterpret_cast<unsigned int*>(smem_raw);
  unsigned short* bop = reinterpret_cast<unsigned short*>(q + (size_t)TC_CT * K * 4 * QL);
  // B operand: [hl][c][n = 2r + out][KS] bf16
  short* s_rng = reinterpret_cast<short*>(bop + (size_t)2 * TC_CT * 2 * TC_R * KS);  // [R][2]
  int* s_meta = reinterpret_cast<int*>(s_rng + 2 * TC_R);                             // [R] W
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int c0 = blockIdx.x * TC_CT;
  // ---- pair arrays of this CTA's columns (once per CTA)
  for (int i = tid; i < TC_CT * K * QL; i += blockDim.x) {
    const int j = i % QL;
    const int t = i / QL;
    const int k = t % K, c = t / K;
    const float2* p = pt + ((size_t)(c0 + c) * K + k) * N;
    const float2 v0 = p[j % N], v1 = p[(j + 1) % N];
    __nv_bfloat16 h0r, l0r, h1r, l1r, h0i, l0i, h1i, l1i;
    split_bf16(v0.x, h0r, l0r);
    split_bf16(v1.x, h1r, l1r);
    split_bf16(v0.y, h0i, l0i);
    split_bf16(v1.y, h1i, l1i);
    unsigned int* base = q + ((size_t)(c * K + k) * 4) * QL + j;
    base[0 * QL] = pack2(h0r, h1r);  // part 0 (real), hi
    base[1 * QL] = pack2(l0r, l1r);  // part 0, lo
    base[2 * QL] = pack2(h0i, h1i);  // part 1 (imag), hi
    base[3 * QL] = pack2(l0i, l1i);  // part 1, lo
  }
  const int g = lane >> 2, t4 = lane & 3;
  const int wc = warp >> 1;               // column of this warp
  const int mh = warp & 1;                // which half of the x' m-tiles
  const int ksteps = (2 * Lp) / 16;
  const int r_begin = blockIdx.y * rot_per_cta;
  const int r_end = min(a.nrot, r_begin + rot_per_cta);
  for (int r0 = r_begin; r0 < r_end; r0 += TC_R) {
    const int nr = min(TC_R, r_end - r0);
    float acc[MTW][4][4];
#pragma unroll
    for (int m = 0; m < MTW; ++m)
#pragma unroll
      for (int nt = 0; nt < 4; ++nt)
#pragma unroll
        for (int e = 0; e < 4; ++e) acc[m][nt][e] = 0.f;
    for (int k = 0; k < K; ++k) {
      __syncthreads();  // previous users of bop / s_rng are done
      if (tid < TC_R) {
        short lo = 1, hi = 0;
        int W = 0;
        if (tid < nr) {
          const RotRec* rec = a.rec + r0 + tid;
          if (rec->valid) {
            lo = rec->xlo[k];
            hi = rec->xhi[k];
            W = rec->W[0];
          }
        }
        s_rng[2 * tid] = lo;
        s_rng[2 * tid + 1] = hi;
        s_meta[tid] = W;
      }
      __syncthreads();
      // skip a channel no rotation of the group touches (uniform across the CTA)
      bool any = false;
      int s_wmax = 0;
      for (int rr = 0; rr < TC_R; ++rr) {
        any |= (s_rng[2 * rr] <= s_rng[2 * rr + 1]);
        s_wmax = max(s_wmax, s_meta[rr]);
      }
      if (!any) continue;
      // ---- stage the ligand operand: rotations x x-planes x columns of channel k.
      // Thread = (rotation, pair of x planes): two 32-byte rows of A (the CTA's 4 columns) in
      // four 16-byte loads, then one 32-bit word (x, x+1) per column, slot and hi/lo.
      for (int i = tid; i < TC_R * (Lp / 2); i += blockDim.x) {
        const int x2 = i % (Lp / 2);
        const int rr = i / (Lp / 2);
        const int x = 2 * x2;
        float4 v[2][2];
#pragma unroll
        for (int d = 0; d < 2; ++d) {
          const bool in = rr < nr && x + d >= s_rng[2 * rr] && x + d <= s_rng[2 * rr + 1];
          if (in) {
            const float4* src = reinterpret_cast<const float4*>(
                a.A + (((size_t)(r0 + rr) * K + k) * a.Lb + x + d) * NCOL + c0);
            v[d][0] = src[0];
            v[d][1] = src[1];
          } else {
            v[d][0] = v[d][1] = make_float4(0.f, 0.f, 0.f, 0.f);
          }
        }
#pragma unroll
        for (int c = 0; c < TC_CT; ++c) {
          // column c of plane x+d: (re, im)
          const float re0 = (c & 1) ? v[0][c >> 1].z : v[0][c >> 1].x;
          const float im0 = (c & 1) ? v[0][c >> 1].w : v[0][c >> 1].y;
          const float re1 = (c & 1) ? v[1][c >> 1].z : v[1][c >> 1].x;
          const float im1 = (c & 1) ? v[1][c >> 1].w : v[1][c >> 1].y;
          __nv_bfloat16 rh0, rl0, rh1, rl1, ih0, il0, ih1, il1, nh0, nl0, nh1, nl1;
          split_bf16(re0, rh0, rl0);
          split_bf16(re1, rh1, rl1);
          split_bf16(im0, ih0, il0);
          split_bf16(im1, ih1, il1);
          split_bf16(-im0, nh0, nl0);
          split_bf16(-im1, nh1, nl1);
          // rows n = 2rr (re out): [x] = ar, [Lp + x] = ai ; n = 2rr+1 (im out): [x] = -ai, [Lp+x] = ar
          unsigned int* bh = reinterpret_cast<unsigned int*>(bop + ((size_t)(0 * TC_CT + c) * 2 * TC_R) * KS);
          unsigned int* bl = reinterpret_cast<unsigned int*>(bop + ((size_t)(1 * TC_CT + c) * 2 * TC_R) * KS);
          const size_t n0 = (size_t)(2 * rr) * (KS / 2), n1 = (size_t)(2 * rr + 1) * (KS / 2);
          const int xw = x2, xwi = (Lp / 2) + x2;
          bh[n0 + xw] = pack2(rh0, rh1);
          bl[n0 + xw] = pack2(rl0, rl1);
          bh[n0 + xwi] = pack2(ih0, ih1);
          bl[n0 + xwi] = pack2(il0, il1);
          bh[n1 + xw] = pack2(nh0, nh1);
          bl[n1 + xw] = pack2(nl0, nl1);
          bh[n1 + xwi] = pack2(rh0, rh1);
          bl[n1 + xwi] = pack2(rl0, rl1);
        }
      }
      __syncthreads();
      // ---- MMAs: this warp's column, its m-tiles, 4 n-tiles, all k-steps of channel k
      const unsigned int* qc = q + ((size_t)(wc * K + k) * 4) * QL;
      const unsigned short* bh = bop + ((size_t)(0 * TC_CT + wc) * 2 * TC_R) * KS;
      const unsigned short* bl = bop + ((size_t)(1 * TC_CT + wc) * 2 * TC_R) * KS;
      for (int s = 0; s < ksteps; ++s) {
        // the two k pairs of this lane: kidx = 16s + 2*t4 and 16s + 2*t4 + 8
        const int ka = 16 * s + 2 * t4, kb = ka + 8;
        const int pa = ka >= Lp, pb = kb >= Lp;
        const int xa = ka - pa * Lp, xb = kb - pb * Lp;
        const unsigned int* qa_h = qc + (2 * pa + 0) * QL;
        const unsigned int* qa_l = qc + (2 * pa + 1) * QL;
        const unsigned int* qb_h = qc + (2 * pb + 0) * QL;
        const unsigned int* qb_l = qc + (2 * pb + 1) * QL;
        unsigned int bfh[4][2], bfl[4][2];
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          const int n = nt * 8 + g;
          bfh[nt][0] = *reinterpret_cast<const unsigned int*>(bh + (size_t)n * KS + ka);
          bfh[nt][1] = *reinterpret_cast<const unsigned int*>(bh + (size_t)n * KS + kb);
          bfl[nt][0] = *reinterpret_cast<const unsigned int*>(bl + (size_t)n * KS + ka);
          bfl[nt][1] = *reinterpret_cast<const unsigned int*>(bl + (size_t)n * KS + kb);
        }
#pragma unroll
        for (int m = 0; m < MTW; ++m) {
          if ((mh * MTW + m) * 16 >= s_wmax) continue;  // rows past every window of the group
          const int row = (mh * MTW + m) * 16 + g;  // x' of a0/a2; +8 for a1/a3
          const unsigned int ah0 = qa_h[xa + row], ah1 = qa_h[xa + row + 8];
          const unsigned int ah2 = qb_h[xb + row], ah3 = qb_h[xb + row + 8];
          const unsigned int al0 = qa_l[xa + row], al1 = qa_l[xa + row + 8];
          const unsigned int al2 = qb_l[xb + row], al3 = qb_l[xb + row + 8];
#pragma unroll
          for (int nt = 0; nt < 4; ++nt) {
            mma_bf16(acc[m][nt], ah0, ah1, ah2, ah3, bfh[nt][0], bfh[nt][1]);
            mma_bf16(acc[m][nt], ah0, ah1, ah2, ah3, bfl[nt][0], bfl[nt][1]);
            mma_bf16(acc[m][nt], al0, al1, al2, al3, bfh[nt][0], bfh[nt][1]);
          }
        }
      }
    }
    __syncthreads();  // s_meta of this group is read below
    // ---- write B rows x' < W for the group's rotations
    // C fragment: c[0] (x' = row, n = 8nt + 2t4 -> rotation 4nt + t4, re), c[1] (same, im),
    // c[2], c[3] (x' = row + 8)
#pragma unroll
    for (int m = 0; m < MTW; ++m) {
      const int row = (mh * MTW + m) * 16 + g;
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int rr = nt * 4 + t4;
        if (rr >= nr) continue;
        const int W = s_meta[rr];
        float2* dst = a.B + (size_t)(r0 + rr) * N * NCOL + c0 + wc;
        if (row < W) dst[(size_t)row * NCOL] = make_float2(acc[m][nt][0], acc[m][nt][1]);
        if (row + 8 < W) dst[(size_t)(row + 8) * NCOL] = make_float2(acc[m][nt][2], acc[m][nt][3]);
      }
    }
  }
}

template <int N>
cudaError_t launch_tc_t(const WaveArgs& a, const float2* pt, cudaStream_t s) {
  constexpr int NCOL = N * (N / 2 + 1);
  const int Lp = (a.Lb + 7) & ~7;
  const size_t sm = xpass_tc_smem_bytes(N, a.K, a.Lb);
  cudaError_t e = cudaFuncSetAttribute(k_xpass_tc<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  const int per = a.chunk > 0 ? ((a.chunk + 15) / 16) * 16 : 64;
  const int chunks = (a.nrot + per - 1) / per;
  k_xpass_tc<N><<<dim3(NCOL / TC_CT, chunks), 32 * TC_WARPS, sm, s>>>(a, pt, Lp, per);
  return cudaGetLastError();
}

}  // namespace

size_t xpass_tc_smem_bytes(int n, int K, int Lb) {
  const int Lp = (Lb + 7) & ~7;
  return sizeof(unsigned int) * (size_t)TC_CT * K * 4 * (n + Lp) +
         sizeof(unsigned short) * (size_t)2 * TC_CT * 2 * TC_R * (2 * Lp + 8) +
         sizeof(short) * 2 * TC_R + sizeof(int) * TC_R + 16;
}

cudaError_t launch_ptilde(int n, int K, const float2* yz, float2* pt, cudaStream_t s) {
  const long total = (long)n * (n / 2 + 1) * K * n;
  const int blocks = (int)std::min<long>(4096, (total + 255) / 256);
  k_ptilde<<<blocks, 256, 0, s>>>(yz, pt, n, K, n * (n / 2 + 1));
  return cudaGetLastError();
}

cudaError_t launch_xpass_tc(const WaveArgs& a, const float2* pt, cudaStream_t s) {
  switch (a.n) {
    case 32: return launch_tc_t<32>(a, pt, s);
    case 64: return launch_tc_t<64>(a, pt, s);
    case 96: return launch_tc_t<96>(a, pt, s);
    case 128: return launch_tc_t<128>(a, pt, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace cdk
