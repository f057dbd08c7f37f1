// search_kernels.cu -- the FP32 FFT translational-rotational search on sm_100a.
//
// One wave of rotations runs five kernels, all on one stream:
//   prep          rotate atoms (reference op order, no contraction), bounding box, windows,
//                 per-channel x-plane ranges          (src/Rotate.cpp, GetMin/MaxCoors.cpp)
//   spread_yz     per (rotation, channel, x plane): spread the atoms that touch the plane
//                 into shared memory (trilinear weights in FillLigandGrid's arithmetic), then
//                 the 2-D real-to-complex FFT over (y,z) -> A      (src/FillLigandGrid.cpp)
//   xpass         per spectral column tile: FFT along x of every channel, the conjugate
//                 product with the resident receptor spectra summed over channels, and the
//                 inverse FFT along x, keeping only the translation window -> B
//                                                       (src/kernel.cu ConjMult + SumGrids)
//   yz_inv_argmin per (rotation, x in window): inverse FFT over y, complex-to-real over z,
//                 min / first argmin over the window, folded into one 64-bit key per rotation
//                                         (src/TranRotaConfSearchNoMini.cu:429-464)
//   finalize      keys -> minE, (i,j,k)
// The energy grid never leaves shared memory. Spectra stay in the digit-reversed order the
// in-place FFT stages produce; the receptor spectra are computed by the same stages, so
// the pointwise product lines up without any permutation.
#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdlib>

#include "cdk_internal.h"
#include "fft.cuh"

namespace cdk {

namespace {

// (a, b) -> packed bf16x2 hi = rn(a), rn(b) and lo = rn(a - hi), rn(b - hi); a in the low half
__device__ __forceinline__ void split_bf16x2(float a, float b, uint32_t& hi, uint32_t& lo) {
  const __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
  const float2 hf = __bfloat1622float2(h);
  const __nv_bfloat162 l = __floats2bfloat162_rn(a - hf.x, b - hf.y);
  hi = *reinterpret_cast<const uint32_t*>(&h);
  lo = *reinterpret_cast<const uint32_t*>(&l);
}

// one 32-byte store (p 32-byte aligned): words w0..w3 then w4..w7
__device__ __forceinline__ void st_v8u(void* p, uint4 lo, uint4 hi) {
  asm volatile("st.global.v8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(p), "r"(lo.x), "r"(lo.y),
               "r"(lo.z), "r"(lo.w), "r"(hi.x), "r"(hi.y), "r"(hi.z), "r"(hi.w)
               : "memory");
}

// Tiled ligand rows (WaveArgs.lop_tiled): (tile r / 128, channel k, chunk jc) is a row set of
// 128 rotations x ncol columns; rotation m = r % 128 keeps its columns side by side, so the lanes
// of a warp (consecutive columns) write one contiguous run. Rows are in natural order: the x
// pass's tensor copies gather column c of the 128 rotations and apply the tensor cores' swizzle.
__device__ __forceinline__ unsigned char* tiled_row(const WaveArgs& a, int r, int k, int jc, int c, int row_bytes) {
  const int ncol = a.n * (a.n / 2 + 1);
  const size_t set = ((size_t)(r / kTileRot) * a.K + k) * 4 + jc;
  return a.lop + ((set * kTileRot + (size_t)(r % kTileRot)) * ncol + c) * (size_t)row_bytes;
}

// split-FP16: one 32-byte row [re | im] of the 8 planes
__device__ __forceinline__ void tiled_row_store(const WaveArgs& a, int r, int k, int jc, int c, uint4 re, uint4 im) {
  st_v8u(tiled_row(a, r, k, jc, c, 32), re, im);
}

// split-BF16: one 64-byte row [hi re | hi im | lo re | lo im]; the x pass reads the lo part 32
// bytes into the same rows. rows[0..3]: hi re, hi im, lo re, lo im.
__device__ __forceinline__ void tiled_row_store64(const WaveArgs& a, int r, int k, int jc, int c, const uint4* rows) {
  uint4* dst = reinterpret_cast<uint4*>(tiled_row(a, r, k, jc, c, 64));
  st_v8u(dst, rows[0], rows[1]);
  st_v8u(dst + 2, rows[2], rows[3]);
}


// ---------------------------------------------------------------------------------------
// exact-order float rotation (src/QuaternionMultiply.cpp:3-11, src/Rotate.cpp:4-27)
__device__ __forceinline__ void qmul_rn(const float* l, const float* r, float* o) {
  o[0] = __fsub_rn(__fsub_rn(__fsub_rn(__fmul_rn(l[0], r[0]), __fmul_rn(l[1], r[1])),
                             __fmul_rn(l[2], r[2])),
                   __fmul_rn(l[3], r[3]));
  o[1] = __fsub_rn(__fadd_rn(__fadd_rn(__fmul_rn(l[0], r[1]), __fmul_rn(l[1], r[0])),
                             __fmul_rn(l[2], r[3])),
                   __fmul_rn(l[3], r[2]));
  o[2] = __fadd_rn(__fadd_rn(__fsub_rn(__fmul_rn(l[0], r[2]), __fmul_rn(l[1], r[3])),
                             __fmul_rn(l[2], r[0])),
                   __fmul_rn(l[3], r[1]));
  o[3] = __fadd_rn(__fsub_rn(__fadd_rn(__fmul_rn(l[0], r[3]), __fmul_rn(l[1], r[2])),
                             __fmul_rn(l[2], r[1])),
                   __fmul_rn(l[3], r[0]));
}

__device__ __forceinline__ void rotate_rn(const float* q, float vx, float vy, float vz,
                                          float* out) {
  float qc[4] = {q[0], -q[1], -q[2], -q[3]};
  float qv[4] = {0.0f, vx, vy, vz};
  float t1[4], t2[4];
  qmul_rn(q, qv, t1);
  qmul_rn(t1, qc, t2);
  out[0] = t2[1];
  out[1] = t2[2];
  out[2] = t2[3];
}

// cell index of a coordinate, FillLigandGrid's double arithmetic (src/FillLigandGrid.cpp:28-30)
__device__ __forceinline__ int cell_of(float x, float mn, float h) {
  return (int)__ddiv_rn(__dsub_rn((double)x, (double)mn), (double)h);
}
// ratio within the cell (src/FillLigandGrid.cpp:33-35): `index * spacing` is a float product
__device__ __forceinline__ double ratio_of(float x, float mn, float h, int i) {
  return __ddiv_rn(__dsub_rn(__dsub_rn((double)x, (double)mn), (double)__fmul_rn((float)i, h)),
                   (double)h);
}

__device__ __forceinline__ unsigned int order_key(float f) {
  unsigned int u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_to_float(unsigned int k) {
  unsigned int u = (k & 0x80000000u) ? (k & 0x7fffffffu) : ~k;
  return __uint_as_float(u);
}

// ---------------------------------------------------------------------------------------
// prep: one warp per rotation
__global__ void __launch_bounds__(128) k_prep(WaveArgs a) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r = blockIdx.x * 4 + warp;
  __shared__ int s_lo[4][KMAX], s_hi[4][KMAX], s_ext[4][3];
  if (lane < KMAX) {
    s_lo[warp][lane] = 0x7fff;
    s_hi[warp][lane] = -1;
  }
  if (lane < 3) s_ext[warp][lane] = 0;
  __syncwarp();
  if (r >= a.nrot) return;
  const RotDesc rd = a.rots[r];
  const ConfDesc cd = a.confs[rd.conf];
  const int nA = min(cd.n_atoms, a.max_atoms);
  const float* xyz = a.coords + (size_t)cd.coord_off * 3;
  float mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  for (int i = lane; i < nA; i += 32) {
    float p[3];
    rotate_rn(rd.q, xyz[i * 3 + 0], xyz[i * 3 + 1], xyz[i * 3 + 2], p);
    a.rot_xyz[(size_t)r * a.max_atoms + i] = make_float4(p[0], p[1], p[2], 0.0f);
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      mn[d] = fminf(mn[d], p[d]);
      mx[d] = fmaxf(mx[d], p[d]);
    }
  }
#pragma unroll
  for (int d = 0; d < 3; ++d)
    for (int o = 16; o > 0; o >>= 1) {
      mn[d] = fminf(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
      mx[d] = fmaxf(mx[d], __shfl_xor_sync(0xffffffffu, mx[d], o));
    }
  const float h = a.spacing;
  int W[3];
#pragma unroll
  for (int d = 0; d < 3; ++d) W[d] = a.n - (int)__fdiv_rn(__fsub_rn(mx[d], mn[d]), h) - 2;
  const bool valid = nA > 0 && W[0] > 0 && W[1] > 0 && W[2] > 0;
  __syncwarp();
  // per-channel x range and touched extents
  const AtomParam* prm = a.params + cd.param_off;
  const int elec = a.K - 1;
  for (int i = lane; i < nA; i += 32) {
    float4 p = a.rot_xyz[(size_t)r * a.max_atoms + i];
    int ci[3] = {cell_of(p.x, mn[0], h), cell_of(p.y, mn[1], h), cell_of(p.z, mn[2], h)};
    const int sl = prm[i].slot;
    if (sl >= 0 && sl < elec) {
      atomicMin(&s_lo[warp][sl], ci[0]);
      atomicMax(&s_hi[warp][sl], ci[0] + 1);
    }
    atomicMin(&s_lo[warp][elec], ci[0]);
    atomicMax(&s_hi[warp][elec], ci[0] + 1);
#pragma unroll
    for (int d = 0; d < 3; ++d) atomicMax(&s_ext[warp][d], ci[d] + 2);
  }
  __syncwarp();
  bool range_bad = false;
  if (a.f16 && a.range_err) {
    // split-FP16 form: |A(x, ky, kz)| <= sum over the channel's atoms of |s_a| (x weights and
    // |Fy|, |Fz| are at most 1), so the scaled ligand rows fit FP16 when this bound does
    bool bad = false;
    if (lane < a.K) {
      float bound = 0.f;
      for (int i = 0; i < nA; ++i) {
        if (lane == elec) bound += fabsf(prm[i].charge);
        else if (prm[i].slot == lane) bound += fabsf(prm[i].w_vdw);
      }
      bad = bound * a.lscale[lane] > 60000.f;
    }
    range_bad = __any_sync(0xffffffffu, bad);
    if (range_bad && lane == 0) atomicOr(a.range_err, 1);
  }
  RotRec* rec = a.rec + r;
  if (lane < KMAX) {
    const bool used = lane < a.K && s_hi[warp][lane] >= 0;
    rec->xlo[lane] = used ? (short)s_lo[warp][lane] : (short)1;
    rec->xhi[lane] = used ? (short)s_hi[warp][lane] : (short)0;
  }
  if (lane == 0) {
    // err 1: the x planes of a channel leave the planned box, or y/z cells the grid;
    // err 2: a scaled ligand value would leave the FP16 range (split-FP16 form). Either makes
    // the rotation invalid (no kernel after this one touches it)
    int err = 0;
    if (valid && (s_ext[warp][0] - 1 >= a.Lb || s_ext[warp][1] > a.n || s_ext[warp][2] > a.n))
      err = 1;
    else if (valid && range_bad)
      err = 2;
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      rec->mn[d] = mn[d];
      rec->W[d] = W[d];
      rec->ext[d] = s_ext[warp][d];
    }
    rec->valid = (valid && !err) ? 1 : 0;
    rec->err = err;
    rec->nA = nA;
    a.keys[r] = ~0ull;
  }
}

// ---------------------------------------------------------------------------------------
// shared helpers for the (y,z) plane transforms
//   P: packed real rows, pair p holds rows 2p (real part) and 2p+1 (imag part), stride n+1
//   O: half spectrum over z, [y][kz] with stride nzh (row y, col kz)

// z: R2C of `npairs` packed row pairs in P, then split into O rows (2p, 2p+1)
template <int N>
__device__ __forceinline__ void plane_forward(float2* P, float2* O, int npairs,
                                              const float2* tw) {
  constexpr int NZH = N / 2 + 1;
  const int tid = threadIdx.x, nthr = blockDim.x;
  fft_lines<N, false>(P, npairs, N + 1, 1, tw, tid, nthr);
  for (int i = tid; i < (N / 2) * NZH; i += nthr) {
    const int p = i / NZH, kz = i - p * NZH;
    float2 A = make_float2(0.f, 0.f), Bv = make_float2(0.f, 0.f);
    if (p < npairs) {
      const float2 zk = P[p * (N + 1) + fft_pos<N>(kz)];
      const float2 zn = P[p * (N + 1) + fft_pos<N>((N - kz) % N)];
      A = make_float2(0.5f * (zk.x + zn.x), 0.5f * (zk.y - zn.y));
      Bv = make_float2(0.5f * (zk.y + zn.y), -0.5f * (zk.x - zn.x));
    }
    O[(2 * p) * NZH + kz] = A;
    O[(2 * p + 1) * NZH + kz] = Bv;
  }
  __syncthreads();
  // y: complex FFT on the nzh columns
  fft_lines<N, false>(O, NZH, 1, NZH, tw, tid, nthr);
}

// ---------------------------------------------------------------------------------------
// spread + forward (y,z) transform of one (rotation, channel, x plane)
template <int N>
__global__ void __launch_bounds__(256) k_spread_yz(WaveArgs a) {
  constexpr int NZH = N / 2 + 1;
  constexpr int NCOL = N * NZH;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* tw = reinterpret_cast<float2*>(smem_raw);
  float2* O = tw + N;
  float2* P = O + N * NZH;
  const int x = blockIdx.x, k = blockIdx.y, r = blockIdx.z;
  const RotRec* rec = a.rec + r;
  if (!rec->valid) return;
  const int xlo = rec->xlo[k], xhi = rec->xhi[k];
  if (x < xlo || x > xhi) return;
  const int tid = threadIdx.x, nthr = blockDim.x;
  for (int i = tid; i < N; i += nthr) tw[i] = a.tw[i];
  const int npairs = min(N / 2, (rec->ext[1] + 1) / 2);
  float* Pf = reinterpret_cast<float*>(P);
  for (int i = tid; i < npairs * (N + 1); i += nthr) P[i] = make_float2(0.f, 0.f);
  __syncthreads();
  // spread the atoms touching plane x (src/FillLigandGrid.cpp:24-66 vdW, :75-118 elec).
  // Warp 0 adds the atoms one after another in ascending atom order, the four (y,z) corners
  // of an atom in four lanes (they never share a cell), each add rounded back to float from
  // double as in the reference: the plane is bit-identical to FillLigandGrid's and the
  // search is deterministic whatever the batch around a rotation.
  const RotDesc rd = a.rots[r];
  const ConfDesc cd = a.confs[rd.conf];
  const AtomParam* prm = a.params + cd.param_off;
  const float mn0 = rec->mn[0], mn1 = rec->mn[1], mn2 = rec->mn[2];
  const float h = a.spacing;
  const bool elec = (k == a.K - 1);
  const int nA = rec->nA;
  if (tid < 32) {
    const int lane = tid;
    for (int base = 0; base < nA; base += 32) {
      const int i = base + lane;
      bool touch = false;
      if (i < nA) {
        const AtomParam ap = prm[i];
        if (elec || ap.slot == k) {
          const int xi = cell_of(a.rot_xyz[(size_t)r * a.max_atoms + i].x, mn0, h);
          touch = (xi == x) || (xi + 1 == x);
        }
      }
      unsigned int m = __ballot_sync(0xffffffffu, touch);
      while (m) {
        const int at = base + __ffs(m) - 1;
        m &= m - 1;
        if (lane < 4) {
          const AtomParam ap = prm[at];
          const float4 p = a.rot_xyz[(size_t)r * a.max_atoms + at];
          const int xi = cell_of(p.x, mn0, h);
          const double xr = ratio_of(p.x, mn0, h, xi);
          const double wx = (xi == x) ? __dsub_rn(1.0, xr) : xr;
          const int yi = cell_of(p.y, mn1, h), zi = cell_of(p.z, mn2, h);
          const double yr = ratio_of(p.y, mn1, h, yi), zr = ratio_of(p.z, mn2, h, zi);
          const double sc = elec ? (double)ap.charge : (double)ap.w_vdw;
          const int dy = lane >> 1, dz = lane & 1;
          const double w = __dmul_rn(__dmul_rn(__dmul_rn(sc, wx), dy ? yr : __dsub_rn(1.0, yr)),
                                     dz ? zr : __dsub_rn(1.0, zr));
          const int y = yi + dy, z = zi + dz;
          if (y < N && z < N) {
            float* cell = &Pf[((y >> 1) * (N + 1) + z) * 2 + (y & 1)];
            *cell = (float)__dadd_rn((double)*cell, w);
          }
        }
        __syncwarp();
      }
    }
  }
  __syncthreads();
  plane_forward<N>(P, O, npairs, tw);
  // write the plane's half spectrum (16-byte stores)
  float4* dst = reinterpret_cast<float4*>(a.A + (((size_t)r * a.K + k) * a.Lb + x) * NCOL);
  const float4* src = reinterpret_cast<const float4*>(O);
  for (int i = tid; i < NCOL / 2; i += nthr) dst[i] = src[i];
}

// ---------------------------------------------------------------------------------------
// Direct (y,z) spectrum of the spread planes of one (rotation, channel).
// The spread is a sum of separable cloud-in-cell kernels, so the 2-D DFT of plane x is
//   A(x, ky, kz) = sum_{atoms a touching x} s_a wx_a(x) Fy_a(ky) Fz_a(kz),
//   Fy_a(ky) = (1 - ry) w^(yi ky) + ry w^((yi+1) ky),   w = exp(-2 pi i / n)
// (the same numbers the spread + radix FFT produce, without the float rounding of the plane).
// CTA per (rotation, channel): per-atom factor tables in shared memory, then every touched
// plane's n*(n/2+1) outputs, written in the (ky position, kz) order of the FFT path.
// Atoms are visited in ascending order for every plane: deterministic.
// One column's 8-plane chunk jc of the plane kernel, written as FP32 planes (A), FP16 rows or
// split-BF16 rows (lop).
template <int N, bool LOP>
__device__ __forceinline__ void plane_chunk_write(const WaveArgs& a, int r, int k, int jc, int x0,
                                                  int xlo, int xhi, int c, const float* ax,
                                                  const float* ay) {
  constexpr int NCOL = N * (N / 2 + 1);
  if constexpr (!LOP) {
#pragma unroll
    for (int d = 0; d < 8; ++d) {
      const int x = x0 + d;
      if (x >= xlo && x <= xhi) a.A[(((size_t)r * a.K + k) * a.Lb + x) * NCOL + c] = make_float2(ax[d], ay[d]);
    }
  } else if (a.f16) {
    // split-FP16 form: FP16 rows of the 8 planes times 2^sigma_k (already in the atoms' x
    // weights): per (rotation, channel) 8 rows [chunk][re, im] of ncol x 16 B in the same 512 B
    // blocks (k_prep has checked that the scaled planes stay inside the FP16 range)
    uint32_t hr[4], hi[4];
#pragma unroll
    for (int d = 0; d < 8; d += 2) {
      const __half2 pr = __floats2half2_rn(ax[d], ax[d + 1]), pi = __floats2half2_rn(ay[d], ay[d + 1]);
      hr[d / 2] = *reinterpret_cast<const uint32_t*>(&pr);
      hi[d / 2] = *reinterpret_cast<const uint32_t*>(&pi);
    }
    if (a.lop_tiled) {
      tiled_row_store(a, r, k, jc, c, make_uint4(hr[0], hr[1], hr[2], hr[3]), make_uint4(hi[0], hi[1], hi[2], hi[3]));
      return;
    }
    uint4* dst = reinterpret_cast<uint4*>(a.lop) +
                 (((size_t)(r >> 3) * a.K + k) * 8 * (NCOL / 4) + (c >> 2)) * 32 + (r & 7) * 4 + (c & 3);
    constexpr size_t RS = (size_t)(NCOL / 4) * 32;  // one row
    dst[(jc * 2 + 0) * RS] = make_uint4(hr[0], hr[1], hr[2], hr[3]);
    dst[(jc * 2 + 1) * RS] = make_uint4(hi[0], hi[1], hi[2], hi[3]);
  } else {
    // split-BF16 rows of the 8 planes (zero outside [xlo, xhi] by construction): per
    // (rotation, channel) 16 rows [hi, lo][chunk][re, im] of ncol x 16 B, the tensor-core x
    // pass's K order, in 512 B blocks of (8 rotations x 4 columns) x 16 B
    uint32_t rh[4], rl[4], ih[4], il[4];
#pragma unroll
    for (int d = 0; d < 8; d += 2) {
      split_bf16x2(ax[d], ax[d + 1], rh[d / 2], rl[d / 2]);
      split_bf16x2(ay[d], ay[d + 1], ih[d / 2], il[d / 2]);
    }
    if (a.lop_tiled) {
      const uint4 rows[4] = {make_uint4(rh[0], rh[1], rh[2], rh[3]), make_uint4(ih[0], ih[1], ih[2], ih[3]),
                             make_uint4(rl[0], rl[1], rl[2], rl[3]), make_uint4(il[0], il[1], il[2], il[3])};
      tiled_row_store64(a, r, k, jc, c, rows);
      return;
    }
    uint4* dst = reinterpret_cast<uint4*>(a.lop) +
                 (((size_t)(r >> 3) * a.K + k) * 16 * (NCOL / 4) + (c >> 2)) * 32 + (r & 7) * 4 + (c & 3);
    constexpr size_t RS = (size_t)(NCOL / 4) * 32;  // one row
    dst[((0 * 4 + jc) * 2 + 0) * RS] = make_uint4(rh[0], rh[1], rh[2], rh[3]);
    dst[((0 * 4 + jc) * 2 + 1) * RS] = make_uint4(ih[0], ih[1], ih[2], ih[3]);
    dst[((1 * 4 + jc) * 2 + 0) * RS] = make_uint4(rl[0], rl[1], rl[2], rl[3]);
    dst[((1 * 4 + jc) * 2 + 1) * RS] = make_uint4(il[0], il[1], il[2], il[3]);
  }
}

// Tiled rows: zeros for a chunk of the tile's stage plan that this rotation's channel does not
// touch (the x pass's tensor copies load the rows of all 128 rotations of a row set)
__device__ __forceinline__ void tiled_zero_chunk(const WaveArgs& a, int r, int k, int jc, int c) {
  const uint4 z = make_uint4(0u, 0u, 0u, 0u);
  if (a.f16) {
    tiled_row_store(a, r, k, jc, c, z, z);
  } else {
    const uint4 zz[4] = {z, z, z, z};
    tiled_row_store64(a, r, k, jc, c, zz);
  }
}

// The K-step range [lo, hi] of channel k in the stage plan of rotation r's tile (k_tile_plan);
// lo > hi when no rotation of the tile touches the channel
__device__ __forceinline__ void tile_plan_range(const WaveArgs& a, int r, int k, int& lo, int& hi) {
  const unsigned long long* tp = a.rec[r - r % kTileRot].tplan;
  const unsigned long long pk = tp[0], pl = tp[1], ph = tp[2];
  const int nact = (int)(tp[3] & 0xFFFFu);
  lo = 15;
  hi = -1;
  for (int ai = 0; ai < nact; ++ai)
    if ((int)((pk >> (4 * ai)) & 15) == k) {
      lo = (int)((pl >> (4 * ai)) & 15);
      hi = (int)((ph >> (4 * ai)) & 15);
    }
}

// plane kernel CTA order for tiled rows: rotation-major by default; the environment variable
// CDK_PLANE_ORDER=1 keeps the channel-major order, for measurement
int plane_rot_major_host() {
  static const int v = [] {
    const char* e = std::getenv("CDK_PLANE_ORDER");
    return (e && std::atoi(e) == 1) ? 0 : 1;
  }();
  return v;
}

constexpr int kPlaneColsPerThread = 2;  // columns per thread in the plane kernel
constexpr int kDirectMaxAtoms = 96;

template <int N, bool LOP>
__global__ void __launch_bounds__(256, kPlaneColsPerThread == 1 ? 5 : 4) k_spread_yz_direct(WaveArgs a, const int* __restrict__ kyof,
                                                           int cap) {
  constexpr int NZH = N / 2 + 1;
  constexpr int NCOL = N * NZH;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* tw = reinterpret_cast<float2*>(smem_raw);            // [N]
  int4* s_apk = reinterpret_cast<int4*>(tw + N);                // [cap] (x cell, w(xi), w(xi+1), -)
  float2* Fy = reinterpret_cast<float2*>(s_apk + cap);          // [cap][N/2][2]: ky positions p, p + N/2
  float2* Fz = Fy + (size_t)cap * N;                            // [cap][NZH]
  int2* s_yz = reinterpret_cast<int2*>(Fz + (size_t)cap * NZH);  // [cap] y and z cells
  float2* s_rr = reinterpret_cast<float2*>(s_yz + cap);           // [cap] y and z ratios
  int* s_atom = reinterpret_cast<int*>(s_rr + cap);               // [cap]
  __shared__ int s_cnt;
  __shared__ uint32_t s_cm[N / 8][3];  // per 8-plane chunk: the channel atoms touching it (bit j)
  // grid (K, nrot), or (nrot, K) for tiled rows: the CTAs in flight then write whole
  // 128-rotation blocks of one channel together
  const bool rot_major = LOP && a.plane_rot_major;
  const int k = rot_major ? blockIdx.y : blockIdx.x, r = rot_major ? blockIdx.x : blockIdx.y;
  const RotRec* rec = a.rec + r;
  if (!rec->valid) return;
  const int xlo = rec->xlo[k], xhi = rec->xhi[k];
  const int tid = threadIdx.x, nthr = blockDim.x;
  // tiled rows: the chunks of the tile's plan outside this rotation's own range get zeros
  int zlo = 15, zhi = -1;
  if (LOP && a.lop_tiled) tile_plan_range(a, r, k, zlo, zhi);
  if (xlo > xhi) {
    for (int q = zlo; q <= zhi; ++q)
      for (int c = tid; c < NCOL; c += nthr) tiled_zero_chunk(a, r, k, q, c);
    return;
  }
  for (int i = tid; i < N; i += nthr) tw[i] = a.tw[i];
  const RotDesc rd = a.rots[r];
  const ConfDesc cd = a.confs[rd.conf];
  const AtomParam* prm = a.params + cd.param_off;
  const float mn0 = rec->mn[0], mn1 = rec->mn[1], mn2 = rec->mn[2];
  const float h = a.spacing;
  const bool elec = (k == a.K - 1);
  const int nA = rec->nA;
  // channel atoms in ascending order (warp 0, ballot compaction)
  if (tid < 32) {
    int cnt = 0;
    for (int base = 0; base < nA; base += 32) {
      const int i = base + tid;
      const bool in = i < nA && (elec || prm[i].slot == k);
      const unsigned int m = __ballot_sync(0xffffffffu, in);
      if (in) s_atom[cnt + __popc(m & ((1u << tid) - 1))] = i;
      cnt += __popc(m);
    }
    if (tid == 0) s_cnt = cnt;
  }
  __syncthreads();
  const int na = s_cnt;
  // split-FP16 rows carry 2^sigma_k: a power of two, folded exactly into the x weights (every
  // product and sum below then scales exactly, outside under- and overflow)
  const float wsc = (LOP && a.f16) ? a.lscale[k] : 1.f;
  // per atom: cells, ratios and x weights (FillLigandGrid's double arithmetic, once per atom)
  for (int j = tid; j < na; j += nthr) {
    const int at = s_atom[j];
    const float4 p = a.rot_xyz[(size_t)r * a.max_atoms + at];
    const int xi = cell_of(p.x, mn0, h), yi = cell_of(p.y, mn1, h), zi = cell_of(p.z, mn2, h);
    const double xr = ratio_of(p.x, mn0, h, xi);
    const double sc = elec ? (double)prm[at].charge : (double)prm[at].w_vdw;
    s_apk[j] = make_int4(xi, __float_as_int(__fmul_rn((float)(sc * (1.0 - xr)), wsc)),
                         __float_as_int((xi + 1 < N) ? __fmul_rn((float)(sc * xr), wsc) : 0.f), 0);
    s_yz[j] = make_int2(yi, zi);
    s_rr[j] = make_float2((float)ratio_of(p.y, mn1, h, yi), (float)ratio_of(p.z, mn2, h, zi));
  }
  __syncthreads();
  // factor tables
  for (int i = tid; i < na * (N + NZH); i += nthr) {
    const int j = i / (N + NZH), f = i - j * (N + NZH);
    if (f < N) {
      const int yi = s_yz[j].x;
      const float ry = s_rr[j].x;
      const int ky = kyof[f];  // natural frequency of position f
      const float2 w0 = tw[(yi * ky) % N], w1 = tw[((yi + 1) * ky) % N];
      // positions f and f + N/2 side by side: a thread's two columns (ky positions p and
      // p + N/2, the same kz) read both factors in one 16-byte load
      Fy[(size_t)j * N + (f % (N / 2)) * 2 + f / (N / 2)] =
          make_float2((1.f - ry) * w0.x + ry * w1.x, (1.f - ry) * w0.y + ry * w1.y);
    } else {
      const int kz = f - N;
      const int zi = s_yz[j].y;
      const float rz = s_rr[j].y;
      const float2 w0 = tw[(zi * kz) % N], w1 = tw[((zi + 1) * kz) % N];
      Fz[(size_t)j * NZH + kz] = make_float2((1.f - rz) * w0.x + rz * w1.x, (1.f - rz) * w0.y + rz * w1.y);
    }
  }
  __syncthreads();
  // per chunk, the atoms whose planes xi, xi + 1 meet it (warp 0, ballots in atom order)
  const int jc0 = xlo >> 3, njc = (xhi >> 3) - jc0 + 1;  // planes < n: njc <= n / 8
  if (tid < 32) {
    for (int q = 0; q < njc; ++q) {
      const int x0 = 8 * (jc0 + q);
      for (int base = 0; base < 96; base += 32) {
        const int j = base + tid;
        const int o = j < na ? s_apk[j].x - x0 : -2;
        const unsigned int m = __ballot_sync(0xffffffffu, o >= -1 && o <= 7);
        if (tid == 0) s_cm[q][base >> 5] = m;
      }
    }
  }
  __syncthreads();
  // Chunks of 8 planes: every thread owns columns, accumulates a chunk's planes in registers
  // and visits the atoms touching the chunk in ascending order; an atom adds to planes xi and
  // xi + 1, whose offsets in the chunk are the same for the whole CTA (a uniform switch).
  // CPT columns per thread (c, c + NCOL / CPT, ...): the atom visit (list walk, weights, the
  // offset switch) is shared by the columns, each column keeping its own accumulation order.
  if (LOP && a.lop_tiled) {
    for (int q = zlo; q <= zhi; ++q)
      if (q < jc0 || q >= jc0 + njc)
        for (int c = tid; c < NCOL; c += nthr) tiled_zero_chunk(a, r, k, q, c);
  }
  constexpr int CPT = kPlaneColsPerThread;
  static_assert(NCOL % CPT == 0, "column split");
  static_assert(CPT != 2 || (NCOL / 2) % NZH == 0, "paired columns share kz");
  for (int cb = tid; cb < NCOL / CPT; cb += nthr) {
    int kyp[CPT], kz[CPT];
#pragma unroll
    for (int u = 0; u < CPT; ++u) {
      const int c = cb + u * (NCOL / CPT);
      kyp[u] = c / NZH;
      kz[u] = c - kyp[u] * NZH;
    }
    for (int q = 0; q < njc; ++q) {
      const int jc = jc0 + q;
      const int x0 = 8 * jc;
      float ax[CPT][8], ay[CPT][8];
#pragma unroll
      for (int u = 0; u < CPT; ++u)
#pragma unroll
        for (int d = 0; d < 8; ++d) ax[u][d] = ay[u][d] = 0.f;
      // only the atoms touching this chunk, in ascending order (the same for the whole CTA)
      for (int wd = 0; wd < 3; ++wd) {
        for (unsigned int mask = s_cm[q][wd]; mask; mask &= mask - 1) {
          const int j = 32 * wd + __ffs(mask) - 1;
          const int4 pk = s_apk[j];
          const int o = pk.x - x0;
          float gx[CPT], gy[CPT];
          if constexpr (CPT == 2) {
            // columns c and c + NCOL/2: ky positions p and p + N/2, one kz
            const float4 fy2 = *reinterpret_cast<const float4*>(Fy + (size_t)j * N + 2 * kyp[0]);
            const float2 fz = Fz[(size_t)j * NZH + kz[0]];
            gx[0] = fy2.x * fz.x - fy2.y * fz.y;
            gy[0] = fy2.x * fz.y + fy2.y * fz.x;
            gx[1] = fy2.z * fz.x - fy2.w * fz.y;
            gy[1] = fy2.z * fz.y + fy2.w * fz.x;
          } else {
#pragma unroll
            for (int u = 0; u < CPT; ++u) {
              const float2 fy = Fy[(size_t)j * N + (kyp[u] % (N / 2)) * 2 + kyp[u] / (N / 2)];
              const float2 fz = Fz[(size_t)j * NZH + kz[u]];
              gx[u] = fy.x * fz.x - fy.y * fz.y;
              gy[u] = fy.x * fz.y + fy.y * fz.x;
            }
          }
          const float w0 = __int_as_float(pk.y), w1 = __int_as_float(pk.z);
          switch (o) {
#define CDK_PLANE_PAIR(D)                                                  \
  case D:                                                                  \
    _Pragma("unroll") for (int u = 0; u < CPT; ++u) {                      \
      ax[u][D] += w0 * gx[u];                                              \
      ay[u][D] += w0 * gy[u];                                              \
      ax[u][D + 1] += w1 * gx[u];                                          \
      ay[u][D + 1] += w1 * gy[u];                                          \
    }                                                                      \
    break;
            case -1:
#pragma unroll
              for (int u = 0; u < CPT; ++u) {
                ax[u][0] += w1 * gx[u];
                ay[u][0] += w1 * gy[u];
              }
              break;
            CDK_PLANE_PAIR(0)
            CDK_PLANE_PAIR(1)
            CDK_PLANE_PAIR(2)
            CDK_PLANE_PAIR(3)
            CDK_PLANE_PAIR(4)
            CDK_PLANE_PAIR(5)
            CDK_PLANE_PAIR(6)
#undef CDK_PLANE_PAIR
            default:  // o == 7: plane xi + 1 is the next chunk's
#pragma unroll
              for (int u = 0; u < CPT; ++u) {
                ax[u][7] += w0 * gx[u];
                ay[u][7] += w0 * gy[u];
              }
              break;
          }
        }
      }
#pragma unroll
      for (int u = 0; u < CPT; ++u)
        plane_chunk_write<N, LOP>(a, r, k, jc, x0, xlo, xhi, cb + u * (NCOL / CPT), ax[u], ay[u]);
    }
  }
}

// ---------------------------------------------------------------------------------------
// x pass for two-stage plans (N = R0*R1), fused stage by stage; CT spectral columns per CTA:
//   phase A  first forward stage straight from A in global memory (only the x planes a
//            channel touches are read; the rest are known zeros), two channels per round;
//            the next round's loads are issued before this round's phase B to hide latency
//   phase B  second forward stage + conj(L_k) * P_k accumulated in registers over all
//            channels (receptor tile resident in shared memory for the CTA's rotations)
//   combine  pair sum through one shuffle, first inverse stage
//   phase C  last inverse stage, written straight to B for x inside the window
template <int N, int CT>
__global__ void __launch_bounds__(256, 2) k_xpass2(WaveArgs a, int rot_per_cta) {
  constexpr int NZH = N / 2 + 1;
  constexpr int NCOL = N * NZH;
  constexpr int R0 = FFTPlan<N>::R0, R1 = FFTPlan<N>::R1, M1 = N / R0;
  constexpr int NA = 2 * CT * M1;  // phase-A items
  constexpr int NB = 2 * CT * R0;  // phase-B items
  static_assert(FFTPlan<N>::NS == 2, "two-stage plans only");
  static_assert(NA <= 256 && NB <= 256, "one item per thread");
  static_assert(NCOL % CT == 0, "column tiles must divide the half spectrum");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int K = a.K;
  float2* tw = reinterpret_cast<float2*>(smem_raw);
  int* s_ch = reinterpret_cast<int*>(tw + N);               // [KMAX] channel ids, [KMAX] count
  short* s_rng = reinterpret_cast<short*>(s_ch + 2 * KMAX);  // [KMAX][2] x range per slot
  float2* Ps = reinterpret_cast<float2*>(s_rng + 4 * KMAX);  // [N][K][CT]
  float2* Wb = Ps + (size_t)N * K * CT;                      // [N][2][CT]
  float2* S = Wb + (size_t)N * 2 * CT;                       // [N][CT]
  const int c0 = blockIdx.x * CT;
  const int tid = threadIdx.x;
  for (int i = tid; i < N; i += 256) tw[i] = a.tw[i];
  for (int i = tid; i < N * K * CT; i += 256) {
    const int c = i % CT, t = i / CT;  // t = pos*K + k
    Ps[i] = a.phat[(size_t)t * NCOL + c0 + c];
  }
  // per-thread roles
  const int a_c = tid % CT, a_half = (tid / CT) & 1, a_np = tid / (2 * CT);
  const int b_half = tid & 1, b_c = (tid >> 1) % CT, b_b = (tid >> 1) / CT;
  const int r_begin = blockIdx.y * rot_per_cta;
  const int r_end = min(a.nrot, r_begin + rot_per_cta);
  for (int r = r_begin; r < r_end; ++r) {
    const RotRec* rec = a.rec + r;
    if (!rec->valid) continue;
    __syncthreads();  // previous rotation is done with s_ch / Wb / S
    if (tid == 0) {
      int nk = 0;
      for (int k = 0; k < K; ++k)
        if (rec->xlo[k] <= rec->xhi[k]) {
          s_rng[2 * nk] = rec->xlo[k];
          s_rng[2 * nk + 1] = rec->xhi[k];
          s_ch[nk++] = k;
        }
      s_ch[KMAX] = nk;
    }
    __syncthreads();
    const int nk = s_ch[KMAX];
    const float2* Ar = a.A + ((size_t)r * K) * a.Lb * NCOL + c0 + a_c;
    // raw loads of one round (channels kk0, kk0+1) for this thread's phase-A item
    auto load_round = [&](int kk0, float2* v) {
      const int kk = kk0 + a_half;
      if (tid < NA && kk < nk) {
        const int k = s_ch[kk];
        const int lo = s_rng[2 * kk], hi = s_rng[2 * kk + 1];
        const float2* src = Ar + (size_t)k * a.Lb * NCOL;
#pragma unroll
        for (int j = 0; j < R0; ++j) {
          const int x = a_np + j * M1;
          v[j] = (x >= lo && x <= hi) ? src[(size_t)x * NCOL] : make_float2(0.f, 0.f);
        }
      } else {
#pragma unroll
        for (int j = 0; j < R0; ++j) v[j] = make_float2(0.f, 0.f);
      }
    };
    float2 acc[R1];
#pragma unroll
    for (int j = 0; j < R1; ++j) acc[j] = make_float2(0.f, 0.f);
    float2 va[R0];
    load_round(0, va);
    for (int k0 = 0; k0 < nk; k0 += 2) {
      // phase A: first forward stage into Wb
      if (tid < NA) {
        Radix<R0, -1>::run(va);
#pragma unroll
        for (int q = 1; q < R0; ++q) va[q] = c_mul(va[q], tw[a_np * q]);
#pragma unroll
        for (int q = 0; q < R0; ++q) Wb[((a_np + q * M1) * 2 + a_half) * CT + a_c] = va[q];
      }
      __syncthreads();
      if (k0 + 2 < nk) load_round(k0 + 2, va);  // in flight during phase B
      // phase B: second forward stage and the conjugate product, accumulated
      const int kk = k0 + b_half;
      if (tid < NB && kk < nk) {
        const int k = s_ch[kk];
        float2 v[R1];
#pragma unroll
        for (int j = 0; j < R1; ++j) v[j] = Wb[((b_b * R1 + j) * 2 + b_half) * CT + b_c];
        Radix<R1, -1>::run(v);
#pragma unroll
        for (int q = 0; q < R1; ++q) {
          const float2 p = Ps[((b_b * R1 + q) * K + k) * CT + b_c];
          acc[q].x += v[q].x * p.x + v[q].y * p.y;
          acc[q].y += v[q].x * p.y - v[q].y * p.x;
        }
      }
      __syncthreads();
    }
    // combine the pair (lanes tid, tid^1), first inverse stage, into S
    if (tid < ((NB + 31) & ~31)) {
      float2 v[R1];
#pragma unroll
      for (int j = 0; j < R1; ++j) {
        v[j].x = acc[j].x + __shfl_xor_sync(0xffffffffu, acc[j].x, 1);
        v[j].y = acc[j].y + __shfl_xor_sync(0xffffffffu, acc[j].y, 1);
      }
      if (tid < NB && b_half == 0) {
        Radix<R1, +1>::run(v);
#pragma unroll
        for (int j = 0; j < R1; ++j) S[(b_b * R1 + j) * CT + b_c] = v[j];
      }
    }
    __syncthreads();
    // phase C: last inverse stage, window rows only
    const int Wx = rec->W[0];
    if (tid < CT * M1) {
      const int c = tid % CT, np = tid / CT;
      float2 v[R0];
#pragma unroll
      for (int q = 0; q < R0; ++q) {
        v[q] = S[(np + q * M1) * CT + c];
        if (q > 0) v[q] = c_mulc(v[q], tw[np * q]);
      }
      Radix<R0, +1>::run(v);
      float2* dst = a.B + (size_t)r * N * NCOL + c0 + c;
#pragma unroll
      for (int j = 0; j < R0; ++j) {
        const int x = np + j * M1;
        if (x < Wx) dst[(size_t)x * NCOL] = v[j];
      }
    }
  }
}

// ---------------------------------------------------------------------------------------
// Plane x of rotation r read from B in any of its layouts; at(f) is column f of the plane.
// Column-pair groups (cs = 1): float2 (f >> 1) 2G + (f & 1) past the plane's first pair; single-
// column groups (cs = 0): float2 f G past the plane's first column. The plain layout is G = 1.
// BL fixes the layout at compile time (the loads of a butterfly then share one base address):
// kBPlain, kBPairs2 (column pairs, G = 2), kBSingle4 (single columns, G = 4); kBAny reads the
// layout from WaveArgs.
constexpr int kBAny = 0, kBPlain = 1, kBPairs2 = 2, kBSingle4 = 3;
template <int BL>
struct BPlane {
  const float2* p;
  int cs, gs;
  __device__ __forceinline__ BPlane(const WaveArgs& a, int r, int x, int n, int ncol) {
    const int G = BL == kBPlain ? 1 : BL == kBPairs2 ? 2 : BL == kBSingle4 ? 4 : (a.bgroup > 1 ? a.bgroup : 1);
    cs = BL == kBSingle4 ? 0 : BL == kBAny ? (a.bcol ? 0 : 1) : 1;
    gs = G << cs;
    p = a.B + ((size_t)r * n + (x - x % G)) * ncol + ((x % G) << cs);
  }
  __device__ __forceinline__ float2 at(int f) const {
    if constexpr (BL == kBPlain) return p[f];
    else if constexpr (BL == kBPairs2) return p[(f >> 1) * 4 + (f & 1)];
    else if constexpr (BL == kBSingle4) return p[f * 4];
    else return p[(size_t)(f >> cs) * gs + (f & cs)];
  }
};
// the compile-time layout of a wave's B (kBAny for the others)
inline int b_layout(const WaveArgs& a) {
  if (a.bcol) return a.bgroup == 4 ? kBSingle4 : kBAny;
  return a.bgroup <= 1 ? kBPlain : a.bgroup == 2 ? kBPairs2 : kBAny;
}

// keep the two smallest keys (b1 < b2) of a stream of distinct keys
__device__ __forceinline__ void top2_insert(unsigned long long k, unsigned long long& b1, unsigned long long& b2) {
  // most candidates lose to the current second-smallest on the energy bits alone (one 32-bit
  // compare); the 64-bit order decides the rest
  if ((unsigned int)(k >> 32) > (unsigned int)(b2 >> 32)) return;
  if (k < b1) {
    b2 = b1;
    b1 = k;
  } else if (k < b2) {
    b2 = k;
  }
}
// merge another pair of two smallest into (b1, b2)
__device__ __forceinline__ void top2_merge(unsigned long long o1, unsigned long long o2, unsigned long long& b1,
                                           unsigned long long& b2) {
  const unsigned long long n1 = o1 < b1 ? o1 : b1;
  const unsigned long long hi = o1 < b1 ? b1 : o1;
  const unsigned long long lo2 = o2 < b2 ? o2 : b2;
  b2 = hi < lo2 ? hi : lo2;
  b1 = n1;
}

// Candidate energies e at linear index lin, into a thread's smallest key (b1) or two smallest
// keys (b1, b2). thr is the float of the largest key kept (+inf while a slot is empty): a value
// strictly above it (as floats, the same order as the keys) cannot enter and is rejected before
// its key is built; equal values, NaN and signed zeros take the exact 64-bit key path.
template <bool TOP2>
__device__ __forceinline__ void keep_min(float e, unsigned int lin, unsigned long long& b1, unsigned long long& b2,
                                         float& thr) {
  if (e > thr) return;
  const unsigned long long k = ((unsigned long long)order_key(e) << 32) | lin;
  if constexpr (TOP2) {
    top2_insert(k, b1, b2);
    thr = b2 == ~0ull ? INFINITY : key_to_float((unsigned int)(b2 >> 32));
  } else {
    if (k < b1) {
      b1 = k;
      thr = key_to_float((unsigned int)(k >> 32));
    }
  }
}

// smallest 64-bit key of the warp: redux on the high words, then on the low words of the lanes
// holding the smallest high word
__device__ __forceinline__ unsigned long long warp_min_key(unsigned long long k) {
  const unsigned int hi = __reduce_min_sync(0xffffffffu, (unsigned int)(k >> 32));
  const unsigned int lo = __reduce_min_sync(0xffffffffu, (unsigned int)(k >> 32) == hi ? (unsigned int)k : 0xffffffffu);
  return ((unsigned long long)hi << 32) | lo;
}
// the warp's two smallest keys from every lane's (b1 < b2) of distinct keys: the smallest b1,
// then the smallest of (b2 on the lane holding it, b1 elsewhere)
template <bool TOP2>
__device__ __forceinline__ void warp_keep_min(unsigned long long& b1, unsigned long long& b2) {
  const unsigned long long k1 = warp_min_key(b1);
  if constexpr (TOP2) b2 = warp_min_key(b1 == k1 ? b2 : b1);
  b1 = k1;
}

// inverse (y,z) of one (rotation, x in window) plane + min / first argmin; TOP2: also the
// plane's second-smallest key, for the FP64 near-tie break (WaveArgs.keys2)
template <int N, bool TOP2, int BL>
__global__ void __launch_bounds__(256, (N <= 64 ? 8 : 2)) k_yz_inv_argmin(WaveArgs a) {
  constexpr int NZH = N / 2 + 1;
  constexpr int NCOL = N * NZH;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* tw = reinterpret_cast<float2*>(smem_raw);
  float2* O = tw + N;
  // n <= 64: the packed rows P overwrite O once O has been read (N/2 x (N+1) <= N x (N/2+1)
  // entries), so a CTA holds one plane and the SM more CTAs; larger n keep P apart (the pack
  // would hold too many values in registers)
  constexpr bool ALIAS = N <= 64;
  float2* P = ALIAS ? O : O + N * NZH;
  static_assert((N / 2) * (N + 1) <= N * NZH, "packed rows fit the plane buffer");
  __shared__ unsigned long long s_best[8], s_best2[8];
  const int x = blockIdx.x, r = blockIdx.y;
  const RotRec* rec = a.rec + r;
  if (!rec->valid) return;
  const int Wx = rec->W[0], Wy = rec->W[1], Wz = rec->W[2];
  if (x >= Wx) return;
  const int tid = threadIdx.x, nthr = blockDim.x;
  for (int i = tid; i < N; i += nthr) tw[i] = a.tw[i];
  // plane x: NCOL / 2 column pairs, 16 B each, contiguous (plain layout) or every G-th of the
  // plane group (grouped layout, G planes per 16 B x column-pair block); or, single-column
  // groups, one float2 of every G
  const BPlane<BL> bp(a, r, x, N, NCOL);
  if constexpr (ALIAS) {
    // y: positions -> natural rows, the first (R1-point, twiddle-free) stage reading its rows
    // straight from B: item (column l, block b) takes positions b R1 + j of column l, plane
    // entry f = row * NZH + l, which is half f % 2 of column pair f / 2
    using PL = FFTPlan<N>;
    constexpr int R0 = PL::R0, R1 = PL::R1;
    static_assert(PL::NS == 2 && StageM<N, 2>::value == 1, "two-stage plan");
    for (int w = tid; w < NZH * R0; w += nthr) {
      const int b = w / NZH, l = w - b * NZH;
      float2 v[R1];
#pragma unroll
      for (int j = 0; j < R1; ++j) v[j] = bp.at((b * R1 + j) * NZH + l);
      Radix<R1, +1>::run(v);
      float2* p = O + l + b * R1 * NZH;
#pragma unroll
      for (int j = 0; j < R1; ++j) p[j * NZH] = v[j];
    }
    __syncthreads();
    fft_stage<N, R0, StageM<N, 1>::value, true>(O, NZH, 1, NZH, tw, tid, nthr);
    __syncthreads();
  } else {
    for (int i = tid; i < NCOL; i += nthr) O[i] = bp.at(i);
    __syncthreads();
    fft_lines<N, true>(O, NZH, 1, NZH, tw, tid, nthr);  // y: positions -> natural rows
  }
  const int npairs = (Wy + 1) / 2;
  const float inv = 1.0f / (float)((double)N * N * N);
  unsigned long long best = ~0ull, best2 = ~0ull;
  float thr = INFINITY;
  if constexpr (ALIAS) {
    // Rows (2p, 2p+1) as one complex line Z_p(k) = Y(2p, k) + i Y(2p+1, k) with the Hermitian
    // extension over z, inverse-transformed in two radix stages (N = R0 R1), one work item per
    // thread and stage (line p fastest). The pack is folded into the first stage's loads and
    // the window argmin into the last stage, so neither the packed input nor the energies take
    // a trip through shared memory.
    using PL = FFTPlan<N>;
    constexpr int R0 = PL::R0, R1 = PL::R1;
    static_assert(PL::NS == 2 && R0 * R1 == N && R1 % 2 == 0, "two-stage plan");
    static_assert((N / 2) * R0 <= 256 && (N / 2) * R1 <= 256, "one item per thread of 256");
    // item w -> (line w % npairs, block w / npairs); (w + 0.5) / npairs stays >= 1/64 away from
    // an integer for w < 256, npairs <= 32, far above the float rounding of the product
    const float rinv = npairs > 0 ? __frcp_rn((float)npairs) : 0.f;
    // stage 1 (R1-point, no twiddles): block b reads natural frequencies k = b + R0 j, which sit
    // at digit-reversed positions b R1 + j; k >= N/2 exactly when j >= R1/2
    const bool has1 = tid < npairs * R0;
    int l1 = 0, b1 = 0;
    float2 v1[R1];
    if (has1) {
      b1 = (int)(((float)tid + 0.5f) * rinv);
      l1 = tid - b1 * npairs;
      const float2* A = O + (2 * l1) * NZH;
      const float2* Bv = A + NZH;
#pragma unroll
      for (int j = 0; j < R1; ++j) {
        const int k = b1 + R0 * j;
        if (j < R1 / 2) {
          const float2 ak = A[k], bk = Bv[k];
          v1[j] = make_float2(ak.x - bk.y, ak.y + bk.x);
          if (j == 0 && b1 == 0) v1[j] = make_float2(ak.x, bk.x);  // k = 0
        } else {
          const int m = N - k;
          const float2 am = A[m], bm = Bv[m];
          v1[j] = make_float2(am.x + bm.y, -am.y + bm.x);
          if (j == R1 / 2 && b1 == 0) v1[j] = make_float2(am.x, bm.x);  // k = N/2
        }
      }
    }
    __syncthreads();  // every read of the y-transformed rows is done: the lines overwrite them
    if (has1) {
      Radix<R1, +1>::run(v1);
      float2* dst = P + l1 * (N + 1) + b1 * R1;
#pragma unroll
      for (int j = 0; j < R1; ++j) dst[j] = v1[j];
    }
    __syncthreads();
    // stage 2 (R0-point, twiddles tw[np k]): item np yields z = np + R1 j; line l holds row 2l in
    // its real part and row 2l + 1 in its imaginary part
    if (tid < npairs * R1) {
      const int np = (int)(((float)tid + 0.5f) * rinv);
      const int l = tid - np * npairs;
      const float2* src = P + l * (N + 1) + np;
      float2 v[R0];
#pragma unroll
      for (int j = 0; j < R0; ++j) v[j] = src[j * R1];
#pragma unroll
      for (int k = 1; k < R0; ++k) v[k] = c_mulc(v[k], tw[np * k]);
      Radix<R0, +1>::run(v);
      const int y0 = 2 * l;
      const bool row0 = y0 < Wy, row1 = y0 + 1 < Wy;
      const unsigned int lin0 = (unsigned int)((x * N + y0) * N + np);
#pragma unroll
      for (int j = 0; j < R0; ++j) {
        if (np + R1 * j < Wz) {
          if (row0) keep_min<TOP2>(v[j].x * inv, lin0 + (unsigned int)(R1 * j), best, best2, thr);
          if (row1) keep_min<TOP2>(v[j].y * inv, lin0 + (unsigned int)(N + R1 * j), best, best2, thr);
        }
      }
    }
  } else {
    // pack rows (2p, 2p+1) as one complex line with Hermitian extension over z (into its own
    // buffer), inverse-transform the lines, then take the window minimum from shared memory
    for (int i = tid; i < npairs * N; i += nthr) {
      const int p = i / N, k = i - p * N;
      const float2* A = O + (2 * p) * NZH;
      const float2* Bv = O + (2 * p + 1) * NZH;
      float2 z;
      if (k == 0 || k == N / 2) {
        z = make_float2(A[k].x, Bv[k].x);
      } else if (k < N / 2) {
        z = make_float2(A[k].x - Bv[k].y, A[k].y + Bv[k].x);
      } else {
        const int m = N - k;
        z = make_float2(A[m].x + Bv[m].y, -A[m].y + Bv[m].x);
      }
      P[p * (N + 1) + fft_pos<N>(k)] = z;
    }
    __syncthreads();
    if constexpr (FFTPlan<N>::NS == 2) {
      ifft_lines_slots<N, N / 2>(P, npairs, N + 1, 1, tw, tid, nthr);
    } else {
      fft_lines<N, true>(P, npairs, N + 1, 1, tw, tid, nthr);
    }
    // window rows by warp, columns by lane (the key carries the index: order does not matter)
    for (int y = tid >> 5; y < Wy; y += nthr >> 5) {
      const float2* row = P + (y >> 1) * (N + 1);
      for (int z = tid & 31; z < Wz; z += 32) {
        const float2 v = row[z];
        const float e = ((y & 1) ? v.y : v.x) * inv;
        keep_min<TOP2>(e, (unsigned int)((x * N + y) * N + z), best, best2, thr);
      }
    }
  }
  warp_keep_min<TOP2>(best, best2);
  if ((tid & 31) == 0) {
    s_best[tid >> 5] = best;
    if constexpr (TOP2) s_best2[tid >> 5] = best2;
  }
  __syncthreads();
  if (tid < 32) {
    const int nw = nthr >> 5;
    best = tid < nw ? s_best[tid] : ~0ull;
    if constexpr (TOP2) best2 = tid < nw ? s_best2[tid] : ~0ull;
    warp_keep_min<TOP2>(best, best2);
    if (tid == 0) {
      atomicMin(a.keys + r, best);
      if constexpr (TOP2) {
        a.keys2[((size_t)r * N + x) * 2] = best;
        a.keys2[((size_t)r * N + x) * 2 + 1] = best2;
      }
    }
  }
}

// Inverse (y,z) of one (rotation, x in window) plane + min / first argmin with warp-local line
// transforms, for n = 8 R1 (R1 = 4, 8, 12, 16). An octet of 8 lanes owns one line (a kz column
// for y, a packed row pair for z). The inverse runs the forward plan's two stages backwards:
// stage 1, radix R1 over the 8 contiguous blocks of R1 digit-reversed positions (lane t holds
// block t in registers); stage 2, radix 8 over the R1 groups {np + R1 j} with twiddles
// tw[np k] (lane t takes groups np = t, t + 8, ...), giving natural index np + R1 j. The
// exchange between the two stages goes through the line's own storage in the plane buffer
// (y: its kz column, rows at stride N/2+1; z: the two rows of its row pair, N + 2 slots), with
// __syncwarp only. Stage-1 output m of block t sits at line position t R1 + (m + t) mod R1 --
// block t rotated by t -- so the 8 lanes' stores of one m, and the 8 lanes' loads of one block
// in stage 2, fall in 8 different banks (odd row stride). In the y pass stage 2 gathers both
// of its groups before any lane writes the natural outputs back into the column. Block-wide
// barriers: after the twiddle load, between the y and z passes (the y output is the z input),
// and in the final reduction. Shared memory is the twiddles and the plane only (68 KB at
// 128^3), so three CTAs of 288 threads (72 registers) fit an SM. Same radix stages, twiddles
// and packing as k_yz_inv_argmin.
// 288 threads = 36 octets: the 33 kz columns (and at most 32 row pairs) of a 64^3 plane in one
// round each, 49 / 65 columns at 96^3 / 128^3 in two
constexpr int kOctWarps = 9;
constexpr int kOctets = 4 * kOctWarps;

template <int N>
constexpr size_t octet_smem() {
  return sizeof(float2) * (N + (size_t)N * (N / 2 + 1));
}

template <int N, bool TOP2, int BL>
__global__ void __launch_bounds__(32 * kOctWarps, 3) k_yz_octet(WaveArgs a) {
  constexpr int NZH = N / 2 + 1, NCOL = N * NZH;
  constexpr int R1 = N / 8;           // stage-1 radix; stage 2 is radix 8
  constexpr int NG = (R1 + 7) / 8;    // stage-2 groups per lane
  static_assert(N % 8 == 0 && (R1 == 4 || R1 == 8 || R1 == 12 || R1 == 16), "n = 8 R1");
  static_assert(NZH % 2 == 1, "odd row stride");
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* s_tw = reinterpret_cast<float2*>(smem_raw);
  float2* s_y = s_tw + N;  // y-transformed rows Y[y][kz]
  __shared__ unsigned long long s_best[kOctWarps], s_best2[kOctWarps];
  const int x = blockIdx.x, r = blockIdx.y;
  const RotRec* rec = a.rec + r;
  if (!rec->valid) return;
  const int Wx = rec->W[0], Wy = rec->W[1], Wz = rec->W[2];
  if (x >= Wx) return;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int o = lane >> 3, t = lane & 7, g = warp * 4 + o;
  for (int i = tid; i < N; i += 32 * kOctWarps) s_tw[i] = a.tw[i];
  const BPlane<BL> bp(a, r, x, N, NCOL);
  __syncthreads();
  // line position of stage-1 output m of block blk
  auto xpos = [](int blk, int m) { return blk * R1 + (m + blk) % R1; };
  // y: columns l = g, g + 36, ...; a warp stops when none of its octets has a column left
  constexpr int YR = (NZH + kOctets - 1) / kOctets;
#pragma unroll 1
  for (int it = 0; it < YR; ++it) {
    if (warp * 4 + kOctets * it >= NZH) break;  // warp-uniform
    const int l = g + kOctets * it;
    const bool act = l < NZH;
    float2* col = s_y + (act ? l : 0);
    float2 v[R1];
#pragma unroll
    for (int j = 0; j < R1; ++j) v[j] = act ? bp.at((t * R1 + j) * NZH + l) : make_float2(0.f, 0.f);
    Radix<R1, +1>::run(v);
    if (act) {
#pragma unroll
      for (int j = 0; j < R1; ++j) col[xpos(t, j) * NZH] = v[j];
    }
    __syncwarp();
    float2 u[NG][8];
#pragma unroll
    for (int q = 0; q < NG; ++q) {
      const int np = t + 8 * q;
#pragma unroll
      for (int j = 0; j < 8; ++j) u[q][j] = (act && np < R1) ? col[xpos(j, np) * NZH] : make_float2(0.f, 0.f);
    }
    __syncwarp();  // every group of the line gathered before any natural output is written
#pragma unroll
    for (int q = 0; q < NG; ++q) {
      const int np = t + 8 * q;
      if (act && np < R1) {
#pragma unroll
        for (int k = 1; k < 8; ++k) u[q][k] = c_mulc(u[q][k], s_tw[np * k]);
        Radix<8, +1>::run(u[q]);
#pragma unroll
        for (int j = 0; j < 8; ++j) col[(np + R1 * j) * NZH] = u[q][j];
      }
    }
  }
  __syncthreads();
  // z: rows (2p, 2p + 1) packed as one complex line, Hermitian extension over z
  const int npairs = (Wy + 1) / 2;
  const float inv = 1.0f / (float)((double)N * N * N);
  unsigned long long best = ~0ull, best2 = ~0ull;
  float thr = INFINITY;
  constexpr int ZR = (N / 2 + kOctets - 1) / kOctets;
#pragma unroll 1
  for (int it = 0; it < ZR; ++it) {
    if (warp * 4 + kOctets * it >= npairs) break;  // warp-uniform
    const int p = g + kOctets * it;
    const bool act = p < npairs;
    float2* rows = s_y + (size_t)(2 * (act ? p : 0)) * NZH;  // rows 2p, 2p + 1: N + 2 slots
    const float2* A = rows;
    const float2* Bv = rows + NZH;
    float2 v[R1];
#pragma unroll
    for (int j = 0; j < R1; ++j) {
      const int k = t + 8 * j;  // natural frequency at digit-reversed position t R1 + j
      if (!act) {
        v[j] = make_float2(0.f, 0.f);
      } else if (j < R1 / 2) {
        const float2 ak = A[k], bk = Bv[k];
        v[j] = make_float2(ak.x - bk.y, ak.y + bk.x);
        if (j == 0 && t == 0) v[j] = make_float2(ak.x, bk.x);  // k = 0
      } else {
        const int m = N - k;
        const float2 am = A[m], bm = Bv[m];
        v[j] = make_float2(am.x + bm.y, -am.y + bm.x);
        if (j == R1 / 2 && t == 0) v[j] = make_float2(am.x, bm.x);  // k = N/2
      }
    }
    __syncwarp();  // the octet has read its rows: their slots become the exchange
    Radix<R1, +1>::run(v);
    if (act) {
#pragma unroll
      for (int j = 0; j < R1; ++j) rows[xpos(t, j)] = v[j];
    }
    __syncwarp();
    const int y0 = 2 * p;
    const bool row0 = act && y0 < Wy, row1 = act && y0 + 1 < Wy;
#pragma unroll
    for (int q = 0; q < NG; ++q) {
      const int np = t + 8 * q;
      if (act && np < R1) {
        float2 u[8];
#pragma unroll
        for (int j = 0; j < 8; ++j) u[j] = rows[xpos(j, np)];
#pragma unroll
        for (int k = 1; k < 8; ++k) u[k] = c_mulc(u[k], s_tw[np * k]);
        Radix<8, +1>::run(u);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          const int z = np + R1 * j;
          if (z < Wz) {
            const unsigned int lin0 = (unsigned int)((x * N + y0) * N + z);
            if (row0) keep_min<TOP2>(u[j].x * inv, lin0, best, best2, thr);
            if (row1) keep_min<TOP2>(u[j].y * inv, lin0 + N, best, best2, thr);
          }
        }
      }
    }
  }
  warp_keep_min<TOP2>(best, best2);
  if (lane == 0) {
    s_best[warp] = best;
    if constexpr (TOP2) s_best2[warp] = best2;
  }
  __syncthreads();
  if (warp == 0) {
    best = lane < kOctWarps ? s_best[lane] : ~0ull;
    if constexpr (TOP2) best2 = lane < kOctWarps ? s_best2[lane] : ~0ull;
    warp_keep_min<TOP2>(best, best2);
    if (lane == 0) {
      atomicMin(a.keys + r, best);
      if constexpr (TOP2) {
        a.keys2[((size_t)r * N + x) * 2] = best;
        a.keys2[((size_t)r * N + x) * 2 + 1] = best2;
      }
    }
  }
}

// FP64 energy of rotation r at translation (ti, tj, tk): the direct trilinear grid-energy sum
// over its rotated atoms (k_prep's rot_xyz and min corner), cells and ratios in
// FillLigandGrid's arithmetic, accumulated in double across the warp's lanes (atoms).
__device__ double pose_energy_fp64(const WaveArgs& a, const float* grids, int r, int ti, int tj, int tk,
                                   int lane) {
  const RotRec* rec = a.rec + r;
  const RotDesc rd = a.rots[r];
  const ConfDesc cd = a.confs[rd.conf];
  const AtomParam* prm = a.params + cd.param_off;
  const int n = a.n, K = a.K;
  const size_t Ng = (size_t)n * n * n;
  const float h = a.spacing;
  double e = 0.0;
  for (int i = lane; i < rec->nA; i += 32) {
    const float4 p4 = a.rot_xyz[(size_t)r * a.max_atoms + i];
    const float p[3] = {p4.x, p4.y, p4.z};
    int ci[3];
    double rr[3];
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      ci[d] = cell_of(p[d], rec->mn[d], h);
      rr[d] = ratio_of(p[d], rec->mn[d], h, ci[d]);
    }
    const AtomParam ap = prm[i];
#pragma unroll
    for (int c = 0; c < 8; ++c) {
      const int dx = (c >> 2) & 1, dy = (c >> 1) & 1, dz = c & 1;
      const int gx = ci[0] + dx + ti, gy = ci[1] + dy + tj, gz = ci[2] + dz + tk;
      if (gx >= n || gy >= n || gz >= n) continue;
      const double w = (dx ? rr[0] : 1.0 - rr[0]) * (dy ? rr[1] : 1.0 - rr[1]) * (dz ? rr[2] : 1.0 - rr[2]);
      const size_t g = ((size_t)gx * n + gy) * n + gz;
      if (ap.slot >= 0 && ap.slot < K - 1) e += (double)ap.w_vdw * w * (double)grids[(size_t)ap.slot * Ng + g];
      e += (double)ap.charge * w * (double)grids[(size_t)(K - 1) * Ng + g];
    }
  }
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
  return e;
}

// FP64 near-tie break of the argmin (precision forms), warp per rotation: the two smallest keys
// over the rotation's window planes; when the second energy lies within tol * max(|E1|, 1) of
// the first, both translations are re-scored in FP64 (pose_energy_fp64) and the lower one is
// kept -- the smaller linear index (x-major first) on an exact FP64 tie. The reported energy
// stays the search's own value at the kept translation. work[4] counts re-scored rotations,
// work[5] the ones whose translation changed.
__global__ void __launch_bounds__(128) k_tiebreak(WaveArgs a, const float* __restrict__ grids, float tol) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int r = blockIdx.x * 4 + warp;
  if (r >= a.nrot) return;
  const RotRec* rec = a.rec + r;
  if (!rec->valid) return;
  const int n = a.n;
  unsigned long long b1 = ~0ull, b2 = ~0ull;
  for (int x = lane; x < rec->W[0]; x += 32)
    top2_merge(a.keys2[((size_t)r * n + x) * 2], a.keys2[((size_t)r * n + x) * 2 + 1], b1, b2);
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long o1 = __shfl_xor_sync(0xffffffffu, b1, o);
    const unsigned long long o2 = __shfl_xor_sync(0xffffffffu, b2, o);
    top2_merge(o1, o2, b1, b2);
  }
  if (b1 == ~0ull || b2 == ~0ull) return;
  const float e1 = key_to_float((unsigned int)(b1 >> 32)), e2 = key_to_float((unsigned int)(b2 >> 32));
  if (!(e2 - e1 <= tol * fmaxf(fabsf(e1), 1.f))) return;
  const unsigned int l1 = (unsigned int)b1, l2 = (unsigned int)b2;
  const double f1 = pose_energy_fp64(a, grids, r, l1 / (n * n), (l1 / n) % n, l1 % n, lane);
  const double f2 = pose_energy_fp64(a, grids, r, l2 / (n * n), (l2 / n) % n, l2 % n, lane);
  if (lane == 0) {
    const bool flip = f2 < f1 || (f2 == f1 && l2 < l1);
    if (flip) a.keys[r] = b2;
    if (a.work) {
      atomicAdd(a.work + 4, 1ull);
      if (flip) atomicAdd(a.work + 5, 1ull);
    }
  }
}

// FP64 re-score of the k lowest-energy poses of a wave (precision forms), one CTA: the k
// smallest final keys (energy, then the rotation's place in the wave) by k rounds of a block
// minimum over each thread's own sorted candidates, then one warp per pose for its FP64 direct
// grid-energy sum at its kept translation. out[j]: the rotation's output slot, the search's
// energy, its translation's linear index and the FP64 energy; unused slots get out = -1.
__global__ void __launch_bounds__(256) k_topk_rescore(WaveArgs a, const float* __restrict__ grids, int k,
                                                      TopPose* __restrict__ out) {
  __shared__ unsigned long long s_min[8];
  __shared__ unsigned long long s_pick[kTopMax];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // per thread: its kTopMax smallest (energy bits, rotation) keys, ascending
  unsigned long long cand[kTopMax];
#pragma unroll
  for (int j = 0; j < kTopMax; ++j) cand[j] = ~0ull;
  for (int r = tid; r < a.nrot; r += blockDim.x) {
    const RotRec* rec = a.rec + r;
    const unsigned long long key = a.keys[r];
    if (!rec->valid || key == ~0ull) continue;
    unsigned long long c = (key & 0xffffffff00000000ull) | (unsigned int)r;
#pragma unroll
    for (int j = 0; j < kTopMax; ++j) {
      const unsigned long long lo = c < cand[j] ? c : cand[j];
      c = c < cand[j] ? cand[j] : c;
      cand[j] = lo;
    }
  }
  int head = 0;
  for (int j = 0; j < k; ++j) {
    unsigned long long m = head < kTopMax ? cand[0] : ~0ull;
    for (int o = 16; o > 0; o >>= 1) {
      const unsigned long long v = __shfl_xor_sync(0xffffffffu, m, o);
      m = v < m ? v : m;
    }
    if (lane == 0) s_min[warp] = m;
    __syncthreads();
    unsigned long long g = s_min[0];
    for (int w = 1; w < 8; ++w) g = s_min[w] < g ? s_min[w] : g;
    if (tid == 0) s_pick[j] = g;
    // the owner pops its head (keys are unique: one rotation each)
    if (g != ~0ull && cand[0] == g) {
#pragma unroll
      for (int q = 0; q + 1 < kTopMax; ++q) cand[q] = cand[q + 1];
      cand[kTopMax - 1] = ~0ull;
      ++head;
    }
    __syncthreads();
  }
  for (int j = warp; j < k; j += 8) {
    const unsigned long long g = s_pick[j];
    TopPose tp;
    tp.out = -1;
    tp.lin = -1;
    tp.e = INFINITY;
    tp.e64 = 0.0;
    if (g != ~0ull) {
      const int r = (int)(unsigned int)g;
      const unsigned int lin = (unsigned int)a.keys[r];
      const int n = a.n;
      const double e64 = pose_energy_fp64(a, grids, r, lin / (n * n), (lin / n) % n, lin % n, lane);
      tp.out = a.rots[r].out;
      tp.lin = (int)lin;
      tp.e = key_to_float((unsigned int)(a.keys[r] >> 32));
      tp.e64 = e64;
    }
    if (lane == 0) out[j] = tp;
  }
}

__global__ void k_finalize(WaveArgs a) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= a.nrot) return;
  const int out = a.rots[r].out;
  const RotRec* rec = a.rec + r;
  if (rec->err == 1) atomicAdd(a.err_count, 1);  // err 2 is reported through range_err
  if (rec->valid) {
    unsigned long long planes = 0;
    for (int k = 0; k < a.K; ++k)
      if (rec->xlo[k] <= rec->xhi[k]) planes += (unsigned long long)(rec->xhi[k] - rec->xlo[k] + 1);
    atomicAdd(a.work, planes);
    atomicAdd(a.work + 1, (unsigned long long)rec->W[0]);
  }
  const unsigned long long key = a.keys[r];
  if (!rec->valid || key == ~0ull) {
    a.minE[out] = INFINITY;
    a.idx[out * 3 + 0] = a.idx[out * 3 + 1] = a.idx[out * 3 + 2] = -1;
    return;
  }
  const unsigned int lin = (unsigned int)(key & 0xffffffffu);
  const int n = a.n;
  a.minE[out] = key_to_float((unsigned int)(key >> 32));
  a.idx[out * 3 + 0] = lin / (n * n);
  a.idx[out * 3 + 1] = (lin / n) % n;
  a.idx[out * 3 + 2] = lin % n;
}

__global__ void k_finalize_server(WaveArgs a, float* ebase, int* ibase) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= a.nrot) return;
  const RotDesc rd = a.rots[r];
  const RotRec* rec = a.rec + r;
  const unsigned long long key = a.keys[r];
  int* idx = ibase + rd.pad0;
  if (rec->err) {
    // a rotation that could not be searched: NaN energy and index -2 (box overflow) or -3
    // (FP16 range), which the server reads back to fail exactly the requests that hold one
    if (rec->err == 1) atomicAdd(a.err_count, 1);
    else atomicOr(a.range_err, 1);
    ebase[rd.out] = __int_as_float(0x7fc00000);
    idx[0] = idx[1] = idx[2] = rec->err == 1 ? -2 : -3;
    return;
  }
  if (!rec->valid || key == ~0ull) {
    ebase[rd.out] = INFINITY;
    idx[0] = idx[1] = idx[2] = -1;
    return;
  }
  const unsigned int lin = (unsigned int)(key & 0xffffffffu);
  const int n = a.n;
  ebase[rd.out] = key_to_float((unsigned int)(key >> 32));
  idx[0] = lin / (n * n);
  idx[1] = (lin / n) % n;
  idx[2] = lin % n;
}

// ---------------------------------------------------------------------------------------
// receptor spectra: dense (y,z) forward of every plane, then x forward per column tile
template <int N>
__global__ void __launch_bounds__(256) k_receptor_yz(const float* grids, float2* out,
                                                      const float2* twg) {
  constexpr int NZH = N / 2 + 1;
  constexpr int NCOL = N * NZH;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* tw = reinterpret_cast<float2*>(smem_raw);
  float2* O = tw + N;
  float2* P = O + N * NZH;
  const int x = blockIdx.x, k = blockIdx.y;
  const int tid = threadIdx.x, nthr = blockDim.x;
  for (int i = tid; i < N; i += nthr) tw[i] = twg[i];
  const float* g = grids + ((size_t)k * N + x) * N * N;
  for (int i = tid; i < N * N; i += nthr) {
    const int y = i / N, z = i - y * N;
    reinterpret_cast<float*>(P)[((y >> 1) * (N + 1) + z) * 2 + (y & 1)] = g[i];
  }
  __syncthreads();
  plane_forward<N>(P, O, N / 2, tw);
  float2* dst = out + ((size_t)k * N + x) * NCOL;
  for (int i = tid; i < NCOL; i += nthr) dst[i] = O[i];
}

template <int N>
__global__ void __launch_bounds__(256) k_receptor_x(const float2* in, float2* phat, int K,
                                                     int ct, const float2* twg) {
  constexpr int NZH = N / 2 + 1;
  constexpr int NCOL = N * NZH;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  float2* tw = reinterpret_cast<float2*>(smem_raw);
  float2* Wb = tw + N;
  const int c0 = blockIdx.x * ct;
  const int k = blockIdx.y;
  const int tid = threadIdx.x, nthr = blockDim.x;
  for (int i = tid; i < N; i += nthr) tw[i] = twg[i];
  for (int i = tid; i < N * ct; i += nthr) {
    const int c = i % ct, x = i / ct;
    Wb[i] = (c0 + c < NCOL) ? in[((size_t)k * N + x) * NCOL + c0 + c] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  fft_lines<N, false>(Wb, ct, 1, ct, tw, tid, nthr);
  for (int i = tid; i < N * ct; i += nthr) {
    const int c = i % ct, xp = i / ct;
    if (c0 + c < NCOL) phat[((size_t)xp * K + k) * NCOL + c0 + c] = Wb[i];
  }
}

template <int N>
constexpr size_t plane_smem() {
  return sizeof(float2) * (N + N * (N / 2 + 1) + (N / 2) * (N + 1));
}

template <int N>
size_t direct_smem(int cap) {
  return sizeof(float2) * (N + (size_t)cap * (N + N / 2 + 1)) + sizeof(int4) * cap +
         sizeof(int) * cap + (sizeof(int2) + sizeof(float2)) * cap;
}

template <int N>
cudaError_t launch_spread_yz_t(const WaveArgs& a, cudaStream_t s) {
  const int cap = a.atom_cap > 0 ? a.atom_cap : a.max_atoms;
  if (a.kyof && cap <= kDirectMaxAtoms) {
    const size_t sm = direct_smem<N>(cap);
    if (a.lop) {
      cudaError_t e = cudaFuncSetAttribute(k_spread_yz_direct<N, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
      if (e != cudaSuccess) return e;
      WaveArgs b = a;
      b.plane_rot_major = (a.lop_tiled && plane_rot_major_host()) ? 1 : 0;
      const dim3 grid = b.plane_rot_major ? dim3(a.nrot, a.K) : dim3(a.K, a.nrot);
      k_spread_yz_direct<N, true><<<grid, 256, sm, s>>>(b, a.kyof, cap);
      return cudaGetLastError();
    }
    cudaError_t e = cudaFuncSetAttribute(k_spread_yz_direct<N, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k_spread_yz_direct<N, false><<<dim3(a.K, a.nrot), 256, sm, s>>>(a, a.kyof, cap);
    return cudaGetLastError();
  }
  if (a.lop) return cudaErrorInvalidValue;  // the FFT plane path writes A only
  const size_t sm = plane_smem<N>();
  cudaError_t e = cudaFuncSetAttribute(k_spread_yz<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  dim3 grid(a.Lb, a.K, a.nrot);
  k_spread_yz<N><<<grid, 256, sm, s>>>(a);
  return cudaGetLastError();
}

template <int N>
cudaError_t launch_yz_inv_t(const WaveArgs& a, cudaStream_t s) {
  // octet kernel at n >= 96 (measured 2.1x faster than block stages at 128^3, 1.05x at 96^3);
  // block stages at n <= 64 (the packed rows alias the plane there, 8 CTAs per SM: 1.6x faster
  // than the octets at 64^3); yz_block_stages: 1 forces block stages, 2 forces octets
  const bool octet = a.yz_block_stages == 2 || (a.yz_block_stages == 0 && N >= 96);
  // the B layout as a template argument (kBAny reads it at run time)
  const int bl = b_layout(a);
#define CDK_YZ_PICK(KERN)                                                                     \
  (bl == kBPlain    ? (a.keys2 ? KERN<N, true, kBPlain> : KERN<N, false, kBPlain>)           \
   : bl == kBPairs2 ? (a.keys2 ? KERN<N, true, kBPairs2> : KERN<N, false, kBPairs2>)         \
   : bl == kBSingle4 ? (a.keys2 ? KERN<N, true, kBSingle4> : KERN<N, false, kBSingle4>)      \
                     : (a.keys2 ? KERN<N, true, kBAny> : KERN<N, false, kBAny>))
  if (octet) {
    constexpr size_t sm = octet_smem<N>();
    auto kern = CDK_YZ_PICK(k_yz_octet);
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    dim3 grid(N, a.nrot);
    kern<<<grid, 32 * kOctWarps, sm, s>>>(a);
    return cudaGetLastError();
  }
  // twiddles + one plane (n <= 64: the packed rows alias it) [+ the packed rows]
  const size_t sm = sizeof(float2) * (N + N * (N / 2 + 1) + (N <= 64 ? 0 : (N / 2) * (N + 1)));
  auto kern = CDK_YZ_PICK(k_yz_inv_argmin);
#undef CDK_YZ_PICK
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  dim3 grid(N, a.nrot);
  kern<<<grid, 256, sm, s>>>(a);
  return cudaGetLastError();
}

template <int N>
cudaError_t launch_xpass_t(const WaveArgs& a, cudaStream_t s) {
  constexpr int NCOL = N * (N / 2 + 1);
  static_assert(FFTPlan<N>::NS == 2, "the x pass runs two-stage radix plans");
  // fixed 16-column tiles; chunks of up to 32 rotations per CTA keep the receptor tile
  // reused while giving the scheduler many CTAs per SM slot
  constexpr int CT = 16;
  if (a.col_tile != CT && a.col_tile != 8) return cudaErrorInvalidValue;
  if (N > 64 && a.col_tile != 8) return cudaErrorInvalidValue;
  const size_t sm = xpass2_smem_bytes(N, a.K, a.col_tile);
  const int per = a.chunk > 0 ? a.chunk : 32;
  const int chunks = (a.nrot + per - 1) / per;
  if (N <= 64 && a.col_tile == CT) {
    cudaError_t e = cudaFuncSetAttribute(k_xpass2<N, (N <= 64 ? 16 : 8)>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k_xpass2<N, (N <= 64 ? 16 : 8)><<<dim3(NCOL / (N <= 64 ? 16 : 8), chunks), 256, sm, s>>>(a, per);
  } else {
    cudaError_t e = cudaFuncSetAttribute(k_xpass2<N, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    if (e != cudaSuccess) return e;
    k_xpass2<N, 8><<<dim3(NCOL / 8, chunks), 256, sm, s>>>(a, per);
  }
  return cudaGetLastError();
}

template <int N>
cudaError_t launch_receptor_t(int K, const float* grids, float2* scratch, float2* phat,
                              const float2* tw, int ct, cudaStream_t s) {
  const size_t sm = plane_smem<N>();
  cudaError_t e = cudaFuncSetAttribute(k_receptor_yz<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  if (e != cudaSuccess) return e;
  k_receptor_yz<N><<<dim3(N, K), 256, sm, s>>>(grids, scratch, tw);
  if ((e = cudaGetLastError()) != cudaSuccess) return e;
  constexpr int NCOL = N * (N / 2 + 1);
  const size_t sm2 = sizeof(float2) * (N + (size_t)N * ct);
  e = cudaFuncSetAttribute(k_receptor_x<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm2);
  if (e != cudaSuccess) return e;
  k_receptor_x<N><<<dim3((NCOL + ct - 1) / ct, K), 256, sm2, s>>>(scratch, phat, K, ct, tw);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------------------
// Rotation grouping for the tensor-core x pass. A tile of 128 rotations loads and multiplies,
// per channel, the union of the 8-plane chunks its rotations touch. Nearly every rotation
// starts at chunk 0; what varies is whether a channel's atoms reach the box's last chunk. A
// stable counting sort of the rotation list on one bit per channel (folded into kGroupBits)
// puts rotations with the same pattern side by side, so tiles skip more chunks. Results do
// not depend on the order: a chunk a rotation does not touch adds exact zeros to its sums, and
// every output goes to its rotation's RotDesc::out.
constexpr int kGroupBits = 10;
constexpr int kGroupBuckets = 1 << kGroupBits;
constexpr int kGroupSeg = 1024;  // rotations per histogram / scatter CTA

// warp per rotation: the rotated x coordinates and their minimum exactly as k_prep computes
// them, then the channels whose atoms reach chunk jc - 1
__global__ void __launch_bounds__(128) k_group_key(const RotDesc* __restrict__ rots,
                                                   const ConfDesc* __restrict__ confs,
                                                   const float* __restrict__ coords,
                                                   const AtomParam* __restrict__ params, long nrot,
                                                   int max_atoms, int K, float h, int jc,
                                                   unsigned short* __restrict__ key) {
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const long r = (long)blockIdx.x * 4 + warp;
  if (r >= nrot) return;
  const RotDesc rd = rots[r];
  const ConfDesc cd = confs[rd.conf];
  const int nA = min(cd.n_atoms, max_atoms);
  const float* xyz = coords + (size_t)cd.coord_off * 3;
  const AtomParam* prm = params + cd.param_off;
  float mn = INFINITY;
  for (int i = lane; i < nA; i += 32) {
    float p[3];
    rotate_rn(rd.q, xyz[i * 3 + 0], xyz[i * 3 + 1], xyz[i * 3 + 2], p);
    mn = fminf(mn, p[0]);
  }
  for (int o = 16; o > 0; o >>= 1) mn = fminf(mn, __shfl_xor_sync(0xffffffffu, mn, o));
  const int elec = K - 1;
  unsigned int bits = 0;
  for (int i = lane; i < nA; i += 32) {
    float p[3];
    rotate_rn(rd.q, xyz[i * 3 + 0], xyz[i * 3 + 1], xyz[i * 3 + 2], p);
    if (min((cell_of(p[0], mn, h) + 1) >> 3, jc - 1) == jc - 1) {
      const int sl = prm[i].slot;
      if (sl >= 0 && sl < elec) bits |= 1u << (sl % kGroupBits);
      bits |= 1u << (elec % kGroupBits);
    }
  }
  bits = __reduce_or_sync(0xffffffffu, bits);
  if (lane == 0) key[r] = (unsigned short)bits;
}

// per segment of kGroupSeg rotations, the count of each key: counts[key * nseg + segment]
__global__ void __launch_bounds__(kGroupSeg) k_group_hist(const unsigned short* __restrict__ key,
                                                          long nrot, int nseg, int* __restrict__ counts) {
  __shared__ int hcount[kGroupBuckets];
  for (int b = threadIdx.x; b < kGroupBuckets; b += blockDim.x) hcount[b] = 0;
  __syncthreads();
  const long r = (long)blockIdx.x * kGroupSeg + threadIdx.x;
  if (r < nrot) atomicAdd(&hcount[key[r]], 1);
  __syncthreads();
  for (int b = threadIdx.x; b < kGroupBuckets; b += blockDim.x)
    counts[(size_t)b * nseg + blockIdx.x] = hcount[b];
}

// exclusive scan of counts in place (key-major, so a key's segments follow one another)
__global__ void __launch_bounds__(1024) k_group_scan(int* __restrict__ counts, long total) {
  __shared__ long part[1024];
  const int tid = threadIdx.x, T = blockDim.x;
  const long per = (total + T - 1) / T;
  const long lo = min(total, (long)tid * per), hi = min(total, lo + per);
  long sum = 0;
  for (long i = lo; i < hi; ++i) sum += counts[i];
  part[tid] = sum;
  __syncthreads();
  for (int off = 1; off < T; off <<= 1) {
    const long v = tid >= off ? part[tid - off] : 0;
    __syncthreads();
    part[tid] += v;
    __syncthreads();
  }
  long run = part[tid] - sum;
  for (long i = lo; i < hi; ++i) {
    const int c = counts[i];
    counts[i] = (int)run;
    run += c;
  }
}

// stable scatter: the warps of a segment place their rotations in warp order, lanes with the
// same key by lane order
__global__ void __launch_bounds__(kGroupSeg) k_group_scatter(const RotDesc* __restrict__ rots,
                                                             const unsigned short* __restrict__ key,
                                                             long nrot, int nseg,
                                                             const int* __restrict__ counts,
                                                             RotDesc* __restrict__ out) {
  __shared__ int base[kGroupBuckets];
  for (int b = threadIdx.x; b < kGroupBuckets; b += blockDim.x) base[b] = counts[(size_t)b * nseg + blockIdx.x];
  const long r = (long)blockIdx.x * kGroupSeg + threadIdx.x;
  const bool live = r < nrot;
  const unsigned int kk = live ? key[r] : 0xffffffffu;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const unsigned int same = __match_any_sync(0xffffffffu, kk);
  const int rank = __popc(same & ((1u << lane) - 1));
  __syncthreads();
  for (int w = 0; w < (int)(blockDim.x >> 5); ++w) {
    if (warp == w) {
      const int b0 = live ? base[kk] : 0;
      __syncwarp();
      if (live) {
        out[b0 + rank] = rots[r];
        if (rank == 0) base[kk] = b0 + __popc(same);
      }
    }
    __syncthreads();
  }
}

}  // namespace

int fft_position(int n, int k) {
  switch (n) {
    case 32: return fft_pos<32>(k);
    case 64: return fft_pos<64>(k);
    case 96: return fft_pos<96>(k);
    case 128: return fft_pos<128>(k);
    default: return k;
  }
}

size_t xpass2_smem_bytes(int n, int K, int col_tile) {
  return sizeof(float2) * n + sizeof(int) * 2 * KMAX + sizeof(short) * 4 * KMAX +
         sizeof(float2) * (size_t)n * col_tile * (K + 2 + 1);
}

int pick_col_tile(int n, int K) {
  // 16 columns when the buffers stay within ~110 KB of shared memory (two CTAs per SM), else 8
  if ((n == 32 || n == 64) && xpass2_smem_bytes(n, K, 16) <= 110 * 1024) return 16;
  return 8;
}

#define CDK_DISPATCH_N(n, fn, ...)                 \
  switch (n) {                                     \
    case 32: return fn<32>(__VA_ARGS__);           \
    case 64: return fn<64>(__VA_ARGS__);           \
    case 96: return fn<96>(__VA_ARGS__);           \
    case 128: return fn<128>(__VA_ARGS__);         \
    default: return cudaErrorInvalidValue;         \
  }

size_t group_rotations_bytes(long nrot) {
  const long nseg = (nrot + kGroupSeg - 1) / kGroupSeg;
  return ((size_t)nrot * sizeof(RotDesc) + 255) / 256 * 256 + ((size_t)nrot * 2 + 255) / 256 * 256 +
         (size_t)kGroupBuckets * nseg * sizeof(int);
}

cudaError_t launch_group_rotations(const RotDesc* rots, const ConfDesc* confs, const float* coords,
                                   const AtomParam* params, long nrot, int max_atoms, int K, float h,
                                   int jc, void* scratch, RotDesc** sorted, cudaStream_t s) {
  if (nrot <= 0 || jc < 1 || K > KMAX) return cudaErrorInvalidValue;
  const long nseg = (nrot + kGroupSeg - 1) / kGroupSeg;
  char* p = static_cast<char*>(scratch);
  RotDesc* out = reinterpret_cast<RotDesc*>(p);
  p += ((size_t)nrot * sizeof(RotDesc) + 255) / 256 * 256;
  unsigned short* key = reinterpret_cast<unsigned short*>(p);
  p += ((size_t)nrot * 2 + 255) / 256 * 256;
  int* counts = reinterpret_cast<int*>(p);
  k_group_key<<<(unsigned)((nrot + 3) / 4), 128, 0, s>>>(rots, confs, coords, params, nrot, max_atoms, K, h, jc, key);
  k_group_hist<<<(unsigned)nseg, kGroupSeg, 0, s>>>(key, nrot, (int)nseg, counts);
  k_group_scan<<<1, 1024, 0, s>>>(counts, (long)kGroupBuckets * nseg);
  k_group_scatter<<<(unsigned)nseg, kGroupSeg, 0, s>>>(rots, key, nrot, (int)nseg, counts, out);
  *sorted = out;
  return cudaGetLastError();
}

cudaError_t launch_prep(const WaveArgs& a, cudaStream_t s) {
  k_prep<<<(a.nrot + 3) / 4, 128, 0, s>>>(a);
  return cudaGetLastError();
}
cudaError_t launch_spread_yz(const WaveArgs& a, cudaStream_t s) {
  if (a.lop_tiled) {
    // the tiled rows zero-fill by the tiles' stage plans: k_tile_plan first
    if (!a.lop || !direct_planes(a) || (reinterpret_cast<uintptr_t>(a.lop) & 127)) return cudaErrorInvalidValue;
    cudaError_t e = launch_tile_plan(a, (a.Lb + 7) / 8, s);
    if (e != cudaSuccess) return e;
  }
  CDK_DISPATCH_N(a.n, launch_spread_yz_t, a, s);
}
bool direct_planes(const WaveArgs& a) {
  const int cap = a.atom_cap > 0 ? a.atom_cap : a.max_atoms;
  return a.kyof != nullptr && cap <= kDirectMaxAtoms;
}
cudaError_t launch_xpass(const WaveArgs& a, cudaStream_t s) {
  CDK_DISPATCH_N(a.n, launch_xpass_t, a, s);
}
cudaError_t launch_yz_inv_argmin(const WaveArgs& a, cudaStream_t s) {
  CDK_DISPATCH_N(a.n, launch_yz_inv_t, a, s);
}
cudaError_t launch_topk_rescore(const WaveArgs& a, const float* grids, int k, TopPose* out, cudaStream_t s) {
  if (!grids || !out || k < 1 || k > kTopMax) return cudaErrorInvalidValue;
  k_topk_rescore<<<1, 256, 0, s>>>(a, grids, k, out);
  return cudaGetLastError();
}
cudaError_t launch_tiebreak(const WaveArgs& a, const float* grids, float tol, cudaStream_t s) {
  if (!a.keys2 || !grids) return cudaErrorInvalidValue;
  k_tiebreak<<<(a.nrot + 3) / 4, 128, 0, s>>>(a, grids, tol);
  return cudaGetLastError();
}
cudaError_t launch_finalize(const WaveArgs& a, cudaStream_t s) {
  k_finalize<<<(a.nrot + 255) / 256, 256, 0, s>>>(a);
  return cudaGetLastError();
}
cudaError_t launch_finalize_server(const WaveArgs& a, float* ebase, int* ibase, cudaStream_t s) {
  k_finalize_server<<<(a.nrot + 255) / 256, 256, 0, s>>>(a, ebase, ibase);
  return cudaGetLastError();
}
cudaError_t launch_receptor_fft(int n, int K, const float* grids, float2* scratch,
                                float2* phat, const float2* tw, int ct, cudaStream_t s) {
  CDK_DISPATCH_N(n, launch_receptor_t, K, grids, scratch, phat, tw, ct, s);
}

}  // namespace cdk
