// compat_kernels.cu -- kernels with the reference's own interfaces and an FP64 re-scorer.
//
//  k_fill_dense   FillLigandGrid (src/FillLigandGrid.cpp:7-120) on the GPU, bit-exact: one
//                 thread owns one (rotation, grid) and adds the atoms in the reference's
//                 order with its mixed float/double arithmetic and no contraction.
//  k_conj_mult    ConjMult (src/kernel.cu:5-14) with a bounds check.
//  k_sum_grids    SumGrids (src/kernel.cu:16-30) with a bounds check.
//  k_rescore_fp64 direct trilinear grid-energy sum of given poses in double.
//  k_build_tables per-search device tables from plain arrays.
//  k_diameter     largest atom-atom distance per search (plans the ligand box).
#include <cuda_runtime.h>

#include "cdk_internal.h"

namespace cdk {

namespace {

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

// one atom into one grid, FillLigandGrid arithmetic, sequential (the owning thread only)
__device__ void spread_exact(float x, float y, float z, const float* mn, float h, double s,
                             int Y, int Z, float* grid) {
  const int xi = (int)__ddiv_rn(__dsub_rn((double)x, (double)mn[0]), (double)h);
  const int yi = (int)__ddiv_rn(__dsub_rn((double)y, (double)mn[1]), (double)h);
  const int zi = (int)__ddiv_rn(__dsub_rn((double)z, (double)mn[2]), (double)h);
  const double xr = __ddiv_rn(__dsub_rn(__dsub_rn((double)x, (double)mn[0]), (double)__fmul_rn((float)xi, h)), (double)h);
  const double yr = __ddiv_rn(__dsub_rn(__dsub_rn((double)y, (double)mn[1]), (double)__fmul_rn((float)yi, h)), (double)h);
  const double zr = __ddiv_rn(__dsub_rn(__dsub_rn((double)z, (double)mn[2]), (double)__fmul_rn((float)zi, h)), (double)h);
  const double wx[2] = {__dsub_rn(1.0, xr), xr}, wy[2] = {__dsub_rn(1.0, yr), yr},
               wz[2] = {__dsub_rn(1.0, zr), zr};
#pragma unroll
  for (int c = 0; c < 8; ++c) {
    const int dx = (c >> 2) & 1, dy = (c >> 1) & 1, dz = c & 1;
    const size_t idx = ((size_t)(xi + dx) * Y + (yi + dy)) * Z + (zi + dz);
    const double w = __dmul_rn(__dmul_rn(__dmul_rn(s, wx[dx]), wy[dy]), wz[dz]);
    grid[idx] = (float)__dadd_rn((double)grid[idx], w);
  }
}

__global__ void k_fill_dense(int nQ, int nAtom, const float* coors, const float* mincoors,
                             const AtomParam* prm, int nVdwUsed, int X, int Y, int Z, float h,
                             float* out) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int K = nVdwUsed + 1;
  if (t >= nQ * K) return;
  const int q = t / K, j = t - q * K;
  const size_t N = (size_t)X * Y * Z;
  float* grid = out + ((size_t)q * K + j) * N;
  const float* c = coors + (size_t)q * nAtom * 3;
  const float* mn = mincoors + q * 3;
  for (int m = 0; m < nAtom; ++m) {
    const AtomParam p = prm[m];
    if (j < nVdwUsed) {
      if (p.slot != j) continue;
      spread_exact(c[m * 3], c[m * 3 + 1], c[m * 3 + 2], mn, h, (double)p.w_vdw, Y, Z, grid);
    } else {
      spread_exact(c[m * 3], c[m * 3 + 1], c[m * 3 + 2], mn, h, (double)p.charge, Y, Z, grid);
    }
  }
}

__global__ void k_conj_mult(const float2* pot, float2* lig, int odist, int K, long total) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const long ip = i % ((long)odist * K);
  const float x = lig[i].x, y = lig[i].y;
  const float2 p = pot[ip];
  lig[i] = make_float2(x * p.x + y * p.y, x * p.y - y * p.x);
}

__global__ void k_sum_grids(const float2* lig, float2* sum, int K, int odist, int idist,
                            long total) {
  const long i = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= total) return;
  const long q = i / odist, f = i - q * odist;
  float sx = 0.f, sy = 0.f;
  for (int k = 0; k < K; ++k) {
    const float2 v = lig[(q * K + k) * odist + f];
    sx += v.x;
    sy += v.y;
  }
  const float d = sqrtf((float)idist);
  sum[i] = make_float2(sx / d, sy / d);
}

// one CTA per pose: rotate, min corner, then sum over atoms x 8 corners x {vdW, elec} in double
__global__ void __launch_bounds__(128) k_rescore_fp64(int n, int K, float h, const float* grids,
                                                      const float* coords, const AtomParam* prm_all,
                                                      const ConfDesc* confs, const RotDesc* rots,
                                                      const int* tidx, int npose, double* energy) {
  const int pose = blockIdx.x;
  if (pose >= npose) return;
  __shared__ float s_mn[3][4];
  __shared__ double s_e[4];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const RotDesc rd = rots[pose];
  const ConfDesc cd = confs[rd.conf];
  const float* xyz = coords + (size_t)cd.coord_off * 3;
  const AtomParam* prm = prm_all + cd.param_off;
  const int nA = cd.n_atoms;
  float mn[3] = {INFINITY, INFINITY, INFINITY};
  for (int i = tid; i < nA; i += blockDim.x) {
    float p[3];
    rotate_rn(rd.q, xyz[i * 3], xyz[i * 3 + 1], xyz[i * 3 + 2], p);
    for (int d = 0; d < 3; ++d) mn[d] = fminf(mn[d], p[d]);
  }
  for (int d = 0; d < 3; ++d) {
    for (int o = 16; o > 0; o >>= 1) mn[d] = fminf(mn[d], __shfl_xor_sync(0xffffffffu, mn[d], o));
    if (lane == 0) s_mn[d][warp] = mn[d];
  }
  __syncthreads();
  for (int d = 0; d < 3; ++d) {
    float v = s_mn[d][0];
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) v = fminf(v, s_mn[d][w]);
    mn[d] = v;
  }
  const size_t N = (size_t)n * n * n;
  const int ti = tidx[pose * 3], tj = tidx[pose * 3 + 1], tk = tidx[pose * 3 + 2];
  double e = 0.0;
  for (int i = tid; i < nA; i += blockDim.x) {
    float p[3];
    rotate_rn(rd.q, xyz[i * 3], xyz[i * 3 + 1], xyz[i * 3 + 2], p);
    int ci[3];
    double rr[3];
    for (int d = 0; d < 3; ++d) {
      ci[d] = (int)__ddiv_rn(__dsub_rn((double)p[d], (double)mn[d]), (double)h);
      rr[d] = __ddiv_rn(__dsub_rn(__dsub_rn((double)p[d], (double)mn[d]), (double)__fmul_rn((float)ci[d], h)), (double)h);
    }
    const AtomParam ap = prm[i];
    for (int c = 0; c < 8; ++c) {
      const int dx = (c >> 2) & 1, dy = (c >> 1) & 1, dz = c & 1;
      const int gx = ci[0] + dx + ti, gy = ci[1] + dy + tj, gz = ci[2] + dz + tk;
      if (gx >= n || gy >= n || gz >= n) continue;
      const double w = (dx ? rr[0] : 1.0 - rr[0]) * (dy ? rr[1] : 1.0 - rr[1]) * (dz ? rr[2] : 1.0 - rr[2]);
      const size_t g = ((size_t)gx * n + gy) * n + gz;
      if (ap.slot >= 0 && ap.slot < K - 1)
        e += (double)ap.w_vdw * w * (double)grids[(size_t)ap.slot * N + g];
      e += (double)ap.charge * w * (double)grids[(size_t)(K - 1) * N + g];
    }
  }
  for (int o = 16; o > 0; o >>= 1) e += __shfl_xor_sync(0xffffffffu, e, o);
  if (lane == 0) s_e[warp] = e;
  __syncthreads();
  if (tid == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += s_e[w];
    energy[pose] = t;
  }
}

}  // namespace

cudaError_t launch_fill_dense(int nQ, int nAtom, const float* coors, const float* mincoors,
                              const AtomParam* params, int nVdwUsed, int X, int Y, int Z,
                              float spacing, float* out, cudaStream_t s) {
  const int total = nQ * (nVdwUsed + 1);
  k_fill_dense<<<(total + 127) / 128, 128, 0, s>>>(nQ, nAtom, coors, mincoors, params, nVdwUsed,
                                                  X, Y, Z, spacing, out);
  return cudaGetLastError();
}

cudaError_t launch_conj_mult(const float2* pot, float2* lig, int odist, int K, int Q,
                             cudaStream_t s) {
  const long total = (long)Q * K * odist;
  k_conj_mult<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(pot, lig, odist, K, total);
  return cudaGetLastError();
}

cudaError_t launch_sum_grids(const float2* lig, float2* sum, int K, int odist, int idist,
                             int Q, cudaStream_t s) {
  const long total = (long)Q * odist;
  k_sum_grids<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(lig, sum, K, odist, idist, total);
  return cudaGetLastError();
}

cudaError_t launch_rescore_fp64(int n, int K, float spacing, const float* grids,
                                const float* coords, const AtomParam* params,
                                const ConfDesc* confs, const RotDesc* rots, const int* tidx,
                                int npose, double* energy, cudaStream_t s) {
  if (npose <= 0) return cudaSuccess;
  k_rescore_fp64<<<npose, 128, 0, s>>>(n, K, spacing, grids, coords, params, confs, rots, tidx,
                                       npose, energy);
  return cudaGetLastError();
}

}  // namespace cdk
