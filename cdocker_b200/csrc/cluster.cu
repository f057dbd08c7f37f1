// cluster.cu -- diverse-conformer selection: greedy leader clustering by superposition RMSD.
//
// The reference picks conformer centres in GeneDiverseConformations
// (src/GeneDiverseConformations.cpp:84-111): conformers are ordered by energy with sort_index
// (include/GeneDiverseConformations.h:9-20, std::sort, not stable), the lowest is the first
// centre, and each following conformer becomes a new centre when its RMSD to every centre found
// so far, after optimal superposition (OpenBabel's OBAlign), exceeds the cut-off (1.5 A). The
// loop stops as soon as the number of centres equals maxNumOfConformations, a test made after
// each candidate from the second on (so a limit of 1 stops only if the second conformer is not a
// centre, and a limit <= 0 never stops).
//
// The outcome depends only on the predicate close(i, j) = rmsd(i, j) <= cutoff for j before i in
// energy order, so the GPU evaluates all of it at once and keeps the sequential part (the scan
// over candidates) to one bit-matrix pass:
//   k_center   per conformer (in energy order): centroid, centred coordinates of the selected
//              atoms, laid out [atom][xyz][conformer] so tiles stage with coalesced loads, and
//              G = sum |x|^2.
//   k_pairs    8 candidates x 32 earlier conformers per CTA (warp = candidate, lane = other
//              conformer); atoms streamed through shared memory in chunks of 32; per pair the 3x3
//              correlation S = sum a b^T, Horn's 4x4 quaternion key matrix, its largest
//              eigenvalue by Newton's method on the characteristic polynomial (Theobald's QCP
//              idea; the coefficients come from traces of N^2 and N^3 and det N), and
//              rmsd = sqrt(max(0, (Ga + Gb - 2 lambda) / n)). Cluster mode packs close(i, j) into
//              one 32-bit word per warp with a ballot; matrix mode writes the RMSD itself.
//   k_greedy   one CTA scans the candidates in order; thread t owns word t of the centre mask,
//              so a candidate costs one row read and one __syncthreads_or.
// All double arithmetic uses explicit round-to-nearest intrinsics (no contraction), sqrt and
// division are IEEE, and every sum runs in atom order: the RMSDs are bit-identical to a host
// double-precision evaluation of the same recipe without fused multiply-adds.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/cdock_b200.h"
#include "cdk_internal.h"

namespace cdk {
namespace {

constexpr int CL_REF = 8;     // candidates per CTA (one per warp)
constexpr int CL_TGT = 32;    // other conformers per CTA (one per lane)
constexpr int CL_CHUNK = 32;  // atoms staged per step
constexpr int CL_MAX_CONF = 32768;      // cluster mode: the centre mask fits one CTA's words
constexpr int CL_MAX_CONF_MATRIX = 16384;

__device__ __forceinline__ double dm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double da(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double ds(double a, double b) { return __dsub_rn(a, b); }

// centred coordinates of conformer order[c] (or c) -> X[(a*3 + d) * ld + c], G[c]
__global__ void k_center(int nConf, int nAtom, const double* __restrict__ coor,
                         const int* __restrict__ sel, int nSel, const int* __restrict__ order,
                         int ld, double* __restrict__ X, double* __restrict__ G) {
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  if (c >= nConf) return;
  const double* p = coor + (size_t)(order ? order[c] : c) * nAtom * 3;
  double s[3] = {0.0, 0.0, 0.0};
  for (int i = 0; i < nSel; ++i)
    for (int d = 0; d < 3; ++d) s[d] = da(s[d], p[sel[i] * 3 + d]);
  double m[3];
  for (int d = 0; d < 3; ++d) m[d] = __ddiv_rn(s[d], (double)nSel);
  double g = 0.0;
  for (int i = 0; i < nSel; ++i) {
    double v[3];
    for (int d = 0; d < 3; ++d) {
      v[d] = ds(p[sel[i] * 3 + d], m[d]);
      X[((size_t)i * 3 + d) * ld + c] = v[d];
    }
    g = da(g, da(da(dm(v[0], v[0]), dm(v[1], v[1])), dm(v[2], v[2])));
  }
  G[c] = g;
}

// minimum RMSD over rotations from the correlation S[p*3+q] = sum a_p b_q of centred sets
__device__ double rmsd_from_corr(const double* S, double Ga, double Gb, int n) {
  const double Sxx = S[0], Sxy = S[1], Sxz = S[2], Syx = S[3], Syy = S[4], Syz = S[5],
               Szx = S[6], Szy = S[7], Szz = S[8];
  double N[4][4];
  N[0][0] = da(da(Sxx, Syy), Szz);
  N[0][1] = ds(Syz, Szy);
  N[0][2] = ds(Szx, Sxz);
  N[0][3] = ds(Sxy, Syx);
  N[1][1] = ds(ds(Sxx, Syy), Szz);
  N[1][2] = da(Sxy, Syx);
  N[1][3] = da(Szx, Sxz);
  N[2][2] = ds(ds(Syy, Sxx), Szz);
  N[2][3] = da(Syz, Szy);
  N[3][3] = ds(ds(Szz, Sxx), Syy);
  N[1][0] = N[0][1];
  N[2][0] = N[0][2];
  N[3][0] = N[0][3];
  N[2][1] = N[1][2];
  N[3][1] = N[1][3];
  N[3][2] = N[2][3];
  // char. polynomial of the traceless N: l^4 + c2 l^2 + c1 l + c0,
  // c2 = -tr(N^2)/2, c1 = -tr(N^3)/3, c0 = det N (Newton's identities)
  double p2 = 0.0;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) p2 = da(p2, dm(N[i][j], N[i][j]));
  double p3 = 0.0;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      const double n2 = da(da(da(dm(N[i][0], N[0][j]), dm(N[i][1], N[1][j])), dm(N[i][2], N[2][j])),
                           dm(N[i][3], N[3][j]));
      p3 = da(p3, dm(n2, N[j][i]));
    }
  // det by 2x2 minors of rows (0,1) and (2,3)
  auto mA = [&](int j, int k) { return ds(dm(N[0][j], N[1][k]), dm(N[0][k], N[1][j])); };
  auto mB = [&](int j, int k) { return ds(dm(N[2][j], N[3][k]), dm(N[2][k], N[3][j])); };
  double det = ds(dm(mA(0, 1), mB(2, 3)), dm(mA(0, 2), mB(1, 3)));
  det = da(det, dm(mA(0, 3), mB(1, 2)));
  det = da(det, dm(mA(1, 2), mB(0, 3)));
  det = ds(det, dm(mA(1, 3), mB(0, 2)));
  det = da(det, dm(mA(2, 3), mB(0, 1)));
  const double c2 = -dm(p2, 0.5);
  const double c1 = -__ddiv_rn(p3, 3.0);
  const double c0 = det;
  // Newton from (Ga + Gb) / 2, an upper bound of the largest root: monotone convergence
  double l = dm(da(Ga, Gb), 0.5);
  for (int it = 0; it < 50; ++it) {
    const double l2 = dm(l, l);
    const double P = da(dm(da(dm(da(l2, c2), l), c1), l), c0);
    const double dP = da(dm(da(dm(4.0, l2), dm(2.0, c2)), l), c1);
    if (dP == 0.0) break;
    const double ln = ds(l, __ddiv_rn(P, dP));
    if (fabs(ds(ln, l)) <= dm(1e-11, fabs(ln))) {
      l = ln;
      break;
    }
    l = ln;
  }
  double e = __ddiv_rn(ds(da(Ga, Gb), dm(2.0, l)), (double)n);
  if (!(e > 0.0)) e = 0.0;
  return __dsqrt_rn(e);
}

// rmsd(candidate i = ref, conformer j = target) for the tile i in [8 by, +8), j in [32 bx, +32).
// bits != nullptr: cluster mode (only j < i, packed); else out[i * nConf + j]
__global__ void __launch_bounds__(256) k_pairs(int nConf, int nSel, int ld,
                                               const double* __restrict__ X,
                                               const double* __restrict__ G, double cutoff,
                                               uint32_t* __restrict__ bits, int W,
                                               double* __restrict__ out) {
  __shared__ double sR[CL_CHUNK][3][CL_REF];
  __shared__ double sT[CL_CHUNK][3][CL_TGT];
  const int i0 = blockIdx.y * CL_REF, j0 = blockIdx.x * CL_TGT;
  if (bits && j0 > i0 + CL_REF - 1) return;  // no j < i in this tile (uniform over the CTA)
  const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
  const int i = i0 + w, j = j0 + lane;
  double S[9];
#pragma unroll
  for (int t = 0; t < 9; ++t) S[t] = 0.0;
  for (int a0 = 0; a0 < nSel; a0 += CL_CHUNK) {
    const int na = min(CL_CHUNK, nSel - a0);
    __syncthreads();
    for (int e = tid; e < na * 3 * CL_REF; e += blockDim.x) {
      const int r = e % CL_REF, ad = e / CL_REF;
      sR[ad / 3][ad % 3][r] = (i0 + r < nConf) ? X[((size_t)(a0 * 3) + ad) * ld + i0 + r] : 0.0;
    }
    for (int e = tid; e < na * 3 * CL_TGT; e += blockDim.x) {
      const int r = e % CL_TGT, ad = e / CL_TGT;
      sT[ad / 3][ad % 3][r] = (j0 + r < nConf) ? X[((size_t)(a0 * 3) + ad) * ld + j0 + r] : 0.0;
    }
    __syncthreads();
    for (int a = 0; a < na; ++a) {
      const double ax = sR[a][0][w], ay = sR[a][1][w], az = sR[a][2][w];
      const double bx = sT[a][0][lane], by = sT[a][1][lane], bz = sT[a][2][lane];
      S[0] = da(S[0], dm(ax, bx));
      S[1] = da(S[1], dm(ax, by));
      S[2] = da(S[2], dm(ax, bz));
      S[3] = da(S[3], dm(ay, bx));
      S[4] = da(S[4], dm(ay, by));
      S[5] = da(S[5], dm(ay, bz));
      S[6] = da(S[6], dm(az, bx));
      S[7] = da(S[7], dm(az, by));
      S[8] = da(S[8], dm(az, bz));
    }
  }
  const bool valid = i < nConf && j < nConf;
  double r = 0.0;
  if (valid && (!bits || j < i)) r = rmsd_from_corr(S, G[i], G[j], nSel);
  if (bits) {
    const unsigned word = __ballot_sync(0xffffffffu, valid && j < i && r <= cutoff);
    if (lane == 0 && i < nConf) bits[(size_t)i * W + blockIdx.x] = word;
  } else if (valid) {
    out[(size_t)i * nConf + j] = r;
  }
}

// the reference's greedy pass over candidates in energy order (positions), one CTA
__global__ void __launch_bounds__(1024) k_greedy(int nConf, int W, const uint32_t* __restrict__ bits,
                                                 const int* __restrict__ order, int maxCenters,
                                                 int* __restrict__ centers, int* __restrict__ count_out) {
  const int t = threadIdx.x;
  uint32_t cm = (t == 0) ? 1u : 0u;  // position 0 is the first centre
  int count = 1;
  if (t == 0) centers[0] = order[0];
  for (int pi = 1; pi < nConf; ++pi) {
    const int last = pi >> 5;
    const uint32_t v = (t <= last && t < W) ? (bits[(size_t)pi * W + t] & cm) : 0u;
    const int close = __syncthreads_or(v != 0u);
    if (!close) {
      if (t == last) cm |= 1u << (pi & 31);
      if (t == 0) centers[count] = order[pi];
      ++count;
    }
    if (count == maxCenters) break;
  }
  if (t == 0) *count_out = count;
}

bool finite_all(const double* p, size_t n) {
  for (size_t i = 0; i < n; ++i)
    if (!std::isfinite(p[i])) return false;
  return true;
}

// selected atoms (mask != 0, or all)
std::vector<int> selected_atoms(int nAtom, const unsigned char* mask) {
  std::vector<int> sel;
  for (int a = 0; a < nAtom; ++a)
    if (!mask || mask[a]) sel.push_back(a);
  return sel;
}

struct ClusterBuffers {
  double *coor = nullptr, *X = nullptr, *G = nullptr, *out = nullptr;
  int *sel = nullptr, *order = nullptr, *centers = nullptr, *count = nullptr;
  uint32_t* bits = nullptr;
  cudaStream_t s = nullptr;
  ~ClusterBuffers() {
    if (s) cudaStreamSynchronize(s);
    cudaFree(coor);
    cudaFree(X);
    cudaFree(G);
    cudaFree(out);
    cudaFree(sel);
    cudaFree(order);
    cudaFree(centers);
    cudaFree(count);
    cudaFree(bits);
    if (s) cudaStreamDestroy(s);
  }
};

#define CL_CUDA(call)                                                     \
  do {                                                                    \
    const cudaError_t e_ = (call);                                        \
    if (e_ != cudaSuccess) {                                              \
      set_error(std::string(#call) + ": " + cudaGetErrorString(e_));      \
      return e_ == cudaErrorMemoryAllocation ? CDK_ERR_NOMEM : CDK_ERR_CUDA; \
    }                                                                     \
  } while (0)

// shared set-up: copies, centring (in `order` when given); returns the leading dimension
int prepare(ClusterBuffers& b, int nConf, int nAtom, const double* coor,
            const std::vector<int>& sel, const std::vector<int>* order, int* ld_out) {
  const int ld = (nConf + CL_TGT - 1) / CL_TGT * CL_TGT;
  const int nSel = (int)sel.size();
  CL_CUDA(cudaStreamCreateWithFlags(&b.s, cudaStreamNonBlocking));
  CL_CUDA(cudaMalloc(&b.coor, sizeof(double) * (size_t)nConf * nAtom * 3));
  CL_CUDA(cudaMalloc(&b.sel, sizeof(int) * nSel));
  CL_CUDA(cudaMalloc(&b.X, sizeof(double) * (size_t)nSel * 3 * ld));
  CL_CUDA(cudaMalloc(&b.G, sizeof(double) * ld));
  CL_CUDA(cudaMemcpyAsync(b.coor, coor, sizeof(double) * (size_t)nConf * nAtom * 3,
                          cudaMemcpyHostToDevice, b.s));
  CL_CUDA(cudaMemcpyAsync(b.sel, sel.data(), sizeof(int) * nSel, cudaMemcpyHostToDevice, b.s));
  if (order) {
    CL_CUDA(cudaMalloc(&b.order, sizeof(int) * nConf));
    CL_CUDA(cudaMemcpyAsync(b.order, order->data(), sizeof(int) * nConf, cudaMemcpyHostToDevice, b.s));
  }
  k_center<<<(nConf + 127) / 128, 128, 0, b.s>>>(nConf, nAtom, b.coor, b.sel, nSel, b.order, ld,
                                                 b.X, b.G);
  CL_CUDA(cudaGetLastError());
  *ld_out = ld;
  return CDK_OK;
}

int check_inputs(int nConf, int nAtom, const double* coor, const unsigned char* mask, int cap,
                 std::vector<int>* sel) {
  if (nConf <= 0 || nAtom <= 0 || !coor) {
    set_error("nConf and nAtom must be positive and coor non-null");
    return CDK_ERR_INVALID;
  }
  if (nConf > cap) {
    set_error("too many conformers (limit " + std::to_string(cap) + ")");
    return CDK_ERR_INVALID;
  }
  if (!finite_all(coor, (size_t)nConf * nAtom * 3)) {
    set_error("non-finite conformer coordinate");
    return CDK_ERR_INVALID;
  }
  *sel = selected_atoms(nAtom, mask);
  if (sel->empty()) {
    set_error("the atom mask selects no atom");
    return CDK_ERR_INVALID;
  }
  return CDK_OK;
}

}  // namespace
}  // namespace cdk

using namespace cdk;

extern "C" int cdk_cluster_conformers(int nConf, int nAtom, const double* coor,
                                      const double* energy, const unsigned char* atomMask,
                                      double cutoff, int maxCenters, int* centers,
                                      int* nCenters) {
  std::vector<int> sel;
  int rc = check_inputs(nConf, nAtom, coor, atomMask, CL_MAX_CONF, &sel);
  if (rc != CDK_OK) return rc;
  if (!energy || !centers || !nCenters || !(cutoff >= 0.0) || !std::isfinite(cutoff)) {
    set_error("energy, centers and nCenters must be non-null and cutoff finite, >= 0");
    return CDK_ERR_INVALID;
  }
  if (!finite_all(energy, (size_t)nConf)) {
    set_error("non-finite conformer energy");
    return CDK_ERR_INVALID;
  }
  // energy order exactly as sort_index<double> (include/GeneDiverseConformations.h:9-20)
  std::vector<size_t> idx((size_t)nConf);
  for (size_t i = 0; i != idx.size(); ++i) idx[i] = i;
  std::sort(idx.begin(), idx.end(), [energy](size_t i1, size_t i2) { return energy[i1] < energy[i2]; });
  std::vector<int> order(idx.begin(), idx.end());
  ClusterBuffers b;
  int ld = 0;
  rc = prepare(b, nConf, nAtom, coor, sel, &order, &ld);
  if (rc != CDK_OK) return rc;
  const int W = (nConf + 31) / 32;
  CL_CUDA(cudaMalloc(&b.bits, sizeof(uint32_t) * (size_t)nConf * W));
  CL_CUDA(cudaMalloc(&b.centers, sizeof(int) * nConf));
  CL_CUDA(cudaMalloc(&b.count, sizeof(int)));
  dim3 grid(W, (nConf + CL_REF - 1) / CL_REF);
  k_pairs<<<grid, 256, 0, b.s>>>(nConf, (int)sel.size(), ld, b.X, b.G, cutoff, b.bits, W, nullptr);
  CL_CUDA(cudaGetLastError());
  k_greedy<<<1, 1024, 0, b.s>>>(nConf, W, b.bits, b.order, maxCenters, b.centers, b.count);
  CL_CUDA(cudaGetLastError());
  int count = 0;
  CL_CUDA(cudaMemcpyAsync(&count, b.count, sizeof(int), cudaMemcpyDeviceToHost, b.s));
  CL_CUDA(cudaStreamSynchronize(b.s));
  if (count < 1 || count > nConf) {
    set_error("clustering returned an invalid centre count");
    return CDK_ERR_CUDA;
  }
  CL_CUDA(cudaMemcpyAsync(centers, b.centers, sizeof(int) * count, cudaMemcpyDeviceToHost, b.s));
  CL_CUDA(cudaStreamSynchronize(b.s));
  *nCenters = count;
  return CDK_OK;
}

extern "C" int cdk_pair_rmsd(int nConf, int nAtom, const double* coor,
                             const unsigned char* atomMask, double* out) {
  std::vector<int> sel;
  int rc = check_inputs(nConf, nAtom, coor, atomMask, CL_MAX_CONF_MATRIX, &sel);
  if (rc != CDK_OK) return rc;
  if (!out) {
    set_error("out must be non-null");
    return CDK_ERR_INVALID;
  }
  ClusterBuffers b;
  int ld = 0;
  rc = prepare(b, nConf, nAtom, coor, sel, nullptr, &ld);
  if (rc != CDK_OK) return rc;
  CL_CUDA(cudaMalloc(&b.out, sizeof(double) * (size_t)nConf * nConf));
  dim3 grid((nConf + CL_TGT - 1) / CL_TGT, (nConf + CL_REF - 1) / CL_REF);
  k_pairs<<<grid, 256, 0, b.s>>>(nConf, (int)sel.size(), ld, b.X, b.G, 0.0, nullptr, 0, b.out);
  CL_CUDA(cudaGetLastError());
  CL_CUDA(cudaMemcpyAsync(out, b.out, sizeof(double) * (size_t)nConf * nConf, cudaMemcpyDeviceToHost, b.s));
  CL_CUDA(cudaStreamSynchronize(b.s));
  return CDK_OK;
}
