// receptor_grids.cu -- receptor potential grids on the GPU.
//
// The reference reads its receptor grids from files written by CHARMM (src/ReadGrids.cpp:6-68);
// computing them is a step outside the search that the grid file format hands over. Here the
// same grids as cdk_synth_receptor_grids (host, multithreaded) are computed on the GPU: nVdw
// soft-core capped Lennard-Jones grids at the probe radii and one Coulomb grid with the
// distance-dependent dielectric eps(r) = 4r, capped at +-elecCap, summed over the receptor atoms
// within `cutoff` of each grid point.
//
// One thread per grid point. The atoms are visited through the host's cell list (cells of edge
// `cutoff`, atoms of a cell in ascending order, the 27 neighbour cells in the host's loop order)
// and every double operation is an explicit round-to-nearest intrinsic (no contraction), so the
// grids are bit-identical to the host function's.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/cdock_b200.h"
#include "cdk_internal.h"

namespace cdk {
namespace {

constexpr int RG_MAX_VDW = 15;

__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }

struct GridGeom {
  int n, nVdw;
  int nc[3];
  float spacing, cutoff, vdwCap, elecCap;
  float origin[3], lo[3];
};

__global__ void __launch_bounds__(128) k_receptor_grids(GridGeom g, const float* __restrict__ xyz,
                                                        const float* __restrict__ radius,
                                                        const float* __restrict__ sqrtEps,
                                                        const float* __restrict__ charge,
                                                        const float* __restrict__ probe,
                                                        const int* __restrict__ cell_start,
                                                        const int* __restrict__ cell_atoms,
                                                        float* __restrict__ out) {
  const size_t N = (size_t)g.n * g.n * g.n;
  const size_t gi = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (gi >= N) return;
  const int k = (int)(gi % g.n), j = (int)((gi / g.n) % g.n), i = (int)(gi / ((size_t)g.n * g.n));
  const double h = (double)g.spacing;
  const double p[3] = {dadd((double)g.origin[0], dmul((double)i, h)),
                       dadd((double)g.origin[1], dmul((double)j, h)),
                       dadd((double)g.origin[2], dmul((double)k, h))};
  const double cut = (double)g.cutoff;
  const double cut2 = dmul(cut, cut);
  double acc[RG_MAX_VDW + 1];
  for (int v = 0; v <= g.nVdw; ++v) acc[v] = 0.0;
  int c[3];
  for (int d = 0; d < 3; ++d)  // clamped as on the host: far cells have no occupied neighbours
    c[d] = (int)floor(fmin(fmax(__ddiv_rn(dsub(p[d], (double)g.lo[d]), cut), -2.0), g.nc[d] + 1.0));
  for (int cx = c[0] - 1; cx <= c[0] + 1; ++cx)
    for (int cy = c[1] - 1; cy <= c[1] + 1; ++cy)
      for (int cz = c[2] - 1; cz <= c[2] + 1; ++cz) {
        if (cx < 0 || cy < 0 || cz < 0 || cx >= g.nc[0] || cy >= g.nc[1] || cz >= g.nc[2]) continue;
        const int cell = (cx * g.nc[1] + cy) * g.nc[2] + cz;
        for (int t = cell_start[cell]; t < cell_start[cell + 1]; ++t) {
          const int a = cell_atoms[t];
          const double dx = dsub(p[0], (double)xyz[a * 3]);
          const double dy = dsub(p[1], (double)xyz[a * 3 + 1]);
          const double dz = dsub(p[2], (double)xyz[a * 3 + 2]);
          const double d2 = dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz));
          if (d2 > cut2) continue;
          const double se = (double)sqrtEps[a];
          for (int v = 0; v < g.nVdw; ++v) {
            const double rmin = dadd((double)radius[a], (double)probe[v]);
            const double dd2 = fmax(d2, dmul(dmul(0.25, rmin), rmin));
            const double s2 = __ddiv_rn(dmul(rmin, rmin), dd2);
            const double s6 = dmul(dmul(s2, s2), s2);
            acc[v] = dadd(acc[v], dmul(se, dsub(dmul(s6, s6), dmul(2.0, s6))));
          }
          acc[g.nVdw] = dadd(acc[g.nVdw], __ddiv_rn(dmul(332.0716, (double)charge[a]), dmul(4.0, fmax(d2, 0.25))));
        }
      }
  for (int v = 0; v < g.nVdw; ++v) out[(size_t)v * N + gi] = (float)fmin(acc[v], (double)g.vdwCap);
  out[(size_t)g.nVdw * N + gi] = (float)fmax(-(double)g.elecCap, fmin(acc[g.nVdw], (double)g.elecCap));
}

}  // namespace
}  // namespace cdk

using namespace cdk;

extern "C" int cdk_receptor_grids_gpu(int device, int n, float spacing, const float* origin, int nAtom,
                                      const float* xyz, const float* radius, const float* sqrtEps,
                                      const float* charge, int nVdw, const float* probe, float vdwCap,
                                      float elecCap, float cutoff, float* out) {
  if (n <= 0 || nAtom < 0 || nVdw < 0 || nVdw > RG_MAX_VDW || !origin || !out ||
      (nAtom && (!xyz || !radius || !sqrtEps || !charge)) || (nVdw && !probe) || !(cutoff > 0)) {
    set_error("invalid argument (nVdw <= 15, cutoff > 0, non-null arrays)");
    return CDK_ERR_INVALID;
  }
  {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev) {
      set_error("no such CUDA device");
      return CDK_ERR_INVALID;
    }
    const cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) {
      set_error(std::string("cudaSetDevice: ") + cudaGetErrorString(e));
      return CDK_ERR_CUDA;
    }
  }
  // the host function's cell list: same bounds, cell edge, atom order within cells
  GridGeom g{};
  g.n = n;
  g.nVdw = nVdw;
  g.spacing = spacing;
  g.cutoff = cutoff;
  g.vdwCap = vdwCap;
  g.elecCap = elecCap;
  float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
  for (int a = 0; a < nAtom; ++a)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], xyz[a * 3 + d]);
      hi[d] = std::max(hi[d], xyz[a * 3 + d]);
    }
  for (int d = 0; d < 3; ++d) {
    g.nc[d] = nAtom ? std::max(1, (int)std::ceil((hi[d] - lo[d]) / cutoff) + 1) : 1;
    g.lo[d] = lo[d];
    g.origin[d] = origin[d];
  }
  const size_t ncell = (size_t)g.nc[0] * g.nc[1] * g.nc[2];
  if (ncell > ((size_t)1 << 26)) {
    set_error("cell list too large: raise cutoff or check the coordinates");
    return CDK_ERR_INVALID;
  }
  std::vector<int> count(ncell + 1, 0), cell_of_atom(nAtom);
  for (int a = 0; a < nAtom; ++a) {
    int c[3];
    for (int d = 0; d < 3; ++d) c[d] = std::min(g.nc[d] - 1, (int)((xyz[a * 3 + d] - lo[d]) / cutoff));
    cell_of_atom[a] = (int)(((size_t)c[0] * g.nc[1] + c[1]) * g.nc[2] + c[2]);
    count[cell_of_atom[a] + 1]++;
  }
  for (size_t c = 0; c < ncell; ++c) count[c + 1] += count[c];
  std::vector<int> atoms(std::max(nAtom, 1)), fill(count.begin(), count.end() - 1);
  for (int a = 0; a < nAtom; ++a) atoms[fill[cell_of_atom[a]]++] = a;  // ascending within a cell

  const size_t N = (size_t)n * n * n;
  float *d_xyz = nullptr, *d_rad = nullptr, *d_se = nullptr, *d_q = nullptr, *d_probe = nullptr, *d_out = nullptr;
  int *d_start = nullptr, *d_atoms = nullptr;
  cudaStream_t s = nullptr;
  int rc = CDK_OK;
  auto cuda_ok = [&](cudaError_t e, const char* what) {
    if (e != cudaSuccess && rc == CDK_OK) {
      set_error(std::string(what) + ": " + cudaGetErrorString(e));
      rc = e == cudaErrorMemoryAllocation ? CDK_ERR_NOMEM : CDK_ERR_CUDA;
    }
    return rc == CDK_OK;
  };
  const size_t na = (size_t)std::max(nAtom, 1);
  if (cuda_ok(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "stream") &&
      cuda_ok(cudaMalloc(&d_xyz, sizeof(float) * 3 * na), "cudaMalloc") &&
      cuda_ok(cudaMalloc(&d_rad, sizeof(float) * na), "cudaMalloc") &&
      cuda_ok(cudaMalloc(&d_se, sizeof(float) * na), "cudaMalloc") &&
      cuda_ok(cudaMalloc(&d_q, sizeof(float) * na), "cudaMalloc") &&
      cuda_ok(cudaMalloc(&d_probe, sizeof(float) * std::max(nVdw, 1)), "cudaMalloc") &&
      cuda_ok(cudaMalloc(&d_start, sizeof(int) * (ncell + 1)), "cudaMalloc") &&
      cuda_ok(cudaMalloc(&d_atoms, sizeof(int) * na), "cudaMalloc") &&
      cuda_ok(cudaMalloc(&d_out, sizeof(float) * (nVdw + 1) * N), "cudaMalloc")) {
    if (nAtom) {
      cuda_ok(cudaMemcpyAsync(d_xyz, xyz, sizeof(float) * 3 * nAtom, cudaMemcpyHostToDevice, s), "H2D");
      cuda_ok(cudaMemcpyAsync(d_rad, radius, sizeof(float) * nAtom, cudaMemcpyHostToDevice, s), "H2D");
      cuda_ok(cudaMemcpyAsync(d_se, sqrtEps, sizeof(float) * nAtom, cudaMemcpyHostToDevice, s), "H2D");
      cuda_ok(cudaMemcpyAsync(d_q, charge, sizeof(float) * nAtom, cudaMemcpyHostToDevice, s), "H2D");
      cuda_ok(cudaMemcpyAsync(d_atoms, atoms.data(), sizeof(int) * nAtom, cudaMemcpyHostToDevice, s), "H2D");
    }
    if (nVdw) cuda_ok(cudaMemcpyAsync(d_probe, probe, sizeof(float) * nVdw, cudaMemcpyHostToDevice, s), "H2D");
    cuda_ok(cudaMemcpyAsync(d_start, count.data(), sizeof(int) * (ncell + 1), cudaMemcpyHostToDevice, s), "H2D");
    if (rc == CDK_OK) {
      k_receptor_grids<<<(unsigned)((N + 127) / 128), 128, 0, s>>>(g, d_xyz, d_rad, d_se, d_q, d_probe, d_start,
                                                                  d_atoms, d_out);
      cuda_ok(cudaGetLastError(), "k_receptor_grids");
    }
    if (rc == CDK_OK)
      cuda_ok(cudaMemcpyAsync(out, d_out, sizeof(float) * (nVdw + 1) * N, cudaMemcpyDeviceToHost, s), "D2H");
    if (s) cuda_ok(cudaStreamSynchronize(s), "k_receptor_grids");
  }
  cudaFree(d_xyz);
  cudaFree(d_rad);
  cudaFree(d_se);
  cudaFree(d_q);
  cudaFree(d_probe);
  cudaFree(d_start);
  cudaFree(d_atoms);
  cudaFree(d_out);
  if (s) cudaStreamDestroy(s);
  return rc;
}
