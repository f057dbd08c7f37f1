// ref_cufft_path.cu -- the reference's cuFFT search path, run as the reference runs it.
//
// TEST INFRASTRUCTURE ONLY (oracle). The search core of the reference lives inline in
// main() (src/TranRotaConfSearchNoMini.cu:156-464), next to OpenMM/OpenBabel code that is not
// available here, so this file restates that orchestration step by step and links it with the
// reference's own unmodified pieces: src/kernel.cu (ConjMult, SumGrids), the host helpers
// (Rotate, GetMinCoors, GetMaxCoors, GetIdxOfAtomsForVdwRadius, FillLigandGrid) and cuFFT.
// oracle/Makefile builds it into oracle/_ref/libcdk_ref_cufft.so.
//
// Differences from main(), all of them needed to run it safely or to measure it:
//  * d_ligand_F and d_ligand_sum_F are padded to the full extent the reference launches
//    touch. ConjMult and SumGrids have no bounds check (src/kernel.cu:8, :18) and their grids
//    ((Q*K*odist)/2^20+1, 1024) x 1024 threads (:232-239) overshoot the Q*K*odist allocation
//    (:220); SumGrids also reads up to K-fold further into d_ligand_F (:25).
//  * errors return a status instead of exit(); per-stage wall times are reported.
//  * the z bound of the translation window uses zdim (the reference reads ydim at :450,
//    the same number on the cubic grids used here).
#include <cuda_runtime.h>
#include <cufft.h>

#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "FillLigandGrid.h"
#include "GetIdxOfAtomsForVdwRadius.h"
#include "GetMaxCoors.h"
#include "GetMinCoors.h"
#include "Rotate.h"
#include "kernel.h"

namespace {
double now_ms() {
  return std::chrono::duration<double, std::milli>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}
}  // namespace

extern "C" {

// One conformer, nQ already-filtered quaternions. grids: all numOfGrids = nVdw+1 receptor
// grids [nVdw+1][X][Y][Z] (elec last), compacted here to the used ones as the driver does
// (:126-146). Outputs minE[nQ] (float) and idx[nQ][3]. times_ms[0..5]: host fill (incl. memset),
// H2D, GPU (R2C + ConjMult + SumGrids + C2R), D2H, host argmin, total.
int refcufft_search(int X, int Y, int Z, float spacing, int nVdw, const float* gridRadii,
                    const float* grids, int nAtom, const float* conf, const float* charge,
                    const float* eps, const float* radii, int nQ, const float* quats,
                    int batchQ, float* minE, int* idx, double* times_ms) {
  const double t_begin = now_ms();
  double t_fill = 0, t_h2d = 0, t_gpu = 0, t_d2h = 0, t_arg = 0;
  std::vector<float> r(radii, radii + nAtom), g(gridRadii, gridRadii + nVdw);
  int nUsed = 0;
  std::vector<int> used;
  std::vector<std::vector<int> > byGrid(nVdw);
  GetIdxOfAtomsForVdwRadius(nAtom, r.data(), nVdw, g.data(), nUsed, used, byGrid);
  const int K = nUsed + 1;
  const size_t N = (size_t)X * Y * Z;
  std::vector<float> usedGrid((size_t)K * N);
  for (int i = 0; i < nUsed; ++i)
    std::memcpy(&usedGrid[i * N], grids + (size_t)used[i] * N, sizeof(float) * N);
  std::memcpy(&usedGrid[nUsed * N], grids + (size_t)nVdw * N, sizeof(float) * N);

  int n[3] = {X, Y, Z};
  int inembed[3] = {X, Y, Z};
  int onembed[3] = {X, Y, Z / 2 + 1};
  const int idist = X * Y * Z;
  const int odist = X * Y * (Z / 2 + 1);
  const int Q = batchQ;

  // padded extents of the reference launches
  const size_t launchConj = ((size_t)Q * K * odist / (1024 * 1024) + 1) * 1024 * 1024;
  const size_t launchSum = ((size_t)Q * odist / (1024 * 1024) + 1) * 1024 * 1024;
  const size_t sumReadQ = (launchSum - 1) / odist + 1;
  size_t ligFElems = launchConj;
  if (sumReadQ * K * odist > ligFElems) ligFElems = sumReadQ * K * odist;
  if ((size_t)Q * K * odist > ligFElems) ligFElems = (size_t)Q * K * odist;

  cufftReal *d_pot_f = nullptr, *d_lig_f = nullptr, *d_sum_f = nullptr;
  cufftComplex *d_pot_F = nullptr, *d_lig_F = nullptr, *d_sum_F = nullptr;
  cufftHandle potPlan = 0, ligPlan = 0, invPlan = 0;
  int status = 0;
#define RC_CHECK(x)      \
  do {                   \
    if ((x) != 0) {      \
      status = __LINE__; \
      goto done;         \
    }                    \
  } while (0)
  {
    RC_CHECK(cudaMalloc((void**)&d_pot_f, sizeof(cufftReal) * K * idist));
    RC_CHECK(cudaMalloc((void**)&d_pot_F, sizeof(cufftComplex) * K * odist));
    RC_CHECK(cudaMemcpy(d_pot_f, usedGrid.data(), sizeof(cufftReal) * K * idist,
                        cudaMemcpyHostToDevice));
    RC_CHECK(cufftPlanMany(&potPlan, 3, n, inembed, 1, idist, onembed, 1, odist, CUFFT_R2C, K));
    RC_CHECK(cufftExecR2C(potPlan, d_pot_f, d_pot_F));

    RC_CHECK(cudaMalloc((void**)&d_lig_f, sizeof(cufftReal) * (size_t)Q * K * idist));
    RC_CHECK(cudaMalloc((void**)&d_lig_F, sizeof(cufftComplex) * ligFElems));
    RC_CHECK(cudaMemset(d_lig_F, 0, sizeof(cufftComplex) * ligFElems));
    RC_CHECK(cufftPlanMany(&ligPlan, 3, n, inembed, 1, idist, onembed, 1, odist, CUFFT_R2C,
                           Q * K));
    RC_CHECK(cudaMalloc((void**)&d_sum_F, sizeof(cufftComplex) * launchSum));
    RC_CHECK(cudaMemset(d_sum_F, 0, sizeof(cufftComplex) * launchSum));
    RC_CHECK(cudaMalloc((void**)&d_sum_f, sizeof(cufftReal) * (size_t)Q * idist));
    RC_CHECK(cufftPlanMany(&invPlan, 3, n, onembed, 1, odist, inembed, 1, idist, CUFFT_C2R, Q));

    dim3 thrConj(1024, 1, 1), blkConj((unsigned)((size_t)Q * K * odist / (1024 * 1024) + 1), 1024, 1);
    dim3 thrSum(1024, 1, 1), blkSum((unsigned)((size_t)Q * odist / (1024 * 1024) + 1), 1024, 1);

    // rotate all quaternions, bounding boxes, lengths (:352-372)
    std::vector<float> coors((size_t)nQ * nAtom * 3), mn((size_t)nQ * 3), mx((size_t)nQ * 3),
        len((size_t)nQ * 3);
    for (int i = 0; i < nQ; ++i)
      for (int j = 0; j < nAtom; ++j)
        Rotate(&quats[i * 4], &conf[j * 3], &coors[(size_t)i * nAtom * 3 + j * 3]);
    GetMinCoors(nQ, nAtom, coors.data(), mn.data());
    GetMaxCoors(nQ, nAtom, coors.data(), mx.data());
    for (int i = 0; i < nQ * 3; ++i) len[i] = mx[i] - mn[i];
    for (int i = 0; i < nQ; ++i) {
      minE[i] = INFINITY;
      idx[i * 3 + 0] = idx[i * 3 + 1] = idx[i * 3 + 2] = -1;
    }
    std::vector<float> lig((size_t)Q * K * N);
    std::vector<float> energy((size_t)Q * idist);
    std::vector<float> ch(charge, charge + nAtom), ep(eps, eps + nAtom);
    const int nBatches = (nQ % Q == 0) ? nQ / Q : nQ / Q + 1;
    for (int b = 0; b < nBatches; ++b) {
      double t0 = now_ms();
      std::memset(lig.data(), 0, sizeof(float) * lig.size());
      int nq = ((b + 1) * Q > nQ) ? nQ - b * Q : Q;
      FillLigandGrid(nq, nAtom, &coors[(size_t)b * Q * nAtom * 3], &mn[(size_t)b * Q * 3],
                     ch.data(), ep.data(), nUsed, used, byGrid, X, Y, Z, spacing, lig.data());
      double t1 = now_ms();
      RC_CHECK(cudaMemcpy(d_lig_f, lig.data(), sizeof(cufftReal) * (size_t)Q * K * idist,
                          cudaMemcpyHostToDevice));
      double t2 = now_ms();
      RC_CHECK(cufftExecR2C(ligPlan, d_lig_f, d_lig_F));
      ConjMult<<<blkConj, thrConj>>>(d_pot_F, d_lig_F, odist, K);
      RC_CHECK(cudaPeekAtLastError());
      SumGrids<<<blkSum, thrSum>>>(d_lig_F, d_sum_F, K, odist, idist);
      RC_CHECK(cudaPeekAtLastError());
      RC_CHECK(cufftExecC2R(invPlan, d_sum_F, d_sum_f));
      RC_CHECK(cudaDeviceSynchronize());
      double t3 = now_ms();
      RC_CHECK(cudaMemcpy(energy.data(), d_sum_f, sizeof(float) * (size_t)Q * idist,
                          cudaMemcpyDeviceToHost));
      double t4 = now_ms();
      // host argmin (:441-464): double division by sqrt(idist), compare against the float min
      for (int q = 0; q < Q; ++q) {
        int iq = b * Q + q;
        if (iq >= nQ) continue;
        int wx = X - int(len[iq * 3 + 0] / spacing) - 2;
        int wy = Y - int(len[iq * 3 + 1] / spacing) - 2;
        int wz = Z - int(len[iq * 3 + 2] / spacing) - 2;
        for (int i = 0; i < wx; ++i)
          for (int j = 0; j < wy; ++j)
            for (int k = 0; k < wz; ++k) {
              size_t tmp = (size_t)q * idist + ((size_t)i * Y + j) * Z + k;
              if (energy[tmp] / std::sqrt((double)idist) < minE[iq]) {
                minE[iq] = energy[tmp] / std::sqrt((double)idist);
                idx[iq * 3 + 0] = i;
                idx[iq * 3 + 1] = j;
                idx[iq * 3 + 2] = k;
              }
            }
      }
      double t5 = now_ms();
      t_fill += t1 - t0;
      t_h2d += t2 - t1;
      t_gpu += t3 - t2;
      t_d2h += t4 - t3;
      t_arg += t5 - t4;
    }
  }
done:
  if (potPlan) cufftDestroy(potPlan);
  if (ligPlan) cufftDestroy(ligPlan);
  if (invPlan) cufftDestroy(invPlan);
  cudaFree(d_pot_f);
  cudaFree(d_pot_F);
  cudaFree(d_lig_f);
  cudaFree(d_lig_F);
  cudaFree(d_sum_F);
  cudaFree(d_sum_f);
  if (times_ms) {
    times_ms[0] = t_fill;
    times_ms[1] = t_h2d;
    times_ms[2] = t_gpu;
    times_ms[3] = t_d2h;
    times_ms[4] = t_arg;
    times_ms[5] = now_ms() - t_begin;
  }
  return status;
#undef RC_CHECK
}

// The reference's kernel.h pair on given spectra, launched as the driver launches them
// (src/TranRotaConfSearchNoMini.cu:232-239, :423-426): ConjMult over the Q x K ligand spectra,
// then SumGrids into Q summed spectra. Host arrays of interleaved complex floats in and out:
// pot [K][odist], lig [Q][K][odist] (ConjMult's in-place result is written back to lig_out),
// sum_out [Q][odist]. The device buffers are padded to the launches' extents (no bounds checks
// in src/kernel.cu) and zero-filled beyond the data. Returns 0 or the failing line.
#define RC_CHECK(x)      \
  do {                   \
    if ((x) != 0) {      \
      status = __LINE__; \
      goto done;         \
    }                    \
  } while (0)
int refcufft_kernels(int odist, int K, int Q, int idist, const float* pot, const float* lig,
                     float* lig_out, float* sum_out) {
  const size_t launchConj = ((size_t)Q * K * odist / (1024 * 1024) + 1) * 1024 * 1024;
  const size_t launchSum = ((size_t)Q * odist / (1024 * 1024) + 1) * 1024 * 1024;
  const size_t sumReadQ = (launchSum - 1) / odist + 1;
  size_t ligElems = launchConj;
  if (sumReadQ * K * odist > ligElems) ligElems = sumReadQ * K * odist;
  if ((size_t)Q * K * odist > ligElems) ligElems = (size_t)Q * K * odist;
  cufftComplex *d_pot = nullptr, *d_lig = nullptr, *d_sum = nullptr;
  int status = 0;
  {
    RC_CHECK(cudaMalloc((void**)&d_pot, sizeof(cufftComplex) * K * odist));
    RC_CHECK(cudaMalloc((void**)&d_lig, sizeof(cufftComplex) * ligElems));
    RC_CHECK(cudaMalloc((void**)&d_sum, sizeof(cufftComplex) * launchSum));
    RC_CHECK(cudaMemset(d_lig, 0, sizeof(cufftComplex) * ligElems));
    RC_CHECK(cudaMemcpy(d_pot, pot, sizeof(cufftComplex) * K * odist, cudaMemcpyHostToDevice));
    RC_CHECK(cudaMemcpy(d_lig, lig, sizeof(cufftComplex) * (size_t)Q * K * odist, cudaMemcpyHostToDevice));
    dim3 thrConj(1024, 1, 1), blkConj((unsigned)((size_t)Q * K * odist / (1024 * 1024) + 1), 1024, 1);
    dim3 thrSum(1024, 1, 1), blkSum((unsigned)((size_t)Q * odist / (1024 * 1024) + 1), 1024, 1);
    ConjMult<<<blkConj, thrConj>>>(d_pot, d_lig, odist, K);
    RC_CHECK(cudaGetLastError());
    RC_CHECK(cudaMemcpy(lig_out, d_lig, sizeof(cufftComplex) * (size_t)Q * K * odist, cudaMemcpyDeviceToHost));
    SumGrids<<<blkSum, thrSum>>>(d_lig, d_sum, K, odist, idist);
    RC_CHECK(cudaGetLastError());
    RC_CHECK(cudaMemcpy(sum_out, d_sum, sizeof(cufftComplex) * (size_t)Q * odist, cudaMemcpyDeviceToHost));
  }
done:
  cudaFree(d_pot);
  cudaFree(d_lig);
  cudaFree(d_sum);
  return status;
}
#undef RC_CHECK

}  // extern "C"
