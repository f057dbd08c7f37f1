// tranrota_driver.cpp -- the reference driver's search block, re-linked against the C++ API.
//
// Test program (built and run by tests/test_cxx_driver.py). It restates the per-conformer
// search loop of src/TranRotaConfSearchNoMini.cu:96-487 -- vdW grid selection and compaction,
// quaternion sampling from one shared mt19937_64, filtering, the translational-rotational
// search, sort_index over the per-rotation minima and the pose rebuild of the nLowest
// orientations -- with every step a call into cdock_b200.hpp (namespace cdk), the way a
// maintainer re-links the reference driver. OpenMM/OpenBabel parts (parameters, conformer
// generation, PDB writing) are replaced by a binary input file and a binary output file.
//
// Input (little-endian): int n, K0 (grids incl. elec), nAtom, nConf, nRotaSample, maxNQ,
// nLowest; uint64 seed; float spacing, mid[3], len[3]; float gridRadii[K0-1],
// gridValues[K0][n][n][n], coor[nConf][nAtom][3], charge[nAtom], eps[nAtom], radii[nAtom].
// Output: int K; per conformer: int nUsed, float quats[nUsed][4], float minE[nUsed],
// int idx[nUsed][3], int nPose, then per pose int idxQ and double coor[nAtom][3].
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "cdock_b200.hpp"

namespace {

template <typename T>
bool rd(FILE* f, T* p, size_t n) {
  return std::fread(p, sizeof(T), n, f) == n;
}
template <typename T>
void wr(FILE* f, const T* p, size_t n) {
  std::fwrite(p, sizeof(T), n, f);
}

}  // namespace

int main(int argc, char** argv) {
  if (argc != 3) {
    std::fprintf(stderr, "usage: %s input.bin output.bin\n", argv[0]);
    return 2;
  }
  FILE* in = std::fopen(argv[1], "rb");
  if (!in) return 2;
  int hdr[7];
  uint64_t seed = 0;
  float spacing = 0.f, mid[3], len[3];
  if (!rd(in, hdr, 7) || !rd(in, &seed, 1) || !rd(in, &spacing, 1) || !rd(in, mid, 3) || !rd(in, len, 3))
    return 2;
  const int n = hdr[0], K0 = hdr[1], nAtom = hdr[2], nConf = hdr[3], nRotaSample = hdr[4];
  const int maxNQ = hdr[5], nLowest = hdr[6];
  const size_t N = (size_t)n * n * n;
  std::vector<float> gridRadii(K0 - 1), gridValues((size_t)K0 * N), coors((size_t)nConf * nAtom * 3);
  std::vector<float> charge(nAtom), eps(nAtom), radii(nAtom);
  if (!rd(in, gridRadii.data(), gridRadii.size()) || !rd(in, gridValues.data(), gridValues.size()) ||
      !rd(in, coors.data(), coors.size()) || !rd(in, charge.data(), nAtom) || !rd(in, eps.data(), nAtom) ||
      !rd(in, radii.data(), nAtom))
    return 2;
  std::fclose(in);

  try {
    // vdW grids the ligand's atoms use, then the electrostatic grid (:122-146)
    const int numOfVdwGrids = K0 - 1;
    int numOfVdwGridsUsed = 0;
    std::vector<int> idxOfVdwUsed;
    std::vector<std::vector<int> > idxOfAtomVdwRadius(numOfVdwGrids);
    cdk::GetIdxOfAtomsForVdwRadius(nAtom, radii.data(), numOfVdwGrids, gridRadii.data(), numOfVdwGridsUsed,
                                   idxOfVdwUsed, idxOfAtomVdwRadius);
    const int numOfGridsUsed = numOfVdwGridsUsed + 1;
    std::vector<float> usedGridValues((size_t)numOfGridsUsed * N);
    for (int i = 0; i < numOfVdwGridsUsed; ++i)
      std::memcpy(&usedGridValues[i * N], &gridValues[(size_t)idxOfVdwUsed[i] * N], sizeof(float) * N);
    std::memcpy(&usedGridValues[numOfVdwGridsUsed * N], &gridValues[(size_t)numOfVdwGrids * N], sizeof(float) * N);
    // the search takes each atom's slot among the used vdW grids
    std::vector<int> slots(nAtom, 0);
    for (int j = 0; j < numOfVdwGridsUsed; ++j)
      for (int a : idxOfAtomVdwRadius[idxOfVdwUsed[j]]) slots[a] = j;

    // grid corner as the driver computes it (:149-151): float arithmetic, widened to double
    const double gridMin[3] = {(double)(mid[0] - len[0] / 2), (double)(mid[1] - len[1] / 2),
                               (double)(mid[2] - len[2] / 2)};

    // the receptor spectra stay resident for every conformer (replaces :156-199)
    cdk::TranRotaSearch search(n, n, n, spacing, numOfGridsUsed, usedGridValues.data());
    std::mt19937_64 gen(seed);  // the reference seeds from std::random_device (:203-204)

    FILE* out = std::fopen(argv[2], "wb");
    if (!out) return 2;
    wr(out, &numOfGridsUsed, 1);
    float* quaternions = nullptr;
    float* quaternionsUsed = nullptr;
    std::vector<float> conformerCoor((size_t)nAtom * 3);
    for (int c = 0; c < nConf; ++c) {
      std::memcpy(conformerCoor.data(), &coors[(size_t)c * nAtom * 3], sizeof(float) * nAtom * 3);
      cdk::QuaternionUniformSampling(gen, quaternions, nRotaSample);
      const int numOfQuaternionsUsed =
          cdk::FilterQuaternions(conformerCoor.data(), nAtom, nRotaSample, quaternions, len[0], len[1], len[2],
                                 maxNQ, quaternionsUsed);
      // rotate, fill, transform, correlate and reduce every used rotation (:333-465)
      std::vector<float> minEnergy;
      std::vector<int> ix, iy, iz;
      search.Search(nAtom, 1, conformerCoor.data(), charge.data(), eps.data(), slots.data(), numOfQuaternionsUsed,
                    quaternionsUsed, minEnergy, ix, iy, iz);
      wr(out, &numOfQuaternionsUsed, 1);
      wr(out, quaternionsUsed, (size_t)numOfQuaternionsUsed * 4);
      wr(out, minEnergy.data(), minEnergy.size());
      for (int q = 0; q < numOfQuaternionsUsed; ++q) {
        const int idx[3] = {ix[q], iy[q], iz[q]};
        wr(out, idx, 3);
      }
      // the nLowest orientations and their poses (:467-487)
      const std::vector<size_t> order = cdk::sort_index(minEnergy);
      const int nPose = std::min(nLowest, numOfQuaternionsUsed);
      wr(out, &nPose, 1);
      std::vector<double> pose((size_t)nAtom * 3);
      for (int l = 0; l < nPose; ++l) {
        const int idxQ = (int)order[l];
        const int idx[3] = {ix[idxQ], iy[idxQ], iz[idxQ]};
        const int rc = cdk_pose_coordinates(nAtom, conformerCoor.data(), quaternionsUsed + 4 * idxQ, gridMin,
                                            spacing, idx, pose.data());
        if (rc != CDK_OK) throw cdk::Error(rc, "cdk_pose_coordinates");
        wr(out, &idxQ, 1);
        wr(out, pose.data(), pose.size());
      }
    }
    delete[] quaternions;
    delete[] quaternionsUsed;
    std::fclose(out);
  } catch (const cdk::Error& e) {
    std::fprintf(stderr, "cdk error %d: %s\n", e.code, e.what());
    return 1;
  }
  return 0;
}
