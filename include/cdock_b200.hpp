// cdock_b200.hpp -- C++ host API with the reference's own entry points for the search path.
//
// The reference's drivers call these helpers by name (src/TranRotaConfSearchNoMini.cu:96-464).
// Each function here keeps the reference's name, argument meaning and ownership rules, inside
// namespace cdk, so a driver re-links by qualifying the calls (or `using namespace cdk;`):
//  - QuaternionUniformSampling, FilterQuaternions: delete[] and re-new[] their float*& output,
//    like src/QuaternionUniformSampling.cpp:8-9 and src/FilterQuaternions.cpp:67-68.
//  - FillLigandGrid runs on the GPU (bit-exact with src/FillLigandGrid.cpp:7-120).
//  - TranRotaSearch replaces the inline cuFFT core (src/TranRotaConfSearchNoMini.cu:156-464).
// Errors throw cdk::Error (the reference exits or prints and returns); the C-ABI in
// cdock_b200.h returns status codes instead.
#pragma once
#include <cstdint>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "cdock_b200.h"

namespace cdk {

struct Error : std::runtime_error {
  int code;
  Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

void QuaternionMultiply(const float* const lq, const float* const rq, float* const result);
void Rotate(const float* const quaternion, const float* const icoor, float* const fcoor);
void GetMinCoors(int nQuaternions, int nAtoms, float* coors, float* mincoors);
void GetMaxCoors(int nQuaternions, int nAtoms, float* coors, float* maxcoors);
void QuaternionUniformSampling(std::mt19937_64& gen, float*& quaters, int nQuaters);
int FilterQuaternions(float* coor, int nAtom, int nQuater, float* quaternions, float gridLenX,
                      float gridLenY, float gridLenZ, int maxNQuaternionsUsed,
                      float*& quaternionsUsed);
void GetIdxOfAtomsForVdwRadius(int nAtoms, float* atomRadii, int numOfVdwGrids,
                               float* gridRadii, int& numOfVdwGridsUsed,
                               std::vector<int>& idxOfVdwUsed,
                               std::vector<std::vector<int> >& idxOfAtomVdwRadius);
void FillLigandGrid(int nQuaternions, int nAtoms, float* coors, float* mincoors,
                    float* atomCharges, float* atomEpsilons, int numOfVdwGridsUsed,
                    std::vector<int> idxOfVdwUsed,
                    std::vector<std::vector<int> >& idxOfAtomVdwRadius, int xdim, int ydim,
                    int zdim, float spacing, float* ligandGridValues);
void ReadGrids(int& numOfGrids, int& xdim, int& ydim, int& zdim, float& midx, float& midy,
               float& midz, float& xlen, float& ylen, float& zlen, float& spacing,
               float& restraint_k, float*& raddi, float*& values, std::string fileName);

// indices of v sorted by value (std::sort, strict <; include/GeneDiverseConformations.h:9-20)
std::vector<size_t> sort_index(const std::vector<float>& v);

// indices of v sorted by value, for the conformer energies (the double instantiation)
std::vector<size_t> sort_index(const std::vector<double>& v);

// The centre selection of GeneDiverseConformations (src/GeneDiverseConformations.cpp:84-122)
// for conformers already generated and minimised: coors [nConf][nAtom][3] and their energies.
// Like the reference, coorsConformers is (re)allocated with new[] and receives the centres'
// coordinates in selection order; the return value is the number of centres.
int SelectDiverseConformations(int nConf, int nAtom, const double* coors,
                               const std::vector<double>& energy, int maxNumOfConformations,
                               double*& coorsConformers, double cutOff = 1.5);

// The search with a resident receptor: construct once per receptor grid set, then Search()
// per conformer batch. Results as the reference's minEnergyQuaternionsUsed / minEnergyIdx*.
class TranRotaSearch {
 public:
  TranRotaSearch(int xdim, int ydim, int zdim, float spacing, int numOfGridsUsed,
                 const float* usedGridValues, const cdk_opts* opts = nullptr);
  ~TranRotaSearch();
  TranRotaSearch(const TranRotaSearch&) = delete;
  TranRotaSearch& operator=(const TranRotaSearch&) = delete;
  // coors: [nConf][nAtom][3]; quaternions: [nConf][nQ][4]; slots from GetIdxOfAtomsForVdwRadius
  void Search(int nAtom, int nConf, const float* coors, const float* charges,
              const float* epsilons, const int* slots, int nQ, const float* quaternions,
              std::vector<float>& minEnergy, std::vector<int>& idxX, std::vector<int>& idxY,
              std::vector<int>& idxZ);
  cdk_ctx* context() { return ctx_; }

 private:
  cdk_ctx* ctx_ = nullptr;
};

}  // namespace cdk
