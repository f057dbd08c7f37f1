// ref_shim.cpp -- extern "C" entry points over the reference's OWN hot-path helpers.
//
// TEST INFRASTRUCTURE ONLY (oracle). oracle/Makefile compiles this file together with the
// unmodified reference sources (src/Rotate.cpp, src/QuaternionMultiply.cpp,
// src/QuaternionUniformSampling.cpp, src/FilterQuaternions.cpp, src/GetMinCoors.cpp,
// src/GetMaxCoors.cpp, src/GetIdxOfAtomsForVdwRadius.cpp, src/FillLigandGrid.cpp,
// src/ReadGrids.cpp) into oracle/_ref/libcdk_ref.so. Nothing here restates the reference:
// each shim only marshals plain arrays into the reference's own C++ signatures, so that the
// tests can pin the oracle restatement (oracle/cdk_oracle.cpp) against the reference itself.
#include <cstdlib>
#include <cstring>
#include <random>
#include <string>
#include <vector>

// GeneDiverseConformations.h declares the conformer generator on OpenBabel and OpenMM types
// (absent here); declaring the two classes lets the header's own sort_index template compile
namespace OpenBabel { class OBMol; }
namespace OpenMM { class System; }
#include <algorithm>
using std::sort;  // the header calls sort unqualified, as its includers bring it in
#include "GeneDiverseConformations.h"
#include "FillLigandGrid.h"
#include "FilterQuaternions.h"
#include "GetIdxOfAtomsForVdwRadius.h"
#include "GetMaxCoors.h"
#include "GetMinCoors.h"
#include "QuaternionUniformSampling.h"
#include "ReadGrids.h"
#include "Rotate.h"

extern "C" {

void ref_srand(unsigned s) { srand(s); }

// the reference's sort_index<float> (include/GeneDiverseConformations.h:9-20)
void ref_sort_index(int n, const float* v, long* out) {
  const std::vector<size_t> id = sort_index<float>(std::vector<float>(v, v + n));
  for (int i = 0; i < n; ++i) out[i] = (long)id[i];
}

void ref_rotate(const float* q, const float* v, float* out) { Rotate(q, v, out); }

// nConf successive QuaternionUniformSampling calls on one generator seeded with `seed`
// (the reference draws a fresh set per conformer from one std::mt19937_64).
void ref_quaternion_uniform_sampling(unsigned long long seed, int nConf, int nQ, float* out) {
  std::mt19937_64 gen(seed);
  float* q = nullptr;
  for (int c = 0; c < nConf; ++c) {
    QuaternionUniformSampling(gen, q, nQ);
    std::memcpy(out + (size_t)c * nQ * 4, q, sizeof(float) * 4 * nQ);
  }
  delete[] q;
}

int ref_filter_quaternions(const float* coor, int nAtom, int nQ, const float* quats, float gx,
                           float gy, float gz, int maxN, float* out) {
  std::vector<float> c(coor, coor + (size_t)nAtom * 3);
  std::vector<float> q(quats, quats + (size_t)nQ * 4);
  float* used = nullptr;
  int n = FilterQuaternions(c.data(), nAtom, nQ, q.data(), gx, gy, gz, maxN, used);
  std::memcpy(out, used, sizeof(float) * 4 * n);
  delete[] used;
  return n;
}

void ref_min_max_coors(int nQ, int nAtom, const float* coors, float* mn, float* mx) {
  std::vector<float> c(coors, coors + (size_t)nQ * nAtom * 3);
  GetMinCoors(nQ, nAtom, c.data(), mn);
  GetMaxCoors(nQ, nAtom, c.data(), mx);
}

// Runs GetIdxOfAtomsForVdwRadius; writes the used grid indices (ascending) and, per atom, the
// position of its grid among the used ones. Returns numOfVdwGridsUsed.
int ref_vdw_slots(int nAtoms, const float* radii, int nVdw, const float* gridRadii,
                  int* used_idx, int* atom_slot) {
  std::vector<float> r(radii, radii + nAtoms), g(gridRadii, gridRadii + nVdw);
  int nUsed = 0;
  std::vector<int> used;
  std::vector<std::vector<int> > byGrid(nVdw);
  GetIdxOfAtomsForVdwRadius(nAtoms, r.data(), nVdw, g.data(), nUsed, used, byGrid);
  for (int j = 0; j < nUsed; ++j) {
    used_idx[j] = used[j];
    for (int a : byGrid[used[j]]) atom_slot[a] = j;
  }
  return nUsed;
}

// FillLigandGrid on nQ rotations; the vdW bucketing comes from GetIdxOfAtomsForVdwRadius on
// the atom radii, exactly as the driver prepares it. out: [nQ][nUsed+1][X][Y][Z], pre-zeroed.
void ref_fill_ligand_grid(int nQ, int nAtom, const float* coors, const float* mincoors,
                          const float* charge, const float* eps, const float* radii,
                          int nVdw, const float* gridRadii, int X, int Y, int Z,
                          float spacing, float* out) {
  std::vector<float> r(radii, radii + nAtom), g(gridRadii, gridRadii + nVdw);
  int nUsed = 0;
  std::vector<int> used;
  std::vector<std::vector<int> > byGrid(nVdw);
  GetIdxOfAtomsForVdwRadius(nAtom, r.data(), nVdw, g.data(), nUsed, used, byGrid);
  std::vector<float> c(coors, coors + (size_t)nQ * nAtom * 3);
  std::vector<float> m(mincoors, mincoors + (size_t)nQ * 3);
  std::vector<float> q(charge, charge + nAtom), e(eps, eps + nAtom);
  FillLigandGrid(nQ, nAtom, c.data(), m.data(), q.data(), e.data(), nUsed, used, byGrid, X, Y,
                 Z, spacing, out);
}

// ReadGrids on a file; header ints [numGrids, x, y, z], floats [mid3, len3, spacing, k].
// Radii and values are copied into caller buffers when they are large enough.
int ref_read_grids(const char* path, int* hdr_i, float* hdr_f, float* radii, long radii_cap,
                   float* values, long values_cap) {
  int nG = 0, x = 0, y = 0, z = 0;
  float mx = 0, my = 0, mz = 0, lx = 0, ly = 0, lz = 0, sp = 0, rk = 0;
  float *rad = nullptr, *val = nullptr;
  ReadGrids(nG, x, y, z, mx, my, mz, lx, ly, lz, sp, rk, rad, val, std::string(path));
  if (rad == nullptr) return -1;
  hdr_i[0] = nG; hdr_i[1] = x; hdr_i[2] = y; hdr_i[3] = z;
  hdr_f[0] = mx; hdr_f[1] = my; hdr_f[2] = mz; hdr_f[3] = lx; hdr_f[4] = ly; hdr_f[5] = lz;
  hdr_f[6] = sp; hdr_f[7] = rk;
  long nr = nG - 1, nv = (long)nG * x * y * z;
  if (radii && nr <= radii_cap) std::memcpy(radii, rad, sizeof(float) * nr);
  if (values && nv <= values_cap) std::memcpy(values, val, sizeof(float) * nv);
  delete[] rad;
  delete[] val;
  return 0;
}

}  // extern "C"
