// reference_api.cpp -- host side of the search path with the reference's semantics.
//
// Everything here must reproduce the reference bit for bit where it decides something
// (which rotations are kept, which vdW grid an atom uses, the order poses are ranked in), so
// the float operation order of the rotation and the library calls that drive the random
// choices are the reference's. Built with -ffp-contract=off: the reference's x86-64 host
// build never fuses a multiply-add.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <random>
#include <sstream>
#include <string>
#include <thread>
#include <vector>

#include "../../../include/cdock_b200.h"
#include "../../../include/cdock_b200.hpp"

namespace cdk {
void set_error(const std::string& msg);

// Hamilton product; the expression order is part of the result (src/QuaternionMultiply.cpp:3-11)
void QuaternionMultiply(const float* const a, const float* const b, float* const r) {
  const float w = a[0] * b[0] - a[1] * b[1] - a[2] * b[2] - a[3] * b[3];
  const float x = a[0] * b[1] + a[1] * b[0] + a[2] * b[3] - a[3] * b[2];
  const float y = a[0] * b[2] - a[1] * b[3] + a[2] * b[0] + a[3] * b[1];
  const float z = a[0] * b[3] + a[1] * b[2] - a[2] * b[1] + a[3] * b[0];
  r[0] = w;
  r[1] = x;
  r[2] = y;
  r[3] = z;
}

// v' = q (0, v) q*  (src/Rotate.cpp:4-27)
void Rotate(const float* const q, const float* const v, float* const out) {
  const float pure[4] = {0.0f, v[0], v[1], v[2]};
  const float conj[4] = {q[0], -q[1], -q[2], -q[3]};
  float qv[4], qvq[4];
  QuaternionMultiply(q, pure, qv);
  QuaternionMultiply(qv, conj, qvq);
  std::memcpy(out, qvq + 1, 3 * sizeof(float));
}

namespace {
template <bool MAX>
void extreme_coors(int nQ, int nAtoms, const float* coors, float* out) {
  for (int i = 0; i < nQ; ++i) {
    const float* c = coors + (size_t)i * nAtoms * 3;
    float e[3] = {c[0], c[1], c[2]};
    for (int a = 1; a < nAtoms; ++a)
      for (int d = 0; d < 3; ++d) {
        const float v = c[a * 3 + d];
        if (MAX ? (v > e[d]) : (v < e[d])) e[d] = v;
      }
    std::memcpy(out + i * 3, e, sizeof(e));
  }
}
}  // namespace

// first-atom seeded, strict compares (src/GetMinCoors.cpp:4-29, src/GetMaxCoors.cpp:3-27)
void GetMinCoors(int nQ, int nAtoms, float* coors, float* mincoors) {
  extreme_coors<false>(nQ, nAtoms, coors, mincoors);
}
void GetMaxCoors(int nQ, int nAtoms, float* coors, float* maxcoors) {
  extreme_coors<true>(nQ, nAtoms, coors, maxcoors);
}

// Shoemake's uniform sampling of SO(3) from three U(0,1) doubles per rotation
// (src/QuaternionUniformSampling.cpp:5-24). Output reallocated as the reference does.
void QuaternionUniformSampling(std::mt19937_64& gen, float*& quaters, int nQuaters) {
  std::uniform_real_distribution<double> unit(0, 1);
  delete[] quaters;
  quaters = new float[4 * (size_t)nQuaters];
  for (int i = 0; i < nQuaters; ++i) {
    const double u1 = unit(gen);
    const double a = 2 * M_PI * unit(gen);
    const double b = 2 * M_PI * unit(gen);
    const double r1 = std::sqrt(1 - u1), r2 = std::sqrt(u1);
    float* q = quaters + 4 * (size_t)i;
    q[0] = (float)(std::cos(b) * r2);
    q[1] = (float)(std::sin(a) * r1);
    q[2] = (float)(std::cos(a) * r1);
    q[3] = (float)(std::sin(b) * r2);
  }
}

// Keeps rotations whose rotated bounding box is shorter than the grid on every axis; more
// than maxN survivors are thinned by std::random_shuffle on the process-wide rand() state
// (src/FilterQuaternions.cpp:11-83).
int FilterQuaternions(float* coor, int nAtom, int nQuater, float* quaternions, float gx,
                      float gy, float gz, int maxN, float*& used) {
  std::vector<int> kept;
  std::vector<float> rc((size_t)nAtom * 3);
  float mn[3], mx[3];
  for (int i = 0; i < nQuater; ++i) {
    for (int a = 0; a < nAtom; ++a) Rotate(quaternions + 4 * (size_t)i, coor + 3 * a, &rc[3 * a]);
    GetMinCoors(1, nAtom, rc.data(), mn);
    GetMaxCoors(1, nAtom, rc.data(), mx);
    const float lx = mx[0] - mn[0], ly = mx[1] - mn[1], lz = mx[2] - mn[2];
    if (lx < gx && ly < gy && lz < gz) kept.push_back(i);
  }
  int count = (int)kept.size();
  if (count > maxN) {
    count = maxN;
    std::random_shuffle(kept.begin(), kept.end());
  }
  delete[] used;
  used = new float[4 * (size_t)count];
  for (int i = 0; i < count; ++i)
    std::memcpy(used + 4 * (size_t)i, quaternions + 4 * (size_t)kept[i], 4 * sizeof(float));
  return count;
}

// Nearest probe radius, first minimum on ties; used grids in ascending order
// (src/GetIdxOfAtomsForVdwRadius.cpp:4-35). The distance is double, as in the reference.
void GetIdxOfAtomsForVdwRadius(int nAtoms, float* atomRadii, int numOfVdwGrids,
                               float* gridRadii, int& numOfVdwGridsUsed,
                               std::vector<int>& idxOfVdwUsed,
                               std::vector<std::vector<int> >& idxOfAtomVdwRadius) {
  for (int a = 0; a < nAtoms; ++a) {
    int best = 0;
    double bestDiff = std::abs(atomRadii[a] - gridRadii[0]);
    for (int g = 1; g < numOfVdwGrids; ++g) {
      const double d = std::abs(atomRadii[a] - gridRadii[g]);
      if (d < bestDiff) {
        bestDiff = d;
        best = g;
      }
    }
    idxOfAtomVdwRadius[best].push_back(a);
  }
  numOfVdwGridsUsed = 0;
  for (int g = 0; g < numOfVdwGrids; ++g)
    if (!idxOfAtomVdwRadius[g].empty()) {
      ++numOfVdwGridsUsed;
      idxOfVdwUsed.push_back(g);
    }
}

void FillLigandGrid(int nQuaternions, int nAtoms, float* coors, float* mincoors,
                    float* atomCharges, float* atomEpsilons, int numOfVdwGridsUsed,
                    std::vector<int> idxOfVdwUsed,
                    std::vector<std::vector<int> >& idxOfAtomVdwRadius, int xdim, int ydim,
                    int zdim, float spacing, float* ligandGridValues) {
  std::vector<int> slot(nAtoms, 0);
  for (int j = 0; j < numOfVdwGridsUsed; ++j)
    for (int a : idxOfAtomVdwRadius[idxOfVdwUsed[j]]) slot[a] = j;
  // the reference adds into the caller's (pre-zeroed) buffer; the GPU fill writes a fresh
  // grid and the sum is added here so that a non-zero caller buffer behaves the same
  const size_t total = (size_t)nQuaternions * (numOfVdwGridsUsed + 1) * xdim * ydim * zdim;
  std::vector<float> fresh(total);
  int rc = cdk_fill_ligand_grid(nQuaternions, nAtoms, coors, mincoors, atomCharges,
                                atomEpsilons, slot.data(), numOfVdwGridsUsed, xdim, ydim, zdim,
                                spacing, fresh.data());
  if (rc) {
    char msg[512];
    cdk_last_error(msg, sizeof msg);
    throw Error(rc, msg);
  }
  for (size_t i = 0; i < total; ++i)
    ligandGridValues[i] = (ligandGridValues[i] == 0.0f) ? fresh[i] : ligandGridValues[i] + fresh[i];
}

namespace {
// parse the reference's grid text format (src/ReadGrids.cpp:6-68)
int read_grids_impl(const std::string& path, int* hi, float* hf, std::vector<float>& radii,
                    std::vector<float>& values) {
  std::ifstream in(path);
  if (!in) {
    set_error("unable to open grid file: " + path);
    return CDK_ERR_IO;
  }
  std::string line;
  for (int i = 0; i < 3; ++i) std::getline(in, line);
  int nG = 0, x = 0, y = 0, z = 0;
  float f[8];
  if (!(in >> nG >> x >> y >> z >> f[0] >> f[1] >> f[2] >> f[3] >> f[4] >> f[5] >> f[6] >> f[7]) ||
      nG < 1 || x < 1 || y < 1 || z < 1) {
    set_error("malformed grid header: " + path);
    return CDK_ERR_IO;
  }
  radii.assign(nG - 1, 0.f);
  for (int i = 0; i < nG - 1; ++i)
    if (!(in >> radii[i])) {
      set_error("malformed grid radii: " + path);
      return CDK_ERR_IO;
    }
  std::getline(in, line);
  const size_t per = (size_t)x * y * z;
  values.assign(per * nG, 0.f);
  for (int g = 0; g < nG; ++g) {
    std::getline(in, line);  // per-grid header line
    for (size_t j = 0; j < per; ++j) {
      float a, b, c;
      if (!(in >> a >> b >> c >> values[g * per + j])) {
        set_error("grid file ended early: " + path);
        return CDK_ERR_IO;
      }
      std::getline(in, line);
    }
  }
  hi[0] = nG;
  hi[1] = x;
  hi[2] = y;
  hi[3] = z;
  std::memcpy(hf, f, sizeof f);
  return CDK_OK;
}
}  // namespace

void ReadGrids(int& numOfGrids, int& xdim, int& ydim, int& zdim, float& midx, float& midy,
               float& midz, float& xlen, float& ylen, float& zlen, float& spacing,
               float& restraint_k, float*& raddi, float*& values, std::string fileName) {
  int hi[4];
  float hf[8];
  std::vector<float> r, v;
  int rc = read_grids_impl(fileName, hi, hf, r, v);
  if (rc) {
    char msg[512];
    cdk_last_error(msg, sizeof msg);
    throw Error(rc, msg);
  }
  numOfGrids = hi[0];
  xdim = hi[1];
  ydim = hi[2];
  zdim = hi[3];
  midx = hf[0];
  midy = hf[1];
  midz = hf[2];
  xlen = hf[3];
  ylen = hf[4];
  zlen = hf[5];
  spacing = hf[6];
  restraint_k = hf[7];
  raddi = new float[r.size()];
  std::copy(r.begin(), r.end(), raddi);
  values = new float[v.size()];
  std::copy(v.begin(), v.end(), values);
}

std::vector<size_t> sort_index(const std::vector<float>& v) {
  std::vector<size_t> id(v.size());
  for (size_t i = 0; i < id.size(); ++i) id[i] = i;
  std::sort(id.begin(), id.end(), [&v](size_t a, size_t b) { return v[a] < v[b]; });
  return id;
}

std::vector<size_t> sort_index(const std::vector<double>& v) {
  std::vector<size_t> id(v.size());
  for (size_t i = 0; i < id.size(); ++i) id[i] = i;
  std::sort(id.begin(), id.end(), [&v](size_t a, size_t b) { return v[a] < v[b]; });
  return id;
}

int SelectDiverseConformations(int nConf, int nAtom, const double* coors,
                               const std::vector<double>& energy, int maxNumOfConformations,
                               double*& coorsConformers, double cutOff) {
  if ((int)energy.size() != nConf) throw Error(CDK_ERR_INVALID, "energy.size() != nConf");
  std::vector<int> centers((size_t)std::max(nConf, 1));
  int n = 0;
  const int rc = cdk_cluster_conformers(nConf, nAtom, coors, energy.data(), nullptr, cutOff,
                                        maxNumOfConformations, centers.data(), &n);
  if (rc) {
    char msg[512];
    cdk_last_error(msg, sizeof msg);
    throw Error(rc, msg);
  }
  delete[] coorsConformers;
  coorsConformers = new double[(size_t)n * nAtom * 3];
  for (int i = 0; i < n; ++i)
    std::memcpy(coorsConformers + (size_t)i * nAtom * 3, coors + (size_t)centers[i] * nAtom * 3,
                sizeof(double) * nAtom * 3);
  return n;
}

TranRotaSearch::TranRotaSearch(int xdim, int ydim, int zdim, float spacing, int K,
                               const float* grids, const cdk_opts* opts) {
  int rc = cdk_ctx_create(xdim, ydim, zdim, spacing, K, grids, opts, &ctx_);
  if (rc) {
    char msg[512];
    cdk_last_error(msg, sizeof msg);
    throw Error(rc, msg);
  }
}

TranRotaSearch::~TranRotaSearch() { cdk_ctx_destroy(ctx_); }

void TranRotaSearch::Search(int nAtom, int nConf, const float* coors, const float* charges,
                            const float* epsilons, const int* slots, int nQ,
                            const float* quaternions, std::vector<float>& minEnergy,
                            std::vector<int>& idxX, std::vector<int>& idxY,
                            std::vector<int>& idxZ) {
  const size_t nRot = (size_t)nConf * nQ;
  minEnergy.assign(nRot, INFINITY);
  std::vector<int> idx(nRot * 3, -1);
  int rc = cdk_search(ctx_, nAtom, nConf, coors, charges, epsilons, slots, nQ, quaternions,
                      minEnergy.data(), idx.data(), nullptr);
  if (rc) {
    char msg[512];
    cdk_last_error(msg, sizeof msg);
    throw Error(rc, msg);
  }
  idxX.resize(nRot);
  idxY.resize(nRot);
  idxZ.resize(nRot);
  for (size_t i = 0; i < nRot; ++i) {
    idxX[i] = idx[i * 3];
    idxY[i] = idx[i * 3 + 1];
    idxZ[i] = idx[i * 3 + 2];
  }
}

}  // namespace cdk

using namespace cdk;

extern "C" {

// Pose of a rotation at its best translation, as the driver rebuilds it
// (src/TranRotaConfSearchNoMini.cu:473-487): the rotated float coordinates widened to double,
// plus (gridMin - mincoor + idx * spacing) per axis, where gridMin = mid - len/2 (:149-151)
// and idx * spacing is the float product of the reference.
int cdk_pose_coordinates(int nAtom, const float* coor, const float* quat, const double* gridMin,
                         float spacing, const int* idx, double* out) {
  if (nAtom <= 0 || !coor || !quat || !gridMin || !idx || !out) {
    set_error("invalid argument");
    return CDK_ERR_INVALID;
  }
  std::vector<float> rc((size_t)nAtom * 3);
  for (int a = 0; a < nAtom; ++a) Rotate(quat, coor + 3 * a, &rc[3 * a]);
  float mn[3];
  GetMinCoors(1, nAtom, rc.data(), mn);
  for (int a = 0; a < nAtom; ++a)
    for (int d = 0; d < 3; ++d) {
      const float step = (float)idx[d] * spacing;
      out[3 * a + d] = (double)rc[3 * a + d] + (gridMin[d] - (double)mn[d] + (double)step);
    }
  return CDK_OK;
}

// sort_index over float minima (include/GeneDiverseConformations.h:9-20): std::sort of the
// indices with strict <, so ties come out in the order the reference's own call leaves them.
int cdk_sort_index(const float* v, long n, long* out) {
  if (n < 0 || (n > 0 && (!v || !out))) {
    set_error("invalid argument");
    return CDK_ERR_INVALID;
  }
  const std::vector<size_t> id = sort_index(std::vector<float>(v, v + n));
  for (long i = 0; i < n; ++i) out[i] = (long)id[i];
  return CDK_OK;
}

int cdk_quaternion_uniform_sampling(uint64_t seed, int nConf, int nQ, float* out) {
  if (!out || nConf < 0 || nQ < 0) {
    set_error("invalid argument");
    return CDK_ERR_INVALID;
  }
  std::mt19937_64 gen(seed);
  float* q = nullptr;
  for (int c = 0; c < nConf; ++c) {
    QuaternionUniformSampling(gen, q, nQ);
    std::memcpy(out + (size_t)c * nQ * 4, q, sizeof(float) * 4 * (size_t)nQ);
  }
  delete[] q;
  return CDK_OK;
}

int cdk_filter_quaternions(const float* coor, int nAtom, int nQ, const float* quats,
                           float gx, float gy, float gz, int maxN, float* out, int* count) {
  if (!coor || !quats || !out || !count || nAtom <= 0 || nQ < 0 || maxN < 0) {
    set_error("invalid argument");
    return CDK_ERR_INVALID;
  }
  std::vector<float> c(coor, coor + (size_t)nAtom * 3), q(quats, quats + (size_t)nQ * 4);
  float* used = nullptr;
  const int n = FilterQuaternions(c.data(), nAtom, nQ, q.data(), gx, gy, gz, maxN, used);
  std::memcpy(out, used, sizeof(float) * 4 * (size_t)n);
  delete[] used;
  *count = n;
  return CDK_OK;
}

int cdk_vdw_slots(int nAtom, const float* radii, int nVdw, const float* gridRadii, int* usedIdx,
                  int* atomSlot, int* nUsed) {
  if (!radii || !gridRadii || !usedIdx || !atomSlot || !nUsed || nAtom <= 0 || nVdw <= 0) {
    set_error("invalid argument");
    return CDK_ERR_INVALID;
  }
  std::vector<float> r(radii, radii + nAtom), g(gridRadii, gridRadii + nVdw);
  std::vector<int> used;
  std::vector<std::vector<int> > byGrid(nVdw);
  int n = 0;
  GetIdxOfAtomsForVdwRadius(nAtom, r.data(), nVdw, g.data(), n, used, byGrid);
  for (int j = 0; j < n; ++j) {
    usedIdx[j] = used[j];
    for (int a : byGrid[used[j]]) atomSlot[a] = j;
  }
  *nUsed = n;
  return CDK_OK;
}

int cdk_read_grids(const char* path, int* hdr_i, float* hdr_f, float* radii, long radii_cap,
                   float* values, long values_cap) {
  if (!path || !hdr_i || !hdr_f) {
    set_error("invalid argument");
    return CDK_ERR_INVALID;
  }
  std::vector<float> r, v;
  int rc = read_grids_impl(path, hdr_i, hdr_f, r, v);
  if (rc) return rc;
  if (radii && (long)r.size() <= radii_cap) std::copy(r.begin(), r.end(), radii);
  if (values && (long)v.size() <= values_cap) std::copy(v.begin(), v.end(), values);
  return CDK_OK;
}

int cdk_write_grids(const char* path, int nG, int x, int y, int z, const float* mid,
                    const float* len, float spacing, float rk, const float* radii,
                    const float* values) {
  if (!path || !mid || !len || !values || nG < 1 || x < 1 || y < 1 || z < 1 ||
      (nG > 1 && !radii)) {
    set_error("invalid argument");
    return CDK_ERR_INVALID;
  }
  FILE* f = std::fopen(path, "w");
  if (!f) {
    set_error(std::string("cannot write ") + path);
    return CDK_ERR_IO;
  }
  std::fprintf(f, "* synthetic receptor potential grids\n* written by cdock_b200\n*\n");
  std::fprintf(f, "%d %d %d %d %.9g %.9g %.9g %.9g %.9g %.9g %.9g %.9g\n", nG, x, y, z, mid[0],
               mid[1], mid[2], len[0], len[1], len[2], spacing, rk);
  for (int i = 0; i < nG - 1; ++i) std::fprintf(f, "%.9g%s", radii[i], i + 1 < nG - 1 ? " " : "");
  std::fprintf(f, "\n");
  const size_t per = (size_t)x * y * z;
  for (int g = 0; g < nG; ++g) {
    std::fprintf(f, "grid %d\n", g);
    for (int i = 0; i < x; ++i)
      for (int j = 0; j < y; ++j)
        for (int k = 0; k < z; ++k)
          std::fprintf(f, "%d %d %d %.9g\n", i, j, k, values[g * per + ((size_t)i * y + j) * z + k]);
  }
  const bool ok = std::fclose(f) == 0;
  if (!ok) {
    set_error(std::string("write failed: ") + path);
    return CDK_ERR_IO;
  }
  return CDK_OK;
}

// Soft-core capped Lennard-Jones per probe radius and a Coulomb grid with eps(r) = 4r:
//   vdW_p(g)  = sum_a sqrtEps_a * [(Rmin/d)^12 - 2 (Rmin/d)^6],  Rmin = r_a + r_p, d >= 0.5 Rmin,
//               then min(., vdwCap)
//   elec(g)   = sum_a 332.0716 q_a / (4 d^2),  d >= 0.5 A, then clamped to [-elecCap, elecCap]
// atoms beyond `cutoff` are skipped (a cell list of cutoff-sized cells).
int cdk_synth_receptor_grids(int n, float spacing, const float* origin, int nAtom,
                             const float* xyz, const float* radius, const float* sqrtEps,
                             const float* charge, int nVdw, const float* probe, float vdwCap,
                             float elecCap, float cutoff, float* out) {
  if (n <= 0 || nAtom < 0 || nVdw < 0 || !origin || !out || (nAtom && (!xyz || !radius || !sqrtEps || !charge)) ||
      (nVdw && !probe) || !(cutoff > 0)) {
    set_error("invalid argument");
    return CDK_ERR_INVALID;
  }
  const size_t N = (size_t)n * n * n;
  // cell list
  float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
  for (int a = 0; a < nAtom; ++a)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], xyz[a * 3 + d]);
      hi[d] = std::max(hi[d], xyz[a * 3 + d]);
    }
  int nc[3];
  for (int d = 0; d < 3; ++d) nc[d] = nAtom ? std::max(1, (int)std::ceil((hi[d] - lo[d]) / cutoff) + 1) : 1;
  std::vector<std::vector<int> > cells((size_t)nc[0] * nc[1] * nc[2]);
  for (int a = 0; a < nAtom; ++a) {
    int c[3];
    for (int d = 0; d < 3; ++d) c[d] = std::min(nc[d] - 1, (int)((xyz[a * 3 + d] - lo[d]) / cutoff));
    cells[((size_t)c[0] * nc[1] + c[1]) * nc[2] + c[2]].push_back(a);
  }
  const double cut2 = (double)cutoff * cutoff;
  auto work = [&](int i0, int i1) {
    std::vector<double> acc(nVdw + 1);
    for (int i = i0; i < i1; ++i)
      for (int j = 0; j < n; ++j)
        for (int k = 0; k < n; ++k) {
          const double p[3] = {origin[0] + (double)i * spacing, origin[1] + (double)j * spacing,
                               origin[2] + (double)k * spacing};
          std::fill(acc.begin(), acc.end(), 0.0);
          int c[3];
          // cells beyond [-2, nc+1] have no occupied neighbours; clamping keeps the
          // conversion to int defined for points far from every atom
          for (int d = 0; d < 3; ++d)
            c[d] = (int)std::floor(std::min(std::max((p[d] - lo[d]) / cutoff, -2.0), nc[d] + 1.0));
          for (int cx = c[0] - 1; cx <= c[0] + 1; ++cx)
            for (int cy = c[1] - 1; cy <= c[1] + 1; ++cy)
              for (int cz = c[2] - 1; cz <= c[2] + 1; ++cz) {
                if (cx < 0 || cy < 0 || cz < 0 || cx >= nc[0] || cy >= nc[1] || cz >= nc[2]) continue;
                for (int a : cells[((size_t)cx * nc[1] + cy) * nc[2] + cz]) {
                  const double dx = p[0] - xyz[a * 3], dy = p[1] - xyz[a * 3 + 1],
                               dz = p[2] - xyz[a * 3 + 2];
                  const double d2 = dx * dx + dy * dy + dz * dz;
                  if (d2 > cut2) continue;
                  for (int v = 0; v < nVdw; ++v) {
                    const double rmin = (double)radius[a] + probe[v];
                    const double dd2 = std::max(d2, 0.25 * rmin * rmin);
                    const double s2 = rmin * rmin / dd2, s6 = s2 * s2 * s2;
                    acc[v] += (double)sqrtEps[a] * (s6 * s6 - 2.0 * s6);
                  }
                  acc[nVdw] += 332.0716 * (double)charge[a] / (4.0 * std::max(d2, 0.25));
                }
              }
          const size_t g = ((size_t)i * n + j) * n + k;
          for (int v = 0; v < nVdw; ++v) out[v * N + g] = (float)std::min(acc[v], (double)vdwCap);
          out[nVdw * N + g] = (float)std::max(-(double)elecCap, std::min(acc[nVdw], (double)elecCap));
        }
  };
  int nt = (int)std::max(1u, std::thread::hardware_concurrency());
  nt = std::min(nt, n);
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; ++t) {
    const int i0 = (int)((long)n * t / nt), i1 = (int)((long)n * (t + 1) / nt);
    pool.emplace_back(work, i0, i1);
  }
  for (auto& th : pool) th.join();
  return CDK_OK;
}

}  // extern "C"
