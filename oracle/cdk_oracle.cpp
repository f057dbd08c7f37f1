// cdk_oracle.cpp -- CPU restatement of CDOCKER's FFT translational-rotational search path.
//
// TEST INFRASTRUCTURE ONLY. This file is the oracle: it is linked by tests/, by
// __graft_entry__.smoke() and by bench.py's cpu_baseline / reference legs as the checker.
// The product (cdocker_b200/) never links, loads or calls it.
//
// Every function restates one step of the reference's algorithm, in the reference's
// arithmetic (float vs double, operation order, loop order, tie rules), citing the
// reference file:line it follows. Built with -ffp-contract=off so that no multiply-add is
// fused, as in the reference's x86-64 host build. Parity is pinned by comparing these
// functions with the reference's own helpers compiled from its sources (oracle/_ref) and by
// the FP64 FFT form in oracle/oracle.py.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <random>
#include <thread>
#include <vector>

namespace {

// Hamilton product, one float op at a time in the reference's order
// (src/QuaternionMultiply.cpp:3-11).
inline void qmul(const float* l, const float* r, float* o) {
  o[0] = l[0] * r[0] - l[1] * r[1] - l[2] * r[2] - l[3] * r[3];
  o[1] = l[0] * r[1] + l[1] * r[0] + l[2] * r[3] - l[3] * r[2];
  o[2] = l[0] * r[2] - l[1] * r[3] + l[2] * r[0] + l[3] * r[1];
  o[3] = l[0] * r[3] + l[1] * r[2] - l[2] * r[1] + l[3] * r[0];
}

// v' = q (0,v) q*  (src/Rotate.cpp:4-27).
inline void rotate(const float* q, const float* v, float* out) {
  float qc[4] = {q[0], -q[1], -q[2], -q[3]};
  float qv[4] = {0.0f, v[0], v[1], v[2]};
  float t1[4], t2[4];
  qmul(q, qv, t1);
  qmul(t1, qc, t2);
  out[0] = t2[1];
  out[1] = t2[2];
  out[2] = t2[3];
}

// Per-axis min / max over atoms, first atom as the seed, strict compares
// (src/GetMinCoors.cpp:4-29, src/GetMaxCoors.cpp:3-27).
inline void minmax(int nAtom, const float* c, float* mn, float* mx) {
  for (int d = 0; d < 3; ++d) mn[d] = mx[d] = c[d];
  for (int a = 1; a < nAtom; ++a)
    for (int d = 0; d < 3; ++d) {
      if (c[a * 3 + d] < mn[d]) mn[d] = c[a * 3 + d];
      if (c[a * 3 + d] > mx[d]) mx[d] = c[a * 3 + d];
    }
}

// One atom's trilinear (cloud-in-cell) spread into a grid of dims (X,Y,Z), z fastest,
// with the reference's mixed double/float arithmetic (src/FillLigandGrid.cpp:24-66):
// cell index and ratios in double, `index * spacing` in float, weight in double, and
// each accumulation rounded back to the float grid.
inline void spread_atom(double x, double y, double z, const float* mn, float spacing,
                        double scale, int Y, int Z, float* grid) {
  int xi = int((x - mn[0]) / spacing);
  int yi = int((y - mn[1]) / spacing);
  int zi = int((z - mn[2]) / spacing);
  double xr = ((x - mn[0]) - (double)((float)xi * spacing)) / spacing;
  double yr = ((y - mn[1]) - (double)((float)yi * spacing)) / spacing;
  double zr = ((z - mn[2]) - (double)((float)zi * spacing)) / spacing;
  const double wx[2] = {1 - xr, xr}, wy[2] = {1 - yr, yr}, wz[2] = {1 - zr, zr};
  // corner order 000,001,010,011,100,101,110,111 (x, y, z bits), as in the reference
  for (int c = 0; c < 8; ++c) {
    int dx = (c >> 2) & 1, dy = (c >> 1) & 1, dz = c & 1;
    size_t idx = ((size_t)(xi + dx) * Y + (yi + dy)) * Z + (zi + dz);
    double w = scale * wx[dx] * wy[dy] * wz[dz];
    grid[idx] = (float)((double)grid[idx] + w);
  }
}

// Nearest probe radius per atom, first minimum on ties (strict <), then the used vdW grids in
// ascending grid order; returns the count (src/GetIdxOfAtomsForVdwRadius.cpp:4-35).
// atom_slot[a] = position of the atom's grid among the used grids.
int vdw_slots(int nAtoms, const float* radii, int nVdw, const float* gridRadii,
              int* used_idx, int* atom_slot) {
  std::vector<int> gidx(nAtoms);
  std::vector<int> count(nVdw, 0);
  for (int i = 0; i < nAtoms; ++i) {
    int idx = 0;
    double diff = std::abs(radii[i] - gridRadii[0]);
    for (int j = 1; j < nVdw; ++j)
      if (std::abs(radii[i] - gridRadii[j]) < diff) {
        idx = j;
        diff = std::abs(radii[i] - gridRadii[j]);
      }
    gidx[i] = idx;
    count[idx]++;
  }
  int nUsed = 0;
  std::vector<int> pos(nVdw, -1);
  for (int j = 0; j < nVdw; ++j)
    if (count[j] > 0) {
      pos[j] = nUsed;
      used_idx[nUsed++] = j;
    }
  for (int i = 0; i < nAtoms; ++i) atom_slot[i] = pos[gidx[i]];
  return nUsed;
}

// Fill one rotation's K = nVdwUsed+1 grids: vdW grids by slot in atom order, then the elec grid
// with every atom (src/FillLigandGrid.cpp:18-66 then :71-118).
void fill_one(int nAtom, const float* coors, const float* mn, const float* charge,
              const float* eps, const int* slot, int nVdwUsed, int X, int Y, int Z,
              float spacing, float* out) {
  size_t N = (size_t)X * Y * Z;
  for (int j = 0; j < nVdwUsed; ++j)
    for (int m = 0; m < nAtom; ++m)
      if (slot[m] == j)
        spread_atom(coors[m * 3 + 0], coors[m * 3 + 1], coors[m * 3 + 2], mn, spacing,
                    (double)std::sqrt(eps[m]), Y, Z, out + (size_t)j * N);
  for (int m = 0; m < nAtom; ++m)
    spread_atom(coors[m * 3 + 0], coors[m * 3 + 1], coors[m * 3 + 2], mn, spacing,
                (double)charge[m], Y, Z, out + (size_t)nVdwUsed * N);
}

// Runs body(r) for r in [0, total) on nthreads host threads (dynamic, one item at a time).
template <class F>
void parallel_for(long total, int nthreads, F body) {
  if (nthreads <= 0) nthreads = (int)std::thread::hardware_concurrency();
  if (nthreads <= 1 || total <= 1) {
    for (long r = 0; r < total; ++r) body(r);
    return;
  }
  std::atomic<long> next(0);
  std::vector<std::thread> pool;
  for (int t = 0; t < nthreads; ++t)
    pool.emplace_back([&]() {
      for (long r = next++; r < total; r = next++) body(r);
    });
  for (auto& th : pool) th.join();
}

}  // namespace

extern "C" {

void orc_rotate(const float* q, const float* v, float* out) { rotate(q, v, out); }

// Shoemake uniform quaternions drawn from one mt19937_64 stream, nConf blocks of nQ in turn,
// as the driver redraws per conformer from a shared generator
// (src/QuaternionUniformSampling.cpp:5-24; src/TranRotaConfSearchNoMini.cu:203-204, :323).
void orc_sample_quaternions(unsigned long long seed, int nConf, int nQ, float* out) {
  std::mt19937_64 gen(seed);
  std::uniform_real_distribution<double> u(0, 1);
  for (long i = 0; i < (long)nConf * nQ; ++i) {
    double s = u(gen);
    double sig1 = std::sqrt(1 - s), sig2 = std::sqrt(s);
    double t1 = 2 * M_PI * u(gen);
    double t2 = 2 * M_PI * u(gen);
    out[i * 4 + 0] = (float)(std::cos(t2) * sig2);
    out[i * 4 + 1] = (float)(std::sin(t1) * sig1);
    out[i * 4 + 2] = (float)(std::cos(t1) * sig1);
    out[i * 4 + 3] = (float)(std::sin(t2) * sig2);
  }
}

void orc_srand(unsigned s) { srand(s); }

// Synthetic receptor potential grids for the benchmark inputs of the reference arm (no
// reference counterpart: the reference reads CHARMM-written grids, src/ReadGrids.cpp:6-68).
// Same definition and operation order as the product's host generator, so the arm searches the
// same grids without loading the product library:
//   vdW_p(g) = min(sum_a sqrtEps_a [(Rmin/d)^12 - 2 (Rmin/d)^6], vdwCap), Rmin = r_a + r_p,
//              d^2 clamped below at (Rmin/2)^2;
//   elec(g)  = clamp(sum_a 332.0716 q_a / (4 max(d^2, 0.25)), +-elecCap);
// atoms within `cutoff` of the point, visited cell by cell (cells of edge `cutoff`, the 27
// around the point's cell in x, y, z order, atoms of a cell in index order).
void orc_synth_receptor_grids(int n, float spacing, const float* origin, int nAtom,
                              const float* xyz, const float* radius, const float* sqrtEps,
                              const float* charge, int nVdw, const float* probe, float vdwCap,
                              float elecCap, float cutoff, float* out) {
  const size_t N = (size_t)n * n * n;
  float lo[3] = {1e30f, 1e30f, 1e30f}, hi[3] = {-1e30f, -1e30f, -1e30f};
  for (int a = 0; a < nAtom; ++a)
    for (int d = 0; d < 3; ++d) {
      lo[d] = std::min(lo[d], xyz[a * 3 + d]);
      hi[d] = std::max(hi[d], xyz[a * 3 + d]);
    }
  int nc[3];
  for (int d = 0; d < 3; ++d) nc[d] = nAtom ? std::max(1, (int)std::ceil((hi[d] - lo[d]) / cutoff) + 1) : 1;
  std::vector<std::vector<int>> cells((size_t)nc[0] * nc[1] * nc[2]);
  for (int a = 0; a < nAtom; ++a) {
    int c[3];
    for (int d = 0; d < 3; ++d) c[d] = std::min(nc[d] - 1, (int)((xyz[a * 3 + d] - lo[d]) / cutoff));
    cells[((size_t)c[0] * nc[1] + c[1]) * nc[2] + c[2]].push_back(a);
  }
  const double cut2 = (double)cutoff * cutoff;
  auto plane = [&](int i) {
    std::vector<double> acc(nVdw + 1);
    for (int j = 0; j < n; ++j)
      for (int k = 0; k < n; ++k) {
        const double p[3] = {origin[0] + (double)i * spacing, origin[1] + (double)j * spacing,
                             origin[2] + (double)k * spacing};
        std::fill(acc.begin(), acc.end(), 0.0);
        int c[3];
        for (int d = 0; d < 3; ++d)
          c[d] = (int)std::floor(std::min(std::max((p[d] - lo[d]) / cutoff, -2.0), nc[d] + 1.0));
        for (int cx = c[0] - 1; cx <= c[0] + 1; ++cx)
          for (int cy = c[1] - 1; cy <= c[1] + 1; ++cy)
            for (int cz = c[2] - 1; cz <= c[2] + 1; ++cz) {
              if (cx < 0 || cy < 0 || cz < 0 || cx >= nc[0] || cy >= nc[1] || cz >= nc[2]) continue;
              for (int a : cells[((size_t)cx * nc[1] + cy) * nc[2] + cz]) {
                const double dx = p[0] - xyz[a * 3], dy = p[1] - xyz[a * 3 + 1], dz = p[2] - xyz[a * 3 + 2];
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
  const int nt = std::max(1, std::min(n, (int)std::thread::hardware_concurrency()));
  std::atomic<int> next(0);
  std::vector<std::thread> pool;
  for (int t = 0; t < nt; ++t)
    pool.emplace_back([&] {
      for (int i = next++; i < n; i = next++) plane(i);
    });
  for (auto& th : pool) th.join();
}

// Keep q whose rotated bounding box is shorter than the grid on every axis; when more than
// maxN pass, std::random_shuffle (rand()-driven) the kept indices and take the first maxN
// (src/FilterQuaternions.cpp:11-83). Returns the count; out holds count*4 floats.
int orc_filter_quaternions(const float* coor, int nAtom, int nQ, const float* q, float gx,
                           float gy, float gz, int maxN, float* out) {
  std::vector<float> rc((size_t)nAtom * 3);
  std::vector<int> keep;
  for (int i = 0; i < nQ; ++i) {
    for (int a = 0; a < nAtom; ++a) rotate(q + i * 4, coor + a * 3, &rc[a * 3]);
    float mn[3], mx[3];
    minmax(nAtom, rc.data(), mn, mx);
    float lx = mx[0] - mn[0], ly = mx[1] - mn[1], lz = mx[2] - mn[2];
    if (lx < gx && ly < gy && lz < gz) keep.push_back(i);
  }
  int n = (int)keep.size();
  if (n > maxN) {
    n = maxN;
    std::random_shuffle(keep.begin(), keep.end());
  }
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < 4; ++d) out[i * 4 + d] = q[keep[i] * 4 + d];
  return n;
}

int orc_vdw_slots(int nAtoms, const float* radii, int nVdw, const float* gridRadii,
                  int* used_idx, int* atom_slot) {
  return vdw_slots(nAtoms, radii, nVdw, gridRadii, used_idx, atom_slot);
}

// Rotate conformer atoms by each quaternion and report per-rotation min corner and lengths
// (src/TranRotaConfSearchNoMini.cu:352-372).
void orc_rotate_bbox(int nAtom, const float* coor, int nQ, const float* q, float* rot_out,
                     float* min_out, float* len_out) {
  for (int i = 0; i < nQ; ++i) {
    float* rc = rot_out + (size_t)i * nAtom * 3;
    for (int a = 0; a < nAtom; ++a) rotate(q + i * 4, coor + a * 3, rc + a * 3);
    float mn[3], mx[3];
    minmax(nAtom, rc, mn, mx);
    for (int d = 0; d < 3; ++d) {
      min_out[i * 3 + d] = mn[d];
      len_out[i * 3 + d] = mx[d] - mn[d];
    }
  }
}

// Dense fill of nQ rotations into [nQ][K][X][Y][Z] (pre-zeroed), rotated coords and min
// corners given (src/FillLigandGrid.cpp:7-120).
void orc_fill_ligand_grid(int nQ, int nAtom, const float* coors, const float* mincoors,
                          const float* charge, const float* eps, const int* slot,
                          int nVdwUsed, int X, int Y, int Z, float spacing, float* out) {
  size_t per = (size_t)(nVdwUsed + 1) * X * Y * Z;
  for (int i = 0; i < nQ; ++i)
    fill_one(nAtom, coors + (size_t)i * nAtom * 3, mincoors + i * 3, charge, eps, slot,
             nVdwUsed, X, Y, Z, spacing, out + i * per);
}

// Translation window bound per axis: n - int(len/h) - 2, with the float division of the
// reference (src/TranRotaConfSearchNoMini.cu:446-450; the z bound there reads ydim, which is
// the same number for the cubic grids this path supports).
int orc_window(int n, float len, float spacing) { return n - int(len / spacing) - 2; }

// Direct-correlation search, cpuNaive's algorithm (src/cpuNaive.cpp:82-216) per rotation:
// rotate, bounding box, a ligand-sized box of dim int(len/h)+2 filled with FillLigandGrid's
// arithmetic, then E[i,j,k] = sum_l sum_m,n,o Lig[l,m,n,o] * P[l,m+i,n+j,o+k] over the
// window [0, n - dim) per axis, in cpuNaive's loop order. First minimum in x-major order,
// strict < (src/TranRotaConfSearchNoMini.cu:441-464). Empty windows give +inf and -1.
//   prec = 0: float accumulation (cpuNaive); prec = 1: double accumulation (FP64 oracle).
//   dense = 1 walks every box cell as cpuNaive does; dense = 0 skips zero cells, which adds
//   the same nonzero terms in the same order (adding +0.0 leaves a sum unchanged).
// grids: [K][X][Y][Z] (z fastest); K = nVdwUsed + 1, elec last. Conformer c of nConf owns
// quaternions [c*nQ, (c+1)*nQ).
void orc_search_direct(int X, int Y, int Z, float spacing, int K, const float* grids,
                       int nAtom, int nConf, const float* coor, const float* charge,
                       const float* eps, const int* slot, int nQ, const float* q, int prec,
                       int dense, int nthreads, float* minE, int* idx, double* minE64) {
  const long total = (long)nConf * nQ;
  const int nVdwUsed = K - 1;
  parallel_for(total, nthreads, [&](long r) {
    const float* cc = coor + (r / nQ) * (size_t)nAtom * 3;
    std::vector<float> rc((size_t)nAtom * 3);
    for (int a = 0; a < nAtom; ++a) rotate(q + r * 4, cc + a * 3, &rc[a * 3]);
    float mn[3], mx[3];
    minmax(nAtom, rc.data(), mn, mx);
    float len[3] = {mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]};
    int dl[3], W[3];
    const int dims[3] = {X, Y, Z};
    for (int d = 0; d < 3; ++d) {
      dl[d] = int(len[d] / spacing) + 2;
      W[d] = dims[d] - dl[d];
    }
    minE[r] = INFINITY;
    if (minE64) minE64[r] = INFINITY;
    idx[r * 3 + 0] = idx[r * 3 + 1] = idx[r * 3 + 2] = -1;
    if (W[0] <= 0 || W[1] <= 0 || W[2] <= 0) return;
    // the fill can touch cell int(len/h)+1 on an axis when double rounding lands on an integer,
    // so the box gets one cell of slack (always zero otherwise).
    const int bx = dl[0] + 1, by = dl[1] + 1, bz = dl[2] + 1;
    const size_t nb = (size_t)bx * by * bz;
    std::vector<float> box((size_t)K * nb, 0.0f);
    fill_one(nAtom, rc.data(), mn, charge, eps, slot, nVdwUsed, bx, by, bz, spacing,
             box.data());
    // nonzero list in cpuNaive order (l, m, n, o)
    std::vector<int> nzl, nzo;
    std::vector<float> nzv;
    for (int l = 0; l < K; ++l)
      for (int m = 0; m < bx; ++m)
        for (int n = 0; n < by; ++n)
          for (int o = 0; o < bz; ++o) {
            float v = box[l * nb + ((size_t)m * by + n) * bz + o];
            if (dense || v != 0.0f) {
              nzl.push_back(l);
              nzo.push_back((m * Y + n) * Z + o);
              nzv.push_back(v);
            }
          }
    const size_t N = (size_t)X * Y * Z;
    float best = INFINITY;
    double best64 = INFINITY;
    int bi = -1, bj = -1, bk = -1;
    for (int i = 0; i < W[0]; ++i)
      for (int j = 0; j < W[1]; ++j)
        for (int k = 0; k < W[2]; ++k) {
          const size_t t = ((size_t)i * Y + j) * Z + k;
          if (prec == 0) {
            float e = 0.0f;
            for (size_t s = 0; s < nzv.size(); ++s)
              e = e + nzv[s] * grids[nzl[s] * N + nzo[s] + t];
            if (e < best) { best = e; best64 = e; bi = i; bj = j; bk = k; }
          } else {
            double e = 0.0;
            for (size_t s = 0; s < nzv.size(); ++s)
              e = e + (double)nzv[s] * (double)grids[nzl[s] * N + nzo[s] + t];
            if (e < best64) { best64 = e; best = (float)e; bi = i; bj = j; bk = k; }
          }
        }
    minE[r] = best;
    if (minE64) minE64[r] = best64;
    idx[r * 3 + 0] = bi;
    idx[r * 3 + 1] = bj;
    idx[r * 3 + 2] = bk;
  });
}

// Full energy map of one rotation over its window, double accumulation: used for near-tie
// analysis (second-best value) in the parity tests. out: [W0][W1][W2]; returns W via w_out.
void orc_energy_map(int X, int Y, int Z, float spacing, int K, const float* grids, int nAtom,
                    const float* coor, const float* charge, const float* eps,
                    const int* slot, const float* q, int* w_out, double* out, long cap) {
  std::vector<float> rc((size_t)nAtom * 3);
  for (int a = 0; a < nAtom; ++a) rotate(q, coor + a * 3, &rc[a * 3]);
  float mn[3], mx[3];
  minmax(nAtom, rc.data(), mn, mx);
  const int dims[3] = {X, Y, Z};
  int dl[3], W[3];
  for (int d = 0; d < 3; ++d) {
    dl[d] = int((mx[d] - mn[d]) / spacing) + 2;
    W[d] = dims[d] - dl[d];
    w_out[d] = W[d];
  }
  if (W[0] <= 0 || W[1] <= 0 || W[2] <= 0) return;
  if ((long)W[0] * W[1] * W[2] > cap) { w_out[0] = -1; return; }
  const int bx = dl[0] + 1, by = dl[1] + 1, bz = dl[2] + 1;
  const size_t nb = (size_t)bx * by * bz;
  std::vector<float> box((size_t)K * nb, 0.0f);
  fill_one(nAtom, rc.data(), mn, charge, eps, slot, K - 1, bx, by, bz, spacing, box.data());
  const size_t N = (size_t)X * Y * Z;
  for (int i = 0; i < W[0]; ++i)
    for (int j = 0; j < W[1]; ++j)
      for (int k = 0; k < W[2]; ++k) {
        const size_t t = ((size_t)i * Y + j) * Z + k;
        double e = 0.0;
        for (int l = 0; l < K; ++l)
          for (int m = 0; m < bx; ++m)
            for (int n = 0; n < by; ++n)
              for (int o = 0; o < bz; ++o) {
                float v = box[l * nb + ((size_t)m * by + n) * bz + o];
                if (v != 0.0f) e += (double)v * grids[l * N + (m * Y + n) * Z + o + t];
              }
        out[((size_t)i * W[1] + j) * W[2] + k] = e;
      }
}

// sort_index: std::sort of indices by value, strict < (include/GeneDiverseConformations.h:9-20).
void orc_sort_index(int n, const float* v, long* out) {
  std::vector<size_t> id(n);
  for (int i = 0; i < n; ++i) id[i] = i;
  std::sort(id.begin(), id.end(), [&](size_t a, size_t b) { return v[a] < v[b]; });
  for (int i = 0; i < n; ++i) out[i] = (long)id[i];
}

}  // extern "C"

// ---------------------------------------------------------------------------------------------
// Diverse-conformer selection (src/GeneDiverseConformations.cpp:84-111): greedy leader
// clustering in energy order (sort_index<double>, include/GeneDiverseConformations.h:9-20) with
// RMSD <= cutOff (1.5) after optimal superposition. OBAlign (OpenBabel, absent here) supplies the
// reference's RMSD; this restatement computes the minimum RMSD over rotations of the centred
// atom sets, in double, by Horn's quaternion key matrix and Newton's method on its
// characteristic polynomial, one operation at a time in a fixed order (no contraction). The
// same recipe, op for op, is what the library's GPU kernels evaluate.
namespace {

void center_conf(const double* p, const std::vector<int>& sel, std::vector<double>& X, double& G) {
  const int n = (int)sel.size();
  double s[3] = {0.0, 0.0, 0.0};
  for (int i = 0; i < n; ++i)
    for (int d = 0; d < 3; ++d) s[d] = s[d] + p[sel[i] * 3 + d];
  double m[3];
  for (int d = 0; d < 3; ++d) m[d] = s[d] / (double)n;
  X.assign((size_t)n * 3, 0.0);
  double g = 0.0;
  for (int i = 0; i < n; ++i) {
    double v[3];
    for (int d = 0; d < 3; ++d) {
      v[d] = p[sel[i] * 3 + d] - m[d];
      X[(size_t)i * 3 + d] = v[d];
    }
    g = g + ((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]);
  }
  G = g;
}

double qcp_rmsd(const double* A, double Ga, const double* B, double Gb, int n) {
  double S[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
  for (int a = 0; a < n; ++a)
    for (int p = 0; p < 3; ++p)
      for (int q = 0; q < 3; ++q) S[p * 3 + q] = S[p * 3 + q] + A[a * 3 + p] * B[a * 3 + q];
  const double Sxx = S[0], Sxy = S[1], Sxz = S[2], Syx = S[3], Syy = S[4], Syz = S[5],
               Szx = S[6], Szy = S[7], Szz = S[8];
  double N[4][4];
  N[0][0] = (Sxx + Syy) + Szz;
  N[0][1] = Syz - Szy;
  N[0][2] = Szx - Sxz;
  N[0][3] = Sxy - Syx;
  N[1][1] = (Sxx - Syy) - Szz;
  N[1][2] = Sxy + Syx;
  N[1][3] = Szx + Sxz;
  N[2][2] = (Syy - Sxx) - Szz;
  N[2][3] = Syz + Szy;
  N[3][3] = (Szz - Sxx) - Syy;
  N[1][0] = N[0][1];
  N[2][0] = N[0][2];
  N[3][0] = N[0][3];
  N[2][1] = N[1][2];
  N[3][1] = N[1][3];
  N[3][2] = N[2][3];
  double p2 = 0.0;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) p2 = p2 + N[i][j] * N[i][j];
  double p3 = 0.0;
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) {
      const double n2 = ((N[i][0] * N[0][j] + N[i][1] * N[1][j]) + N[i][2] * N[2][j]) + N[i][3] * N[3][j];
      p3 = p3 + n2 * N[j][i];
    }
  auto mA = [&](int j, int k) { return N[0][j] * N[1][k] - N[0][k] * N[1][j]; };
  auto mB = [&](int j, int k) { return N[2][j] * N[3][k] - N[2][k] * N[3][j]; };
  double det = mA(0, 1) * mB(2, 3) - mA(0, 2) * mB(1, 3);
  det = det + mA(0, 3) * mB(1, 2);
  det = det + mA(1, 2) * mB(0, 3);
  det = det - mA(1, 3) * mB(0, 2);
  det = det + mA(2, 3) * mB(0, 1);
  const double c2 = -(p2 * 0.5), c1 = -(p3 / 3.0), c0 = det;
  double l = (Ga + Gb) * 0.5;
  for (int it = 0; it < 50; ++it) {
    const double l2 = l * l;
    const double P = ((l2 + c2) * l + c1) * l + c0;
    const double dP = (4.0 * l2 + 2.0 * c2) * l + c1;
    if (dP == 0.0) break;
    const double ln = l - P / dP;
    if (std::fabs(ln - l) <= 1e-11 * std::fabs(ln)) {
      l = ln;
      break;
    }
    l = ln;
  }
  double e = ((Ga + Gb) - 2.0 * l) / (double)n;
  if (!(e > 0.0)) e = 0.0;
  return std::sqrt(e);
}

std::vector<int> mask_sel(int nAtom, const unsigned char* mask) {
  std::vector<int> sel;
  for (int a = 0; a < nAtom; ++a)
    if (!mask || mask[a]) sel.push_back(a);
  return sel;
}

}  // namespace

extern "C" {

// out[i*nConf + j] = rmsd(reference i, target j)
void orc_pair_rmsd(int nConf, int nAtom, const double* coor, const unsigned char* mask, double* out) {
  const std::vector<int> sel = mask_sel(nAtom, mask);
  const int n = (int)sel.size();
  std::vector<std::vector<double>> X(nConf);
  std::vector<double> G(nConf);
  for (int c = 0; c < nConf; ++c) center_conf(coor + (size_t)c * nAtom * 3, sel, X[c], G[c]);
  for (int i = 0; i < nConf; ++i)
    for (int j = 0; j < nConf; ++j) out[(size_t)i * nConf + j] = qcp_rmsd(X[i].data(), G[i], X[j].data(), G[j], n);
}

// the reference's loop (src/GeneDiverseConformations.cpp:84-111), candidate = reference mol
// (align.SetRefMol, :96), centre = target (:100); returns the centre count
int orc_cluster_conformers(int nConf, int nAtom, const double* coor, const double* energy,
                           const unsigned char* mask, double cutOff, int maxNum, int* centers) {
  const std::vector<int> sel = mask_sel(nAtom, mask);
  const int n = (int)sel.size();
  std::vector<double> e(energy, energy + nConf);
  std::vector<size_t> idx(e.size());
  for (size_t i = 0; i != idx.size(); ++i) idx[i] = i;
  std::sort(idx.begin(), idx.end(), [&e](size_t i1, size_t i2) { return e[i1] < e[i2]; });
  std::vector<std::vector<double>> X(nConf);
  std::vector<double> G(nConf);
  for (int c = 0; c < nConf; ++c) center_conf(coor + (size_t)c * nAtom * 3, sel, X[c], G[c]);
  std::vector<size_t> idxCenter;
  idxCenter.push_back(idx[0]);
  for (int i = 1; i < nConf; i++) {
    const size_t r = idx[i];
    bool ifNewCenter = true;
    for (size_t j = 0; j < idxCenter.size(); j++) {
      const size_t t = idxCenter[j];
      if (qcp_rmsd(X[r].data(), G[r], X[t].data(), G[t], n) <= cutOff) {
        ifNewCenter = false;
        break;
      }
    }
    if (ifNewCenter) idxCenter.push_back(idx[i]);
    if ((int)idxCenter.size() == maxNum) break;
  }
  for (size_t i = 0; i < idxCenter.size(); ++i) centers[i] = (int)idxCenter[i];
  return (int)idxCenter.size();
}

}  // extern "C"
