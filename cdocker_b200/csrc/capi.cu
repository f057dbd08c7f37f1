// capi.cu -- the C-ABI: receptor context, search orchestration, kernel.h-compatible calls.
//
// The search replaces the inline core of the reference drivers
// (src/TranRotaConfSearchNoMini.cu:156-464): the receptor spectra are computed once at context
// creation and stay resident; a search is cut into waves of rotations, each wave running the
// five kernels of search_kernels.cu back to back on one stream. Only the per-rotation minimum
// energy and best translation leave the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/cdock_b200.h"
#include "cdk_internal.h"

namespace cdk {

static thread_local std::string g_last_error;
void set_error(const std::string& msg) { g_last_error = msg; }

namespace {

__global__ void k_build_tables(int nAtom, int nConf, int nQ, const float* quats,
                               const float* charge, const float* eps, const int* slot,
                               ConfDesc* confs, RotDesc* rots, AtomParam* params) {
  const long t = (long)blockIdx.x * blockDim.x + threadIdx.x;
  const long nRot = (long)nConf * nQ;
  if (t < nRot) {
    RotDesc d;
    for (int i = 0; i < 4; ++i) d.q[i] = quats[t * 4 + i];
    d.conf = (int)(t / nQ);
    d.out = (int)t;
    d.pad0 = d.pad1 = 0;
    rots[t] = d;
  }
  if (t < nConf) {
    ConfDesc c;
    c.coord_off = (int)t * nAtom;
    c.param_off = 0;
    c.n_atoms = nAtom;
    c.pad = 0;
    confs[t] = c;
  }
  if (t < nAtom) {
    AtomParam p;
    p.w_vdw = sqrtf(eps[t]);  // IEEE sqrt, as std::sqrt(float) in FillLigandGrid (:43)
    p.charge = charge[t];
    p.slot = slot[t];
    p.pad = 0;
    params[t] = p;
  }
}

// largest atom-atom distance over all conformers, as float bits (non-negative floats order
// like their bit patterns), plus a flag for slots outside [0, K-2]
__global__ void k_diameter(int nAtom, int nConf, const float* coor, const int* slot, int K,
                           unsigned int* out) {
  const long total = (long)nConf * nAtom * nAtom;
  for (long t = (long)blockIdx.x * blockDim.x + threadIdx.x; t < total;
       t += (long)gridDim.x * blockDim.x) {
    const long c = t / ((long)nAtom * nAtom);
    const int i = (int)((t / nAtom) % nAtom), j = (int)(t % nAtom);
    if (j <= i) continue;
    const float* a = coor + (c * nAtom + i) * 3;
    const float* b = coor + (c * nAtom + j) * 3;
    const double dx = (double)a[0] - b[0], dy = (double)a[1] - b[1], dz = (double)a[2] - b[2];
    const float d = (float)sqrt(dx * dx + dy * dy + dz * dz);
    atomicMax(out, __float_as_uint(d));
  }
  const long t0 = (long)blockIdx.x * blockDim.x + threadIdx.x;
  if (t0 < nAtom && (slot[t0] < 0 || slot[t0] > K - 2)) atomicOr(out + 1, 1u);
  if (t0 < (long)nConf * nAtom * 3 && !isfinite(coor[t0])) atomicOr(out + 1, 2u);
}

struct Arena {
  void* base = nullptr;
  size_t cap = 0;
};

bool grow(Arena& a, size_t bytes) {
  if (bytes <= a.cap) return true;
  if (a.base) cudaFree(a.base);
  a.base = nullptr;
  a.cap = 0;
  if (cudaMalloc(&a.base, bytes) != cudaSuccess) return false;
  a.cap = bytes;
  return true;
}

size_t align_up(size_t x) { return (x + 255) & ~size_t(255); }

}  // namespace
}  // namespace cdk

using namespace cdk;

struct cdk_ctx {
  int dev = 0;
  int n = 0, K = 0;
  float spacing = 0.f;
  cdk_opts opts{};
  cudaStream_t stream = nullptr;
  float* d_grids = nullptr;   // [K][n^3], kept for the FP64 re-score
  float2* d_phat = nullptr;   // [n][K][ncol]
  float2* d_ptilde = nullptr; // [ncol][K][n] receptor transformed over (y,z) only, x n (BF16X3 form)
  void* d_top = nullptr;      // operator image of the streamed tensor-core x pass (built on first use)
  float lscale[KMAX] = {};    // split-FP16 form: ligand scale 2^sigma_k (the operator carries 2^-sigma_k)
  float2* d_tw = nullptr;     // [n]
  int* d_kyof = nullptr;      // [n] natural frequency at each digit-reversed position
  Arena wave;                 // per-wave scratch
  Arena tables;               // per-search tables
  Arena io;                   // staging of host-buffer searches
  Arena group;                // rotation grouping of the tensor-core x pass (sorted list, keys)
  Arena topk;                 // precision forms: per wave the k lowest poses with FP64 re-scores
  int topk_k = 0, topk_waves = 0;  // of the last search
  unsigned int* d_misc = nullptr;  // [0] diameter bits, [1] flags, [2] error count, [3] fault,
                                   // [4] FP16 range flag
  unsigned long long* d_work = nullptr;  // [8] work counters (WaveArgs.work)
  unsigned long long* h_work = nullptr;
  unsigned int* h_misc = nullptr;  // pinned mirror
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  // per-kernel timing (opts.reserved[0] != 0): events around every launch of every wave
  std::vector<cudaEvent_t> kev;
  int kev_used = 0;
  // CUDA graph of the last search shape (opts.use_graphs)
  struct GraphKey {
    const void* p[7];
    int nAtom, nConf, nQ, Lb;
    cudaStream_t s;
    bool operator==(const GraphKey& o) const {
      for (int i = 0; i < 7; ++i)
        if (p[i] != o.p[i]) return false;
      return nAtom == o.nAtom && nConf == o.nConf && nQ == o.nQ && Lb == o.Lb && s == o.s;
    }
  } gkey{};
  int gkey_seen = 0;  // 1 after one plain run with gkey, 2 once the graph exists
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t gexec = nullptr;
  // autotuned x-pass configuration (opts.reserved[2] = 1), per (Lb)
  int tuned_Lb = -1, tuned_col_tile = 0, tuned_chunk = 0;
  // autotuned tensor-core x pass (Hankel operator), per (Lb, form): columns per CTA, ring cap
  int tuned_hx_Lb = -1, tuned_hx_cols = 0, tuned_hx_nb = 0, tuned_hx_ks = 0;
  // the ligand box whose x pass the autotuner has settled (whatever kernel it runs, including
  // those with nothing to tune); searches of that box may be captured into graphs
  int tuned_any_Lb = -1;
  double tune_ms[8] = {};
  double stats[CDK_NSTATS] = {};
};

namespace {

#define CDK_CUDA(call)                                                                 \
  do {                                                                                 \
    cudaError_t e_ = (call);                                                           \
    if (e_ != cudaSuccess) {                                                           \
      set_error(std::string(#call) + ": " + cudaGetErrorString(e_));                   \
      return CDK_ERR_CUDA;                                                             \
    }                                                                                  \
  } while (0)

bool supported_n(int n) { return n == 32 || n == 64 || n == 96 || n == 128; }

// Times the x pass (the dominant kernel) on the search's first wave under each candidate
// configuration -- column tile and rotations per CTA for the FP32 form, rotations per CTA for
// the tensor-core form -- and keeps the fastest for this ligand box. The candidates all compute
// the same numbers (deterministic kernels), so the timing runs leave no trace in the results.
int autotune_xpass(cdk_ctx* c, WaveArgs a, const RotDesc* d_rots, long nRot, int wave, bool tc,
                   cudaStream_t s) {
  a.nrot = (int)std::min<long>(wave, nRot);
  a.rots = d_rots;
  CDK_CUDA(launch_prep(a, s));
  CDK_CUDA(launch_spread_yz(a, s));
  struct Cand { int ct, chunk; };
  std::vector<Cand> cands;
  if (tc && c->opts.reserved[3] != 1 && umma_supported(c->n, a.Lb)) {
    cands.push_back({a.col_tile, 0});  // fixed 128-rotation tiles
  } else if (tc) {
    for (int ch : {32, 64, 128, 256}) cands.push_back({a.col_tile, ch});
  } else {
    for (int ct : (c->n <= 64 ? std::vector<int>{16, 8} : std::vector<int>{8}))
      for (int ch : {16, 32, 64}) {
        if (xpass2_smem_bytes(c->n, c->K, ct) > 227 * 1024) continue;
        cands.push_back({ct, ch});
      }
  }
  cudaEvent_t e0, e1;
  CDK_CUDA(cudaEventCreate(&e0));
  CDK_CUDA(cudaEventCreate(&e1));
  double best = 1e30;
  Cand pick = cands[0];
  int i = 0;
  for (const Cand& cd : cands) {
    WaveArgs t = a;
    t.col_tile = cd.ct;
    t.chunk = cd.chunk;
    float ms = 0.f, total = 0.f;
    for (int rep = 0; rep < 2; ++rep) {
      CDK_CUDA(cudaEventRecord(e0, s));
      if (tc && c->opts.reserved[3] != 1 && umma_supported(c->n, a.Lb))
        CDK_CUDA(launch_xpass_umma(t, c->d_ptilde, s));
      else if (tc) CDK_CUDA(launch_xpass_tc(t, c->d_ptilde, s));
      else CDK_CUDA(launch_xpass(t, s));
      CDK_CUDA(cudaEventRecord(e1, s));
      CDK_CUDA(cudaEventSynchronize(e1));
      CDK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (rep == 1) total = ms;  // second run: warm caches
    }
    if (i < 8) c->tune_ms[i] = total;
    ++i;
    if (total < best) {
      best = total;
      pick = cd;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->tuned_Lb = a.Lb;
  c->tuned_col_tile = pick.ct;
  c->tuned_chunk = pick.chunk;
  return CDK_OK;
}

// Times the Hankel tensor-core x pass on the search's first wave (rotations in the order the
// waves use) under each candidate shape -- one or two columns per CTA (n <= 64), 1 to 3 K-steps
// per ring stage, ring caps of 4, 8, 16 and 32 stages -- and keeps the fastest for this ligand box. The candidates run the same
// MMAs per column in the same order, so the results are identical whichever wins.
int autotune_hankel(cdk_ctx* c, WaveArgs a, const RotDesc* order, long nRot, int wave, bool f16,
                    const float* osc, cudaStream_t s) {
  a.nrot = (int)std::min<long>(wave, nRot);
  a.rots = order;
  CDK_CUDA(launch_prep(a, s));
  CDK_CUDA(launch_spread_yz(a, s));
  struct Cand { int cols, nb, ks; };
  std::vector<Cand> cands;
  for (int cols : {1, 2})
    for (int ks : {1, 2, 3})
      for (int nb : {4, 8, 16, 32}) {
        HankelPlan p{};
        if (!hankel_plan(c->n, c->K, a.Lb, f16, cols, &p, nb, ks) || p.cols != cols || p.ks != ks) continue;
        bool dup = false;
        for (const Cand& q : cands) dup |= (q.cols == cols && q.nb == p.nb && q.ks == ks);
        if (!dup) cands.push_back({cols, p.nb, ks});
      }
  if (cands.empty()) return CDK_OK;
  cudaEvent_t e0, e1;
  CDK_CUDA(cudaEventCreate(&e0));
  CDK_CUDA(cudaEventCreate(&e1));
  double best = 1e30;
  Cand pick = cands[0];
  int i = 0;
  for (const Cand& cd : cands) {
    HankelPlan p{};
    hankel_plan(c->n, c->K, a.Lb, f16, cd.cols, &p, cd.nb, cd.ks);
    hankel_b_layout(p, a);
    float ms = 0.f, total = 0.f;
    for (int rep = 0; rep < 2; ++rep) {
      CDK_CUDA(cudaEventRecord(e0, s));
      CDK_CUDA(launch_xpass_hankel(a, c->d_ptilde, osc, p, s));
      CDK_CUDA(cudaEventRecord(e1, s));
      CDK_CUDA(cudaEventSynchronize(e1));
      CDK_CUDA(cudaEventElapsedTime(&ms, e0, e1));
      if (rep == 1) total = ms;  // second run: warm caches
    }
    if (i < 8) c->tune_ms[i] = total;
    ++i;
    if (total < best) {
      best = total;
      pick = cd;
    }
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  c->tuned_hx_Lb = a.Lb;
  c->tuned_hx_cols = pick.cols;
  c->tuned_hx_nb = pick.nb;
  c->tuned_hx_ks = pick.ks;
  return CDK_OK;
}

// the search proper on device tables; nRot rotations, outputs indexed by RotDesc.out
int run_waves(cdk_ctx* c, const float* d_coor, const AtomParam* d_params, const ConfDesc* d_confs,
              const RotDesc* d_rots, long nRot, int maxAtoms, int Lb, float* d_minE, int* d_idx,
              cudaStream_t s) {
  const int n = c->n, K = c->K;
  const size_t ncol = (size_t)n * (n / 2 + 1);
  const bool tc = c->opts.form != CDK_FORM_FP32;
  const bool f16form = c->opts.form == CDK_FORM_FP16X2;
  // tensor-core x pass with streamed ligand rows (direct planes: ligands <= 96 atoms): the
  // Hankel-operator kernel at every n (box <= 32 planes, operator fits shared memory); the older
  // 64^3 kernel with streamed operator tiles on request (reserved[3] = 3)
  WaveArgs probe{};
  probe.kyof = (c->opts.reserved[1] & 1) ? nullptr : c->d_kyof;
  probe.max_atoms = maxAtoms;
  probe.atom_cap = maxAtoms;
  // automatic choice (reserved[3] = 0): the Hankel kernel over tiled rows (64^3: 5 % faster per
  // search than the streamed-tile kernel in the split-BF16 form); 3 forces streamed tiles (64^3,
  // box <= 32 planes), 4 the Hankel kernel
  const int variant = c->opts.reserved[3];
  const bool can_stream = tc && stream_supported(n, Lb) && direct_planes(probe);
  const bool streamed = can_stream && use_stream_tiles(variant);
  HankelPlan hp{};
  const bool hankel = tc && !streamed && (variant == 0 || variant == 4) && direct_planes(probe) &&
                      hankel_plan(n, K, Lb, f16form, c->opts.reserved[5] & 3, &hp, 0, (c->opts.reserved[5] >> 2) & 7);
  if (streamed && !c->d_top) {
    const size_t tb = stream_top_bytes(n, K);
    if (cudaMalloc(&c->d_top, tb) != cudaSuccess) {
      c->d_top = nullptr;
      set_error("cudaMalloc of the tensor-core operator image failed (" + std::to_string(tb >> 20) + " MiB)");
      return CDK_ERR_NOMEM;
    }
    std::vector<float> osc(K);
    for (int k = 0; k < K; ++k) osc[k] = 1.f / c->lscale[k];
    // stream-ordered before the waves
    CDK_CUDA(launch_top_build(n, K, c->d_ptilde, c->d_top, f16form ? osc.data() : nullptr, s));
  }
  std::vector<float> osc(K);
  for (int k = 0; k < K; ++k) osc[k] = 1.f / c->lscale[k];
  const bool rows = hankel || streamed;  // the plane kernel writes split / FP16 ligand rows
  if (tc && f16form && !rows) {
    set_error("the split-FP16 form runs on the tensor-core x pass with ligand rows only (ligands "
              "of at most 96 atoms, a ligand box of at most 32 planes, K x n small enough for the "
              "operator to fit shared memory); use CDK_FORM_BF16X3");
    return CDK_ERR_UNSUPPORTED;
  }
  const bool f16 = f16form && rows;
  // the Hankel x pass loads tiled ligand rows by tensor copies, or untiled rows by per-thread copies
  const bool tiled = hankel && hankel_tiled(c->opts.reserved[5]);
  const size_t lop_per = rows ? stream_lop_bytes_per_rotation(n, K, f16) : 0;
  int wave = c->opts.wave_rotations;
  if (wave <= 0) {
    // keep A + B of one wave near 16 GiB at n <= 64 (under a tenth of the B200's HBM): at 64^3,
    // waves of ~4,900 rotations instead of ~1,800 make the split-FP16 search 2-4 % faster (fewer
    // kernel tails per rotation; measured up to 8,192); 32 GiB at n >= 96, where a rotation's
    // rows and window planes take 10-30 MB
    const double per = (rows ? (double)lop_per : (double)K * Lb * ncol * 8) + (double)n * ncol * 8;
    const double target = (n <= 64 ? 16.0 : 32.0) * (1ull << 30);
    wave = (int)std::min<double>(8192.0, std::max(64.0, target / per));
  }
  wave = (int)std::min<long>(wave, std::min<long>(nRot, 65535));
  if (wave < 1) wave = 1;
  const size_t b_rotxyz = align_up((size_t)wave * maxAtoms * sizeof(float4));
  const size_t b_rec = align_up((size_t)wave * sizeof(RotRec));
  const size_t b_keys = align_up((size_t)wave * sizeof(unsigned long long));
  // precision forms: the FP64 near-tie break (reserved[7] = 1 turns it off) keeps every window
  // plane's two smallest keys; per wave the k lowest poses are re-scored in FP64 (reserved[6]:
  // 0 = 8 in the precision forms and none in the FP32 form, -1 = none, 1..32 = k)
  const bool tiebreak = tc && c->opts.reserved[7] == 0;
  const int topk = c->opts.reserved[6] < 0 ? 0 : c->opts.reserved[6] > 0 ? std::min(c->opts.reserved[6], (int)kTopMax)
                                                                        : (tc ? 8 : 0);
  const size_t b_keys2 = tiebreak ? align_up((size_t)wave * n * 2 * sizeof(unsigned long long)) : 0;
  const size_t b_A = align_up(rows ? lop_wave_bytes(wave, tiled, lop_per)
                                   : (size_t)wave * K * Lb * ncol * sizeof(float2));
  const size_t b_B = align_up((size_t)wave * n * ncol * sizeof(float2));
  if (!grow(c->wave, b_rotxyz + b_rec + b_keys + b_A + b_B + b_keys2)) {
    set_error("cudaMalloc of the wave scratch failed (" +
              std::to_string((b_rotxyz + b_rec + b_keys + b_A + b_B + b_keys2) >> 20) + " MiB)");
    return CDK_ERR_NOMEM;
  }
  char* base = static_cast<char*>(c->wave.base);
  WaveArgs a{};
  a.n = n;
  a.K = K;
  a.Lb = Lb;
  a.spacing = c->spacing;
  a.max_atoms = maxAtoms;
  a.atom_cap = maxAtoms;
  a.coords = d_coor;
  a.params = d_params;
  a.confs = d_confs;
  a.rot_xyz = reinterpret_cast<float4*>(base);
  a.rec = reinterpret_cast<RotRec*>(base + b_rotxyz);
  a.keys = reinterpret_cast<unsigned long long*>(base + b_rotxyz + b_rec);
  a.A = rows ? nullptr : reinterpret_cast<float2*>(base + b_rotxyz + b_rec + b_keys);
  a.lop = rows ? reinterpret_cast<unsigned char*>(base + b_rotxyz + b_rec + b_keys) : nullptr;
  a.lop_tiled = tiled ? 1 : 0;
  a.B = reinterpret_cast<float2*>(base + b_rotxyz + b_rec + b_keys + b_A);
  a.keys2 = tiebreak ? reinterpret_cast<unsigned long long*>(base + b_rotxyz + b_rec + b_keys + b_A + b_B) : nullptr;
  a.phat = c->d_phat;
  a.tw = c->d_tw;
  a.minE = d_minE;
  a.idx = d_idx;
  a.err_count = reinterpret_cast<int*>(c->d_misc + 2);
  a.fault = reinterpret_cast<int*>(c->d_misc + 3);
  a.f16 = f16 ? 1 : 0;
  for (int k = 0; k < KMAX; ++k) a.lscale[k] = c->lscale[k];
  a.range_err = reinterpret_cast<int*>(c->d_misc + 4);
  // the shared-memory streamed x pass writes B in plane groups (whole sectors per store)
  a.bgroup = rows ? stream_bgroup() : 1;
  a.col_tile = c->opts.col_tile > 0 ? c->opts.col_tile : pick_col_tile(n, K);
  a.kyof = (c->opts.reserved[1] & 1) ? nullptr : c->d_kyof;  // reserved[1] bit 0: FFT planes
  // bit 1: block-stage yz kernel at every n; bit 2: octet yz kernel at every n
  a.yz_block_stages = (c->opts.reserved[1] & 2) ? 1 : (c->opts.reserved[1] & 4) ? 2 : 0;
  a.chunk = 0;
  if (c->tuned_Lb == Lb) {
    if (c->tuned_col_tile) a.col_tile = c->tuned_col_tile;
    a.chunk = c->tuned_chunk;
  }
  if (tc && !rows && xpass_tc_smem_bytes(n, K, Lb) > 227 * 1024) {
    set_error("ligand box too large for the tensor-core x pass at this grid size and K");
    return CDK_ERR_UNSUPPORTED;
  }
  if (xpass2_smem_bytes(n, K, a.col_tile) > 227 * 1024 ||
      (n <= 64 && a.col_tile != 8 && a.col_tile != 16) || (n > 64 && a.col_tile != 8)) {
    set_error("column tile must be 8 or 16 (n <= 64) or 8 (n > 64) and fit shared memory");
    return CDK_ERR_INVALID;
  }
  CDK_CUDA(cudaMemsetAsync(c->d_misc + 2, 0, 3 * sizeof(unsigned int), s));
  CDK_CUDA(cudaMemsetAsync(c->d_work, 0, 8 * sizeof(unsigned long long), s));
  const bool umma = tc && !rows && c->opts.reserved[3] != 1 && umma_supported(n, Lb);
  a.work = c->d_work;
  const bool prof = c->opts.reserved[0] != 0;
  const long nwaves = (nRot + wave - 1) / wave;
  c->topk_k = topk;
  c->topk_waves = 0;
  if (topk > 0 && !grow(c->topk, (size_t)nwaves * topk * sizeof(TopPose))) {
    set_error("cudaMalloc of the top-pose buffer failed");
    return CDK_ERR_NOMEM;
  }
  if (prof) {
    const size_t need = (size_t)nwaves * (kLaunchesPerWave + 1);
    while (c->kev.size() < need) {
      cudaEvent_t e;
      CDK_CUDA(cudaEventCreate(&e));
      c->kev.push_back(e);
    }
  }
  c->kev_used = 0;
  // inside a stream capture the per-kernel events become external event-record nodes of the
  // graph (a plain record there would only order the capture), so replays record them too
  cudaStreamCaptureStatus cap_state = cudaStreamCaptureStatusNone;
  CDK_CUDA(cudaStreamIsCapturing(s, &cap_state));
  const unsigned int evflags = cap_state == cudaStreamCaptureStatusActive ? cudaEventRecordExternal
                                                                          : cudaEventRecordDefault;
  if (c->opts.reserved[2] && c->tuned_Lb != Lb && !rows) {
    int rc = autotune_xpass(c, a, d_rots, nRot, wave, tc, s);
    if (rc) return rc;
    a.col_tile = c->tuned_col_tile ? c->tuned_col_tile : a.col_tile;
    a.chunk = c->tuned_chunk;
  }
  long launches = 1, waves = 0;
  // tensor-core x pass: rotations reaching the same ligand-box chunks side by side (fewer
  // K-steps per 128-rotation tile; reserved[4] = 1 keeps the given order)
  const RotDesc* order = d_rots;
  const int jc = (Lb + 7) / 8;
  if (rows && c->opts.reserved[4] == 0 && nRot > 128 && jc > 1) {
    const size_t gb = group_rotations_bytes(nRot);
    if (!grow(c->group, gb)) {
      set_error("cudaMalloc of the rotation-grouping scratch failed (" + std::to_string(gb >> 20) + " MiB)");
      return CDK_ERR_NOMEM;
    }
    RotDesc* sorted = nullptr;
    CDK_CUDA(launch_group_rotations(d_rots, d_confs, d_coor, d_params, nRot, maxAtoms, K, c->spacing, jc,
                                    c->group.base, &sorted, s));
    order = sorted;
    launches += 4;
  }
  if (hankel && c->opts.reserved[2] && c->tuned_hx_Lb != Lb) {
    int rc = autotune_hankel(c, a, order, nRot, wave, f16form, osc.data(), s);
    if (rc) return rc;
  }
  if (hankel && c->tuned_hx_Lb == Lb && c->tuned_hx_cols > 0)
    hankel_plan(n, K, Lb, f16form, c->tuned_hx_cols, &hp, c->tuned_hx_nb, c->tuned_hx_ks);
  if (hankel) hankel_b_layout(hp, a);
  if (c->opts.reserved[2]) c->tuned_any_Lb = Lb;
  for (long r0 = 0; r0 < nRot; r0 += wave) {
    a.nrot = (int)std::min<long>(wave, nRot - r0);
    a.rots = order + r0;
    cudaEvent_t* ev = prof ? &c->kev[(size_t)waves * (kLaunchesPerWave + 1)] : nullptr;
    if (prof) CDK_CUDA(cudaEventRecordWithFlags(ev[0], s, evflags));
    CDK_CUDA(launch_prep(a, s));
    if (prof) CDK_CUDA(cudaEventRecordWithFlags(ev[1], s, evflags));
    CDK_CUDA(launch_spread_yz(a, s));
    if (prof) CDK_CUDA(cudaEventRecordWithFlags(ev[2], s, evflags));
    if (hankel) CDK_CUDA(launch_xpass_hankel(a, c->d_ptilde, osc.data(), hp, s));
    else if (streamed) CDK_CUDA(launch_xpass_stream(a, c->d_top, s));
    else if (umma) CDK_CUDA(launch_xpass_umma(a, c->d_ptilde, s));
    else if (tc) CDK_CUDA(launch_xpass_tc(a, c->d_ptilde, s));
    else CDK_CUDA(launch_xpass(a, s));
    if (prof) CDK_CUDA(cudaEventRecordWithFlags(ev[3], s, evflags));
    CDK_CUDA(launch_yz_inv_argmin(a, s));
    if (tiebreak) CDK_CUDA(launch_tiebreak(a, c->d_grids, f16form ? 1e-3f : 1e-4f, s));
    if (topk > 0)
      CDK_CUDA(launch_topk_rescore(a, c->d_grids, topk, static_cast<TopPose*>(c->topk.base) + (size_t)waves * topk, s));
    if (prof) CDK_CUDA(cudaEventRecordWithFlags(ev[4], s, evflags));
    CDK_CUDA(launch_finalize(a, s));
    if (prof) CDK_CUDA(cudaEventRecordWithFlags(ev[5], s, evflags));
    launches += kLaunchesPerWave + (rows ? 1 : 0) + (tiebreak ? 1 : 0) + (topk > 0 ? 1 : 0);  // + k_tile_plan
    ++waves;
  }
  c->kev_used = prof ? (int)waves : 0;
  c->topk_waves = topk > 0 ? (int)waves : 0;
  c->stats[0] = (double)launches;
  c->stats[1] = (double)waves;
  c->stats[2] = (double)nRot;
  c->stats[4] = (double)Lb;
  c->stats[5] = (double)wave;
  c->stats[13] = hankel ? (double)hp.cols : streamed ? 4.0 : (double)a.col_tile;
  c->stats[14] = rows || umma ? 128.0 : (double)(a.chunk > 0 ? a.chunk : (tc ? 64 : 32));
  c->stats[16] = hankel ? (f16 ? 7.0 : 6.0) : streamed ? (f16 ? 5.0 : 3.0) : umma ? 2.0 : tc ? 1.0 : 0.0;
  c->stats[15] = (double)(c->gkey_seen);
  return CDK_OK;
}

// Checks inputs on the device (slots, finite coordinates) and plans the ligand box from the
// largest atom-atom distance. Synchronises the stream once (4-byte read back).
int plan_box(cdk_ctx* c, int nAtom, int nConf, const float* d_coor, const int* d_slot,
             cudaStream_t s, int* Lb) {
  CDK_CUDA(cudaMemsetAsync(c->d_misc, 0, 2 * sizeof(unsigned int), s));
  const long pairs = (long)nConf * nAtom * nAtom;
  long blocks = std::max<long>((pairs + 255) / 256, ((long)nConf * nAtom * 3 + 255) / 256);
  blocks = std::min<long>(blocks, 4096);
  k_diameter<<<(unsigned)std::max<long>(1, blocks), 256, 0, s>>>(nAtom, nConf, d_coor, d_slot,
                                                                c->K, c->d_misc);
  CDK_CUDA(cudaGetLastError());
  CDK_CUDA(cudaMemcpyAsync(c->h_misc, c->d_misc, 2 * sizeof(unsigned int),
                           cudaMemcpyDeviceToHost, s));
  CDK_CUDA(cudaStreamSynchronize(s));
  if (c->h_misc[1] & 1u) {
    set_error("atom slot outside [0, K-2]");
    return CDK_ERR_INVALID;
  }
  if (c->h_misc[1] & 2u) {
    set_error("non-finite ligand coordinate");
    return CDK_ERR_INVALID;
  }
  float diam;
  std::memcpy(&diam, &c->h_misc[0], sizeof(float));
  // the spread touches x planes up to int(len/h)+1 with len <= diameter; two planes of slack
  // absorb rounding of rotated coordinates and non-unit quaternions
  const int lb = (int)std::floor(diam / c->spacing + 1e-3) + 3;
  *Lb = std::min(c->n, std::max(lb, 2));
  return CDK_OK;
}

int search_device_impl(cdk_ctx* c, int nAtom, int nConf, const float* d_coor,
                       const float* d_charge, const float* d_eps, const int* d_slot, int nQ,
                       const float* d_quats, float* d_minE, int* d_idx, cudaStream_t s) {
  if (nAtom <= 0 || nConf <= 0 || nQ < 0) {
    set_error("nAtom and nConf must be positive, nQ non-negative");
    return CDK_ERR_INVALID;
  }
  if (nAtom > c->opts.max_atoms) {
    set_error("ligand has more atoms than the context's max_atoms");
    return CDK_ERR_INVALID;
  }
  const long nRot = (long)nConf * nQ;
  if (nRot == 0) return CDK_OK;
  if (nRot > (1l << 31) / 4) {
    set_error("too many rotations in one call");
    return CDK_ERR_INVALID;
  }
  CDK_CUDA(cudaSetDevice(c->dev));
  int Lb = 0;
  int rc = plan_box(c, nAtom, nConf, d_coor, d_slot, s, &Lb);
  if (rc) return rc;
  const size_t b_conf = align_up(sizeof(ConfDesc) * nConf);
  const size_t b_rot = align_up(sizeof(RotDesc) * nRot);
  const size_t b_par = align_up(sizeof(AtomParam) * nAtom);
  if (!grow(c->tables, b_conf + b_rot + b_par)) {
    set_error("cudaMalloc of the search tables failed");
    return CDK_ERR_NOMEM;
  }
  char* tb = static_cast<char*>(c->tables.base);
  ConfDesc* confs = reinterpret_cast<ConfDesc*>(tb);
  RotDesc* rots = reinterpret_cast<RotDesc*>(tb + b_conf);
  AtomParam* params = reinterpret_cast<AtomParam*>(tb + b_conf + b_rot);
  CDK_CUDA(cudaEventRecord(c->ev0, s));
  const long tmax = std::max<long>(nRot, std::max(nConf, nAtom));
  // CUDA graph: the first search of a shape runs plainly (growing the scratch), the second
  // captures build-tables + every wave into one graph, later ones replay it
  cdk_ctx::GraphKey key{{d_coor, d_charge, d_eps, d_slot, d_quats, d_minE, d_idx}, nAtom, nConf, nQ, Lb, s};
  // a search that autotunes (a new ligand box) runs plainly: timing runs do not go into graphs
  const bool graphs = c->opts.use_graphs != 0 && !(c->opts.reserved[2] && c->tuned_any_Lb != Lb);
  if (graphs && c->gkey_seen == 2 && c->gkey == key) {
    CDK_CUDA(cudaGraphLaunch(c->gexec, s));
    CDK_CUDA(cudaEventRecord(c->ev1, s));
    c->stats[15] = 2;
    return CDK_OK;
  }
  const bool capture = graphs && c->gkey_seen == 1 && c->gkey == key;
  if (capture) CDK_CUDA(cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal));
  k_build_tables<<<(unsigned)((tmax + 255) / 256), 256, 0, s>>>(
      nAtom, nConf, nQ, d_quats, d_charge, d_eps, d_slot, confs, rots, params);
  cudaError_t le = cudaGetLastError();
  rc = (le == cudaSuccess) ? run_waves(c, d_coor, params, confs, rots, nRot, nAtom, Lb, d_minE, d_idx, s)
                           : CDK_ERR_CUDA;
  if (capture) {
    cudaGraph_t g = nullptr;
    cudaError_t ce = cudaStreamEndCapture(s, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (ce != cudaSuccess) {
      set_error(std::string("graph capture: ") + cudaGetErrorString(ce));
      return CDK_ERR_CUDA;
    }
    if (c->gexec) cudaGraphExecDestroy(c->gexec);
    if (c->graph) cudaGraphDestroy(c->graph);
    c->graph = g;
    CDK_CUDA(cudaGraphInstantiate(&c->gexec, g, 0));
    CDK_CUDA(cudaGraphLaunch(c->gexec, s));
    c->gkey_seen = 2;
    c->stats[15] = 2;
  } else {
    if (rc) return rc;
    if (graphs) {
      c->gkey = key;
      c->gkey_seen = 1;
    }
  }
  if (le != cudaSuccess) {
    set_error(std::string("k_build_tables: ") + cudaGetErrorString(le));
    return CDK_ERR_CUDA;
  }
  CDK_CUDA(cudaEventRecord(c->ev1, s));
  return CDK_OK;
}

int check_errors_after(cdk_ctx* c, cudaStream_t s) {
  CDK_CUDA(cudaMemcpyAsync(c->h_misc + 2, c->d_misc + 2, 3 * sizeof(unsigned int),
                           cudaMemcpyDeviceToHost, s));
  CDK_CUDA(cudaStreamSynchronize(s));
  if (c->h_misc[3] != 0) {
    set_error("a bounded device wait (tensor-core commit) gave up; results are invalid");
    return CDK_ERR_CUDA;
  }
  float ms = 0.f;
  if (cudaEventElapsedTime(&ms, c->ev0, c->ev1) == cudaSuccess) c->stats[3] = ms;
  (void)cudaGetLastError();
  CDK_CUDA(cudaMemcpy(c->h_work, c->d_work, 8 * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  c->stats[6] = (double)c->h_work[0];
  c->stats[7] = (double)c->h_work[1];
  c->stats[17] = (double)c->h_work[2];
  c->stats[18] = (double)c->h_work[3];
  c->stats[19] = (double)c->h_work[4];
  c->stats[20] = (double)c->h_work[5];
  for (int k = 0; k < kLaunchesPerWave; ++k) c->stats[8 + k] = 0.0;
  for (int w = 0; w < c->kev_used; ++w) {
    cudaEvent_t* ev = &c->kev[(size_t)w * (kLaunchesPerWave + 1)];
    for (int k = 0; k < kLaunchesPerWave; ++k) {
      float t = 0.f;
      if (cudaEventElapsedTime(&t, ev[k], ev[k + 1]) == cudaSuccess) c->stats[8 + k] += t;
    }
  }
  // a timing query that failed (an event never recorded) must not surface as the error of a
  // later call
  (void)cudaGetLastError();
  if (c->h_misc[2] != 0) {
    set_error(std::to_string(c->h_misc[2]) +
              " rotation(s) overflowed the planned ligand box; results for them are invalid");
    return CDK_ERR_OVERFLOW;
  }
  if (c->h_misc[4] != 0) {
    set_error("a scaled ligand spectrum value left the FP16 range of the split-FP16 form "
              "(charges or sqrt-epsilon sums too large for this receptor); use CDK_FORM_BF16X3");
    return CDK_ERR_UNSUPPORTED;
  }
  return CDK_OK;
}

}  // namespace

namespace cdk {
bool ctx_view(const cdk_ctx* c, CtxView* v) {
  if (!c || !v) return false;
  v->dev = c->dev;
  v->n = c->n;
  v->K = c->K;
  v->spacing = c->spacing;
  v->col_tile_opt = c->opts.col_tile;
  v->max_atoms = c->opts.max_atoms;
  v->phat = c->d_phat;
  v->tw = c->d_tw;
  v->kyof = (c->opts.reserved[1] & 1) ? nullptr : c->d_kyof;
  v->h_misc = c->h_misc;
  v->stream = c->stream;
  v->form = c->opts.form;
  v->tc_variant = c->opts.reserved[3];
  v->hx_shape = c->opts.reserved[5];
  v->top = c->d_top;
  v->ptilde = c->d_ptilde;
  v->grids = c->d_grids;
  v->tiebreak = c->opts.form != CDK_FORM_FP32 && c->opts.reserved[7] == 0;
  for (int k = 0; k < KMAX; ++k) v->lscale[k] = c->lscale[k];
  return true;
}

int ctx_ensure_top(cdk_ctx* c) {
  if (c->d_top) return CDK_OK;
  if (c->opts.form == CDK_FORM_FP32 || !c->d_ptilde) {
    set_error("the operator image needs a precision-form context");
    return CDK_ERR_INVALID;
  }
  const size_t tb = stream_top_bytes(c->n, c->K);
  if (tb == 0) {
    set_error("no streamed tensor-core x pass at this grid size");
    return CDK_ERR_UNSUPPORTED;
  }
  if (cudaMalloc(&c->d_top, tb) != cudaSuccess) {
    c->d_top = nullptr;
    set_error("cudaMalloc of the tensor-core operator image failed (" + std::to_string(tb >> 20) + " MiB)");
    return CDK_ERR_NOMEM;
  }
  std::vector<float> osc(c->K);
  for (int k = 0; k < c->K; ++k) osc[k] = 1.f / c->lscale[k];
  cudaError_t e = launch_top_build(c->n, c->K, c->d_ptilde, c->d_top,
                                   c->opts.form == CDK_FORM_FP16X2 ? osc.data() : nullptr, c->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) {
    set_error(std::string("operator image: ") + cudaGetErrorString(e));
    return CDK_ERR_CUDA;
  }
  return CDK_OK;
}
}  // namespace cdk

extern "C" {

const char* cdk_version(void) { return "cdock_b200 0.1 (sm_100a)"; }

int cdk_last_error(char* buf, size_t cap) {
  const std::string& m = g_last_error;
  if (buf && cap) {
    size_t k = std::min(cap - 1, m.size());
    std::memcpy(buf, m.data(), k);
    buf[k] = 0;
  }
  return (int)m.size();
}

void cdk_opts_default(cdk_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->device = 0;
  o->form = CDK_FORM_FP32;
  o->wave_rotations = 0;
  o->max_atoms = 256;
  o->col_tile = 0;
  o->use_graphs = 0;
}

int cdk_ctx_create(int nx, int ny, int nz, float spacing, int K, const float* grids,
                   const cdk_opts* opts, cdk_ctx** out) {
  if (!out || !grids) {
    set_error("null argument");
    return CDK_ERR_INVALID;
  }
  *out = nullptr;
  if (nx != ny || ny != nz || !supported_n(nx)) {
    set_error("grid must be cubic with edge 32, 64, 96 or 128");
    return CDK_ERR_UNSUPPORTED;
  }
  if (K < 2 || K > KMAX) {
    set_error("K must be in [2, 16]");
    return CDK_ERR_UNSUPPORTED;
  }
  if (!(spacing > 0.f) || !std::isfinite(spacing)) {
    set_error("spacing must be positive");
    return CDK_ERR_INVALID;
  }
  cdk_ctx* c = new cdk_ctx();
  if (opts) c->opts = *opts;
  else cdk_opts_default(&c->opts);
  if (c->opts.max_atoms <= 0) c->opts.max_atoms = 256;
  if (c->opts.form != CDK_FORM_FP32 && c->opts.form != CDK_FORM_BF16X3 && c->opts.form != CDK_FORM_FP16X2) {
    delete c;
    set_error("unknown form");
    return CDK_ERR_UNSUPPORTED;
  }
  c->dev = c->opts.device;
  c->n = nx;
  c->K = K;
  c->spacing = spacing;
  auto fail = [&](int code) {
    cdk_ctx_destroy(c);
    return code;
  };
#define CTX_CUDA(call)                                                   \
  do {                                                                   \
    cudaError_t e_ = (call);                                             \
    if (e_ != cudaSuccess) {                                             \
      set_error(std::string(#call) + ": " + cudaGetErrorString(e_));     \
      return fail(e_ == cudaErrorMemoryAllocation ? CDK_ERR_NOMEM : CDK_ERR_CUDA); \
    }                                                                    \
  } while (0)
  CTX_CUDA(cudaSetDevice(c->dev));
  CTX_CUDA(cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
  CTX_CUDA(cudaEventCreate(&c->ev0));
  CTX_CUDA(cudaEventCreate(&c->ev1));
  const int n = nx;
  const size_t N = (size_t)n * n * n, ncol = (size_t)n * (n / 2 + 1);
  CTX_CUDA(cudaMalloc(&c->d_grids, sizeof(float) * K * N));
  CTX_CUDA(cudaMalloc(&c->d_phat, sizeof(float2) * K * n * ncol));
  CTX_CUDA(cudaMalloc(&c->d_tw, sizeof(float2) * n));
  CTX_CUDA(cudaMalloc(&c->d_misc, 8 * sizeof(unsigned int)));
  CTX_CUDA(cudaMallocHost(&c->h_misc, 8 * sizeof(unsigned int)));
  CTX_CUDA(cudaMalloc(&c->d_work, 8 * sizeof(unsigned long long)));
  CTX_CUDA(cudaMallocHost(&c->h_work, 8 * sizeof(unsigned long long)));
  std::vector<float2> tw(n);
  for (int j = 0; j < n; ++j) {
    const double ang = -2.0 * M_PI * j / n;
    tw[j] = make_float2((float)std::cos(ang), (float)std::sin(ang));
  }
  CTX_CUDA(cudaMemcpyAsync(c->d_tw, tw.data(), sizeof(float2) * n, cudaMemcpyHostToDevice,
                           c->stream));
  {
    std::vector<int> kyof(n);
    for (int k = 0; k < n; ++k) kyof[fft_position(n, k)] = k;
    CTX_CUDA(cudaMalloc(&c->d_kyof, sizeof(int) * n));
    CTX_CUDA(cudaMemcpy(c->d_kyof, kyof.data(), sizeof(int) * n, cudaMemcpyHostToDevice));
  }
  CTX_CUDA(cudaMemcpyAsync(c->d_grids, grids, sizeof(float) * K * N, cudaMemcpyHostToDevice,
                           c->stream));
  float2* scratch = nullptr;
  CTX_CUDA(cudaMalloc(&scratch, sizeof(float2) * K * n * ncol));
  cudaError_t e = launch_receptor_fft(n, K, c->d_grids, scratch, c->d_phat, c->d_tw,
                                      pick_col_tile(n, 1), c->stream);
  if (e == cudaSuccess && c->opts.form != CDK_FORM_FP32) {
    e = cudaMalloc(&c->d_ptilde, sizeof(float2) * K * n * ncol);
    if (e == cudaSuccess) e = launch_ptilde(n, K, scratch, c->d_ptilde, c->stream);
  }
  cudaError_t e2 = cudaStreamSynchronize(c->stream);
  cudaFree(scratch);
  CTX_CUDA(e);
  CTX_CUDA(e2);
  for (int k = 0; k < KMAX; ++k) c->lscale[k] = 1.f;
  if (c->opts.form == CDK_FORM_FP16X2) {
    // per channel the power of two that brings max |P~| into [2^14, 2^15): the operator image
    // holds P~ 2^-sigma and the ligand rows carry 2^sigma (FP16 ends at 65504)
    std::vector<float2> pt((size_t)K * n * ncol);
    CTX_CUDA(cudaMemcpy(pt.data(), c->d_ptilde, sizeof(float2) * pt.size(), cudaMemcpyDeviceToHost));
    std::vector<float> mx(K, 0.f);
    for (size_t i = 0; i < pt.size(); ++i) {
      const int k = (int)((i / n) % K);  // [ncol][K][n]
      mx[k] = std::max(mx[k], std::max(std::fabs(pt[i].x), std::fabs(pt[i].y)));
    }
    for (int k = 0; k < K; ++k) {
      int sigma = 0;
      if (mx[k] > 0.f && std::isfinite(mx[k]))
        sigma = std::min(30, std::max(-30, (int)std::floor(std::log2(mx[k])) - 14));
      c->lscale[k] = std::ldexp(1.0f, sigma);
    }
  }
#undef CTX_CUDA
  *out = c;
  return CDK_OK;
}

int cdk_ctx_destroy(cdk_ctx* c) {
  if (!c) return CDK_OK;
  cudaSetDevice(c->dev);
  if (c->stream) cudaStreamSynchronize(c->stream);
  cudaFree(c->d_grids);
  cudaFree(c->d_phat);
  cudaFree(c->d_ptilde);
  cudaFree(c->d_top);
  cudaFree(c->d_tw);
  cudaFree(c->d_kyof);
  cudaFree(c->d_misc);
  if (c->h_misc) cudaFreeHost(c->h_misc);
  cudaFree(c->d_work);
  if (c->h_work) cudaFreeHost(c->h_work);
  for (cudaEvent_t e : c->kev) cudaEventDestroy(e);
  if (c->gexec) cudaGraphExecDestroy(c->gexec);
  if (c->graph) cudaGraphDestroy(c->graph);
  cudaFree(c->wave.base);
  cudaFree(c->tables.base);
  cudaFree(c->io.base);
  cudaFree(c->group.base);
  cudaFree(c->topk.base);
  if (c->ev0) cudaEventDestroy(c->ev0);
  if (c->ev1) cudaEventDestroy(c->ev1);
  if (c->stream) cudaStreamDestroy(c->stream);
  delete c;
  return CDK_OK;
}

int cdk_search_device(cdk_ctx* c, int nAtom, int nConf, const float* d_coor,
                      const float* d_charge, const float* d_eps, const int* d_slot, int nQ,
                      const float* d_quats, float* d_minE, int* d_idx, void* stream) {
  if (!c || !d_coor || !d_charge || !d_eps || !d_slot || !d_minE || !d_idx ||
      (nQ > 0 && !d_quats)) {
    set_error("null argument");
    return CDK_ERR_INVALID;
  }
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
  int rc = search_device_impl(c, nAtom, nConf, d_coor, d_charge, d_eps, d_slot, nQ, d_quats,
                              d_minE, d_idx, s);
  if (rc) return rc;
  return check_errors_after(c, s);
}

int cdk_search(cdk_ctx* c, int nAtom, int nConf, const float* coor, const float* charge,
               const float* eps, const int* slot, int nQ, const float* quats, float* minE,
               int* idx, void* stream) {
  if (!c || !coor || !charge || !eps || !slot || !minE || !idx || (nQ > 0 && !quats)) {
    set_error("null argument");
    return CDK_ERR_INVALID;
  }
  if (nAtom <= 0 || nConf <= 0 || nQ < 0) {
    set_error("nAtom and nConf must be positive, nQ non-negative");
    return CDK_ERR_INVALID;
  }
  const long nRot = (long)nConf * nQ;
  if (nRot == 0) return CDK_OK;
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
  CDK_CUDA(cudaSetDevice(c->dev));
  const size_t b_coor = align_up(sizeof(float) * 3 * nAtom * (size_t)nConf);
  const size_t b_atom = align_up(sizeof(float) * nAtom);
  const size_t b_q = align_up(sizeof(float) * 4 * nRot);
  const size_t b_e = align_up(sizeof(float) * nRot);
  const size_t b_i = align_up(sizeof(int) * 3 * nRot);
  if (!grow(c->io, b_coor + 3 * b_atom + b_q + b_e + b_i)) {
    set_error("cudaMalloc of the input staging failed");
    return CDK_ERR_NOMEM;
  }
  char* p = static_cast<char*>(c->io.base);
  float* d_coor = reinterpret_cast<float*>(p);
  float* d_charge = reinterpret_cast<float*>(p + b_coor);
  float* d_eps = reinterpret_cast<float*>(p + b_coor + b_atom);
  int* d_slot = reinterpret_cast<int*>(p + b_coor + 2 * b_atom);
  float* d_q = reinterpret_cast<float*>(p + b_coor + 3 * b_atom);
  float* d_e = reinterpret_cast<float*>(p + b_coor + 3 * b_atom + b_q);
  int* d_i = reinterpret_cast<int*>(p + b_coor + 3 * b_atom + b_q + b_e);
  CDK_CUDA(cudaMemcpyAsync(d_coor, coor, sizeof(float) * 3 * nAtom * (size_t)nConf,
                           cudaMemcpyHostToDevice, s));
  CDK_CUDA(cudaMemcpyAsync(d_charge, charge, sizeof(float) * nAtom, cudaMemcpyHostToDevice, s));
  CDK_CUDA(cudaMemcpyAsync(d_eps, eps, sizeof(float) * nAtom, cudaMemcpyHostToDevice, s));
  CDK_CUDA(cudaMemcpyAsync(d_slot, slot, sizeof(int) * nAtom, cudaMemcpyHostToDevice, s));
  CDK_CUDA(cudaMemcpyAsync(d_q, quats, sizeof(float) * 4 * nRot, cudaMemcpyHostToDevice, s));
  int rc = search_device_impl(c, nAtom, nConf, d_coor, d_charge, d_eps, d_slot, nQ, d_q, d_e,
                              d_i, s);
  if (rc) return rc;
  CDK_CUDA(cudaMemcpyAsync(minE, d_e, sizeof(float) * nRot, cudaMemcpyDeviceToHost, s));
  CDK_CUDA(cudaMemcpyAsync(idx, d_i, sizeof(int) * 3 * nRot, cudaMemcpyDeviceToHost, s));
  return check_errors_after(c, s);
}

int cdk_rescore_fp64(cdk_ctx* c, int nAtom, int nConf, const float* coor, const float* charge,
                     const float* eps, const int* slot, int nPose, const int* rot_conf,
                     const float* quats, const int* tidx, double* energy, void* stream) {
  if (!c || !coor || !charge || !eps || !slot || !rot_conf || !quats || !tidx || !energy ||
      nAtom <= 0 || nConf <= 0 || nPose < 0) {
    set_error("invalid argument");
    return CDK_ERR_INVALID;
  }
  if (nPose == 0) return CDK_OK;
  for (int i = 0; i < nAtom; ++i)
    if (slot[i] < 0 || slot[i] > c->K - 2) {
      set_error("atom slot outside [0, K-2]");
      return CDK_ERR_INVALID;
    }
  for (int i = 0; i < nPose; ++i)
    if (rot_conf[i] < 0 || rot_conf[i] >= nConf) {
      set_error("pose conformer index out of range");
      return CDK_ERR_INVALID;
    }
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : c->stream;
  CDK_CUDA(cudaSetDevice(c->dev));
  std::vector<ConfDesc> confs(nConf);
  for (int i = 0; i < nConf; ++i) confs[i] = ConfDesc{i * nAtom, 0, nAtom, 0};
  std::vector<RotDesc> rots(nPose);
  for (int i = 0; i < nPose; ++i) {
    for (int d = 0; d < 4; ++d) rots[i].q[d] = quats[i * 4 + d];
    rots[i].conf = rot_conf[i];
    rots[i].out = i;
    rots[i].pad0 = rots[i].pad1 = 0;
  }
  std::vector<AtomParam> prm(nAtom);
  for (int i = 0; i < nAtom; ++i) prm[i] = AtomParam{std::sqrt(eps[i]), charge[i], slot[i], 0};
  const size_t b_coor = align_up(sizeof(float) * 3 * nAtom * (size_t)nConf);
  const size_t b_conf = align_up(sizeof(ConfDesc) * nConf);
  const size_t b_rot = align_up(sizeof(RotDesc) * nPose);
  const size_t b_prm = align_up(sizeof(AtomParam) * nAtom);
  const size_t b_t = align_up(sizeof(int) * 3 * nPose);
  const size_t b_e = align_up(sizeof(double) * nPose);
  void* buf = nullptr;
  CDK_CUDA(cudaMallocAsync(&buf, b_coor + b_conf + b_rot + b_prm + b_t + b_e, s));
  char* p = static_cast<char*>(buf);
  float* d_coor = reinterpret_cast<float*>(p);
  ConfDesc* d_conf = reinterpret_cast<ConfDesc*>(p + b_coor);
  RotDesc* d_rot = reinterpret_cast<RotDesc*>(p + b_coor + b_conf);
  AtomParam* d_prm = reinterpret_cast<AtomParam*>(p + b_coor + b_conf + b_rot);
  int* d_t = reinterpret_cast<int*>(p + b_coor + b_conf + b_rot + b_prm);
  double* d_e = reinterpret_cast<double*>(p + b_coor + b_conf + b_rot + b_prm + b_t);
  cudaMemcpyAsync(d_coor, coor, sizeof(float) * 3 * nAtom * (size_t)nConf, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(d_conf, confs.data(), sizeof(ConfDesc) * nConf, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(d_rot, rots.data(), sizeof(RotDesc) * nPose, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(d_prm, prm.data(), sizeof(AtomParam) * nAtom, cudaMemcpyHostToDevice, s);
  cudaMemcpyAsync(d_t, tidx, sizeof(int) * 3 * nPose, cudaMemcpyHostToDevice, s);
  cudaError_t e = launch_rescore_fp64(c->n, c->K, c->spacing, c->d_grids, d_coor, d_prm, d_conf,
                                      d_rot, d_t, nPose, d_e, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(energy, d_e, sizeof(double) * nPose, cudaMemcpyDeviceToHost, s);
  cudaFreeAsync(buf, s);
  cudaError_t e2 = cudaStreamSynchronize(s);
  CDK_CUDA(e);
  CDK_CUDA(e2);
  return CDK_OK;
}

int cdk_fill_ligand_grid(int nQ, int nAtom, const float* coors, const float* mincoors,
                         const float* charge, const float* eps, const int* slot, int nVdwUsed,
                         int x, int y, int z, float spacing, float* out) {
  if (nQ <= 0 || nAtom <= 0 || nVdwUsed < 0 || x < 2 || y < 2 || z < 2 || !coors ||
      !mincoors || !charge || !eps || !slot || !out) {
    set_error("invalid argument");
    return CDK_ERR_INVALID;
  }
  // every corner the spread touches must lie inside the grid (the reference does not check)
  for (int q = 0; q < nQ; ++q)
    for (int a = 0; a < nAtom; ++a) {
      const int dims[3] = {x, y, z};
      for (int d = 0; d < 3; ++d) {
        const double v = ((double)coors[((size_t)q * nAtom + a) * 3 + d] - mincoors[q * 3 + d]) / spacing;
        if (!(v >= 0.0) || (int)v + 1 >= dims[d]) {
          set_error("an atom's cell lies outside the grid");
          return CDK_ERR_INVALID;
        }
      }
      if (nVdwUsed > 0 && (slot[a] < 0 || slot[a] >= nVdwUsed)) {
        set_error("atom slot outside [0, nVdwUsed-1]");
        return CDK_ERR_INVALID;
      }
    }
  std::vector<AtomParam> prm(nAtom);
  for (int i = 0; i < nAtom; ++i) prm[i] = AtomParam{std::sqrt(eps[i]), charge[i], slot[i], 0};
  const size_t N = (size_t)x * y * z;
  const size_t outElems = (size_t)nQ * (nVdwUsed + 1) * N;
  float *d_c = nullptr, *d_m = nullptr, *d_o = nullptr;
  AtomParam* d_p = nullptr;
  int rc = CDK_OK;
  cudaStream_t s = nullptr;
  if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess ||
      cudaMalloc(&d_c, sizeof(float) * 3 * nAtom * (size_t)nQ) != cudaSuccess ||
      cudaMalloc(&d_m, sizeof(float) * 3 * nQ) != cudaSuccess ||
      cudaMalloc(&d_p, sizeof(AtomParam) * nAtom) != cudaSuccess ||
      cudaMalloc(&d_o, sizeof(float) * outElems) != cudaSuccess) {
    set_error("device allocation failed");
    rc = CDK_ERR_NOMEM;
  } else {
    cudaMemcpyAsync(d_c, coors, sizeof(float) * 3 * nAtom * (size_t)nQ, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_m, mincoors, sizeof(float) * 3 * nQ, cudaMemcpyHostToDevice, s);
    cudaMemcpyAsync(d_p, prm.data(), sizeof(AtomParam) * nAtom, cudaMemcpyHostToDevice, s);
    cudaMemsetAsync(d_o, 0, sizeof(float) * outElems, s);
    cudaError_t e = launch_fill_dense(nQ, nAtom, d_c, d_m, d_p, nVdwUsed, x, y, z, spacing, d_o, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(out, d_o, sizeof(float) * outElems, cudaMemcpyDeviceToHost, s);
    cudaError_t e2 = cudaStreamSynchronize(s);
    if (e != cudaSuccess || e2 != cudaSuccess) {
      set_error(std::string("fill: ") + cudaGetErrorString(e != cudaSuccess ? e : e2));
      rc = CDK_ERR_CUDA;
    }
  }
  cudaFree(d_c);
  cudaFree(d_m);
  cudaFree(d_p);
  cudaFree(d_o);
  if (s) cudaStreamDestroy(s);
  return rc;
}

int cdk_conj_mult(const void* d_potential_F, void* d_ligand_F, int odist, int K, int Q,
                  void* stream) {
  if (!d_potential_F || !d_ligand_F || odist <= 0 || K <= 0 || Q <= 0) {
    set_error("invalid argument");
    return CDK_ERR_INVALID;
  }
  CDK_CUDA(launch_conj_mult(static_cast<const float2*>(d_potential_F),
                            static_cast<float2*>(d_ligand_F), odist, K, Q,
                            static_cast<cudaStream_t>(stream)));
  return CDK_OK;
}

int cdk_sum_grids(const void* d_ligand_F, void* d_sum_F, int K, int odist, int idist, int Q,
                  void* stream) {
  if (!d_ligand_F || !d_sum_F || odist <= 0 || K <= 0 || Q <= 0 || idist <= 0) {
    set_error("invalid argument");
    return CDK_ERR_INVALID;
  }
  CDK_CUDA(launch_sum_grids(static_cast<const float2*>(d_ligand_F), static_cast<float2*>(d_sum_F),
                            K, odist, idist, Q, static_cast<cudaStream_t>(stream)));
  return CDK_OK;
}

int cdk_ctx_top_poses(cdk_ctx* c, int cap, int* rot, float* minE, int* idx, double* e64, int* count) {
  if (!c || !count || cap < 0 || (cap > 0 && (!rot || !minE || !idx || !e64))) {
    set_error("invalid argument");
    return CDK_ERR_INVALID;
  }
  const int total = c->topk_k * c->topk_waves;
  *count = total;
  if (total == 0 || cap == 0) return CDK_OK;
  CDK_CUDA(cudaSetDevice(c->dev));
  std::vector<TopPose> h((size_t)total);
  CDK_CUDA(cudaMemcpy(h.data(), c->topk.base, sizeof(TopPose) * total, cudaMemcpyDeviceToHost));
  const int n = c->n;
  for (int i = 0; i < total && i < cap; ++i) {
    rot[i] = h[i].out;
    minE[i] = h[i].e;
    e64[i] = h[i].e64;
    const int lin = h[i].lin;
    idx[3 * i + 0] = lin < 0 ? -1 : lin / (n * n);
    idx[3 * i + 1] = lin < 0 ? -1 : (lin / n) % n;
    idx[3 * i + 2] = lin < 0 ? -1 : lin % n;
  }
  return CDK_OK;
}

int cdk_ctx_stats(cdk_ctx* c, double* out, int n) {
  if (!c || !out) return CDK_ERR_INVALID;
  for (int i = 0; i < n && i < CDK_NSTATS; ++i) out[i] = c->stats[i];
  return CDK_OK;
}

}  // extern "C"
