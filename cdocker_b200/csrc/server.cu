// server.cu -- continuous-batching docking server over one resident receptor context.
//
// The reference searches one ligand at a time (src/TranRotaConfSearchNoMini.cu:297-465). Here a
// worker thread keeps the receptor spectra resident and packs the rotations of many requests
// -- ligands of different sizes, conformer and rotation counts -- into shared waves:
//   * admission: a request is admitted when its inputs and outputs fit the server's device
//     arena (a fixed budget of HBM carved once at creation); otherwise it waits in FIFO order
//     (or submit returns CDK_ERR_BUSY when the wait queue is full);
//   * packing: each wave takes rotations from the admitted requests in admission order, so a
//     request that arrives while others run joins the next wave (continuous batching);
//   * completion: when the wave holding a request's last rotation has finished, its results
//     are copied back and its arena space is released for the next admissions.
// Every rotation's arithmetic is independent of the other rotations of its wave (the spread
// adds atoms in a fixed order, the channel sum runs in a fixed order), so a request's results
// are the same alone and in any mix.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/cdock_b200.h"
#include "cdk_internal.h"

namespace cdk {
namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
  return std::chrono::duration<double, std::milli>(b - a).count();
}

// first-fit allocator over [0, cap) in 256-byte units (host bookkeeping of device space)
class RangeAlloc {
 public:
  explicit RangeAlloc(size_t cap) { free_[0] = cap; }
  bool alloc(size_t bytes, size_t* off) {
    bytes = (bytes + 255) & ~size_t(255);
    for (auto it = free_.begin(); it != free_.end(); ++it) {
      if (it->second >= bytes) {
        *off = it->first;
        const size_t rest = it->second - bytes;
        const size_t start = it->first + bytes;
        free_.erase(it);
        if (rest) free_[start] = rest;
        return true;
      }
    }
    return false;
  }
  void release(size_t off, size_t bytes) {
    bytes = (bytes + 255) & ~size_t(255);
    auto it = free_.emplace(off, bytes).first;
    auto nx = std::next(it);
    if (nx != free_.end() && it->first + it->second == nx->first) {
      it->second += nx->second;
      free_.erase(nx);
    }
    if (it != free_.begin()) {
      auto pv = std::prev(it);
      if (pv->first + pv->second == it->first) {
        pv->second += it->second;
        free_.erase(it);
      }
    }
  }

 private:
  std::map<size_t, size_t> free_;
};

struct Request {
  uint64_t id = 0;
  int nAtom = 0, nConf = 0, nQ = 0;
  int Lb = 0;
  std::vector<float> coor, quats;
  std::vector<AtomParam> params;
  std::vector<ConfDesc> confs;  // kept alive for the asynchronous upload
  // device placement (byte offsets into the arena)
  size_t off = 0, bytes = 0;
  size_t off_coor = 0, off_param = 0, off_e = 0, off_i = 0;
  long nRot = 0, next_rot = 0, done_rot = 0;
  int conf_base = 0;  // first ConfDesc slot of this request in the server's conformer table
  Clock::time_point t_submit, t_admit, t_done;
  bool admitted = false, finished = false;
  std::vector<float> out_e;
  std::vector<int> out_i;
  int status = CDK_OK;    // first error of any wave that held rotations of this request
  std::string errmsg;
  bool scan = false;      // a wave of this request flagged rotations: scan its outputs
};

// first error wins; later ones keep the original cause
void fail_request(Request* r, int code, const std::string& msg) {
  if (r->status == CDK_OK) {
    r->status = code;
    r->errmsg = msg;
  }
}

// Per-wave status words on the device (one block per wave slot, cleared before the wave's
// launches and read back after them): [0] rotations over the planned box, [1] a bounded device
// wait gave up, [2] a scaled ligand value left the FP16 range.
constexpr int kSlotWords = 16;

struct WaveSlot {
  RotDesc* h_rots = nullptr;  // pinned
  RotDesc* d_rots = nullptr;
  cudaEvent_t done = nullptr;
  std::vector<std::pair<uint64_t, long>> parts;  // (request, rotations of it in this wave)
  bool busy = false;
  unsigned int* h_status = nullptr;  // pinned mirror of the slot's status words
  cudaError_t launch_err = cudaSuccess;  // first failed launch of this wave
};

}  // namespace
}  // namespace cdk

using namespace cdk;

struct cdk_server {
  cdk_ctx* ctx = nullptr;
  CtxView v{};
  cdk_server_opts opts{};
  cudaStream_t stream = nullptr;
  // device memory carved once
  char* arena = nullptr;          // request inputs and outputs
  size_t arena_bytes = 0;
  ConfDesc* d_confs = nullptr;    // conformer table, one slot range per request
  int conf_cap = 0;
  void* scratch = nullptr;        // wave scratch (rot_xyz, rec, keys, A or split rows, B)
  bool streamed = false;          // precision form: tensor-core x pass with ligand rows where it applies
  float osc[KMAX] = {};           // split-FP16 form: operator scale 2^-sigma_k per channel
  unsigned int* d_misc = nullptr;  // [16 s .. 16 s + 2] status words of wave slot s; work
                                   // counters (4 x u64) at byte 128
  WaveSlot slots[2];
  RangeAlloc* alloc = nullptr;
  RangeAlloc* conf_alloc = nullptr;
  // state shared with the worker
  std::mutex mu;
  std::condition_variable cv, done_cv;
  std::deque<Request*> waiting;
  std::vector<Request*> active;  // admitted, rotations left to schedule or in flight
  std::map<uint64_t, Request*> all;
  uint64_t next_id = 1;
  bool stop = false;
  std::thread worker;
  // statistics
  long waves = 0, rotations = 0, launches = 0, tc_waves = 0;
  long inject_fault_wave = -1;  // opts.reserved[0] > 0: wave number whose fault word the host sets
  double busy_ms = 0.0;
  std::vector<double> latencies;
  std::string error;
};

namespace {

int lb_of(const std::vector<float>& coor, int nAtom, int nConf, float spacing, int n) {
  double best = 0.0;
  for (int c = 0; c < nConf; ++c)
    for (int i = 0; i < nAtom; ++i)
      for (int j = i + 1; j < nAtom; ++j) {
        const float* a = &coor[((size_t)c * nAtom + i) * 3];
        const float* b = &coor[((size_t)c * nAtom + j) * 3];
        const double dx = (double)a[0] - b[0], dy = (double)a[1] - b[1], dz = (double)a[2] - b[2];
        best = std::max(best, std::sqrt(dx * dx + dy * dy + dz * dz));
      }
  const int lb = (int)std::floor((float)best / spacing + 1e-3) + 3;
  return std::min(n, std::max(2, lb));
}

// arena block of one request: coordinates (moved up to a 48-byte multiple, so that an atom
// offset of 12-byte coordinates is exact; the leading 256 bytes pay for that move), parameters,
// minE, idx
size_t req_bytes(int nAtom, int nConf, long nRot) {
  auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
  return 256 + up(sizeof(float) * 3 * (size_t)nAtom * nConf) + up(sizeof(AtomParam) * (size_t)nAtom) +
         up(sizeof(float) * (size_t)nRot) + up(sizeof(int) * 3 * (size_t)nRot);
}

// admit waiting requests in FIFO order while the arena has room (called with mu held)
void admit(cdk_server* s) {
  while (!s->waiting.empty()) {
    Request* r = s->waiting.front();
    size_t off = 0, coff = 0;
    if (!s->alloc->alloc(r->bytes, &off)) break;
    if (!s->conf_alloc->alloc((size_t)r->nConf * 256, &coff)) {
      s->alloc->release(off, r->bytes);
      break;
    }
    s->waiting.pop_front();
    auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
    r->off = off;
    r->off_coor = (off + 47) / 48 * 48;
    r->off_param = up(r->off_coor + sizeof(float) * 3 * (size_t)r->nAtom * r->nConf);
    r->off_e = r->off_param + up(sizeof(AtomParam) * (size_t)r->nAtom);
    r->off_i = r->off_e + up(sizeof(float) * (size_t)r->nRot);
    r->conf_base = (int)(coff / 256);
    r->admitted = true;
    r->t_admit = Clock::now();
    // inputs to the device (stream order puts them before the waves that read them)
    cudaMemcpyAsync(s->arena + r->off_coor, r->coor.data(), sizeof(float) * r->coor.size(),
                    cudaMemcpyHostToDevice, s->stream);
    cudaMemcpyAsync(s->arena + r->off_param, r->params.data(),
                    sizeof(AtomParam) * r->params.size(), cudaMemcpyHostToDevice, s->stream);
    r->confs.resize(r->nConf);
    for (int c = 0; c < r->nConf; ++c)
      r->confs[c] = ConfDesc{(int)((r->off_coor + (size_t)c * r->nAtom * 12) / 12),
                             (int)(r->off_param / 16), r->nAtom, 0};
    cudaMemcpyAsync(s->d_confs + r->conf_base, r->confs.data(), sizeof(ConfDesc) * r->nConf,
                    cudaMemcpyHostToDevice, s->stream);
    s->active.push_back(r);
  }
}

// a finished wave: its status words fail the requests it held (wave-wide causes: a failed
// launch, a device wait that gave up; per-rotation causes -- box overflow, FP16 range -- only
// mark the requests for a scan of their own outputs), then requests whose last rotation it
// held are completed: results copied back, arena space released
void retire(cdk_server* s, WaveSlot& w, int slot) {
  cudaError_t se = cudaEventSynchronize(w.done);
  const unsigned int* st = w.h_status;
  std::vector<Request*> finished;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    for (auto& pr : w.parts) {
      auto it = s->all.find(pr.first);
      if (it == s->all.end()) continue;
      Request* r = it->second;
      if (w.launch_err != cudaSuccess)
        fail_request(r, CDK_ERR_CUDA, std::string("a kernel launch of its wave failed: ") +
                                          cudaGetErrorString(w.launch_err));
      else if (se != cudaSuccess)
        fail_request(r, CDK_ERR_CUDA, std::string("its wave did not complete: ") + cudaGetErrorString(se));
      else if (st[1] != 0)
        fail_request(r, CDK_ERR_CUDA, "a bounded device wait (tensor-core commit) gave up in its wave; "
                                      "results are invalid");
      else if (st[0] != 0 || st[2] != 0)
        r->scan = true;
      r->done_rot += pr.second;
      if (r->done_rot == r->nRot) finished.push_back(r);
    }
  }
  (void)slot;
  w.parts.clear();
  w.busy = false;
  w.launch_err = cudaSuccess;
  for (Request* r : finished) {
    r->out_e.resize(r->nRot);
    r->out_i.resize(3 * r->nRot);
    cudaError_t e1 = cudaMemcpy(r->out_e.data(), s->arena + r->off_e, sizeof(float) * r->nRot,
                                cudaMemcpyDeviceToHost);
    cudaError_t e2 = cudaMemcpy(r->out_i.data(), s->arena + r->off_i, sizeof(int) * 3 * r->nRot,
                                cudaMemcpyDeviceToHost);
    std::lock_guard<std::mutex> lk(s->mu);
    if (e1 != cudaSuccess || e2 != cudaSuccess)
      fail_request(r, CDK_ERR_CUDA, std::string("copy of the results failed: ") +
                                        cudaGetErrorString(e1 != cudaSuccess ? e1 : e2));
    if (r->scan) {
      // k_finalize_server marks a rotation that could not be searched with index -2 (box
      // overflow) or -3 (FP16 range)
      long ovf = 0, rng = 0;
      for (long g = 0; g < r->nRot; ++g) {
        ovf += r->out_i[3 * g] == -2;
        rng += r->out_i[3 * g] == -3;
      }
      if (ovf)
        fail_request(r, CDK_ERR_OVERFLOW, std::to_string(ovf) +
                                              " rotation(s) of this request overflowed the planned ligand box");
      else if (rng)
        fail_request(r, CDK_ERR_UNSUPPORTED,
                     "a scaled ligand value of this request left the FP16 range of the split-FP16 form "
                     "(charges or sqrt-epsilon sums too large for this receptor); use CDK_FORM_BF16X3");
    }
    r->t_done = Clock::now();
    r->finished = true;
    s->latencies.push_back(ms_between(r->t_submit, r->t_done));
    s->alloc->release(r->off, r->bytes);
    s->conf_alloc->release((size_t)r->conf_base * 256, (size_t)r->nConf * 256);
    s->active.erase(std::remove(s->active.begin(), s->active.end(), r), s->active.end());
  }
  if (!finished.empty()) s->done_cv.notify_all();
}

void worker_loop(cdk_server* s) {
  cudaSetDevice(s->v.dev);
  const int n = s->v.n, K = s->v.K;
  const size_t ncol = (size_t)n * (n / 2 + 1);
  const int W = s->opts.wave_rotations;
  const int Lmax = s->opts.max_box;
  auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
  char* sc = static_cast<char*>(s->scratch);
  WaveArgs a{};
  a.n = n;
  a.K = K;
  a.spacing = s->v.spacing;
  a.max_atoms = s->opts.max_atoms;
  a.coords = reinterpret_cast<const float*>(s->arena);
  a.params = reinterpret_cast<const AtomParam*>(s->arena);
  a.confs = s->d_confs;
  a.rot_xyz = reinterpret_cast<float4*>(sc);
  sc += up((size_t)W * a.max_atoms * sizeof(float4));
  a.rec = reinterpret_cast<RotRec*>(sc);
  sc += up((size_t)W * sizeof(RotRec));
  a.keys = reinterpret_cast<unsigned long long*>(sc);
  sc += up((size_t)W * sizeof(unsigned long long));
  a.A = reinterpret_cast<float2*>(sc);
  const bool f16 = s->streamed && s->v.form == CDK_FORM_FP16X2;
  // ligand rows of either layout (tiled rows round the wave up to whole 128-rotation tiles)
  const size_t rows = s->streamed ? lop_wave_bytes(W, true, stream_lop_bytes_per_rotation(n, K, f16)) : 0;
  unsigned char* lop_base = reinterpret_cast<unsigned char*>(sc);
  sc += up(std::max((size_t)W * K * Lmax * ncol * sizeof(float2), rows));
  a.B = reinterpret_cast<float2*>(sc);
  sc += up((size_t)W * n * ncol * sizeof(float2));
  // precision forms: every window plane's two smallest keys for the FP64 near-tie break, as
  // in a plain search (so results are the same alone and in the mix)
  a.keys2 = s->v.tiebreak ? reinterpret_cast<unsigned long long*>(sc) : nullptr;
  a.phat = s->v.phat;
  a.tw = s->v.tw;
  a.work = reinterpret_cast<unsigned long long*>(s->d_misc + 32);
  for (int k = 0; k < KMAX; ++k) a.lscale[k] = s->v.lscale[k];
  a.col_tile = s->v.col_tile_opt > 0 ? s->v.col_tile_opt : pick_col_tile(n, K);
  a.kyof = s->v.kyof;
  a.minE = nullptr;
  a.idx = nullptr;
  int cur = 0;
  for (;;) {
    // build the next wave from the admitted requests
    WaveSlot& w = s->slots[cur];
    if (w.busy) retire(s, w, cur);
    int nr = 0, lb = 2, cap = 1;
    {
      std::unique_lock<std::mutex> lk(s->mu);
      admit(s);
      auto has_work = [&] {
        for (Request* r : s->active)
          if (r->next_rot < r->nRot) return true;
        return false;
      };
      if (!has_work()) {
        WaveSlot& other = s->slots[cur ^ 1];
        if (other.busy) {
          lk.unlock();
          retire(s, other, cur ^ 1);
          continue;
        }
        if (s->stop && s->waiting.empty()) break;
        s->cv.wait_for(lk, std::chrono::milliseconds(2));
        continue;
      }
      // every wave's RotDesc.out indexes a per-request output block: the wave carries
      // requests whose outputs share one base, so outputs go through one base pointer with
      // per-request offsets folded into `out` (units of one rotation)
      for (Request* r : s->active) {
        if (nr == W) break;
        if (r->next_rot >= r->nRot) continue;
        const long take = std::min<long>(W - nr, r->nRot - r->next_rot);
        // outputs: minE at float index off_e/4 + g, idx at int index off_i/4 + 3g, both
        // relative to the arena base (launch_finalize_server)
        const long obase = (long)(r->off_e / sizeof(float));
        const long ibase = (long)(r->off_i / sizeof(int));
        for (long t = 0; t < take; ++t) {
          const long g = r->next_rot + t;
          RotDesc& d = w.h_rots[nr + t];
          std::memcpy(d.q, &r->quats[g * 4], 4 * sizeof(float));
          d.conf = r->conf_base + (int)(g / r->nQ);
          d.out = (int)(obase + g);
          d.pad0 = (int)(ibase + 3 * g);
          d.pad1 = 0;
        }
        w.parts.emplace_back(r->id, take);
        r->next_rot += take;
        nr += (int)take;
        lb = std::max(lb, r->Lb);
        cap = std::max(cap, r->nAtom);
      }
    }
    // this slot's status words: cleared before the wave, read back after it
    unsigned int* d_st = s->d_misc + kSlotWords * cur;
    a.err_count = reinterpret_cast<int*>(d_st);
    a.fault = reinterpret_cast<int*>(d_st + 1);
    a.range_err = reinterpret_cast<int*>(d_st + 2);
    cudaError_t le = cudaMemcpyAsync(w.d_rots, w.h_rots, sizeof(RotDesc) * nr, cudaMemcpyHostToDevice, s->stream);
    auto note = [&](cudaError_t e) {
      if (le == cudaSuccess && e != cudaSuccess) le = e;
    };
    note(cudaMemsetAsync(d_st, 0, kSlotWords * sizeof(unsigned int), s->stream));
    a.nrot = nr;
    a.Lb = lb;
    a.atom_cap = cap;
    a.rots = w.d_rots;
    // the same x-pass choice as a plain search on the context (results alone and in the mix
    // stay identical): streamed tiles at 64^3 where they apply, the Hankel kernel elsewhere
    HankelPlan hp{};
    const bool tile_wave = s->streamed && s->v.top != nullptr && use_stream_tiles(s->v.tc_variant) &&
                           stream_supported(n, lb) && direct_planes(a);
    const bool tc_wave = tile_wave || (s->streamed && s->v.tc_variant != 3 && direct_planes(a) &&
                                       hankel_plan(n, K, lb, f16, 0, &hp));
    a.lop = tc_wave ? lop_base : nullptr;
    // the Hankel x pass loads tiled rows (split-FP16) or untiled rows, as in a plain search
    a.lop_tiled = (tc_wave && !tile_wave && hankel_tiled(s->v.hx_shape)) ? 1 : 0;
    a.f16 = (tc_wave && f16) ? 1 : 0;
    a.bgroup = tc_wave ? stream_bgroup() : 1;
    a.bcol = 0;
    if (tc_wave && !tile_wave) hankel_b_layout(hp, a);
    if (le == cudaSuccess) {
      note(launch_prep(a, s->stream));
      note(launch_spread_yz(a, s->stream));
      note(tile_wave ? launch_xpass_stream(a, s->v.top, s->stream)
                     : tc_wave ? launch_xpass_hankel(a, s->v.ptilde, s->osc, hp, s->stream)
                               : launch_xpass(a, s->stream));
      note(launch_yz_inv_argmin(a, s->stream));
      if (a.keys2)
        note(launch_tiebreak(a, s->v.grids, s->v.form == CDK_FORM_FP16X2 ? 1e-3f : 1e-4f, s->stream));
      note(launch_finalize_server(a, reinterpret_cast<float*>(s->arena),
                                  reinterpret_cast<int*>(s->arena), s->stream));
    }
    if (s->waves == s->inject_fault_wave) {
      // fault injection from the host (a test switch): the word a bounded device wait sets
      // when it gives up, written after the wave's kernels
      const unsigned int one = 1;
      note(cudaMemcpyAsync(d_st + 1, &one, sizeof(one), cudaMemcpyHostToDevice, s->stream));
      note(cudaStreamSynchronize(s->stream));
    }
    note(cudaMemcpyAsync(w.h_status, d_st, 4 * sizeof(unsigned int), cudaMemcpyDeviceToHost, s->stream));
    note(cudaEventRecord(w.done, s->stream));
    w.launch_err = le;
    if (le != cudaSuccess) {
      std::lock_guard<std::mutex> lk(s->mu);
      s->error = std::string("wave launch: ") + cudaGetErrorString(le);
    }
    w.busy = true;
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->waves++;
      s->tc_waves += tc_wave ? 1 : 0;
      s->rotations += nr;
      s->launches += kLaunchesPerWave + (tc_wave ? 1 : 0) + (a.keys2 ? 1 : 0);  // + k_tile_plan, tie break
    }
    cur ^= 1;
  }
  for (int k = 0; k < 2; ++k)
    if (s->slots[k].busy) retire(s, s->slots[k], k);
}

}  // namespace

extern "C" {

void cdk_server_opts_default(cdk_server_opts* o) {
  if (!o) return;
  std::memset(o, 0, sizeof(*o));
  o->arena_bytes = (size_t)1 << 30;
  o->wave_rotations = 1024;
  o->max_box = 0;
  o->max_atoms = 128;
  o->max_conformers = 1 << 16;
  o->max_waiting = 4096;
}

int cdk_server_create(cdk_ctx* ctx, const cdk_server_opts* opts, cdk_server** out) {
  if (!ctx || !out) {
    set_error("null argument");
    return CDK_ERR_INVALID;
  }
  *out = nullptr;
  cdk_server* s = new cdk_server();
  s->ctx = ctx;
  ctx_view(ctx, &s->v);
  if (opts) s->opts = *opts;
  else cdk_server_opts_default(&s->opts);
  if (s->opts.wave_rotations <= 0 || s->opts.wave_rotations > 65535) s->opts.wave_rotations = 1024;
  if (s->opts.max_atoms <= 0) s->opts.max_atoms = 128;
  if (s->opts.max_box <= 0) s->opts.max_box = std::min(s->v.n, 40);
  if (s->opts.max_conformers <= 0) s->opts.max_conformers = 1 << 16;
  if (s->opts.arena_bytes < ((size_t)1 << 20)) s->opts.arena_bytes = (size_t)1 << 20;
  const int n = s->v.n, K = s->v.K, W = s->opts.wave_rotations;
  const size_t ncol = (size_t)n * (n / 2 + 1);
  auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
  // precision-form contexts run the tensor-core x pass (resident Hankel operator, streamed
  // ligand rows) on waves it applies to (ligand box <= 32 planes, ligands <= 96 atoms on the
  // direct plane path); other waves and FP32 contexts run the FP32 radix x pass
  HankelPlan probe{};
  const bool tcv = s->v.tc_variant == 0 || s->v.tc_variant == 3 || s->v.tc_variant == 4;
  s->streamed = ((s->v.form == CDK_FORM_BF16X3 && tcv) || s->v.form == CDK_FORM_FP16X2) &&
                s->v.kyof != nullptr && s->v.ptilde != nullptr &&
                (stream_supported(n, std::min(s->opts.max_box, 32)) ||
                 hankel_plan(n, K, std::min(s->opts.max_box, 32), s->v.form == CDK_FORM_FP16X2, 0, &probe));
  if (s->streamed && use_stream_tiles(s->v.tc_variant) && stream_top_bytes(n, K) > 0) {
    // 64^3: the streamed-tile kernel's operator image, built once per context
    const int rc = ctx_ensure_top(ctx);
    if (rc != CDK_OK) {
      delete s;
      return rc;
    }
    ctx_view(ctx, &s->v);
  }
  for (int k = 0; k < KMAX; ++k) s->osc[k] = s->v.lscale[k] != 0.f ? 1.f / s->v.lscale[k] : 1.f;
  const size_t planes = (size_t)W * K * s->opts.max_box * ncol * sizeof(float2);
  const size_t rows = s->streamed ? lop_wave_bytes(W, true,
                                                   stream_lop_bytes_per_rotation(n, K, s->v.form == CDK_FORM_FP16X2))
                                  : 0;
  const size_t scratch = up((size_t)W * s->opts.max_atoms * sizeof(float4)) +
                         up((size_t)W * sizeof(RotRec)) + up((size_t)W * 8) +
                         up(std::max(planes, rows)) + up((size_t)W * n * ncol * sizeof(float2)) +
                         (s->v.tiebreak ? up((size_t)W * n * 2 * sizeof(unsigned long long)) : 0);
  auto fail = [&](const std::string& m, int code) {
    set_error(m);
    cdk_server_destroy(s);
    return code;
  };
  if (cudaSetDevice(s->v.dev) != cudaSuccess) return fail("cudaSetDevice failed", CDK_ERR_CUDA);
  if (cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking) != cudaSuccess)
    return fail("stream creation failed", CDK_ERR_CUDA);
  if (cudaMalloc(&s->arena, s->opts.arena_bytes) != cudaSuccess ||
      cudaMalloc(&s->d_confs, sizeof(ConfDesc) * (size_t)s->opts.max_conformers) != cudaSuccess ||
      cudaMalloc(&s->scratch, scratch) != cudaSuccess ||
      cudaMalloc(&s->d_misc, 256) != cudaSuccess)
    return fail("server device allocation failed (" + std::to_string((s->opts.arena_bytes + scratch) >> 20) + " MiB)", CDK_ERR_NOMEM);
  cudaMemset(s->d_misc, 0, 256);
  s->inject_fault_wave = s->opts.reserved[0] > 0 ? (long)s->opts.reserved[0] - 1 : -1;
  s->arena_bytes = s->opts.arena_bytes;
  s->conf_cap = s->opts.max_conformers;
  for (auto& w : s->slots) {
    if (cudaMallocHost(&w.h_rots, sizeof(RotDesc) * W) != cudaSuccess ||
        cudaMalloc(&w.d_rots, sizeof(RotDesc) * W) != cudaSuccess ||
        cudaMallocHost(&w.h_status, 4 * sizeof(unsigned int)) != cudaSuccess ||
        cudaEventCreateWithFlags(&w.done, cudaEventDisableTiming) != cudaSuccess)
      return fail("server wave buffers failed", CDK_ERR_NOMEM);
  }
  s->alloc = new RangeAlloc(s->arena_bytes);
  s->conf_alloc = new RangeAlloc((size_t)s->conf_cap * 256);
  s->worker = std::thread(worker_loop, s);
  *out = s;
  return CDK_OK;
}

int cdk_server_submit(cdk_server* s, int nAtom, int nConf, const float* coor,
                      const float* charge, const float* eps, const int* slot, int nQ,
                      const float* quats, uint64_t* ticket) {
  if (!s || !coor || !charge || !eps || !slot || !quats || !ticket || nAtom <= 0 ||
      nConf <= 0 || nQ <= 0) {
    set_error("invalid argument");
    return CDK_ERR_INVALID;
  }
  if (nAtom > s->opts.max_atoms) {
    set_error("ligand larger than the server's max_atoms");
    return CDK_ERR_INVALID;
  }
  for (int i = 0; i < nAtom; ++i)
    if (slot[i] < 0 || slot[i] > s->v.K - 2) {
      set_error("atom slot outside [0, K-2]");
      return CDK_ERR_INVALID;
    }
  Request* r = new Request();
  r->nAtom = nAtom;
  r->nConf = nConf;
  r->nQ = nQ;
  r->nRot = (long)nConf * nQ;
  r->coor.assign(coor, coor + (size_t)nAtom * nConf * 3);
  r->quats.assign(quats, quats + (size_t)r->nRot * 4);
  r->params.resize(nAtom);
  for (int i = 0; i < nAtom; ++i) r->params[i] = AtomParam{std::sqrt(eps[i]), charge[i], slot[i], 0};
  r->Lb = lb_of(r->coor, nAtom, nConf, s->v.spacing, s->v.n);
  if (r->Lb > s->opts.max_box) {
    delete r;
    set_error("ligand box larger than the server's max_box");
    return CDK_ERR_INVALID;
  }
  r->bytes = req_bytes(nAtom, nConf, r->nRot);
  if (r->bytes > s->arena_bytes || nConf > s->conf_cap) {
    delete r;
    set_error("request larger than the whole server arena");
    return CDK_ERR_INVALID;
  }
  r->t_submit = Clock::now();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if ((int)s->waiting.size() >= s->opts.max_waiting) {
      delete r;
      set_error("server queue full");
      return CDK_ERR_BUSY;
    }
    r->id = s->next_id++;
    s->all[r->id] = r;
    s->waiting.push_back(r);
    *ticket = r->id;
  }
  s->cv.notify_one();
  return CDK_OK;
}

int cdk_server_poll(cdk_server* s, uint64_t ticket, int wait_ms, float* minE, int* idx,
                    double* timing) {
  if (!s) {
    set_error("null server");
    return CDK_ERR_INVALID;
  }
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->all.find(ticket);
  if (it == s->all.end()) {
    set_error("unknown ticket");
    return CDK_ERR_INVALID;
  }
  Request* r = it->second;
  if (!r->finished && wait_ms != 0) {
    auto pred = [&] { return r->finished; };
    if (wait_ms < 0) s->done_cv.wait(lk, pred);
    else s->done_cv.wait_for(lk, std::chrono::milliseconds(wait_ms), pred);
  }
  if (!r->finished) return CDK_ERR_BUSY;
  const int status = r->status;
  const std::string msg = r->errmsg;
  if (minE) std::memcpy(minE, r->out_e.data(), sizeof(float) * r->nRot);
  if (idx) std::memcpy(idx, r->out_i.data(), sizeof(int) * 3 * r->nRot);
  if (timing) {
    timing[0] = ms_between(r->t_submit, r->t_admit);
    timing[1] = ms_between(r->t_admit, r->t_done);
    timing[2] = ms_between(r->t_submit, r->t_done);
  }
  s->all.erase(it);
  delete r;
  if (status != CDK_OK) set_error(msg);
  return status;
}

int cdk_server_stats(cdk_server* s, double* out, int n) {
  if (!s || !out) return CDK_ERR_INVALID;
  std::lock_guard<std::mutex> lk(s->mu);
  std::vector<double> lat = s->latencies;
  std::sort(lat.begin(), lat.end());
  auto pct = [&](double p) {
    if (lat.empty()) return 0.0;
    size_t k = (size_t)std::ceil(p * lat.size()) - 1;
    return lat[std::min(k, lat.size() - 1)];
  };
  const double vals[9] = {(double)s->waves, (double)s->rotations, (double)s->launches,
                          (double)lat.size(), pct(0.50), pct(0.99),
                          (double)s->waiting.size(), (double)s->active.size(),
                          (double)s->tc_waves};
  for (int i = 0; i < n && i < 9; ++i) out[i] = vals[i];
  return CDK_OK;
}

int cdk_server_destroy(cdk_server* s) {
  if (!s) return CDK_OK;
  if (s->worker.joinable()) {
    {
      std::lock_guard<std::mutex> lk(s->mu);
      s->stop = true;
    }
    s->cv.notify_all();
    s->worker.join();
  }
  cudaSetDevice(s->v.dev);
  if (s->stream) cudaStreamSynchronize(s->stream);
  for (auto& w : s->slots) {
    if (w.h_rots) cudaFreeHost(w.h_rots);
    if (w.h_status) cudaFreeHost(w.h_status);
    cudaFree(w.d_rots);
    if (w.done) cudaEventDestroy(w.done);
  }
  cudaFree(s->arena);
  cudaFree(s->d_confs);
  cudaFree(s->scratch);
  cudaFree(s->d_misc);
  if (s->stream) cudaStreamDestroy(s->stream);
  for (auto& kv : s->all) delete kv.second;
  delete s->alloc;
  delete s->conf_alloc;
  delete s;
  return CDK_OK;
}

}  // extern "C"
